// rz_single.cu -- single-list Redzone, persistent grid-wide schedule (and the single-CTA case).
//
// Redzone follows Algorithm 2 of the reference (RemoveFromList_GPUWide, redzone.hxx:626-941) and
// its CPU form (redzone_CPU, Redzone_CPU.hxx:150-248). The phases are the reference's; the data
// layout and synchronisation are this library's own:
//   * Phase A (mark, reference :698-706): every index in the red zone [cut, n) sets one bit of a
//     k-bit bitmap in scratch (atomicOr) instead of writing an in-band 0x80000000 sentinel into
//     the caller's tail, so any payload width works and the tail is never written.
//   * Barrier: epoch-tagged arrival flags with bounded waits (rz_common.cuh) replace
//     cg::grid.sync() and BlockStorage_t::Wait(): one release store per CTA, no reset.
//   * Phase B (fill holes, reference :752-822): items are processed in tiles of B*IPT, item
//     (j, t) of a tile at i = base + j*B + t, so every warp load of the index list and of the tail
//     window is a contiguous 128-byte (or 32*W-byte) segment. Valid/valid pairs are moved at once;
//     orphans get their rank in i order from per-(j, warp) ballot counts and one scan per tile,
//     and are written to per-CTA regions of scratch lists (the caller's index list is const).
//     Each tile clears the bitmap words it read, which leaves the bitmap zero for the next call.
//   * Phase C (pair orphans, reference :834-934): each CTA publishes its two orphan counts as
//     epoch-tagged words; only CTAs that own destination orphans wait for the others, prefix the
//     counts and binary-search the owner of each source rank (instead of the reference's
//     LoadBalance linear search, :477-524).
//   * Red-list schedule (one tile per CTA, k <= kRedlistMaxK): in phase A each CTA also writes its
//     red entries {i, idx[i] - cut} in i order to its region of a list and arrives with a 64-bit
//     word tag << 32 | count. If the grid holds at most kFastMaxRed red entries, every CTA reads
//     them all into shared memory: V (tail positions whose item is removed) and P (positions whose
//     hole needs no fill) as k-bit maps, destination orphans = V \ P counted per tile, source
//     orphans = P \ V in order; each CTA then fills its holes and pairs its own destination
//     orphans with no further exchange (phases B and C in one step, one grid-wide wait in all).
//     Above that count the CTAs continue with the bitmap phases B and C.
// The O(n) partition comparator is in rz_partition.cu; the cluster schedule in rz_cluster.cu.
#include <algorithm>
#include <atomic>
#include <cstdio>

#include "rz_common.cuh"
#include "rz_internal.h"
#include "rz_single_kernel.cuh"

namespace rz {

// ------------------------------------------------------------------------------------------------
// Redzone, one list, G persistent CTAs (G == 1 degenerates to block-level synchronisation).
// ------------------------------------------------------------------------------------------------
template <int W, int IPT>
__global__ void redzone_single_kernel(const SingleParams p) {
    redzone_single_body<W, IPT>(p);
}

// ------------------------------------------------------------------------------------------------
// RZ_VALIDATE: full duplicate / range check with an n-bit occupancy map (left zero on exit).
// ------------------------------------------------------------------------------------------------
__global__ void validate_mark_kernel(const uint32_t* __restrict__ idx, uint32_t k, uint32_t n,
                                     uint32_t* __restrict__ seen, uint32_t* status) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        const uint32_t r = __ldg(&idx[i]);
        if (r >= n) {
            atomicOr(status, ST_RANGE);
            continue;
        }
        const uint32_t bit = 1u << (r & 31u);
        if (atomicOr(&seen[r >> 5], bit) & bit) atomicOr(status, ST_DUPLICATE);
    }
}
__global__ void validate_clear_kernel(const uint32_t* __restrict__ idx, uint32_t k, uint32_t n,
                                      uint32_t* __restrict__ seen) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        const uint32_t r = __ldg(&idx[i]);
        if (r < n) seen[r >> 5] = 0u;
    }
}

// ------------------------------------------------------------------------------------------------
// Barrier-timeout test kernel: the grid's own arrival protocol, waiting for one CTA more than the
// grid has, so the bounded wait must expire.
// ------------------------------------------------------------------------------------------------
__global__ void barrier_timeout_kernel(uint32_t* arrive, uint32_t* status, uint32_t spin_limit, uint32_t tag) {
    flag_arrive(arrive, blockIdx.x, tag);
    flag_wait_all(arrive, gridDim.x + 1u, tag, status, spin_limit);
}

// ------------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------------
using SingleFn = void (*)(const SingleParams);

template <int W>
static SingleFn single_fn(int items) {
    switch (items) {
        case 1: return redzone_single_kernel<W, 1>;
        case 2: return redzone_single_kernel<W, 2>;
        case 4: return redzone_single_kernel<W, 4>;
        case 8: return redzone_single_kernel<W, 8>;
        default: return nullptr;
    }
}
static SingleFn single_fn(int w, int items) {
    switch (w) {
        case 4: return single_fn<4>(items);
        case 8: return single_fn<8>(items);
        case 16: return single_fn<16>(items);
        case 32: return single_fn<32>(items);
        default: return nullptr;
    }
}

static int wi(int w) { return w == 4 ? 0 : w == 8 ? 1 : w == 16 ? 2 : 3; }
static int ii(int items) { return items == 1 ? 0 : items == 2 ? 1 : items == 4 ? 2 : 3; }

int redzone_max_block(int w, int items) {
    static int cache[4][4] = {};
    SingleFn f = single_fn(w, items);
    if (!f) return 0;
    int& c = cache[wi(w)][ii(items)];
    if (c == 0) {
        cudaFuncAttributes a{};
        if (cudaFuncGetAttributes(&a, (const void*)f) != cudaSuccess) return 0;
        c = a.maxThreadsPerBlock & ~31;
    }
    return c;
}

int redzone_occupancy(int w, int items, int block, size_t dynamic_smem) {
    SingleFn f = single_fn(w, items);
    if (!f) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)f, block, dynamic_smem) != cudaSuccess)
        return 0;
    return nb;
}

// Opt the kernel in to the red-list schedule's dynamic shared memory (once per device and variant).
static int allow_redlist_smem(rz_ctx* ctx, int w, int items) {
    static std::atomic<uint64_t> done[4][4];
    const uint64_t bit = 1ull << (ctx->device & 63);
    std::atomic<uint64_t>& d = done[wi(w)][ii(items)];
    if (d.load() & bit) return RZ_OK;
    RZ_CUDA_TRY(ctx, cudaFuncSetAttribute((const void*)single_fn(w, items), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(redlist_smem_bytes(kRedlistMaxK))));
    d.fetch_or(bit);
    return RZ_OK;
}

int clamp_cfg(const rz_ctx* ctx, uint32_t k, uint32_t w, rz_launch_cfg* cfg) {
    if (cfg->items != 1 && cfg->items != 2 && cfg->items != 4 && cfg->items != 8) return RZ_ERR_INVALID_ARG;
    if (cfg->block < 32 || cfg->block > 1024 || (cfg->block & 31)) return RZ_ERR_INVALID_ARG;
    const int maxb = redzone_max_block(int(w), cfg->items);
    if (maxb <= 0) return RZ_ERR_INVALID_ARG;
    if (cfg->block > maxb) cfg->block = maxb;
    if (cfg->ctas_per_sm < 1) cfg->ctas_per_sm = 1;
    (void)ctx;
    (void)k;
    return RZ_OK;
}

int default_cfg(const rz_ctx* ctx, uint32_t n, uint32_t k, uint32_t w, rz_launch_cfg* cfg) {
    (void)n;
    cfg->use_partition = 0;
    cfg->schedule = RZ_SCHED_AUTO;
    // Measured on B200 (n = 2^28, L2 flushed): up to k = 2^12 the scan-all schedule (one grid, each
    // CTA reads the whole list: 7.9 against 8.5 us per call at k = 2^10); the cluster-scan schedule,
    // which needs no grid-wide wait, from k = 2^13 to 2^17 (7.2 against 11.1 us per call at
    // k = 2^16, graph steady state). Where the cluster scan does not run (wider
    // items at k > 2^16, k > 2^17): the grid schedule with 512-item tiles at 2^15, 1024-item tiles
    // to 2^17 (64 CTAs at 2^16 -- fewer, fuller CTAs shorten the grid-wide wait), and 4096-item
    // tiles on two CTAs per SM beyond.
    if (k <= kScanAllMaxK) {
        cfg->block = 256;
        cfg->items = 1;
        cfg->ctas_per_sm = 4;  // used only by a fallback (misaligned index list)
        cfg->schedule = RZ_SCHED_SCANALL;
        return RZ_OK;
    }
    if (k >= kCscanMinK && cscan_default_cfg(ctx, k, w, cfg)) return RZ_OK;
    if (k <= kClusterMaxK) {
        cfg->block = 256; cfg->items = 4; cfg->ctas_per_sm = 4;
    } else if (k <= (1u << 15)) {
        cfg->block = 256; cfg->items = 2; cfg->ctas_per_sm = 4;
    } else if (k <= (1u << 16)) {
        cfg->block = 256; cfg->items = 4; cfg->ctas_per_sm = 2;
    } else if (k <= (1u << 17)) {
        cfg->block = 256; cfg->items = 4; cfg->ctas_per_sm = w >= 16 ? 2 : 1;
    } else {
        cfg->block = 1024; cfg->items = 4; cfg->ctas_per_sm = 2;
    }
    return clamp_cfg(ctx, k, w, cfg);
}

int launch_validate(rz_ctx* ctx, uint32_t n, const uint32_t* idx, uint32_t k, cudaStream_t s) {
    int st = ensure_seen(ctx, n);
    if (st != RZ_OK) return st;
    const int grid = std::max(1, std::min<int>(ctx->sms * 4, int((k + 255) / 256)));
    validate_mark_kernel<<<grid, 256, 0, s>>>(idx, k, n, ctx->ws.seen, ctx->ws.status);
    validate_clear_kernel<<<grid, 256, 0, s>>>(idx, k, n, ctx->ws.seen);
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    return RZ_OK;
}

int launch_redzone(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx, uint32_t k,
                   const rz_launch_cfg& cfg_in, uint32_t flags, cudaStream_t s, LaunchInfo* info) {
    rz_launch_cfg cfg = cfg_in;
    int st = clamp_cfg(ctx, k, w, &cfg);
    if (st != RZ_OK) return st;
    st = ensure_lists(ctx, k);
    if (st != RZ_OK) return st;
    st = reset_if_dirty(ctx, s);
    if (st != RZ_OK) return st;
    const bool validate = (flags & RZ_VALIDATE) != 0;
    int launches = 0;
    if (validate) {
        st = launch_validate(ctx, n, idx, k, s);
        if (st != RZ_OK) return st;
        launches += 2;
    }
    int sched = cfg.schedule;
    if (flags & RZ_FORCE_BLOCK) sched = RZ_SCHED_BLOCK;
    if (flags & RZ_FORCE_GRID) sched = RZ_SCHED_GRID;
    if (sched == RZ_SCHED_AUTO) sched = (k <= kClusterMaxK) ? RZ_SCHED_CLUSTER : RZ_SCHED_GRID;
    if (sched == RZ_SCHED_SCANALL) {
        LaunchInfo ci;
        ci.launches = launches;
        st = launch_scanall(ctx, data, n, w, idx, k, cfg, validate, s, &ci);
        if (st == RZ_OK) {
            if (info) *info = ci;
            return RZ_OK;
        }
        if (st != RZ_ERR_UNSUPPORTED) return st;
        sched = k <= kClusterMaxK ? RZ_SCHED_CLUSTER : RZ_SCHED_GRID;  // misaligned list, or k too large
    }
    if (sched == RZ_SCHED_SPLIT) {
        LaunchInfo ci;
        ci.launches = launches;
        st = launch_split(ctx, data, n, w, idx, k, cfg, validate, s, &ci);
        if (st == RZ_OK) {
            if (info) *info = ci;
            return RZ_OK;
        }
        if (st != RZ_ERR_UNSUPPORTED) return st;
        sched = RZ_SCHED_GRID;  // k beyond the shared-memory maps
    }
    if (sched == RZ_SCHED_CSCAN) {
        LaunchInfo ci;
        ci.launches = launches;
        st = launch_cscan(ctx, data, n, w, idx, k, cfg, validate, s, &ci);
        if (st == RZ_OK) {
            if (info) *info = ci;
            return RZ_OK;
        }
        if (st != RZ_ERR_UNSUPPORTED) return st;
        sched = RZ_SCHED_GRID;  // k beyond one register pass per slice, or no room for the cluster
    }
    if (sched == RZ_SCHED_CLUSTER) {
        LaunchInfo ci;
        ci.launches = launches;
        st = launch_cluster(ctx, data, n, w, idx, k, cfg, validate, s, &ci);
        if (st == RZ_OK) {
            if (info) *info = ci;
            return RZ_OK;
        }
        if (st != RZ_ERR_UNSUPPORTED) return st;
        sched = RZ_SCHED_GRID;  // bitmap slice too large for shared memory: use the grid schedule
    }
    const uint32_t tile = uint32_t(cfg.block) * uint32_t(cfg.items);
    const uint32_t ntiles = (k + tile - 1) / tile;
    // Red-list schedule when every tile gets its own co-resident CTA with the shared memory for
    // the k-bit maps; otherwise the bitmap schedule without dynamic shared memory.
    bool fast = false;
    size_t dsmem = 0;
    long grid = 1;
    const bool few_red = k <= kFastMaxK || double(k) * double(k) <= double(kFastMaxRed) * double(n);
    if (sched != RZ_SCHED_BLOCK && k <= kRedlistMaxK && few_red && ctx->ws.redlist && ctx->ws.red_cap > k &&
        ntiles > 1) {
        st = allow_redlist_smem(ctx, int(w), cfg.items);
        if (st != RZ_OK) return st;
        const size_t need = redlist_smem_bytes(k);
        const int occf = redzone_occupancy(int(w), cfg.items, cfg.block, need);
        const long gf = std::min<long>(std::min<long>((long)cfg.ctas_per_sm, (long)occf) * ctx->sms, (long)kMaxGrid);
        if (occf > 0 && (long)ntiles <= gf) {
            fast = true;
            dsmem = need;
            grid = ntiles;
        }
    }
    if (!fast) {
        int occ = redzone_occupancy(int(w), cfg.items, cfg.block);
        if (occ <= 0) return RZ_ERR_INVALID_ARG;
        grid = std::min<long>((long)cfg.ctas_per_sm, (long)occ) * ctx->sms;
        grid = std::min<long>(grid, (long)ntiles);
        grid = std::min<long>(grid, (long)kMaxGrid);
        if (sched == RZ_SCHED_BLOCK) grid = 1;
        if (grid < 1) grid = 1;
        // Re-balance: use as many CTAs as needed for the resulting tiles-per-CTA (no idle CTAs).
        const uint32_t tpc = (ntiles + uint32_t(grid) - 1) / uint32_t(grid);
        grid = (ntiles + tpc - 1) / tpc;
    }

    SingleParams p;
    p.data = static_cast<uint8_t*>(data);
    p.idx = idx;
    p.n = n;
    p.k = k;
    p.bitmap = ctx->ws.bitmap;
    p.dlist = ctx->ws.dlist;
    p.slist = ctx->ws.slist;
    p.epoch = ctx->ws.epoch;
    p.arrive = ctx->ws.arrive;
    p.cnt_words = ctx->ws.cnt_words;
    p.status = ctx->ws.status;
    p.dev_len = ctx->ws.dev_len;
    p.stamps = ctx->ws.stamps_on ? ctx->ws.stamps : nullptr;
    p.spin_limit = kSpinLimit;
    p.validate = validate ? 1u : 0u;
    p.redlist = fast ? ctx->ws.redlist : nullptr;
    p.arrive64 = fast ? ctx->ws.arrive64 : nullptr;

    SingleFn f = single_fn(int(w), cfg.items);
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(unsigned(grid));
    lc.blockDim = dim3(unsigned(cfg.block));
    lc.dynamicSmemBytes = dsmem;
    lc.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = grid > 1 ? 1 : 0;
    lc.attrs = attr;
    lc.numAttrs = 1;
    RZ_CUDA_TRY(ctx, cudaLaunchKernelEx(&lc, f, p));
    launches += 1;
    if (info) {
        info->grid = int(grid);
        info->block = cfg.block;
        info->items = cfg.items;
        info->launches = launches;
    }
    return RZ_OK;
}

// An empty kernel: what a launch of a given shape costs between two events with no work in it.
__global__ void empty_launch_kernel() {}

int test_empty_launch(rz_ctx* ctx, int grid, int block, int cluster, int smem, cudaStream_t s) {
    if (grid < 1 || block < 1 || block > 1024 || cluster < 1 || cluster > 8 || grid % cluster || smem < 0)
        return RZ_ERR_INVALID_ARG;
    if (smem > 48 * 1024)
        RZ_CUDA_TRY(ctx, cudaFuncSetAttribute(empty_launch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(unsigned(grid));
    lc.blockDim = dim3(unsigned(block));
    lc.dynamicSmemBytes = size_t(smem);
    lc.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(cluster);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = cluster > 1 ? 1 : 0;
    RZ_CUDA_TRY(ctx, cudaLaunchKernelEx(&lc, empty_launch_kernel));
    return RZ_OK;
}

__device__ __forceinline__ void fill_item(uint32_t& v, uint32_t i) { v = i; }
__device__ __forceinline__ void fill_item(uint2& v, uint32_t i) { v = make_uint2(i, ~i); }
__device__ __forceinline__ void fill_item(uint4& v, uint32_t i) { v = make_uint4(i, ~i, i, ~i); }
__device__ __forceinline__ void fill_item(u32x8& v, uint32_t i) {
    v.a = make_uint4(i, ~i, i, ~i);
    v.b = v.a;
}

// Plain scattered stores data[pos[i]] = item i: the rate the memory system sustains for the hole
// writes of a removal, with nothing else in the kernel. Positions >= n are skipped.
template <int W>
__global__ void __launch_bounds__(256) scatter_kernel(uint8_t* __restrict__ data, uint32_t n,
                                                      const uint32_t* __restrict__ pos, uint32_t count) {
    using T = typename Payload<W>::T;
    T* d = reinterpret_cast<T*>(data);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t q = __ldg(&pos[i]);
        T v;
        fill_item(v, i);
        if (q < n) d[q] = v;
    }
}

int test_scatter(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* pos, uint32_t count, cudaStream_t s) {
    if (count == 0) return RZ_OK;
    const int grid = ctx->sms * 8;
    switch (w) {
        case 4: scatter_kernel<4><<<grid, 256, 0, s>>>(static_cast<uint8_t*>(data), n, pos, count); break;
        case 8: scatter_kernel<8><<<grid, 256, 0, s>>>(static_cast<uint8_t*>(data), n, pos, count); break;
        case 16: scatter_kernel<16><<<grid, 256, 0, s>>>(static_cast<uint8_t*>(data), n, pos, count); break;
        case 32: scatter_kernel<32><<<grid, 256, 0, s>>>(static_cast<uint8_t*>(data), n, pos, count); break;
        default: return RZ_ERR_INVALID_ARG;
    }
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    return RZ_OK;
}

int test_barrier_timeout(rz_ctx* ctx, uint32_t spin_limit, uint32_t* status_out) {
    cudaStream_t s = nullptr;
    int st = reset_if_dirty(ctx, s);
    if (st != RZ_OK) return st;
    // A tag no real call uses; the slots it leaves behind are reset below.
    barrier_timeout_kernel<<<1, 32, 0, s>>>(ctx->ws.arrive, ctx->ws.status, spin_limit, 0xfffffff0u);
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    RZ_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    uint32_t h = 0;
    RZ_CUDA_TRY(ctx, cudaMemcpy(&h, ctx->ws.status, sizeof(h), cudaMemcpyDeviceToHost));
    RZ_CUDA_TRY(ctx, cudaMemset(ctx->ws.status, 0, sizeof(uint32_t)));
    ctx->ws.dirty = true;  // re-zero the barrier state before the next call
    *status_out = h;
    return RZ_OK;
}

}  // namespace rz
