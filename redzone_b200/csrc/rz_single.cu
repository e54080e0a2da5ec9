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
// The O(n) partition comparator is in rz_partition.cu; the cluster schedule in rz_cluster.cu.
#include <algorithm>
#include <cstdio>

#include "rz_common.cuh"
#include "rz_internal.h"

namespace rz {

struct SingleParams {
    uint8_t* data;
    const uint32_t* idx;
    uint32_t n, k;
    uint32_t* bitmap;
    uint32_t* dlist;
    uint32_t* slist;
    uint32_t* epoch;
    uint32_t* arrive;
    unsigned long long* cnt_words;
    uint32_t* status;
    unsigned long long* dev_len;
    unsigned long long* stamps;  // nullable: 8 globaltimer stamps per CTA
    uint32_t spin_limit;
    uint32_t validate;
};

// ------------------------------------------------------------------------------------------------
// Redzone, one list, G persistent CTAs (G == 1 degenerates to block-level synchronisation).
// ------------------------------------------------------------------------------------------------
template <int W, int IPT>
__global__ void redzone_single_kernel(const SingleParams p) {
    using T = typename Payload<W>::T;
    RZ_STAMP(p, 0);
    T* __restrict__ head = reinterpret_cast<T*>(p.data);
    const uint32_t n = p.n, k = p.k, cut = n - k;
    const T* __restrict__ tail = reinterpret_cast<const T*>(p.data) + cut;
    const int B = blockDim.x, nw = B >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t TILE = uint32_t(B) * IPT;
    const uint32_t ntiles = (k + TILE - 1) / TILE;
    const uint32_t G = gridDim.x;
    const uint32_t tpc = (ntiles + G - 1) / G;
    const uint32_t t0 = min(blockIdx.x * tpc, ntiles);
    const uint32_t t1 = min(t0 + tpc, ntiles);
    const bool single = (tpc == 1);
    const uint32_t chunk_base = t0 * TILE;

    __shared__ uint32_t s_cnt[2][8 * 32 + 1];
    __shared__ uint32_t s_scan[33];
    __shared__ uint32_t s_pd[kMaxGrid + 1];
    __shared__ uint32_t s_ps[kMaxGrid + 1];
    __shared__ int s_abort;
    __shared__ uint32_t s_tag;

    if (threadIdx.x == 0) {
        s_tag = (G > 1) ? ld_acquire(p.epoch) + 1u : 0u;
        s_abort = p.validate ? ((__ldcg(p.status) & (ST_DUPLICATE | ST_RANGE)) != 0) : 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && p.dev_len) *p.dev_len = (unsigned long long)(n - k);

    uint32_t rr[IPT];
    T src[IPT];

    // ---- phase A: mark the red zone ---------------------------------------------------------
    // The loads are issued before the first __syncthreads so they overlap the epoch read.
    for (uint32_t t = t0; t < t1; ++t) {
        const uint32_t base = t * TILE;
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
            rr[j] = (i < k) ? __ldg(&p.idx[i]) : 0xffffffffu;
        }
        if (single) {
            // Pull this CTA's tail window into L2 while the grid waits at the barrier. A prefetch
            // is not an outstanding access the arrival's release has to wait for (a load is).
            const uint32_t cnt = min(TILE, k - base);
            prefetch_l2(tail + base, size_t(cnt) * W);
        }
        if (t == t0) {
            __syncthreads();  // s_abort / s_tag
            if (s_abort) return;  // validation failed: leave the caller's data untouched
        }
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
            const uint32_t r = rr[j];
            if (i < k && r >= cut) {
                if (r >= n) {
                    atomicOr(p.status, ST_RANGE);
                } else {
                    const uint32_t off = r - cut;
                    const uint32_t bit = 1u << (off & 31u);
                    if (p.validate) {
                        if (atomicOr(&p.bitmap[off >> 5], bit) & bit) atomicOr(p.status, ST_DUPLICATE);
                    } else {
                        atomicOr(&p.bitmap[off >> 5], bit);
                    }
                }
            }
        }
    }
    if (t0 >= t1) {
        __syncthreads();
        if (s_abort) return;
    }
    RZ_STAMP(p, 1);
    const uint32_t tag = s_tag;
    if (G > 1) {
        flag_arrive(p.arrive, blockIdx.x, tag);
        RZ_STAMP(p, 5);
        if (!flag_wait_all(p.arrive, G, tag, p.status, p.spin_limit)) return;
        // Every CTA has read the epoch (it arrived): advance it for the next call.
        if (blockIdx.x == 0 && threadIdx.x == 0) *p.epoch = tag;
    } else {
        __syncthreads();
    }
    RZ_STAMP(p, 2);

    // ---- phase B: classify, fill holes, collect orphans --------------------------------------
    // With one tile per CTA the hole writes are issued only after the orphan counts have been
    // published (below), so the publishing release does not wait for ~k scattered stores.
    uint32_t dcnt = 0, scnt = 0;
    const int E = IPT * nw;
    bool dv[IPT], sv[IPT];
#pragma unroll
    for (int j = 0; j < IPT; ++j) dv[j] = sv[j] = false;
    for (uint32_t t = t0, tt = 0; t < t1; ++t, ++tt) {
        const uint32_t base = t * TILE;
        if (!single) {
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
                rr[j] = (i < k) ? __ldg(&p.idx[i]) : 0xffffffffu;
            }
        }
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
            if (i < k) {
                const uint32_t word = __ldcg(&p.bitmap[i >> 5]);
                if (single) src[j] = tail[i];  // L2 hit (prefetched), issued with the bitmap load
                sv[j] = ((word >> (i & 31u)) & 1u) == 0u;
                dv[j] = rr[j] < cut;
            } else {
                sv[j] = false;
                dv[j] = false;
            }
        }
        if (!single) {
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
                if (dv[j] && sv[j]) src[j] = tail[i];
            }
#pragma unroll
            for (int j = 0; j < IPT; ++j)
                if (dv[j] && sv[j]) head[rr[j]] = src[j];
        }

        uint32_t dmask[IPT], smask[IPT];
        uint32_t* cbuf = s_cnt[tt & 1u];
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            dmask[j] = __ballot_sync(0xffffffffu, dv[j] && !sv[j]);
            smask[j] = __ballot_sync(0xffffffffu, sv[j] && !dv[j]);
            if (lane == 0) cbuf[j * nw + warp] = (uint32_t(__popc(dmask[j])) << 16) | uint32_t(__popc(smask[j]));
        }
        // Clear the bitmap words of this tile (lane 0 owns the 32 items of its warp and round).
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
                if (i < k) p.bitmap[i >> 5] = 0u;
            }
        }
        __syncthreads();
        if (warp == 0) {
            const int per = (E + 31) >> 5;
            const int lo = lane * per, hi = min(lo + per, E);
            uint32_t s = 0;
            for (int e = lo; e < hi; ++e) s += cbuf[e];
            const uint32_t inc = warp_inclusive_scan(s);
            uint32_t run = inc - s;
            for (int e = lo; e < hi; ++e) {
                const uint32_t x = cbuf[e];
                cbuf[e] = run;
                run += x;
            }
            if (lane == 31) cbuf[E] = inc;
        }
        __syncthreads();
        const uint32_t tot = cbuf[E];
        if (tot != 0u) {
            const uint32_t lt = lanemask_lt();
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t ex = cbuf[j * nw + warp];
                const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
                if (dv[j] && !sv[j]) {
                    const uint32_t rank = (ex >> 16) + __popc(dmask[j] & lt);
                    p.dlist[chunk_base + dcnt + rank] = rr[j];
                }
                if (sv[j] && !dv[j]) {
                    const uint32_t rank = (ex & 0xffffu) + __popc(smask[j] & lt);
                    p.slist[chunk_base + scnt + rank] = cut + i;
                }
            }
        }
        dcnt += tot >> 16;
        scnt += tot & 0xffffu;
    }
    RZ_STAMP(p, 3);

    // ---- phase C: pair destination orphans with source orphans of equal global rank ------------
    if (G > 1) {
        __syncthreads();  // this CTA's orphan-list writes precede the release below
        if (threadIdx.x == 0) {
            const unsigned long long hi = (unsigned long long)tag << 32;
            st_release_u64(&p.cnt_words[blockIdx.x], hi | dcnt);
            st_release_u64(&p.cnt_words[G + blockIdx.x], hi | scnt);
        }
    }
    if (single) {
#pragma unroll
        for (int j = 0; j < IPT; ++j)
            if (dv[j] && sv[j]) head[rr[j]] = src[j];
    }
    if (G > 1) {
        if (dcnt == 0u) {
            RZ_STAMP(p, 4);
            return;
        }
        int ok = 1;
        for (uint32_t c = threadIdx.x; c < 2 * G && ok; c += B) {
            uint32_t it = 0;
            unsigned long long w = ld_relaxed_u64(&p.cnt_words[c]);
            while (uint32_t(w >> 32) != tag) {
                if (++it > p.spin_limit) {
                    ok = 0;
                    break;
                }
                w = ld_relaxed_u64(&p.cnt_words[c]);
            }
            if (c < G) s_pd[c] = uint32_t(w);
            else s_ps[c - G] = uint32_t(w);
        }
        if (!__syncthreads_and(ok)) {
            if (threadIdx.x == 0) atomicOr(p.status, ST_TIMEOUT);
            return;
        }
        if (threadIdx.x == 0) fence_acq_rel_gpu();  // the other CTAs' source-orphan lists
        __syncthreads();
        block_scan_array(s_pd, int(G), s_scan);
        block_scan_array(s_ps, int(G), s_scan);
    } else {
        if (dcnt == 0u) {
            RZ_STAMP(p, 4);
            return;
        }
        if (threadIdx.x == 0) {
            s_pd[0] = 0; s_pd[1] = dcnt;
            s_ps[0] = 0; s_ps[1] = scnt;
        }
        __syncthreads();
    }
    const uint32_t myd = s_pd[blockIdx.x];
    const uint32_t tot_s = s_ps[G];
    for (uint32_t r = threadIdx.x; r < dcnt; r += B) {
        const uint32_t jr = myd + r;
        if (jr >= tot_s) {
            atomicOr(p.status, ST_INCONSISTENT);
            continue;
        }
        const int c2 = owner_of_rank(s_ps, int(G), jr);
        const uint32_t base2 = min(uint32_t(c2) * tpc, ntiles) * TILE;
        const uint32_t pos = __ldcg(&p.slist[base2 + (jr - s_ps[c2])]);
        const uint32_t dest = __ldcg(&p.dlist[chunk_base + r]);
        head[dest] = reinterpret_cast<const T*>(p.data)[pos];
    }
    RZ_STAMP(p, 4);
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

int redzone_occupancy(int w, int items, int block) {
    SingleFn f = single_fn(w, items);
    if (!f) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)f, block, 0) != cudaSuccess) return 0;
    return nb;
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
    if (k <= kClusterMaxK) {
        // One 16-CTA cluster; up to 2^16 items this is a single tile per CTA.
        cfg->block = 1024; cfg->items = 4; cfg->ctas_per_sm = 4;
    } else {
        cfg->block = 512; cfg->items = 4; cfg->ctas_per_sm = 2;
    }
    if (w >= 16 && cfg->items > 2) cfg->items = 2;
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
    int occ = redzone_occupancy(int(w), cfg.items, cfg.block);
    if (occ <= 0) return RZ_ERR_INVALID_ARG;
    long grid = std::min<long>((long)cfg.ctas_per_sm, (long)occ) * ctx->sms;
    grid = std::min<long>(grid, (long)ntiles);
    grid = std::min<long>(grid, (long)kMaxGrid);
    if (sched == RZ_SCHED_BLOCK) grid = 1;
    if (grid < 1) grid = 1;
    // Re-balance: use as many CTAs as needed for the resulting tiles-per-CTA (no idle CTAs).
    const uint32_t tpc = (ntiles + uint32_t(grid) - 1) / uint32_t(grid);
    grid = (ntiles + tpc - 1) / tpc;

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

    SingleFn f = single_fn(int(w), cfg.items);
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(unsigned(grid));
    lc.blockDim = dim3(unsigned(cfg.block));
    lc.dynamicSmemBytes = 0;
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
