// rz_single.cu -- single-list Redzone (persistent, grid-wide) and the O(n) partition comparator.
//
// Redzone follows Algorithm 2 of the reference (RemoveFromList_GPUWide, redzone.hxx:626-941) and
// its CPU form (redzone_CPU, Redzone_CPU.hxx:150-248). The phases are the reference's; the data
// layout and synchronisation are this library's own:
//   * Phase A (mark, reference :698-706): every index in the red zone [cut, n) sets one bit of a
//     k-bit bitmap in scratch (atomicOr) instead of writing an in-band 0x80000000 sentinel into
//     the caller's tail, so any payload width works and the tail is never written.
//   * Grid barrier: a bounded generation barrier (rz_common.cuh) replaces cg::grid.sync().
//   * Phase B (fill holes, reference :752-822): items are processed in tiles of B*IPT, item
//     (j, t) of a tile at i = base + j*B + t, so every warp load of the index list and of the tail
//     window is a contiguous 128-byte (or 32*W-byte) segment. Valid/valid pairs are moved at once;
//     orphans get their rank in i order from per-(j, warp) ballot counts and one scan per tile,
//     and are written to per-CTA regions of scratch lists (the caller's index list is const).
//     Each tile clears the bitmap words it read, which leaves the bitmap zero for the next call.
//   * Phase C (pair orphans, reference :834-934): only CTAs that own destination orphans wait for
//     the others; they prefix the per-CTA counts and binary-search the owner of each source rank
//     (instead of the reference's LoadBalance linear search, :477-524).
// The partition comparator is a mark pass plus a single-pass, in-place, stable compaction with
// decoupled look-back (the O(n) algorithms of cuCompactor.cuh:29-87 and Thrust_remove.hxx:15-17).
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
    uint32_t* counts;
    GridSync* sync;
    uint32_t* status;
    unsigned long long* dev_len;
    uint32_t spin_limit;
    uint32_t validate;
};

// ------------------------------------------------------------------------------------------------
// Redzone, one list, G persistent CTAs (G == 1 degenerates to block-level synchronisation).
// ------------------------------------------------------------------------------------------------
template <int W, int IPT>
__global__ void redzone_single_kernel(const SingleParams p) {
    using T = typename Payload<W>::T;
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

    if (p.validate) {
        // Validation ran earlier in the stream; on failure leave the caller's data untouched.
        if (threadIdx.x == 0) s_abort = (__ldcg(p.status) & (ST_DUPLICATE | ST_RANGE)) != 0;
        __syncthreads();
        if (s_abort) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && p.dev_len) *p.dev_len = (unsigned long long)(n - k);

    uint32_t rr[IPT];
    T src[IPT];

    // ---- phase A: mark the red zone ---------------------------------------------------------
    for (uint32_t t = t0; t < t1; ++t) {
        const uint32_t base = t * TILE;
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
            rr[j] = (i < k) ? __ldg(&p.idx[i]) : 0xffffffffu;
        }
        if (single) {
            // Issue the tail loads now; they complete while the grid waits at the barrier.
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
                if (i < k) src[j] = tail[i];
            }
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
                    const uint32_t old = atomicOr(&p.bitmap[off >> 5], bit);
                    if (p.validate && (old & bit)) atomicOr(p.status, ST_DUPLICATE);
                }
            }
        }
    }
    if (G > 1) {
        if (!grid_barrier(p.sync, G, true, p.status, p.spin_limit)) return;
    } else {
        __threadfence_block();
        __syncthreads();
    }

    // ---- phase B: classify, fill holes, collect orphans --------------------------------------
    uint32_t dcnt = 0, scnt = 0;
    const int E = IPT * nw;
    for (uint32_t t = t0, tt = 0; t < t1; ++t, ++tt) {
        const uint32_t base = t * TILE;
        if (!single) {
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
                rr[j] = (i < k) ? __ldg(&p.idx[i]) : 0xffffffffu;
            }
        }
        bool dv[IPT], sv[IPT];
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
            if (i < k) {
                const uint32_t word = __ldcg(&p.bitmap[i >> 5]);
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
        }
#pragma unroll
        for (int j = 0; j < IPT; ++j)
            if (dv[j] && sv[j]) head[rr[j]] = src[j];

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

    // ---- phase C: pair destination orphans with source orphans of equal global rank ------------
    if (G > 1) {
        if (threadIdx.x == 0) {
            p.counts[blockIdx.x] = dcnt;
            p.counts[G + blockIdx.x] = scnt;
            __threadfence();
        }
        if (!grid_barrier(p.sync, G, dcnt > 0u, p.status, p.spin_limit)) return;
        if (dcnt == 0u) return;
        for (uint32_t c = threadIdx.x; c < G; c += B) {
            s_pd[c] = __ldcg(&p.counts[c]);
            s_ps[c] = __ldcg(&p.counts[G + c]);
        }
        __syncthreads();
        block_scan_array(s_pd, int(G), s_scan);
        block_scan_array(s_ps, int(G), s_scan);
    } else {
        if (dcnt == 0u) return;
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
// O(n) partition comparator: mark, then stable in-place compaction with decoupled look-back.
// ------------------------------------------------------------------------------------------------
__global__ void partition_mark_kernel(const uint32_t* __restrict__ idx, uint32_t k, uint32_t n,
                                      uint32_t* __restrict__ bits, uint32_t* status, uint32_t validate) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        const uint32_t r = __ldg(&idx[i]);
        if (r >= n) {
            atomicOr(status, ST_RANGE);
            continue;
        }
        const uint32_t bit = 1u << (r & 31u);
        const uint32_t old = atomicOr(&bits[r >> 5], bit);
        if (validate && (old & bit)) atomicOr(status, ST_DUPLICATE);
    }
}

// Look-back state word: bits 62-63 = flag (1 aggregate, 2 inclusive prefix), bits 0-61 = value.
constexpr unsigned long long kFlagAgg = 1ull << 62;
constexpr unsigned long long kFlagInc = 2ull << 62;
constexpr unsigned long long kValMask = (1ull << 62) - 1;

template <int W, int IPT>
__global__ void partition_compact_kernel(uint8_t* data, uint32_t n, uint32_t* __restrict__ bits,
                                         unsigned long long* state, uint32_t* status,
                                         uint32_t spin_limit, unsigned long long* dev_len,
                                         uint32_t new_len) {
    using T = typename Payload<W>::T;
    T* A = reinterpret_cast<T*>(data);
    const int B = blockDim.x, nw = B >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t TILE = uint32_t(B) * IPT;
    unsigned long long* ticket = state;       // state[0] = ticket counter
    unsigned long long* tstate = state + 1;   // per-tile look-back words
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_cnt[8 * 32 + 1];
    __shared__ unsigned long long s_excl;
    // The tile's values pass through shared memory: the store needs each load's result, so once
    // the barrier below completes every load of this tile has landed. Only then may the tile
    // publish its count, which lets later tiles write over this tile's input range.
    __shared__ T s_stage[IPT * 256];
    if (threadIdx.x == 0) s_tile = uint32_t(atomicAdd(ticket, 1ull));
    if (blockIdx.x == 0 && threadIdx.x == 0 && dev_len) *dev_len = new_len;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t base = tile * TILE;

    T v[IPT];
    bool keep[IPT];
    if (B > 256) return;  // s_stage is sized for 256 threads (the only block size launched)
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
        keep[j] = false;
        if (i < n) {
            v[j] = A[i];
            const uint32_t word = __ldcg(&bits[i >> 5]);
            keep[j] = ((word >> (i & 31u)) & 1u) == 0u;
        }
    }
#pragma unroll
    for (int j = 0; j < IPT; ++j)
        if (base + uint32_t(j) * B + threadIdx.x < n) s_stage[j * B + threadIdx.x] = v[j];
    uint32_t km[IPT];
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        km[j] = __ballot_sync(0xffffffffu, keep[j]);
        if (lane == 0) s_cnt[j * nw + warp] = __popc(km[j]);
    }
    if (lane == 0) {
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
            if (i < n) bits[i >> 5] = 0u;
        }
    }
    __syncthreads();
    const int E = IPT * nw;
    if (warp == 0) {
        const int per = (E + 31) >> 5;
        const int lo = lane * per, hi = min(lo + per, E);
        uint32_t s = 0;
        for (int e = lo; e < hi; ++e) s += s_cnt[e];
        const uint32_t inc = warp_inclusive_scan(s);
        uint32_t run = inc - s;
        for (int e = lo; e < hi; ++e) {
            const uint32_t x = s_cnt[e];
            s_cnt[e] = run;
            run += x;
        }
        if (lane == 31) s_cnt[E] = inc;
    }
    __syncthreads();
    if (warp == 0) {
        const unsigned long long agg = s_cnt[E];
        if (lane == 0) {
            __threadfence();
            st_release_u64(&tstate[tile], (tile == 0 ? kFlagInc : kFlagAgg) | agg);
        }
        unsigned long long excl = 0;
        if (tile > 0) {
            int64_t pred = int64_t(tile) - 1 - lane;
            bool done = false;
            uint32_t it = 0;
            while (!done) {
                unsigned long long s = kFlagInc;  // lanes before tile 0 act as a zero prefix
                if (pred >= 0) {
                    s = ld_acquire_u64(&tstate[pred]);
                    while ((s >> 62) == 0ull) {
                        if (++it > spin_limit) break;
                        __nanosleep(32);
                        s = ld_acquire_u64(&tstate[pred]);
                    }
                }
                if (__any_sync(0xffffffffu, it > spin_limit)) {
                    if (lane == 0) atomicOr(status, ST_TIMEOUT);
                    excl = 0;
                    break;
                }
                const uint32_t incmask = __ballot_sync(0xffffffffu, (s >> 62) == 2ull);
                // Lanes up to and including the nearest inclusive prefix contribute.
                const int stop = incmask ? __ffs(incmask) - 1 : 32;
                unsigned long long val = (lane <= stop) ? (pred >= 0 ? (s & kValMask) : 0ull) : 0ull;
#pragma unroll
                for (int d = 16; d > 0; d >>= 1) val += __shfl_down_sync(0xffffffffu, val, d);
                excl += __shfl_sync(0xffffffffu, val, 0);
                if (incmask) done = true;
                else pred -= 32;
            }
            if (lane == 0) st_release_u64(&tstate[tile], kFlagInc | (excl + agg));
        }
        if (lane == 0) s_excl = excl;
    }
    __syncthreads();
    const unsigned long long excl = s_excl;
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        if (keep[j]) {
            const unsigned long long dst = excl + s_cnt[j * nw + warp] + __popc(km[j] & lt);
            A[dst] = s_stage[j * B + threadIdx.x];
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Barrier-timeout test kernel: one CTA waits for an arrival count that can never be reached.
// ------------------------------------------------------------------------------------------------
__global__ void barrier_timeout_kernel(GridSync* gs, uint32_t* status, uint32_t spin_limit) {
    grid_barrier(gs, gridDim.x + 1u, true, status, spin_limit);
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
    if (k <= 2048u) {
        cfg->block = 256; cfg->items = 8; cfg->ctas_per_sm = 1;
    } else if (k <= (1u << 22)) {
        cfg->block = 256; cfg->items = 4; cfg->ctas_per_sm = 1;
    } else {
        cfg->block = 512; cfg->items = 4; cfg->ctas_per_sm = 2;
    }
    if (w >= 16 && cfg->items > 4) cfg->items = 4;
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
    const uint32_t tile = uint32_t(cfg.block) * uint32_t(cfg.items);
    const uint32_t ntiles = (k + tile - 1) / tile;
    int occ = redzone_occupancy(int(w), cfg.items, cfg.block);
    if (occ <= 0) return RZ_ERR_INVALID_ARG;
    long grid = std::min<long>((long)cfg.ctas_per_sm, (long)occ) * ctx->sms;
    if (cfg.ctas_per_sm <= 0) grid = ctx->sms;
    grid = std::min<long>(grid, (long)ntiles);
    grid = std::min<long>(grid, (long)kMaxGrid);
    if (flags & RZ_FORCE_BLOCK) grid = 1;
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
    p.counts = ctx->ws.counts;
    p.sync = ctx->ws.sync;
    p.status = ctx->ws.status;
    p.dev_len = ctx->ws.dev_len;
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

template <int W>
static void (*part_fn())(uint8_t*, uint32_t, uint32_t*, unsigned long long*, uint32_t*, uint32_t,
                         unsigned long long*, uint32_t) {
    constexpr int IPT = W == 4 ? 8 : W == 8 ? 8 : W == 16 ? 4 : 2;
    return partition_compact_kernel<W, IPT>;
}
static int part_items(int w) { return w == 4 ? 8 : w == 8 ? 8 : w == 16 ? 4 : 2; }

int launch_partition(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx, uint32_t k,
                     uint32_t flags, cudaStream_t s, LaunchInfo* info) {
    const int block = 256;
    const int items = part_items(int(w));
    const uint32_t tile = uint32_t(block * items);
    const uint32_t ntiles = (n + tile - 1) / tile;
    int st = ensure_partition(ctx, n, ntiles);
    if (st != RZ_OK) return st;
    st = reset_if_dirty(ctx, s);
    if (st != RZ_OK) return st;
    const bool validate = (flags & RZ_VALIDATE) != 0;
    RZ_CUDA_TRY(ctx, cudaMemsetAsync(ctx->ws.tile_state, 0, sizeof(unsigned long long) * (size_t(ntiles) + 1), s));
    const int mgrid = std::max(1, std::min<int>(ctx->sms * 8, int((k + 255) / 256)));
    partition_mark_kernel<<<mgrid, 256, 0, s>>>(idx, k, n, ctx->ws.part_bits, ctx->ws.status, validate ? 1u : 0u);
    auto* f = w == 4 ? part_fn<4>() : w == 8 ? part_fn<8>() : w == 16 ? part_fn<16>() : part_fn<32>();
    f<<<ntiles, block, 0, s>>>(static_cast<uint8_t*>(data), n, ctx->ws.part_bits, ctx->ws.tile_state,
                               ctx->ws.status, kSpinLimit, ctx->ws.dev_len, n - k);
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    if (info) {
        info->grid = int(ntiles);
        info->block = block;
        info->items = items;
        info->launches = 2;  // the look-back state memset is a copy-engine node, not a kernel
    }
    return RZ_OK;
}

int test_barrier_timeout(rz_ctx* ctx, uint32_t spin_limit, uint32_t* status_out) {
    cudaStream_t s = nullptr;
    int st = reset_if_dirty(ctx, s);
    if (st != RZ_OK) return st;
    barrier_timeout_kernel<<<1, 32, 0, s>>>(ctx->ws.sync, ctx->ws.status, spin_limit);
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    RZ_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    uint32_t h = 0;
    RZ_CUDA_TRY(ctx, cudaMemcpy(&h, ctx->ws.status, sizeof(h), cudaMemcpyDeviceToHost));
    RZ_CUDA_TRY(ctx, cudaMemset(ctx->ws.status, 0, sizeof(uint32_t)));
    // The abandoned arrival left the barrier counter at 1: reset the barrier state.
    RZ_CUDA_TRY(ctx, cudaMemset(ctx->ws.sync, 0, sizeof(GridSync)));
    *status_out = h;
    return RZ_OK;
}

}  // namespace rz
