// rz_cluster.cu -- single-list Redzone on one thread-block cluster (up to 16 CTAs on one GPC).
//
// Same phases and result as the grid-wide kernel in rz_single.cu (reference Algorithm 2,
// redzone.hxx:626-941), with the synchronisation moved on-chip:
//   * the k-bit red-zone bitmap lives in distributed shared memory: CTA c owns the bits of the
//     tail slots it classifies in phase B, and phase A marks them with remote atomics
//     (atomicOr through cluster.map_shared_rank) instead of L2 atomics;
//   * the three phase boundaries are hardware cluster barriers (barrier.cluster arrive/wait),
//     which need no polling, no timeout and no scratch state;
//   * per-CTA orphan counts are pushed into every CTA's shared memory before the last barrier,
//     so the prefix over CTAs is read locally (no CTA touches remote shared memory after it).
// For small and medium k this removes the two L2 round-trip-bound grid barriers, which dominate
// the grid kernel's latency; the grid kernel remains the schedule for large k.
#include <cooperative_groups.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "rz_common.cuh"
#include "rz_internal.h"

namespace cg = cooperative_groups;

namespace rz {

constexpr int kMaxCluster = 16;

struct ClusterParams {
    uint8_t* data;
    const uint32_t* idx;
    uint32_t n, k;
    uint32_t* dlist;
    uint32_t* slist;
    uint32_t* status;
    unsigned long long* dev_len;
    unsigned long long* stamps;  // nullable: 8 globaltimer stamps per CTA
    uint32_t validate;
};

template <int W, int IPT>
__global__ void redzone_cluster_kernel(const ClusterParams p) {
    using T = typename Payload<W>::T;
    RZ_STAMP(p, 0);
    cg::cluster_group cluster = cg::this_cluster();
    T* __restrict__ head = reinterpret_cast<T*>(p.data);
    const uint32_t n = p.n, k = p.k, cut = n - k;
    const T* __restrict__ tail = reinterpret_cast<const T*>(p.data) + cut;
    const int B = blockDim.x, nw = B >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t C = cluster.num_blocks();
    const uint32_t c = cluster.block_rank();
    const uint32_t TILE = uint32_t(B) * IPT;
    const uint32_t ntiles = (k + TILE - 1) / TILE;
    const uint32_t tpc = (ntiles + C - 1) / C;
    const uint32_t chunk_items = tpc * TILE;  // items (and bitmap bits) owned by each CTA
    const uint32_t t0 = min(c * tpc, ntiles);
    const uint32_t t1 = min(t0 + tpc, ntiles);
    const bool single = (tpc == 1);
    const uint32_t chunk_base = t0 * TILE;
    const uint32_t words = chunk_items >> 5;

    extern __shared__ uint32_t s_bits[];  // this CTA's slice of the red-zone bitmap
    __shared__ uint32_t s_cnt[2][8 * 32 + 1];
    __shared__ uint32_t s_counts[2 * kMaxCluster];  // dcnt[c'] at [c'], scnt[c'] at [16 + c']
    __shared__ uint32_t s_ps[kMaxCluster + 1];
    __shared__ uint32_t s_pd[kMaxCluster + 1];
    __shared__ int s_abort;

    if (p.validate) {
        // Every CTA reads the same status word written by the validation kernels, so the
        // decision is uniform over the cluster and no CTA is left waiting at a barrier.
        if (threadIdx.x == 0) s_abort = (__ldcg(p.status) & (ST_DUPLICATE | ST_RANGE)) != 0;
        __syncthreads();
        if (s_abort) return;
    }
    if (c == 0 && threadIdx.x == 0 && p.dev_len) *p.dev_len = (unsigned long long)(n - k);

    for (uint32_t w = threadIdx.x; w < words; w += B) s_bits[w] = 0u;

    uint32_t rr[IPT];
    T src[IPT];
    if (single && t0 < t1) {
        const uint32_t base = t0 * TILE;
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
            rr[j] = (i < k) ? __ldg(&p.idx[i]) : 0xffffffffu;
        }
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
            if (i < k) src[j] = tail[i];
        }
    }
    cluster.sync();  // every slice is zeroed and every CTA of the cluster is running

    // ---- phase A: mark red-zone sources in the owners' bitmap slices ----------------------------
    for (uint32_t t = t0; t < t1; ++t) {
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
            const uint32_t r = rr[j];
            if (i < k && r >= cut) {
                if (r >= n) {
                    atomicOr(p.status, ST_RANGE);
                } else {
                    const uint32_t off = r - cut;
                    const uint32_t owner = off / chunk_items;
                    const uint32_t local = off - owner * chunk_items;
                    uint32_t* slice = cluster.map_shared_rank(s_bits, owner);
                    const uint32_t bit = 1u << (local & 31u);
                    const uint32_t old = atomicOr(slice + (local >> 5), bit);
                    if (p.validate && (old & bit)) atomicOr(p.status, ST_DUPLICATE);
                }
            }
        }
    }
    RZ_STAMP(p, 1);
    cluster.sync();  // all marks have landed
    RZ_STAMP(p, 2);

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
                const uint32_t word = s_bits[(i - chunk_base) >> 5];
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
                if (dv[j] && !sv[j]) p.dlist[chunk_base + dcnt + (ex >> 16) + __popc(dmask[j] & lt)] = rr[j];
                if (sv[j] && !dv[j]) p.slist[chunk_base + scnt + (ex & 0xffffu) + __popc(smask[j] & lt)] = cut + i;
            }
        }
        dcnt += tot >> 16;
        scnt += tot & 0xffffu;
    }

    // ---- phase C: exchange counts on-chip, then pair orphans by global rank ---------------------
    RZ_STAMP(p, 3);
    if (threadIdx.x < C) {
        uint32_t* rc = cluster.map_shared_rank(s_counts, threadIdx.x);
        rc[c] = dcnt;
        rc[kMaxCluster + c] = scnt;
    }
    cluster.sync();  // counts and the global orphan lists are visible cluster-wide
    if (dcnt == 0u) {
        RZ_STAMP(p, 4);
        return;
    }
    if (threadIdx.x == 0) {
        uint32_t d = 0, s = 0;
        for (uint32_t q = 0; q < C; ++q) {
            s_pd[q] = d;
            s_ps[q] = s;
            d += s_counts[q];
            s += s_counts[kMaxCluster + q];
        }
        s_pd[C] = d;
        s_ps[C] = s;
    }
    __syncthreads();
    const uint32_t myd = s_pd[c];
    const uint32_t tot_s = s_ps[C];
    for (uint32_t r = threadIdx.x; r < dcnt; r += B) {
        const uint32_t jr = myd + r;
        if (jr >= tot_s) {
            atomicOr(p.status, ST_INCONSISTENT);
            continue;
        }
        const int c2 = owner_of_rank(s_ps, int(C), jr);
        const uint32_t base2 = min(uint32_t(c2) * tpc, ntiles) * TILE;
        const uint32_t pos = __ldcg(&p.slist[base2 + (jr - s_ps[c2])]);
        const uint32_t dest = __ldcg(&p.dlist[chunk_base + r]);
        head[dest] = reinterpret_cast<const T*>(p.data)[pos];
    }
    RZ_STAMP(p, 4);
}

// ------------------------------------------------------------------------------------------------
using ClusterFn = void (*)(const ClusterParams);

template <int W>
static ClusterFn cluster_fn(int items) {
    switch (items) {
        case 1: return redzone_cluster_kernel<W, 1>;
        case 2: return redzone_cluster_kernel<W, 2>;
        case 4: return redzone_cluster_kernel<W, 4>;
        case 8: return redzone_cluster_kernel<W, 8>;
        default: return nullptr;
    }
}
static ClusterFn cluster_fn(int w, int items) {
    switch (w) {
        case 4: return cluster_fn<4>(items);
        case 8: return cluster_fn<8>(items);
        case 16: return cluster_fn<16>(items);
        case 32: return cluster_fn<32>(items);
        default: return nullptr;
    }
}

int cluster_max_block(int w, int items) {
    ClusterFn f = cluster_fn(w, items);
    if (!f) return 0;
    cudaFuncAttributes a{};
    if (cudaFuncGetAttributes(&a, (const void*)f) != cudaSuccess) return 0;
    return a.maxThreadsPerBlock & ~31;
}

// Largest power-of-two cluster size <= want that the device can co-schedule for this kernel and
// shared-memory footprint (0 if none). Cached per (kernel, block, smem, want).
static int feasible_cluster(rz_ctx* ctx, ClusterFn f, int block, size_t smem, int want) {
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, size_t, int>, int> cache;
    std::lock_guard<std::mutex> g(mu);
    auto key = std::make_tuple((const void*)f, block, smem, want);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    int result = 0;
    for (int cs = want; cs >= 1; cs >>= 1) {
        cudaLaunchConfig_t lc{};
        lc.gridDim = dim3(unsigned(cs));
        lc.blockDim = dim3(unsigned(block));
        lc.dynamicSmemBytes = smem;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = unsigned(cs);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        lc.attrs = attr;
        lc.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, (const void*)f, &lc) == cudaSuccess && nclusters > 0) {
            result = cs;
            break;
        }
        cudaGetLastError();
    }
    (void)ctx;
    cache[key] = result;
    return result;
}

int launch_cluster(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx, uint32_t k,
                   const rz_launch_cfg& cfg, bool validate, cudaStream_t s, LaunchInfo* info) {
    ClusterFn f = cluster_fn(int(w), cfg.items);
    if (!f) return RZ_ERR_INVALID_ARG;
    int block = std::min(cfg.block, cluster_max_block(int(w), cfg.items));
    if (block < 32) return RZ_ERR_INVALID_ARG;
    const uint32_t tile = uint32_t(block) * uint32_t(cfg.items);
    const uint32_t ntiles = (k + tile - 1) / tile;
    int want = 4 * std::max(1, std::min(4, cfg.ctas_per_sm));
    while (want > 1 && uint32_t(want) > ntiles) want >>= 1;
    const uint32_t tpc = (ntiles + uint32_t(want) - 1) / uint32_t(want);
    size_t smem = size_t(tpc) * tile / 8;  // one bit per owned item
    if (smem + 16384 > ctx->smem_optin) return RZ_ERR_UNSUPPORTED;
    static bool attrs_set[4][4] = {};
    const int wi = w == 4 ? 0 : w == 8 ? 1 : w == 16 ? 2 : 3;
    const int ii = cfg.items == 1 ? 0 : cfg.items == 2 ? 1 : cfg.items == 4 ? 2 : 3;
    if (!attrs_set[wi][ii]) {
        RZ_CUDA_TRY(ctx, cudaFuncSetAttribute((const void*)f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        RZ_CUDA_TRY(ctx, cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              int(ctx->smem_optin) - 16384));
        attrs_set[wi][ii] = true;
    }
    int cs = feasible_cluster(ctx, f, block, smem, want);
    if (cs < 1) return RZ_ERR_UNSUPPORTED;
    if (cs != want) {
        // A smaller cluster owns more items per CTA: recompute the bitmap slice size.
        const uint32_t tpc2 = (ntiles + uint32_t(cs) - 1) / uint32_t(cs);
        smem = size_t(tpc2) * tile / 8;
        if (smem + 16384 > ctx->smem_optin) return RZ_ERR_UNSUPPORTED;
    }
    int st = ensure_lists(ctx, k);
    if (st != RZ_OK) return st;

    ClusterParams p;
    p.data = static_cast<uint8_t*>(data);
    p.idx = idx;
    p.n = n;
    p.k = k;
    p.dlist = ctx->ws.dlist;
    p.slist = ctx->ws.slist;
    p.status = ctx->ws.status;
    p.dev_len = ctx->ws.dev_len;
    p.stamps = ctx->ws.stamps_on ? ctx->ws.stamps : nullptr;
    p.validate = validate ? 1u : 0u;

    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(unsigned(cs));
    lc.blockDim = dim3(unsigned(block));
    lc.dynamicSmemBytes = smem;
    lc.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(cs);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    RZ_CUDA_TRY(ctx, cudaLaunchKernelEx(&lc, f, p));
    if (info) {
        info->grid = cs;
        info->block = block;
        info->items = cfg.items;
        info->launches += 1;
    }
    return RZ_OK;
}

}  // namespace rz
