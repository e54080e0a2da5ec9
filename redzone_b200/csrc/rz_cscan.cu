// rz_cscan.cu -- single-list Redzone without any grid-wide wait: the cluster-scan schedule.
//
// The canonical pairing (reference Algorithm 2, redzone.hxx:626-941; the rule is the same as in
// rz_single.cu) depends only on the red entries {(i, idx[i]) : idx[i] >= cut}: V = {idx[i] - cut}
// (tail positions whose item is removed) and P = {i} (holes that need no fill); destination
// orphans are V \ P and source orphans P \ V, each ranked by position. So a CTA that knows every
// red entry can fill its own holes and pair its own destination orphans with no other CTA.
//
// Schedule: G CTAs, one 1024..8192-item tile each, grouped in independent clusters of Q = 8.
// Every cluster finds all red entries on its own: CTA q of a cluster loads slice q of the index
// list (k/Q entries, 16-byte loads held in registers: one DRAM round trip) and PUSHES the slice's
// red entries, in position order, into a per-rank region of every cluster member's shared memory
// (remote stores through distributed shared memory), together with the slice's count. One
// hardware cluster barrier (release/acquire) makes every push visible; after it each CTA works
// from its own shared memory only. No grid barrier, no flags in global memory, no cooperative
// launch, no scratch state between calls. The whole index list is read once per cluster (L2 hits
// after the first).
// When a slice has more than kCscanRegCap red entries or the cluster more than kFastMaxRed (only
// at k^2/n >~ 1000 or with clustered removals near the end), the CTAs instead OR the slices'
// partial k-bit maps, read through distributed shared memory, and rank orphans by prefix counts
// over the map words (slower, exact).
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <tuple>

#include "rz_common.cuh"
#include "rz_internal.h"
#include "rz_pairfill.cuh"
#include "rz_single_kernel.cuh"

namespace cg = cooperative_groups;

namespace rz {

constexpr uint32_t kCscanQ = 8;          // CTAs per cluster (portable size)
constexpr int kCscanVec = 8;             // 16-byte slice loads per thread: 32 entries
constexpr uint32_t kCscanWarpSpan = 32u * 4u * kCscanVec;  // slice entries per warp (1024)
constexpr uint32_t kCscanRegCap = 256;   // red entries one CTA pushes to each cluster member
constexpr int kCscanMaxBlock = 512;

struct CscanParams {
    uint8_t* data;
    const uint32_t* idx;  // 16-byte aligned
    uint32_t n, k;
    uint32_t* status;
    unsigned long long* dev_len;
    unsigned long long* stamps;  // nullable: 8 globaltimer stamps per CTA
    uint32_t validate;
};

// Dynamic shared memory: the pairing layout of rz_pairfill.cuh (full V and P maps, the slow
// path's two prefix arrays, red positions / values / source orphans), then this slice's V and P
// maps and the Q push regions (kCscanRegCap uint2 each).
__host__ __device__ inline size_t cscan_smem_bytes(uint32_t k) {
    const size_t kw = (k + 31) / 32;
    return (pairfill_words(uint32_t(kw)) + 2 * kw) * 4 + size_t(kCscanQ) * kCscanRegCap * 8;
}

__device__ __forceinline__ void cluster_arrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_arrive_relaxed() {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
// Phase stamps of this kernel stay in thread 0's registers until the end: a global store before a
// release barrier would make that barrier wait for it, and so distort what is measured.
#define CS_STAMP(slot)                                      \
    do {                                                    \
        if (p.stamps && threadIdx.x == 0) st_[slot] = globaltimer(); \
    } while (0)

__device__ __forceinline__ uint4 ldg_nc_v4(const uint32_t* p) {
    uint4 v;
    asm volatile("ld.global.nc.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}
// Component c of v (c is a constant after unrolling).
__device__ __forceinline__ uint32_t lane_of(const uint4& v, int c) {
    return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
}

// MAXB: the launch bound (256, or 512 for the largest slices; 512 threads leave 128 registers
// per thread, which the wider payloads at 4..8 items per thread exceed).
template <int W, int IPT, int MAXB>
__global__ void __launch_bounds__(MAXB, 1) redzone_cscan_kernel(const CscanParams p) {
    using T = typename Payload<W>::T;
    // Barrier phase 0 (remote shared memory may be written only once every CTA of the cluster
    // runs): arrive now, wait just before the first push.
    cluster_arrive_relaxed();
    unsigned long long st_[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    CS_STAMP(0);
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t n = p.n, k = p.k, cut = n - k;
    const int B = blockDim.x, nw = B >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t q = cluster.block_rank();

    // ---- the critical path starts with this CTA's slice of the index list: issue it first ------
    // Slices are multiples of 4 entries (16-byte aligned); warp w of CTA q reads entries
    // [sb + w * 1024, +1024), lane l the four at +128 j + 4 l of round j.
    const uint32_t SL = ((k + kCscanQ - 1) / kCscanQ + 3u) & ~3u;
    const uint32_t sb = min(q * SL, k), se = min(sb + SL, k);
    const uint32_t wbase = sb + uint32_t(warp) * kCscanWarpSpan;
    uint4 sv[kCscanVec];
#pragma unroll
    for (int j = 0; j < kCscanVec; ++j) {
        const uint32_t e = wbase + uint32_t(j) * 128u + uint32_t(lane) * 4u;
        if (e + 4u <= se) {
            sv[j] = ldg_nc_v4(p.idx + e);
        } else {
            sv[j].x = e < se ? __ldg(p.idx + e) : 0u;
            sv[j].y = e + 1u < se ? __ldg(p.idx + e + 1u) : 0u;
            sv[j].z = e + 2u < se ? __ldg(p.idx + e + 2u) : 0u;
            sv[j].w = 0u;  // e + 3 >= se here
        }
    }

    T* __restrict__ head = reinterpret_cast<T*>(p.data);
    const T* __restrict__ tail = reinterpret_cast<const T*>(p.data) + cut;
    const uint32_t TILE = uint32_t(B) * IPT;
    const uint32_t ntiles = (k + TILE - 1) / TILE;
    const uint32_t t = blockIdx.x;  // this CTA's tile (none when t >= ntiles)
    const uint32_t chunk_base = min(t, ntiles) * TILE;
    const uint32_t kw = (k + 31) >> 5;

    extern __shared__ __align__(16) uint32_t s_dyn[];
    __shared__ uint32_t s_cnt[2][16 * 16 + 1];
    __shared__ uint32_t s_scan[33];
    const PairFillSmem pf{s_dyn, kw, s_cnt, s_scan};
    uint32_t* mapV = pf.mapV();
    uint32_t* mapP = pf.mapP();
    uint32_t* s_pos = pf.pos();
    uint32_t* s_val = pf.val();
    uint32_t* pV = s_dyn + pairfill_words(kw);  // this slice's red entries only (read by the cluster: slow path)
    uint32_t* pP = pV + kw;
    uint2* s_reg = reinterpret_cast<uint2*>(pP + kw);  // push region r: [r * cap, +cap)
    __shared__ uint32_t s_qcnt[kCscanQ];     // pushed: red entries of each rank's slice
    __shared__ uint32_t s_qc[kCscanQ + 1];   // their prefix
    __shared__ uint32_t s_total;
    __shared__ int s_abort;

    if (threadIdx.x == 0) s_abort = p.validate ? ((__ldcg(p.status) & (ST_DUPLICATE | ST_RANGE)) != 0) : 0;

    // ---- this CTA's tile: index and tail item (needed only by the final moves) ----------------
    uint32_t rr[IPT];
    T src[IPT];
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        const uint32_t i = chunk_base + uint32_t(j) * B + threadIdx.x;
        rr[j] = 0xffffffffu;
        if (t < ntiles && i < k) {
            rr[j] = __ldg(&p.idx[i]);
            src[j] = tail[i];
        }
    }
    for (uint32_t w = threadIdx.x; w < kw; w += B) {  // the four maps
        mapV[w] = 0u;
        mapP[w] = 0u;
        pV[w] = 0u;
        pP[w] = 0u;
    }
    __syncthreads();  // s_abort, zeroed maps
    if (s_abort) {
        // Validation failed: leave the caller's data untouched. Every CTA still passes the same
        // three cluster-barrier phases as the normal path (cluster barriers have no time limit,
        // so their count must match on every path).
        cluster_wait();
        cluster_arrive();
        cluster_wait();
        cluster_arrive();
        cluster_wait();
        return;
    }
    CS_STAMP(1);

    // ---- this slice's red entries: one bit per register entry (bit 4 j + c) -------------------
    uint32_t bits = 0, oor = 0;
#pragma unroll
    for (int j = 0; j < kCscanVec; ++j) {
        const uint32_t e = wbase + uint32_t(j) * 128u + uint32_t(lane) * 4u;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const uint32_t v = lane_of(sv[j], c);
            const bool in = e + uint32_t(c) < se;
            bits |= uint32_t(in && v - cut < k) << (4 * j + c);
            oor |= uint32_t(in && v >= n);
        }
    }
    if (__any_sync(0xffffffffu, oor != 0u) && lane == 0) atomicOr(p.status, ST_RANGE);
    const uint32_t wred = __reduce_add_sync(0xffffffffu, uint32_t(__popc(bits)));
    if (lane == 0) s_scan[warp] = wred;
    __syncthreads();
    if (warp == 0) {
        const uint32_t x = lane < nw ? s_scan[lane] : 0u;
        const uint32_t inc = warp_inclusive_scan(x);
        if (lane < nw) s_scan[lane] = inc - x;
        if (lane == 31) s_scan[32] = inc;
    }
    __syncthreads();
    cluster_wait();  // phase 0: every CTA of the cluster runs
    // The slice's count goes to every member (an overflowing count sends all of them to the slow
    // path, where the regions are not read).
    if (threadIdx.x < kCscanQ) *cluster.map_shared_rank(&s_qcnt[q], threadIdx.x) = s_scan[32];
    // Entries in position order (round j, then lane, then c): a warp scan per round that has any.
    const uint32_t wany = __reduce_or_sync(0xffffffffu, bits);
    if (wany) {
        uint32_t run = s_scan[warp];
#pragma unroll
        for (int j = 0; j < kCscanVec; ++j) {
            if (((wany >> (4 * j)) & 15u) == 0u) continue;  // warp-uniform
            const uint32_t nib = (bits >> (4 * j)) & 15u;
            const uint32_t x = uint32_t(__popc(nib));
            const uint32_t inc = warp_inclusive_scan(x);
            uint32_t r = run + inc - x;
            run += __shfl_sync(0xffffffffu, inc, 31);
            const uint32_t e0 = wbase + uint32_t(j) * 128u + uint32_t(lane) * 4u;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if (!((nib >> c) & 1u)) continue;
                const uint32_t e = e0 + uint32_t(c), v = lane_of(sv[j], c) - cut;
                atomicOr(&pV[v >> 5], 1u << (v & 31u));
                atomicOr(&pP[e >> 5], 1u << (e & 31u));
                if (r < kCscanRegCap) {
                    const uint2 en = make_uint2(e, v);
#pragma unroll
                    for (uint32_t d = 0; d < kCscanQ; ++d) cluster.map_shared_rank(s_reg, d)[q * kCscanRegCap + r] = en;
                }
                ++r;
            }
        }
    }
    CS_STAMP(5);
    cluster_arrive();  // phase 1: every push and partial map of this CTA is complete
    cluster_wait();
    CS_STAMP(2);

    // ---- the cluster's red entries, from this CTA's own shared memory ---------------------------
    if (threadIdx.x < 32) {
        const uint32_t c = uint32_t(lane) < kCscanQ ? s_qcnt[lane] : 0u;
        const uint32_t inc = warp_inclusive_scan(c);
        if (uint32_t(lane) < kCscanQ) s_qc[lane] = inc - c;
        const bool ovf = __any_sync(0xffffffffu, c > kCscanRegCap);
        if (lane == 31) s_total = (ovf || inc > kFastMaxRed) ? 0xffffffffu : inc;
    }
    __syncthreads();
    const uint32_t R = s_total;
    const bool fast = R <= kFastMaxRed;
    if (fast) {
        cluster_arrive_relaxed();  // phase 2: no remote access from here on
        for (uint32_t e = threadIdx.x; e < R; e += B) {
            uint32_t r = 0;
#pragma unroll
            for (uint32_t u = 1; u < kCscanQ; ++u) r += s_qc[u] <= e ? 1u : 0u;
            const uint2 en = s_reg[r * kCscanRegCap + (e - s_qc[r])];
            s_pos[e] = en.x;
            s_val[e] = en.y;
            atomicOr(&mapV[en.y >> 5], 1u << (en.y & 31u));
            atomicOr(&mapP[en.x >> 5], 1u << (en.x & 31u));
        }
    } else {
        for (uint32_t w = threadIdx.x; w < kw; w += B) {
            uint32_t v = 0, pm = 0;
#pragma unroll
            for (uint32_t d = 0; d < kCscanQ; ++d) {
                v |= *cluster.map_shared_rank(&pV[w], d);
                pm |= *cluster.map_shared_rank(&pP[w], d);
            }
            mapV[w] = v;
            mapP[w] = pm;
        }
        cluster_arrive();  // phase 2: this CTA's remote reads are done
    }
    __syncthreads();
    CS_STAMP(6);

    uint32_t stot, dbase;
    derive_pairing<IPT>(pf, R, k, chunk_base, t < ntiles, p.status, stot, dbase);
    CS_STAMP(3);

    // ---- this tile: fill holes, pair destination orphans ---------------------------------------
    if (t < ntiles) fill_holes<W, IPT>(pf, R, k, cut, chunk_base, stot, dbase, rr, src, head, tail);
    CS_STAMP(4);
    cluster_wait();  // phase 2: no CTA leaves while another may still read its shared memory
    if (blockIdx.x == 0 && threadIdx.x == 0 && p.dev_len) *p.dev_len = (unsigned long long)(n - k);
    if (p.stamps && threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < 8; ++i) p.stamps[blockIdx.x * kStampsPerCta + i] = st_[i];
    }
}

using CscanFn = void (*)(const CscanParams);

template <int W, int MAXB>
static CscanFn cscan_fn(int items) {
    switch (items) {
        case 1: return redzone_cscan_kernel<W, 1, MAXB>;
        case 2: return redzone_cscan_kernel<W, 2, MAXB>;
        case 4: return redzone_cscan_kernel<W, 4, MAXB>;
        case 8: return redzone_cscan_kernel<W, 8, MAXB>;
        default: return nullptr;
    }
}
template <int MAXB>
static CscanFn cscan_fn(int w, int items) {
    switch (w) {
        case 4: return cscan_fn<4, MAXB>(items);
        case 8: return cscan_fn<8, MAXB>(items);
        case 16: return cscan_fn<16, MAXB>(items);
        case 32: return cscan_fn<32, MAXB>(items);
        default: return nullptr;
    }
}

// Whether at least one Q-CTA cluster of (function, block, dynamic shared memory) can be resident:
// queried once per combination and device.
static bool cscan_cluster_fits(rz_ctx* ctx, CscanFn f, cudaLaunchConfig_t* lc) {
    static std::mutex mu;
    static std::map<std::tuple<int, const void*, unsigned, size_t>, bool> known;
    const auto key = std::make_tuple(ctx->device, (const void*)f, lc->blockDim.x, lc->dynamicSmemBytes);
    {
        std::lock_guard<std::mutex> g(mu);
        auto it = known.find(key);
        if (it != known.end()) return it->second;
    }
    int nclusters = 0;
    bool ok = cudaOccupancyMaxActiveClusters(&nclusters, (const void*)f, lc) == cudaSuccess && nclusters >= 1;
    if (!ok) cudaGetLastError();
    std::lock_guard<std::mutex> g(mu);
    known[key] = ok;
    return ok;
}

// Slice fit, register bound and shared memory of a (k, w, block, items) launch.
static bool cscan_fits(const rz_ctx* ctx, uint32_t k, uint32_t w, int block, int items) {
    if (block > kCscanMaxBlock || block < 32 || (block & 31)) return false;
    if (block > 256 && items * int(w) > 32) return false;  // 512 threads with wide items would spill
    const uint64_t sl = ((uint64_t(k) + kCscanQ - 1) / kCscanQ + 3) & ~uint64_t(3);
    if (sl > uint64_t(kCscanWarpSpan) * uint64_t(block / 32)) return false;
    return cscan_smem_bytes(k) + 4096 <= ctx->smem_optin;
}

bool cscan_default_cfg(const rz_ctx* ctx, uint32_t k, uint32_t w, rz_launch_cfg* cfg) {
    if (k > kCscanMaxK) return false;
    // About 64 CTAs (8 clusters): 256 threads with 1..4 items each, 512 threads beyond k = 2^16
    // (a 256-thread CTA holds a slice of at most 8192 entries).
    const int block = k > (1u << 16) ? 512 : 256;
    int items = 1;
    while (items < 4 && uint64_t(block) * items * 64 < k) items *= 2;
    if (!cscan_fits(ctx, k, w, block, items)) return false;
    cfg->block = block;
    cfg->items = items;
    cfg->ctas_per_sm = 2;  // used only by a grid-schedule fallback (misaligned index list)
    cfg->use_partition = 0;
    cfg->schedule = RZ_SCHED_CSCAN;
    return true;
}

int launch_cscan(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx, uint32_t k,
                 const rz_launch_cfg& cfg, bool validate, cudaStream_t s, LaunchInfo* info) {
    const int block = cfg.block;
    CscanFn f = block > 256 ? cscan_fn<512>(int(w), cfg.items) : cscan_fn<256>(int(w), cfg.items);
    if (!f || k == 0) return RZ_ERR_INVALID_ARG;
    // Every slice must fit the registers of one pass (ceil4(ceil(k / Q)) <= 32 * block) and the
    // index list is read in 16-byte units.
    if (!cscan_fits(ctx, k, w, block, cfg.items)) return RZ_ERR_UNSUPPORTED;
    if (reinterpret_cast<uintptr_t>(idx) & 15u) return RZ_ERR_UNSUPPORTED;
    const size_t smem = cscan_smem_bytes(k);
    static std::atomic<uint64_t> attr_done[2][4][4];
    const int bi = block > 256 ? 1 : 0;
    const int wi = w == 4 ? 0 : w == 8 ? 1 : w == 16 ? 2 : 3;
    const int ii = cfg.items == 1 ? 0 : cfg.items == 2 ? 1 : cfg.items == 4 ? 2 : 3;
    const uint64_t bit = 1ull << (ctx->device & 63);
    if (!(attr_done[bi][wi][ii].load() & bit)) {
        RZ_CUDA_TRY(ctx, cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              int(ctx->smem_optin) - 4096));
        attr_done[bi][wi][ii].fetch_or(bit);
    }
    const uint32_t tile = uint32_t(block) * uint32_t(cfg.items);
    const uint32_t ntiles = (k + tile - 1) / tile;
    const uint32_t grid = (ntiles + kCscanQ - 1) / kCscanQ * kCscanQ;

    CscanParams p;
    p.data = static_cast<uint8_t*>(data);
    p.idx = idx;
    p.n = n;
    p.k = k;
    p.status = ctx->ws.status;
    p.dev_len = ctx->ws.dev_len;
    p.stamps = ctx->ws.stamps_on ? ctx->ws.stamps : nullptr;
    p.validate = validate ? 1u : 0u;

    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(grid);
    lc.blockDim = dim3(unsigned(block));
    lc.dynamicSmemBytes = smem;
    lc.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kCscanQ;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    if (!cscan_cluster_fits(ctx, f, &lc)) return RZ_ERR_UNSUPPORTED;
    RZ_CUDA_TRY(ctx, cudaLaunchKernelEx(&lc, f, p));
    if (info) {
        info->grid = int(grid);
        info->block = block;
        info->items = cfg.items;
        info->launches += 1;
    }
    return RZ_OK;
}

}  // namespace rz
