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
// list (k/Q entries, held in registers: one DRAM round trip), lists the slice's red entries in
// position order in its shared memory and marks them in two partial k-bit maps. One hardware
// cluster barrier; then each CTA reads the Q lists through distributed shared memory (in rank
// order = position order) into its own maps and red-entry arrays, and derives everything from
// them. No grid barrier, no flags in global memory, no cooperative launch, no scratch state
// between calls. The whole index list is read once per cluster (L2 hits after the first).
// When the cluster's red entries exceed kFastMaxRed (only at k^2/n >~ 1000), the CTAs OR the
// partial maps instead and rank orphans by prefix counts over the map words (slower, exact).
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>

#include "rz_common.cuh"
#include "rz_internal.h"
#include "rz_single_kernel.cuh"

namespace cg = cooperative_groups;

namespace rz {

constexpr uint32_t kCscanQ = 8;       // CTAs per cluster (portable size)
constexpr int kCscanPer = 32;         // slice entries per thread (registers): k <= 32 * B * Q
constexpr uint32_t kCscanLcap = kFastMaxRed;  // red entries one CTA's list can hold

struct CscanParams {
    uint8_t* data;
    const uint32_t* idx;
    uint32_t n, k;
    uint32_t* status;
    unsigned long long* dev_len;
    unsigned long long* stamps;  // nullable: 8 globaltimer stamps per CTA
    uint32_t validate;
};

// Dynamic shared memory: full V and P maps, partial (this slice's) V and P maps, per-word prefix
// arrays of the slow path (two k-bit-map-sized arrays), red positions / values / source orphans
// (kFastMaxRed each) and this slice's list (kCscanLcap uint2).
__host__ __device__ inline size_t cscan_smem_bytes(uint32_t k) {
    const size_t kw = (k + 31) / 32;
    return (6 * kw + 3 * size_t(kFastMaxRed) + 2 * size_t(kCscanLcap)) * 4;
}

__device__ __forceinline__ void cluster_arrive() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

template <int W, int IPT>
__global__ void __launch_bounds__(256) redzone_cscan_kernel(const CscanParams p) {
    using T = typename Payload<W>::T;
    RZ_STAMP(p, 0);
    cg::cluster_group cluster = cg::this_cluster();
    T* __restrict__ head = reinterpret_cast<T*>(p.data);
    const uint32_t n = p.n, k = p.k, cut = n - k;
    const T* __restrict__ tail = reinterpret_cast<const T*>(p.data) + cut;
    const int B = blockDim.x, nw = B >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t Q = cluster.num_blocks(), q = cluster.block_rank();
    const uint32_t TILE = uint32_t(B) * IPT;
    const uint32_t ntiles = (k + TILE - 1) / TILE;
    const uint32_t t = blockIdx.x;  // this CTA's tile (none when t >= ntiles)
    const uint32_t chunk_base = min(t, ntiles) * TILE;
    const uint32_t kw = (k + 31) >> 5;
    const int E = IPT * nw;
    const uint32_t lt = lanemask_lt();

    extern __shared__ uint32_t s_dyn[];
    uint32_t* mapV = s_dyn;
    uint32_t* mapP = mapV + kw;
    uint32_t* pV = mapP + kw;   // this slice's red entries only (read by the cluster)
    uint32_t* pP = pV + kw;
    uint32_t* s_dpre = pP + kw;  // slow path: per-word prefix of destination orphans
    uint32_t* s_spre = s_dpre + kw;  // slow path: per-word prefix of source orphans
    uint32_t* s_pos = s_spre + kw;
    uint32_t* s_val = s_pos + kFastMaxRed;
    uint32_t* s_src = s_val + kFastMaxRed;
    uint2* s_list = reinterpret_cast<uint2*>(s_src + kFastMaxRed);
    __shared__ uint32_t s_cnt[2][8 * 32 + 1];
    __shared__ uint32_t s_scan[33];
    __shared__ uint32_t s_qc[kCscanQ + 1];  // red entries per cluster rank, then their prefix
    __shared__ uint32_t s_lcount, s_ovf, s_total;
    __shared__ int s_abort;

    if (threadIdx.x == 0) s_abort = p.validate ? ((__ldcg(p.status) & (ST_DUPLICATE | ST_RANGE)) != 0) : 0;
    if (blockIdx.x == 0 && threadIdx.x == 0 && p.dev_len) *p.dev_len = (unsigned long long)(n - k);

    // ---- loads: this CTA's tile (index + tail item) and its slice of the whole index list ----
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
    const uint32_t SL = (k + Q - 1) / Q;
    const uint32_t sb = min(q * SL, k), se = min(sb + SL, k);
    const uint32_t wbase = sb + uint32_t(warp) * 32u * kCscanPer;  // warp-contiguous, lane-strided
    uint32_t sv[kCscanPer];
#pragma unroll
    for (int j = 0; j < kCscanPer; ++j) {
        const uint32_t e = wbase + uint32_t(j) * 32u + uint32_t(lane);
        sv[j] = e < se ? __ldg(&p.idx[e]) : 0u;
    }
    for (uint32_t w = threadIdx.x; w < 4 * kw; w += B) s_dyn[w] = 0u;  // all four maps
    __syncthreads();  // s_abort, zeroed maps
    if (s_abort) {
        // Validation failed: leave the caller's data untouched. Every CTA still passes the same
        // two cluster-barrier phases as the normal path (cluster barriers have no time limit, so
        // their count must match on every path).
        cluster_arrive();
        cluster_wait();
        cluster_arrive();
        cluster_wait();
        return;
    }
    RZ_STAMP(p, 1);

    // ---- this slice's red entries, in position order: count, one block scan, write ----------
    uint32_t wcount = 0;
#pragma unroll
    for (int j = 0; j < kCscanPer; ++j) {
        const uint32_t e = wbase + uint32_t(j) * 32u + uint32_t(lane);
        const bool in = e < se;
        if (in && sv[j] >= n && sv[j] >= cut) atomicOr(p.status, ST_RANGE);
        const bool red = in && sv[j] >= cut && sv[j] < n;
        if (red) {
            const uint32_t v = sv[j] - cut;
            atomicOr(&pV[v >> 5], 1u << (v & 31u));
            atomicOr(&pP[e >> 5], 1u << (e & 31u));
        }
        wcount += __popc(__ballot_sync(0xffffffffu, red));
    }
    if (lane == 0) s_scan[warp] = wcount;
    __syncthreads();
    if (warp == 0) {
        const uint32_t x = lane < nw ? s_scan[lane] : 0u;
        const uint32_t inc = warp_inclusive_scan(x);
        if (lane < nw) s_scan[lane] = inc - x;
        if (lane == 31) {
            s_lcount = min(inc, kCscanLcap);
            s_ovf = inc > kCscanLcap ? 1u : 0u;
        }
    }
    __syncthreads();
    {
        uint32_t run = s_scan[warp];
#pragma unroll
        for (int j = 0; j < kCscanPer; ++j) {
            const uint32_t e = wbase + uint32_t(j) * 32u + uint32_t(lane);
            const bool red = e < se && sv[j] >= cut && sv[j] < n;
            const uint32_t m = __ballot_sync(0xffffffffu, red);
            const uint32_t r = run + __popc(m & lt);
            if (red && r < kCscanLcap) s_list[r] = make_uint2(e, sv[j] - cut);
            run += __popc(m);
        }
    }
    RZ_STAMP(p, 5);
    cluster.sync();  // every list, partial map and count of the cluster is complete
    RZ_STAMP(p, 2);

    // ---- the cluster's red entries, read through distributed shared memory -----------------
    if (threadIdx.x < 32) {
        uint32_t c = 0, o = 0;
        if (uint32_t(lane) < Q) {
            c = *cluster.map_shared_rank(&s_lcount, uint32_t(lane));
            o = *cluster.map_shared_rank(&s_ovf, uint32_t(lane));
        }
        const uint32_t inc = warp_inclusive_scan(c);
        if (uint32_t(lane) < Q) s_qc[lane] = inc - c;
        const uint32_t any_ovf = __any_sync(0xffffffffu, o != 0u);
        if (lane == 31) s_total = any_ovf ? 0xffffffffu : inc;
    }
    __syncthreads();
    const uint32_t R = s_total;
    const bool fast = R <= kFastMaxRed;
    if (fast) {
        for (uint32_t qq = 0; qq < Q; ++qq) {
            const uint32_t at = s_qc[qq];
            const uint32_t cnt = (qq + 1 < Q ? s_qc[qq + 1] : R) - at;
            const uint2* rl = cluster.map_shared_rank(s_list, qq);
            for (uint32_t e = threadIdx.x; e < cnt; e += B) {
                const uint2 en = rl[e];
                s_pos[at + e] = en.x;
                s_val[at + e] = en.y;
                atomicOr(&mapV[en.y >> 5], 1u << (en.y & 31u));
                atomicOr(&mapP[en.x >> 5], 1u << (en.x & 31u));
            }
        }
    } else {
        for (uint32_t w = threadIdx.x; w < kw; w += B) {
            uint32_t v = 0, pm = 0;
            for (uint32_t qq = 0; qq < Q; ++qq) {
                v |= *cluster.map_shared_rank(&pV[w], qq);
                pm |= *cluster.map_shared_rank(&pP[w], qq);
            }
            mapV[w] = v;
            mapP[w] = pm;
        }
    }
    cluster_arrive();  // this CTA's remote reads are done (it may leave once all have arrived)
    __syncthreads();
    RZ_STAMP(p, 6);

    uint32_t stot = 0;  // source orphans of the whole list
    uint32_t dbase = 0;  // destination orphans before this tile (fast path)
    uint32_t* cbuf = s_cnt[1];
    if (fast) {
        // Ranks inside this tile: one word of the V \ P map per (round, warp).
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i0 = chunk_base + uint32_t(j) * B + uint32_t(warp) * 32u;
                cbuf[j * nw + warp] = (t < ntiles && i0 < k) ? __popc(mapV[i0 >> 5] & ~mapP[i0 >> 5]) : 0u;
            }
        }
        // Source orphans compacted in position order; destination orphans before this tile and
        // in all: rounds of B red entries, per-warp ballot counts, one barrier per round.
        uint32_t dall = 0;
        for (uint32_t q0 = 0, rd = 0; q0 == 0 || q0 < R; q0 += B, ++rd) {
            uint32_t* wc = s_cnt[0] + 96u * (rd & 1u);
            const uint32_t e = q0 + threadIdx.x;
            uint32_t ps = 0;
            bool sf = false, af = false, df = false;
            if (e < R) {
                ps = s_pos[e];
                const uint32_t v = s_val[e];
                sf = !((mapV[ps >> 5] >> (ps & 31u)) & 1u);
                af = !((mapP[v >> 5] >> (v & 31u)) & 1u);
                df = af && v < chunk_base;
            }
            const uint32_t bs = __ballot_sync(0xffffffffu, sf);
            const uint32_t bd = __ballot_sync(0xffffffffu, df);
            const uint32_t ba = __ballot_sync(0xffffffffu, af);
            if (lane == 0) {
                wc[warp] = __popc(bs);
                wc[32 + warp] = __popc(bd);
                wc[64 + warp] = __popc(ba);
            }
            __syncthreads();
            uint32_t pre = 0, ts = 0;
            for (int w2 = 0; w2 < nw; ++w2) {
                const uint32_t x = wc[w2];
                pre += w2 < warp ? x : 0u;
                ts += x;
                dbase += wc[32 + w2];
                dall += wc[64 + w2];
            }
            if (sf) s_src[stot + pre + __popc(bs & lt)] = ps;
            stot += ts;
        }
        if (threadIdx.x == 0 && blockIdx.x == 0 && dall != stot) atomicOr(p.status, ST_INCONSISTENT);
        if (warp == 0) warp0_scan_counts(cbuf, E, lane);
        __syncthreads();
    } else {
        // Per-word prefixes of destination (V & ~P) and source (P & ~V) orphans, in word order:
        // warp w owns a contiguous block of words, lane l reads word j * 32 + l of it.
        const uint32_t per = (kw + B - 1) / B;
        const uint32_t wb = uint32_t(warp) * 32u * per;
        uint32_t ssum = 0, dsum = 0;  // counts can reach k here: summed separately, not packed
        for (uint32_t j = 0; j < per; ++j) {
            const uint32_t w = wb + j * 32u + uint32_t(lane);
            if (w < kw) {
                const uint32_t v = mapV[w], pm = mapP[w];
                ssum += uint32_t(__popc(pm & ~v));
                dsum += uint32_t(__popc(v & ~pm));
            }
        }
        ssum = warp_inclusive_scan(ssum);
        dsum = warp_inclusive_scan(dsum);
        if (lane == 31) {
            s_cnt[0][warp] = ssum;
            s_cnt[0][32 + warp] = dsum;
        }
        __syncthreads();
        if (warp == 0) {
            const uint32_t xs = lane < nw ? s_cnt[0][lane] : 0u, xd = lane < nw ? s_cnt[0][32 + lane] : 0u;
            const uint32_t is = warp_inclusive_scan(xs), id = warp_inclusive_scan(xd);
            if (lane < nw) {
                s_cnt[0][64 + lane] = is - xs;
                s_cnt[0][96 + lane] = id - xd;
            }
            if (lane == 31) {
                s_cnt[0][128] = is;
                s_cnt[0][129] = id;
            }
        }
        __syncthreads();
        uint32_t cs = s_cnt[0][64 + warp], cd = s_cnt[0][96 + warp];
        for (uint32_t j = 0; j < per; ++j) {
            const uint32_t w = wb + j * 32u + uint32_t(lane);
            uint32_t v = 0, pm = 0;
            if (w < kw) {
                v = mapV[w];
                pm = mapP[w];
            }
            const uint32_t xs = uint32_t(__popc(pm & ~v)), xd = uint32_t(__popc(v & ~pm));
            const uint32_t is = warp_inclusive_scan(xs), id = warp_inclusive_scan(xd);
            if (w < kw) {
                s_spre[w] = cs + is - xs;
                s_dpre[w] = cd + id - xd;
            }
            cs += __shfl_sync(0xffffffffu, is, 31);
            cd += __shfl_sync(0xffffffffu, id, 31);
        }
        stot = s_cnt[0][128];
        if (threadIdx.x == 0 && blockIdx.x == 0 && s_cnt[0][129] != stot) atomicOr(p.status, ST_INCONSISTENT);
        __syncthreads();
    }
    RZ_STAMP(p, 3);

    // ---- this tile: fill holes, pair destination orphans ---------------------------------------
    if (t < ntiles) {
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t i = chunk_base + uint32_t(j) * B + threadIdx.x;
            if (i >= k || rr[j] >= cut) continue;  // past the list, or a hole needing no fill
            const uint32_t vw = mapV[i >> 5];
            if (!((vw >> lane) & 1u)) {
                head[rr[j]] = src[j];  // valid source, valid destination
                continue;
            }
            const uint32_t below = __popc(vw & ~mapP[i >> 5] & lt);
            const uint32_t rank = fast ? dbase + cbuf[j * nw + warp] + below : s_dpre[i >> 5] + below;
            if (rank >= stot) continue;  // only with invalid input (reported above)
            uint32_t spos;
            if (fast) {
                spos = s_src[rank];
            } else {
                // The word holding the rank-th source orphan: last word whose prefix <= rank.
                uint32_t lo = 0, hi = kw;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (s_spre[mid] <= rank) lo = mid; else hi = mid;
                }
                uint32_t sw = mapP[lo] & ~mapV[lo];
                for (uint32_t c = rank - s_spre[lo]; c > 0u; --c) sw &= sw - 1u;  // drop lower ones
                spos = lo * 32u + uint32_t(__ffs(sw) - 1);
            }
            head[rr[j]] = tail[spos];
        }
    }
    RZ_STAMP(p, 4);
    cluster_wait();  // no CTA leaves while another may still read its shared memory
}

using CscanFn = void (*)(const CscanParams);

template <int W>
static CscanFn cscan_fn(int items) {
    switch (items) {
        case 1: return redzone_cscan_kernel<W, 1>;
        case 2: return redzone_cscan_kernel<W, 2>;
        case 4: return redzone_cscan_kernel<W, 4>;
        case 8: return redzone_cscan_kernel<W, 8>;
        default: return nullptr;
    }
}
static CscanFn cscan_fn(int w, int items) {
    switch (w) {
        case 4: return cscan_fn<4>(items);
        case 8: return cscan_fn<8>(items);
        case 16: return cscan_fn<16>(items);
        case 32: return cscan_fn<32>(items);
        default: return nullptr;
    }
}

int launch_cscan(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx, uint32_t k,
                 const rz_launch_cfg& cfg, bool validate, cudaStream_t s, LaunchInfo* info) {
    CscanFn f = cscan_fn(int(w), cfg.items);
    if (!f || k == 0) return RZ_ERR_INVALID_ARG;
    const int block = cfg.block;
    if (block > 256 || block < 32) return RZ_ERR_UNSUPPORTED;  // the slice lives in registers
    // Every slice must fit the registers of one pass: k <= kCscanPer * block * Q.
    if (uint64_t(k) > uint64_t(kCscanPer) * uint64_t(block) * kCscanQ) return RZ_ERR_UNSUPPORTED;
    const size_t smem = cscan_smem_bytes(k);
    if (smem + 4096 > ctx->smem_optin) return RZ_ERR_UNSUPPORTED;
    static std::atomic<uint64_t> attr_done[4][4];
    const int wi = w == 4 ? 0 : w == 8 ? 1 : w == 16 ? 2 : 3;
    const int ii = cfg.items == 1 ? 0 : cfg.items == 2 ? 1 : cfg.items == 4 ? 2 : 3;
    const uint64_t bit = 1ull << (ctx->device & 63);
    if (!(attr_done[wi][ii].load() & bit)) {
        RZ_CUDA_TRY(ctx, cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              int(ctx->smem_optin) - 4096));
        attr_done[wi][ii].fetch_or(bit);
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
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, (const void*)f, &lc) != cudaSuccess || nclusters < 1) {
        cudaGetLastError();
        return RZ_ERR_UNSUPPORTED;
    }
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
