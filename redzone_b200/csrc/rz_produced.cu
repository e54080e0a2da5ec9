// rz_produced.cu -- removal of a list made on the GPU, with the red-zone marking fused into its
// producer (the paper's "mark during producer", p.14). No counterpart in the reference's code:
// there, phase 1 (redzone.hxx:698-707) scans the finished list for entries >= n - k.
//
// The producer (rz_emit, include/redzone_device.cuh) appends each deleted row to a list and,
// when the row is >= n - capacity, also to a candidate list of (slot, row) pairs. Every red entry
// (idx[i] >= n - k, with k <= capacity) is among the candidates, so a CTA of the removal learns
// all red entries by reading the candidates -- typically a few dozen pairs -- instead of its
// share of a k-entry list plus an exchange with the other CTAs. The removal kernel therefore has
// no barrier of any kind between CTAs: each CTA reads its tile (index and tail item) and the
// candidates at once, builds the V and P maps in shared memory, orders the red entries by
// position and derives the canonical pairing exactly as the cluster-scan schedule does
// (rz_pairfill.cuh). k itself is read on the device: the host never waits for the producer.
// If the candidates overflowed their buffer, each CTA reads the whole list instead (exact,
// slower); if the list outgrew its capacity, nothing moves and the status says so.
//
// The same pairing kernel also serves two schedules of rz_remove on an ordinary index list:
//   scan-all (RZ_SCHED_SCANALL, the default for short lists): every CTA reads the whole list for
//     the red entries -- one grid, no wait of any kind;
//   split (RZ_SCHED_SPLIT): a scan grid lists the red entries as candidates and this kernel runs
//     as its programmatic dependent, loading its tile while the scan runs.
#include <algorithm>
#include <atomic>
#include <new>

#include "../../include/redzone_device.cuh"
#include "rz_common.cuh"
#include "rz_internal.h"
#include "rz_pairfill.cuh"

struct rz_producer {
    rz_ctx* ctx = nullptr;
    uint32_t* idx = nullptr;
    uint32_t* counts = nullptr;  // [0] rows, [1] candidates (own 256-byte block)
    uint32_t* cand = nullptr;    // (slot, row) pairs
    uint32_t capacity = 0;
    uint32_t cand_capacity = 0;
    uint32_t n = 0;
    bool have_n = false;
};

namespace rz {

constexpr uint32_t kProducedMaxK = 1u << 18;  // list capacity: four k-bit maps in shared memory
constexpr int kProducedBlock = 256;

// Dynamic shared memory for a list of at most `capacity` rows: V and P maps and the two prefix
// arrays of the slow path (capacity bits each), then ordered red positions / values, source
// orphans, and the unordered red entries as collected (kFastMaxRed words each).
static size_t produced_smem_bytes(uint32_t capacity) {
    return (pairfill_words((capacity + 31) / 32) + 2 * size_t(kFastMaxRed)) * 4;
}

// Produced lists: k = counts[0], candidates counted in counts[1]. Split schedule (rz_remove with
// a device index list, see below): k = k_fixed, candidates counted in *cand_count, written by the
// scan kernel this kernel waits for (pdl); the last CTA to read the count resets it (done).
struct ProducedParams {
    uint8_t* data;
    const uint32_t* idx;
    const uint32_t* counts;      // produced lists only
    const uint32_t* cand_count;  // counts + 1, or the split scan's counter
    uint32_t* done;              // split schedule: CTAs that have read *cand_count
    const uint2* cand;
    uint32_t n, k_fixed, capacity, cand_capacity;
    uint32_t* status;
    unsigned long long* dev_len;
    uint32_t validate;
    uint32_t pdl;                // wait for the preceding (scan) grid before reading candidates
    uint32_t full_scan;          // scan-all schedule: every CTA reads the whole (16-byte aligned) list
};

template <int W, int IPT>
__global__ void __launch_bounds__(kProducedBlock, 1) redzone_produced_kernel(const ProducedParams p) {
    using T = typename Payload<W>::T;
    const uint32_t k = p.k_fixed ? p.k_fixed : __ldcg(&p.counts[0]);
    const uint32_t n = p.n;
    if (k > p.capacity) {  // uniform: every CTA reads the same counts
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(p.status, ST_CAPACITY);
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && p.dev_len) *p.dev_len = (unsigned long long)(n - k);
    const uint32_t B = blockDim.x, TILE = B * IPT;
    const uint32_t ntiles = (k + TILE - 1) / TILE;
    const uint32_t t = blockIdx.x;
    if (t >= ntiles || k == n) return;  // no tile here, or nothing survives (nothing moves)
    const uint32_t cut = n - k, kw = (k + 31) >> 5, kwc = (p.capacity + 31) >> 5;
    const uint32_t chunk_base = t * TILE;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = int(B >> 5);
    T* __restrict__ head = reinterpret_cast<T*>(p.data);
    const T* __restrict__ tail = reinterpret_cast<const T*>(p.data) + cut;

    extern __shared__ __align__(16) uint32_t s_dyn[];
    __shared__ uint32_t s_cnt[2][16 * 16 + 1];
    __shared__ uint32_t s_scan[33];
    const PairFillSmem pf{s_dyn, kwc, s_cnt, s_scan};
    uint32_t* mapV = pf.mapV();
    uint32_t* mapP = pf.mapP();
    uint32_t* s_spre = pf.spre();
    uint32_t* s_pos = pf.pos();
    uint32_t* s_val = pf.val();
    uint32_t* u_pos = s_dyn + pairfill_words(kwc);  // red entries as collected (any order)
    uint32_t* u_val = u_pos + kFastMaxRed;
    __shared__ uint32_t s_R, s_m;
    __shared__ int s_abort;

    if (threadIdx.x == 0) {
        s_R = 0;
        s_abort = p.validate ? ((__ldcg(p.status) & (ST_DUPLICATE | ST_RANGE)) != 0) : 0;
    }
    uint32_t rr[IPT];
    T src[IPT];
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        const uint32_t i = chunk_base + uint32_t(j) * B + threadIdx.x;
        rr[j] = 0xffffffffu;
        if (i < k) {
            rr[j] = __ldcg(&p.idx[i]);
            src[j] = tail[i];
        }
    }
    for (uint32_t w = threadIdx.x; w < kw; w += B) {
        mapV[w] = 0u;
        mapP[w] = 0u;
    }
    // Everything above overlaps the scan grid of the split schedule; the candidates need it done.
    if (p.pdl) asm volatile("griddepcontrol.wait;" ::: "memory");
    if (threadIdx.x == 0) {
        s_m = __ldcg(p.cand_count);
        if (p.done) {
            // Self-cleaning counter: the last CTA to have read it resets it for the next call.
            __threadfence();
            if (atomicAdd(p.done, 1u) == gridDim.x - 1) {
                *const_cast<uint32_t*>(p.cand_count) = 0u;
                *p.done = 0u;
            }
        }
    }
    __syncthreads();
    if (s_abort) return;  // validation failed: nothing moves
    const uint32_t m = s_m;

    // ---- the red entries: from the candidates, or (candidates overflowed) from the whole list ---
    const bool from_cand = !p.full_scan && m <= p.cand_capacity;
    if (p.full_scan) {
        // Scan-all schedule: the list's 16-byte units, four loads in flight per thread (the list
        // comes from L2 for all but the first CTA to touch a line); the last k % 4 entries below.
        // The range flag is kept in a register: a global atomic inside the loop could alias the
        // list for the compiler and serialise the loads.
        const uint32_t nq = k / 4;
        const uint4* q4 = reinterpret_cast<const uint4*>(p.idx);
        bool oor = false;
#pragma unroll 4
        for (uint32_t u = threadIdx.x; u < nq; u += B) {
            const uint4 x = __ldcg(q4 + u);
            const uint32_t vv[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const uint32_t row = vv[c], slot = 4 * u + uint32_t(c);
                if (row >= n) {
                    oor = true;
                } else if (row >= cut) {
                    const uint32_t v = row - cut;
                    atomicOr(&mapV[v >> 5], 1u << (v & 31u));
                    atomicOr(&mapP[slot >> 5], 1u << (slot & 31u));
                    const uint32_t r = atomicAdd(&s_R, 1u);
                    if (r < kFastMaxRed) {
                        u_pos[r] = slot;
                        u_val[r] = v;
                    }
                }
            }
        }
        if (oor) atomicOr(p.status, ST_RANGE);
    }
    // Candidates, or the whole list one entry per step (candidates overflowed), or the scan-all
    // schedule's last k % 4 entries.
    const uint32_t scan_n = p.full_scan ? (k & 3u) : (from_cand ? m : k);
    const uint32_t ebase = p.full_scan ? (k & ~3u) : 0u;
    for (uint32_t e0 = threadIdx.x; e0 < scan_n; e0 += B) {
        const uint32_t e = ebase + e0;
        uint32_t slot, row;
        if (from_cand) {
            const uint2 c = __ldcg(&p.cand[e]);
            slot = c.x;
            row = c.y;
        } else {
            slot = e;
            row = __ldcg(&p.idx[e]);
        }
        if (row >= n) {
            atomicOr(p.status, ST_RANGE);
            continue;
        }
        if (row < cut || slot >= k) continue;
        const uint32_t v = row - cut;
        atomicOr(&mapV[v >> 5], 1u << (v & 31u));
        atomicOr(&mapP[slot >> 5], 1u << (slot & 31u));
        const uint32_t r = atomicAdd(&s_R, 1u);
        if (r < kFastMaxRed) {
            u_pos[r] = slot;
            u_val[r] = v;
        }
    }
    __syncthreads();
    const uint32_t R = s_R > kFastMaxRed ? 0xffffffffu : s_R;

    // ---- red entries in position order ----------------------------------------------------------
    if (R <= 32u) {
        if (warp == 0) {
            const uint32_t ps = uint32_t(lane) < R ? u_pos[lane] : 0xffffffffu;
            uint32_t rank = 0;
            for (uint32_t d = 0; d < R; ++d) rank += __shfl_sync(0xffffffffu, ps, int(d)) < ps ? 1u : 0u;
            if (uint32_t(lane) < R) {
                s_pos[rank] = ps;
                s_val[rank] = u_val[lane];
            }
        }
    } else if (R <= kFastMaxRed) {
        // rank(slot) = set bits of P before it: per-word prefix of the P map (into s_spre, which
        // only the slow path uses otherwise), warp w owning a contiguous block of words.
        const uint32_t per = (kw + B - 1) / B;
        const uint32_t wb = uint32_t(warp) * 32u * per;
        uint32_t sum = 0;
        for (uint32_t j = 0; j < per; ++j) {
            const uint32_t w = wb + j * 32u + uint32_t(lane);
            if (w < kw) sum += uint32_t(__popc(mapP[w]));
        }
        sum = warp_inclusive_scan(sum);
        if (lane == 31) s_cnt[0][warp] = sum;
        __syncthreads();
        if (warp == 0) {
            const uint32_t x = lane < nw ? s_cnt[0][lane] : 0u;
            const uint32_t inc = warp_inclusive_scan(x);
            if (lane < nw) s_cnt[0][32 + lane] = inc - x;
        }
        __syncthreads();
        uint32_t run = s_cnt[0][32 + warp];
        for (uint32_t j = 0; j < per; ++j) {
            const uint32_t w = wb + j * 32u + uint32_t(lane);
            const uint32_t x = w < kw ? uint32_t(__popc(mapP[w])) : 0u;
            const uint32_t inc = warp_inclusive_scan(x);
            if (w < kw) s_spre[w] = run + inc - x;
            run += __shfl_sync(0xffffffffu, inc, 31);
        }
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < R; e += B) {
            const uint32_t ps = u_pos[e];
            const uint32_t rank = s_spre[ps >> 5] + uint32_t(__popc(mapP[ps >> 5] & ((1u << (ps & 31u)) - 1u)));
            s_pos[rank] = ps;
            s_val[rank] = u_val[e];
        }
    }
    __syncthreads();

    uint32_t stot, dbase;
    derive_pairing<IPT>(pf, R, k, chunk_base, true, p.status, stot, dbase);
    fill_holes<W, IPT>(pf, R, k, cut, chunk_base, stot, dbase, rr, src, head, tail);
}

using ProducedFn = void (*)(const ProducedParams);

template <int W>
static ProducedFn produced_fn(int items) {
    switch (items) {
        case 1: return redzone_produced_kernel<W, 1>;
        case 2: return redzone_produced_kernel<W, 2>;
        case 4: return redzone_produced_kernel<W, 4>;
        case 8: return redzone_produced_kernel<W, 8>;
        default: return nullptr;
    }
}
static ProducedFn produced_fn(uint32_t w, int items) {
    switch (w) {
        case 4: return produced_fn<4>(items);
        case 8: return produced_fn<8>(items);
        case 16: return produced_fn<16>(items);
        case 32: return produced_fn<32>(items);
        default: return nullptr;
    }
}

// Split schedule, first grid: every red entry (i, idx[i] >= cut) of a device index list, appended
// (any order) to a candidate buffer with one atomic per warp; out-of-range entries are reported.
// The pairing grid is launched as its programmatic dependent, so its tile loads overlap this.
__global__ void __launch_bounds__(256) split_scan_kernel(const uint32_t* __restrict__ idx, uint32_t k, uint32_t n,
                                                         uint32_t vec, uint2* __restrict__ cand,
                                                         uint32_t* __restrict__ cand_count, uint32_t* status) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const uint32_t cut = n - k;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    const uint32_t nq = vec ? k / 4 : 0;
    const uint32_t lane = threadIdx.x & 31;
    // Every lane of a warp runs the same number of iterations (the append is warp-wide).
    const uint32_t total = nq + (k - 4 * nq);  // quads, then the remaining single entries
    const uint32_t total_round = (total + 31u) & ~31u;
    bool oor = false;
    for (uint32_t u = gtid; u < total_round; u += stride) {
        uint32_t e0, v[4], cnt = 0;
        if (u < nq) {
            const uint4 q = __ldg(reinterpret_cast<const uint4*>(idx) + u);
            e0 = 4 * u;
            v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
            cnt = 4;
        } else {
            e0 = 4 * nq + (u - nq);
            v[0] = u < total ? __ldg(&idx[e0]) : 0u;
            v[1] = v[2] = v[3] = 0u;
            cnt = u < total ? 1u : 0u;
        }
        uint32_t redbits = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const bool in = uint32_t(c) < cnt;
            oor |= in && v[c] >= n;
            redbits |= uint32_t(in && v[c] >= cut && v[c] < n) << c;
        }
        const uint32_t mine = uint32_t(__popc(redbits));
        const uint32_t inc = warp_inclusive_scan(mine);
        const uint32_t wtot = __shfl_sync(0xffffffffu, inc, 31);
        if (wtot == 0u) continue;
        uint32_t base = 0;
        if (lane == 31) base = atomicAdd(cand_count, wtot);
        base = __shfl_sync(0xffffffffu, base, 31) + inc - mine;
#pragma unroll
        for (int c = 0; c < 4; ++c)
            if ((redbits >> c) & 1u) cand[base++] = make_uint2(e0 + uint32_t(c), v[c]);
    }
    if (__any_sync(0xffffffffu, oor) && lane == 0) atomicOr(status, ST_RANGE);
}

// Let the pairing kernel for (w, items) use the device's large shared memory; once per device.
static int allow_produced_smem(rz_ctx* ctx, ProducedFn f, uint32_t w, int items) {
    static std::atomic<uint64_t> done[4][4];
    const int wi = w == 4 ? 0 : w == 8 ? 1 : w == 16 ? 2 : 3;
    const int ii = items == 1 ? 0 : items == 2 ? 1 : items == 4 ? 2 : 3;
    const uint64_t bit = 1ull << (ctx->device & 63);
    if (!(done[wi][ii].load() & bit)) {
        RZ_CUDA_TRY(ctx, cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              int(ctx->smem_optin) - 4096));
        done[wi][ii].fetch_or(bit);
    }
    return RZ_OK;
}

// The library's own producer: every row i < n with keys[i] < threshold. Each thread reads 16
// keys per step (four 16-byte loads in flight: a 4-byte load per step would leave the kernel
// waiting on memory latency) and emits them warp-wide; keys not 16-byte aligned, and the last
// n % 16, take the one-key loop.
__global__ void produce_where_less_kernel(const rz_producer_view v, const uint32_t* __restrict__ keys,
                                          uint32_t threshold, uint32_t vec) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t gtid = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t nvec = vec ? v.n / 16u : 0u;
    // Every lane of a warp runs the same number of iterations (rz_emit is called warp-wide).
    const uint64_t nvec_round = (nvec + 31u) & ~uint64_t(31);
    for (uint64_t c = gtid; c < nvec_round; c += stride) {
        const bool ok = c < nvec;
        uint4 q[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            q[u] = ok ? __ldg(reinterpret_cast<const uint4*>(keys) + c * 4 + u) : make_uint4(~0u, ~0u, ~0u, ~0u);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const uint32_t row = uint32_t(c * 16 + 4 * u);
            rz_emit(v, row, ok && q[u].x < threshold);
            rz_emit(v, row + 1, ok && q[u].y < threshold);
            rz_emit(v, row + 2, ok && q[u].z < threshold);
            rz_emit(v, row + 3, ok && q[u].w < threshold);
        }
    }
    const uint64_t rest = nvec * 16;
    const uint64_t n_round = rest + ((uint64_t(v.n) - rest + 31u) & ~uint64_t(31));
    for (uint64_t i = rest + gtid; i < n_round; i += stride) {
        const bool take = i < v.n && __ldg(&keys[i]) < threshold;
        rz_emit(v, uint32_t(i), take);
    }
}

// Split schedule of rz_remove (RZ_SCHED_SPLIT): the scan grid above, then the pairing grid of the
// produced-list path as its programmatic dependent. One 256 * items tile per pairing CTA;
// RZ_ERR_UNSUPPORTED when the shared-memory maps would not fit or k > kFastMaxK.
int launch_split(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx, uint32_t k,
                 const rz_launch_cfg& cfg, bool validate, cudaStream_t s, LaunchInfo* info) {
    if (k == 0 || k > kFastMaxK || !ctx->ws.redlist || ctx->ws.red_cap < size_t(k) + 1) return RZ_ERR_UNSUPPORTED;
    const size_t smem = produced_smem_bytes(k);
    if (smem + 4096 > ctx->smem_optin) return RZ_ERR_UNSUPPORTED;
    int items = cfg.items;
    ProducedFn f = produced_fn(w, items);
    if (!f) return RZ_ERR_INVALID_ARG;
    const int ast = allow_produced_smem(ctx, f, w, items);
    if (ast != RZ_OK) return ast;
    const uint32_t vec = (reinterpret_cast<uintptr_t>(idx) & 15u) == 0 ? 1u : 0u;
    const uint32_t units = vec ? k / 4 + (k & 3u) : k;
    const uint32_t sgrid = std::max<uint32_t>(1u, std::min<uint32_t>((units + 255) / 256, uint32_t(ctx->sms) * 4));
    uint2* cand = ctx->ws.redlist;
    uint32_t* counter = ctx->ws.split_count;
    split_scan_kernel<<<sgrid, 256, 0, s>>>(idx, k, n, vec, cand, counter, ctx->ws.status);
    RZ_CUDA_TRY(ctx, cudaGetLastError());

    const uint32_t tile = uint32_t(kProducedBlock) * uint32_t(items);
    const uint32_t grid = (k + tile - 1) / tile;
    ProducedParams pp;
    pp.data = static_cast<uint8_t*>(data);
    pp.idx = idx;
    pp.counts = nullptr;
    pp.cand_count = counter;
    pp.done = counter + 1;
    pp.cand = cand;
    pp.n = n;
    pp.k_fixed = k;
    pp.capacity = k;
    pp.cand_capacity = k + 1;
    pp.status = ctx->ws.status;
    pp.dev_len = ctx->ws.dev_len;
    pp.validate = validate ? 1u : 0u;
    pp.pdl = 1;
    pp.full_scan = 0;
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(grid);
    lc.blockDim = dim3(kProducedBlock);
    lc.dynamicSmemBytes = smem;
    lc.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    RZ_CUDA_TRY(ctx, cudaLaunchKernelEx(&lc, f, pp));
    if (info) {
        info->grid = int(grid);
        info->block = kProducedBlock;
        info->items = items;
        info->launches += 2;
    }
    return RZ_OK;
}

// Scan-all schedule of rz_remove (RZ_SCHED_SCANALL): the pairing grid alone, each CTA reading the
// whole list for the red entries. No second grid, no wait of any kind; the cost of the scan grows
// with k per CTA, so it is the default only for short lists. Needs a 16-byte-aligned list.
int launch_scanall(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx, uint32_t k,
                   const rz_launch_cfg& cfg, bool validate, cudaStream_t s, LaunchInfo* info) {
    if (k == 0 || k > kFastMaxK || (reinterpret_cast<uintptr_t>(idx) & 15u)) return RZ_ERR_UNSUPPORTED;
    const size_t smem = produced_smem_bytes(k);
    if (smem + 4096 > ctx->smem_optin) return RZ_ERR_UNSUPPORTED;
    const int items = cfg.items;
    ProducedFn f = produced_fn(w, items);
    if (!f) return RZ_ERR_INVALID_ARG;
    const int ast = allow_produced_smem(ctx, f, w, items);
    if (ast != RZ_OK) return ast;
    const uint32_t tile = uint32_t(kProducedBlock) * uint32_t(items);
    const uint32_t grid = (k + tile - 1) / tile;
    ProducedParams pp;
    pp.data = static_cast<uint8_t*>(data);
    pp.idx = idx;
    pp.counts = nullptr;
    pp.cand_count = ctx->ws.split_count;  // read, not used
    pp.done = nullptr;
    pp.cand = nullptr;
    pp.n = n;
    pp.k_fixed = k;
    pp.capacity = k;
    pp.cand_capacity = 0;
    pp.status = ctx->ws.status;
    pp.dev_len = ctx->ws.dev_len;
    pp.validate = validate ? 1u : 0u;
    pp.pdl = 0;
    pp.full_scan = 1;
    f<<<grid, kProducedBlock, smem, s>>>(pp);
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    if (info) {
        info->grid = int(grid);
        info->block = kProducedBlock;
        info->items = items;
        info->launches += 1;
    }
    return RZ_OK;
}

}  // namespace rz

using namespace rz;

extern "C" {

int rz_producer_create(rz_ctx* ctx, int64_t capacity, int64_t cand_capacity, rz_producer** out) {
    if (!ctx || !out || capacity < 1 || cand_capacity < 0) return RZ_ERR_INVALID_ARG;
    *out = nullptr;
    if (capacity > int64_t(kProducedMaxK) || cand_capacity > int64_t(1) << 24) return RZ_ERR_UNSUPPORTED;
    if (produced_smem_bytes(uint32_t(capacity)) + 4096 > ctx->smem_optin) return RZ_ERR_UNSUPPORTED;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    rz_producer* p = new (std::nothrow) rz_producer();
    if (!p) return RZ_ERR_NO_MEMORY;
    p->ctx = ctx;
    p->capacity = uint32_t(capacity);
    p->cand_capacity = uint32_t(cand_capacity);
    // One allocation: counts (256 bytes) | list | candidates.
    const size_t list_bytes = (size_t(capacity) * 4 + 255) / 256 * 256;
    const size_t bytes = 256 + list_bytes + size_t(std::max<int64_t>(cand_capacity, 1)) * 8;
    void* mem = nullptr;
    cudaError_t e = cudaMalloc(&mem, bytes);
    if (e == cudaSuccess) e = cudaMemset(mem, 0, 256);
    if (e != cudaSuccess) {
        if (mem) cudaFree(mem);
        delete p;
        return e == cudaErrorMemoryAllocation ? RZ_ERR_NO_MEMORY : cuda_fail(ctx, e, "producer buffers");
    }
    uint8_t* b = static_cast<uint8_t*>(mem);
    p->counts = reinterpret_cast<uint32_t*>(b);
    p->idx = reinterpret_cast<uint32_t*>(b + 256);
    p->cand = reinterpret_cast<uint32_t*>(b + 256 + list_bytes);
    *out = p;
    return RZ_OK;
}

void rz_producer_destroy(rz_producer* p) {
    if (!p) return;
    cudaSetDevice(p->ctx->device);
    cudaDeviceSynchronize();
    cudaFree(p->counts);
    delete p;
}

int rz_producer_reset(rz_producer* p, int64_t n, rz_stream_t stream) {
    if (!p || n < 1) return RZ_ERR_INVALID_ARG;
    if (n >= (int64_t(1) << 32)) return RZ_ERR_UNSUPPORTED;
    std::lock_guard<std::recursive_mutex> g(p->ctx->mu);
    cudaSetDevice(p->ctx->device);
    RZ_CUDA_TRY(p->ctx, cudaMemsetAsync(p->counts, 0, 2 * sizeof(uint32_t), reinterpret_cast<cudaStream_t>(stream)));
    p->n = uint32_t(n);
    p->have_n = true;
    return RZ_OK;
}

int rz_producer_get_view(const rz_producer* p, rz_producer_view* out) {
    if (!p || !out || !p->have_n) return RZ_ERR_INVALID_ARG;
    out->idx = p->idx;
    out->counts = p->counts;
    out->cand = p->cand;
    out->capacity = p->capacity;
    out->cand_capacity = p->cand_capacity;
    out->n = p->n;
    out->floor = p->n > p->capacity ? p->n - p->capacity : 0u;
    return RZ_OK;
}

int rz_produce_where_less(rz_producer* p, const uint32_t* d_keys, uint32_t threshold, rz_stream_t stream) {
    if (!p || !d_keys || !p->have_n) return RZ_ERR_INVALID_ARG;
    rz_ctx* ctx = p->ctx;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    rz_producer_view v;
    rz_producer_get_view(p, &v);
    const uint32_t vec = (reinterpret_cast<uintptr_t>(d_keys) & 15u) == 0 ? 1u : 0u;
    const uint64_t units = vec ? (uint64_t(p->n) + 15) / 16 : uint64_t(p->n);
    const int grid = int(std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(ctx->sms) * 8, (units + 255) / 256)));
    produce_where_less_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(v, d_keys, threshold, vec);
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    return RZ_OK;
}

int rz_producer_download(const rz_producer* p, uint32_t* h_idx, int64_t max, int64_t* k, int64_t* candidates,
                         rz_stream_t stream) {
    if (!p || max < 0 || (max > 0 && !h_idx)) return RZ_ERR_INVALID_ARG;
    rz_ctx* ctx = p->ctx;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t c[2] = {0, 0};
    RZ_CUDA_TRY(ctx, cudaMemcpyAsync(c, p->counts, sizeof(c), cudaMemcpyDeviceToHost, s));
    RZ_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    const int64_t m = std::min<int64_t>(std::min<int64_t>(c[0], p->capacity), max);
    if (m > 0) {
        RZ_CUDA_TRY(ctx, cudaMemcpyAsync(h_idx, p->idx, size_t(m) * 4, cudaMemcpyDeviceToHost, s));
        RZ_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    }
    if (k) *k = c[0];
    if (candidates) *candidates = c[1];
    return RZ_OK;
}

int rz_remove_produced(rz_ctx* ctx, rz_producer* p, void* d_data, uint32_t elem_bytes, int64_t* new_len,
                       uint32_t flags, rz_stream_t stream) {
    if (!ctx || !p || !d_data || !p->have_n) return RZ_ERR_INVALID_ARG;
    if (elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16 && elem_bytes != 32) return RZ_ERR_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(d_data) % (elem_bytes >= 16 ? 16 : elem_bytes)) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int st = reset_if_dirty(ctx, s);
    if (st != RZ_OK) return st;
    ctx->last_kernels = 0;
    const bool validate = (flags & RZ_VALIDATE) != 0;
    if (validate) {
        // The validation passes need k on the host: the one synchronisation of this path.
        uint32_t hk = 0;
        RZ_CUDA_TRY(ctx, cudaMemcpyAsync(&hk, p->counts, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        RZ_CUDA_TRY(ctx, cudaStreamSynchronize(s));
        if (hk > p->capacity) {
            if (new_len) *new_len = int64_t(p->n) - int64_t(hk);
            return RZ_ERR_NO_MEMORY;
        }
        if (hk > 0) {
            st = launch_validate(ctx, p->n, p->idx, hk, s);
            if (st != RZ_OK) return st;
            ctx->last_kernels += 2;
        }
    }
    // About 64 tiles for a full list: 256 threads, 1..8 items each.
    int items = 1;
    while (items < 8 && uint64_t(kProducedBlock) * items * 64 < p->capacity) items *= 2;
    ProducedFn f = produced_fn(elem_bytes, items);
    if (!f) return RZ_ERR_INVALID_ARG;
    const size_t smem = produced_smem_bytes(p->capacity);
    st = allow_produced_smem(ctx, f, elem_bytes, items);
    if (st != RZ_OK) return st;
    const uint32_t tile = uint32_t(kProducedBlock) * uint32_t(items);
    const uint32_t grid = std::max<uint32_t>(1u, (p->capacity + tile - 1) / tile);
    ProducedParams pp;
    pp.data = static_cast<uint8_t*>(d_data);
    pp.idx = p->idx;
    pp.counts = p->counts;
    pp.cand_count = p->counts + 1;
    pp.done = nullptr;
    pp.cand = reinterpret_cast<const uint2*>(p->cand);
    pp.n = p->n;
    pp.k_fixed = 0;
    pp.capacity = p->capacity;
    pp.cand_capacity = p->cand_capacity;
    pp.status = ctx->ws.status;
    pp.dev_len = ctx->ws.dev_len;
    pp.validate = validate ? 1u : 0u;
    pp.pdl = 0;
    pp.full_scan = 0;
    f<<<grid, kProducedBlock, smem, s>>>(pp);
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    ctx->last_kernels += 1;
    ctx->last_grid = int(grid);
    ctx->last_block = kProducedBlock;
    if (flags & RZ_SYNC) return read_status(ctx, s, new_len);
    if (new_len) *new_len = -1;  // on the device until the stream reaches this point
    return RZ_OK;
}

}  // extern "C"
