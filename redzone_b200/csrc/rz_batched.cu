// rz_batched.cu -- many independent lists in one persistent launch (replayed from a CUDA graph).
//
// Each list gets exactly the single-list result (same rule, same bits as rz_remove). The launch
// consumes a host-built work queue with a ticket counter. A list of at most one tile is one
// SINGLE item; a longer list is cut into tiles, and tiles into groups of `span` tiles (so each
// work item carries enough work to amortise its dispatch). Work items, in queue order:
//   MARK(l, g)     the tiles of group g mark their red-zone indices in the list's bitmap
//   SINGLE(l)      the whole list in one CTA, bitmap and both orphan lists in shared memory
//   CLASSIFY(l, g) waits until every MARK group of list l is done, then fills holes and lists
//                  orphans tile by tile (the grid kernel's phase B)
//   PAIR(l, g)     waits until every CLASSIFY group of l is done, then pairs the destination
//                  orphans of its tiles by global rank (the grid kernel's phase C)
// A waiting item only ever waits for items with smaller tickets, which running CTAs took and finish
// without waiting on anything later, so the queue cannot deadlock; every wait is bounded anyway.
// The queue runs phase by phase over all lists (SINGLE items between the MARK and CLASSIFY items,
// so that the marks have landed by the time the first CLASSIFY item is taken), or, with
// rz_batch_cfg.wave > 0, as a wavefront over the lists (order_queue). Reference: the per-block
// body of Algorithm 1 (RemoveFromList2, redzone.hxx:237-444) and the phases of Algorithm 2
// (redzone.hxx:626-941).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "rz_batch_order.h"
#include "rz_common.cuh"
#include "rz_internal.h"

namespace rz {

enum : uint32_t { K_MARK = 0, K_SINGLE = 1, K_CLASSIFY = 2, K_PAIR = 3 };
constexpr uint32_t kMaxTilesPerList = kBatchMaxTilesPerList;
constexpr uint32_t kNoItem = 0xffffffffu;
constexpr int kMarkLoads = 8;   // index loads in flight per thread in a MARK item

struct ListRec {            // one per list, device-resident
    uint8_t* data;
    const uint32_t* idx;
    uint32_t n, k;
    uint32_t nch;           // tiles of the i range; 1 = SINGLE list
    uint32_t span;          // tiles per MARK / CLASSIFY / PAIR item
    uint32_t ngroups;       // ceil(nch / span)
    uint32_t bitmap_off;    // word offset of the list's bitmap (multi-tile lists)
    uint64_t list_off;      // entry offset of the list's orphan lists (multi-tile lists)
    uint32_t cnt_off;       // word offset of the list's per-tile counts (2 * nch words)
    uint32_t pad;
};

struct BatchParams {
    const ListRec* lists;
    const uint2* queue;     // {list, kind << 28 | group}
    uint32_t nitems;
    uint32_t* counters;     // [0] ticket, then per list: marks_done, classify_done (in groups)
    uint32_t* bitmap;
    uint32_t* dlist;
    uint32_t* slist;
    uint32_t* chunk_cnt;
    uint32_t* status;
    uint32_t spin_limit;
};

__device__ __forceinline__ bool wait_count(const uint32_t* ctr, uint32_t target, uint32_t spin_limit) {
    uint32_t it = 0;
    while (ld_relaxed(ctr) < target) {
        if (++it > spin_limit) return false;
    }
    fence_acq_rel_gpu();
    return true;
}

// Ranks of this tile's orphans in i order (round-major items: i = base + j*B + t). Returns the
// packed total (D << 16 | S) and leaves per-(round, warp) exclusive prefixes in s_cnt.
template <int IPT>
__device__ __forceinline__ uint32_t rank_orphans(const bool* dv, const bool* sv, uint32_t* dmask, uint32_t* smask,
                                                 uint32_t* s_cnt) {
    const int nw = blockDim.x >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        dmask[j] = __ballot_sync(0xffffffffu, dv[j] && !sv[j]);
        smask[j] = __ballot_sync(0xffffffffu, sv[j] && !dv[j]);
        if (lane == 0) s_cnt[j * nw + warp] = (uint32_t(__popc(dmask[j])) << 16) | uint32_t(__popc(smask[j]));
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
    return s_cnt[E];
}

template <int IPT>
__device__ __forceinline__ void write_orphans(const bool* dv, const bool* sv, const uint32_t* dmask,
                                              const uint32_t* smask, const uint32_t* rr, const uint32_t* s_cnt,
                                              uint32_t base, uint32_t cut, uint32_t* dl, uint32_t* sl) {
    const int nw = blockDim.x >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5, B = blockDim.x;
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        const uint32_t ex = s_cnt[j * nw + warp];
        const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
        if (dv[j] && !sv[j]) dl[(ex >> 16) + __popc(dmask[j] & lt)] = rr[j];
        if (sv[j] && !dv[j]) sl[(ex & 0xffffu) + __popc(smask[j] & lt)] = cut + i;
    }
    (void)lane;
}

// Two 512-thread CTAs per SM (at most 64 registers) where one thread's items take at most 64
// bytes: measured on the 4096-list workload, the doubled resident warps keep more random hole
// writes in flight (best configuration 12.73 -> 10.17 ms). Wider variants would spill at 64
// registers (144-644 bytes) and keep the compiler's choice (up to 128).
template <int W, int IPT>
constexpr int batched_min_blocks() { return W * IPT <= 64 ? 2 : 1; }

template <int W, int IPT>
__global__ void __launch_bounds__(512, batched_min_blocks<W, IPT>()) redzone_batched_kernel(const BatchParams p) {
    using T = typename Payload<W>::T;
    const int B = blockDim.x, lane = threadIdx.x & 31;
    const uint32_t TILE = uint32_t(B) * IPT;
    extern __shared__ __align__(16) uint32_t smem[];
    // SINGLE items: bitmap (TILE bits) | D positions (TILE) | S positions (TILE).
    uint32_t* s_bits = smem;
    uint32_t* s_dl = smem + TILE / 32;
    uint32_t* s_sl = s_dl + TILE;
    __shared__ uint32_t s_cnt[2][8 * 32 + 1];  // rank counts; CLASSIFY alternates them between tiles
    __shared__ uint32_t s_item[2];
    __shared__ int s_ok;
    __shared__ uint32_t s_pfx[2 * kMaxTilesPerList + 2];  // PAIR: per-tile prefixes of D and S
    __shared__ uint32_t s_scan[33];

    const uint64_t pol_stream = l2_policy_evict_first(), pol_hole = l2_policy_evict_last();
    // The next ticket is taken one item ahead, so its atomic overlaps the current item's work.
    uint32_t next_t = 0;
    if (threadIdx.x == 0) next_t = atomicAdd(&p.counters[0], 1u);
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t t = next_t;
            if (t < p.nitems) {
                const uint2 q = p.queue[t];
                s_item[0] = q.x;
                s_item[1] = q.y;
                next_t = atomicAdd(&p.counters[0], 1u);
            } else {
                s_item[0] = kNoItem;
            }
        }
        __syncthreads();
        const uint32_t l = s_item[0];
        if (l == kNoItem) return;
        const uint32_t kind = s_item[1] >> 28, grp = s_item[1] & 0x0fffffffu;
        const ListRec L = p.lists[l];
        const uint32_t n = L.n, k = L.k, cut = n - k;
        T* __restrict__ head = reinterpret_cast<T*>(L.data);
        const T* __restrict__ tail = reinterpret_cast<const T*>(L.data) + cut;
        uint32_t* marks_done = &p.counters[1 + 2 * l];
        uint32_t* classify_done = &p.counters[2 + 2 * l];
        const uint32_t t_begin = grp * L.span, t_end = min(t_begin + L.span, L.nch);

        if (kind == K_MARK) {
            // The group's index entries in any order, kMarkLoads loads in flight per thread:
            // marking waits on index bytes in flight, not on its (fire-and-forget) atomics.
            const uint32_t lo = t_begin * TILE, hi = min(t_end * TILE, k);
            for (uint32_t b = lo + threadIdx.x; b < hi; b += uint32_t(kMarkLoads) * B) {
                uint32_t r[kMarkLoads];
#pragma unroll
                for (int j = 0; j < kMarkLoads; ++j) {
                    const uint32_t i = b + uint32_t(j) * B;
                    r[j] = i < hi ? __ldg(&L.idx[i]) : 0u;
                }
#pragma unroll
                for (int j = 0; j < kMarkLoads; ++j) {
                    const uint32_t i = b + uint32_t(j) * B;
                    if (i < hi && r[j] >= cut) {
                        if (r[j] >= n) atomicOr(p.status, ST_RANGE);
                        else atomicOr(&p.bitmap[L.bitmap_off + ((r[j] - cut) >> 5)], 1u << ((r[j] - cut) & 31u));
                    }
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                atomicAdd(marks_done, 1u);
            }
            continue;
        }

        uint32_t rr[IPT];
        T src[IPT];
        bool dv[IPT], sv[IPT];
        uint32_t dmask[IPT], smask[IPT];

        if (kind == K_SINGLE) {
            // ---- whole list in this CTA (k <= TILE) -------------------------------------------
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i = uint32_t(j) * B + threadIdx.x;
                rr[j] = 0xffffffffu;
                if (i < k) {
                    rr[j] = ld_hint(&L.idx[i], pol_stream);
                    src[j] = ld_hint(tail + i, pol_stream);  // loaded with the index, needed or not: one round trip
                }
            }
            for (uint32_t w = threadIdx.x; w < TILE / 32; w += B) s_bits[w] = 0u;
            __syncthreads();
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i = uint32_t(j) * B + threadIdx.x;
                if (i < k && rr[j] >= cut) {
                    if (rr[j] >= n) atomicOr(p.status, ST_RANGE);
                    else atomicOr(&s_bits[(rr[j] - cut) >> 5], 1u << ((rr[j] - cut) & 31u));
                }
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i = uint32_t(j) * B + threadIdx.x;
                if (i < k) {
                    sv[j] = ((s_bits[i >> 5] >> (i & 31u)) & 1u) == 0u;
                    dv[j] = rr[j] < cut;
                } else {
                    sv[j] = dv[j] = false;
                }
            }
#pragma unroll
            for (int j = 0; j < IPT; ++j)
                if (dv[j] && sv[j]) st_hint(head + rr[j], src[j], pol_hole);
            const uint32_t tot = rank_orphans<IPT>(dv, sv, dmask, smask, s_cnt[0]);
            if (tot != 0u) {
                write_orphans<IPT>(dv, sv, dmask, smask, rr, s_cnt[0], 0, cut, s_dl, s_sl);
                __syncthreads();
                const uint32_t dcnt = tot >> 16, scnt = tot & 0xffffu;
                const uint32_t m = min(dcnt, scnt);
                for (uint32_t r = threadIdx.x; r < m; r += B)
                    st_hint(head + s_dl[r], reinterpret_cast<const T*>(L.data)[s_sl[r]], pol_hole);
                if (dcnt > scnt && threadIdx.x == 0) atomicOr(p.status, ST_INCONSISTENT);
            }
            continue;
        }

        if (kind == K_CLASSIFY) {
            // ---- holes and orphan lists of the group's tiles -----------------------------------
            if (threadIdx.x == 0) s_ok = wait_count(marks_done, L.ngroups, p.spin_limit);
            __syncthreads();
            if (!s_ok) {
                if (threadIdx.x == 0) atomicOr(p.status, ST_TIMEOUT);
                continue;
            }
            for (uint32_t c = t_begin; c < t_end; ++c) {
                const uint32_t base = c * TILE;
                // The next tile's indices and tail window go to L2 while this one is processed.
                if (c + 1 < t_end) {
                    const uint32_t nb = base + TILE, cnt = min(TILE, k - nb);
                    prefetch_l2(L.idx + nb, size_t(cnt) * 4);
                    prefetch_l2(tail + nb, size_t(cnt) * W);
                }
                // Index, bitmap word and tail item are loaded together (the tail item whether it
                // is needed or not): one round trip per tile instead of two dependent ones.
                uint32_t word[IPT];
#pragma unroll
                for (int j = 0; j < IPT; ++j) {
                    const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
                    if (i < k) {
                        rr[j] = ld_hint(&L.idx[i], pol_stream);
                        word[j] = __ldcg(&p.bitmap[L.bitmap_off + (i >> 5)]);
                        src[j] = ld_hint(tail + i, pol_stream);
                    } else {
                        rr[j] = 0xffffffffu;
                        word[j] = 0u;
                    }
                }
#pragma unroll
                for (int j = 0; j < IPT; ++j) {
                    const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
                    if (i < k) {
                        sv[j] = ((word[j] >> (i & 31u)) & 1u) == 0u;
                        dv[j] = rr[j] < cut;
                    } else {
                        sv[j] = dv[j] = false;
                    }
                }
#pragma unroll
                for (int j = 0; j < IPT; ++j)
                    if (dv[j] && sv[j]) st_hint(head + rr[j], src[j], pol_hole);
                __syncwarp();  // every lane has read its bitmap word before lane 0 clears it
                if (lane == 0) {
#pragma unroll
                    for (int j = 0; j < IPT; ++j) {
                        const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
                        if (i < k) p.bitmap[L.bitmap_off + (i >> 5)] = 0u;  // leave the bitmap zero
                    }
                }
                // Alternate count buffers: tile c + 1 writes the other one, and tile c + 2 writes
                // this one only after every thread has passed tile c + 1's barriers, i.e. after
                // every read of this tile's counts.
                uint32_t* cnt = s_cnt[c & 1u];
                const uint32_t tot = rank_orphans<IPT>(dv, sv, dmask, smask, cnt);
                if (tot != 0u)
                    write_orphans<IPT>(dv, sv, dmask, smask, rr, cnt, base, cut,
                                       p.dlist + L.list_off + base, p.slist + L.list_off + base);
                if (threadIdx.x == 0) {
                    p.chunk_cnt[L.cnt_off + c] = tot >> 16;
                    p.chunk_cnt[L.cnt_off + L.nch + c] = tot & 0xffffu;
                }
            }
            __syncthreads();  // every thread's hole, list and count stores precede the release
            if (threadIdx.x == 0) {
                __threadfence();
                atomicAdd(classify_done, 1u);
            }
            continue;
        }

        // ---- K_PAIR: destination orphans of the group's tiles -----------------------------------
        // Counts persist between launches, so they are read only after every CLASSIFY group of
        // this list is done in this launch.
        if (threadIdx.x == 0) s_ok = wait_count(classify_done, L.ngroups, p.spin_limit);
        __syncthreads();
        if (!s_ok) {
            if (threadIdx.x == 0) atomicOr(p.status, ST_TIMEOUT);
            continue;
        }
        uint32_t any = 0;
        for (uint32_t c = t_begin + threadIdx.x; c < t_end; c += B) any |= __ldcg(&p.chunk_cnt[L.cnt_off + c]);
        if (!__syncthreads_or(any != 0u)) continue;  // no destination orphans in this group
        const uint32_t nch = L.nch;
        for (uint32_t q = threadIdx.x; q < nch; q += B) {
            s_pfx[q] = __ldcg(&p.chunk_cnt[L.cnt_off + q]);
            s_pfx[kMaxTilesPerList + 1 + q] = __ldcg(&p.chunk_cnt[L.cnt_off + nch + q]);
        }
        __syncthreads();
        uint32_t* pfx_d = s_pfx;
        uint32_t* pfx_s = s_pfx + kMaxTilesPerList + 1;
        block_scan_array(pfx_d, int(nch), s_scan);
        block_scan_array(pfx_s, int(nch), s_scan);
        const uint32_t tot_s = pfx_s[nch];
        for (uint32_t c = t_begin; c < t_end; ++c) {
            const uint32_t dc = pfx_d[c + 1] - pfx_d[c];
            for (uint32_t r = threadIdx.x; r < dc; r += B) {
                const uint32_t jr = pfx_d[c] + r;
                if (jr >= tot_s) {
                    atomicOr(p.status, ST_INCONSISTENT);
                    continue;
                }
                const int c2 = owner_of_rank(pfx_s, int(nch), jr);
                const uint32_t pos = __ldcg(&p.slist[L.list_off + uint64_t(c2) * TILE + (jr - pfx_s[c2])]);
                const uint32_t dest = __ldcg(&p.dlist[L.list_off + uint64_t(c) * TILE + r]);
                st_hint(head + dest, reinterpret_cast<const T*>(L.data)[pos], pol_hole);
            }
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Host side: plans (queue + scratch owned by the plan) and graph-captured launches.
// ------------------------------------------------------------------------------------------------
using BatchFn = void (*)(const BatchParams);

template <int W>
static BatchFn batch_fn(int items) {
    switch (items) {
        case 1: return redzone_batched_kernel<W, 1>;
        case 2: return redzone_batched_kernel<W, 2>;
        case 4: return redzone_batched_kernel<W, 4>;
        case 8: return redzone_batched_kernel<W, 8>;
        default: return nullptr;
    }
}
static BatchFn batch_fn(int w, int items) {
    switch (w) {
        case 4: return batch_fn<4>(items);
        case 8: return batch_fn<8>(items);
        case 16: return batch_fn<16>(items);
        case 32: return batch_fn<32>(items);
        default: return nullptr;
    }
}

// Tiles per work item for a list of `nch` tiles: 4 by default. Measured on B200 against the
// earlier rule (up to 8 tiles, at least ~32 items per list), both with the default wavefront lag:
// 5-26 % faster on seven list mixes (4, 8, 16 and 32-byte items, lists of 2^8 to 2^22 items),
// equal on mixes of lists short enough to be one item either way.
static uint32_t span_for(uint32_t nch, int32_t cfg_span) {
    return std::min<uint32_t>(cfg_span > 0 ? uint32_t(cfg_span) : 4u, nch);
}


}  // namespace rz

struct rz_batch_plan {
    rz_ctx* ctx = nullptr;
    uint32_t w = 0;
    rz_batch_cfg cfg{};
    int grid = 0;
    size_t smem = 0;
    uint32_t nlists = 0, nitems = 0;
    uint64_t total_k = 0;
    void* dev = nullptr;            // one allocation: lists | queue | counters | tile counts | bitmap | orphan lists
    rz::BatchParams params{};
    size_t counters_bytes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace rz {

// Items are read and written as whole w-byte units (16-byte vectors for w >= 16) and index
// entries as 4-byte words: both must be aligned to them.
static bool list_aligned(const rz_list_desc& d, uint32_t w) {
    const uintptr_t a = w >= 16 ? 16 : w;
    return (reinterpret_cast<uintptr_t>(d.data) % a) == 0 && (reinterpret_cast<uintptr_t>(d.idx) % 4) == 0;
}

static int plan_build(rz_ctx* ctx, const rz_list_desc* lists, int32_t nlists, uint32_t w, const rz_batch_cfg& cfg_in,
                      rz_batch_plan* plan) {
    rz_batch_cfg cfg = cfg_in;
    if (cfg.block < 32 || cfg.block > 1024 || (cfg.block & 31)) return RZ_ERR_INVALID_ARG;
    if (cfg.ctas_per_sm < 1) cfg.ctas_per_sm = 1;
    BatchFn f = batch_fn(int(w), cfg.items);
    if (!f) return RZ_ERR_INVALID_ARG;
    cudaFuncAttributes fa{};
    RZ_CUDA_TRY(ctx, cudaFuncGetAttributes(&fa, (const void*)f));
    cfg.block = std::min(cfg.block, fa.maxThreadsPerBlock & ~31);
    const uint32_t TILE = uint32_t(cfg.block) * uint32_t(cfg.items);
    if (TILE > 8192) return RZ_ERR_INVALID_ARG;  // the tile scan holds at most 8 rounds x 32 warps
    const size_t smem = size_t(TILE / 32 + 2 * TILE) * 4;

    int occ = 0;
    cudaError_t e = cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)f, cfg.block, smem);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch plan occupancy");
    if (occ < 1) return RZ_ERR_UNSUPPORTED;
    const int full_grid = std::max(1, std::min(cfg.ctas_per_sm, occ) * ctx->sms);

    std::vector<ListRec> recs(static_cast<size_t>(nlists));
    std::vector<uint2> mark, single, classify, pair;
    std::vector<uint32_t> groups;
    plan->total_k = 0;
    uint64_t bitmap_words = 0, list_entries = 0, cnt_words = 0;
    for (int32_t l = 0; l < nlists; ++l) {
        const rz_list_desc& d = lists[l];
        if (d.n < 0 || d.k < 0 || d.k > d.n || d.n >= (int64_t(1) << 32)) return RZ_ERR_INVALID_ARG;
        if (d.k > 0 && (!d.data || !d.idx)) return RZ_ERR_INVALID_ARG;
        if (!list_aligned(d, w)) return RZ_ERR_INVALID_ARG;
        ListRec r{};
        r.data = static_cast<uint8_t*>(d.data);
        r.idx = d.idx;
        r.n = uint32_t(d.n);
        r.k = uint32_t(d.k);
        const uint32_t nch = (r.k + TILE - 1) / TILE;
        r.nch = nch;
        if (r.k == 0 || r.k == r.n) {
            recs[size_t(l)] = r;
            continue;  // nothing moves
        }
        if (nch > kMaxTilesPerList) return RZ_ERR_UNSUPPORTED;  // raise items or block for lists this long
        if (nch == 1) {
            r.span = 1;
            r.ngroups = 1;
            single.push_back(make_uint2(uint32_t(l), (K_SINGLE << 28)));
        } else {
            r.span = span_for(nch, cfg.span);
            r.ngroups = (nch + r.span - 1) / r.span;
            r.bitmap_off = uint32_t(bitmap_words);
            r.list_off = list_entries;
            r.cnt_off = uint32_t(cnt_words);
            bitmap_words += (uint64_t(r.k) + 31) / 32;
            list_entries += uint64_t(nch) * TILE;
            cnt_words += 2ull * nch;
            groups.push_back(r.ngroups);
            for (uint32_t g = 0; g < r.ngroups; ++g) {
                mark.push_back(make_uint2(uint32_t(l), (K_MARK << 28) | g));
                classify.push_back(make_uint2(uint32_t(l), (K_CLASSIFY << 28) | g));
                pair.push_back(make_uint2(uint32_t(l), (K_PAIR << 28) | g));
            }
        }
        plan->total_k += r.k;
        recs[size_t(l)] = r;
    }
    if (bitmap_words >= (1ull << 32) || cnt_words >= (1ull << 32)) return RZ_ERR_UNSUPPORTED;
    // Big SINGLE lists first: the tail of the queue is then made of short items.
    std::sort(single.begin(), single.end(), [&](const uint2& a, const uint2& b) {
        return recs[a.x].k > recs[b.x].k;
    });
    std::vector<uint2> queue;
    order_queue(mark, single, classify, pair, groups, size_t(std::max(0, cfg.wave)) * size_t(full_grid) / 2, queue);

    const size_t b_lists = sizeof(ListRec) * std::max<size_t>(recs.size(), 1);
    const size_t b_queue = sizeof(uint2) * std::max<size_t>(queue.size(), 1);
    const size_t b_ctr = sizeof(uint32_t) * (1 + 2 * size_t(nlists));
    const size_t b_cnt = sizeof(uint32_t) * std::max<uint64_t>(cnt_words, 1);
    const size_t b_bits = sizeof(uint32_t) * std::max<uint64_t>(bitmap_words, 1);
    const size_t b_list = sizeof(uint32_t) * std::max<uint64_t>(list_entries, 1);
    auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t off_queue = up(b_lists), off_ctr = off_queue + up(b_queue), off_cnt = off_ctr + up(b_ctr),
                 off_bits = off_cnt + up(b_cnt), off_dl = off_bits + up(b_bits), off_sl = off_dl + up(b_list),
                 total = off_sl + up(b_list);
    void* dev = nullptr;
    RZ_CUDA_TRY(ctx, cudaMalloc(&dev, total));
    uint8_t* b = static_cast<uint8_t*>(dev);
    e = recs.empty() ? cudaSuccess : cudaMemcpy(b, recs.data(), sizeof(ListRec) * recs.size(),
                                                            cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !queue.empty())
        e = cudaMemcpy(b + off_queue, queue.data(), sizeof(uint2) * queue.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(b + off_ctr, 0, off_bits - off_ctr + up(b_bits));
    if (e != cudaSuccess) {
        cudaFree(dev);
        return cuda_fail(ctx, e, "batch plan upload");
    }
    plan->ctx = ctx;
    plan->w = w;
    plan->cfg = cfg;
    plan->smem = smem;
    plan->grid = std::max(1, std::min<int>(full_grid, int(queue.size())));
    plan->nlists = uint32_t(nlists);
    plan->nitems = uint32_t(queue.size());
    plan->dev = dev;
    plan->counters_bytes = b_ctr;
    BatchParams& p = plan->params;
    p.lists = reinterpret_cast<const ListRec*>(b);
    p.queue = reinterpret_cast<const uint2*>(b + off_queue);
    p.nitems = plan->nitems;
    p.counters = reinterpret_cast<uint32_t*>(b + off_ctr);
    p.chunk_cnt = reinterpret_cast<uint32_t*>(b + off_cnt);
    p.bitmap = reinterpret_cast<uint32_t*>(b + off_bits);
    p.dlist = reinterpret_cast<uint32_t*>(b + off_dl);
    p.slist = reinterpret_cast<uint32_t*>(b + off_sl);
    p.status = ctx->ws.status;
    p.spin_limit = kSpinLimit;
    return RZ_OK;
}

// Enqueue one execution of the plan: counters reset + the persistent kernel.
static int plan_enqueue(rz_batch_plan* plan, cudaStream_t s) {
    rz_ctx* ctx = plan->ctx;
    RZ_CUDA_TRY(ctx, cudaMemsetAsync(plan->params.counters, 0, plan->counters_bytes, s));
    if (plan->nitems == 0) return RZ_OK;
    BatchFn f = batch_fn(int(plan->w), plan->cfg.items);
    f<<<plan->grid, plan->cfg.block, plan->smem, s>>>(plan->params);
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    return RZ_OK;
}

bool default_batch_cfg(const rz_ctx* ctx, uint32_t w, rz_batch_cfg* cfg);  // rz_autotune.cpp

// The default (or tuned) configuration, with items and then block raised until every list fits
// in kMaxTilesPerList tiles (a plan created without a configuration must not fail on long lists).
static void default_fitting(const rz_ctx* ctx, const rz_list_desc* lists, int32_t nlists, uint32_t w,
                            rz_batch_cfg* cfg) {
    default_batch_cfg(ctx, w, cfg);
    int64_t kmax = 0;
    for (int32_t l = 0; l < nlists; ++l)
        if (lists[l].k < lists[l].n) kmax = std::max<int64_t>(kmax, lists[l].k);
    while (int64_t(cfg->block) * cfg->items * kMaxTilesPerList < kmax) {
        if (cfg->items < 8) cfg->items *= 2;
        else if (cfg->block < 512) cfg->block *= 2;
        else break;
    }
}

// ------------------------------------------------------------------------------------------------
// Arenas: batched launches without per-launch allocation (used by the streaming service). An
// arena owns device scratch and pinned host staging sized for at most `max_lists` lists with at
// most `max_k` removals in total; a launch builds its queue and list records in the host staging,
// uploads them on the launch stream and runs the kernel. The caller must not reuse an arena until
// its previous launch has completed (the upload reads the staging asynchronously).
// ------------------------------------------------------------------------------------------------
struct BatchArena {
    rz_ctx* ctx = nullptr;
    uint32_t w = 0;
    rz_batch_cfg cfg{};
    uint32_t tile = 0;
    size_t smem = 0;
    int grid = 0;
    size_t max_lists = 0, max_items = 0, max_bits = 0, max_entries = 0, max_cnt = 0;
    uint8_t* dev = nullptr;
    uint8_t* host = nullptr;  // pinned
    size_t off_queue = 0, off_ctr = 0, off_cnt = 0, off_bits = 0, off_dl = 0, off_sl = 0, total = 0;
};

int arena_create(rz_ctx* ctx, uint32_t w, const rz_batch_cfg* cfg_in, size_t max_lists, size_t max_k,
                 BatchArena** out) {
    rz_batch_cfg cfg{};
    if (cfg_in) cfg = *cfg_in;
    else default_batch_cfg(ctx, w, &cfg);
    BatchFn f = batch_fn(int(w), cfg.items);
    if (!f || max_lists == 0) return RZ_ERR_INVALID_ARG;
    cudaFuncAttributes fa{};
    RZ_CUDA_TRY(ctx, cudaFuncGetAttributes(&fa, (const void*)f));
    cfg.block = std::min(cfg.block, fa.maxThreadsPerBlock & ~31);
    BatchArena* a = new (std::nothrow) BatchArena();
    if (!a) return RZ_ERR_NO_MEMORY;
    a->ctx = ctx;
    a->w = w;
    a->cfg = cfg;
    a->tile = uint32_t(cfg.block) * uint32_t(cfg.items);
    a->smem = size_t(a->tile / 32 + 2 * a->tile) * 4;
    a->max_lists = max_lists;
    const size_t max_tiles = max_k / a->tile + max_lists;  // sum over lists of ceil(k / tile)
    a->max_items = 3 * max_tiles + max_lists;
    a->max_bits = max_k / 32 + max_lists;
    a->max_entries = max_tiles * a->tile;
    a->max_cnt = 2 * max_tiles;
    auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
    a->off_queue = up(sizeof(ListRec) * max_lists);
    a->off_ctr = a->off_queue + up(sizeof(uint2) * a->max_items);
    a->off_cnt = a->off_ctr + up(4 * (1 + 2 * max_lists));
    a->off_bits = a->off_cnt + up(4 * a->max_cnt);
    a->off_dl = a->off_bits + up(4 * a->max_bits);
    a->off_sl = a->off_dl + up(4 * a->max_entries);
    a->total = a->off_sl + up(4 * a->max_entries);
    cudaError_t e = cudaMalloc(&a->dev, a->total);
    if (e == cudaSuccess) e = cudaMemset(a->dev, 0, a->total);
    if (e == cudaSuccess) e = cudaMallocHost(&a->host, a->off_ctr);
    int occ = 0;
    if (e == cudaSuccess) e = cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(a->smem));
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)f, cfg.block, a->smem);
    if (e != cudaSuccess || occ < 1) {
        const int st = e != cudaSuccess ? cuda_fail(ctx, e, "arena_create") : RZ_ERR_UNSUPPORTED;
        if (a->dev) cudaFree(a->dev);
        if (a->host) cudaFreeHost(a->host);
        delete a;
        return st;
    }
    a->grid = std::max(1, std::min(cfg.ctas_per_sm, occ) * ctx->sms);
    *out = a;
    return RZ_OK;
}

void arena_destroy(BatchArena* a) {
    if (!a) return;
    cudaFree(a->dev);
    cudaFreeHost(a->host);
    delete a;
}

// Build the plan for `lists` into the arena and launch it on `s` (no allocation). Lists must
// respect the arena's limits (RZ_ERR_UNSUPPORTED otherwise, before anything is enqueued).
int arena_launch(BatchArena* a, const rz_list_desc* lists, int nlists, cudaStream_t s) {
    rz_ctx* ctx = a->ctx;
    if (nlists < 0 || size_t(nlists) > a->max_lists) return RZ_ERR_UNSUPPORTED;
    ListRec* recs = reinterpret_cast<ListRec*>(a->host);
    uint2* queue = reinterpret_cast<uint2*>(a->host + a->off_queue);
    const uint32_t TILE = a->tile;
    // Count first (so limits are checked before anything is written or enqueued).
    size_t nmark = 0, nsingle = 0, bits = 0, entries = 0, cnt = 0;
    for (int l = 0; l < nlists; ++l) {
        const rz_list_desc& d = lists[l];
        if (d.n < 0 || d.k < 0 || d.k > d.n || d.n >= (int64_t(1) << 32)) return RZ_ERR_INVALID_ARG;
        if (d.k > 0 && (!d.data || !d.idx)) return RZ_ERR_INVALID_ARG;
        if (!list_aligned(d, a->w)) return RZ_ERR_INVALID_ARG;
        if (d.k == 0 || d.k == d.n) continue;
        const uint32_t nch = uint32_t((uint64_t(d.k) + TILE - 1) / TILE);
        if (nch > kMaxTilesPerList) return RZ_ERR_UNSUPPORTED;
        if (nch == 1) {
            ++nsingle;
        } else {
            const uint32_t span = span_for(nch, a->cfg.span);
            nmark += (nch + span - 1) / span;
            bits += (uint64_t(d.k) + 31) / 32;
            entries += size_t(nch) * TILE;
            cnt += 2 * size_t(nch);
        }
    }
    if (3 * nmark + nsingle > a->max_items || bits > a->max_bits || entries > a->max_entries || cnt > a->max_cnt)
        return RZ_ERR_UNSUPPORTED;
    std::vector<uint2> mark, single, classify, pair, ordered;
    std::vector<uint32_t> groups;
    mark.reserve(nmark);
    classify.reserve(nmark);
    pair.reserve(nmark);
    single.reserve(nsingle);
    bits = entries = cnt = 0;
    for (int l = 0; l < nlists; ++l) {
        const rz_list_desc& d = lists[l];
        ListRec r{};
        r.data = static_cast<uint8_t*>(d.data);
        r.idx = d.idx;
        r.n = uint32_t(d.n);
        r.k = uint32_t(d.k);
        const uint32_t nch = uint32_t((uint64_t(d.k) + TILE - 1) / TILE);
        r.nch = nch;
        if (!(d.k == 0 || d.k == d.n)) {
            if (nch == 1) {
                r.span = r.ngroups = 1;
                single.push_back(make_uint2(uint32_t(l), K_SINGLE << 28));
            } else {
                r.span = span_for(nch, a->cfg.span);
                r.ngroups = (nch + r.span - 1) / r.span;
                r.bitmap_off = uint32_t(bits);
                r.list_off = entries;
                r.cnt_off = uint32_t(cnt);
                bits += (uint64_t(d.k) + 31) / 32;
                entries += size_t(nch) * TILE;
                cnt += 2 * size_t(nch);
                groups.push_back(r.ngroups);
                for (uint32_t g = 0; g < r.ngroups; ++g) {
                    mark.push_back(make_uint2(uint32_t(l), (K_MARK << 28) | g));
                    classify.push_back(make_uint2(uint32_t(l), (K_CLASSIFY << 28) | g));
                    pair.push_back(make_uint2(uint32_t(l), (K_PAIR << 28) | g));
                }
            }
        }
        recs[l] = r;
    }
    std::sort(single.begin(), single.end(), [&](const uint2& x, const uint2& y) { return recs[x.x].k > recs[y.x].k; });
    order_queue(mark, single, classify, pair, groups, size_t(std::max(0, a->cfg.wave)) * size_t(a->grid) / 2,
                ordered);
    std::copy(ordered.begin(), ordered.end(), queue);
    const size_t nitems = ordered.size();
    if (nlists > 0)
        RZ_CUDA_TRY(ctx, cudaMemcpyAsync(a->dev, a->host, sizeof(ListRec) * size_t(nlists), cudaMemcpyHostToDevice, s));
    if (nitems)
        RZ_CUDA_TRY(ctx, cudaMemcpyAsync(a->dev + a->off_queue, a->host + a->off_queue, sizeof(uint2) * nitems,
                                         cudaMemcpyHostToDevice, s));
    RZ_CUDA_TRY(ctx, cudaMemsetAsync(a->dev + a->off_ctr, 0, 4 * (1 + 2 * size_t(nlists)), s));
    if (nitems == 0) return RZ_OK;
    BatchParams p;
    p.lists = reinterpret_cast<const ListRec*>(a->dev);
    p.queue = reinterpret_cast<const uint2*>(a->dev + a->off_queue);
    p.nitems = uint32_t(nitems);
    p.counters = reinterpret_cast<uint32_t*>(a->dev + a->off_ctr);
    p.chunk_cnt = reinterpret_cast<uint32_t*>(a->dev + a->off_cnt);
    p.bitmap = reinterpret_cast<uint32_t*>(a->dev + a->off_bits);
    p.dlist = reinterpret_cast<uint32_t*>(a->dev + a->off_dl);
    p.slist = reinterpret_cast<uint32_t*>(a->dev + a->off_sl);
    p.status = ctx->ws.status;
    p.spin_limit = kSpinLimit;
    BatchFn f = batch_fn(int(a->w), a->cfg.items);
    f<<<std::min<int>(a->grid, int(nitems)), a->cfg.block, a->smem, s>>>(p);
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    return RZ_OK;
}

}  // namespace rz

using namespace rz;

extern "C" {

int rz_batch_plan_create(rz_ctx* ctx, const rz_list_desc* lists, int32_t nlists, uint32_t elem_bytes,
                         const rz_batch_cfg* cfg, rz_batch_plan** out) {
    if (!ctx || !out || (nlists > 0 && !lists) || nlists < 0) return RZ_ERR_INVALID_ARG;
    if (elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16 && elem_bytes != 32) return RZ_ERR_INVALID_ARG;
    *out = nullptr;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    rz_batch_cfg c{};
    bool predicted = false;
    if (cfg) c = *cfg;
    else if (!(predicted = predict_batch_cfg(ctx, lists, nlists, elem_bytes, &c)))
        default_fitting(ctx, lists, nlists, elem_bytes, &c);
    rz_batch_plan* plan = new (std::nothrow) rz_batch_plan();
    if (!plan) return RZ_ERR_NO_MEMORY;
    int st = plan_build(ctx, lists, nlists, elem_bytes, c, plan);
    if (st == RZ_ERR_UNSUPPORTED && predicted) {
        // The network's choice cannot plan these lists (a tile too small for the longest one):
        // fall back to the default with a tile that fits.
        default_fitting(ctx, lists, nlists, elem_bytes, &c);
        st = plan_build(ctx, lists, nlists, elem_bytes, c, plan);
    }
    if (st != RZ_OK) {
        delete plan;
        return st;
    }
    *out = plan;
    return RZ_OK;
}

int rz_batch_plan_launch(rz_batch_plan* plan, rz_stream_t stream) {
    if (!plan) return RZ_ERR_INVALID_ARG;
    rz_ctx* ctx = plan->ctx;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!plan->exec) {
        // Capture once on a private stream; every later launch is one graph launch.
        cudaStream_t cs = nullptr;
        RZ_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        int st = RZ_OK;
        if (e == cudaSuccess) st = plan_enqueue(plan, cs);
        cudaGraph_t graph = nullptr;
        const cudaError_t e2 = (e == cudaSuccess) ? cudaStreamEndCapture(cs, &graph) : e;
        cudaStreamDestroy(cs);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamBeginCapture");
        if (st != RZ_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e2 != cudaSuccess) return cuda_fail(ctx, e2, "cudaStreamEndCapture");
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e3 = cudaGraphInstantiate(&exec, graph, 0);
        if (e3 != cudaSuccess) {
            cudaGraphDestroy(graph);
            return cuda_fail(ctx, e3, "cudaGraphInstantiate");
        }
        plan->graph = graph;
        plan->exec = exec;
    }
    RZ_CUDA_TRY(ctx, cudaGraphLaunch(plan->exec, s));
    ctx->last_kernels = plan->nitems ? 1 : 0;
    ctx->last_grid = plan->grid;
    ctx->last_block = plan->cfg.block;
    return RZ_OK;
}

int rz_batch_plan_info(const rz_batch_plan* plan, int32_t* grid, int32_t* block, int32_t* items, int64_t* work_items,
                       int64_t* total_k) {
    if (!plan) return RZ_ERR_INVALID_ARG;
    if (grid) *grid = plan->grid;
    if (block) *block = plan->cfg.block;
    if (items) *items = plan->cfg.items;
    if (work_items) *work_items = plan->nitems;
    if (total_k) *total_k = int64_t(plan->total_k);
    return RZ_OK;
}

void rz_batch_plan_destroy(rz_batch_plan* plan) {
    if (!plan) return;
    cudaSetDevice(plan->ctx->device);
    cudaDeviceSynchronize();
    if (plan->exec) cudaGraphExecDestroy(plan->exec);
    if (plan->graph) cudaGraphDestroy(plan->graph);
    cudaFree(plan->dev);
    delete plan;
}

int rz_remove_batched(rz_ctx* ctx, const rz_list_desc* lists, int32_t nlists, uint32_t elem_bytes, uint32_t flags,
                      rz_stream_t stream) {
    rz_batch_plan* plan = nullptr;
    int st = rz_batch_plan_create(ctx, lists, nlists, elem_bytes, nullptr, &plan);
    if (st != RZ_OK) return st;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    st = plan_enqueue(plan, reinterpret_cast<cudaStream_t>(stream));
    if (st == RZ_OK) st = read_status(ctx, reinterpret_cast<cudaStream_t>(stream));
    ctx->last_kernels = plan->nitems ? 1 : 0;
    ctx->last_grid = plan->grid;
    ctx->last_block = plan->cfg.block;
    (void)flags;
    rz_batch_plan_destroy(plan);
    return st;
}

}  // extern "C"
