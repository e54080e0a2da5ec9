// rz_single_kernel.cuh -- body of the single-list Redzone kernel (grid-wide persistent schedule),
// shared by the kernel that runs on context scratch (rz_single.cu) and the variant that runs on a
// fixed device-global scratch array (rz_noalloc.cu). The algorithm is described in rz_single.cu.
#pragma once

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
    // Red-list schedule (nullable; set only with one tile per CTA, k <= kRedlistMaxK and the dynamic
    // shared memory it needs): red entries per CTA region and tagged per-CTA entry counts.
    uint2* redlist;
    unsigned long long* arrive64;
};

// Exclusive scan in place of cbuf[0..E) by warp 0 (E <= 256, a few entries per lane); cbuf[E]
// receives the total.
__device__ __forceinline__ void warp0_scan_counts(uint32_t* cbuf, int E, int lane) {
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

// Dynamic shared memory of the red-list schedule for k removals: V and P maps (k bits each),
// then red positions, red values and source orphans (kFastMaxRed words each).
__host__ __device__ inline size_t redlist_smem_bytes(uint32_t k) {
    return (size_t(2) * ((k + 31) / 32) + size_t(3) * kFastMaxRed) * 4;
}

constexpr uint32_t kDeepMarkLoads = 8;  // phase A index loads in flight per thread (several tiles per CTA)

// ------------------------------------------------------------------------------------------------
// Redzone, one list, G persistent CTAs (G == 1 degenerates to block-level synchronisation).
// ------------------------------------------------------------------------------------------------
template <int W, int IPT>
__device__ __forceinline__ void redzone_single_body(const SingleParams& p) {
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
    __shared__ uint32_t s_red_total;     // red-list schedule: red entries of the whole grid
    extern __shared__ uint32_t s_dyn[];  // red-list schedule only
    const bool fast = p.redlist != nullptr && single && G > 1;

    if (threadIdx.x == 0) {
        s_tag = (G > 1) ? ld_acquire(p.epoch) + 1u : 0u;
        s_abort = p.validate ? ((__ldcg(p.status) & (ST_DUPLICATE | ST_RANGE)) != 0) : 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && p.dev_len) *p.dev_len = (unsigned long long)(n - k);

    uint32_t rr[IPT];
    T src[IPT];
#pragma unroll
    for (int j = 0; j < IPT; ++j) rr[j] = 0xffffffffu;

    // ---- phase A: mark the red zone ---------------------------------------------------------
    // The loads are issued before the first __syncthreads so they overlap the epoch read.
    // Several tiles per CTA: the CTA's index entries in any order, kDeepMarkLoads loads in flight
    // per thread (a mark needs nothing but its own entry; phase B re-reads the indices).
    if (!single && t0 < t1) {
        constexpr uint32_t U = kDeepMarkLoads;
        const uint32_t hi = min(t1 * TILE, k), step = U * uint32_t(B);
        uint32_t b = t0 * TILE + threadIdx.x;
        uint32_t r[U];
#pragma unroll
        for (uint32_t j = 0; j < U; ++j) {
            const uint32_t i = b + j * B;
            r[j] = (i < hi) ? __ldg(&p.idx[i]) : 0u;
        }
        __syncthreads();  // s_abort / s_tag
        if (s_abort) return;  // validation failed: leave the caller's data untouched
        for (;;) {
#pragma unroll
            for (uint32_t j = 0; j < U; ++j) {
                const uint32_t i = b + j * B;
                if (i < hi && r[j] >= cut) {
                    if (r[j] >= n) {
                        atomicOr(p.status, ST_RANGE);
                    } else {
                        const uint32_t off = r[j] - cut;
                        const uint32_t bit = 1u << (off & 31u);
                        if (p.validate) {
                            if (atomicOr(&p.bitmap[off >> 5], bit) & bit) atomicOr(p.status, ST_DUPLICATE);
                        } else {
                            atomicOr(&p.bitmap[off >> 5], bit);
                        }
                    }
                }
            }
            if (b >= hi || hi - b <= step) break;
            b += step;
#pragma unroll
            for (uint32_t j = 0; j < U; ++j) {
                const uint32_t i = b + j * B;
                r[j] = (i < hi) ? __ldg(&p.idx[i]) : 0u;
            }
        }
    }
    if (single && t0 < t1) {  // one tile: its indices stay in registers for phase B
        const uint32_t base = t0 * TILE;
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
            rr[j] = (i < k) ? __ldg(&p.idx[i]) : 0xffffffffu;
        }
        // Pull this CTA's tail window into L2 while the grid waits at the barrier. A prefetch
        // is not an outstanding access the arrival's release has to wait for (a load is).
        prefetch_l2(tail + base, size_t(min(TILE, k - base)) * W);
        __syncthreads();  // s_abort / s_tag
        if (s_abort) return;  // validation failed: leave the caller's data untouched
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
    const int E = IPT * nw;

    // ---- red-list schedule: publish this CTA's red entries {position, value - cut}, in position
    // order, and clear the shared-memory maps used after the barrier.
    uint32_t red_mine = 0;
    if (fast) {
        const uint32_t kw = (k + 31) >> 5;
        for (uint32_t q = threadIdx.x; q < 2 * kw; q += B) s_dyn[q] = 0u;
        if (threadIdx.x == 0) s_red_total = 0u;
        uint32_t* cbuf = s_cnt[0];
        uint32_t rm[IPT];
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t i = chunk_base + uint32_t(j) * B + threadIdx.x;
            rm[j] = __ballot_sync(0xffffffffu, i < k && rr[j] >= cut && rr[j] < n);
            if (lane == 0) cbuf[j * nw + warp] = __popc(rm[j]);
        }
        __syncthreads();
        if (warp == 0) warp0_scan_counts(cbuf, E, lane);
        __syncthreads();
        const uint32_t lt = lanemask_lt();
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            if ((rm[j] >> lane) & 1u) {
                const uint32_t i = chunk_base + uint32_t(j) * B + threadIdx.x;
                p.redlist[chunk_base + cbuf[j * nw + warp] + __popc(rm[j] & lt)] = make_uint2(i, rr[j] - cut);
            }
        }
        red_mine = cbuf[E];
    }

    constexpr uint32_t kEarly = 4;  // red entries per CTA pulled while polling (red-list schedule)
    uint2 early[kEarly];
    if (G > 1) {
        if (fast) {
            // Arrival carries the red-entry count: tag << 32 | count, released after the entries.
            __syncthreads();
            if (threadIdx.x == 0)
                st_release_u64(&p.arrive64[blockIdx.x], ((unsigned long long)tag << 32) | red_mine);
            RZ_STAMP(p, 5);
            // Acquire polls. As soon as CTA c's arrival is seen, its poller pulls CTA c's first
            // kEarly red entries into registers and the shared maps, so that part of the gather
            // overlaps the wait for the slower CTAs (measured: -0.6 us steady state).
            int ok = 1;
            for (uint32_t c = threadIdx.x; c < G && ok; c += B) {
                uint32_t it = 0;
                unsigned long long w = ld_acquire_u64(&p.arrive64[c]);
                while (uint32_t(w >> 32) != tag) {
                    if (++it > p.spin_limit) {
                        ok = 0;
                        break;
                    }
                    w = ld_acquire_u64(&p.arrive64[c]);
                }
                const uint32_t cnt = uint32_t(w);
                s_pd[c] = cnt;
                atomicAdd(&s_red_total, cnt);
                if (c == threadIdx.x && ok) {
                    const uint2* ent = p.redlist + size_t(c) * TILE;
#pragma unroll
                    for (uint32_t e = 0; e < kEarly; ++e) {
                        if (e < cnt) {
                            early[e] = __ldcg(&ent[e]);
                            atomicOr(&s_dyn[early[e].y >> 5], 1u << (early[e].y & 31u));               // V map
                            atomicOr(&s_dyn[((k + 31) >> 5) + (early[e].x >> 5)], 1u << (early[e].x & 31u));  // P map
                        }
                    }
                }
            }
            if (!__syncthreads_and(ok)) {
                if (threadIdx.x == 0) atomicOr(p.status, ST_TIMEOUT);
                return;
            }
            RZ_STAMP(p, 7);
            if (s_red_total > kFastMaxRed) {
                // The bitmap phases read the other CTAs' marks: one acquire fence for the block.
                // (The red-list path reads only entries that its own pollers acquired.)
                if (threadIdx.x == 0) fence_acq_rel_gpu();
                __syncthreads();
            }
        } else {
            flag_arrive(p.arrive, blockIdx.x, tag);
            RZ_STAMP(p, 5);
            if (!flag_wait_all(p.arrive, G, tag, p.status, p.spin_limit)) return;
        }
        // Every CTA has read the epoch (it arrived): advance it for the next call.
        if (blockIdx.x == 0 && threadIdx.x == 0) *p.epoch = tag;
    } else {
        __syncthreads();
    }
    RZ_STAMP(p, 2);

    if (fast) {
        if (s_red_total <= kFastMaxRed) {
            // ---- every CTA derives the pairing from the red list -------------------------------
            // V = tail positions i with cut + i in idx (sources that are removed), P = positions
            // i with idx[i] >= cut (holes that need no filling). Destination orphans are V \ P
            // and source orphans P \ V, both ranked in position order (the canonical rule).
            const uint32_t R = s_red_total;
            const uint32_t kw = (k + 31) >> 5;
            uint32_t* mapV = s_dyn;
            uint32_t* mapP = s_dyn + kw;
            uint32_t* s_pos = mapP + kw;  // red positions, in position order
            uint32_t* s_val = s_pos + kFastMaxRed;
            uint32_t* s_src = s_val + kFastMaxRed;  // source orphans, in position order
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i = chunk_base + uint32_t(j) * B + threadIdx.x;
                if (i < k) src[j] = tail[i];  // L2 hit: prefetched in phase A
            }
            // Red entries before each CTA: warp 0 scans the G counts (a few per lane, in order).
            if (warp == 0) {
                const uint32_t per = (G + 31) >> 5;
                const uint32_t ca = min(uint32_t(lane) * per, G), cb = min(ca + per, G);
                uint32_t s = 0;
                for (uint32_t c = ca; c < cb; ++c) s += s_pd[c];
                uint32_t run = warp_inclusive_scan(s) - s;
                for (uint32_t c = ca; c < cb; ++c) {
                    const uint32_t x = s_pd[c];
                    s_ps[c] = run;  // exclusive prefix; s_pd keeps the counts
                    run += x;
                }
            }
            __syncthreads();
            // Gather, in position order: the poller of CTA c places CTA c's entries at their
            // ranks -- the first kEarly from registers (already in the maps), the rest now.
            for (uint32_t c = threadIdx.x; c < G; c += B) {
                const uint32_t cnt = s_pd[c], at = s_ps[c];
                const uint2* ent = p.redlist + size_t(c) * TILE;
                const uint32_t e0 = (c == threadIdx.x) ? min(cnt, kEarly) : 0u;
                if (c == threadIdx.x) {
#pragma unroll
                    for (uint32_t e = 0; e < kEarly; ++e) {
                        if (e < e0) {
                            s_pos[at + e] = early[e].x;
                            s_val[at + e] = early[e].y;
                        }
                    }
                }
                for (uint32_t e = e0; e < cnt; ++e) {
                    const uint2 en = __ldcg(&ent[e]);
                    s_pos[at + e] = en.x;
                    s_val[at + e] = en.y;
                    atomicOr(&mapV[en.y >> 5], 1u << (en.y & 31u));
                    atomicOr(&mapP[en.x >> 5], 1u << (en.x & 31u));
                }
            }
            __syncthreads();
            RZ_STAMP(p, 6);
            // Ranks inside this tile: one word of the V \ P map per (round, warp).
            uint32_t* cbuf = s_cnt[1];
            if (lane == 0) {
#pragma unroll
                for (int j = 0; j < IPT; ++j) {
                    const uint32_t i0 = chunk_base + uint32_t(j) * B + uint32_t(warp) * 32u;
                    cbuf[j * nw + warp] = i0 < k ? __popc(mapV[i0 >> 5] & ~mapP[i0 >> 5]) : 0u;
                }
            }
            // Source orphans (P \ V) compacted in position order, destination orphans (V \ P)
            // before this tile and in all: rounds of B red entries, per-warp ballot counts, one
            // barrier per round (double-buffered counts; the first round always runs, so the
            // tile's word counts above are published by it too).
            const uint32_t lt = lanemask_lt();
            uint32_t stot = 0, dbase = 0, dall = 0;
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
            __syncthreads();  // s_src and the tile's ranks are complete
            RZ_STAMP(p, 3);
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i = chunk_base + uint32_t(j) * B + threadIdx.x;
                if (i >= k || rr[j] >= cut) continue;  // past the list, or a hole needing no fill
                const uint32_t vw = mapV[i >> 5];
                if (!((vw >> lane) & 1u)) {
                    head[rr[j]] = src[j];  // valid source, valid destination
                } else {
                    const uint32_t rank = dbase + cbuf[j * nw + warp] + __popc(vw & ~mapP[i >> 5] & lt);
                    if (rank < stot) head[rr[j]] = tail[s_src[rank]];
                }
            }
            if (lane == 0) {  // leave the global red-zone bitmap zero for the next call
#pragma unroll
                for (int j = 0; j < IPT; ++j) {
                    const uint32_t i = chunk_base + uint32_t(j) * B + threadIdx.x;
                    if (i < k) p.bitmap[i >> 5] = 0u;
                }
            }
            RZ_STAMP(p, 4);
            return;
        }
    }

    // ---- phase B: classify, fill holes, collect orphans --------------------------------------
    // With one tile per CTA the hole writes are issued only after the orphan counts have been
    // published (below), so the publishing release does not wait for ~k scattered stores.
    uint32_t dcnt = 0, scnt = 0;
    bool dv[IPT], sv[IPT];
#pragma unroll
    for (int j = 0; j < IPT; ++j) dv[j] = sv[j] = false;
    for (uint32_t t = t0, tt = 0; t < t1; ++t, ++tt) {
        const uint32_t base = t * TILE;
        if (!single && t + 1 < t1) {
            // The next tile's indices and tail window go to L2 while this one is processed.
            const uint32_t nb = base + TILE, cnt = min(TILE, k - nb);
            prefetch_l2(p.idx + nb, size_t(cnt) * 4);
            prefetch_l2(tail + nb, size_t(cnt) * W);
        }
        // Index (re-read when a CTA has several tiles), bitmap word and tail item are loaded
        // together, the tail item whether it is needed or not: one round trip per tile.
        uint32_t word[IPT];
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
            if (i < k) {
                if (!single) rr[j] = __ldg(&p.idx[i]);
                word[j] = __ldcg(&p.bitmap[i >> 5]);
                src[j] = tail[i];  // with one tile per CTA: an L2 hit (prefetched in phase A)
            } else {
                if (!single) rr[j] = 0xffffffffu;
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
                sv[j] = false;
                dv[j] = false;
            }
        }
        if (!single) {
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
        // With one tile per CTA the clear waits until the counts are published (below), so the
        // publishing release does not wait for these stores either.
        if (!single && lane == 0) {
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
                if (i < k) p.bitmap[i >> 5] = 0u;
            }
        }
        __syncthreads();
        if (tt == 0) RZ_STAMP(p, 6);
        if (warp == 0) warp0_scan_counts(cbuf, E, lane);  // packed D << 16 | S counts
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
                    // 4-byte items: the list holds the source item itself (in registers: every
                    // tile loads its tail items; tail items are never written), which saves
                    // phase C a dependent random load per orphan. Otherwise it holds the source
                    // position.
                    if constexpr (W == 4) {
                        p.slist[chunk_base + scnt + rank] = uint32_t(src[j]);
                    } else {
                        p.slist[chunk_base + scnt + rank] = cut + i;
                    }
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
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i = t0 * TILE + uint32_t(j) * B + threadIdx.x;
                if (i < k) p.bitmap[i >> 5] = 0u;
            }
        }
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
        RZ_STAMP(p, 7);
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
        const uint32_t ent = __ldcg(&p.slist[base2 + (jr - s_ps[c2])]);
        const uint32_t dest = __ldcg(&p.dlist[chunk_base + r]);
        if constexpr (W == 4) {
            head[dest] = T(ent);
        } else {
            head[dest] = reinterpret_cast<const T*>(p.data)[ent];
        }
    }
    RZ_STAMP(p, 4);
}

}  // namespace rz
