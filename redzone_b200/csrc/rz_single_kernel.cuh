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
};

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
                    // 4-byte items with one tile per CTA: the list holds the source item itself
                    // (already in registers; tail items are never written), which saves phase C
                    // a dependent load. Otherwise it holds the source position.
                    if constexpr (W == 4) {
                        p.slist[chunk_base + scnt + rank] = single ? uint32_t(src[j]) : cut + i;
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
            head[dest] = single ? T(ent) : reinterpret_cast<const T*>(p.data)[ent];
        } else {
            head[dest] = reinterpret_cast<const T*>(p.data)[ent];
        }
    }
    RZ_STAMP(p, 4);
}

}  // namespace rz
