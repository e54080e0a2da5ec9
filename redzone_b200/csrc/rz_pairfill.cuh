// rz_pairfill.cuh -- the last two steps of a single-list removal in a CTA that knows every red
// entry: derive the canonical pairing, then fill its own tile's holes.
//
// Shared by the kernels in which each CTA holds complete V and P maps in shared memory (the
// cluster-scan schedule, rz_cscan.cu, and the produced-list path, rz_produced.cu). The rule is
// the reference's (Algorithm 2, redzone.hxx:777-813 and 852-933): with cut = n - k and red
// entries {(i, idx[i]) : idx[i] >= cut}, V = {idx[i] - cut} (tail positions whose item is
// removed) and P = {i} (holes that need no fill); destination orphans are V \ P and source
// orphans P \ V, each ranked by position, and the r-th destination orphan takes the item of the
// r-th source orphan.
#pragma once

#include "rz_common.cuh"
#include "rz_internal.h"
#include "rz_single_kernel.cuh"

namespace rz {

// Shared-memory state of one CTA: from `base`, the V map, the P map and the slow path's per-word
// destination / source orphan prefixes (`stride` words each, stride >= ceil(k / 32)), then the
// red positions, red values and source orphans (kFastMaxRed words each). With R <= kFastMaxRed
// ("fast"), positions / values hold the red entries in position order; otherwise only the maps
// are used. cnt is two 257-word count buffers, scan at least 2 words.
struct PairFillSmem {
    uint32_t* base;
    uint32_t stride;
    uint32_t (*cnt)[16 * 16 + 1];
    uint32_t* scan;
    __device__ __forceinline__ uint32_t* mapV() const { return base; }
    __device__ __forceinline__ uint32_t* mapP() const { return base + stride; }
    __device__ __forceinline__ uint32_t* dpre() const { return base + 2 * stride; }
    __device__ __forceinline__ uint32_t* spre() const { return base + 3 * stride; }
    __device__ __forceinline__ uint32_t* pos() const { return base + 4 * stride; }
    __device__ __forceinline__ uint32_t* val() const { return base + 4 * stride + kFastMaxRed; }
    __device__ __forceinline__ uint32_t* src() const { return base + 4 * stride + 2 * kFastMaxRed; }
};
// Words of the layout above (the kernel's own arrays may follow).
__host__ __device__ inline size_t pairfill_words(uint32_t stride) { return 4 * size_t(stride) + 3 * size_t(kFastMaxRed); }

// The pairing as this CTA needs it: the number of source orphans (stot), the destination orphans
// before its tile (dbase, fast path) and per-(round, warp) ranks inside the tile (cnt[1]).
// has_tile: the CTA owns tile [chunk_base, chunk_base + blockDim.x * IPT).
template <int IPT>
__device__ __forceinline__ void derive_pairing(const PairFillSmem& s, uint32_t R, uint32_t k, uint32_t chunk_base,
                                               bool has_tile, uint32_t* status, uint32_t& stot,
                                               uint32_t& dbase) {
    const uint32_t B = blockDim.x, kw = (k + 31) >> 5;
    const int nw = int(B >> 5), lane = threadIdx.x & 31, warp = threadIdx.x >> 5, E = IPT * nw;
    const uint32_t lt = lanemask_lt();
    const bool fast = R <= kFastMaxRed;
    uint32_t* mapV = s.mapV();
    uint32_t* mapP = s.mapP();
    uint32_t* cbuf = s.cnt[1];
    stot = 0;
    dbase = 0;
    if (fast && R <= 32u && E <= 32) {
        // Few red entries (the usual case: about k^2/n of them): warp 0 pairs them, one lane per
        // entry, while another warp scans this tile's V \ P word counts; one barrier.
        if (warp == 0) {
            uint32_t ps = 0;
            bool sf = false, af = false, df = false;
            if (uint32_t(lane) < R) {
                ps = s.pos()[lane];
                const uint32_t v = s.val()[lane];
                sf = !((mapV[ps >> 5] >> (ps & 31u)) & 1u);
                af = !((mapP[v >> 5] >> (v & 31u)) & 1u);
                df = af && v < chunk_base;
            }
            const uint32_t bs = __ballot_sync(0xffffffffu, sf);
            const uint32_t bd = __ballot_sync(0xffffffffu, df);
            const uint32_t ba = __ballot_sync(0xffffffffu, af);
            if (sf) s.src()[__popc(bs & lt)] = ps;
            if (lane == 0) {
                s.scan[0] = __popc(bs);
                s.scan[1] = __popc(bd);
                if (blockIdx.x == 0 && __popc(ba) != __popc(bs)) atomicOr(status, ST_INCONSISTENT);
            }
        }
        if (warp == (nw > 1 ? 1 : 0)) {
            // cbuf[j * nw + w] = V \ P bits of this tile before word (j, w).
            uint32_t x = 0;
            if (lane < E) {
                const uint32_t i0 = chunk_base + uint32_t(lane / nw) * B + uint32_t(lane % nw) * 32u;
                x = (has_tile && i0 < k) ? __popc(mapV[i0 >> 5] & ~mapP[i0 >> 5]) : 0u;
            }
            const uint32_t inc = warp_inclusive_scan(x);
            if (lane < E) cbuf[lane] = inc - x;
        }
        __syncthreads();
        stot = s.scan[0];
        dbase = s.scan[1];
    } else if (fast) {
        // Ranks inside this tile: one word of the V \ P map per (round, warp).
        if (lane == 0) {
#pragma unroll
            for (int j = 0; j < IPT; ++j) {
                const uint32_t i0 = chunk_base + uint32_t(j) * B + uint32_t(warp) * 32u;
                cbuf[j * nw + warp] = (has_tile && i0 < k) ? __popc(mapV[i0 >> 5] & ~mapP[i0 >> 5]) : 0u;
            }
        }
        // Source orphans compacted in position order; destination orphans before this tile and
        // in all: rounds of B red entries, per-warp ballot counts, one barrier per round.
        uint32_t dall = 0;
        for (uint32_t q0 = 0, rd = 0; q0 == 0 || q0 < R; q0 += B, ++rd) {
            uint32_t* wc = s.cnt[0] + 96u * (rd & 1u);
            const uint32_t e = q0 + threadIdx.x;
            uint32_t ps = 0;
            bool sf = false, af = false, df = false;
            if (e < R) {
                ps = s.pos()[e];
                const uint32_t v = s.val()[e];
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
            if (sf) s.src()[stot + pre + __popc(bs & lt)] = ps;
            stot += ts;
        }
        if (threadIdx.x == 0 && blockIdx.x == 0 && dall != stot) atomicOr(status, ST_INCONSISTENT);
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
            s.cnt[0][warp] = ssum;
            s.cnt[0][32 + warp] = dsum;
        }
        __syncthreads();
        if (warp == 0) {
            const uint32_t xs = lane < nw ? s.cnt[0][lane] : 0u, xd = lane < nw ? s.cnt[0][32 + lane] : 0u;
            const uint32_t is = warp_inclusive_scan(xs), id = warp_inclusive_scan(xd);
            if (lane < nw) {
                s.cnt[0][64 + lane] = is - xs;
                s.cnt[0][96 + lane] = id - xd;
            }
            if (lane == 31) {
                s.cnt[0][128] = is;
                s.cnt[0][129] = id;
            }
        }
        __syncthreads();
        uint32_t cs = s.cnt[0][64 + warp], cd = s.cnt[0][96 + warp];
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
                s.spre()[w] = cs + is - xs;
                s.dpre()[w] = cd + id - xd;
            }
            cs += __shfl_sync(0xffffffffu, is, 31);
            cd += __shfl_sync(0xffffffffu, id, 31);
        }
        stot = s.cnt[0][128];
        if (threadIdx.x == 0 && blockIdx.x == 0 && s.cnt[0][129] != stot) atomicOr(status, ST_INCONSISTENT);
        __syncthreads();
    }
}

// This tile's holes: a hole below the cut whose own tail item survives takes it (src, already in
// registers); one whose tail item is removed takes the item of the source orphan of its rank.
template <int W, int IPT>
__device__ __forceinline__ void fill_holes(const PairFillSmem& s, uint32_t R, uint32_t k, uint32_t cut,
                                           uint32_t chunk_base, uint32_t stot, uint32_t dbase,
                                           const uint32_t (&rr)[IPT], const typename Payload<W>::T (&src)[IPT],
                                           typename Payload<W>::T* __restrict__ head,
                                           const typename Payload<W>::T* __restrict__ tail) {
    const uint32_t B = blockDim.x, kw = (k + 31) >> 5;
    const int nw = int(B >> 5), lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = lanemask_lt();
    const bool fast = R <= kFastMaxRed;
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        const uint32_t i = chunk_base + uint32_t(j) * B + threadIdx.x;
        if (i >= k || rr[j] >= cut) continue;  // past the list, or a hole needing no fill
        const uint32_t vw = s.mapV()[i >> 5];
        if (!((vw >> lane) & 1u)) {
            head[rr[j]] = src[j];  // valid source, valid destination
            continue;
        }
        const uint32_t below = __popc(vw & ~s.mapP()[i >> 5] & lt);
        const uint32_t rank = fast ? dbase + s.cnt[1][j * nw + warp] + below : s.dpre()[i >> 5] + below;
        if (rank >= stot) continue;  // only with invalid input (reported by derive_pairing)
        uint32_t spos;
        if (fast) {
            spos = s.src()[rank];
        } else {
            // The word holding the rank-th source orphan: last word whose prefix <= rank.
            uint32_t lo = 0, hi = kw;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (s.spre()[mid] <= rank) lo = mid; else hi = mid;
            }
            uint32_t sw = s.mapP()[lo] & ~s.mapV()[lo];
            for (uint32_t c = rank - s.spre()[lo]; c > 0u; --c) sw &= sw - 1u;  // drop lower ones
            spos = lo * 32u + uint32_t(__ffs(sw) - 1);
        }
        head[rr[j]] = tail[spos];
    }
}

}  // namespace rz
