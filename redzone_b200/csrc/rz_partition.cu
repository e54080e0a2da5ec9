// rz_partition.cu -- the O(n) comparator: mark, then stable in-place compaction.
//
// The reference's O(n) paths mark the k removed slots (remove_phase1, DataStruct.hxx:11-18) and
// then run a partition-style compaction: InK's count / scan / scatter (cuCompactor.cuh:29-141,
// out of place) or thrust::remove (Thrust_remove.hxx:15-17, in place). Here the same three steps
// run in place on B200:
//   1. mark:  the k removed positions set bits of an n-bit map in scratch (any payload width);
//   2. count: kept items per tile from the bit map alone (n/8 bytes), then one CTA turns the
//             per-tile counts into exclusive output offsets;
//   3. move:  each tile stages its kept items in shared memory, raises its "staged" flag, and
//             writes them to offset[t] + rank.
// In-place safety without a chained look-back: tile t writes [offset[t], offset[t] + kept[t]),
// a range shorter than one tile that ends at or before the end of tile t's own input, so it
// overlaps the input of at most two tiles u <= t; tile t waits only for those tiles' staged flags.
// Tiles are taken in ticket order, so every tile waited for is held by a running CTA that waits
// for nothing before staging. The move kernel is one HBM pass (read n*w + n/8, write (n-k)*w).
#include <algorithm>
#include <atomic>
#include <climits>

#include "rz_common.cuh"
#include "rz_internal.h"

namespace rz {

constexpr int kPartBlock = 512;

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

// Kept items of each tile (one warp per tile, grid-stride over tiles). The bit map is padded with
// zero words to whole tiles, so every tile's BW words are read as BW/4 16-byte loads, all issued
// before any is used; only bits past n are masked.
template <uint32_t BW>
__global__ void partition_count_kernel(const uint32_t* __restrict__ bits, uint32_t n, uint32_t ntiles,
                                       uint32_t* __restrict__ kept) {
    constexpr uint32_t TILE = BW * 32u;
    constexpr int V = int((BW / 4 + 31) / 32);  // 16-byte loads per lane
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += warps) {
        const uint4* src = reinterpret_cast<const uint4*>(bits + size_t(t) * BW);
        uint4 v[V];
#pragma unroll
        for (int j = 0; j < V; ++j) {
            const uint32_t q = uint32_t(j) * 32u + uint32_t(lane);
            v[j] = q < BW / 4 ? __ldg(&src[q]) : make_uint4(0u, 0u, 0u, 0u);
        }
        uint32_t removed = 0;
#pragma unroll
        for (int j = 0; j < V; ++j) {
            const uint32_t q = uint32_t(j) * 32u + uint32_t(lane);
            const uint32_t w[4] = {v[j].x, v[j].y, v[j].z, v[j].w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const uint32_t first = t * TILE + (q * 4u + uint32_t(e)) * 32u;
                uint32_t word = w[e];
                if (first >= n) word = 0u;
                else if (n - first < 32u) word &= (1u << (n - first)) - 1u;  // bits past n are not items
                removed += __popc(word);
            }
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) removed += __shfl_down_sync(0xffffffffu, removed, d);
        if (lane == 0) kept[t] = min(TILE, n - t * TILE) - removed;
    }
}

// Exclusive scan of kept[0..ntiles) into offset[0..ntiles) and the per-tile records
// {offset, kept, 0, 0} the pipelined move copies with each tile; one CTA of 1024 threads.
// Chunks of kScanChunk counts are loaded coalesced (all loads in flight at once) into shared
// memory, each thread sums a contiguous run of 32, one block scan, and the results are written
// back coalesced; a running carry joins the chunks.
constexpr uint32_t kScanChunk = 32768;
// One padding word per 32 keeps both the coalesced and the per-thread-run accesses free of bank
// conflicts.
__device__ __forceinline__ uint32_t scan_pad(uint32_t i) { return i + (i >> 5); }
constexpr size_t kScanSmem = size_t(kScanChunk + kScanChunk / 32) * 4;
__global__ void __launch_bounds__(1024) partition_scan_kernel(const uint32_t* __restrict__ kept, uint32_t ntiles,
                                                              uint32_t* __restrict__ offset, uint4* __restrict__ recs) {
    extern __shared__ uint32_t s_kept[];  // [kScanChunk + kScanChunk / 32], padded
    __shared__ uint32_t scratch[33];
    constexpr uint32_t B = 1024, PER = kScanChunk / B;
    uint32_t carry = 0;
    for (uint32_t c0 = 0; c0 < ntiles; c0 += kScanChunk) {
        const uint32_t cn = min(kScanChunk, ntiles - c0);
        {
            uint32_t v[PER];
#pragma unroll
            for (uint32_t j = 0; j < PER; ++j) {
                const uint32_t q = j * B + threadIdx.x;
                v[j] = q < cn ? kept[c0 + q] : 0u;
            }
#pragma unroll
            for (uint32_t j = 0; j < PER; ++j) s_kept[scan_pad(j * B + threadIdx.x)] = v[j];
        }
        __syncthreads();
        uint32_t s = 0;
#pragma unroll
        for (uint32_t j = 0; j < PER; ++j) s += s_kept[scan_pad(threadIdx.x * PER + j)];
        uint32_t total;
        uint32_t run = carry + block_exclusive_scan(s, scratch, &total);
#pragma unroll
        for (uint32_t j = 0; j < PER; ++j) {
            const uint32_t x = s_kept[scan_pad(threadIdx.x * PER + j)];
            s_kept[scan_pad(threadIdx.x * PER + j)] = run;
            run += x;
        }
        __syncthreads();
        const uint32_t end = carry + total;  // offset just past this chunk
#pragma unroll 4
        for (uint32_t j = 0; j < PER; ++j) {
            const uint32_t q = j * B + threadIdx.x;
            if (q < cn) {
                const uint32_t o = s_kept[scan_pad(q)];
                const uint32_t o_next = q + 1 < cn ? s_kept[scan_pad(q + 1)] : end;
                offset[c0 + q] = o;
                recs[c0 + q] = make_uint4(o, o_next - o, 0u, 0u);
            }
        }
        carry = end;
        __syncthreads();  // s_kept is reused by the next chunk
    }
}

// One tile per CTA, taken in ticket order (used for payloads that are not 16-byte aligned, and
// when phase stamps are on).
template <int W, int IPT>
__global__ void __launch_bounds__(kPartBlock) partition_move_kernel(
    uint8_t* data, uint32_t n, uint32_t ntiles, uint32_t* __restrict__ bits, const uint32_t* __restrict__ offset,
    uint32_t* staged, unsigned long long* ticket, uint32_t tag, uint32_t* status, uint32_t spin_limit,
    unsigned long long* dev_len, uint32_t new_len, unsigned long long* stamps, uint32_t stamp_stride) {
    using T = typename Payload<W>::T;
    T* A = reinterpret_cast<T*>(data);
    constexpr int B = kPartBlock, NW = B / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr uint32_t TILE = uint32_t(B) * IPT;
    __shared__ T s_stage[IPT * B];
    __shared__ uint32_t s_cnt[IPT * NW + 1];
    __shared__ uint32_t s_tile;
    if (blockIdx.x == 0 && threadIdx.x == 0 && dev_len) *dev_len = new_len;
    const unsigned long long t_start = stamps ? globaltimer() : 0ull;

    if (threadIdx.x == 0) s_tile = uint32_t(atomicAdd(ticket, 1ull));
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= ntiles) return;
    unsigned long long* my_stamps =
        (stamps && tile % stamp_stride == 0 && tile / stamp_stride < uint32_t(kMaxGrid))
            ? stamps + size_t(tile / stamp_stride) * kStampsPerCta : nullptr;
    if (my_stamps && threadIdx.x == 0) {
        my_stamps[0] = t_start;
        my_stamps[1] = globaltimer();
    }
    const uint32_t base = tile * TILE;
    const uint32_t off = __ldg(&offset[tile]);
    T v[IPT];
    uint32_t wd[IPT];
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
        if (i < n) {
            v[j] = A[i];
            wd[j] = __ldcg(&bits[i >> 5]);
        } else {
            wd[j] = 0xffffffffu;  // past the end: treated as removed
        }
    }
    bool keep[IPT];
    uint32_t km[IPT];
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        const uint32_t i = base + uint32_t(j) * B + threadIdx.x;
        keep[j] = ((wd[j] >> (i & 31u)) & 1u) == 0u;
        if (keep[j]) s_stage[j * B + threadIdx.x] = v[j];
        km[j] = __ballot_sync(0xffffffffu, keep[j]);
        if (lane == 0) {
            s_cnt[j * NW + warp] = __popc(km[j]);
            if (i < n) bits[i >> 5] = 0u;  // leave the removal map zero for the next call
        }
    }
    // Every kept value of this tile is in shared memory once this barrier completes (each
    // st.shared consumed its load), so the tile's input range may be overwritten from here on.
    __syncthreads();
    if (threadIdx.x == 0) st_release(&staged[tile], tag);
    if (warp == 0) {
        constexpr int E = IPT * NW;
        constexpr int per = (E + 31) / 32;
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
        // Wait for the (at most two) tiles whose input this tile's output overlaps.
        if (inc > 0 && lane < 2) {
            const uint32_t u0 = off / TILE;
            const uint32_t u = u0 + uint32_t(lane);
            const uint32_t u_last = (off + inc - 1) / TILE;
            if (u <= u_last && u < tile) {
                uint32_t it = 0;
                while (ld_acquire(&staged[u]) != tag) {
                    if (++it > spin_limit) {
                        atomicOr(status, ST_TIMEOUT);
                        break;
                    }
                }
            }
        }
    }
    __syncthreads();
    if (my_stamps && threadIdx.x == 0) my_stamps[2] = globaltimer();
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int j = 0; j < IPT; ++j) {
        if (keep[j]) {
            const uint32_t dst = off + s_cnt[j * NW + warp] + __popc(km[j] & lt);
            A[dst] = s_stage[j * B + threadIdx.x];
        }
    }
    if (my_stamps && threadIdx.x == 0) my_stamps[3] = globaltimer();
}

// ------------------------------------------------------------------------------------------------
// Move step, warp-specialised pipeline: persistent CTAs (one per SM), a ring of kMoveStages
// shared-memory stages of 32 KB. One producer thread takes tickets (the next one prefetched) and
// fills free stages with 1-D TMA bulk copies of the tile payload, its bitmap words and its
// {offset, kept} record; it raises a tile's staged flag as soon as that copy has landed, in issue
// order, whatever the consumers are doing. Two consumer groups of 8 warps take alternate ring
// positions, so one group's flag wait and barrier overlap the other group's stores. Inside a
// group warp w owns a contiguous eighth of the tile: lane j holds the keep word of round j, one
// warp scan ranks the rounds, one group barrier shares the eight warp totals, and every kept
// item is written to offset + rank. Every wait is bounded; on expiry the CTA stops consuming, the
// producer waits (bounded) for its copies in flight, and the status word gets ST_TIMEOUT.
// Requires a 16-byte-aligned payload.
// ------------------------------------------------------------------------------------------------
constexpr int kMoveStages = 6;
constexpr uint32_t kTileBytes = 32768;
constexpr int kMoveGroups = 2;
constexpr int kGroupThreads = 256;
constexpr int kMoveBlock = kMoveGroups * kGroupThreads + 32;

template <int W>
constexpr size_t move_smem_bytes() {
    return size_t(kMoveStages) * kTileBytes + size_t(kMoveStages) * (kTileBytes / W / 8) + size_t(kMoveStages) * 16;
}

template <int W>
__global__ void __launch_bounds__(kMoveBlock, 1) partition_move_ws_kernel(
    uint8_t* data, uint32_t n, uint32_t ntiles, uint32_t* __restrict__ bits, const uint4* __restrict__ recs,
    uint32_t* staged, unsigned long long* ticket, uint32_t tag, uint32_t* status, uint32_t spin_limit,
    unsigned long long* dev_len, uint32_t new_len) {
    using T = typename Payload<W>::T;
    constexpr uint32_t TILE = kTileBytes / W;  // items per tile
    constexpr uint32_t BW = TILE / 32;         // bitmap words per tile
    constexpr int S = kMoveStages;
    constexpr int GW = kGroupThreads / 32;     // warps per consumer group
    constexpr uint32_t PER_WARP = TILE / GW;   // items per warp and tile
    constexpr int R = int(PER_WARP / 32);      // rounds per warp = bitmap words per warp
    static_assert(R >= 1 && R <= 32, "one keep word per lane");
    T* A = reinterpret_cast<T*>(data);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    extern __shared__ __align__(128) uint8_t smem[];
    T* stage = reinterpret_cast<T*>(smem);                                   // [S][TILE]
    uint32_t* sbits = reinterpret_cast<uint32_t*>(smem + S * kTileBytes);    // [S][BW]
    uint4* srec = reinterpret_cast<uint4*>(smem + S * kTileBytes + S * BW * 4);  // [S]
    __shared__ __align__(8) unsigned long long full[S], empty[S];
    __shared__ uint32_t s_tile[S];
    __shared__ uint32_t s_wtot[kMoveGroups][GW];
    __shared__ uint32_t s_go[kMoveGroups][2];  // [group][barrier A / barrier B] outcome
    __shared__ volatile uint32_t s_abort;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], GW);
        }
        s_abort = 0u;
        fence_mbar_init();
        if (blockIdx.x == 0 && dev_len) *dev_len = new_len;
    }
    __syncthreads();

    if (warp == kMoveGroups * GW) {
        // ---------------- producer ----------------
        if (lane != 0) return;
        uint32_t issued = 0, pub = 0, ends = 0, idle = 0;
        bool done = false;
        unsigned long long next = atomicAdd(ticket, 1ull);
        while (true) {
            bool prog = false;
            // Raise the staged flags of landed copies, in issue order.
            while (pub < issued) {
                const int s = int(pub % S);
                if (!mbar_test_wait(&full[s], (pub / S) & 1u)) break;
                const uint32_t t = s_tile[s];
                if (t < ntiles) st_relaxed(&staged[t], tag);
                ++pub;
                prog = true;
            }
            if (s_abort) break;
            if (ends < uint32_t(kMoveGroups)) {
                const uint32_t p = issued;
                const int s = int(p % S);
                // A stage is free once its previous position is published and consumed.
                const bool free = p < uint32_t(S) || (pub + S > p && mbar_test_wait(&empty[s], ((p / S) - 1u) & 1u));
                if (free) {
                    fence_proxy_async_smem();  // the consumers' generic reads of the stage come first
                    const uint32_t t = done ? ntiles : uint32_t(min(next, (unsigned long long)ntiles));
                    s_tile[s] = t;
                    if (t < ntiles) {
                        next = atomicAdd(ticket, 1ull);  // prefetch: used at the next issue
                        const uint32_t base = t * TILE;
                        const uint32_t items = min(TILE, n - base);
                        const uint32_t bulk = (items * W) & ~15u;
                        mbar_arrive_expect_tx(&full[s], bulk + BW * 4 + 16);
                        if (bulk) tma_load_1d(stage + size_t(s) * TILE, data + size_t(base) * W, bulk, &full[s]);
                        tma_load_1d(sbits + s * BW, bits + size_t(t) * BW, BW * 4, &full[s]);
                        tma_load_1d(&srec[s], recs + t, 16, &full[s]);
                    } else {
                        done = true;
                        ++ends;
                        mbar_arrive(&full[s]);  // end marker: completes the phase with no bytes
                    }
                    ++issued;
                    prog = true;
                }
            } else if (pub == issued) {
                break;
            }
            if (prog) {
                idle = 0;
            } else if (++idle > spin_limit) {
                s_abort = 1u;
                atomicOr(status, ST_TIMEOUT);
                break;
            }
        }
        // Never leave with copies in flight into this CTA's shared memory.
        for (; pub < issued; ++pub) {
            uint32_t it = 0;
            while (!mbar_test_wait(&full[pub % S], (pub / S) & 1u) && ++it <= spin_limit) {
            }
        }
        return;
    }

    // ---------------- consumers ----------------
    const int g = warp / GW, gw = warp % GW;
    const int gt = threadIdx.x - g * kGroupThreads;
    const uint32_t bar_id = 1u + uint32_t(g);
    const uint32_t lt = lanemask_lt();
    for (uint32_t p = uint32_t(g);; p += kMoveGroups) {
        const int s = int(p % S);
        const uint32_t par = (p / S) & 1u;
        // One thread waits (bounded) for the stage; the group learns the outcome at the barrier.
        if (gt == 0) {
            uint32_t it = 0;
            bool ok = true;
            while (!mbar_try_wait(&full[s], par)) {
                if (s_abort || ++it > spin_limit) {
                    ok = false;
                    break;
                }
            }
            if (!ok && !s_abort) {
                s_abort = 1u;
                atomicOr(status, ST_TIMEOUT);
            }
            s_go[g][0] = ok ? 1u : 0u;
        }
        named_bar(bar_id, kGroupThreads);
        if (!s_go[g][0]) break;
        mbar_try_wait(&full[s], par);  // completed: acquires the copied bytes for this thread
        const uint32_t t = s_tile[s];
        if (t >= ntiles) break;
        const uint32_t base = t * TILE;
        const uint32_t items = min(TILE, n - base);
        const uint4 rec = srec[s];
        const uint32_t off = rec.x, total = rec.y;
        T* st = stage + size_t(s) * TILE;
        // The ragged end of the last tile (fewer than 16 bytes) comes through plain loads.
        const uint32_t bulk_items = ((items * W) & ~15u) / W;
        for (uint32_t q = bulk_items + uint32_t(gt); q < items; q += kGroupThreads) st[q] = A[base + q];
        // Keep word of round `lane` of this warp (bits past n are not items).
        uint32_t kw = 0u;
        if (lane < R) {
            const uint32_t wi = uint32_t(gw) * R + uint32_t(lane);
            const uint32_t first = base + wi * 32u;
            const uint32_t valid = first >= n ? 0u : (n - first >= 32u ? 0xffffffffu : (1u << (n - first)) - 1u);
            kw = ~sbits[s * BW + wi] & valid;
            bits[size_t(t) * BW + wi] = 0u;  // leave the removal map zero for the next call
        }
        const uint32_t c = __popc(kw);
        const uint32_t inc = warp_inclusive_scan(c);
        if (lane == 31) s_wtot[g][gw] = inc;
        // Wait for the (at most two) tiles whose input this tile's output overlaps.
        if (gw == 0) {
            if (lane < 2 && total > 0) {
                const uint32_t u = off / TILE + uint32_t(lane);
                if (u <= (off + total - 1u) / TILE && u < t) {
                    uint32_t it = 0;
                    while (ld_acquire(&staged[u]) != tag) {
                        if (s_abort || ++it > spin_limit) {
                            if (!s_abort) atomicOr(status, ST_TIMEOUT);
                            s_abort = 1u;
                            break;
                        }
                    }
                }
            }
            __syncwarp();
            if (lane == 0) s_go[g][1] = s_abort ? 0u : 1u;
        }
        named_bar(bar_id, kGroupThreads);
        if (!s_go[g][1]) break;
        uint32_t wpre = 0;
#pragma unroll
        for (int q = 0; q < GW; ++q) wpre += q < gw ? s_wtot[g][q] : 0u;
        const uint32_t excl = inc - c;
        const T* src = st + size_t(gw) * PER_WARP;
        const uint32_t dst0 = off + wpre;
#pragma unroll 8
        for (int j = 0; j < R; ++j) {
            const uint32_t km = __shfl_sync(0xffffffffu, kw, j);
            const uint32_t ej = __shfl_sync(0xffffffffu, excl, j);
            if ((km >> lane) & 1u) A[dst0 + ej + __popc(km & lt)] = src[j * 32 + lane];
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

using MoveFn = void (*)(uint8_t*, uint32_t, uint32_t, uint32_t*, const uint32_t*, uint32_t*, unsigned long long*,
                        uint32_t, uint32_t*, uint32_t, unsigned long long*, uint32_t, unsigned long long*, uint32_t);
using MoveWsFn = void (*)(uint8_t*, uint32_t, uint32_t, uint32_t*, const uint4*, uint32_t*, unsigned long long*,
                          uint32_t, uint32_t*, uint32_t, unsigned long long*, uint32_t);

// 32 KB of payload per tile for every width.
static int part_items(int w) { return w == 4 ? 16 : w == 8 ? 8 : w == 16 ? 4 : 2; }
static MoveFn move_fn(int w) {
    switch (w) {
        case 4: return partition_move_kernel<4, 16>;
        case 8: return partition_move_kernel<8, 8>;
        case 16: return partition_move_kernel<16, 4>;
        default: return partition_move_kernel<32, 2>;
    }
}
static MoveWsFn move_ws_fn(int w, size_t* smem) {
    switch (w) {
        case 4: *smem = move_smem_bytes<4>(); return partition_move_ws_kernel<4>;
        case 8: *smem = move_smem_bytes<8>(); return partition_move_ws_kernel<8>;
        case 16: *smem = move_smem_bytes<16>(); return partition_move_ws_kernel<16>;
        default: *smem = move_smem_bytes<32>(); return partition_move_ws_kernel<32>;
    }
}

int launch_partition(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx, uint32_t k,
                     uint32_t flags, cudaStream_t s, LaunchInfo* info) {
    const int items = part_items(int(w));
    const uint32_t tile = uint32_t(kPartBlock * items);  // == kTileBytes / w for every width
    const uint32_t ntiles = (n + tile - 1) / tile;
    // The bit map is padded to whole tiles: the pipelined move copies a tile's words in one piece.
    int st = ensure_partition(ctx, size_t(ntiles) * tile, ntiles);
    if (st != RZ_OK) return st;
    st = reset_if_dirty(ctx, s);
    if (st != RZ_OK) return st;
    const bool validate = (flags & RZ_VALIDATE) != 0;
    // Scratch layout in tile_state: the ticket on its own 128-byte line, then staged, kept and
    // offset as 32-bit arrays of ntiles rounded up to a multiple of 4, then the 16-byte records.
    // Ticket and staged flags are cleared by one memset per call (which keeps the call correct
    // when it is replayed from a CUDA graph).
    const uint32_t ntp = (ntiles + 3u) & ~3u;
    unsigned long long* ticket = ctx->ws.tile_state;
    uint32_t* staged = reinterpret_cast<uint32_t*>(ctx->ws.tile_state + 16);
    uint32_t* kept = staged + ntp;
    uint32_t* offset = kept + ntp;
    uint4* recs = reinterpret_cast<uint4*>(offset + ntp);
    const uint32_t tag = 1u;
    RZ_CUDA_TRY(ctx, cudaMemsetAsync(ticket, 0, 128 + size_t(ntiles) * 4, s));
    const int mgrid = std::max(1, std::min<int>(ctx->sms * 8, int((k + 255) / 256)));
    partition_mark_kernel<<<mgrid, 256, 0, s>>>(idx, k, n, ctx->ws.part_bits, ctx->ws.status, validate ? 1u : 0u);
    const int cgrid = std::max(1, std::min<int>(ctx->sms * 8, int((ntiles + 7) / 8)));
    switch (w) {
        case 4: partition_count_kernel<kTileBytes / 4 / 32><<<cgrid, 256, 0, s>>>(ctx->ws.part_bits, n, ntiles, kept); break;
        case 8: partition_count_kernel<kTileBytes / 8 / 32><<<cgrid, 256, 0, s>>>(ctx->ws.part_bits, n, ntiles, kept); break;
        case 16: partition_count_kernel<kTileBytes / 16 / 32><<<cgrid, 256, 0, s>>>(ctx->ws.part_bits, n, ntiles, kept); break;
        default: partition_count_kernel<kTileBytes / 32 / 32><<<cgrid, 256, 0, s>>>(ctx->ws.part_bits, n, ntiles, kept); break;
    }
    // Function attributes belong to a device: one bit per device (first 64 devices).
    static std::atomic<uint64_t> scan_attr{0};
    const uint64_t dev_bit = 1ull << (ctx->device & 63);
    if (!(scan_attr.load() & dev_bit)) {
        RZ_CUDA_TRY(ctx, cudaFuncSetAttribute((const void*)partition_scan_kernel,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize, int(kScanSmem)));
        scan_attr.fetch_or(dev_bit);
    }
    partition_scan_kernel<<<1, 1024, kScanSmem, s>>>(kept, ntiles, offset, recs);
    int grid = int(ntiles), block = kPartBlock;
    if ((reinterpret_cast<uintptr_t>(data) & 15u) == 0 && !ctx->ws.stamps_on) {
        size_t smem = 0;
        MoveWsFn f = move_ws_fn(int(w), &smem);
        static std::atomic<uint64_t> attr_set[4];
        const int wi = w == 4 ? 0 : w == 8 ? 1 : w == 16 ? 2 : 3;
        if (!(attr_set[wi].load() & dev_bit)) {
            RZ_CUDA_TRY(ctx, cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
            attr_set[wi].fetch_or(dev_bit);
        }
        grid = std::max(1, std::min<int>(ctx->sms, int(ntiles)));
        block = kMoveBlock;
        f<<<grid, kMoveBlock, smem, s>>>(static_cast<uint8_t*>(data), n, ntiles, ctx->ws.part_bits, recs, staged,
                                         ticket, tag, ctx->ws.status, kSpinLimit, ctx->ws.dev_len, n - k);
    } else {
        const uint32_t stride = std::max<uint32_t>(1u, (ntiles + kMaxGrid - 1) / kMaxGrid);
        move_fn(int(w))<<<ntiles, kPartBlock, 0, s>>>(
            static_cast<uint8_t*>(data), n, ntiles, ctx->ws.part_bits, offset, staged, ticket, tag, ctx->ws.status,
            kSpinLimit, ctx->ws.dev_len, n - k, ctx->ws.stamps_on ? ctx->ws.stamps : nullptr, stride);
        grid = std::min<int>(int(ntiles), kMaxGrid);
    }
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    if (info) {
        info->grid = grid;
        info->block = block;
        info->items = items;
        info->launches += 4;  // mark, count, scan, move (the ticket memset runs on the copy engine)
    }
    return RZ_OK;
}

}  // namespace rz
