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

// Kept items of each tile (one warp per tile, grid-stride over tiles).
__global__ void partition_count_kernel(const uint32_t* __restrict__ bits, uint32_t n, uint32_t tile_items,
                                       uint32_t ntiles, uint32_t* __restrict__ kept) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t wpt = tile_items >> 5;  // bitmap words per tile
    for (uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < ntiles; t += warps) {
        const uint32_t w0 = t * wpt;
        uint32_t removed = 0;
        for (uint32_t q = lane; q < wpt; q += 32) {
            const uint32_t wi = w0 + q;
            const uint32_t first = wi << 5;
            if (first >= n) break;
            uint32_t word = __ldg(&bits[wi]);
            const uint32_t valid = n - first;
            if (valid < 32) word &= (1u << valid) - 1u;  // bits past n are not items
            removed += __popc(word);
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) removed += __shfl_down_sync(0xffffffffu, removed, d);
        if (lane == 0) {
            const uint32_t items = min(tile_items, n - t * tile_items);
            kept[t] = items - removed;
        }
    }
}

// Exclusive scan of kept[0..ntiles) into offset[0..ntiles), one CTA of 1024 threads.
__global__ void __launch_bounds__(1024) partition_scan_kernel(const uint32_t* __restrict__ kept, uint32_t ntiles,
                                                              uint32_t* __restrict__ offset) {
    __shared__ uint32_t scratch[33];
    const uint32_t B = blockDim.x;
    const uint32_t per = (ntiles + B - 1) / B;
    const uint32_t lo = threadIdx.x * per, hi = min(lo + per, ntiles);
    uint32_t s = 0;
    for (uint32_t t = lo; t < hi; ++t) s += kept[t];
    uint32_t total;
    uint32_t run = block_exclusive_scan(s, scratch, &total);
    for (uint32_t t = lo; t < hi; ++t) {
        offset[t] = run;
        run += kept[t];
    }
}

// One tile per CTA, taken in ticket order.
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
// Move step, pipelined: persistent CTAs (one per SM), kStages tiles of 32 KB in flight per CTA.
// Thread 0 takes tickets and issues 1-D TMA bulk copies (tile payload + its bitmap words) into a
// ring of shared-memory stages; a tile's staged flag is raised as soon as its copy has landed
// (also for tiles still waiting in the ring), so successors waiting on it are not held up by this
// CTA's processing order. The other threads turn the staged bitmap into ranks and write the kept
// items out while the next tiles' copies are in flight. Requires a 16-byte-aligned payload.
// ------------------------------------------------------------------------------------------------
constexpr int kStages = 4;
constexpr uint32_t kTileBytes = 32768;
constexpr int kTmaBlock = 256;

template <int W>
__global__ void __launch_bounds__(kTmaBlock, 1) partition_move_tma_kernel(
    uint8_t* data, uint32_t n, uint32_t ntiles, uint32_t* __restrict__ bits, const uint32_t* __restrict__ offset,
    uint32_t* staged, unsigned long long* ticket, uint32_t tag, uint32_t* status, uint32_t spin_limit,
    unsigned long long* dev_len, uint32_t new_len) {
    using T = typename Payload<W>::T;
    constexpr uint32_t TILE = kTileBytes / W;   // items per tile
    constexpr uint32_t BW = TILE / 32;          // bitmap words per tile
    constexpr int B = kTmaBlock, NW = B / 32;
    constexpr int ROUNDS = TILE / B;            // items per thread per tile
    T* A = reinterpret_cast<T*>(data);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

    extern __shared__ __align__(128) uint8_t smem[];
    T* stage = reinterpret_cast<T*>(smem);                                       // [kStages][TILE]
    uint32_t* sbits = reinterpret_cast<uint32_t*>(smem + kStages * kTileBytes);  // [kStages][BW]
    __shared__ __align__(8) unsigned long long bars[kStages];
    __shared__ uint32_t s_tile[kStages];
    __shared__ uint32_t s_cnt[ROUNDS * NW + 1];
    if (blockIdx.x == 0 && threadIdx.x == 0 && dev_len) *dev_len = new_len;

    uint32_t published = 0;  // thread 0: stages whose staged flag is raised for the current tile
    auto issue = [&](int s) {  // thread 0: refill stage s with the next ticket
        const uint32_t t = uint32_t(atomicAdd(ticket, 1ull));
        s_tile[s] = t;
        published &= ~(1u << s);
        if (t >= ntiles) return;
        const uint32_t base = t * TILE;
        const uint32_t items = min(TILE, n - base);
        const uint32_t bulk = (items * W) & ~15u;
        mbar_arrive_expect_tx(&bars[s], bulk + BW * 4);
        if (bulk) tma_load_1d(stage + size_t(s) * TILE, data + size_t(base) * W, bulk, &bars[s]);
        tma_load_1d(sbits + s * BW, bits + size_t(t) * BW, BW * 4, &bars[s]);
    };
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
        for (int s = 0; s < kStages; ++s) issue(s);
    }
    __syncthreads();

    uint32_t parity = 0;  // bit s: phase parity of stage s
    int timed_out = 0;
    for (int s = 0;; s = (s + 1 == kStages) ? 0 : s + 1) {
        const uint32_t t = s_tile[s];
        if (t >= ntiles) break;  // tickets grow along the ring, so every later stage is empty too
        const uint32_t base = t * TILE;
        const uint32_t items = min(TILE, n - base);
        // Wait for this stage's copy (bounded; a copy of valid memory always lands).
        {
            uint32_t it = 0;
            while (!mbar_try_wait(&bars[s], (parity >> s) & 1u)) {
                if (++it > spin_limit) {
                    timed_out = 1;
                    break;
                }
            }
            parity ^= 1u << s;
        }
        T* st = stage + size_t(s) * TILE;
        const uint32_t* sb = sbits + s * BW;
        // The ragged end of the last tile (fewer than 16 bytes) comes through plain loads.
        const uint32_t bulk_items = ((items * W) & ~15u) / W;
        for (uint32_t q = bulk_items + threadIdx.x; q < items; q += B) st[q] = A[base + q];
        __syncthreads();
        if (threadIdx.x == 0) {
            // This tile's input is read; so is that of every other stage whose copy has landed,
            // except a last tile with a ragged end (read by plain loads when it is processed).
            if (!(published & (1u << s))) st_release(&staged[t], tag);
            const bool last_ragged = ((n - (ntiles - 1) * TILE) * W) % 16 != 0;
            for (int o = 1; o < kStages; ++o) {
                const int so = (s + o) % kStages;
                const uint32_t to = s_tile[so];
                if (to >= ntiles || (published & (1u << so))) continue;
                if (last_ragged && to == ntiles - 1) continue;
                if (mbar_try_wait(&bars[so], (parity >> so) & 1u)) {
                    st_release(&staged[to], tag);
                    published |= 1u << so;
                }
            }
        }
        // Ranks of the kept items, round-major (round j covers items j*B .. j*B+B-1).
        uint32_t km[ROUNDS];
#pragma unroll
        for (int j = 0; j < ROUNDS; ++j) {
            const uint32_t q = uint32_t(j) * B + threadIdx.x;
            const bool keep = q < items && ((sb[q >> 5] >> (q & 31u)) & 1u) == 0u;
            km[j] = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) s_cnt[j * NW + warp] = __popc(km[j]);
        }
        // Leave the removal map zero for the next call (coalesced: one word per thread).
        for (uint32_t q = threadIdx.x; q < BW; q += B)
            if (base + q * 32 < n) bits[size_t(t) * BW + q] = 0u;
        __syncthreads();
        const uint32_t off = __ldg(&offset[t]);
        if (warp == 0) {
            constexpr int E = ROUNDS * NW;
            constexpr int per = (E + 31) / 32;
            const int lo = lane * per, hi = min(lo + per, E);
            uint32_t sum = 0;
            for (int e = lo; e < hi; ++e) sum += s_cnt[e];
            const uint32_t inc = warp_inclusive_scan(sum);
            uint32_t run = inc - sum;
            for (int e = lo; e < hi; ++e) {
                const uint32_t x = s_cnt[e];
                s_cnt[e] = run;
                run += x;
            }
            const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
            // Wait for the (at most two) tiles whose input this tile's output overlaps.
            if (total > 0 && lane < 2) {
                const uint32_t u = off / TILE + uint32_t(lane);
                if (u <= (off + total - 1) / TILE && u < t) {
                    uint32_t it = 0;
                    while (ld_acquire(&staged[u]) != tag) {
                        if (++it > spin_limit) {
                            timed_out = 1;
                            break;
                        }
                    }
                }
            }
        }
        __syncthreads();
        const uint32_t lt = lanemask_lt();
#pragma unroll
        for (int j = 0; j < ROUNDS; ++j) {
            const uint32_t q = uint32_t(j) * B + threadIdx.x;
            if ((km[j] >> lane) & 1u) A[off + s_cnt[j * NW + warp] + __popc(km[j] & lt)] = st[q];
        }
        __syncthreads();  // stage s is consumed
        if (threadIdx.x == 0) {
            fence_proxy_async_smem();  // generic reads of the stage precede the next async write
            issue(s);
        }
        __syncthreads();
    }
    if (timed_out) atomicOr(status, ST_TIMEOUT);
}

using MoveFn = void (*)(uint8_t*, uint32_t, uint32_t, uint32_t*, const uint32_t*, uint32_t*, unsigned long long*,
                        uint32_t, uint32_t*, uint32_t, unsigned long long*, uint32_t, unsigned long long*, uint32_t);
using MoveTmaFn = void (*)(uint8_t*, uint32_t, uint32_t, uint32_t*, const uint32_t*, uint32_t*, unsigned long long*,
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
static MoveTmaFn move_tma_fn(int w) {
    switch (w) {
        case 4: return partition_move_tma_kernel<4>;
        case 8: return partition_move_tma_kernel<8>;
        case 16: return partition_move_tma_kernel<16>;
        default: return partition_move_tma_kernel<32>;
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
    // Scratch layout in tile_state: the ticket on its own 128-byte line, then staged[ntiles],
    // kept[ntiles] and offset[ntiles] as 32-bit arrays. Ticket and staged flags are cleared by
    // one memset per call (which keeps the call correct when it is replayed from a CUDA graph).
    unsigned long long* ticket = ctx->ws.tile_state;
    uint32_t* staged = reinterpret_cast<uint32_t*>(ctx->ws.tile_state + 16);
    uint32_t* kept = staged + ntiles;
    uint32_t* offset = kept + ntiles;
    const uint32_t tag = 1u;
    RZ_CUDA_TRY(ctx, cudaMemsetAsync(ticket, 0, 128 + size_t(ntiles) * 4, s));
    const int mgrid = std::max(1, std::min<int>(ctx->sms * 8, int((k + 255) / 256)));
    partition_mark_kernel<<<mgrid, 256, 0, s>>>(idx, k, n, ctx->ws.part_bits, ctx->ws.status, validate ? 1u : 0u);
    const int cgrid = std::max(1, std::min<int>(ctx->sms * 8, int((ntiles + 7) / 8)));
    partition_count_kernel<<<cgrid, 256, 0, s>>>(ctx->ws.part_bits, n, tile, ntiles, kept);
    partition_scan_kernel<<<1, 1024, 0, s>>>(kept, ntiles, offset);
    int grid = int(ntiles), block = kPartBlock;
    if ((reinterpret_cast<uintptr_t>(data) & 15u) == 0 && !ctx->ws.stamps_on) {
        MoveTmaFn f = move_tma_fn(int(w));
        const size_t smem = size_t(kStages) * kTileBytes + size_t(kStages) * (kTileBytes / w / 8);
        static bool attr_set[4] = {false, false, false, false};
        const int wi = w == 4 ? 0 : w == 8 ? 1 : w == 16 ? 2 : 3;
        if (!attr_set[wi]) {
            RZ_CUDA_TRY(ctx, cudaFuncSetAttribute((const void*)f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
            attr_set[wi] = true;
        }
        grid = std::max(1, std::min<int>(ctx->sms, int(ntiles)));
        block = kTmaBlock;
        f<<<grid, kTmaBlock, smem, s>>>(static_cast<uint8_t*>(data), n, ntiles, ctx->ws.part_bits, offset, staged,
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
