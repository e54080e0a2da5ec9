// rz_common.cuh -- device-side building blocks shared by every Redzone kernel in this library.
//
// Contents: payload types for the four supported element widths, acquire/release memory
// operations in inline PTX, a self-resetting generation barrier with a bounded wait (the
// replacement for cg::this_grid().sync() and BlockStorage_t::Wait(), redzone.hxx:56-80 and
// :707,846,912,935,940), and a few warp/block scan helpers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "rz_internal.h"

namespace rz {

// Device status bits, OR-ed into a caller-visible status word. The host maps them to rz_status.
enum : uint32_t {
    ST_DUPLICATE = 1u << 0,
    ST_RANGE = 1u << 1,
    ST_TIMEOUT = 1u << 2,
    ST_INCONSISTENT = 1u << 3,  // orphan counts disagree (only possible with invalid input)
};

// 32-byte payload (u64 key + three u64 words in the streaming table; 8 x u32 otherwise).
struct alignas(16) u32x8 {
    uint4 a, b;
};

template <int W> struct Payload;
template <> struct Payload<4> { using T = uint32_t; };
template <> struct Payload<8> { using T = uint2; };
template <> struct Payload<16> { using T = uint4; };
template <> struct Payload<32> { using T = u32x8; };

// ---- memory-ordering primitives (gpu scope) ------------------------------------------------
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t atom_add_acq_rel(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---- generation barrier -----------------------------------------------------------------------
// {count, gen} live in library scratch. Each participating CTA reads `gen`, then arrives on
// `count`; the last arriver resets `count` and publishes gen+1 with release semantics. Because
// the last arriver always leaves count at zero, the pair needs no per-call reset and is safe
// under CUDA-graph replay. A CTA that passes `wait=false` arrives without waiting (used when it
// has no work after the barrier). Every wait is bounded by `spin_limit` polls; on expiry the CTA
// records ST_TIMEOUT and the function returns false, so no kernel ever hangs.
__device__ __forceinline__ bool grid_barrier(GridSync* gs, uint32_t expected, bool wait,
                                             uint32_t* status, uint32_t spin_limit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const uint32_t g0 = ld_acquire(&gs->gen);
        const uint32_t old = atom_add_acq_rel(&gs->count, 1u);
        if (old == expected - 1) {
            atomicExch(&gs->count, 0u);
            __threadfence();
            st_release(&gs->gen, g0 + 1u);
        } else if (wait) {
            uint32_t it = 0;
            uint32_t ns = 32;
            while (ld_acquire(&gs->gen) == g0) {
                if (++it > spin_limit) {
                    ok = 0;
                    atomicOr(status, ST_TIMEOUT);
                    break;
                }
                __nanosleep(ns);
                if (ns < 256) ns <<= 1;
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ---- scans ------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += u;
    }
    return v;
}

// Exclusive scan of one value per thread over the whole block (blockDim.x <= 1024, multiple of
// 32). `scratch` must hold 33 words. Returns the exclusive prefix; *total gets the block sum.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* scratch, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t inc = warp_inclusive_scan(v);
    __syncthreads();
    if (lane == 31) scratch[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < nw ? scratch[lane] : 0u;
        const uint32_t winc = warp_inclusive_scan(w);
        if (lane < nw) scratch[lane] = winc - w;
        if (lane == 31) scratch[32] = winc;
    }
    __syncthreads();
    const uint32_t r = scratch[warp] + inc - v;
    *total = scratch[32];
    return r;
}

// Exclusive scan, in place, of cnt[0..m) in shared memory by the whole block; cnt[m] receives
// the total. `scratch` must hold 33 words.
__device__ __forceinline__ void block_scan_array(uint32_t* cnt, int m, uint32_t* scratch) {
    const int B = blockDim.x;
    const int per = (m + B - 1) / B;
    const int lo = threadIdx.x * per;
    const int hi = min(lo + per, m);
    uint32_t s = 0;
    for (int c = lo; c < hi; ++c) s += cnt[c];
    uint32_t total;
    uint32_t run = block_exclusive_scan(s, scratch, &total);
    __syncthreads();
    for (int c = lo; c < hi; ++c) {
        const uint32_t x = cnt[c];
        cnt[c] = run;
        run += x;
    }
    if (threadIdx.x == 0) cnt[m] = total;
    __syncthreads();
}

// Largest c in [0, m) with pfx[c] <= j, where pfx is a non-decreasing exclusive prefix of
// length m+1 and j < pfx[m]. Empty segments (pfx[c] == pfx[c+1]) are skipped.
__device__ __forceinline__ int owner_of_rank(const uint32_t* pfx, int m, uint32_t j) {
    int lo = 0, hi = m;  // invariant: pfx[lo] <= j < pfx[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pfx[mid] <= j) lo = mid; else hi = mid;
    }
    return lo;
}

}  // namespace rz
