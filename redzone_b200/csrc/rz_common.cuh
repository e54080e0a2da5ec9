// rz_common.cuh -- device-side building blocks shared by every Redzone kernel in this library.
//
// Contents: payload types for the four supported element widths, acquire/release memory
// operations in inline PTX, epoch-tagged arrival flags with bounded waits (the replacement for
// cg::this_grid().sync() and BlockStorage_t::Wait(), redzone.hxx:56-80 and
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
    ST_CAPACITY = 1u << 4,      // a produced list outgrew its capacity (nothing was moved)
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

// ---- L2 eviction priorities (createpolicy + L2::cache_hint) ----------------------------------
// Read-once streams (a list's index entries and tail items on their last read) go in as
// evict-first, hole stores as evict-last: partially written hole lines then stay in L2 while
// more writes to the same sectors may arrive, instead of being pushed out by the stream.
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint32_t ld_hint(const uint32_t* a, uint64_t pol) {
    uint32_t v;
    asm volatile("ld.global.nc.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ uint2 ld_hint(const uint2* a, uint64_t pol) {
    uint2 v;
    asm volatile("ld.global.nc.L2::cache_hint.v2.b32 {%0, %1}, [%2], %3;" : "=r"(v.x), "=r"(v.y) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ uint4 ld_hint(const uint4* a, uint64_t pol) {
    uint4 v;
    asm volatile("ld.global.nc.L2::cache_hint.v4.b32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ u32x8 ld_hint(const u32x8* a, uint64_t pol) {
    u32x8 v;
    v.a = ld_hint(&a->a, pol);
    v.b = ld_hint(&a->b, pol);
    return v;
}
__device__ __forceinline__ void st_hint(uint32_t* a, uint32_t v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.b32 [%0], %1, %2;" ::"l"(a), "r"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_hint(uint2* a, uint2 v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.v2.b32 [%0], {%1, %2}, %3;" ::"l"(a), "r"(v.x), "r"(v.y), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_hint(uint4* a, uint4 v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.v4.b32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(a), "r"(v.x), "r"(v.y),
                 "r"(v.z), "r"(v.w), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_hint(u32x8* a, const u32x8& v, uint64_t pol) {
    st_hint(&a->a, v.a, pol);
    st_hint(&a->b, v.b, pol);
}

// ---- epoch-tagged arrival flags --------------------------------------------------------------
// The grid schedule's barriers. Each call reads an epoch E once at kernel start and tags every
// arrival with E+1; a CTA arrives with one release store to its own slot and waits by polling the
// other CTAs' slots for the tag. Flags from earlier calls carry older tags, so nothing is reset
// between calls (graph replays included). CTA 0 advances the stored epoch once every CTA has
// arrived at the first barrier, i.e. after every CTA of this call has read it.
__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Record a phase timestamp for this CTA when tracing is enabled (params carry `stamps`).
#define RZ_STAMP(p, slot)                                                                          \
    do {                                                                                           \
        if ((p).stamps && threadIdx.x == 0)                                                        \
            (p).stamps[blockIdx.x * ::rz::kStampsPerCta + (slot)] = ::rz::globaltimer();           \
    } while (0)

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
// Named barrier over `count` threads (a multiple of 32); id 0 is __syncthreads().
__device__ __forceinline__ void named_bar(uint32_t id, uint32_t count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Arrive: the barrier orders every thread's prior writes before thread 0's release store.
__device__ __forceinline__ void flag_arrive(uint32_t* flags, uint32_t slot, uint32_t tag) {
    __syncthreads();
    if (threadIdx.x == 0) st_release(&flags[slot], tag);
}

// Wait until flags[0..G) all hold `tag`; bounded by spin_limit polls per slot. The polls are
// relaxed and back-to-back (each is an L2 round trip; __nanosleep backoff was measured to add
// microseconds of wake-up latency per barrier on B200); one acquire fence by thread 0, ordered
// before the rest of the block by the closing barrier, makes the other CTAs' released writes
// visible. Returns false (and records ST_TIMEOUT) if some slot never gets there.
__device__ __forceinline__ bool flag_wait_all(const uint32_t* flags, uint32_t G, uint32_t tag, uint32_t* status,
                                              uint32_t spin_limit) {
    int ok = 1;
    for (uint32_t c = threadIdx.x; c < G && ok; c += blockDim.x) {
        uint32_t it = 0;
        while (ld_relaxed(&flags[c]) != tag) {
            if (++it > spin_limit) {
                ok = 0;
                break;
            }
        }
    }
    const int all = __syncthreads_and(ok);
    if (!all) {
        if (threadIdx.x == 0) atomicOr(status, ST_TIMEOUT);
        return false;
    }
    if (threadIdx.x == 0) fence_acq_rel_gpu();
    __syncthreads();
    return true;
}

// Prefetch the 128-byte lines that start inside [p, p + bytes) into L2, spread over the block's
// threads (every prefetched address lies inside the range; the first partial line is left to the
// demand load). A prefetch is not a memory access a fence waits for, so issuing it before a
// barrier costs nothing there.
__device__ __forceinline__ void prefetch_l2(const void* p, size_t bytes) {
    const uintptr_t b = reinterpret_cast<uintptr_t>(p);
    const uintptr_t lo = (b + 127) & ~uintptr_t(127);
    const uintptr_t hi = b + bytes;
    for (uintptr_t a = lo + uintptr_t(threadIdx.x) * 128; a < hi; a += uintptr_t(blockDim.x) * 128)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
}

// ---- mbarrier + 1-D TMA bulk copies (each into its own CTA only) ---------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Arrive once and add `bytes` to the transaction count the current phase waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// Plain arrive (no transaction bytes).
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Non-blocking test of a phase (never suspends the thread).
__device__ __forceinline__ bool mbar_test_wait(unsigned long long* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Global -> shared bulk copy completing on `bar`. Both addresses 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void tma_load_1d(void* dst_smem, const void* src, uint32_t bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst_smem)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
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
