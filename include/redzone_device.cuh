// redzone_device.cuh -- device-side half of the producer API (rz_producer_* in redzone.h).
//
// A caller's CUDA kernel that decides which rows of a list to delete emits them here instead of
// writing its own index list; rz_remove_produced then removes them. Emitting also does the
// red-zone marking the removal would otherwise do by scanning the whole list (the paper's "mark
// during producer", p.14): a row that may fall in the red zone [n - k, n) -- any row >= n -
// capacity, since k <= capacity -- is also recorded as a candidate (slot, row) pair. For a list
// whose deletions are spread out, candidates are about capacity * k / n of the k rows.
//
//   __global__ void my_producer(rz_producer_view v, const Record* recs, uint32_t n) {
//       for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
//           rz_emit(v, i, should_delete(recs[i]));
//   }
//
// Contract: every row is emitted at most once per round and is < v.n. Any thread may call
// rz_emit, in any order; the list order is the order in which slots were taken, and the removal
// is canonical for that list.
#pragma once

#include <stdint.h>

#include "redzone.h"

// Emit `row` when `take` is true. Call it from every active lane of a warp together (lanes with
// nothing to delete pass take = false): one atomic per warp reserves the slots.
__device__ __forceinline__ void rz_emit(const rz_producer_view& v, uint32_t row, bool take) {
    const unsigned act = __activemask();
    const unsigned m = __ballot_sync(act, take);
    if (m == 0u) return;
    unsigned lane;
    asm("mov.u32 %0, %%laneid;" : "=r"(lane));
    const unsigned leader = unsigned(__ffs(m) - 1);
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&v.counts[0], uint32_t(__popc(m)));
    base = __shfl_sync(act, base, int(leader));
    if (!take) return;
    const uint32_t slot = base + uint32_t(__popc(m & ((1u << lane) - 1u)));
    if (slot < v.capacity) v.idx[slot] = row;  // beyond capacity the count alone records it
    if (row >= v.floor) {
        const uint32_t c = atomicAdd(&v.counts[1], 1u);
        if (c < v.cand_capacity) {
            v.cand[2 * size_t(c)] = slot;
            v.cand[2 * size_t(c) + 1] = row;
        }
    }
}
