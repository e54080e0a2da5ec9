// rz_keep.cu -- preserve-list compaction: data[0..m) = (old) data[keep[0..m)], O(m) work.
//
// The inverse form of removal that the paper names as future work: when the kept items are fewer
// than the removed ones, gathering them costs m random reads instead of the n - m moves a removal
// would make. In place in two steps on the caller's stream: a gather kernel reads every kept item
// into context scratch (the reads may come from any position, including [0, m), so nothing is
// written to the payload while they run), then one device copy puts the m items at the front.
// An entry >= n is skipped (its slot keeps its own item) and sets ST_RANGE.
#include <algorithm>

#include "rz_common.cuh"
#include "rz_internal.h"

namespace rz {

constexpr int kKeepIpt = 4;  // items per thread per step, all loads issued before any store

template <int W>
__global__ void __launch_bounds__(256) keep_gather_kernel(const uint8_t* __restrict__ data, uint32_t n,
                                                          const uint32_t* __restrict__ keep, uint32_t m,
                                                          uint8_t* __restrict__ stage, uint32_t* status) {
    using T = typename Payload<W>::T;
    const T* A = reinterpret_cast<const T*>(data);
    T* S = reinterpret_cast<T*>(stage);
    const uint32_t stride = gridDim.x * blockDim.x * kKeepIpt;
    for (uint32_t base = blockIdx.x * blockDim.x * kKeepIpt + threadIdx.x; base < m; base += stride) {
        uint32_t r[kKeepIpt];
        T v[kKeepIpt];
#pragma unroll
        for (int q = 0; q < kKeepIpt; ++q) {
            const uint32_t j = base + uint32_t(q) * blockDim.x;
            r[q] = j < m ? __ldg(&keep[j]) : 0u;
        }
#pragma unroll
        for (int q = 0; q < kKeepIpt; ++q) {
            const uint32_t j = base + uint32_t(q) * blockDim.x;
            if (j < m) {
                if (r[q] < n) {
                    v[q] = A[r[q]];
                } else {
                    v[q] = A[j];  // out of range: the slot keeps its own item
                    atomicOr(status, ST_RANGE);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < kKeepIpt; ++q) {
            const uint32_t j = base + uint32_t(q) * blockDim.x;
            if (j < m) S[j] = v[q];
        }
    }
}

int launch_keep(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* keep, uint32_t m, void* stage,
                cudaStream_t s) {
    if (m == 0) return RZ_OK;
    const long per_cta = 256L * kKeepIpt;
    const int grid = int(std::min<long>(long(ctx->sms) * 8, (long(m) + per_cta - 1) / per_cta));
    const uint8_t* d = static_cast<const uint8_t*>(data);
    uint8_t* st = static_cast<uint8_t*>(stage);
    switch (w) {
        case 4: keep_gather_kernel<4><<<grid, 256, 0, s>>>(d, n, keep, m, st, ctx->ws.status); break;
        case 8: keep_gather_kernel<8><<<grid, 256, 0, s>>>(d, n, keep, m, st, ctx->ws.status); break;
        case 16: keep_gather_kernel<16><<<grid, 256, 0, s>>>(d, n, keep, m, st, ctx->ws.status); break;
        default: keep_gather_kernel<32><<<grid, 256, 0, s>>>(d, n, keep, m, st, ctx->ws.status); break;
    }
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    RZ_CUDA_TRY(ctx, cudaMemcpyAsync(data, stage, size_t(m) * w, cudaMemcpyDeviceToDevice, s));
    return RZ_OK;
}

}  // namespace rz
