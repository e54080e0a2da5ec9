// rz_comparators.cu -- the reference's O(n) GPU comparator, for the benchmark only.
//
// The reference times Redzone against a mark-then-compact pass built on Thrust
// (Thrust_remove.hxx:15-17 and DataStruct.hxx:11-18): every removed slot is overwritten with the
// marker -1, then thrust::remove(thrust::device, list, list + n, -1) compacts the list, stably.
// rz_test_thrust_remove runs that same library call on the caller's int list, so the benchmark
// can time it beside this library's own O(n) partition (rz_partition) and the O(k) removal. It is
// a measurement aid: no removal path of this library calls it, and like the reference's it
// assumes that -1 occurs in the list only where the marks put it.
#include <thrust/execution_policy.h>
#include <thrust/remove.h>

#include "rz_internal.h"

namespace rz {

__global__ void thrust_mark_kernel(int32_t* __restrict__ list, uint32_t n, const uint32_t* __restrict__ idx,
                                   uint32_t k) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
        const uint32_t q = __ldg(&idx[i]);
        if (q < n) list[q] = -1;
    }
}

}  // namespace rz

extern "C" int rz_test_thrust_remove(rz_ctx* ctx, int32_t* d_list, int64_t n, const uint32_t* d_idx, int64_t k,
                                     int64_t* new_len, rz_stream_t stream) {
    using namespace rz;
    if (!ctx || n < 0 || k < 0 || k > n || (n > 0 && !d_list) || (k > 0 && !d_idx)) return RZ_ERR_INVALID_ARG;
    if (n >= (int64_t(1) << 31)) return RZ_ERR_UNSUPPORTED;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (k > 0) {
        thrust_mark_kernel<<<ctx->sms * 4, 256, 0, s>>>(d_list, uint32_t(n), d_idx, uint32_t(k));
        RZ_CUDA_TRY(ctx, cudaGetLastError());
    }
    int32_t* end = d_list + n;
    try {
        end = thrust::remove(thrust::cuda::par.on(s), d_list, d_list + n, int32_t(-1));
    } catch (...) {
        ctx->last_cuda_error = "thrust::remove failed";
        return RZ_ERR_CUDA;
    }
    if (new_len) *new_len = int64_t(end - d_list);
    return RZ_OK;
}
