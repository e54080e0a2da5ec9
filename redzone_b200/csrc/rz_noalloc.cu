// rz_noalloc.cu -- rz_remove_noalloc: single-list Redzone for callers that cannot allocate.
//
// Some callers cannot call cudaMalloc at all: code running inside a memory-pool budget that is
// already fully committed, allocator-free real-time paths that must not take the driver's
// allocation lock (or synchronise, as cudaFree does), plugin hosts that hand out device buffers
// but own every allocation themselves. rz_remove needs a context, and a context allocates its
// scratch (bitmap, orphan lists, barrier words) and grows it with k. This file gives those
// callers one entry point whose scratch is a fixed-size, file-scope device array instead: it
// allocates nothing, ever. The caller still passes the payload and the index list.
//
// Limits and rules of use:
//   * k <= kNoAllocMaxK (2^20) removals per call and n < 2^32 items; larger calls are rejected
//     with RZ_ERR_UNSUPPORTED before anything is launched.
//   * The array (kScratchWords * 4 bytes, about 8.4 MB) lives in every GPU that loads this
//     library, until the process exits.
//   * Set-up: the first call on a device, with that device current, looks up the array's device
//     address (cudaGetSymbolAddress) and caches it. Make that first call before any stream
//     capture on that device.
//   * The stream must belong to the current device (checked); a cudaDeviceReset discards the
//     array's address, so this library must not be used on a device after it was reset.
//   * All calls share the one array and it keeps the last call's contents. Each call clears, on
//     its stream, the parts that must start at zero (the red-zone bitmap words it uses and the
//     barrier words), so a call that ended early cannot leave state behind for the next one.
//     Two calls that overlap on the GPU (different streams without ordering) race on the array:
//     order them on one stream, or with events.
//   * Errors found on the device (an index >= n, a bounded wait that gave up, inconsistent
//     orphan counts) are ORed into a status word of the array that no call clears; the caller
//     reads and clears it with rz_noalloc_sync_status, which covers every call since its last use.
//   * Indices >= n are skipped safely (never used as addresses) and reported as above; duplicate
//     indices are the caller's responsibility, as with rz_remove without RZ_VALIDATE.
// The kernel is the grid-wide Redzone body of rz_single_kernel.cuh with its scratch pointers
// aimed into the array; results are bit-identical to rz_remove.
#include <algorithm>
#include <mutex>

#include "rz_common.cuh"
#include "rz_internal.h"
#include "rz_single_kernel.cuh"

namespace rz {
namespace {

constexpr uint32_t kNoAllocMaxK = 1u << 20;
constexpr int kNoAllocBlock = 256;
constexpr int kNoAllocItems = 4;
constexpr int kMaxDevices = 64;

// Word offsets of the regions inside the array (every region starts on a 256-byte boundary).
constexpr size_t kOffStatus = 0;                                   // 64 words
constexpr size_t kOffEpoch = 64;                                   // 64 words
constexpr size_t kOffArrive = 128;                                 // kMaxGrid words
constexpr size_t kOffCnt = kOffArrive + kMaxGrid;                  // 2*kMaxGrid u64 = 4*kMaxGrid words
constexpr size_t kOffBitmap = kOffCnt + 4 * size_t(kMaxGrid);      // kNoAllocMaxK/32 words
constexpr size_t kOffDlist = kOffBitmap + kNoAllocMaxK / 32;       // kNoAllocMaxK words
constexpr size_t kOffSlist = kOffDlist + kNoAllocMaxK;             // kNoAllocMaxK words
constexpr size_t kScratchWords = kOffSlist + kNoAllocMaxK + 64;
static_assert(kOffCnt % 64 == 0 && kOffBitmap % 64 == 0 && kOffDlist % 64 == 0 && kOffSlist % 64 == 0,
              "regions must stay 256-byte aligned");

}  // namespace

// The scratch. Host code must not use this name as an address (on the host it is only a
// stand-in for the symbol): the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kScratchWords];

template <int W>
__global__ void redzone_noalloc_kernel(const SingleParams p) {
    redzone_single_body<W, kNoAllocItems>(p);
}

namespace {

using NoAllocFn = void (*)(const SingleParams);

NoAllocFn noalloc_fn(uint32_t w) {
    switch (w) {
        case 4: return redzone_noalloc_kernel<4>;
        case 8: return redzone_noalloc_kernel<8>;
        case 16: return redzone_noalloc_kernel<16>;
        case 32: return redzone_noalloc_kernel<32>;
        default: return nullptr;
    }
}

struct DeviceSetup {
    uint32_t* scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int sms = 0;
};

std::mutex g_setup_mu;
DeviceSetup g_setup[kMaxDevices];

// Once per device, with that device current: resolve the array's device address.
cudaError_t setup_device(int dev, DeviceSetup* out) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    DeviceSetup& s = g_setup[dev];
    if (!s.scratch) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        s.sms = sms;
        s.scratch = static_cast<uint32_t*>(ptr);
    }
    *out = s;
    return cudaSuccess;
}

// The legacy and per-thread default streams (handles 0, 1, 2) belong to the current device.
bool stream_on_device(cudaStream_t s, int dev) {
    if (reinterpret_cast<uintptr_t>(s) <= 2) return true;
    int sdev = -1;
    if (cudaStreamGetDevice(s, &sdev) != cudaSuccess) return false;
    return sdev == dev;
}

}  // namespace
}  // namespace rz

extern "C" int rz_noalloc_sync_status(rz_stream_t stream) {
    using namespace rz;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return RZ_ERR_CUDA;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!stream_on_device(s, dev)) return RZ_ERR_INVALID_ARG;
    uint32_t* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        base = g_setup[dev].scratch;
    }
    if (!base) return cudaStreamSynchronize(s) == cudaSuccess ? RZ_OK : RZ_ERR_CUDA;  // no call on this device yet
    uint32_t bits = 0;  // pageable host word: the copy completes before the call returns
    if (cudaMemcpyAsync(&bits, base + kOffStatus, sizeof(bits), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return RZ_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return RZ_ERR_CUDA;
    if (bits) {
        if (cudaMemsetAsync(base + kOffStatus, 0, sizeof(uint32_t), s) != cudaSuccess) return RZ_ERR_CUDA;
        if (cudaStreamSynchronize(s) != cudaSuccess) return RZ_ERR_CUDA;
    }
    return map_status(bits);
}

extern "C" int rz_remove_noalloc(void* d_data, int64_t n, uint32_t elem_bytes, const uint32_t* d_idx, int64_t k,
                                 int64_t* new_len, rz_stream_t stream) {
    using namespace rz;
    if (n < 0 || k < 0 || k > n) return RZ_ERR_INVALID_ARG;
    if (elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16 && elem_bytes != 32) return RZ_ERR_INVALID_ARG;
    if (n >= (int64_t(1) << 32) || k > int64_t(kNoAllocMaxK)) return RZ_ERR_UNSUPPORTED;
    if (k > 0 && (!d_data || !d_idx)) return RZ_ERR_INVALID_ARG;
    const uintptr_t align = elem_bytes >= 16 ? 16 : elem_bytes;
    if (reinterpret_cast<uintptr_t>(d_data) % align || reinterpret_cast<uintptr_t>(d_idx) % 4)
        return RZ_ERR_INVALID_ARG;
    if (new_len) *new_len = n - k;
    if (k == 0 || k == n) return RZ_OK;  // nothing moves

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return RZ_ERR_CUDA;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!stream_on_device(s, dev)) return RZ_ERR_INVALID_ARG;
    DeviceSetup ds;
    if (setup_device(dev, &ds) != cudaSuccess) return RZ_ERR_CUDA;
    uint32_t* base = ds.scratch;

    // Clear what must start at zero: epoch, barrier words, and the bitmap words of k bits. The
    // status word is left alone: it collects device errors until rz_noalloc_sync_status reads it.
    if (cudaMemsetAsync(base + kOffEpoch, 0, (kOffBitmap - kOffEpoch) * 4, s) != cudaSuccess) return RZ_ERR_CUDA;
    if (cudaMemsetAsync(base + kOffBitmap, 0, ((size_t(k) + 31) / 32) * 4, s) != cudaSuccess) return RZ_ERR_CUDA;

    NoAllocFn f = noalloc_fn(elem_bytes);
    const uint32_t tile = uint32_t(kNoAllocBlock) * kNoAllocItems;
    const uint32_t ntiles = uint32_t((k + tile - 1) / tile);
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, (const void*)f, kNoAllocBlock, 0) != cudaSuccess || occ < 1)
        return RZ_ERR_CUDA;
    long grid = std::min<long>({long(occ) * ds.sms, long(ntiles), long(kMaxGrid)});
    const uint32_t tpc = (ntiles + uint32_t(grid) - 1) / uint32_t(grid);
    grid = (ntiles + tpc - 1) / tpc;

    SingleParams p;
    p.data = static_cast<uint8_t*>(d_data);
    p.idx = d_idx;
    p.n = uint32_t(n);
    p.k = uint32_t(k);
    p.bitmap = base + kOffBitmap;
    p.dlist = base + kOffDlist;
    p.slist = base + kOffSlist;
    p.epoch = base + kOffEpoch;
    p.arrive = base + kOffArrive;
    p.cnt_words = reinterpret_cast<unsigned long long*>(base + kOffCnt);
    p.status = base + kOffStatus;
    p.dev_len = nullptr;
    p.stamps = nullptr;
    p.spin_limit = kSpinLimit;
    p.validate = 0;
    p.redlist = nullptr;  // bitmap schedule only: the fixed scratch array has no red list
    p.arrive64 = nullptr;

    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(unsigned(grid));
    lc.blockDim = dim3(unsigned(kNoAllocBlock));
    lc.dynamicSmemBytes = 0;
    lc.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = grid > 1 ? 1 : 0;
    lc.attrs = attr;
    lc.numAttrs = 1;
    if (cudaLaunchKernelEx(&lc, f, p) != cudaSuccess) return RZ_ERR_CUDA;
    return RZ_OK;
}
