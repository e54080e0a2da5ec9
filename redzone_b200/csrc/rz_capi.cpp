// rz_capi.cpp -- the extern "C" boundary declared in include/redzone.h: context, scratch and
// dispatch of single-list removals. Kernels live in rz_single.cu; batching, tuning, the learned
// predictor and the service are in their own translation units.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <new>

#include "rz_internal.h"

namespace rz {

int cuda_fail(rz_ctx* ctx, cudaError_t e, const char* where) {
    if (ctx) {
        char buf[512];
        std::snprintf(buf, sizeof(buf), "%s: %s (%s)", where, cudaGetErrorName(e), cudaGetErrorString(e));
        ctx->last_cuda_error = buf;
    }
    return e == cudaErrorMemoryAllocation ? RZ_ERR_NO_MEMORY : RZ_ERR_CUDA;
}

template <typename T>
static int grow(rz_ctx* ctx, T*& ptr, size_t& cap, size_t want, bool zero) {
    if (want <= cap && ptr) return RZ_OK;
    size_t nc = std::max<size_t>(want, cap * 2);
    nc = std::max<size_t>(nc, 1024);
    // The scratch limit (rz_set_scratch_limit) counts every grown buffer; refusing leaves the old
    // buffer in place, so a refused call changes nothing.
    const size_t held_after = ctx->scratch_held - (ptr ? cap * sizeof(T) : 0) + nc * sizeof(T);
    if (held_after > ctx->scratch_limit) {
        if (want * sizeof(T) + ctx->scratch_held - (ptr ? cap * sizeof(T) : 0) > ctx->scratch_limit) {
            ctx->last_cuda_error = "context scratch limit reached";
            return RZ_ERR_NO_MEMORY;
        }
        nc = want;  // the doubling would pass the limit; the exact size still fits
    }
    if (ptr) {
        RZ_CUDA_TRY(ctx, cudaDeviceSynchronize());
        RZ_CUDA_TRY(ctx, cudaFree(ptr));
        ctx->scratch_held -= cap * sizeof(T);
        ptr = nullptr;
        cap = 0;
    }
    void* p = nullptr;
    RZ_CUDA_TRY(ctx, cudaMalloc(&p, nc * sizeof(T)));
    if (zero) RZ_CUDA_TRY(ctx, cudaMemset(p, 0, nc * sizeof(T)));
    ptr = static_cast<T*>(p);
    cap = nc;
    ctx->scratch_held += nc * sizeof(T);
    return RZ_OK;
}

int ensure_lists(rz_ctx* ctx, size_t k) {
    int st = grow(ctx, ctx->ws.bitmap, ctx->ws.bitmap_words, (k + 31) / 32 + 1, true);
    if (st != RZ_OK) return st;
    size_t cap = ctx->ws.list_cap;
    st = grow(ctx, ctx->ws.dlist, cap, k + 1, false);
    if (st != RZ_OK) return st;
    size_t cap2 = ctx->ws.list_cap;
    st = grow(ctx, ctx->ws.slist, cap2, k + 1, false);
    if (st != RZ_OK) return st;
    ctx->ws.list_cap = std::min(cap, cap2);
    if (k <= kRedlistMaxK) return grow(ctx, ctx->ws.redlist, ctx->ws.red_cap, k + 1, false);
    return RZ_OK;
}

int ensure_seen(rz_ctx* ctx, size_t n) {
    return grow(ctx, ctx->ws.seen, ctx->ws.seen_words, (n + 31) / 32 + 1, true);
}

int ensure_partition(rz_ctx* ctx, size_t n, size_t ntiles) {
    int st = grow(ctx, ctx->ws.part_bits, ctx->ws.part_words, (n + 31) / 32 + 1, true);
    if (st != RZ_OK) return st;
    // Ticket line (16 words), three 32-bit arrays of ntiles rounded up to 4 (staged, kept,
    // offset), then one 16-byte record per tile.
    const size_t ntp = (ntiles + 3) & ~size_t(3);
    return grow(ctx, ctx->ws.tile_state, ctx->ws.tile_cap, 16 + 3 * ntp / 2 + 2 * ntiles + 1, true);
}

int reset_if_dirty(rz_ctx* ctx, cudaStream_t s) {
    if (!ctx->ws.dirty) return RZ_OK;
    Workspace& w = ctx->ws;
    if (w.bitmap) RZ_CUDA_TRY(ctx, cudaMemsetAsync(w.bitmap, 0, w.bitmap_words * 4, s));
    if (w.seen) RZ_CUDA_TRY(ctx, cudaMemsetAsync(w.seen, 0, w.seen_words * 4, s));
    if (w.part_bits) RZ_CUDA_TRY(ctx, cudaMemsetAsync(w.part_bits, 0, w.part_words * 4, s));
    RZ_CUDA_TRY(ctx, cudaMemsetAsync(w.epoch, 0, 4, s));
    RZ_CUDA_TRY(ctx, cudaMemsetAsync(w.split_count, 0, 8, s));
    RZ_CUDA_TRY(ctx, cudaMemsetAsync(w.arrive, 0, kMaxGrid * 4, s));
    RZ_CUDA_TRY(ctx, cudaMemsetAsync(w.cnt_words, 0, 2 * kMaxGrid * 8, s));
    RZ_CUDA_TRY(ctx, cudaMemsetAsync(w.arrive64, 0, kMaxGrid * 8, s));
    w.dirty = false;
    return RZ_OK;
}

int map_status(uint32_t bits) {
    if (bits & 16u) return RZ_ERR_NO_MEMORY;
    if (bits & 2u) return RZ_ERR_OUT_OF_RANGE;
    if (bits & 1u) return RZ_ERR_DUPLICATE;
    if (bits & 4u) return RZ_ERR_TIMEOUT;
    if (bits & 8u) return RZ_ERR_DUPLICATE;
    return RZ_OK;
}

// The status word (offset 0) and the device length (offset 512) of the workspace block come back
// in one copy on the call's stream into pinned memory. The caller waits for it by polling an
// event recorded after the copy, so a synchronous call returns within about a microsecond of
// the copy landing; after kPollLimit of polling it blocks in cudaEventSynchronize instead.
static constexpr std::chrono::microseconds kPollLimit{2000};

int wait_event(rz_ctx* ctx, cudaEvent_t ev) {
    const auto t0 = std::chrono::steady_clock::now();
    bool polled = false;
    for (;;) {
        const cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) return cuda_fail(ctx, e, "cudaEventQuery");
        polled = true;
        if (std::chrono::steady_clock::now() - t0 > kPollLimit) {
            RZ_CUDA_TRY(ctx, cudaEventSynchronize(ev));
            break;
        }
    }
    // "Not ready" is not a failure: do not leave it behind as the thread's last error.
    if (polled && cudaPeekAtLastError() == cudaErrorNotReady) cudaGetLastError();
    return RZ_OK;
}

static int fetch_result(rz_ctx* ctx, cudaStream_t s, uint32_t* status, unsigned long long* len) {
    RZ_CUDA_TRY(ctx, cudaMemcpyAsync(ctx->ws.h_result, ctx->ws.status, kResultBytes, cudaMemcpyDeviceToHost, s));
    RZ_CUDA_TRY(ctx, cudaEventRecord(ctx->done_event, s));
    const int st = wait_event(ctx, ctx->done_event);
    if (st != RZ_OK) return st;
    std::memcpy(status, ctx->ws.h_result, sizeof(uint32_t));
    if (len) std::memcpy(len, ctx->ws.h_result + 512, sizeof(unsigned long long));
    return RZ_OK;
}

int read_status(rz_ctx* ctx, cudaStream_t s, int64_t* new_len) {
    uint32_t h = 0;
    unsigned long long dl = 0;
    int st = fetch_result(ctx, s, &h, new_len ? &dl : nullptr);
    if (st != RZ_OK) return st;
    if (new_len) *new_len = int64_t(dl);
    if (h) {
        RZ_CUDA_TRY(ctx, cudaMemset(ctx->ws.status, 0, sizeof(uint32_t)));
        // A failed call may have left barrier state or bitmap bits behind.
        ctx->ws.dirty = true;
    }
    return map_status(h);
}

static int check_args(const void* data, int64_t n, uint32_t w, const uint32_t* idx, int64_t k) {
    if (n < 0 || k < 0 || k > n) return RZ_ERR_INVALID_ARG;
    if (w != 4 && w != 8 && w != 16 && w != 32) return RZ_ERR_INVALID_ARG;
    if (n >= (int64_t(1) << 32)) return RZ_ERR_UNSUPPORTED;
    if (k > 0 && (!data || !idx)) return RZ_ERR_INVALID_ARG;
    const uintptr_t align = w >= 16 ? 16 : w;
    if (reinterpret_cast<uintptr_t>(data) % align) return RZ_ERR_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(idx) % 4) return RZ_ERR_INVALID_ARG;
    return RZ_OK;
}

}  // namespace rz

using namespace rz;

extern "C" {

int rz_create(rz_ctx** out, int device) {
    if (!out) return RZ_ERR_INVALID_ARG;
    *out = nullptr;
    rz_ctx* ctx = new (std::nothrow) rz_ctx();
    if (!ctx) return RZ_ERR_NO_MEMORY;
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        int st = cuda_fail(ctx, e, "cudaSetDevice");
        delete ctx;
        return st;
    }
    cudaDeviceProp prop{};
    e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) {
        int st = cuda_fail(ctx, e, "cudaGetDeviceProperties");
        delete ctx;
        return st;
    }
    ctx->sms = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    Workspace& w = ctx->ws;
    void* p = nullptr;
    // One allocation: status | epoch (split-schedule counters at +128) | dev_len (one 256-byte
    // line each) | arrival tags |
    // tagged orphan counts | tagged red-entry counts | phase stamps.
    const size_t off_arrive = 768;
    const size_t off_cnt = off_arrive + size_t(kMaxGrid) * 4;
    const size_t off_arr64 = off_cnt + size_t(2 * kMaxGrid) * 8;
    const size_t off_stamps = off_arr64 + size_t(kMaxGrid) * 8;
    const size_t bytes = off_stamps + size_t(kMaxGrid) * kStampsPerCta * 8;
    e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) e = cudaMemset(p, 0, bytes);
    if (e != cudaSuccess) {
        int st = cuda_fail(ctx, e, "workspace");
        delete ctx;
        return st;
    }
    uint8_t* b = static_cast<uint8_t*>(p);
    w.status = reinterpret_cast<uint32_t*>(b);
    w.epoch = reinterpret_cast<uint32_t*>(b + 256);
    w.split_count = reinterpret_cast<uint32_t*>(b + 384);
    w.dev_len = reinterpret_cast<unsigned long long*>(b + 512);
    w.arrive = reinterpret_cast<uint32_t*>(b + off_arrive);
    w.cnt_words = reinterpret_cast<unsigned long long*>(b + off_cnt);
    w.arrive64 = reinterpret_cast<unsigned long long*>(b + off_arr64);
    w.stamps = reinterpret_cast<unsigned long long*>(b + off_stamps);
    void* hr = nullptr;
    e = cudaMallocHost(&hr, kResultBytes);
    if (e != cudaSuccess) {
        int st = cuda_fail(ctx, e, "pinned result buffer");
        cudaFree(p);
        delete ctx;
        return st;
    }
    w.h_result = static_cast<uint8_t*>(hr);
    e = cudaEventCreateWithFlags(&ctx->done_event, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        int st = cuda_fail(ctx, e, "completion event");
        cudaFreeHost(hr);
        cudaFree(p);
        delete ctx;
        return st;
    }
    *out = ctx;
    return RZ_OK;
}

void rz_destroy(rz_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    Workspace& w = ctx->ws;
    cudaFree(w.status);
    if (w.h_result) cudaFreeHost(w.h_result);
    if (ctx->done_event) cudaEventDestroy(ctx->done_event);
    cudaFree(w.bitmap);
    cudaFree(w.dlist);
    cudaFree(w.slist);
    cudaFree(w.redlist);
    cudaFree(w.seen);
    cudaFree(w.part_bits);
    cudaFree(w.tile_state);
    cudaFree(w.idx_stage);
    cudaFree(w.keep_stage);
    release_extras(ctx);
    delete ctx;
}

int rz_status_string(int code, char* buf, size_t len) {
    const char* s = "unknown status";
    switch (code) {
        case RZ_OK: s = "ok"; break;
        case RZ_ERR_INVALID_ARG: s = "invalid argument"; break;
        case RZ_ERR_DUPLICATE: s = "duplicate removal index"; break;
        case RZ_ERR_OUT_OF_RANGE: s = "removal index out of range"; break;
        case RZ_ERR_NO_MEMORY: s = "out of device memory"; break;
        case RZ_ERR_TIMEOUT: s = "bounded device wait timed out"; break;
        case RZ_ERR_CUDA: s = "CUDA runtime error"; break;
        case RZ_ERR_UNSUPPORTED: s = "unsupported"; break;
        case RZ_ERR_BUSY: s = "admission refused"; break;
        default: break;
    }
    if (!buf || len == 0) return int(std::strlen(s));
    std::snprintf(buf, len, "%s", s);
    return int(std::strlen(buf));
}

int rz_last_cuda_error(const rz_ctx* ctx, char* buf, size_t len) {
    if (!ctx || !buf || len == 0) return 0;
    std::snprintf(buf, len, "%s", ctx->last_cuda_error.c_str());
    return int(std::strlen(buf));
}

int rz_sync_status(rz_ctx* ctx, rz_stream_t stream) {
    if (!ctx) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return read_status(ctx, reinterpret_cast<cudaStream_t>(stream));
}

int rz_num_sms(const rz_ctx* ctx) { return ctx ? ctx->sms : 0; }

int rz_set_scratch_limit(rz_ctx* ctx, int64_t bytes) {
    if (!ctx) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    ctx->scratch_limit = bytes < 0 ? ~size_t(0) : size_t(bytes);
    return RZ_OK;
}

int64_t rz_scratch_bytes(const rz_ctx* ctx) { return ctx ? int64_t(ctx->scratch_held) : 0; }

int rz_default_cfg(const rz_ctx* ctx, int64_t n, int64_t k, uint32_t elem_bytes, rz_launch_cfg* cfg) {
    if (!ctx || !cfg || k < 0 || n < k) return RZ_ERR_INVALID_ARG;
    if (n >= (int64_t(1) << 32)) return RZ_ERR_UNSUPPORTED;
    return default_cfg(ctx, uint32_t(n), uint32_t(k), elem_bytes, cfg);
}

int rz_remove_cfg(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes, const uint32_t* d_idx,
                  int64_t k, const rz_launch_cfg* cfg, uint32_t flags, rz_stream_t stream) {
    if (!ctx || !cfg) return RZ_ERR_INVALID_ARG;
    int st = check_args(d_data, n, elem_bytes, d_idx, k);
    if (st != RZ_OK) return st;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    ctx->last_kernels = 0;
    ctx->last_grid = 0;
    ctx->last_block = 0;
    if (k == 0 || k == n) {
        // Nothing moves (reference: redzone.hxx:651, Redzone_CPU.hxx handles it implicitly).
        if (flags & RZ_VALIDATE && k > 0) {
            st = launch_validate(ctx, uint32_t(n), d_idx, uint32_t(k), s);
            if (st != RZ_OK) return st;
            ctx->last_kernels = 2;
        }
        return (flags & RZ_SYNC) ? read_status(ctx, s) : RZ_OK;
    }
    LaunchInfo info;
    if (cfg->use_partition || (flags & RZ_FORCE_PARTITION))
        st = launch_partition(ctx, d_data, uint32_t(n), elem_bytes, d_idx, uint32_t(k), flags, s, &info);
    else
        st = launch_redzone(ctx, d_data, uint32_t(n), elem_bytes, d_idx, uint32_t(k), *cfg, flags, s, &info);
    if (st != RZ_OK) return st;
    ctx->last_kernels = info.launches;
    ctx->last_grid = info.grid;
    ctx->last_block = info.block;
    return (flags & RZ_SYNC) ? read_status(ctx, s) : RZ_OK;
}

int rz_remove(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes, const uint32_t* d_idx, int64_t k,
              int64_t* new_len, uint32_t flags, rz_stream_t stream) {
    if (!ctx) return RZ_ERR_INVALID_ARG;
    int st = check_args(d_data, n, elem_bytes, d_idx, k);
    if (st != RZ_OK) return st;
    if (new_len) *new_len = n - k;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    rz_launch_cfg cfg{};
    bool have = false;
    if (flags & RZ_USE_PREDICTOR)
        have = predict_cfg(ctx, uint32_t(n), uint32_t(k), elem_bytes, d_idx,
                              reinterpret_cast<cudaStream_t>(stream), &cfg);
    if (!have) have = tuned_cfg(ctx, uint32_t(n), uint32_t(k), elem_bytes, &cfg);
    if (!have) {
        st = default_cfg(ctx, uint32_t(n), uint32_t(k), elem_bytes, &cfg);
        if (st != RZ_OK) return st;
    }
    // The partition path reorders survivors; it runs only when the caller allows that order.
    if (cfg.use_partition && !(flags & RZ_ALLOW_STABLE)) cfg.use_partition = 0;
    return rz_remove_cfg(ctx, d_data, n, elem_bytes, d_idx, k, &cfg, flags, stream);
}

int rz_append_remove(rz_ctx* ctx, void* d_data, int64_t n, int64_t capacity, uint32_t elem_bytes,
                     const void* d_gain, int64_t g, const uint32_t* d_idx, int64_t k, int64_t* new_len,
                     uint32_t flags, rz_stream_t stream) {
    if (!ctx || g < 0 || n < 0 || (g > 0 && !d_gain) || capacity < n + g) return RZ_ERR_INVALID_ARG;
    int st = check_args(d_data, n + g, elem_bytes, d_idx, k);
    if (st != RZ_OK) return st;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    if (g > 0) {
        uint8_t* dst = static_cast<uint8_t*>(d_data) + size_t(n) * elem_bytes;
        RZ_CUDA_TRY(ctx, cudaMemcpyAsync(dst, d_gain, size_t(g) * elem_bytes, cudaMemcpyDeviceToDevice,
                                         reinterpret_cast<cudaStream_t>(stream)));
    }
    return rz_remove(ctx, d_data, n + g, elem_bytes, d_idx, k, new_len, flags, stream);
}

int rz_keep(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes, const uint32_t* d_keep, int64_t m,
            int64_t* new_len, uint32_t flags, rz_stream_t stream) {
    if (!ctx) return RZ_ERR_INVALID_ARG;
    // The keep list may be any length up to n and in any order: the same checks as a removal
    // list of the same length.
    int st = check_args(d_data, n, elem_bytes, d_keep, m);
    if (st != RZ_OK) return st;
    if (new_len) *new_len = m;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    st = grow(ctx, ctx->ws.keep_stage, ctx->ws.keep_cap, (size_t(m) * elem_bytes + 15) / 16 + 1, false);
    if (st != RZ_OK) return st;
    st = launch_keep(ctx, d_data, uint32_t(n), elem_bytes, d_keep, uint32_t(m), ctx->ws.keep_stage, s);
    if (st != RZ_OK) return st;
    ctx->last_kernels = m > 0 ? 1 : 0;
    if (flags & RZ_SYNC) return read_status(ctx, s);
    return RZ_OK;
}

int rz_partition(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes, const uint32_t* d_idx, int64_t k,
                 int64_t* new_len, uint32_t flags, rz_stream_t stream) {
    if (!ctx) return RZ_ERR_INVALID_ARG;
    int st = check_args(d_data, n, elem_bytes, d_idx, k);
    if (st != RZ_OK) return st;
    if (new_len) *new_len = n - k;
    rz_launch_cfg cfg{256, 8, 1, 1, RZ_SCHED_AUTO};
    return rz_remove_cfg(ctx, d_data, n, elem_bytes, d_idx, k, &cfg, flags | RZ_FORCE_PARTITION, stream);
}

int rz_remove_host_idx(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes, const uint32_t* h_idx,
                       int64_t k, int64_t* new_len, uint32_t flags, rz_stream_t stream) {
    if (!ctx) return RZ_ERR_INVALID_ARG;
    int st = check_args(d_data, n, elem_bytes, h_idx, k);
    if (st != RZ_OK) return st;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    st = grow(ctx, ctx->ws.idx_stage, ctx->ws.stage_cap, size_t(k) + 1, false);
    if (st != RZ_OK) return st;
    uint32_t* d_stage = ctx->ws.idx_stage;
    if (k > 0) RZ_CUDA_TRY(ctx, cudaMemcpyAsync(d_stage, h_idx, size_t(k) * 4, cudaMemcpyHostToDevice, s));
    int64_t nl = 0;
    st = rz_remove(ctx, d_data, n, elem_bytes, d_stage, k, &nl, flags & ~RZ_SYNC, stream);
    if (st != RZ_OK) return st;
    // Read the device-tracked length back with the status: the step's result crosses to the host.
    unsigned long long dl = 0;
    uint32_t h = 0;
    st = fetch_result(ctx, s, &h, &dl);
    if (st != RZ_OK) return st;
    if (h) {
        RZ_CUDA_TRY(ctx, cudaMemset(ctx->ws.status, 0, sizeof(uint32_t)));
        ctx->ws.dirty = true;
    }
    if (new_len) *new_len = (k > 0 && k < n) ? int64_t(dl) : n - k;
    return map_status(h);
}

int rz_last_launch(const rz_ctx* ctx, int32_t* kernels, int32_t* grid, int32_t* block) {
    if (!ctx) return RZ_ERR_INVALID_ARG;
    if (kernels) *kernels = ctx->last_kernels;
    if (grid) *grid = ctx->last_grid;
    if (block) *block = ctx->last_block;
    return RZ_OK;
}

int rz_phase_stamps(rz_ctx* ctx, int enable) {
    if (!ctx) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    ctx->ws.stamps_on = enable != 0;
    return RZ_OK;
}

int rz_read_phase_stamps(rz_ctx* ctx, uint64_t* out, int32_t max_ctas, int32_t* nctas) {
    if (!ctx || !out || max_ctas < 0) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    const int n = std::min<int>(max_ctas, std::min(ctx->last_grid, kMaxGrid));
    RZ_CUDA_TRY(ctx, cudaDeviceSynchronize());
    if (n > 0)
        RZ_CUDA_TRY(ctx, cudaMemcpy(out, ctx->ws.stamps, size_t(n) * kStampsPerCta * 8, cudaMemcpyDeviceToHost));
    if (nctas) *nctas = n;
    return RZ_OK;
}

int rz_test_empty_launch(rz_ctx* ctx, int32_t grid, int32_t block, int32_t cluster, int32_t smem_bytes,
                         rz_stream_t stream) {
    if (!ctx) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return test_empty_launch(ctx, grid, block, cluster, smem_bytes, reinterpret_cast<cudaStream_t>(stream));
}

int rz_test_scatter(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes, const uint32_t* d_pos, int64_t count,
                    rz_stream_t stream) {
    if (!ctx || n < 0 || count < 0 || (count > 0 && (!d_data || !d_pos))) return RZ_ERR_INVALID_ARG;
    if (n >= (int64_t(1) << 32) || count >= (int64_t(1) << 32)) return RZ_ERR_UNSUPPORTED;
    const uintptr_t align = elem_bytes >= 16 ? 16 : elem_bytes;
    if (align == 0 || reinterpret_cast<uintptr_t>(d_data) % align) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return test_scatter(ctx, d_data, uint32_t(n), elem_bytes, d_pos, uint32_t(count),
                        reinterpret_cast<cudaStream_t>(stream));
}

int rz_test_barrier_timeout(rz_ctx* ctx, uint32_t spin_limit, uint32_t* status_bits) {
    if (!ctx || !status_bits) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return test_barrier_timeout(ctx, spin_limit, status_bits);
}

}  // extern "C"
