// rz_async.cpp -- rz_remove_host_idx_async / rz_wait: the host-index removal, pipelined.
//
// rz_remove_host_idx copies the host index list, runs the removal, reads the result back and
// waits, so consecutive calls run strictly one after another: copy, kernel, read-back, host
// wake-up. A host program that feeds the GPU a stream of removal lists (the reference's
// redzone_CPU call shape, Redzone_CPU.hxx:150, called in a loop) can instead issue calls without
// waiting and collect each result later. Per context there is a ring of kSlots slots, each with a
// device copy of one index list, its own device status word and length word (the call's kernels
// write those instead of the context's, so calls in flight never share them), a pinned copy of
// both, and three events. Three streams:
//   copy stream : H2D h_idx -> slot.d_idx ; record slot.copied
//   call stream : wait slot.copied ; [zero slot.status, after a call that reported an error] ;
//                 removal kernel(s) ; record slot.kdone
//   read stream : wait slot.kdone ; D2H slot.status|flag|length (16 bytes) -> slot.h_res ;
//                 record slot.done
// rz_wait spins on the landing flag (a word that is zero on the device and armed on the host)
// instead of querying the event: no CUDA call per wait (the event remains the fallback).
// The index copy of call i+1 runs while call i's kernel runs, and call i's read-back while call
// i+1's kernel runs, so with a few calls in flight the call stream runs the kernels back to back.
// The read-back is one 16-byte copy and nothing else: measured on B200 with a 256 KB list per
// call, a 4-byte memset on the read stream after each copy took the loop from 9.5 to 15.5 us per
// step, and a store of the result to mapped host memory from the kernel itself to 12.2 us (the
// kernel cannot end until the store has crossed PCIe, behind the list copies). So a slot's status
// word is cleared on the call stream, and only after a call that reported an error.
// A slot is reused only after its previous call was collected (rz_wait) or, when the caller
// issues more than kSlots calls ahead, after the issuing call has waited for it and kept its
// result for a later rz_wait.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <deque>
#include <new>

#include "rz_internal.h"

namespace rz {

namespace {

constexpr int kSlots = 8;
constexpr size_t kStashMax = 1024;  // results of calls evicted from their slot before rz_wait
constexpr size_t kSlotResBytes = 256;   // a slot's device status (offset 0) and length (offset 8)
constexpr size_t kSlotReadBytes = 16;   // what comes back per call: status word, landing flag, length
constexpr uint32_t kArmed = 0xffffffffu;  // the host's landing flag before the read-back arrives
constexpr auto kLandPoll = std::chrono::microseconds(2000);

struct Slot {
    uint32_t* d_idx = nullptr;
    size_t cap = 0;                  // entries of d_idx
    uint8_t* d_res = nullptr;        // device: status word at 0, device length at 8
    uint8_t* h_res = nullptr;        // pinned copy of the same kSlotReadBytes
    bool clear_status = false;       // the last call reported an error: zero the status before reuse
    cudaEvent_t copied = nullptr;
    cudaEvent_t kdone = nullptr;
    cudaEvent_t done = nullptr;
    uint64_t ticket = 0;
    int64_t k = 0, n = 0;
    bool pending = false;
};

struct Result {
    uint64_t ticket;
    int status;
    int64_t new_len;
};

}  // namespace

struct AsyncPipe {
    cudaStream_t copy_stream = nullptr;
    cudaStream_t read_stream = nullptr;
    uint8_t* d_res = nullptr;        // kSlots * kSlotResBytes
    Slot slots[kSlots];
    std::deque<Result> stash;
    uint64_t next_ticket = 1;
};

namespace {

void pipe_free(AsyncPipe* p) {
    for (Slot& s : p->slots) {
        cudaFree(s.d_idx);
        if (s.h_res) cudaFreeHost(s.h_res);
        if (s.copied) cudaEventDestroy(s.copied);
        if (s.kdone) cudaEventDestroy(s.kdone);
        if (s.done) cudaEventDestroy(s.done);
    }
    cudaFree(p->d_res);
    if (p->copy_stream) cudaStreamDestroy(p->copy_stream);
    if (p->read_stream) cudaStreamDestroy(p->read_stream);
    delete p;
}

int pipe_create(rz_ctx* ctx, AsyncPipe** out) {
    AsyncPipe* p = new (std::nothrow) AsyncPipe();
    if (!p) return RZ_ERR_NO_MEMORY;
    cudaError_t e = cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->read_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_res, kSlots * kSlotResBytes);
    if (e == cudaSuccess) e = cudaMemset(p->d_res, 0, kSlots * kSlotResBytes);
    for (int i = 0; i < kSlots && e == cudaSuccess; ++i) {
        Slot& s = p->slots[i];
        s.d_res = p->d_res + size_t(i) * kSlotResBytes;
        void* h = nullptr;
        e = cudaMallocHost(&h, kSlotReadBytes);
        if (e != cudaSuccess) break;
        s.h_res = static_cast<uint8_t*>(h);
        e = cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.kdone, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        const int st = cuda_fail(ctx, e, "asynchronous pipeline");
        pipe_free(p);
        return st;
    }
    *out = p;
    return RZ_OK;
}

// The finished call of a pending slot: its status and device-tracked length, as read back. A
// device error marks the context scratch for a reset before its next call, and the slot's status
// word for clearing before the slot's next call.
int collect(rz_ctx* ctx, Slot& s, Result* r) {
    // The read-back copies 16 bytes whose word at offset 4 is zero on the device; the host set its
    // copy of that word to kArmed when it issued the call, so zero there means the copy has landed
    // (one 16-byte write). Spin on it for up to kLandPoll, then wait for the slot's event.
    volatile const uint32_t* flag = reinterpret_cast<volatile const uint32_t*>(s.h_res + 4);
    bool landed = *flag == 0u;
    if (!landed) {
        const auto t0 = std::chrono::steady_clock::now();
        while (!(landed = (*flag == 0u)) && std::chrono::steady_clock::now() - t0 < kLandPoll) {
        }
    }
    if (!landed) {
        const int st = wait_event(ctx, s.done);
        if (st != RZ_OK) return st;
    }
    std::atomic_thread_fence(std::memory_order_acquire);
    uint32_t bits = 0;
    unsigned long long len = 0;
    std::memcpy(&bits, s.h_res, sizeof(bits));
    std::memcpy(&len, s.h_res + 8, sizeof(len));
    s.pending = false;
    if (bits) {
        ctx->ws.dirty = true;
        s.clear_status = true;
    }
    r->ticket = s.ticket;
    r->status = map_status(bits);
    r->new_len = (s.k > 0 && s.k < s.n) ? int64_t(len) : s.n - s.k;
    return RZ_OK;
}

// Aim the context's status and length words at a slot's for the duration of one launch: every
// kernel takes both pointers from the context when it is launched.
struct ResultRedirect {
    rz_ctx* ctx;
    uint32_t* status;
    unsigned long long* dev_len;
    ResultRedirect(rz_ctx* c, uint8_t* d_res) : ctx(c), status(c->ws.status), dev_len(c->ws.dev_len) {
        ctx->ws.status = reinterpret_cast<uint32_t*>(d_res);
        ctx->ws.dev_len = reinterpret_cast<unsigned long long*>(d_res + 8);
    }
    ~ResultRedirect() {
        ctx->ws.status = status;
        ctx->ws.dev_len = dev_len;
    }
};

}  // namespace

void release_async(rz_ctx* ctx) {
    AsyncPipe* p = static_cast<AsyncPipe*>(ctx->async_pipe);
    if (!p) return;
    cudaStreamSynchronize(p->copy_stream);
    cudaStreamSynchronize(p->read_stream);
    for (Slot& s : p->slots)
        if (s.done) cudaEventSynchronize(s.done);
    pipe_free(p);
    ctx->async_pipe = nullptr;
}

}  // namespace rz

using namespace rz;

extern "C" {

int rz_remove_host_idx_async(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes, const uint32_t* h_idx,
                             int64_t k, uint32_t flags, rz_stream_t stream, uint64_t* ticket) {
    if (!ctx || !ticket) return RZ_ERR_INVALID_ARG;
    *ticket = 0;
    if (n < 0 || k < 0 || k > n || (k > 0 && (!d_data || !h_idx))) return RZ_ERR_INVALID_ARG;
    if (n >= (int64_t(1) << 32)) return RZ_ERR_UNSUPPORTED;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    if (!ctx->async_pipe) {
        AsyncPipe* p = nullptr;
        const int st = pipe_create(ctx, &p);
        if (st != RZ_OK) return st;
        ctx->async_pipe = p;
    }
    AsyncPipe& P = *static_cast<AsyncPipe*>(ctx->async_pipe);
    const uint64_t t = P.next_ticket;
    Slot& s = P.slots[t % kSlots];
    if (s.pending) {
        // The caller is more than kSlots calls ahead: finish the slot's call and keep its result.
        Result r;
        const int st = collect(ctx, s, &r);
        if (st != RZ_OK) return st;
        P.stash.push_back(r);
        if (P.stash.size() > kStashMax) P.stash.pop_front();
    }
    if (size_t(k) + 1 > s.cap) {
        // Grow the slot's staging (its previous call, if any, has finished).
        const size_t want = std::max<size_t>(size_t(k) + 1, 2 * s.cap);
        if (s.d_idx) {
            RZ_CUDA_TRY(ctx, cudaFree(s.d_idx));
            ctx->scratch_held -= s.cap * 4;
            s.d_idx = nullptr;
            s.cap = 0;
        }
        if (ctx->scratch_held + want * 4 > ctx->scratch_limit) {
            ctx->last_cuda_error = "context scratch limit reached";
            return RZ_ERR_NO_MEMORY;
        }
        void* d = nullptr;
        RZ_CUDA_TRY(ctx, cudaMalloc(&d, want * 4));
        s.d_idx = static_cast<uint32_t*>(d);
        s.cap = want;
        ctx->scratch_held += want * 4;
    }
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(stream);
    // Copy stream: the index list arrives.
    if (k > 0)
        RZ_CUDA_TRY(ctx, cudaMemcpyAsync(s.d_idx, h_idx, size_t(k) * 4, cudaMemcpyHostToDevice, P.copy_stream));
    RZ_CUDA_TRY(ctx, cudaEventRecord(s.copied, P.copy_stream));
    // Call stream: the removal, writing the slot's status and length words. The status word is
    // zero (it starts so; after a call that reported an error it is cleared here first).
    RZ_CUDA_TRY(ctx, cudaStreamWaitEvent(cs, s.copied, 0));
    if (s.clear_status) {
        RZ_CUDA_TRY(ctx, cudaMemsetAsync(s.d_res, 0, sizeof(uint32_t), cs));
        s.clear_status = false;
    }
    int st;
    {
        ResultRedirect redirect(ctx, s.d_res);
        st = rz_remove(ctx, d_data, n, elem_bytes, s.d_idx, k, nullptr, flags & ~uint32_t(RZ_SYNC), stream);
    }
    if (st != RZ_OK) return st;
    RZ_CUDA_TRY(ctx, cudaEventRecord(s.kdone, cs));
    // Read stream: the result comes back while the call stream runs the next removal.
    RZ_CUDA_TRY(ctx, cudaStreamWaitEvent(P.read_stream, s.kdone, 0));
    *reinterpret_cast<volatile uint32_t*>(s.h_res + 4) = kArmed;
    RZ_CUDA_TRY(ctx, cudaMemcpyAsync(s.h_res, s.d_res, kSlotReadBytes, cudaMemcpyDeviceToHost, P.read_stream));
    RZ_CUDA_TRY(ctx, cudaEventRecord(s.done, P.read_stream));
    s.ticket = t;
    s.k = k;
    s.n = n;
    s.pending = true;
    P.next_ticket = t + 1;
    *ticket = t;
    return RZ_OK;
}

int rz_wait(rz_ctx* ctx, uint64_t ticket, int64_t* new_len) {
    if (!ctx || ticket == 0) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    AsyncPipe* p = static_cast<AsyncPipe*>(ctx->async_pipe);
    if (!p || ticket >= p->next_ticket) return RZ_ERR_INVALID_ARG;
    Slot& s = p->slots[ticket % kSlots];
    Result r{};
    if (s.pending && s.ticket == ticket) {
        const int st = collect(ctx, s, &r);
        if (st != RZ_OK) return st;
    } else {
        auto it = std::find_if(p->stash.begin(), p->stash.end(), [&](const Result& x) { return x.ticket == ticket; });
        if (it == p->stash.end()) return RZ_ERR_INVALID_ARG;  // already collected, or too old
        r = *it;
        p->stash.erase(it);
    }
    if (new_len) *new_len = r.new_len;
    return r.status;
}

}  // extern "C"
