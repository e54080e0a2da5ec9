// redzone.hpp -- C++ shim over redzone.h with the reference's call shape.
//
// The reference's GPU entry point is a device-side template,
//   template <int WarpCount, int BlockCount, int prefetchcount, bool DebugPrint, typename T>
//   __device__ void RemoveFromList_GPUWide(T* List, const int Length, int* Removals,
//                                          const int RemoveCount, BlockStorage_t<BlockCount>&);
// (redzone.hxx:626-627), which the caller must launch cooperatively with exactly BlockCount
// blocks. redzone::RemoveFromList below keeps the argument order and meaning (list, length,
// removal indices, removal count), takes any 4/8/16/32-byte trivially copyable T, is called from
// the host, and returns the new length. It never writes Removals (the reference does) and reports
// failures as rz_status instead of exiting.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>

#include "redzone.h"

namespace redzone {

class Error : public std::runtime_error {
public:
    explicit Error(int code)
        : std::runtime_error(message(code)), code_(code) {}
    int code() const { return code_; }

private:
    static std::string message(int code) {
        char buf[128];
        rz_status_string(code, buf, sizeof(buf));
        return std::string("redzone: ") + buf;
    }
    int code_;
};

// One context per device and thread of control; owns the library scratch.
class Context {
public:
    explicit Context(int device = 0) {
        const int st = rz_create(&ctx_, device);
        if (st != RZ_OK) throw Error(st);
    }
    ~Context() { rz_destroy(ctx_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    rz_ctx* get() const { return ctx_; }

private:
    rz_ctx* ctx_ = nullptr;
};

// In-place removal of Removals[0..RemoveCount) from List[0..Length) (device pointers).
// Asynchronous on `stream` unless RZ_SYNC is in `flags`. Returns Length - RemoveCount.
template <typename T>
int64_t RemoveFromList(Context& ctx, T* List, int64_t Length, const uint32_t* Removals, int64_t RemoveCount,
                       rz_stream_t stream = nullptr, uint32_t flags = 0) {
    static_assert(std::is_trivially_copyable<T>::value, "items are moved as raw bytes");
    static_assert(sizeof(T) == 4 || sizeof(T) == 8 || sizeof(T) == 16 || sizeof(T) == 32,
                  "item size must be 4, 8, 16 or 32 bytes");
    int64_t new_len = 0;
    const int st = rz_remove(ctx.get(), List, Length, uint32_t(sizeof(T)), Removals, RemoveCount, &new_len, flags,
                             stream);
    if (st != RZ_OK) throw Error(st);
    return new_len;
}

// The reference's int-typed removal list (Removals is int*): same bits, read as unsigned.
template <typename T>
int64_t RemoveFromList(Context& ctx, T* List, int Length, const int* Removals, int RemoveCount,
                       rz_stream_t stream = nullptr, uint32_t flags = 0) {
    return RemoveFromList(ctx, List, int64_t(Length), reinterpret_cast<const uint32_t*>(Removals),
                          int64_t(RemoveCount), stream, flags);
}

}  // namespace redzone
