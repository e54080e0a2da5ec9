// rz_keyidx.cu -- a key -> row index kept current under Redzone moves, for delete-by-key.
//
// Records are 8, 16 or 32 bytes and start with a uint64 key (two reserved values: all ones marks
// an empty slot, all ones minus one an erased one). The index is an open-addressing hash table on
// the device: capacity a power of two, linear probing from the SplitMix64 finaliser of the key
// (Steele, Lea and Flood, "Fast splittable pseudorandom number generators", 2014).
//
// Removal by key keeps the index exact in O(k): the canonical rule moves an item only into a hole
// below the cut (every other surviving item keeps its row), so after the removal each hole's new
// occupant is re-pointed at the hole, and the deleted keys are erased. Nothing is rescanned.
#include <algorithm>
#include <new>

#include "rz_common.cuh"
#include "rz_internal.h"

namespace rz {

constexpr unsigned long long kEmptyKey = ~0ull;
constexpr unsigned long long kErasedKey = ~0ull - 1ull;
constexpr uint32_t kNoRow = 0xffffffffu;
enum : uint32_t { IX_DUPLICATE = 1u, IX_MISSING = 2u, IX_FULL = 4u, IX_RESERVED = 8u };

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ unsigned long long record_key(const uint8_t* data, uint32_t w, uint32_t row) {
    return *reinterpret_cast<const unsigned long long*>(data + size_t(row) * w);
}

// Slot holding `key`, or kNoRow (stops at the first empty slot; erased slots are passed over).
__device__ __forceinline__ uint32_t find_slot(const unsigned long long* keys, uint32_t mask, unsigned long long key) {
    uint32_t s = uint32_t(mix64(key)) & mask;
    for (uint32_t probe = 0; probe <= mask; ++probe, s = (s + 1u) & mask) {
        const unsigned long long k0 = keys[s];
        if (k0 == key) return s;
        if (k0 == kEmptyKey) return kNoRow;
    }
    return kNoRow;
}

__global__ void ix_insert_kernel(unsigned long long* keys, uint32_t* rows, uint32_t mask, const uint8_t* data,
                                 uint32_t w, uint32_t first, uint32_t count, uint32_t* status) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
        const uint32_t row = first + q;
        const unsigned long long key = record_key(data, w, row);
        if (key >= kErasedKey) {
            atomicOr(status, IX_RESERVED);
            continue;
        }
        uint32_t s = uint32_t(mix64(key)) & mask;
        bool done = false;
        for (uint32_t probe = 0; probe <= mask && !done; ++probe, s = (s + 1u) & mask) {
            unsigned long long k0 = keys[s];
            while (k0 == kEmptyKey || k0 == kErasedKey) {
                const unsigned long long prev = atomicCAS(&keys[s], k0, key);
                if (prev == k0) {
                    rows[s] = row;
                    done = true;
                    break;
                }
                k0 = prev;  // someone else took the slot: look at what they put there
            }
            if (!done && k0 == key) {
                atomicOr(status, IX_DUPLICATE);
                done = true;
            }
        }
        if (!done) atomicOr(status, IX_FULL);
    }
}

// Rows of the keys to delete (kNoRow and IX_MISSING when absent) and their slots.
__global__ void ix_lookup_kernel(const unsigned long long* keys, const uint32_t* rows, uint32_t mask,
                                 const unsigned long long* q, uint32_t count, uint32_t* out_rows,
                                 uint32_t* out_slots, uint32_t* status) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const unsigned long long key = q[i];
        const uint32_t s = key >= kErasedKey ? kNoRow : find_slot(keys, mask, key);
        if (s == kNoRow) {
            out_rows[i] = kNoRow;
            if (out_slots) atomicOr(status, IX_MISSING);
        } else {
            out_rows[i] = rows[s];
        }
        if (out_slots) out_slots[i] = s;
    }
}

__global__ void ix_erase_kernel(unsigned long long* keys, const uint32_t* slots, uint32_t count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        keys[slots[i]] = kErasedKey;
}

// After the removal: every hole below the cut holds a moved item; point its key at the hole.
__global__ void ix_repoint_kernel(const unsigned long long* keys, uint32_t* rows, uint32_t mask, const uint8_t* data,
                                  uint32_t w, const uint32_t* holes, uint32_t count, uint32_t cut) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t h = holes[i];
        if (h >= cut) continue;
        const uint32_t s = find_slot(keys, mask, record_key(data, w, h));
        if (s != kNoRow) rows[s] = h;
    }
}

static int grid_for(const rz_ctx* ctx, int64_t count) {
    return int(std::max<int64_t>(1, std::min<int64_t>(int64_t(ctx->sms) * 8, (count + 255) / 256)));
}

}  // namespace rz

struct rz_keyindex {
    rz_ctx* ctx = nullptr;
    unsigned long long* keys = nullptr;
    uint32_t* rows = nullptr;
    uint32_t mask = 0;
    uint32_t* status = nullptr;      // device
    uint32_t* h_status = nullptr;    // pinned
    uint32_t* del_rows = nullptr;    // removal list of the current call
    uint32_t* del_slots = nullptr;
    size_t del_cap = 0;
};

using namespace rz;

static int ix_status(rz_keyindex* ix, cudaStream_t s, uint32_t* bits) {
    RZ_CUDA_TRY(ix->ctx, cudaMemcpyAsync(ix->h_status, ix->status, 4, cudaMemcpyDeviceToHost, s));
    RZ_CUDA_TRY(ix->ctx, cudaStreamSynchronize(s));
    *bits = *ix->h_status;
    if (*bits) RZ_CUDA_TRY(ix->ctx, cudaMemsetAsync(ix->status, 0, 4, s));
    return RZ_OK;
}

static int ix_map(uint32_t bits) {
    if (bits & IX_RESERVED) return RZ_ERR_INVALID_ARG;
    if (bits & IX_FULL) return RZ_ERR_NO_MEMORY;
    if (bits & IX_DUPLICATE) return RZ_ERR_DUPLICATE;
    if (bits & IX_MISSING) return RZ_ERR_OUT_OF_RANGE;
    return RZ_OK;
}

static bool key_record(uint32_t w) { return w == 8 || w == 16 || w == 32; }

extern "C" {

int rz_keyindex_create(rz_ctx* ctx, int64_t capacity, rz_keyindex** out) {
    if (!ctx || !out || capacity < 1 || capacity > (int64_t(1) << 31)) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    uint64_t cap = 2;
    while (cap < uint64_t(capacity)) cap <<= 1;
    rz_keyindex* ix = new (std::nothrow) rz_keyindex();
    if (!ix) return RZ_ERR_NO_MEMORY;
    ix->ctx = ctx;
    ix->mask = uint32_t(cap - 1);
    cudaError_t e = cudaMalloc(&ix->keys, cap * 8);
    if (e == cudaSuccess) e = cudaMalloc(&ix->rows, cap * 4);
    if (e == cudaSuccess) e = cudaMalloc(&ix->status, 4);
    if (e == cudaSuccess) e = cudaMemset(ix->status, 0, 4);
    if (e == cudaSuccess) e = cudaMemset(ix->keys, 0xff, cap * 8);
    if (e == cudaSuccess) e = cudaMallocHost(&ix->h_status, 4);
    if (e != cudaSuccess) {
        const int st = cuda_fail(ctx, e, "rz_keyindex_create");
        cudaFree(ix->keys);
        cudaFree(ix->rows);
        cudaFree(ix->status);
        delete ix;
        return st;
    }
    *out = ix;
    return RZ_OK;
}

void rz_keyindex_destroy(rz_keyindex* ix) {
    if (!ix) return;
    cudaSetDevice(ix->ctx->device);
    cudaFree(ix->keys);
    cudaFree(ix->rows);
    cudaFree(ix->status);
    cudaFree(ix->del_rows);
    cudaFree(ix->del_slots);
    if (ix->h_status) cudaFreeHost(ix->h_status);
    delete ix;
}

int rz_keyindex_insert(rz_keyindex* ix, const void* d_data, int64_t first, int64_t count, uint32_t record_bytes,
                       rz_stream_t stream) {
    if (!ix || !key_record(record_bytes) || first < 0 || count < 0 || first + count > (int64_t(1) << 32) - 1 ||
        (count > 0 && !d_data))
        return RZ_ERR_INVALID_ARG;
    rz_ctx* ctx = ix->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (count > 0) {
        ix_insert_kernel<<<grid_for(ctx, count), 256, 0, s>>>(ix->keys, ix->rows, ix->mask,
                                                              static_cast<const uint8_t*>(d_data), record_bytes,
                                                              uint32_t(first), uint32_t(count), ix->status);
        RZ_CUDA_TRY(ctx, cudaGetLastError());
    }
    uint32_t bits = 0;
    const int st = ix_status(ix, s, &bits);
    return st != RZ_OK ? st : ix_map(bits);
}

int rz_keyindex_build(rz_keyindex* ix, const void* d_data, int64_t n, uint32_t record_bytes, rz_stream_t stream) {
    if (!ix) return RZ_ERR_INVALID_ARG;
    rz_ctx* ctx = ix->ctx;
    {
        std::lock_guard<std::recursive_mutex> lock(ctx->mu);
        cudaSetDevice(ctx->device);
        RZ_CUDA_TRY(ctx, cudaMemsetAsync(ix->keys, 0xff, (size_t(ix->mask) + 1) * 8,
                                         reinterpret_cast<cudaStream_t>(stream)));
    }
    return rz_keyindex_insert(ix, d_data, 0, n, record_bytes, stream);
}

int rz_keyindex_find(rz_keyindex* ix, const uint64_t* d_keys, int64_t count, uint32_t* d_rows, rz_stream_t stream) {
    if (!ix || count < 0 || (count > 0 && (!d_keys || !d_rows)) || count > (int64_t(1) << 32) - 1)
        return RZ_ERR_INVALID_ARG;
    rz_ctx* ctx = ix->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    if (count == 0) return RZ_OK;
    ix_lookup_kernel<<<grid_for(ctx, count), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        ix->keys, ix->rows, ix->mask, reinterpret_cast<const unsigned long long*>(d_keys), uint32_t(count), d_rows,
        nullptr, ix->status);
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    return RZ_OK;
}

int rz_remove_by_key(rz_ctx* ctx, rz_keyindex* ix, void* d_data, int64_t n, uint32_t record_bytes,
                     const uint64_t* d_keys, int64_t k, int64_t* new_len, uint32_t flags, rz_stream_t stream) {
    if (!ctx || !ix || ix->ctx != ctx || !key_record(record_bytes) || n < 0 || k < 0 || k > n ||
        n >= (int64_t(1) << 32) || (k > 0 && (!d_keys || !d_data)))
        return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (new_len) *new_len = n - k;
    if (k == 0) return RZ_OK;
    if (size_t(k) > ix->del_cap) {
        cudaFree(ix->del_rows);
        cudaFree(ix->del_slots);
        ix->del_rows = ix->del_slots = nullptr;
        ix->del_cap = 0;
        const size_t cap = std::max<size_t>(size_t(k), 1024);
        RZ_CUDA_TRY(ctx, cudaMalloc(&ix->del_rows, cap * 4));
        RZ_CUDA_TRY(ctx, cudaMalloc(&ix->del_slots, cap * 4));
        ix->del_cap = cap;
    }
    // 1. rows of the keys; any missing key fails the call before anything changes.
    ix_lookup_kernel<<<grid_for(ctx, k), 256, 0, s>>>(ix->keys, ix->rows, ix->mask,
                                                     reinterpret_cast<const unsigned long long*>(d_keys),
                                                     uint32_t(k), ix->del_rows, ix->del_slots, ix->status);
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    uint32_t bits = 0;
    int st = ix_status(ix, s, &bits);
    if (st != RZ_OK) return st;
    if (bits) return ix_map(bits);
    // 2. the removal itself (duplicates among the keys give duplicate rows: RZ_VALIDATE catches
    //    them before any data moves), then 3. erase the deleted keys and re-point the moved ones.
    int64_t nl = 0;
    st = rz_remove(ctx, d_data, n, record_bytes, ix->del_rows, k, &nl, (flags | RZ_VALIDATE) & ~RZ_SYNC, stream);
    if (st != RZ_OK) return st;
    st = read_status(ctx, s);
    if (st != RZ_OK) return st;
    ix_erase_kernel<<<grid_for(ctx, k), 256, 0, s>>>(ix->keys, ix->del_slots, uint32_t(k));
    ix_repoint_kernel<<<grid_for(ctx, k), 256, 0, s>>>(ix->keys, ix->rows, ix->mask, static_cast<const uint8_t*>(d_data),
                                                      record_bytes, ix->del_rows, uint32_t(k), uint32_t(n - k));
    RZ_CUDA_TRY(ctx, cudaGetLastError());
    if (flags & RZ_SYNC) RZ_CUDA_TRY(ctx, cudaStreamSynchronize(s));
    return RZ_OK;
}

}  // extern "C"
