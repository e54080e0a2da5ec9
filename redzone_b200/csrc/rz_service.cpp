// rz_service.cpp -- streaming delete service over a device-resident table.
//
// The table is split into `shards` independent sub-tables (each a contiguous run of
// shard_capacity records with its own live length). Delete batches (a shard and distinct live row
// indices) are submitted from the host at any time. A worker thread runs continuous batching:
//   * admission: a pending batch is admitted when its shard has no launch in flight (batches on
//     one shard are applied in submission order, since a removal moves that shard's rows), a slot
//     is free, and its indices fit the slot's share of the device index budget;
//   * coalescing: the admitted batches of one slot (distinct shards) run as one batched Redzone
//     launch (rz_batched.cu arenas: no allocation per launch);
//   * overlap: each slot has its own stream, so launches of different slots run concurrently and
//     batches keep being admitted while others are on the GPU;
//   * lengths: a device array holds every shard's live length; a small kernel after each launch
//     updates it on the GPU (the host keeps a mirror to plan the next launches);
//   * refill: before a batch would take a shard below floor_rows, the shard is refilled to its
//     capacity by appending fresh records (the paper's add-then-remove, Sec. 4.6); the new keys
//     depend only on the shard's own history, so results do not depend on the interleaving.
// Per-batch latency is submit -> completion as seen by the worker (CUDA event).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <random>
#include <thread>
#include <vector>

#include "rz_internal.h"

namespace rz {

using Clock = std::chrono::steady_clock;

struct SvcBatch {
    uint64_t ticket;
    int32_t shard;
    const uint32_t* h_idx;
    int64_t count;
    std::vector<uint32_t> owned;  // copy when the caller did not lend the buffer
    Clock::time_point arrival;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    BatchArena* arena = nullptr;
    uint32_t* d_idx = nullptr;     // index staging, capacity `cap_idx`
    size_t cap_idx = 0;
    int64_t* h_upd = nullptr;      // pinned: {shard, gain, k} triples for the length kernel
    bool busy = false;
    std::vector<SvcBatch> batches;
};

// Append g fresh records to shard s at rows [len, len + g): key = s << 40 | (appended + j).
__global__ void fill_records_kernel(uint32_t* rows, uint32_t words, uint64_t g, uint64_t key0) {
    for (uint64_t j = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; j < g; j += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t key = key0 + j;
        uint32_t* r = rows + j * words;
        r[0] = uint32_t(key);
        if (words > 1) r[1] = uint32_t(key >> 32);
        for (uint32_t q = 2; q < words; ++q) r[q] = uint32_t(key * 0x9e3779b97f4a7c15ull >> (8 * (q & 3))) ^ q;
    }
}

// Device-side length tracking: len[shard] += gain - k for each admitted batch of the launch.
__global__ void update_lengths_kernel(long long* len, const int64_t* upd, int m) {
    for (int q = threadIdx.x; q < m; q += blockDim.x) {
        const int64_t s = upd[3 * q], gain = upd[3 * q + 1], k = upd[3 * q + 2];
        len[s] += gain - k;
    }
}

}  // namespace rz

struct rz_service {
    rz_ctx* ctx = nullptr;
    uint8_t* table = nullptr;
    rz_service_cfg cfg{};
    std::vector<int64_t> len;         // host mirror of live lengths
    std::vector<int64_t> appended;    // records appended per shard so far (refill keys)
    std::vector<char> shard_busy;
    long long* d_len = nullptr;       // device-tracked lengths
    int64_t* d_upd = nullptr;         // per-slot update triples (device)
    std::vector<rz::Slot> slots;
    std::deque<rz::SvcBatch> pending;
    std::mutex mu;
    std::condition_variable cv, idle_cv;
    std::thread worker;
    std::atomic<bool> stop{false};
    uint64_t next_ticket = 1;
    int64_t in_flight = 0;            // submitted, not yet completed
    // stats
    int64_t submitted = 0, completed = 0, rejected = 0, rows_deleted = 0, launches = 0, refills = 0,
            rows_appended = 0, batches_launched = 0;
    std::vector<double> lat_us;
    rz::Clock::time_point first_submit{}, last_complete{};
    bool any_submit = false;
    int error = RZ_OK;
};

namespace rz {

static void launch_group(rz_service* S, Slot& slot) {
    rz_ctx* ctx = S->ctx;
    const uint32_t w = S->cfg.record_bytes;
    const int m = int(slot.batches.size());
    std::vector<rz_list_desc> lists(static_cast<size_t>(m));
    size_t off = 0;
    for (int q = 0; q < m; ++q) {
        SvcBatch& b = slot.batches[size_t(q)];
        const int s = b.shard;
        int64_t gain = 0;
        if (S->len[size_t(s)] - b.count < S->cfg.floor_rows) {
            gain = S->cfg.shard_capacity - S->len[size_t(s)];
            if (gain > 0) {
                uint8_t* rows = S->table + (size_t(s) * S->cfg.shard_capacity + size_t(S->len[size_t(s)])) * w;
                const uint64_t key0 = (uint64_t(s) << 40) | uint64_t(S->appended[size_t(s)]);
                const int grid = int(std::min<int64_t>(ctx->sms * 4, (gain + 255) / 256));
                fill_records_kernel<<<grid, 256, 0, slot.stream>>>(reinterpret_cast<uint32_t*>(rows), w / 4,
                                                                   uint64_t(gain), key0);
                S->appended[size_t(s)] += gain;
                S->len[size_t(s)] += gain;
                S->refills++;
                S->rows_appended += gain;
            }
        }
        cudaMemcpyAsync(slot.d_idx + off, b.h_idx, size_t(b.count) * 4, cudaMemcpyHostToDevice, slot.stream);
        lists[size_t(q)] = rz_list_desc{S->table + size_t(s) * S->cfg.shard_capacity * w, slot.d_idx + off,
                                        S->len[size_t(s)], b.count};
        slot.h_upd[3 * q] = s;
        slot.h_upd[3 * q + 1] = gain;
        slot.h_upd[3 * q + 2] = b.count;
        S->len[size_t(s)] -= b.count;
        off += size_t(b.count);
    }
    int st = arena_launch(slot.arena, lists.data(), m, slot.stream);
    const size_t si = size_t(&slot - S->slots.data());
    int64_t* d_upd = S->d_upd + si * size_t(3 * S->cfg.max_batches_per_launch);
    if (st == RZ_OK && cudaMemcpyAsync(d_upd, slot.h_upd, size_t(3 * m) * 8, cudaMemcpyHostToDevice, slot.stream) != cudaSuccess)
        st = RZ_ERR_CUDA;
    if (st == RZ_OK) update_lengths_kernel<<<1, 64, 0, slot.stream>>>(S->d_len, d_upd, m);
    if (st == RZ_OK && cudaEventRecord(slot.done, slot.stream) != cudaSuccess) st = RZ_ERR_CUDA;
    if (st != RZ_OK) S->error = st;
    slot.busy = true;
    S->launches++;
    S->batches_launched += m;
}

static void worker_loop(rz_service* S) {
    cudaSetDevice(S->ctx->device);
    const size_t slot_cap = S->slots.empty() ? 0 : S->slots[0].cap_idx;
    while (true) {
        bool progressed = false;
        // 1. completions
        for (Slot& slot : S->slots) {
            if (!slot.busy || cudaEventQuery(slot.done) != cudaSuccess) continue;
            const auto now = Clock::now();
            std::lock_guard<std::mutex> g(S->mu);
            for (SvcBatch& b : slot.batches) {
                S->lat_us.push_back(std::chrono::duration<double, std::micro>(now - b.arrival).count());
                S->shard_busy[size_t(b.shard)] = 0;
                S->completed++;
                S->rows_deleted += b.count;
                S->in_flight--;
            }
            S->last_complete = now;
            slot.batches.clear();
            slot.busy = false;
            progressed = true;
            S->idle_cv.notify_all();
        }
        // 2. admission: fill every free slot with pending batches of idle, distinct shards
        {
            std::unique_lock<std::mutex> g(S->mu);
            for (Slot& slot : S->slots) {
                if (slot.busy || S->pending.empty()) continue;
                std::vector<char> blocked(S->shard_busy.begin(), S->shard_busy.end());
                size_t used = 0;
                for (auto it = S->pending.begin(); it != S->pending.end();) {
                    if (int(slot.batches.size()) >= S->cfg.max_batches_per_launch) break;
                    const int s = it->shard;
                    if (blocked[size_t(s)]) {  // shard busy, or an earlier batch of it is waiting
                        blocked[size_t(s)] = 1;
                        ++it;
                        continue;
                    }
                    if (used + size_t(it->count) > slot_cap) break;  // the slot's index memory is full
                    used += size_t(it->count);
                    blocked[size_t(s)] = 1;
                    S->shard_busy[size_t(s)] = 1;
                    slot.batches.push_back(std::move(*it));
                    it = S->pending.erase(it);
                }
                if (!slot.batches.empty()) {
                    launch_group(S, slot);  // enqueues only; the lock guards the counters it updates
                    progressed = true;
                }
            }
            if (S->stop && S->pending.empty()) {
                bool busy = false;
                for (Slot& slot : S->slots) busy |= slot.busy;
                if (!busy) return;
            }
            if (!progressed) {
                bool busy = false;
                for (Slot& slot : S->slots) busy |= slot.busy;
                // Nothing in flight: sleep until a submission; otherwise poll the events again soon.
                if (!busy) S->cv.wait_for(g, std::chrono::milliseconds(2));
            }
        }
    }
}

}  // namespace rz

using namespace rz;

extern "C" {

int rz_service_create(rz_ctx* ctx, void* d_table, const int64_t* initial_len, const rz_service_cfg* cfg,
                      rz_service** out) {
    if (!ctx || !d_table || !cfg || !out) return RZ_ERR_INVALID_ARG;
    const rz_service_cfg& c = *cfg;
    if (c.shards < 1 || c.slots < 1 || c.shard_capacity < 1 || c.shard_capacity >= (int64_t(1) << 32) ||
        (c.record_bytes != 4 && c.record_bytes != 8 && c.record_bytes != 16 && c.record_bytes != 32) ||
        c.max_batches_per_launch < 1 || c.max_batches_per_launch > 4096 || c.index_budget_bytes < 4 * c.slots ||
        c.floor_rows < 0 || c.floor_rows > c.shard_capacity)
        return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    rz_service* S = new (std::nothrow) rz_service();
    if (!S) return RZ_ERR_NO_MEMORY;
    S->ctx = ctx;
    S->table = static_cast<uint8_t*>(d_table);
    S->cfg = c;
    S->len.assign(size_t(c.shards), c.shard_capacity);
    if (initial_len)
        for (int s = 0; s < c.shards; ++s) S->len[size_t(s)] = std::min(initial_len[s], c.shard_capacity);
    S->appended.assign(size_t(c.shards), 0);
    S->shard_busy.assign(size_t(c.shards), 0);
    int st = RZ_OK;
    cudaError_t e = cudaMalloc(&S->d_len, sizeof(long long) * size_t(c.shards));
    if (e == cudaSuccess) e = cudaMemcpy(S->d_len, S->len.data(), 8 * size_t(c.shards), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&S->d_upd, size_t(c.slots) * 3 * size_t(c.max_batches_per_launch) * 8);
    const size_t cap_idx = size_t(c.index_budget_bytes / 4 / c.slots);
    S->slots.resize(size_t(c.slots));
    for (Slot& slot : S->slots) {
        if (e != cudaSuccess) break;
        e = cudaStreamCreateWithFlags(&slot.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&slot.d_idx, cap_idx * 4);
        if (e == cudaSuccess) e = cudaMallocHost(&slot.h_upd, size_t(3 * c.max_batches_per_launch) * 8);
        slot.cap_idx = cap_idx;
        if (e == cudaSuccess) {
            st = arena_create(ctx, c.record_bytes, nullptr, size_t(c.max_batches_per_launch), cap_idx, &slot.arena);
            if (st != RZ_OK) break;
        }
    }
    if (e != cudaSuccess) st = cuda_fail(ctx, e, "rz_service_create");
    if (st != RZ_OK) {
        for (Slot& slot : S->slots) {
            if (slot.stream) cudaStreamDestroy(slot.stream);
            if (slot.done) cudaEventDestroy(slot.done);
            cudaFree(slot.d_idx);
            if (slot.h_upd) cudaFreeHost(slot.h_upd);
            arena_destroy(slot.arena);
        }
        cudaFree(S->d_len);
        cudaFree(S->d_upd);
        delete S;
        return st;
    }
    S->worker = std::thread(worker_loop, S);
    *out = S;
    return RZ_OK;
}

int rz_service_submit(rz_service* S, int32_t shard, const uint32_t* h_idx, int64_t count, uint32_t flags,
                      uint64_t* ticket) {
    if (!S || shard < 0 || shard >= S->cfg.shards || count < 0 || (count > 0 && !h_idx)) return RZ_ERR_INVALID_ARG;
    if (size_t(count) > S->slots[0].cap_idx) {
        std::lock_guard<std::mutex> g(S->mu);
        S->rejected++;
        return RZ_ERR_BUSY;  // larger than one slot's index memory: can never be admitted
    }
    SvcBatch b;
    b.shard = shard;
    b.count = count;
    if (flags & RZ_SUBMIT_BORROW) {
        b.h_idx = h_idx;
    } else {
        b.owned.assign(h_idx, h_idx + count);
        b.h_idx = b.owned.data();
    }
    b.arrival = Clock::now();
    {
        std::lock_guard<std::mutex> g(S->mu);
        if (!S->any_submit) {
            S->first_submit = b.arrival;
            S->any_submit = true;
        }
        b.ticket = S->next_ticket++;
        if (ticket) *ticket = b.ticket;
        S->submitted++;
        S->in_flight++;
        S->pending.push_back(std::move(b));
    }
    S->cv.notify_one();
    return RZ_OK;
}

int rz_service_drain(rz_service* S, int32_t timeout_ms) {
    if (!S) return RZ_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> g(S->mu);
    const bool ok = S->idle_cv.wait_for(g, std::chrono::milliseconds(timeout_ms), [&] { return S->in_flight == 0; });
    if (S->error != RZ_OK) return S->error;
    return ok ? RZ_OK : RZ_ERR_TIMEOUT;
}

int rz_service_stats_get(rz_service* S, rz_service_stats* out) {
    if (!S || !out) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(S->mu);
    rz_service_stats r{};
    r.submitted = S->submitted;
    r.completed = S->completed;
    r.rejected = S->rejected;
    r.rows_deleted = S->rows_deleted;
    r.launches = S->launches;
    r.refills = S->refills;
    r.rows_appended = S->rows_appended;
    r.mean_batches_per_launch = S->launches ? double(S->batches_launched) / double(S->launches) : 0.0;
    if (!S->lat_us.empty()) {
        std::vector<double> v = S->lat_us;
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) { return v[std::min(v.size() - 1, size_t(p * double(v.size() - 1) + 0.5))]; };
        r.p50_us = pct(0.50);
        r.p99_us = pct(0.99);
        r.max_us = v.back();
        double s = 0;
        for (double x : v) s += x;
        r.mean_us = s / double(v.size());
    }
    if (S->any_submit && S->completed)
        r.busy_seconds = std::chrono::duration<double>(S->last_complete - S->first_submit).count();
    *out = r;
    return RZ_OK;
}

int rz_service_reset_stats(rz_service* S) {
    if (!S) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(S->mu);
    S->submitted = S->completed = S->rejected = S->rows_deleted = S->launches = S->refills = S->rows_appended = 0;
    S->batches_launched = 0;
    S->lat_us.clear();
    S->any_submit = false;
    return RZ_OK;
}

int rz_service_lengths(rz_service* S, int64_t* host_view, int64_t* device_view) {
    if (!S) return RZ_ERR_INVALID_ARG;
    if (host_view) {
        std::lock_guard<std::mutex> g(S->mu);
        std::memcpy(host_view, S->len.data(), 8 * S->len.size());
    }
    if (device_view) {
        cudaSetDevice(S->ctx->device);
        for (Slot& slot : S->slots) cudaStreamSynchronize(slot.stream);
        RZ_CUDA_TRY(S->ctx, cudaMemcpy(device_view, S->d_len, 8 * S->len.size(), cudaMemcpyDeviceToHost));
    }
    return RZ_OK;
}

int rz_service_checkpoint(rz_service* S, int64_t* lengths, int64_t* appended, int32_t timeout_ms) {
    if (!S || !lengths || !appended) return RZ_ERR_INVALID_ARG;
    const int st = rz_service_drain(S, timeout_ms);
    if (st != RZ_OK) return st;
    std::lock_guard<std::mutex> g(S->mu);
    std::memcpy(lengths, S->len.data(), 8 * S->len.size());
    std::memcpy(appended, S->appended.data(), 8 * S->appended.size());
    return RZ_OK;
}

int rz_service_restore(rz_service* S, const int64_t* lengths, const int64_t* appended) {
    if (!S || !lengths || !appended) return RZ_ERR_INVALID_ARG;
    for (size_t s = 0; s < S->len.size(); ++s)
        if (lengths[s] < 0 || lengths[s] > S->cfg.shard_capacity || appended[s] < 0) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> g(S->mu);
    if (S->in_flight != 0) return RZ_ERR_BUSY;
    for (const Slot& slot : S->slots)
        if (slot.busy) return RZ_ERR_BUSY;
    std::memcpy(S->len.data(), lengths, 8 * S->len.size());
    std::memcpy(S->appended.data(), appended, 8 * S->appended.size());
    cudaSetDevice(S->ctx->device);
    RZ_CUDA_TRY(S->ctx, cudaMemcpy(S->d_len, S->len.data(), 8 * S->len.size(), cudaMemcpyHostToDevice));
    return RZ_OK;
}

void rz_service_destroy(rz_service* S) {
    if (!S) return;
    {
        std::lock_guard<std::mutex> g(S->mu);
        S->stop = true;
    }
    S->cv.notify_all();
    if (S->worker.joinable()) S->worker.join();
    cudaSetDevice(S->ctx->device);
    for (Slot& slot : S->slots) {
        cudaStreamSynchronize(slot.stream);
        cudaStreamDestroy(slot.stream);
        cudaEventDestroy(slot.done);
        cudaFree(slot.d_idx);
        cudaFreeHost(slot.h_upd);
        arena_destroy(slot.arena);
    }
    cudaFree(S->d_len);
    cudaFree(S->d_upd);
    delete S;
}

int rz_service_run_poisson(rz_service* S, const uint32_t* const* pool, const int64_t* pool_counts, int32_t pool_size,
                           double rate, double seconds, uint64_t seed, rz_service_stats* out) {
    if (!S || !pool || !pool_counts || pool_size < 1 || rate <= 0 || seconds <= 0) return RZ_ERR_INVALID_ARG;
    std::mt19937_64 rng(seed);
    std::exponential_distribution<double> gap(rate);
    std::uniform_int_distribution<int> pick(0, pool_size - 1), shard(0, S->cfg.shards - 1);
    const auto t0 = Clock::now();
    double t = 0;
    int st = RZ_OK;
    while (true) {
        t += gap(rng);
        if (t > seconds) break;
        const auto due = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(t));
        while (Clock::now() < due) {
        }
        const int q = pick(rng);
        const int rc = rz_service_submit(S, shard(rng), pool[q], pool_counts[q], RZ_SUBMIT_BORROW, nullptr);
        if (rc != RZ_OK && rc != RZ_ERR_BUSY) {
            st = rc;
            break;
        }
    }
    const int dr = rz_service_drain(S, 600000);
    if (st == RZ_OK) st = dr;
    if (out) rz_service_stats_get(S, out);
    return st;
}

}  // extern "C"
