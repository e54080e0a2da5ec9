// e2e_driver.cpp -- end-to-end timing of the host-index removal from C++, the way a program that
// called the reference's redzone_CPU (Redzone_CPU.hxx:150) in a loop would call this library
// instead: its removal lists live on the host (pinned), the list it removes from lives on the
// GPU, and every call's status and new length come back to the host.
//
//   rz_e2e <log2 n> <log2 k> <steps> <depth> [sets]
//
// Makes a device list of n int32 items (iota) and `sets` (default 64) host index lists of k
// distinct uniform positions each (seeded), then times `steps` calls of
// rz_remove_host_idx_async with up to `depth` calls in flight, every call collected with rz_wait
// (status checked, new length checked), between two CUDA events on the call stream; also the
// synchronous rz_remove_host_idx one call at a time. Prints one JSON object. Built by
// redzone_b200/build.py next to the library; bench.py runs it.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <unordered_set>
#include <vector>

#include "redzone.h"

static uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static int fail(const char* what, int code) {
    std::printf("{\"error\": \"%s\", \"status\": %d}\n", what, code);
    return 1;
}

int main(int argc, char** argv) {
    if (argc < 5) return fail("usage: rz_e2e <log2 n> <log2 k> <steps> <depth> [sets]", -1);
    const int64_t n = int64_t(1) << std::atoi(argv[1]);
    const int64_t k = int64_t(1) << std::atoi(argv[2]);
    const int steps = std::atoi(argv[3]);
    const int depth = std::atoi(argv[4]);
    const int sets = argc > 5 ? std::atoi(argv[5]) : 64;
    if (k > n / 2 || steps < 1 || depth < 1 || sets < 1) return fail("bad arguments", -1);

    // Host index lists: k distinct uniform positions each, pinned.
    uint32_t* h_idx = nullptr;
    if (cudaMallocHost(&h_idx, size_t(sets) * size_t(k) * 4) != cudaSuccess) return fail("cudaMallocHost", -1);
    for (int s = 0; s < sets; ++s) {
        uint64_t state = 0x5EEDull * 1000003ull + uint64_t(s);
        std::unordered_set<uint32_t> seen;
        seen.reserve(size_t(k) * 2);
        uint32_t* out = h_idx + size_t(s) * size_t(k);
        int64_t got = 0;
        while (got < k) {
            const uint32_t v = uint32_t(splitmix(state) % uint64_t(n));
            if (seen.insert(v).second) out[got++] = v;
        }
    }
    // Device list: iota.
    int32_t* d_list = nullptr;
    if (cudaMalloc(&d_list, size_t(n) * 4) != cudaSuccess) return fail("cudaMalloc", -1);
    {
        std::vector<int32_t> iota(static_cast<size_t>(n));
        for (int64_t i = 0; i < n; ++i) iota[size_t(i)] = int32_t(i);
        if (cudaMemcpy(d_list, iota.data(), size_t(n) * 4, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail("upload", -1);
    }
    rz_ctx* ctx = nullptr;
    int st = rz_create(&ctx, 0);
    if (st != RZ_OK) return fail("rz_create", st);
    cudaStream_t stream = nullptr;
    cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
    rz_stream_t rs = reinterpret_cast<rz_stream_t>(stream);

    auto issue = [&](int i, uint64_t* t) -> int {
        return rz_remove_host_idx_async(ctx, d_list, n, 4, h_idx + size_t(i % sets) * size_t(k), k, 0, rs, t);
    };
    auto collect = [&](uint64_t t) -> int {
        int64_t len = -1;
        const int s2 = rz_wait(ctx, t, &len);
        if (s2 != RZ_OK) return s2;
        return len == n - k ? RZ_OK : RZ_ERR_INVALID_ARG;
    };
    // Warm-up: the staging slots grow on first use.
    for (int i = 0; i < depth + 2; ++i) {
        uint64_t t = 0;
        if ((st = issue(i, &t)) != RZ_OK || (st = collect(t)) != RZ_OK) return fail("warm-up", st);
    }
    cudaStreamSynchronize(stream);

    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::deque<uint64_t> inflight;
    double issue_s = 0;
    cudaEventRecord(e0, stream);
    for (int i = 0; i < steps; ++i) {
        uint64_t t = 0;
        const auto h0 = std::chrono::steady_clock::now();
        st = issue(i, &t);
        issue_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - h0).count();
        if (st != RZ_OK) return fail("rz_remove_host_idx_async", st);
        inflight.push_back(t);
        if (int(inflight.size()) == depth) {
            if ((st = collect(inflight.front())) != RZ_OK) return fail("rz_wait", st);
            inflight.pop_front();
        }
    }
    while (!inflight.empty()) {
        if ((st = collect(inflight.front())) != RZ_OK) return fail("rz_wait", st);
        inflight.pop_front();
    }
    cudaEventRecord(e1, stream);
    cudaEventSynchronize(e1);
    float pipelined_ms = 0;
    cudaEventElapsedTime(&pipelined_ms, e0, e1);

    // The synchronous call, one at a time.
    const int sync_steps = steps < 200 ? steps : 200;
    cudaEventRecord(e0, stream);
    for (int i = 0; i < sync_steps; ++i) {
        int64_t len = -1;
        st = rz_remove_host_idx(ctx, d_list, n, 4, h_idx + size_t(i % sets) * size_t(k), k, &len, 0, rs);
        if (st != RZ_OK || len != n - k) return fail("rz_remove_host_idx", st);
    }
    cudaEventRecord(e1, stream);
    cudaEventSynchronize(e1);
    float sync_ms = 0;
    cudaEventElapsedTime(&sync_ms, e0, e1);

    std::printf("{\"ms_per_step\": %.6f, \"steps\": %d, \"depth\": %d, \"sets\": %d, \"host_issue_us_per_call\": %.3f, "
                "\"serial_ms_per_step\": %.6f, \"h2d_bytes_per_step\": %lld, \"d2h_bytes_per_step\": 16}\n",
                pipelined_ms / steps, steps, depth, sets, 1e6 * issue_s / steps, sync_ms / sync_steps,
                (long long)(k * 4));
    rz_destroy(ctx);
    cudaStreamDestroy(stream);
    cudaFree(d_list);
    cudaFreeHost(h_idx);
    return 0;
}
