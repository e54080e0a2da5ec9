// A host program written against include/redzone.hpp, the reference-shaped C++ call: it makes
// a device list, removes the indices read from a file with redzone::RemoveFromList (int list and
// 16-byte records), and writes the surviving prefixes for the Python test to check against the
// oracle. It also checks that a duplicate index under RZ_VALIDATE comes back as redzone::Error.
//   shim_main <index file (uint32)> <n> <out file>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <vector>

#include "redzone.hpp"

struct Rec {
    uint32_t a, b, c, d;
};

static void fail(const char* what) {
    std::fprintf(stderr, "shim_main: %s\n", what);
    std::exit(1);
}

int main(int argc, char** argv) {
    if (argc != 4) fail("usage: shim_main <index file> <n> <out file>");
    const long n = std::atol(argv[2]);
    std::FILE* f = std::fopen(argv[1], "rb");
    if (!f) fail("cannot open the index file");
    std::vector<int> idx;
    int v;
    while (std::fread(&v, sizeof(v), 1, f) == 1) idx.push_back(v);
    std::fclose(f);
    const int k = int(idx.size());

    std::vector<int> list(n);
    std::vector<Rec> recs(n);
    for (long i = 0; i < n; ++i) {
        list[i] = int(i);
        recs[i] = Rec{uint32_t(i), uint32_t(i) ^ 0xA5A5A5A5u, uint32_t(3 * i), ~uint32_t(i)};
    }
    int *d_list = nullptr, *d_idx = nullptr;
    Rec* d_recs = nullptr;
    if (cudaMalloc(&d_list, n * sizeof(int)) != cudaSuccess || cudaMalloc(&d_recs, n * sizeof(Rec)) != cudaSuccess ||
        cudaMalloc(&d_idx, (k + 1) * sizeof(int)) != cudaSuccess)
        fail("cudaMalloc");
    cudaMemcpy(d_list, list.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(d_recs, recs.data(), n * sizeof(Rec), cudaMemcpyHostToDevice);
    cudaMemcpy(d_idx, idx.data(), k * sizeof(int), cudaMemcpyHostToDevice);

    redzone::Context ctx(0);
    // The reference's argument order and types: (List, Length, Removals, RemoveCount).
    const int64_t len1 = redzone::RemoveFromList(ctx, d_list, int(n), d_idx, k, nullptr, RZ_SYNC);
    const int64_t len2 = redzone::RemoveFromList(ctx, d_recs, int(n), d_idx, k, nullptr, RZ_SYNC);
    if (len1 != n - k || len2 != n - k) fail("new length");
    cudaMemcpy(list.data(), d_list, n * sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(recs.data(), d_recs, n * sizeof(Rec), cudaMemcpyDeviceToHost);

    // A repeated index with RZ_VALIDATE: the call throws and leaves the list as it was.
    int code = 0;
    if (k >= 2) {
        cudaMemcpy(d_idx + 1, d_idx, sizeof(int), cudaMemcpyDeviceToDevice);
        try {
            redzone::RemoveFromList(ctx, d_list, int(n), d_idx, k, nullptr, RZ_VALIDATE | RZ_SYNC);
        } catch (const redzone::Error& e) {
            code = e.code();
        }
    }
    std::vector<int> after(n);
    cudaMemcpy(after.data(), d_list, n * sizeof(int), cudaMemcpyDeviceToHost);
    for (long i = 0; i < n; ++i)
        if (after[i] != list[i]) fail("a rejected call changed the list");

    std::FILE* o = std::fopen(argv[3], "wb");
    if (!o) fail("cannot open the output file");
    std::fwrite(&code, sizeof(code), 1, o);
    std::fwrite(list.data(), sizeof(int), size_t(n - k), o);
    std::fwrite(recs.data(), sizeof(Rec), size_t(n - k), o);
    std::fclose(o);
    cudaFree(d_list);
    cudaFree(d_recs);
    cudaFree(d_idx);
    return 0;
}
