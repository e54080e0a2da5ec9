// rz_autotune.cpp -- exhaustive autotuner and tuning tables.
//
// The reference fixes its launch configuration at compile time (GPUBlockCount / GPUBlockSize,
// tests.cu:1-2; prefetch depth 5, redzone.hxx:1134). Here every call can pick its configuration:
// rz_autotune_single times the 63-point space (block 128/256/512/1024 x items per thread 1/2/4/8
// x grid scale 1/2/4 with the schedule chosen by k, eight cluster-scan, four scan-all and three
// split launches) plus the O(n) partition path with CUDA events and an L2 flush between
// repetitions; rz_autotune_batched does the same for the batched kernel's tile and grid. The
// winners go into a per-context table keyed by (payload width, log2 k) that rz_remove and
// rz_batch_plan_create consult, and which can be saved to and loaded from a text file.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "rz_internal.h"

namespace rz {

struct TuneTable {
    std::map<std::pair<uint32_t, int>, rz_launch_cfg> single;  // (w, log2k) -> cfg
    std::map<uint32_t, rz_batch_cfg> batched;                  // w -> cfg
    void* scrub = nullptr;                                      // 256 MiB L2 flush buffer (tuning only)
};

static TuneTable* table(rz_ctx* ctx) {
    if (!ctx->tune_table) ctx->tune_table = new TuneTable();
    return static_cast<TuneTable*>(ctx->tune_table);
}

static int log2_bucket(uint32_t k) {
    int b = 0;
    while ((1u << (b + 1)) <= k && b < 31) ++b;
    // round to nearest power of two
    if (b < 31 && double(k) >= 1.4142135623730951 * double(1u << b)) ++b;
    return b;
}

bool tuned_cfg(rz_ctx* ctx, uint32_t n, uint32_t k, uint32_t w, rz_launch_cfg* cfg) {
    (void)n;
    if (!ctx->tune_table) return false;
    TuneTable* t = table(ctx);
    const int b = log2_bucket(k);
    const rz_launch_cfg* best = nullptr;
    int bestd = 1 << 30;
    for (auto& kv : t->single) {
        if (kv.first.first != w) continue;
        const int d = std::abs(kv.first.second - b);
        if (d < bestd) {
            bestd = d;
            best = &kv.second;
        }
    }
    if (!best || bestd > 2) return false;
    *cfg = *best;
    return true;
}

// The best fixed configuration of the batched kernel over 1,000 timed list mixes on B200:
// 512 x 4 x 4, wavefront order, for items of up to 16 bytes (7.1 % mean regret against
// exhaustive autotune on the 100 held-out mixes). For 32-byte items 256 x 4 x 4, wavefront order:
// the streaming service's records (2^27 x 32 bytes) sustain 4.7e9 rows/s with it, and on an
// earlier build 4.45e9 against 4.13e9 with 256 x 8 x 4 phase by phase, the best fixed choice on
// the timed mixes of that build.
bool default_batch_cfg(const rz_ctx* ctx, uint32_t w, rz_batch_cfg* cfg) {
    cfg->block = 512;
    cfg->items = 4;
    cfg->ctas_per_sm = 4;
    cfg->span = 0;
    cfg->wave = kDefaultWave;
    if (w >= 32) cfg->block = 256;
    if (ctx->tune_table) {
        TuneTable* t = static_cast<TuneTable*>(ctx->tune_table);
        auto it = t->batched.find(w);
        if (it != t->batched.end()) {
            *cfg = it->second;
            return true;
        }
    }
    return false;
}

void release_tune(rz_ctx* ctx) {
    if (!ctx->tune_table) return;
    TuneTable* t = static_cast<TuneTable*>(ctx->tune_table);
    if (t->scrub) cudaFree(t->scrub);
    delete t;
    ctx->tune_table = nullptr;
}

static int ensure_scrub(rz_ctx* ctx) {
    TuneTable* t = table(ctx);
    if (!t->scrub) RZ_CUDA_TRY(ctx, cudaMalloc(&t->scrub, size_t(256) << 20));
    return RZ_OK;
}

// The space in a fixed order (the predictor's class index is the position here). A cluster-scan,
// scan-all or split point that does not run for an instance (k > 2^17, a slice too long for the
// block, wide items on 512 threads, a misaligned index list) runs another schedule (the grid, or
// the cluster schedule for a short list) with the same block and items.
void config_space(rz_launch_cfg* out) {
    static const int blocks[4] = {128, 256, 512, 1024};
    static const int items[4] = {1, 2, 4, 8};
    static const int gs[3] = {1, 2, 4};
    static const int cscan[8][2] = {{128, 2}, {128, 4}, {256, 1}, {256, 2}, {256, 4}, {256, 8}, {512, 2}, {512, 4}};
    int q = 0;
    for (int b : blocks)
        for (int i : items)
            for (int g : gs) out[q++] = rz_launch_cfg{b, i, g, 0, RZ_SCHED_AUTO};
    for (const auto& c : cscan) out[q++] = rz_launch_cfg{c[0], c[1], 2, 0, RZ_SCHED_CSCAN};
    for (int i : {1, 2, 4, 8}) out[q++] = rz_launch_cfg{256, i, 2, 0, RZ_SCHED_SCANALL};
    for (int i : {1, 2, 4}) out[q++] = rz_launch_cfg{256, i, 2, 0, RZ_SCHED_SPLIT};
}

}  // namespace rz

using namespace rz;

extern "C" {

int rz_config_space(rz_launch_cfg* out, int32_t max) {
    rz_launch_cfg space[kConfigSpace];
    config_space(space);
    for (int q = 0; q < kConfigSpace && q < max && out; ++q) out[q] = space[q];
    return kConfigSpace;
}

int rz_autotune_single(rz_ctx* ctx, void* d_data, int64_t n, uint32_t w, const uint32_t* d_idx, int64_t k,
                       int32_t reps, rz_tune_entry* out, int32_t max_out, int32_t* count) {
    if (!ctx || !out || max_out < 1 || reps < 1) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    int st = ensure_scrub(ctx);
    if (st != RZ_OK) return st;
    TuneTable* t = table(ctx);
    rz_launch_cfg space[kConfigSpace + 1];
    config_space(space);
    space[kConfigSpace] = rz_launch_cfg{256, 8, 1, 1, RZ_SCHED_AUTO};  // the partition path
    cudaStream_t s = nullptr;
    RZ_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<rz_tune_entry> res;
    for (int q = 0; q <= kConfigSpace; ++q) {
        std::vector<float> ms;
        st = rz_remove_cfg(ctx, d_data, n, w, d_idx, k, &space[q], 0, reinterpret_cast<rz_stream_t>(s));  // warm-up
        if (st != RZ_OK) break;
        for (int r = 0; r < reps; ++r) {
            cudaMemsetAsync(t->scrub, r & 0xff, size_t(256) << 20, s);
            cudaEventRecord(e0, s);
            st = rz_remove_cfg(ctx, d_data, n, w, d_idx, k, &space[q], 0, reinterpret_cast<rz_stream_t>(s));
            cudaEventRecord(e1, s);
            if (st != RZ_OK) break;
            cudaEventSynchronize(e1);
            float x = 0;
            cudaEventElapsedTime(&x, e0, e1);
            ms.push_back(x);
        }
        if (st != RZ_OK) break;
        std::sort(ms.begin(), ms.end());
        res.push_back(rz_tune_entry{space[q], ms[ms.size() / 2]});
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (st != RZ_OK) return st;
    const int rd = read_status(ctx, nullptr);
    if (rd != RZ_OK) return rd;
    std::sort(res.begin(), res.end(), [](const rz_tune_entry& a, const rz_tune_entry& b) { return a.ms < b.ms; });
    const int m = std::min<int>(max_out, int(res.size()));
    for (int q = 0; q < m; ++q) out[q] = res[size_t(q)];
    if (count) *count = m;
    return RZ_OK;
}

int rz_autotune_batched(rz_ctx* ctx, const rz_list_desc* lists, int32_t nlists, uint32_t w, int32_t reps,
                        rz_batch_cfg* best, float* best_ms) {
    if (!ctx || !best || reps < 1) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    int st = ensure_scrub(ctx);
    if (st != RZ_OK) return st;
    TuneTable* t = table(ctx);
    std::vector<rz_batch_cfg> cands(kBatchCfgSpace);
    batch_config_space(cands.data());
    cudaStream_t s = nullptr;
    RZ_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float bms = 1e30f;
    for (const rz_batch_cfg& c : cands) {
        rz_batch_plan* plan = nullptr;
        const int ps = rz_batch_plan_create(ctx, lists, nlists, w, &c, &plan);
        if (ps != RZ_OK) continue;  // infeasible (e.g. a list needs more chunks than the tile allows)
        std::vector<float> ms;
        st = rz_batch_plan_launch(plan, reinterpret_cast<rz_stream_t>(s));
        for (int r = 0; r < reps && st == RZ_OK; ++r) {
            cudaMemsetAsync(t->scrub, r & 0xff, size_t(256) << 20, s);
            cudaEventRecord(e0, s);
            st = rz_batch_plan_launch(plan, reinterpret_cast<rz_stream_t>(s));
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float x = 0;
            cudaEventElapsedTime(&x, e0, e1);
            ms.push_back(x);
        }
        cudaStreamSynchronize(s);
        rz_batch_plan_destroy(plan);
        if (st != RZ_OK) break;
        std::sort(ms.begin(), ms.end());
        const float med = ms[ms.size() / 2];
        if (med < bms) {
            bms = med;
            *best = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if (st != RZ_OK) return st;
    if (bms >= 1e29f) return RZ_ERR_UNSUPPORTED;
    if (best_ms) *best_ms = bms;
    return read_status(ctx, nullptr);
}

int rz_tune_table_set_single(rz_ctx* ctx, uint32_t w, int32_t log2k, const rz_launch_cfg* cfg) {
    if (!ctx || !cfg) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    table(ctx)->single[{w, log2k}] = *cfg;
    return RZ_OK;
}

int rz_tune_table_set_batched(rz_ctx* ctx, uint32_t w, const rz_batch_cfg* cfg) {
    if (!ctx || !cfg) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    table(ctx)->batched[w] = *cfg;
    return RZ_OK;
}

int rz_tune_table_save(rz_ctx* ctx, const char* path) {
    if (!ctx || !path) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    FILE* f = std::fopen(path, "w");
    if (!f) return RZ_ERR_INVALID_ARG;
    std::fprintf(f, "# redzone_b200 tuning table\n");
    TuneTable* t = table(ctx);
    for (auto& kv : t->single)
        std::fprintf(f, "single %u %d %d %d %d %d %d\n", kv.first.first, kv.first.second, kv.second.block,
                     kv.second.items, kv.second.ctas_per_sm, kv.second.use_partition, kv.second.schedule);
    for (auto& kv : t->batched)
        std::fprintf(f, "batched %u %d %d %d %d\n", kv.first, kv.second.block, kv.second.items, kv.second.ctas_per_sm,
                     kv.second.wave);
    std::fclose(f);
    return RZ_OK;
}

int rz_tune_table_load(rz_ctx* ctx, const char* path) {
    if (!ctx || !path) return RZ_ERR_INVALID_ARG;
    std::lock_guard<std::recursive_mutex> g(ctx->mu);
    FILE* f = std::fopen(path, "r");
    if (!f) return RZ_ERR_INVALID_ARG;
    TuneTable* t = table(ctx);
    char line[256];
    int bad = 0;
    while (std::fgets(line, sizeof(line), f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        char kind[16] = {0};
        unsigned w = 0;
        int a = 0, b = 0, c = 0, d = 0, e = 0, sc = 0;
        if (std::sscanf(line, "%15s", kind) != 1) continue;
        if (std::strcmp(kind, "single") == 0) {
            const int got = std::sscanf(line, "%*s %u %d %d %d %d %d %d", &w, &a, &b, &c, &d, &e, &sc);
            if (got < 6) {
                ++bad;
                continue;
            }
            t->single[{w, a}] = rz_launch_cfg{b, c, d, e, got >= 7 ? sc : RZ_SCHED_AUTO};
        } else if (std::strcmp(kind, "batched") == 0) {
            int wave = 0;  // optional fifth number (older tables have four)
            if (std::sscanf(line, "%*s %u %d %d %d %d", &w, &a, &b, &c, &wave) < 4) {
                ++bad;
                continue;
            }
            t->batched[w] = rz_batch_cfg{a, b, c, 0, wave};
        } else {
            ++bad;
        }
    }
    std::fclose(f);
    return bad ? RZ_ERR_INVALID_ARG : RZ_OK;
}

}  // extern "C"
