// rz_internal.h -- host-side declarations shared by the translation units of the library.
#pragma once

#include <cstddef>
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/redzone.h"

namespace rz {

constexpr int kMaxGrid = 1024;           // upper bound on CTAs of the persistent single-list kernel
constexpr int kStampsPerCta = 8;         // phase timestamps recorded per CTA when enabled
constexpr uint32_t kSpinLimit = 1u << 22;  // polls of a bounded device wait (~0.5-1 s with backoff)
// Red-list schedule of the grid kernel (one tile per CTA): every CTA publishes its red-zone
// entries with its arrival, and when the whole grid has at most kFastMaxRed of them each CTA
// derives the orphan pairing from that list in shared memory (no orphan-count exchange).
constexpr uint32_t kFastMaxK = 1u << 17;   // k bound: two k-bit maps live in shared memory
// The grid kernel's red-list schedule goes further: its two k-bit maps take 128 KB at 2^19 (one
// CTA per SM). Above kFastMaxK it is chosen only when uniform removals would leave at most
// kFastMaxRed red entries (k^2 / n), since a grid with more falls back to the bitmap phases.
constexpr uint32_t kRedlistMaxK = 1u << 19;
constexpr uint32_t kFastMaxRed = 1024;     // red entries of the whole grid

// Library scratch owned by one context. Every buffer is zero where the kernels require it on
// entry and is left zero on exit (the kernels clear what they set), so no per-call memset is
// needed; `dirty` forces a full re-zero after a call that ended with a device error.
struct Workspace {
    uint32_t* status = nullptr;      // device status word (ST_* bits)
    uint32_t* bitmap = nullptr;      // red-zone bitmap, k bits
    size_t bitmap_words = 0;
    uint32_t* dlist = nullptr;       // destination orphans (per-CTA regions), k entries
    uint32_t* slist = nullptr;       // source-orphan positions (per-CTA regions), k entries
    size_t list_cap = 0;
    uint32_t* seen = nullptr;        // RZ_VALIDATE: n-bit occupancy map
    size_t seen_words = 0;
    uint32_t* part_bits = nullptr;   // partition path: n-bit removal map
    size_t part_words = 0;
    unsigned long long* tile_state = nullptr;  // partition path: ticket, staged/kept/offset per tile
    size_t tile_cap = 0;
    unsigned long long* dev_len = nullptr;     // device copy of the last new length
    uint32_t* idx_stage = nullptr;   // rz_remove_host_idx: device copy of host indices
    size_t stage_cap = 0;
    uint4* keep_stage = nullptr;     // rz_keep: the kept items, 16-byte units
    size_t keep_cap = 0;
    uint32_t* epoch = nullptr;       // grid schedule: call epoch (advanced by CTA 0 each call)
    uint32_t* split_count = nullptr; // split schedule: red entries listed, pairing CTAs done (reset by the last)
    uint32_t* arrive = nullptr;      // grid schedule: per-CTA arrival tags, kMaxGrid
    unsigned long long* cnt_words = nullptr;  // grid schedule: tagged orphan counts, 2*kMaxGrid
    unsigned long long* arrive64 = nullptr;   // red-list schedule: tag << 32 | red entries, kMaxGrid
    uint2* redlist = nullptr;        // red-list schedule: {position, value - cut} per red entry, k
    size_t red_cap = 0;
    unsigned long long* stamps = nullptr;     // optional phase timestamps, 8 per CTA
    uint8_t* h_result = nullptr;     // pinned host copy of [status .. dev_len] (one D2H per sync)
    bool stamps_on = false;
    bool dirty = false;
};

}  // namespace rz

struct rz_ctx {
    int device = 0;
    int sms = 0;
    size_t smem_optin = 0;
    rz::Workspace ws;
    std::string last_cuda_error;
    std::recursive_mutex mu;
    int last_kernels = 0;        // kernels launched by the most recent removal call
    int last_grid = 0;
    int last_block = 0;
    void* predictor = nullptr;   // rz::Predictor*, owned (see rz_mlp.cu)
    void* tune_table = nullptr;  // rz::TuneTable*, owned (see rz_autotune.cpp)
    void* async_pipe = nullptr;  // rz::AsyncPipe*, owned (see rz_async.cpp)
    size_t scratch_held = 0;     // bytes of grown context scratch
    size_t scratch_limit = ~size_t(0);  // rz_set_scratch_limit: growth beyond it -> RZ_ERR_NO_MEMORY
    cudaEvent_t done_event = nullptr;    // completion of a synchronous call's last copy (polled)
};

namespace rz {

// Record a CUDA error in the context and map it to RZ_ERR_CUDA.
int cuda_fail(rz_ctx* ctx, cudaError_t e, const char* where);
#define RZ_CUDA_TRY(ctx, call)                                   \
    do {                                                         \
        cudaError_t _e = (call);                                 \
        if (_e != cudaSuccess) return ::rz::cuda_fail((ctx), _e, #call); \
    } while (0)

// Grow-only scratch allocation; returns RZ_OK or an error code.
int ensure_lists(rz_ctx* ctx, size_t k);
int ensure_seen(rz_ctx* ctx, size_t n);
int ensure_partition(rz_ctx* ctx, size_t n, size_t ntiles);
int reset_if_dirty(rz_ctx* ctx, cudaStream_t s);

// Kernel launchers (rz_single.cu).
struct LaunchInfo {
    int grid = 0;
    int block = 0;
    int items = 0;
    int launches = 0;  // kernels launched by this call
};
int launch_redzone(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx,
                   uint32_t k, const rz_launch_cfg& cfg, uint32_t flags, cudaStream_t s,
                   LaunchInfo* info);
int launch_partition(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx,
                     uint32_t k, uint32_t flags, cudaStream_t s, LaunchInfo* info);
// Cluster-scan schedule (rz_cscan.cu); RZ_ERR_UNSUPPORTED when a slice of the index list does not
// fit one register pass, the maps do not fit in shared memory, the index list is not 16-byte
// aligned or no cluster can be co-scheduled.
int launch_cscan(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx, uint32_t k,
                 const rz_launch_cfg& cfg, bool validate, cudaStream_t s, LaunchInfo* info);
// The default cluster-scan launch for (k, w), if that schedule runs it: false otherwise.
bool cscan_default_cfg(const rz_ctx* ctx, uint32_t k, uint32_t w, rz_launch_cfg* cfg);
constexpr uint32_t kScanAllMaxK = 1u << 12;      // the default uses the scan-all schedule up to here
constexpr uint32_t kCscanMinK = (1u << 12) + 1;  // the default uses the cluster scan from here
constexpr uint32_t kCscanMaxK = 1u << 17;       // ... to here (one register pass per slice)
// Cluster schedule (rz_cluster.cu); RZ_ERR_UNSUPPORTED when the bitmap slice does not fit in
// shared memory or no cluster of the requested size can be co-scheduled.
// Split schedule (rz_produced.cu); RZ_ERR_UNSUPPORTED for k > kFastMaxK or too little shared memory.
int launch_split(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx, uint32_t k,
                 const rz_launch_cfg& cfg, bool validate, cudaStream_t s, LaunchInfo* info);
// Scan-all schedule (rz_produced.cu); RZ_ERR_UNSUPPORTED for k > kFastMaxK, a misaligned list or
// too little shared memory.
int launch_scanall(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx, uint32_t k,
                   const rz_launch_cfg& cfg, bool validate, cudaStream_t s, LaunchInfo* info);
int launch_cluster(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* idx, uint32_t k,
                   const rz_launch_cfg& cfg, bool validate, cudaStream_t s, LaunchInfo* info);
int cluster_max_block(int w, int items);
constexpr uint32_t kClusterMaxK = 1u << 14;  // RZ_SCHED_AUTO uses the cluster schedule up to here
// The launch-configuration space in its canonical order (rz_autotune.cpp): 48 grid / cluster
// points (block x items x grid scale, schedule chosen by k), 8 cluster-scan, 4 scan-all and 3
// split points.
constexpr int kConfigSpace = 63;
void config_space(rz_launch_cfg* out);
int launch_validate(rz_ctx* ctx, uint32_t n, const uint32_t* idx, uint32_t k, cudaStream_t s);
// rz_keep: gather data[keep[j]] into `stage` (m items), then copy the stage to data[0..m).
int launch_keep(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* keep, uint32_t m, void* stage,
                cudaStream_t s);
// Largest block size the single-list kernel for (w, items) can launch with.
int redzone_max_block(int w, int items);
// CTAs per SM the single-list kernel for (w, items, block) can keep resident.
int redzone_occupancy(int w, int items, int block, size_t dynamic_smem = 0);
int default_cfg(const rz_ctx* ctx, uint32_t n, uint32_t k, uint32_t w, rz_launch_cfg* cfg);
int clamp_cfg(const rz_ctx* ctx, uint32_t k, uint32_t w, rz_launch_cfg* cfg);

// Hooks implemented by the tuning / learned-predictor translation units.
bool predict_cfg(rz_ctx* ctx, uint32_t n, uint32_t k, uint32_t w, const uint32_t* d_idx,
                 cudaStream_t s, rz_launch_cfg* cfg);
bool tuned_cfg(rz_ctx* ctx, uint32_t n, uint32_t k, uint32_t w, rz_launch_cfg* cfg);
// The batched configuration space (rz_batch_config_space): block {128,256,512} x items {2,4,8} x
// CTAs per SM {1,2,4} x work order {phase by phase, wavefront with kDefaultWave}.
constexpr int kDefaultWave = 4;  // a lag of 2 grids' worth of items: 9.06 ms on 4096 lists against 9.40 with 6
constexpr uint32_t kBatchMaxTilesPerList = 1024;  // tiles one list of the batched kernel may span
constexpr int kBatchCfgSpace = 54;
void batch_config_space(rz_batch_cfg* out);
// The batched configuration the attached list-mix predictor picks (false without one).
bool predict_batch_cfg(rz_ctx* ctx, const rz_list_desc* lists, int nlists, uint32_t w, rz_batch_cfg* cfg);
void release_extras(rz_ctx* ctx);
// The status word (offset 0) and the device length (offset 512) of the workspace block: one
// device-to-host copy of this many bytes brings both back.
constexpr size_t kResultBytes = 512 + sizeof(unsigned long long);
// Wait for an event: poll (about 2 ms), then block. RZ_OK or RZ_ERR_CUDA.
int wait_event(rz_ctx* ctx, cudaEvent_t ev);
// Map device status bits (ST_* of rz_common.cuh) to an rz_status code, most severe first.
int map_status(uint32_t bits);
// Wait for the stream, then map the device status to rz_status (clearing it); with new_len, also
// read back the device-tracked length of the last call.
int read_status(rz_ctx* ctx, cudaStream_t s, int64_t* new_len = nullptr);

// Batched launches into preallocated scratch (rz_batched.cu), for the streaming service.
struct BatchArena;
int arena_create(rz_ctx* ctx, uint32_t w, const rz_batch_cfg* cfg, size_t max_lists, size_t max_k, BatchArena** out);
void arena_destroy(BatchArena* a);
int arena_launch(BatchArena* a, const rz_list_desc* lists, int nlists, cudaStream_t s);

// Test hook: run a grid barrier whose expected arrival count exceeds the grid, so that the
// bounded wait must expire; returns the device status bits observed.
int test_barrier_timeout(rz_ctx* ctx, uint32_t spin_limit, uint32_t* status_out);
// Diagnostic: plain scattered stores of `count` items at positions pos[] (the hole writes alone).
int test_scatter(rz_ctx* ctx, void* data, uint32_t n, uint32_t w, const uint32_t* pos, uint32_t count, cudaStream_t s);
// Diagnostic: launch an empty kernel of the given shape (cluster size 1-8 dividing grid).
int test_empty_launch(rz_ctx* ctx, int grid, int block, int cluster, int smem, cudaStream_t s);

}  // namespace rz
