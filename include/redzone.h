/*
 * redzone.h -- C-ABI of the B200-native Redzone O(k) in-place stream compaction library.
 *
 * The reference (JBontes/redzone) exposes two entry points for this path, both void and both
 * clobbering the removal list:
 *   - redzone.hxx:626-627   template<...> __device__ void RemoveFromList_GPUWide(T* List,
 *                           const int Length, int* Removals, const int RemoveCount,
 *                           BlockStorage_t<BlockCount>& BlockStore)   (cooperative launch by the
 *                           caller, T must be 4 bytes, new length implicitly Length-RemoveCount)
 *   - Redzone_CPU.hxx:150   void redzone_CPU(int* list, int listsize, int* removals,
 *                           int removecount, int(&times)[4])
 * This header replaces both with plain-pointer C functions. Every pointer named d_* is a device
 * pointer owned by the caller; the library owns its scratch. Nothing here aborts or traps:
 * errors come back as rz_status codes.
 *
 * Result contract (identical to the reference on the surviving prefix):
 *   cut = n - k. For i in [0,k): dest = idx[i], src = cut + i. A source is valid iff src is not
 *   itself in idx; a destination is valid iff dest < cut. Valid/valid pairs move data[src] to
 *   data[dest]. Valid destinations without a valid source form the destination-orphan list D
 *   (in i order); valid sources without a valid destination form the source-orphan list S (in i
 *   order); then data[D[j]] = data[S[j]]. Kept items below cut that are not removed never move.
 *   The tail [cut, n) is unspecified after the call (this implementation leaves it untouched);
 *   the index list is never written (the reference clobbers it).
 */
#ifndef REDZONE_B200_H
#define REDZONE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same object as cudaStream_t / CUstream; declared here so the header needs no CUDA headers. */
typedef struct CUstream_st* rz_stream_t;

typedef struct rz_ctx rz_ctx;

typedef enum rz_status {
    RZ_OK = 0,
    RZ_ERR_INVALID_ARG = 1,   /* null pointer, k > n, unsupported element size, misalignment   */
    RZ_ERR_DUPLICATE = 2,     /* RZ_VALIDATE: an index occurs twice                             */
    RZ_ERR_OUT_OF_RANGE = 3,  /* RZ_VALIDATE: an index >= n                                     */
    RZ_ERR_NO_MEMORY = 4,     /* scratch allocation failed or exceeded the context budget       */
    RZ_ERR_TIMEOUT = 5,       /* a bounded device wait (grid barrier, look-back) gave up        */
    RZ_ERR_CUDA = 6,          /* a CUDA runtime call failed (see rz_last_cuda_error)           */
    RZ_ERR_UNSUPPORTED = 7,   /* n >= 2^32, or a feature this build does not provide            */
    RZ_ERR_BUSY = 8           /* service: admission refused (memory budget or slots exhausted)  */
} rz_status;

/* Flags for rz_remove / rz_remove_batched. */
#define RZ_VALIDATE        0x1u  /* check indices for range and duplicates (O(k) extra passes)   */
#define RZ_SYNC            0x2u  /* synchronise the stream and return the device status          */
#define RZ_FORCE_PARTITION 0x4u  /* run the O(n) stable partition instead of Redzone             */
#define RZ_FORCE_BLOCK     0x8u  /* force the single-CTA schedule                                */
#define RZ_FORCE_GRID      0x10u /* force the grid-wide persistent schedule                      */
#define RZ_USE_PREDICTOR   0x20u /* let the trained MLP pick the launch configuration            */
#define RZ_ALLOW_STABLE    0x40u /* caller accepts the partition path's (stable) survivor order  */
#define RZ_CLOBBER_INDICES 0x80u /* caller allows the index list to be overwritten, as the       */
                                 /* reference does; accepted, but no path here ever writes it     */

/* Schedules of the single-list Redzone kernel. */
#define RZ_SCHED_AUTO    0  /* cluster for small/medium k, grid-wide otherwise                    */
#define RZ_SCHED_BLOCK   1  /* one CTA, block-level synchronisation                              */
#define RZ_SCHED_CLUSTER 2  /* one thread-block cluster; red-zone bitmap in distributed smem      */
#define RZ_SCHED_GRID    3  /* persistent grid, bounded global barriers                           */
#define RZ_SCHED_CSCAN   4  /* independent 8-CTA clusters, each finds every red entry; no grid wait */
#define RZ_SCHED_SPLIT   5  /* a scan grid lists the red entries; the pairing grid (launched as its */
                            /* programmatic dependent) reads them; no wait inside either grid     */
#define RZ_SCHED_SCANALL 6  /* one grid, every CTA reads the whole list; no wait (short lists)    */

/* Launch configuration of the single-list kernels (one entry of the 63-point tuning space:
 * block x items x grid scale with the schedule chosen by k, or a cluster-scan, scan-all or split
 * launch; plus the Redzone-vs-partition bit). */
typedef struct rz_launch_cfg {
    int32_t block;          /* threads per CTA: 128, 256, 512 or 1024                             */
    int32_t items;          /* items per thread per tile: 1, 2, 4 or 8                            */
    int32_t ctas_per_sm;    /* grid scale g in {1,2,4}: grid schedule = g CTAs per SM (capped by  */
                            /* occupancy and tile count); cluster schedule = 4g CTAs per cluster */
    int32_t use_partition;  /* 1 = O(n) partition path, 0 = Redzone                                */
    int32_t schedule;       /* RZ_SCHED_*                                                          */
} rz_launch_cfg;

/* ---- context ------------------------------------------------------------------------------ */
int  rz_create(rz_ctx** ctx, int device);
void rz_destroy(rz_ctx* ctx);
/* Human-readable name of a status code; returns the number of bytes written (without NUL). */
int  rz_status_string(int code, char* buf, size_t len);
/* Text of the last CUDA error seen by this context (empty if none). */
int  rz_last_cuda_error(const rz_ctx* ctx, char* buf, size_t len);
/* Synchronise `stream` and return (and clear) the device-side status of calls made on it. */
int  rz_sync_status(rz_ctx* ctx, rz_stream_t stream);
/* Number of SMs of the context's device. */
int  rz_num_sms(const rz_ctx* ctx);
/* Cap the context scratch the library may grow (bytes; negative = no cap). A call that would need
 * more returns RZ_ERR_NO_MEMORY and changes nothing; scratch already held is kept. Also the way
 * tests inject an allocation failure. rz_scratch_bytes reports what the context holds. */
int  rz_set_scratch_limit(rz_ctx* ctx, int64_t bytes);
int64_t rz_scratch_bytes(const rz_ctx* ctx);

/* ---- single list -------------------------------------------------------------------------- */
/*
 * Remove the k distinct positions d_idx[0..k) from d_data[0..n) (elem_bytes in {4,8,16,32}),
 * in place, asynchronously on `stream`. *new_len (host pointer, may be NULL) receives n-k.
 * Replaces RemoveFromList_GPUWide (redzone.hxx:626) and redzone_CPU (Redzone_CPU.hxx:150).
 */
int rz_remove(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes,
              const uint32_t* d_idx, int64_t k, int64_t* new_len, uint32_t flags,
              rz_stream_t stream);

/* As rz_remove with an explicit launch configuration (used by the autotuner and tests). */
int rz_remove_cfg(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes,
                  const uint32_t* d_idx, int64_t k, const rz_launch_cfg* cfg, uint32_t flags,
                  rz_stream_t stream);

/*
 * Host-buffer form of rz_remove: copies h_idx (k entries, ideally pinned) to the device, runs
 * the removal on the device-resident d_data, synchronises and returns the status. This is the
 * end-to-end call a host program makes when its removal lists are produced on the CPU.
 */
int rz_remove_host_idx(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes,
                       const uint32_t* h_idx, int64_t k, int64_t* new_len, uint32_t flags,
                       rz_stream_t stream);

/*
 * Pipelined form of rz_remove_host_idx for a host program that hands the GPU one removal list
 * after another (redzone_CPU, Redzone_CPU.hxx:150, called in a loop): returns without waiting.
 * The index list is copied on the context's own copy stream, so the copy of one call overlaps
 * the kernel of the one before; the removal runs on `stream` after its copy; the call's own
 * status and device-tracked length (16 bytes) are read back into pinned memory on a third stream
 * while the next removal runs. *ticket names the call for rz_wait. h_idx (ideally pinned) must stay
 * unchanged until rz_wait for the call returns. Calls are ordered on `stream` as issued. Up to 8
 * calls per context are in flight; issuing a 9th waits for the oldest (its result is kept for
 * rz_wait). The staging buffers grow to the largest k seen (context scratch). Each call reports
 * only its own device errors.
 */
int rz_remove_host_idx_async(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes,
                             const uint32_t* h_idx, int64_t k, uint32_t flags, rz_stream_t stream,
                             uint64_t* ticket);
/* Wait for the call `ticket` of rz_remove_host_idx_async; returns its status and sets *new_len
 * (may be NULL) to the length the device tracked. Each ticket is collected once. */
int rz_wait(rz_ctx* ctx, uint64_t ticket, int64_t* new_len);

/*
 * Add-then-remove (the paper's growth step, Sec. 4.6): append g items from d_gain (device) at
 * rows [n, n + g) of d_data, whose allocation must hold capacity >= n + g items, then remove the k
 * distinct rows d_idx (each < n + g, so appended rows may be removed too) from the grown list with
 * the Redzone rule. *new_len = n + g - k. No counterpart in the reference's code; it replaces a
 * caller's copy followed by RemoveFromList_GPUWide (redzone.hxx:626) on Length + g.
 */
int rz_append_remove(rz_ctx* ctx, void* d_data, int64_t n, int64_t capacity, uint32_t elem_bytes,
                     const void* d_gain, int64_t g, const uint32_t* d_idx, int64_t k, int64_t* new_len,
                     uint32_t flags, rz_stream_t stream);

/*
 * Preserve-list compaction, the inverse form of removal: d_data[0..m) = (old) d_data[d_keep[j]]
 * for j in [0, m), in the order of d_keep (any order; each entry < n). O(m) work -- cheaper than
 * removing the other n - m items when m < n/2. The kept items pass through context scratch
 * (m * elem_bytes, grown on first use). Entries >= n are skipped and reported as
 * RZ_ERR_OUT_OF_RANGE (with RZ_SYNC or rz_sync_status). *new_len = m. No counterpart in the
 * reference's code (the paper names it as future work).
 */
int rz_keep(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes, const uint32_t* d_keep, int64_t m,
            int64_t* new_len, uint32_t flags, rz_stream_t stream);

/*
 * Key -> row index for delete-by-key (no counterpart in the reference's code; the paper names a
 * key index kept under Redzone moves as future work). Records are 8, 16 or 32 bytes and begin
 * with a uint64 key; the two largest key values are reserved. The index is a device hash table of
 * `capacity` slots (rounded up to a power of two; keep it at least twice the live keys).
 *   rz_keyindex_build  -- clear, then index rows [0, n); RZ_ERR_DUPLICATE on a repeated key.
 *   rz_keyindex_insert -- index rows [first, first + count) (e.g. after rz_append_remove); the
 *                         keys must not be indexed already. Both are synchronous.
 *   rz_keyindex_find   -- rows of `count` keys into d_rows (0xffffffff when absent), async.
 *   rz_remove_by_key   -- remove the rows holding the k given keys with the Redzone rule and keep
 *                         the index exact: deleted keys are erased and each item moved into a hole
 *                         is re-pointed at it (O(k); no other row changes). Synchronous up to the
 *                         removal: a missing key returns RZ_ERR_OUT_OF_RANGE and a repeated one
 *                         RZ_ERR_DUPLICATE before any row moves. *new_len = n - k.
 */
typedef struct rz_keyindex rz_keyindex;
int rz_keyindex_create(rz_ctx* ctx, int64_t capacity, rz_keyindex** out);
void rz_keyindex_destroy(rz_keyindex* ix);
int rz_keyindex_build(rz_keyindex* ix, const void* d_data, int64_t n, uint32_t record_bytes, rz_stream_t stream);
int rz_keyindex_insert(rz_keyindex* ix, const void* d_data, int64_t first, int64_t count, uint32_t record_bytes,
                       rz_stream_t stream);
int rz_keyindex_find(rz_keyindex* ix, const uint64_t* d_keys, int64_t count, uint32_t* d_rows, rz_stream_t stream);
int rz_remove_by_key(rz_ctx* ctx, rz_keyindex* ix, void* d_data, int64_t n, uint32_t record_bytes,
                     const uint64_t* d_keys, int64_t k, int64_t* new_len, uint32_t flags, rz_stream_t stream);

/*
 * Removal lists made on the GPU, with the red-zone marking fused into the producer (the paper's
 * "mark during producer" optimisation, p.14; no counterpart in the reference's code, whose
 * phase 1, redzone.hxx:698-707, scans the finished list). A caller's kernel that decides which
 * rows to delete calls rz_emit (include/redzone_device.cuh) for each of them; rz_emit appends the
 * row to the producer's list and, when the row could fall in the red zone [n - k, n) (it is
 * >= n - capacity), also to a short candidate list of (slot, row) pairs. rz_remove_produced then
 * removes the emitted rows with the canonical rule; every CTA learns the red entries from the
 * candidates, so no CTA scans the whole list and none waits for another, and k never has to
 * reach the host.
 *   rz_producer_create  -- capacity: most rows one round may emit (<= 2^18); cand_capacity:
 *                          candidate slots (about capacity^2 / n + margin; when exceeded, the
 *                          removal falls back to reading the list itself, still exact).
 *   rz_producer_reset   -- start a round for a list of n rows (n < 2^32): zeroes the counts on
 *                          `stream`. Take the view after each reset.
 *   rz_producer_get_view -- the plain struct a producer kernel passes to rz_emit.
 *   rz_remove_produced  -- remove the rows emitted since the reset from d_data[0..n), asynchronous;
 *                          the new length n - k is on the device (counts[0] gives k) and, with
 *                          RZ_SYNC, in *new_len. A round that emitted more than `capacity` rows
 *                          fails with RZ_ERR_NO_MEMORY and moves nothing. RZ_VALIDATE reads k back
 *                          (one synchronisation) and checks the list first.
 *   rz_produce_where_less -- a producer provided by the library: emits every row i < n with
 *                          d_keys[i] < threshold.
 *   rz_producer_download -- synchronous copy of the round's list to the host (up to max entries);
 *                          *k and *candidates receive the counts.
 */
typedef struct rz_producer_view {
    uint32_t* idx;            /* the removal list, capacity entries                               */
    uint32_t* counts;         /* [0] rows emitted (k), [1] candidates emitted                     */
    uint32_t* cand;           /* candidates: (slot in idx, row) pairs, cand_capacity of them       */
    uint32_t capacity;
    uint32_t cand_capacity;
    uint32_t n;               /* length of the list the round removes from                        */
    uint32_t floor;           /* max(0, n - capacity): rows >= floor are candidates                */
} rz_producer_view;
typedef struct rz_producer rz_producer;
int rz_producer_create(rz_ctx* ctx, int64_t capacity, int64_t cand_capacity, rz_producer** out);
void rz_producer_destroy(rz_producer* p);
int rz_producer_reset(rz_producer* p, int64_t n, rz_stream_t stream);
int rz_producer_get_view(const rz_producer* p, rz_producer_view* out);
int rz_remove_produced(rz_ctx* ctx, rz_producer* p, void* d_data, uint32_t elem_bytes, int64_t* new_len,
                       uint32_t flags, rz_stream_t stream);
int rz_produce_where_less(rz_producer* p, const uint32_t* d_keys, uint32_t threshold, rz_stream_t stream);
int rz_producer_download(const rz_producer* p, uint32_t* h_idx, int64_t max, int64_t* k, int64_t* candidates,
                         rz_stream_t stream);

/*
 * O(n) stable partition comparator (mark, per-tile counts and their scan, then a pipelined
 * in-place move), in place. Survivors keep their relative order, as with thrust::remove
 * (Thrust_remove.hxx:15-17) and InK compact (cuCompactor.cuh:104-141).
 */
int rz_partition(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes,
                 const uint32_t* d_idx, int64_t k, int64_t* new_len, uint32_t flags,
                 rz_stream_t stream);

/*
 * The reference's O(n) GPU comparator, for measurement only (no removal path of this library uses
 * it): mark every removed slot of the int list with -1, then thrust::remove(list, list + n, -1),
 * stable (Thrust_remove.hxx:15-17 with the marking of DataStruct.hxx:11-18), on `stream`.
 * *new_len receives the length Thrust returns. Assumes -1 occurs only where the marks put it.
 */
int rz_test_thrust_remove(rz_ctx* ctx, int32_t* d_list, int64_t n, const uint32_t* d_idx, int64_t k,
                          int64_t* new_len, rz_stream_t stream);

/*
 * rz_remove for callers that cannot allocate device memory (an exhausted or foreign-owned memory
 * pool, a real-time path that must not take the allocator's lock or synchronise, a plugin host
 * that owns every allocation). No counterpart in the reference: its GPU path takes a
 * caller-allocated BlockStorage_t instead. Needs no context and calls no allocating routine; its
 * scratch is a fixed device-global array of about 8.4 MB that every GPU loading this library
 * holds until exit. Limits: k <= 2^20 (RZ_ERR_UNSUPPORTED above that), n < 2^32. The first call
 * on a device, with that device current, looks up the array's address: make it before any stream
 * capture, and do not use the library on a device after a cudaDeviceReset. `stream` must belong
 * to the current device (RZ_ERR_INVALID_ARG otherwise). Calls share the array, so calls that
 * overlap on the GPU race; order them on one stream. Asynchronous on `stream`; same result as
 * rz_remove; no RZ_VALIDATE. Errors found on the device (an index >= n, which is skipped; a
 * bounded wait that gave up) are collected in the array and read with rz_noalloc_sync_status.
 */
int rz_remove_noalloc(void* d_data, int64_t n, uint32_t elem_bytes, const uint32_t* d_idx, int64_t k,
                      int64_t* new_len, rz_stream_t stream);
/* Companion of rz_remove_noalloc (no counterpart in the reference): synchronise `stream` (on the
 * current device), then return and clear the device-side status of every rz_remove_noalloc call on
 * this device since the last rz_noalloc_sync_status -- RZ_ERR_OUT_OF_RANGE, RZ_ERR_TIMEOUT,
 * RZ_ERR_DUPLICATE (inconsistent orphan counts, only from invalid input) or RZ_OK. Allocates
 * nothing. */
int rz_noalloc_sync_status(rz_stream_t stream);

/* The configuration rz_remove would choose for (n, k, elem_bytes) without a predictor or tuning
 * table: the scan-all schedule up to k = 2^12, the cluster scan up to 2^17 (where it runs), the
 * grid schedule beyond. */
int rz_default_cfg(const rz_ctx* ctx, int64_t n, int64_t k, uint32_t elem_bytes,
                   rz_launch_cfg* cfg);

/* ---- many lists in one launch --------------------------------------------------------------- */
/* One list: device pointers to its payload (n items) and its k distinct removal indices. */
/* One list of a batch: data aligned to min(elem_bytes, 16) bytes, idx to 4 bytes
 * (RZ_ERR_INVALID_ARG otherwise). */
typedef struct rz_list_desc {
    void* data;
    const uint32_t* idx;
    int64_t n;
    int64_t k;
} rz_list_desc;

/* Tile and schedule of the batched kernel: tile = block * items; lists with k <= tile run whole
 * in one CTA, longer lists are split into tiles and handed out `span` tiles per work item
 * (0 = automatic: 4); ctas_per_sm sets the persistent grid. */
typedef struct rz_batch_cfg {
    int32_t block;
    int32_t items;
    int32_t ctas_per_sm;
    int32_t span;
    int32_t wave;  /* work order: 0 = phase by phase over all lists (every list's marks, then the    */
                   /* holes of every list, then every list's orphans); w > 0 = list by list, a     */
                   /* list's phases w/2 grids' worth of work items apart (keeps its writes in L2) */
} rz_batch_cfg;

typedef struct rz_batch_plan rz_batch_plan;

/*
 * Plan the removal of every list of `lists` (host array) in one persistent launch. The plan owns
 * its work queue and scratch. cfg == NULL uses the configuration the list-mix predictor picks
 * when one is attached (rz_set_batch_predictor; only configurations whose tile lets the longest
 * list fit in 1024 tiles are candidates), else the context's tuned batched configuration, else the
 * built-in default (512 x 4 x 4, wavefront order; 256 x 4 x 4 for 32-byte items), its tile
 * raised until the longest list fits.
 * An explicit configuration whose tile is too small for a list fails with RZ_ERR_UNSUPPORTED.
 * Each list's result equals rz_remove on that list (the reference's per-list calls,
 * redzone.hxx:1089-1166, one launch each).
 */
int  rz_batch_plan_create(rz_ctx* ctx, const rz_list_desc* lists, int32_t nlists, uint32_t elem_bytes,
                          const rz_batch_cfg* cfg, rz_batch_plan** plan);
/* Run the plan on `stream`: captured into a CUDA graph on the first launch, replayed after. */
int  rz_batch_plan_launch(rz_batch_plan* plan, rz_stream_t stream);
int  rz_batch_plan_info(const rz_batch_plan* plan, int32_t* grid, int32_t* block, int32_t* items,
                        int64_t* work_items, int64_t* total_k);
void rz_batch_plan_destroy(rz_batch_plan* plan);
/* One-shot form: plan, run, synchronise, return the device status. */
int  rz_remove_batched(rz_ctx* ctx, const rz_list_desc* lists, int32_t nlists, uint32_t elem_bytes,
                       uint32_t flags, rz_stream_t stream);

/* ---- streaming delete service ---------------------------------------------------------------- */
/*
 * A device-resident table split into `shards` independent sub-tables of shard_capacity records;
 * delete batches (one shard, distinct live row indices) are submitted from the host while earlier
 * ones run. A worker thread admits a batch when its shard has nothing in flight, a slot (stream)
 * is free and its indices fit the slot's share of index_budget_bytes; it coalesces the admitted
 * batches of a slot into one batched Redzone launch; slots overlap on the GPU. Live lengths are
 * tracked on the device. Before a batch would take a shard below floor_rows the shard is refilled
 * to capacity with fresh records (add-then-remove). No counterpart in the reference, which only
 * benchmarks one removal at a time (tests.cu:135-157).
 */
typedef struct rz_service rz_service;

typedef struct rz_service_cfg {
    int32_t shards;
    int32_t slots;                   /* launches in flight at once, one stream each               */
    int64_t shard_capacity;          /* records per shard (< 2^32)                                  */
    uint32_t record_bytes;           /* 4, 8, 16 or 32                                              */
    int32_t max_batches_per_launch;  /* coalescing limit (distinct shards per launch)               */
    int64_t index_budget_bytes;      /* device memory for in-flight indices, split over the slots */
    int64_t floor_rows;              /* refill threshold                                            */
} rz_service_cfg;

typedef struct rz_service_stats {
    int64_t submitted, completed, rejected, rows_deleted, launches, refills, rows_appended;
    double p50_us, p99_us, mean_us, max_us;  /* per-batch latency, submit -> completion         */
    double mean_batches_per_launch;
    double busy_seconds;                     /* first submit -> last completion                */
} rz_service_stats;

#define RZ_SUBMIT_BORROW 0x1u  /* h_idx stays valid and unchanged until the batch completes */

int  rz_service_create(rz_ctx* ctx, void* d_table, const int64_t* initial_len, const rz_service_cfg* cfg,
                       rz_service** svc);
/* RZ_ERR_BUSY: the batch is larger than one slot's index memory and can never be admitted. */
int  rz_service_submit(rz_service* svc, int32_t shard, const uint32_t* h_idx, int64_t count,
                       uint32_t flags, uint64_t* ticket);
int  rz_service_drain(rz_service* svc, int32_t timeout_ms);
int  rz_service_stats_get(rz_service* svc, rz_service_stats* out);
int  rz_service_reset_stats(rz_service* svc);
/* Live lengths as the host plans them and as the device tracks them (either pointer may be NULL). */
int  rz_service_lengths(rz_service* svc, int64_t* host_view, int64_t* device_view);
/* Checkpoint / resume. rz_service_checkpoint drains (up to timeout_ms), then writes every shard's
 * live length and the count of records refills have appended to it (both `shards` entries); with
 * the caller's copy of its table (rows [0, length) of each shard) that is the whole state.
 * rz_service_restore loads such a state into an idle service (RZ_ERR_BUSY if work is pending);
 * later refills then append exactly the records the original service would have. */
int  rz_service_checkpoint(rz_service* svc, int64_t* lengths, int64_t* appended, int32_t timeout_ms);
int  rz_service_restore(rz_service* svc, const int64_t* lengths, const int64_t* appended);
void rz_service_destroy(rz_service* svc);
/* Load generator: Poisson arrivals at `rate` batches/s for `seconds`; each arrival submits a random
 * batch of `pool` (pinned index arrays, lent to the service) to a uniformly random shard; then
 * drains and returns the statistics. */
int  rz_service_run_poisson(rz_service* svc, const uint32_t* const* pool, const int64_t* pool_counts,
                            int32_t pool_size, double rate, double seconds, uint64_t seed,
                            rz_service_stats* out);

/* ---- autotuning ------------------------------------------------------------------------------ */
typedef struct rz_tune_entry {
    rz_launch_cfg cfg;
    float ms;               /* median time of the configuration */
} rz_tune_entry;

/*
 * Time the 63 launch configurations (48 of block x items x grid scale with the schedule chosen
 * by k, 8 cluster-scan, 4 scan-all and 3 split launches) and the partition path on the caller's
 * data, which every run rewrites (timing does not depend on the values). L2 is flushed between
 * repetitions. Writes up to max_out entries sorted by time.
 */
int rz_autotune_single(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes, const uint32_t* d_idx,
                       int64_t k, int32_t reps, rz_tune_entry* out, int32_t max_out, int32_t* count);
/* The launch-configuration space in its canonical order (the predictor's class index is the
 * position): writes up to max entries, returns the size of the space. Host only, no GPU needed. */
int rz_config_space(rz_launch_cfg* out, int32_t max);
/* Time candidate batched configurations on `lists`; *best receives the fastest. */
int rz_autotune_batched(rz_ctx* ctx, const rz_list_desc* lists, int32_t nlists, uint32_t elem_bytes,
                        int32_t reps, rz_batch_cfg* best, float* best_ms);
/*
 * Tuning tables (text; '#' comments; lines "single <w> <log2k> <block> <items> <g> <partition>
 * [<schedule>]" and "batched <w> <block> <items> <ctas_per_sm> [<wave>]"). rz_remove and rz_batch_plan_create use the
 * loaded entries (nearest log2 k bucket of the same width).
 */
int rz_tune_table_load(rz_ctx* ctx, const char* path);
int rz_tune_table_save(rz_ctx* ctx, const char* path);
int rz_tune_table_set_single(rz_ctx* ctx, uint32_t elem_bytes, int32_t log2k, const rz_launch_cfg* cfg);
int rz_tune_table_set_batched(rz_ctx* ctx, uint32_t elem_bytes, const rz_batch_cfg* cfg);

/* ---- learned configuration predictor ---------------------------------------------------------- */
/*
 * A 12 -> 64 -> 64 -> 64 FP32 MLP (ReLU hidden layers) trained and evaluated by the library's
 * own CUDA kernels. Outputs 0..62 are logits over the 63 launch configurations (the order of
 * rz_autotune_single's space), output 63 the logit of "the O(n) partition path is faster". The
 * reference has no counterpart: its configuration is fixed at compile time (tests.cu:1-2).
 * Features (rz_mlp_features, computed on the GPU from the index list): log2 n, log2 k, k/n,
 * payload bytes, mean and variance of the log-gap of the sorted 4096-index sample, fraction of
 * the sample in the red zone, 5-bucket run-length histogram (each scaled to about [0, 1]).
 */
typedef struct rz_mlp rz_mlp;
int  rz_mlp_param_count(void);
int  rz_mlp_create(rz_ctx* ctx, uint64_t seed, rz_mlp** mlp);
void rz_mlp_destroy(rz_mlp* mlp);
int  rz_mlp_get_params(rz_mlp* mlp, float* h_params, int32_t count);
int  rz_mlp_set_params(rz_mlp* mlp, const float* h_params, int32_t count);
int  rz_mlp_features(rz_ctx* ctx, const uint32_t* d_idx, int64_t n, int64_t k, uint32_t elem_bytes,
                     float* h_features12);
/* Logits (nsamp x 64) for host features (nsamp x 12). */
int  rz_mlp_forward(rz_mlp* mlp, const float* h_x, int64_t nsamp, float* h_out);
/* Mean loss and gradient of every parameter over one batch; targets nsamp x 64 (63 probabilities
 * over configurations + the partition bit). Used to check the kernels against a CPU oracle. */
int  rz_mlp_gradients(rz_mlp* mlp, const float* h_x, const float* h_t, int64_t nsamp, float* h_grad,
                      float* h_loss);
/* Adam on the GPU over nsamp samples, `epochs` passes of seeded mini-batches. */
int  rz_mlp_train(rz_mlp* mlp, const float* h_x, const float* h_t, int64_t nsamp, int32_t epochs,
                  int32_t batch, float lr, uint64_t seed, float* h_last_loss);
/* Make rz_remove(..., RZ_USE_PREDICTOR) consult `mlp` (NULL detaches it). */
int  rz_set_predictor(rz_ctx* ctx, rz_mlp* mlp);
/* The configuration the attached predictor picks for an instance. */
int  rz_predict_cfg(rz_ctx* ctx, const uint32_t* d_idx, int64_t n, int64_t k, uint32_t elem_bytes,
                    rz_launch_cfg* cfg);
/*
 * The same network trained for mixes of lists: it picks the batched kernel's configuration
 * (block {128,256,512} x items {2,4,8} x CTAs per SM {1,2,4} x work order {0, 6}: the 54 points
 * of rz_batch_config_space, in that order = outputs 0..53; the other outputs are ignored; the
 * autotuner searches the same space) from 12 features of the mix that rz_batch_features
 * computes on the host from the list sizes: log2 of the list count, total n and total k, total
 * k / n, payload bytes, mean and spread of log2 n, mean k/n, the share of removals in lists with
 * k <= 256 / 1024 / 4096, log2 of the largest k. No counterpart in the reference (it has no
 * batching). rz_set_batch_predictor attaches it (NULL detaches): rz_batch_plan_create and
 * rz_remove_batched then use its choice; rz_predict_batch_cfg returns it.
 */
int  rz_batch_config_space(rz_batch_cfg* out, int32_t max);
int  rz_batch_features(const rz_list_desc* lists, int32_t nlists, uint32_t elem_bytes, float* h_features12);
int  rz_set_batch_predictor(rz_ctx* ctx, rz_mlp* mlp);
int  rz_predict_batch_cfg(rz_ctx* ctx, const rz_list_desc* lists, int32_t nlists, uint32_t elem_bytes,
                          rz_batch_cfg* cfg);

/* ---- diagnostics -------------------------------------------------------------------------- */
/* Number of kernels the context's most recent removal call launched (memsets not counted), and
 * the grid / block it used for its main kernel. */
int rz_last_launch(const rz_ctx* ctx, int32_t* kernels, int32_t* grid, int32_t* block);

/*
 * Phase tracing of the single-list Redzone kernels (the reference's clock64 phase stamps,
 * redzone.hxx:629,708-712,847-851,936-939, kept per CTA and in %globaltimer nanoseconds).
 * When enabled, thread 0 of every CTA records 8 slots: 0 start, 1 marks issued, 2 first barrier
 * passed, 3 holes filled / orphans listed, 4 done; 5-7 unused. rz_read_phase_stamps synchronises
 * the device and copies the stamps of the most recent call (8 * nctas values).
 */
int rz_phase_stamps(rz_ctx* ctx, int enable);
int rz_read_phase_stamps(rz_ctx* ctx, uint64_t* out, int32_t max_ctas, int32_t* nctas);

/* Measurement aid: launch an empty kernel of `grid` x `block` threads (clusters of `cluster` CTAs,
 * 1-8, dividing grid; `smem_bytes` of dynamic shared memory) on `stream`. Timed between the same
 * events as a removal, it gives the floor that every launch of that shape pays. */
int rz_test_empty_launch(rz_ctx* ctx, int32_t grid, int32_t block, int32_t cluster, int32_t smem_bytes,
                         rz_stream_t stream);

/* Measurement aid: plain scattered stores d_data[d_pos[i]] = (an item made from i) for i in
 * [0, count), positions >= n skipped, on `stream`, with nothing else in the kernel. Given the hole
 * positions of a removal it measures the rate at which this GPU absorbs those writes alone: the
 * ceiling a removal whose time goes to its hole writes can reach. It overwrites d_data. */
int rz_test_scatter(rz_ctx* ctx, void* d_data, int64_t n, uint32_t elem_bytes, const uint32_t* d_pos, int64_t count,
                    rz_stream_t stream);

/*
 * Failure-detection check for the bounded device waits that replace the reference's grid
 * barriers (cg::grid.sync, redzone.hxx:707-940, and BlockStorage_t::Wait, redzone.hxx:59-80,
 * which can spin forever): launches one CTA that waits at a barrier nobody else reaches, with
 * `spin_limit` polls. The wait must give up, record the timeout and return; *status_bits gets
 * the device status word (bit 2 = timeout). The context's barrier state is reset afterwards.
 */
int rz_test_barrier_timeout(rz_ctx* ctx, uint32_t spin_limit, uint32_t* status_bits);

#ifdef __cplusplus
}
#endif

#endif /* REDZONE_B200_H */
