/*
 * srdl.h -- C ABI of libsrdl, the sm_100a semi-naive Datalog runtime.
 *
 * Plain pointers and sizes only.  All functions return 0 on success unless
 * stated otherwise; on failure srdl_last_error() describes the error of the
 * calling thread.  Status codes: 1 bad argument, 2 bad state, 3 CUDA error,
 * 4 malformed plan, 5 capacity exceeded, 6 I/O error, 7 unsupported
 * construct, 8 timed out.
 *
 * Two layers:
 *  - database handles (srdl_open ... srdl_close) that interpret a plan JSON
 *    produced from the srdatalog MIR; the per-program shim emitted by
 *    srdatalog_b200.build_project wraps one handle behind the reference's
 *    srdatalog_* names;
 *  - stream-ordered, allocation-free kernel primitives on device pointers
 *    (index build, delta, merge) for callers that keep their own relations.
 */
#ifndef SRDL_H
#define SRDL_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SRDL_ABI_VERSION 1

typedef struct srdl_db srdl_db;

/* Message for the last failed call on this thread (never NULL). */
const char* srdl_last_error(void);
int srdl_version(void);

/* Parse a plan and create a database bound to CUDA device `device`.  No GPU
 * work happens until srdl_init_device / srdl_run.  Replaces the
 * per-program SemiNaiveDatabase the generated shim allocates lazily
 * (src/srdatalog/codegen/jit/main_file.py:680-695). */
int srdl_open(const char* plan_json, int device, srdl_db** out);

/* Free every host and device resource of the database.  Replaces
 * srdatalog_shutdown (main_file.py:772-775). */
int srdl_close(srdl_db* db);

/* Select the device, create the stream and memory pool.  Replaces
 * srdatalog_init -> SRDatalog::GPU::init_cuda (main_file.py:683-688;
 * RT/gpu/init.h:50). */
int srdl_init_device(srdl_db* db);

/* Stage n_rows row-major uint32 rows of an input relation (host memory;
 * copied to the device by srdl_run).  No reference counterpart: the
 * reference only loads files. */
int srdl_load_rows(srdl_db* db, const char* rel, const uint32_t* rows, uint64_t n_rows);

/* Stage one CSV file for an input relation.  Replaces srdatalog_load_csv
 * (main_file.py:690-727) -> SRDatalog::load_from_file (RT/runtime/io.h:384). */
int srdl_load_csv(srdl_db* db, const char* rel, const char* path);

/* Stage `dir`/<input_file> for every input relation.  Replaces
 * srdatalog_load_all -> <Runner>::load_data (main_file.py:729-741, 204-213). */
int srdl_load_all(srdl_db* db, const char* dir);

/* Stage n_rows row-major uint32 pairs that already live in device memory
 * (binary input relations only).  They are copied once, on the database's
 * stream; srdl_run then starts from HBM-resident inputs.  No reference
 * counterpart. */
int srdl_load_device_rows(srdl_db* db, const char* rel, const uint32_t* d_rows, uint64_t n_rows);

/* Launch all further work of `db` on `stream` (a cudaStream_t owned by the
 * caller, who keeps it alive until srdl_close); device state of earlier runs
 * is released first.  No reference counterpart. */
int srdl_set_stream(srdl_db* db, void* stream);

/* Record CUDA events around every kernel family of srdl_run and report their
 * device time and algorithmic bytes in srdl_stats_json ("kernels"). */
int srdl_set_profiling(srdl_db* db, int enable);

/* Per-handle options (the autotuner's knobs, which never change a result,
 * and the run's memory limit):
 *   "bitmap_mb"        budget for bitmaps of long child lists (MB, 0 = none;
 *                      default SRDL_BITMAP_MB or 768)
 *   "hash_min"         hash child lists longer than this (0 = never; default
 *                      SRDL_HASH_MIN or 0)
 *   "lsm_compact_pct"  Device2LevelIndex: merge HEAD into FULL once HEAD
 *                      exceeds this percentage of FULL (default 10, the
 *                      reference's kCompactRatio, device_2level_index.h:300)
 *   "radix_bits"       widest radix-sort digit, 1..8 (default 8): a sort of
 *                      b-bit keys runs ceil(b / radix_bits) passes
 *   "join_blocks_per_sm"  join launches use at most this many blocks per
 *                      SM, 1..64 (default 16): the candidates per warp
 *   "join_chunk"       largest chunk of candidates a warp of the two-source
 *                      column join takes from its queue, 64..2^20 (default
 *                      4096): smaller chunks keep the rows in flight closer
 *   "pivot_min"        count-only two-source joins: rows whose probed list
 *                      belongs to the table's first (sorted) column, has a
 *                      bitmap and at least this many values are counted by
 *                      a kernel holding that bitmap in shared memory
 *                      (default 0: off -- on the R-MAT triangle the cj2
 *                      kernel's L2-resident bitmap probes measured faster)
 *   "device_loop"      1 (default; SRDL_DEVICE_LOOP=0 changes it) runs the
 *                      iterations of a qualifying recursive step after the
 *                      first as one CUDA graph that loops on the device
 *                      until the delta is empty; 0 keeps every iteration on
 *                      the host path.  Results are the same either way
 *   "device_loop_cap_limit"  largest buffer capacity (rows) the device loop
 *                      may choose, 0 = none (default); small values force
 *                      its overflow path, which hands iterations back to the
 *                      host path (for tests)
 *   "mem_limit_mb"     device memory a run may hold (MB, 0 = no limit,
 *                      the default): past it the run stops with status 5
 *                      (see srdl_mem_stats)
 *   "shard_world",     evaluate as shard "shard_rank" of "shard_world"
 *   "shard_rank"       (default 0 of 1): rules the plan marks
 *                      "shard": "key" keep only bindings whose "shard_var"
 *                      value v has owner(v) = ((v * 0x9E3779B1) mod 2^32)
 *                      * world >> 32 equal to the rank; rules marked
 *                      "shard": "work" expand only this shard's interleaved
 *                      segments of one join level's work items.  The marks
 *                      come from srdatalog_b200.shard.shard_plan; results
 *                      of the shards add up to the unsharded result.
 *                      srdl_run fails with status 1 if rank >= world.
 * Unknown names return 1 (argument error); negative values are rejected.
 * No reference counterpart: the reference fixes these at code-generation
 * time and evaluates on one GPU. */
int srdl_set_option(srdl_db* db, const char* name, int64_t value);

/* Exchange of derived tuples between shards (plans marked by
 * srdatalog_b200.shard.shard_plan carry "exchange" ops where a recursive
 * rule derives tuples keyed by another shard's values).  With shard_world
 * > 1, an exchange op partitions the relation's NEW tuples by the owner of
 * their first declared column and calls fn three ways:
 *   phase 0  counts[0..world) in: keys this shard sends to each shard;
 *            out: keys it receives from each shard;
 *   phase 1  d_send: the keys grouped by destination shard (ascending;
 *            uint64 in the relation's canonical index order), d_recv: room
 *            for the received keys, grouped by source shard; the transfer
 *            must be complete when fn returns;
 *   phase 2  (once per recursive iteration, before deciding to stop)
 *            counts[0] in: this shard's new-delta size; out: the sum over
 *            all shards.
 * `stream` is the database's cudaStream_t (synchronised before phase 1).
 * fn returns 0 on success; anything else fails the run (status 2).
 * fn = NULL removes it.  No reference counterpart. */
typedef int (*srdl_exchange_fn)(void* user, int phase, const char* rel, uint64_t* counts,
                                const uint64_t* d_send, uint64_t* d_recv, void* stream);
int srdl_set_exchange(srdl_db* db, srdl_exchange_fn fn, void* user);

/* Stream-ordered device copy (any direction under unified addressing),
 * complete on return: for exchange callbacks that move keys between
 * buffers the caller owns. */
int srdl_copy_device(void* dst, const void* src, uint64_t bytes, void* stream);

/* Kernels this process has launched through libsrdl so far. */
uint64_t srdl_launch_count(void);

/* For the count-only rule `rule`, also count bindings per group of the
 * rule's first bound variable: group g holds values in [bounds[g],
 * bounds[g+1]) (n_bounds = groups + 1, host array, non-decreasing;
 * n_bounds = 0 removes the grouping).  Splits the count of a disjoint-union
 * batch per instance.  The rule's last level must be a two-source column
 * join without filters (status 7 otherwise).  No reference counterpart. */
int srdl_set_count_groups(srdl_db* db, const char* rule, const uint32_t* bounds,
                          uint64_t n_bounds);

/* Per-group counts of the last run (n_groups = bounds - 1). */
int srdl_group_counts(srdl_db* db, const char* rule, uint64_t* out, uint64_t n_groups);

/* Drop every staged input (host and device rows) so the handle can be
 * reloaded with another input; the plan stays.  No reference counterpart. */
int srdl_clear_inputs(srdl_db* db);

/* counts[j] = rows of FULL(rel) whose first declared column lies in
 * [bounds[j], bounds[j+1]) for j < n_bounds-1 (host arrays; bounds
 * non-decreasing).  Splits a disjoint-union batch into per-instance sizes.
 * No reference counterpart. */
int srdl_range_counts(srdl_db* db, const char* rel, const uint32_t* bounds, uint64_t n_bounds,
                      uint64_t* counts);

/* Instances of a batched run: instance j owns the values [bounds[j],
 * bounds[j+1]) (host array, non-decreasing, n_bounds = instances + 1; 0
 * clears).  Every later srdl_run records on the device, for each recursive
 * step whose computed relations are binary, the iterations each instance's
 * own run would take (its last iteration with a non-empty delta, plus one,
 * capped at the step's iterations).  No reference counterpart. */
int srdl_set_instances(srdl_db* db, const uint32_t* bounds, uint64_t n_bounds);

/* Per-instance iterations of plan step `step` in the last run (out: one
 * uint32 per instance).  Non-recursive steps give 1.  Status 7 when the
 * step was not recorded (a computed relation is not binary). */
int srdl_instance_iterations(srdl_db* db, uint64_t step, uint32_t* out, uint64_t n_instances);

/* Per-range fingerprints of FULL(rel), a binary relation: sums[j] = the sum
 * mod 2^64, over its rows (x, y) with bounds[j] <= x < bounds[j+1], of
 * m(x - bounds[j] ^ 0x243F6A8885A308D3) * m(y - bounds[j] ^
 * 0x13198A2E03707344), m the SplitMix64 output function.  An order-free
 * digest of each instance's rows in its own values.  No reference
 * counterpart. */
int srdl_range_checksums(srdl_db* db, const char* rel, const uint32_t* bounds, uint64_t n_bounds,
                         uint64_t* sums);

/* Rows currently staged for `rel` by the load calls (host-side count). */
uint64_t srdl_staged_rows(srdl_db* db, const char* rel);

/* Copy staged inputs to the device and evaluate the plan; recursive strata
 * stop at an empty delta or after max_iters iterations (0 = unlimited).
 * Results stay on the device until the next run or srdl_close.  Replaces
 * srdatalog_run (main_file.py:743-753) -> copy_host_to_device
 * (RT/gpu/runtime/query.h:107) + <Runner>::run. */
int srdl_run(srdl_db* db, uint64_t max_iters);

/* Rows in the FULL version of `rel` (canonical index).  Replaces
 * srdatalog_size (main_file.py:755-767), which read the host DB. */
uint64_t srdl_size(srdl_db* db, const char* rel);

/* Bindings counted by a count-only rule (with_count) in the last run.
 * Replaces the ">>>> <Rule> count: N" stdout line of the generated runner
 * (tests/fixtures/jit/lsqb_triangle_count/orchestrator.cpp:40-47). */
uint64_t srdl_count(srdl_db* db, const char* rule);

/* Copy up to cap_rows rows of FULL(rel) into out_rows (row-major uint32, in
 * declared column order, lexicographically sorted) and return the total
 * row count (negative status on error; out_rows may be NULL to query the
 * size).  No reference counterpart: the reference cannot read results back. */
int64_t srdl_dump(srdl_db* db, const char* rel, uint32_t* out_rows, uint64_t cap_rows);

/* JSON run statistics (iterations per step, timings, derived rows). */
int srdl_stats_json(srdl_db* db, char* buf, uint64_t cap);

/* Device memory of the database's stream, measured by its caching arena:
 * out4[0] bytes held by live buffers now, out4[1] the most held during the
 * last srdl_run (its peak, recorded whether it succeeded or not), out4[2]
 * bytes cached for reuse, out4[3] the run limit set by the "mem_limit_mb"
 * option (0: none).  A run that would hold more than the limit stops with
 * status 5; its database keeps nothing of that run.  No reference
 * counterpart (the reference runs one query and never limits it). */
int srdl_mem_stats(srdl_db* db, uint64_t* out4);

/* Give the blocks the database's stream caches for reuse back to the device
 * (a server does this for idle handles when its memory budget is tight; the
 * next run allocates afresh).  No reference counterpart. */
int srdl_trim_cache(srdl_db* db);

/* SHA-256 of FULL(rel) as srdl_dump returns it (rows sorted, declared
 * column order, row-major little-endian uint32) into out32[32]: the parity
 * check's digest, computed next to the data.  srdl_sha256 hashes any host
 * buffer the same way.  No reference counterpart. */
int srdl_hash(srdl_db* db, const char* rel, unsigned char* out32);
int srdl_sha256(const void* data, uint64_t n_bytes, unsigned char* out32);

/* ------------------------------------------------------------------------
 * Kernel primitives.  Keys are uint64 = (index column 0 << 32) | column 1;
 * every value must be < 2^value_bits.  Pointers are device pointers, work
 * is enqueued on `stream` (a cudaStream_t, NULL = legacy default stream),
 * the result count is written to device memory, and nothing is allocated:
 * temporaries live in the caller's scratch region.
 * ---------------------------------------------------------------------- */

/* Scratch bytes srdl_sort_unique_u64 needs for n keys. */
uint64_t srdl_sort_unique_scratch_bytes(uint64_t n, int value_bits);

/* Sort n keys ascending and drop duplicates: d_out gets the distinct keys,
 * *d_n_out their count.  d_out needs room for n keys and may alias d_in.
 * Replaces rebuild_index_fn (RT/gpu/runtime/gpu_mir_helpers.h:204-232) ->
 * zip_sort_columns (RT/gpu/sort.h:297-302) + deduplicate_aggregate_and_unique
 * (RT/gpu/deduplication.h:178-258). */
int srdl_sort_unique_u64(const uint64_t* d_in, uint64_t n, int value_bits, uint64_t* d_out,
                         uint64_t* d_n_out, void* d_scratch, uint64_t scratch_bytes,
                         void* stream);

/* Scratch bytes srdl_set_difference_u64 needs for na keys of `a`. */
uint64_t srdl_set_difference_scratch_bytes(uint64_t na);

/* d_out = a - b for sorted duplicate-free arrays; *d_n_out = |d_out|.
 * Replaces compute_delta_index_fn (gpu_mir_helpers.h:88-122) ->
 * DSAI::set_difference_update (RT/gpu/device_sorted_array_index.ipp:966-1130). */
int srdl_set_difference_u64(const uint64_t* d_a, uint64_t na, const uint64_t* d_b, uint64_t nb,
                            uint64_t* d_out, uint64_t* d_n_out, void* d_scratch,
                            uint64_t scratch_bytes, void* stream);

/* d_out = a U b for disjoint sorted duplicate-free arrays (na + nb keys).
 * Replaces merge_index_fn (gpu_mir_helpers.h:136-159) -> DSAI::merge
 * (RT/gpu/device_sorted_array_index.ipp:709-847). */
int srdl_merge_u64(const uint64_t* d_a, uint64_t na, const uint64_t* d_b, uint64_t nb,
                   uint64_t* d_out, void* stream);

/* Allocation-free variant of srdl_sort_unique_u64, for callers that may not
 * allocate device memory on their call path (a host engine whose memory
 * manager owns and pre-plans every device allocation, or a latency-critical
 * caller that cannot afford cudaMalloc).  No counterpart in the reference.
 * Same contract as srdl_sort_unique_u64 without the scratch arguments: the
 * temporaries live in a 20 MiB file-scope device array that every GPU loading
 * libsrdl keeps until process exit.  At most
 * srdl_sort_unique_noalloc_max_keys() (1,048,576) keys per call; more returns
 * status 5.  The first call on a device resolves the array's address (call it
 * once before any stream capture).  Calls that overlap on the GPU share the
 * array and race: serialise them.  Calls no cudaMalloc/cudaFree. */
int srdl_sort_unique_u64_noalloc(const uint64_t* d_in, uint64_t n, int value_bits,
                                 uint64_t* d_out, uint64_t* d_n_out, void* stream);
uint64_t srdl_sort_unique_noalloc_max_keys(void);

#ifdef __cplusplus
}
#endif

#endif /* SRDL_H */
