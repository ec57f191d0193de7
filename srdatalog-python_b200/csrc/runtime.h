// runtime.h -- host-side database: plan, relation store, executor.
//
// Replaces the generated <Project>_Runner (step_N bodies, orchestrator_jit.py:
// 600-747), the device DB (RT/gpu/runtime/query.h:107 copy_host_to_device)
// and the mir_helpers primitive provider (RT/gpu/runtime/gpu_mir_helpers.h).
// The plan is interpreted; kernels are fixed.
#pragma once

#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/srdl.h"
#include "json.h"
#include "kernels.h"

namespace srdl {

enum Ver { kFull = 0, kDelta = 1, kNew = 2 };

// Caching arena for the allocations of one stream.  Freed blocks are kept in
// per-size-class free lists and handed to the next allocation of that class
// on the same stream (safe in stream order), so a fixpoint's iterations,
// which allocate the same few sizes over and over, stop calling the driver:
// a stream-ordered allocation that has to re-map pool memory can wait for
// the kernels already queued, leaving the GPU idle behind it.  Classes are
// 4 KB, quarter steps between powers of two below 1 MB, and powers of two
// from 1 MB up, so a relation that grows over the iterations keeps reusing
// the same few blocks; a request takes the smallest cached block of up to
// twice its class.  When the device runs out of memory, every arena frees
// its cached blocks and the allocation is retried once.
class StreamArena;
void arena_attach(cudaStream_t s);   // one reference per database using `s`
void arena_detach(cudaStream_t s);   // last reference frees the cached blocks
// Device bytes of the stream's arena: handed out to live buffers now, the
// most handed out since the last reset_peak, cached for reuse, and the limit
// on the bytes it holds, handed out plus cached (0: none).  Under a limit the
// cache is dropped before a new block would pass it, and a request that
// would take the handed-out bytes alone past it fails with status 5
// (kErrCapacity) instead of allocating: a server admits work against a
// device-memory budget and holds each run to its reservation this way.
struct ArenaUse {
  size_t in_use = 0, peak = 0, cached = 0, limit = 0;
};
ArenaUse arena_use(cudaStream_t s);
void arena_set_limit(cudaStream_t s, size_t bytes);
void arena_reset_peak(cudaStream_t s);
void arena_trim(cudaStream_t s);  // frees the cached blocks (stream-ordered)

// Owning device allocation: from the stream's arena when one is attached,
// else straight from the stream-ordered pool.
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(size_t bytes, cudaStream_t st);
  ~DevBuf() { reset(); }
  DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
  DevBuf& operator=(DevBuf&& o) noexcept;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  void reset();
  template <typename T>
  T* as() const { return reinterpret_cast<T*>(p_); }
  size_t bytes() const { return bytes_; }

 private:
  void* p_ = nullptr;
  size_t bytes_ = 0;
  cudaStream_t st_ = 0;
  std::shared_ptr<StreamArena> arena_;
  size_t cls_ = 0;  // size of the arena block backing p_
};

struct Split3;

// One sorted, duplicate-free key array plus the join-side trie pieces,
// built on first use by a join.
struct Index {
  DevBuf keys;
  uint64_t n = 0;
  bool trie = false;
  uint64_t epoch = 0;  // FULL: the last delta (Relation::delta_epoch) merged into this permutation
  DevBuf lo, roots, dir;
  DevBuf nroots_d;  // device-resident count of `roots`
  uint32_t dir_n = 0;
  bool hash_done = false;  // hashed child lists built (or found unnecessary)
  DevBuf hdir, hpool;
  bool bitmap_done = false;  // bitmaps of long child lists built (or found unnecessary)
  DevBuf bdir, bpool;
  uint32_t bwords = 0;
  // Ternary relations (packed keys): the pair and row views of this array in
  // each column order a join has read it in, built on first use.
  std::map<std::vector<int>, std::shared_ptr<Split3>> split;
};

// Read views of a ternary relation in one column order (c0, c1, c2): `pair`
// holds the distinct (c0, c1) as binary keys, `rows` every tuple as
// (position of its (c0, c1) in `pair`) << 32 | c2.
struct Split3 {
  Index pair, rows;
};

struct Chunk {
  DevBuf keys;
  uint64_t n = 0;
  std::vector<int> order;  // index permutation the keys are packed in
  bool sorted = false;     // already sorted and unique in `order` (a copied index)
};

struct RelVersion {
  std::map<std::vector<int>, Index> idx;
  std::vector<Chunk> chunks;  // NEW: unsorted join output
  void clear() {
    idx.clear();
    chunks.clear();
  }
  bool has_index() const { return !idx.empty(); }
};

struct Relation {
  std::string name;
  int arity = 2;
  std::string input_file;
  bool print_size = false;
  std::string index_type;
  std::vector<int> canonical;
  RelVersion v[3];
  std::vector<uint32_t> facts;   // rows the plan itself carries (head constants), row-major
  std::vector<uint32_t> staged;  // host rows loaded before run (row-major)
  uint32_t staged_max = 0;       // largest value in `staged` (kept as rows are added)
  uint32_t* pinned = nullptr;    // page-locked copy of `staged` used for the upload
  size_t pinned_cap = 0;         // words allocated; grows, freed only at close
  bool pinned_valid = false;     // holds the current `staged`
  DevBuf dstaged;                // device rows loaded before run (row-major pairs)
  uint64_t dstaged_n = 0;
  uint32_t dstaged_max = 0;
  bool loaded = false;
  bool pending_delta = false;    // NEW was sorted straight into a delta
  Index pending;
  // Device2LevelIndex policy (index_type): FULL in the canonical permutation
  // is kept as a large sorted segment (v[kFull]) plus a small sorted HEAD that
  // receives each iteration's DELTA; HEAD is merged into FULL when it passes a
  // tenth of FULL, at the end of the stratum, or before any read that wants
  // FULL as one array (every such read goes through ensure_index).  FULL's
  // other permutations are dropped whenever HEAD changes and are rebuilt from
  // the merged canonical array on demand.
  bool lsm = false;
  // Materialised relations of arity 3 or 4: a tuple is stored as one uint64,
  // its columns (in index order) packed pack_bits apiece into P and split at
  // pack_half bits, key = (P >> pack_half) << 32 | (P mod 2^pack_half), so
  // key order is tuple order and the binary-key sort, difference and merge
  // apply unchanged.  pack_half = 0: the tuple does not fit 64 bits.
  int pack_bits = 0, pack_half = 0;
  Index head;
  // Every compute_delta_index makes a new DELTA (delta_epoch).  full_epoch is
  // the last one any permutation of FULL has absorbed, base_epoch the one
  // before it: a permutation at base_epoch still lacks the latest delta and is
  // merged with it; one older than that is rebuilt from an up-to-date one.
  uint64_t delta_epoch = 0, full_epoch = 0, base_epoch = 0;
};

// Plan-level descriptions (parsed once from JSON).
struct SourceDesc {
  std::string rel;
  Ver ver;
  std::vector<int> index;
  std::vector<std::string> prefix;
};

struct PipeOp {
  enum Kind { Scan, ColumnJoin, Cartesian, Filter, Insert, Negation } kind;
  std::vector<SourceDesc> sources;           // scan: one
  std::vector<std::string> vars;             // scan / cartesian / insert / filter vars
  std::string var;                           // column join var
  std::vector<std::vector<std::string>> var_from_source;
  std::string code;                          // filter
  std::string rel;                           // insert
  std::vector<int> index;                    // insert dedup index
  std::vector<uint32_t> const_prefix;        // negation: constant values leading the probed prefix
};

struct Op {
  // Hook: an injected C++ hook of the reference (mir/types.py:358), kept in
  // the plan and skipped (there is no C++ code generation here).
  // Exchange: send NEW tuples to the shards owning their first column.
  enum Kind { Execute, Rebuild, Clear, CheckSize, ComputeDelta, Merge, RebuildFrom, Reconstruct, Hook, Exchange } kind;
  std::string rel, rule;
  Ver ver = kFull;
  std::vector<int> index, source_index;
  bool count = false;
  std::vector<PipeOp> pipeline;
  // Sharding of a rule when the database is one of several shards:
  //   Work: the last level's work items are split evenly; this shard expands
  //         its contiguous window (count-only rules over replicated inputs);
  //   Key : only bindings whose `shard_var` value this shard owns
  //         (shard_owner) are kept, filtered where the variable is bound.
  enum Shard { NoShard, Work, Key } shard = NoShard;
  std::string shard_var;
};

struct Step {
  bool recursive = false;
  std::vector<Op> ops;
};

// Per-kernel-family device time (CUDA events on the database stream) and
// the algorithmic bytes / work units those launches had to process.
struct KernelStats {
  double ms = 0, bytes = 0, units = 0;
  uint64_t scopes = 0;
};

struct AllocStats {
  double ms, max_ms;
  uint64_t calls;
};
AllocStats alloc_stats();
void reset_alloc_max();

struct StepStats {
  uint64_t iterations = 0;
  double ms = 0;
};

// Host wall time spent in each kind of plan operation during the last run
// (launch, allocation and synchronisation time; the kernels run behind it).
struct OpStats {
  double ms = 0, max_ms = 0;
  uint64_t calls = 0;
};

// A pipeline's join levels, built from the plan (sources resolved to
// index views), before any is run.
struct PipePlan {
  std::vector<LevelSpec> levels;
  const PipeOp* insert = nullptr;
  Relation* target = nullptr;
  int nslots = 0;
  int key_slot[4] = {-1, -1, -1, -1};  // emitted key columns (materialising rules)
  bool sharded = false;
  size_t work_split = 0;
};

class Database {
 public:
  Database(const std::string& plan_json, int device);
  ~Database();

  void load_rows(const std::string& rel, const uint32_t* rows, uint64_t n);
  void load_device_rows(const std::string& rel, const uint32_t* d_rows, uint64_t n);
  void clear_inputs();
  // Count-only rule `rule`: also count per group of its first variable's
  // values, [bounds[g], bounds[g+1]) (n_bounds = groups + 1; 0 clears).
  void set_count_groups(const std::string& rule, const uint32_t* bounds, uint64_t n_bounds);
  void group_counts(const std::string& rule, uint64_t* out, uint64_t n_groups) const;
  // counts[j] = rows of FULL(rel) whose first declared column is in
  // [bounds[j], bounds[j+1]), for j < n_bounds - 1.
  void range_counts(const std::string& rel, const uint32_t* bounds, uint64_t n_bounds,
                    uint64_t* counts);
  // Instances of a batched run: instance j owns the values [bounds[j],
  // bounds[j+1]) (n_bounds = instances + 1; 0 clears).  Every later run
  // records on the device, per recursive step whose computed relations are
  // binary, the iterations each instance's own run would take.
  void set_instances(const uint32_t* bounds, uint64_t n_bounds);
  void instance_iterations(uint64_t step, uint32_t* out, uint64_t n_instances) const;
  // sums[j] = sum over the rows (x, y) of FULL(rel) with x in [bounds[j],
  // bounds[j+1]) of mix_a(x - bounds[j]) * mix_b(y - bounds[j]) mod 2^64
  // (binary relations; the row fingerprint of instances.cu).
  void range_checksums(const std::string& rel, const uint32_t* bounds, uint64_t n_bounds, uint64_t* sums);
  void set_stream(cudaStream_t s);
  void set_profiling(bool on) { profile_ = on; }
  void set_option(const std::string& name, int64_t value);
  void set_exchange(srdl_exchange_fn fn, void* user) {
    xfn_ = fn;
    xuser_ = user;
  }
  void load_csv(const std::string& rel, const std::string& path);
  void load_all(const std::string& dir);
  void run(uint64_t max_iters);
  uint64_t size(const std::string& rel);
  uint64_t count(const std::string& rule) const;
  // Rows of FULL in declared column order, lexicographically sorted.
  int64_t dump(const std::string& rel, uint32_t* out, uint64_t cap_rows);
  std::string stats_json() const;
  // Arena bytes of this database's stream: in use now, the last run's peak,
  // cached, and the limit.
  ArenaUse mem_stats() const;
  // Frees the blocks this database's stream arena caches for reuse.
  void trim_cache() {
    if (dev_ready_) arena_trim(L_.stream);
  }
  bool any_loaded() const;
  void stage_facts(Relation& r);
  uint64_t staged_rows(const std::string& name) {
    Relation& r = rel(name);
    return r.staged.size() / r.arity + r.dstaged_n;
  }
  void init_device();
  Relation& rel(const std::string& name);
  bool has_rel(const std::string& name) const { return rels_.count(name) > 0; }
  const std::vector<std::string>& input_relations() const { return inputs_; }

 private:
  // ------------------------------------------------------------ state
  int device_;
  bool dev_ready_ = false;
  Launch L_;
  std::string name_;
  std::map<std::string, std::unique_ptr<Relation>> rels_;
  std::vector<std::string> inputs_;
  std::vector<Step> steps_;
  std::map<std::string, uint64_t> counts_;
  std::map<std::string, std::vector<uint32_t>> group_bounds_;
  std::map<std::string, std::vector<uint64_t>> group_counts_;
  std::vector<StepStats> step_stats_;
  // batched runs (instances.cu): instance bounds, per recursive step the
  // last iteration with a delta row of every instance (device), and the
  // iterations of every instance's own run (host, after the step)
  std::vector<uint32_t> inst_bounds_;
  DevBuf inst_bounds_d_;
  std::map<size_t, DevBuf> inst_last_;
  std::map<size_t, std::vector<uint32_t>> inst_iters_;
  uint32_t* loop_marks_ = nullptr;  // the step on the device loop: its instance marks (or null)
  void instances_begin();
  uint32_t* instance_marks(size_t si);
  void mark_instances(size_t si, const Step& st, uint32_t iter);
  void instances_end(size_t si, uint64_t iters);
  Index& binary_full_index(Relation& r, bool* swapped);
  uint32_t dom_max_ = 0;
  int bits_ = 1;
  uint64_t derived_ = 0;
  double run_ms_ = 0;
  bool own_stream_ = true;
  bool profile_ = false;
  bool trace_ = std::getenv("SRDL_TRACE") != nullptr;  // per-sort sizes on stderr
  int64_t opt_bitmap_mb_ = -1;      // -1: SRDL_BITMAP_MB or the default
  int64_t opt_hash_min_ = -1;       // -1: SRDL_HASH_MIN or off
  int64_t opt_lsm_pct_ = 10;        // HEAD -> FULL merge threshold (% of FULL)
  uint64_t opt_mem_limit_ = 0;      // bytes a run may hold on the device (0: no limit)
  int64_t opt_pivot_min_ = 0;       // count joins: shortest bitmapped list the pivot kernel takes (0: off)
  ArenaUse mem_run_{};              // the last run's arena use (peak: its most held)
  int64_t shard_rank_ = 0, shard_world_ = 1;  // this database's shard among shard_world_
  srdl_exchange_fn xfn_ = nullptr;  // moves tuples between shards (exchange ops)
  void* xuser_ = nullptr;
  struct KEvent {
    std::string name;
    cudaEvent_t a, b;
    double bytes, units;
  };
  std::vector<KEvent> kev_;
  std::vector<cudaEvent_t> ev_pool_;
  std::map<std::string, KernelStats> kstats_;
  std::map<std::string, OpStats> opstats_;
  AllocStats alloc_{0, 0, 0};
  double pool_reserved_gb_ = 0;
  uint64_t launches_ = 0;
  // The device loop (loop.cu): statistics of the last run, on/off.
  struct LoopStats {
    uint64_t entries = 0, iterations = 0, overflows = 0, skipped = 0;
    double capture_ms = 0, run_ms = 0;
    std::string last_error;
  };
  LoopStats loop_stats_;
  int64_t opt_device_loop_ = -1;     // -1: SRDL_DEVICE_LOOP (0 turns it off) or on
  // The loop's graph is captured and launched on a stream of its own (the
  // database's stream may be a default stream, which cannot be captured),
  // ordered after and before the database's stream by two events.
  cudaStream_t loop_stream_ = nullptr;
  cudaEvent_t loop_ev_[2] = {nullptr, nullptr};
  uint64_t opt_loop_cap_limit_ = 0;  // largest capacity the loop may choose (0: none; tests force overflows)
  // Largest candidate count seen per join level of each execute op, and the
  // largest NEW (before dedup), DELTA and final FULL sizes per relation, kept
  // across runs: the device loop sizes its buffers from them.
  std::map<const Op*, std::vector<uint64_t>> level_max_;
  std::map<std::string, uint64_t> new_max_, delta_max_, full_max_;
  size_t prof_begin(const std::string& name);
  void prof_end(size_t id, double bytes, double units);
  void prof_collect();
  DevBuf d_small_;  // device scalars read back by the host
  uint64_t* h_small_ = nullptr;  // pinned mirror

  // ------------------------------------------------------------ helpers
  void parse_plan(const std::string& plan_json);
  void reset_device_state();
  void upload_inputs();
  uint64_t read_scalar(int slot);
  Index& ensure_index(Relation& r, Ver v, const std::vector<int>& perm);
  // FULL's large segment in `perm` without merging HEAD into it.
  Index& full_base(Relation& r, const std::vector<int>& perm);
  // Merges r's HEAD into canonical FULL (drops FULL's other permutations).
  void compact_head(Relation& r);
  // d <- d - HEAD when d is in the canonical permutation of an LSM relation.
  void subtract_head(Relation& r, const std::vector<int>& perm, Index& d);
  // hi_max: largest first-column value of the keys (-1: the input domain's)
  void ensure_trie(Relation& r, Index& ix, int64_t hi_max = -1);
  TrieView view(Relation& r, Index& ix);
  TrieView view2(Index& ix);  // a binary view of derived keys (ternary pair / row views)
  Split3& ensure_split(Relation& r, Index& canon, const std::vector<int>& order);
  void ensure_hash(Index& ix);
  void ensure_bitmaps(Index& ix);
  void sort_into(Index& out, const uint64_t* in, uint64_t n, bool swap, const Index* full,
                 const Index* head = nullptr, int key_bits = 0);
  void run_steps(uint64_t max_iters);
  // Device loop: whether a recursive step qualifies (why not, when it does
  // not), and running its iterations from it0 on the device; returns
  // kLoopDone (fixpoint or iteration limit reached), kLoopOverflow (a
  // capacity was too small: iteration it0 + *done is to be redone on the
  // host) or kLoopSkipped (nothing done).
  enum { kLoopDone = 0, kLoopOverflow = 1, kLoopSkipped = 2 };
  bool loop_eligible(const Step& st, std::string& why);
  int run_device_loop(const Step& st, uint64_t it0, uint64_t max_iters, uint64_t* done);
  void exec_ops(const Step& st, uint64_t iteration);
  // dviews: DELTA views that replace the relation's DELTA index (device loop)
  PipePlan plan_pipeline(const Op& op, bool recursive, uint64_t iteration,
                         const std::map<std::string, TrieView>* dviews);
  void exec_pipeline(const Op& op, bool recursive, uint64_t iteration);
  void op_rebuild(const Step& st, size_t pos, const Op& op);
  void op_compute_delta(const Op& op);
  void op_merge(const Op& op);
  void op_exchange(const Op& op);
  // Sum of a count over all shards (the exchange callback's phase 2).
  uint64_t shards_sum(uint64_t local);
};

std::vector<int> identity_perm(int arity);

}  // namespace srdl
