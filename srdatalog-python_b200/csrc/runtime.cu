// runtime.cu -- Database: plan parsing, input staging, relation indexes.
#include <algorithm>
#include <atomic>
#include <mutex>
#include <unordered_map>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <sstream>

#include "runtime.h"

namespace srdl {

// Dense directories are built while the value domain stays below this many
// entries (64 MB of uint32 offsets); above it, lookups binary-search keys.
constexpr uint64_t kDenseDirMax = 1ull << 24;
constexpr int kSmallSlots = 16;

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

std::vector<int> identity_perm(int arity) {
  std::vector<int> p(arity);
  for (int i = 0; i < arity; i++) p[i] = i;
  return p;
}

// ------------------------------------------------------------------ DevBuf

// Host time spent inside device allocations (process-wide), for the stats.
static std::atomic<uint64_t> g_alloc_ns{0}, g_alloc_max_ns{0}, g_alloc_calls{0};

AllocStats alloc_stats() {
  return {g_alloc_ns.load() * 1e-6, g_alloc_max_ns.load() * 1e-6, g_alloc_calls.load()};
}
void reset_alloc_max() { g_alloc_max_ns.store(0); }

static size_t size_class(size_t b) {
  if (b <= 4096) return 4096;
  const int k = 63 - __builtin_clzll((unsigned long long)b);
  const size_t base = size_t(1) << k;
  if (b == base) return b;
  if (b >= (size_t(1) << 20)) return base << 1;  // 1 MB and up: powers of two
  const size_t q = base / 4;
  return base + ((b - base + q - 1) / q) * q;
}

// Timed driver allocation; on an out-of-memory answer every arena gives its
// cached blocks back, the device drains, and the allocation is tried once more.
static void release_all_arenas();
static void* driver_alloc(size_t bytes, cudaStream_t st) {
  const auto t0 = std::chrono::steady_clock::now();
  void* p = nullptr;
  cudaError_t e = cudaMallocAsync(&p, bytes, st);
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    release_all_arenas();
    SRDL_CUDA(cudaDeviceSynchronize());
    e = cudaMallocAsync(&p, bytes, st);
  }
  SRDL_CUDA(e);
  const uint64_t ns = (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                          std::chrono::steady_clock::now() - t0)
                          .count();
  g_alloc_ns += ns;
  g_alloc_calls++;
  uint64_t prev = g_alloc_max_ns.load();
  while (ns > prev && !g_alloc_max_ns.compare_exchange_weak(prev, ns)) {
  }
  return p;
}

class StreamArena {
 public:
  explicit StreamArena(cudaStream_t s) : st_(s) {}
  // Smallest cached block of class [cls, 2*cls], else a new one of class cls;
  // *got = the class of the block handed out.  With a limit, the bytes the
  // arena holds (handed out + cached) stay within it: a new block first
  // drops the cache when it would pass the limit, and a request that the
  // handed-out bytes alone would take past it is refused (status 5).
  void* take(size_t cls, size_t* got) {
    {
      std::lock_guard<std::mutex> g(mu_);
      auto it = free_.lower_bound(cls);
      const bool hit = it != free_.end() && it->first <= 2 * cls;
      const size_t c = hit ? it->first : cls;
      if (limit_ && in_use_ + c > limit_)
        throw Error{kErrCapacity, "device memory limit of the run exceeded: " +
                                      std::to_string(in_use_ + c) + " bytes needed, limit " +
                                      std::to_string(limit_) + " (mem_limit_mb)"};
      in_use_ += c;
      peak_ = in_use_ > peak_ ? in_use_ : peak_;
      if (hit) {
        void* p = it->second;
        *got = it->first;
        cached_ -= it->first;
        free_.erase(it);
        return p;
      }
      if (limit_ && in_use_ + cached_ > limit_) drop_cache();
    }
    *got = cls;
    try {
      return driver_alloc(cls, st_);
    } catch (...) {
      std::lock_guard<std::mutex> g(mu_);
      in_use_ -= cls;
      throw;
    }
  }
  void give(void* p, size_t cls) {
    std::lock_guard<std::mutex> g(mu_);
    in_use_ -= cls;
    if (closed_) {
      cudaFreeAsync(p, st_);
      return;
    }
    free_.emplace(cls, p);
    cached_ += cls;
  }
  // Frees every cached block (stream-ordered); with `close`, later returns
  // are freed at once instead of cached.
  void release(bool close) {
    std::lock_guard<std::mutex> g(mu_);
    drop_cache();
    if (close) closed_ = true;
  }
  ArenaUse use() {
    std::lock_guard<std::mutex> g(mu_);
    ArenaUse u;
    u.in_use = in_use_;
    u.peak = peak_;
    u.cached = cached_;
    u.limit = limit_;
    return u;
  }
  // A limit below what the arena holds drops the cache at once.
  void set_limit(size_t b) {
    std::lock_guard<std::mutex> g(mu_);
    limit_ = b;
    if (limit_ && in_use_ + cached_ > limit_) drop_cache();
  }
  void reset_peak() {
    std::lock_guard<std::mutex> g(mu_);
    peak_ = in_use_;
  }
  int refs = 0;

 private:
  void drop_cache() {  // mu_ held
    for (auto& kv : free_) cudaFreeAsync(kv.second, st_);
    free_.clear();
    cached_ = 0;
  }
  cudaStream_t st_;
  std::mutex mu_;
  std::multimap<size_t, void*> free_;
  size_t cached_ = 0, in_use_ = 0, peak_ = 0, limit_ = 0;
  bool closed_ = false;
};

static std::mutex g_arena_mu;
static std::unordered_map<cudaStream_t, std::shared_ptr<StreamArena>>& arenas() {
  static auto* m = new std::unordered_map<cudaStream_t, std::shared_ptr<StreamArena>>();
  return *m;
}

static std::shared_ptr<StreamArena> arena_for(cudaStream_t s) {
  std::lock_guard<std::mutex> g(g_arena_mu);
  auto it = arenas().find(s);
  return it == arenas().end() ? nullptr : it->second;
}

void arena_attach(cudaStream_t s) {
  std::lock_guard<std::mutex> g(g_arena_mu);
  auto& a = arenas()[s];
  if (!a) a = std::make_shared<StreamArena>(s);
  a->refs++;
}

void arena_detach(cudaStream_t s) {
  std::shared_ptr<StreamArena> a;
  {
    std::lock_guard<std::mutex> g(g_arena_mu);
    auto it = arenas().find(s);
    if (it == arenas().end()) return;
    if (--it->second->refs > 0) return;
    a = it->second;
    arenas().erase(it);
  }
  a->release(true);
}

ArenaUse arena_use(cudaStream_t s) {
  auto a = arena_for(s);
  return a ? a->use() : ArenaUse{};
}

void arena_set_limit(cudaStream_t s, size_t bytes) {
  if (auto a = arena_for(s)) a->set_limit(bytes);
}

void arena_reset_peak(cudaStream_t s) {
  if (auto a = arena_for(s)) a->reset_peak();
}

void arena_trim(cudaStream_t s) {
  if (auto a = arena_for(s)) a->release(false);
}

static void release_all_arenas() {
  std::vector<std::shared_ptr<StreamArena>> all;
  {
    std::lock_guard<std::mutex> g(g_arena_mu);
    for (auto& kv : arenas()) all.push_back(kv.second);
  }
  for (auto& a : all) a->release(false);
}

DevBuf::DevBuf(size_t bytes, cudaStream_t st) : bytes_(bytes), st_(st) {
  if (!bytes) return;
  arena_ = arena_for(st);
  if (arena_) p_ = arena_->take(size_class(bytes), &cls_);
  else p_ = driver_alloc((bytes + 255) & ~size_t(255), st);
}

DevBuf& DevBuf::operator=(DevBuf&& o) noexcept {
  if (this != &o) {
    reset();
    p_ = o.p_;
    bytes_ = o.bytes_;
    st_ = o.st_;
    arena_ = std::move(o.arena_);
    cls_ = o.cls_;
    o.p_ = nullptr;
    o.bytes_ = 0;
  }
  return *this;
}

void DevBuf::reset() {
  if (p_) {
    if (arena_) arena_->give(p_, cls_);
    else cudaFreeAsync(p_, st_);
  }
  arena_.reset();
  p_ = nullptr;
  bytes_ = 0;
}

// ------------------------------------------------------------------ plan

static Ver parse_ver(const std::string& s) {
  if (s == "FULL") return kFull;
  if (s == "DELTA") return kDelta;
  if (s == "NEW") return kNew;
  throw Error{kErrPlan, "plan: bad version " + s};
}

static SourceDesc parse_source(const Json& j) {
  SourceDesc s;
  s.rel = j.at("rel").s();
  s.ver = parse_ver(j.at("ver").s());
  s.index = j.at("index").ints();
  s.prefix = j.at("prefix").strs();
  return s;
}

Database::Database(const std::string& plan_json, int device) : device_(device) {
  parse_plan(plan_json);
}

Database::~Database() {
  if (dev_ready_) {
    cudaSetDevice(device_);
    for (auto& kv : rels_)
      for (auto& v : kv.second->v) v.clear();
    for (auto& kv : rels_) kv.second->pending = Index{};
    for (auto& kv : rels_) kv.second->head = Index{};
    for (auto& kv : rels_) kv.second->dstaged.reset();
    d_small_.reset();
    // (every buffer of the stream's arena goes back before it closes: a
    // block returned later would be freed on the destroyed stream)
    inst_last_.clear();
    inst_bounds_d_.reset();
    arena_detach(L_.stream);
    cudaStreamSynchronize(L_.stream);
    if (h_small_) cudaFreeHost(h_small_);
    for (auto& kv : rels_)
      if (kv.second->pinned) cudaFreeHost(kv.second->pinned);
    for (auto& e : kev_) {
      cudaEventDestroy(e.a);
      cudaEventDestroy(e.b);
    }
    for (auto e : ev_pool_) cudaEventDestroy(e);
    if (loop_stream_) cudaStreamDestroy(loop_stream_);
    for (auto e : loop_ev_)
      if (e) cudaEventDestroy(e);
    if (own_stream_) cudaStreamDestroy(L_.stream);
    (void)cudaGetLastError();  // teardown errors must not surface in a later call
  }
}

void Database::parse_plan(const std::string& plan_json) {
  Json p = JsonParser(plan_json).parse();
  SRDL_REQUIRE(p.at("version").i() == 1, kErrPlan, "plan: unsupported version");
  name_ = p.has("name") ? p.at("name").s() : "plan";
  for (auto& r : p.at("relations").a()) {
    auto rel = std::make_unique<Relation>();
    rel->name = r.at("name").s();
    rel->arity = (int)r.at("arity").i();
    SRDL_REQUIRE(rel->arity >= 1, kErrPlan, "plan: relation arity must be >= 1");
    rel->input_file = r.at("input_file").s();
    rel->print_size = r.at("print_size").flag();
    rel->index_type = r.at("index_type").s();
    rel->lsm = rel->index_type.find("Device2LevelIndex") != std::string::npos;
    rel->canonical = r.at("canonical").ints();
    SRDL_REQUIRE((int)rel->canonical.size() == rel->arity, kErrPlan,
                 "plan: canonical index arity mismatch for " + rel->name);
    if (r.has("facts")) {
      for (auto& row : r.at("facts").a()) {
        const auto& vals = row.a();
        SRDL_REQUIRE((int)vals.size() == rel->arity, kErrPlan,
                     "plan: facts row of the wrong arity for " + rel->name);
        for (auto& x : vals) {
          SRDL_REQUIRE(x.i() >= 0 && x.i() <= 0xffffffffLL, kErrPlan,
                       "plan: facts value out of range for " + rel->name);
          rel->facts.push_back((uint32_t)x.i());
        }
      }
    }
    if (!rel->input_file.empty()) inputs_.push_back(rel->name);
    const std::string name = rel->name;
    const bool has_facts = !rel->facts.empty();
    rels_[name] = std::move(rel);
    if (has_facts) stage_facts(*rels_[name]);
  }
  for (auto& sj : p.at("steps").a()) {
    Step st;
    st.recursive = sj.at("recursive").flag();
    for (auto& oj : sj.at("ops").a()) {
      Op op;
      const std::string k = oj.at("op").s();
      if (k == "execute_pipeline") {
        op.kind = Op::Execute;
        op.rule = oj.at("rule").s();
        op.count = oj.at("count").flag();
        if (oj.has("shard")) {
          const std::string sh = oj.at("shard").s();
          if (sh == "work") {
            op.shard = Op::Work;
          } else if (sh == "key") {
            op.shard = Op::Key;
            op.shard_var = oj.at("shard_var").s();
          } else {
            // "exchange": the rule runs unrestricted, its tuples go to their
            // owners by the exchange op that follows it
            SRDL_REQUIRE(sh.empty() || sh == "exchange", kErrPlan,
                         "rule " + op.rule + ": unknown shard mode " + sh);
          }
        }
        for (auto& pj : oj.at("pipeline").a()) {
          PipeOp po;
          const std::string pk = pj.at("op").s();
          if (pk == "scan") {
            po.kind = PipeOp::Scan;
            po.sources.push_back(parse_source(pj));
            po.vars = pj.at("vars").strs();
          } else if (pk == "column_join") {
            po.kind = PipeOp::ColumnJoin;
            po.var = pj.at("var").s();
            for (auto& s : pj.at("sources").a()) po.sources.push_back(parse_source(s));
          } else if (pk == "cartesian_join") {
            po.kind = PipeOp::Cartesian;
            po.vars = pj.at("vars").strs();
            for (auto& s : pj.at("sources").a()) po.sources.push_back(parse_source(s));
            for (auto& v : pj.at("var_from_source").a()) po.var_from_source.push_back(v.strs());
          } else if (pk == "negation") {
            po.kind = PipeOp::Negation;
            po.sources.push_back(parse_source(pj));
            if (pj.has("const_prefix"))
              for (auto& cj : pj.at("const_prefix").a()) {
                const long long v = cj.i();
                SRDL_REQUIRE(v >= 0 && v <= 0xFFFFFFFFll, kErrPlan, "plan: negation constant out of range");
                po.const_prefix.push_back((uint32_t)v);
              }
            const size_t nb = po.const_prefix.size() + po.sources[0].prefix.size();
            SRDL_REQUIRE(nb >= 1 && nb <= 2, kErrUnsupported,
                         "plan: negation needs one or two bound values");
          } else if (pk == "filter") {
            po.kind = PipeOp::Filter;
            po.vars = pj.at("vars").strs();
            po.code = pj.at("code").s();
          } else if (pk == "insert_into") {
            po.kind = PipeOp::Insert;
            po.rel = pj.at("rel").s();
            po.vars = pj.at("vars").strs();
            po.index = pj.at("index").ints();
          } else {
            throw Error{kErrUnsupported, "plan: pipeline op '" + pk + "' is not supported"};
          }
          for (auto& s : po.sources)
            SRDL_REQUIRE(rels_.count(s.rel), kErrPlan, "plan: unknown relation " + s.rel);
          op.pipeline.push_back(std::move(po));
        }
      } else if (k == "inject_cpp_hook") {
        op.kind = Op::Hook;
      } else {
        op.rel = oj.at("rel").s();
        SRDL_REQUIRE(rels_.count(op.rel), kErrPlan, "plan: unknown relation " + op.rel);
        if (k == "rebuild_index") {
          op.kind = Op::Rebuild;
          op.ver = parse_ver(oj.at("ver").s());
          op.index = oj.at("index").ints();
        } else if (k == "clear_relation") {
          op.kind = Op::Clear;
          op.ver = parse_ver(oj.at("ver").s());
        } else if (k == "check_size") {
          op.kind = Op::CheckSize;
          op.ver = parse_ver(oj.at("ver").s());
        } else if (k == "compute_delta_index") {
          op.kind = Op::ComputeDelta;
          op.index = oj.at("index").ints();
        } else if (k == "merge_index") {
          op.kind = Op::Merge;
          op.index = oj.at("index").ints();
        } else if (k == "exchange") {
          op.kind = Op::Exchange;
        } else if (k == "rebuild_index_from_index") {
          op.kind = Op::RebuildFrom;
          op.ver = parse_ver(oj.at("ver").s());
          op.index = oj.at("index").ints();
          op.source_index = oj.at("source_index").ints();
        } else if (k == "post_stratum_reconstruct") {
          op.kind = Op::Reconstruct;
          op.index = oj.at("index").ints();
        } else {
          throw Error{kErrUnsupported, "plan: op '" + k + "' is not supported"};
        }
      }
      st.ops.push_back(std::move(op));
    }
    steps_.push_back(std::move(st));
  }
  step_stats_.resize(steps_.size());
}

Relation& Database::rel(const std::string& name) {
  auto it = rels_.find(name);
  SRDL_REQUIRE(it != rels_.end(), kErrArg, "unknown relation " + name);
  return *it->second;
}

bool Database::any_loaded() const {
  // rows a plan carries (facts) do not count as loaded inputs
  for (auto& kv : rels_)
    if (kv.second->loaded && kv.second->facts.empty()) return true;
  return false;
}

void Database::stage_facts(Relation& r) {
  load_rows(r.name, r.facts.data(), r.facts.size() / r.arity);
}

// ------------------------------------------------------------------ device

void Database::init_device() {
  SRDL_CUDA(cudaSetDevice(device_));
  if (dev_ready_) return;
  int sms = 0;
  SRDL_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
  L_.num_sms = sms;
  if (own_stream_) SRDL_CUDA(cudaStreamCreateWithFlags(&L_.stream, cudaStreamNonBlocking));
  // Keep freed blocks in the pool: iterations reuse the same sizes.
  cudaMemPool_t pool;
  SRDL_CUDA(cudaDeviceGetDefaultMemPool(&pool, device_));
  uint64_t thr = ~0ull;
  SRDL_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  arena_attach(L_.stream);
  SRDL_CUDA(cudaMallocHost(&h_small_, kSmallSlots * sizeof(uint64_t)));
  d_small_ = DevBuf(kSmallSlots * sizeof(uint64_t), L_.stream);
  dev_ready_ = true;
}

uint64_t Database::read_scalar(int slot) {
  SRDL_CUDA(cudaMemcpyAsync(h_small_ + slot, d_small_.as<uint64_t>() + slot, sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, L_.stream));
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  return h_small_[slot];
}

void Database::set_stream(cudaStream_t s) {
  SRDL_CUDA(cudaSetDevice(device_));
  if (!dev_ready_) {
    L_.stream = s;
    own_stream_ = false;
    return;
  }
  // Release everything allocated on the old stream before switching.
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  reset_device_state();
  arena_attach(s);
  for (auto& kv : rels_) {
    if (kv.second->dstaged_n) SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  }
  DevBuf keep_small(kSmallSlots * sizeof(uint64_t), s);
  std::vector<std::pair<Relation*, DevBuf>> moved;
  for (auto& kv : rels_) {
    Relation& r = *kv.second;
    if (!r.dstaged_n) continue;
    DevBuf nb(r.dstaged_n * 8, s);
    SRDL_CUDA(cudaMemcpyAsync(nb.as<void>(), r.dstaged.as<void>(), r.dstaged_n * 8,
                              cudaMemcpyDeviceToDevice, L_.stream));
    SRDL_CUDA(cudaStreamSynchronize(L_.stream));
    r.dstaged = std::move(nb);
  }
  d_small_ = std::move(keep_small);
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  arena_detach(L_.stream);
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  if (own_stream_) SRDL_CUDA(cudaStreamDestroy(L_.stream));
  L_.stream = s;
  own_stream_ = false;
}

cudaEvent_t make_event() {
  cudaEvent_t e;
  SRDL_CUDA(cudaEventCreate(&e));
  return e;
}

size_t Database::prof_begin(const std::string& name) {
  if (!profile_) return (size_t)-1;
  KEvent k{name, nullptr, nullptr, 0, 0};
  for (cudaEvent_t* e : {&k.a, &k.b}) {
    if (!ev_pool_.empty()) {
      *e = ev_pool_.back();
      ev_pool_.pop_back();
    } else {
      *e = make_event();
    }
  }
  SRDL_CUDA(cudaEventRecord(k.a, L_.stream));
  kev_.push_back(k);
  return kev_.size() - 1;
}

void Database::prof_end(size_t id, double bytes, double units) {
  if (id == (size_t)-1) return;
  SRDL_CUDA(cudaEventRecord(kev_[id].b, L_.stream));
  kev_[id].bytes = bytes;
  kev_[id].units = units;
}

void Database::prof_collect() {
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  for (auto& k : kev_) {
    float ms = 0;
    SRDL_CUDA(cudaEventElapsedTime(&ms, k.a, k.b));
    KernelStats& s = kstats_[k.name];
    s.ms += ms;
    s.bytes += k.bytes;
    s.units += k.units;
    s.scopes++;
    ev_pool_.push_back(k.a);
    ev_pool_.push_back(k.b);
  }
  kev_.clear();
}

void Database::reset_device_state() {
  for (auto& kv : rels_) {
    for (auto& v : kv.second->v) v.clear();
    kv.second->pending = Index{};
    kv.second->pending_delta = false;
    kv.second->head = Index{};
    kv.second->delta_epoch = kv.second->full_epoch = kv.second->base_epoch = 0;
  }
  counts_.clear();
  group_counts_.clear();
  kstats_.clear();
  loop_stats_ = LoopStats{};
  derived_ = 0;
  for (auto& s : step_stats_) s = StepStats{};
}

// ------------------------------------------------------------------ loading

void Database::load_rows(const std::string& name, const uint32_t* rows, uint64_t n) {
  Relation& r = rel(name);
  SRDL_REQUIRE(rows || n == 0, kErrArg, "load_rows: null rows");
  SRDL_REQUIRE(r.arity <= 4, kErrUnsupported,
               "relation " + name + ": only relations of arity 1 to 4 can be loaded");
  r.staged.insert(r.staged.end(), rows, rows + n * r.arity);
  // The value bound is taken once here, not on every run (a run re-uploads
  // the rows but never rescans them on the host).
  uint32_t mx = r.staged_max;
  for (uint64_t i = 0; i < n * r.arity; i++) mx = rows[i] > mx ? rows[i] : mx;
  r.staged_max = mx;
  r.pinned_valid = false;  // page-locked mirror is stale
  r.loaded = true;
}

void Database::set_count_groups(const std::string& rule, const uint32_t* bounds,
                                uint64_t n_bounds) {
  if (n_bounds == 0) {
    group_bounds_.erase(rule);
    group_counts_.erase(rule);
    return;
  }
  SRDL_REQUIRE(bounds && n_bounds >= 2 && n_bounds <= (1ull << 31), kErrArg,
               "set_count_groups: need 2 or more bounds");
  for (uint64_t j = 0; j + 1 < n_bounds; j++)
    SRDL_REQUIRE(bounds[j] <= bounds[j + 1], kErrArg, "set_count_groups: bounds must be non-decreasing");
  bool known = false;
  for (auto& st : steps_)
    for (auto& op : st.ops)
      if (op.kind == Op::Execute && op.rule == rule) {
        SRDL_REQUIRE(op.count, kErrArg, "set_count_groups: rule " + rule + " is not count-only");
        known = true;
      }
  SRDL_REQUIRE(known, kErrArg, "set_count_groups: unknown rule " + rule);
  group_bounds_[rule].assign(bounds, bounds + n_bounds);
  group_counts_.erase(rule);
}

void Database::group_counts(const std::string& rule, uint64_t* out, uint64_t n_groups) const {
  auto it = group_bounds_.find(rule);
  SRDL_REQUIRE(it != group_bounds_.end(), kErrArg, "group_counts: no groups set for " + rule);
  SRDL_REQUIRE(n_groups == it->second.size() - 1, kErrArg, "group_counts: wrong group count");
  auto c = group_counts_.find(rule);
  for (uint64_t g = 0; g < n_groups; g++) out[g] = c == group_counts_.end() ? 0 : c->second[g];
}

void Database::clear_inputs() {
  for (auto& kv : rels_) {
    Relation& r = *kv.second;
    r.staged.clear();
    r.staged.shrink_to_fit();
    r.staged_max = 0;
    r.pinned_valid = false;
    r.dstaged.reset();
    r.dstaged_n = 0;
    r.dstaged_max = 0;
    r.loaded = false;
    if (!r.facts.empty()) stage_facts(r);
  }
}

void Database::range_counts(const std::string& name, const uint32_t* bounds, uint64_t n_bounds,
                            uint64_t* counts) {
  Relation& r = rel(name);
  SRDL_REQUIRE(bounds || n_bounds == 0, kErrArg, "range_counts: null bounds");
  if (n_bounds < 2) return;
  for (uint64_t j = 0; j + 1 < n_bounds; j++)
    SRDL_REQUIRE(bounds[j] <= bounds[j + 1], kErrArg, "range_counts: bounds must be non-decreasing");
  if (!r.v[kFull].has_index() || r.arity > 2) {
    for (uint64_t j = 0; j + 1 < n_bounds; j++) counts[j] = 0;
    return;
  }
  SRDL_CUDA(cudaSetDevice(device_));
  if (r.head.n) compact_head(r);
  // a binary relation's two columns lie in the same range, so any FULL
  // permutation's high word tells the range (no extra permutation sorted)
  Index& ix = r.arity == 2 ? binary_full_index(r, nullptr) : ensure_index(r, kFull, identity_perm(r.arity));
  DevBuf d_bounds(n_bounds * 4, L_.stream);
  DevBuf d_pos(n_bounds * 8, L_.stream);
  SRDL_CUDA(cudaMemcpyAsync(d_bounds.as<void>(), bounds, n_bounds * 4, cudaMemcpyHostToDevice,
                            L_.stream));
  bounds_positions(L_, ix.keys.as<uint64_t>(), ix.n, d_bounds.as<uint32_t>(), n_bounds,
                   d_pos.as<uint64_t>());
  std::vector<uint64_t> pos(n_bounds);
  SRDL_CUDA(cudaMemcpyAsync(pos.data(), d_pos.as<void>(), n_bounds * 8, cudaMemcpyDeviceToHost,
                            L_.stream));
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  for (uint64_t j = 0; j + 1 < n_bounds; j++) counts[j] = pos[j + 1] - pos[j];
}

void Database::load_device_rows(const std::string& name, const uint32_t* d_rows, uint64_t n) {
  Relation& r = rel(name);
  SRDL_REQUIRE(d_rows || n == 0, kErrArg, "load_device_rows: null rows");
  SRDL_REQUIRE(r.arity == 2, kErrUnsupported, "load_device_rows: binary relations only");
  SRDL_REQUIRE(r.dstaged_n == 0, kErrState, "load_device_rows: relation already has device rows");
  init_device();
  r.dstaged = DevBuf(std::max<uint64_t>(n, 1) * 8, L_.stream);
  if (n)
    SRDL_CUDA(cudaMemcpyAsync(r.dstaged.as<void>(), d_rows, n * 8, cudaMemcpyDeviceToDevice,
                              L_.stream));
  max_u32(L_, r.dstaged.as<uint32_t>(), n * 2, reinterpret_cast<uint32_t*>(d_small_.as<uint64_t>() + 4));
  SRDL_CUDA(cudaMemsetAsync(reinterpret_cast<uint32_t*>(d_small_.as<uint64_t>() + 4) + 1, 0, 4, L_.stream));
  r.dstaged_max = (uint32_t)read_scalar(4);
  r.dstaged_n = n;
  r.loaded = true;
}

// Sorted unique keys of `in` (packed in some order) into `out`, optionally
// dropping keys present in `full`.
void Database::sort_into(Index& out, const uint64_t* in, uint64_t n, bool swap, const Index* full,
                         const Index* head, int key_bits) {
  // key halves hold at most key_bits bits (0: the value bits of the inputs)
  const int kb = key_bits > 0 ? key_bits : bits_;
  out.keys = DevBuf(std::max<uint64_t>(n, 1) * 8, L_.stream);
  out.trie = false;
  out.split.clear();
  if (n == 0) {
    out.n = 0;
    return;
  }
  DevBuf scratch(sort_scratch_bytes(n, kb), L_.stream);
  Scratch s{scratch.as<char>(), scratch.bytes(), 0};
  const bool hd = head && head->n;
  const bool diff = (full && full->n) || hd;
  size_t pid = prof_begin(diff ? "sort_dedup_diff" : "sort_dedup");
  sort_dedup(L_, in, n, kb, swap, full && full->n ? full->keys.as<uint64_t>() : nullptr,
             full ? full->n : 0, out.keys.as<uint64_t>(), d_small_.as<uint64_t>(), s,
             hd ? head->keys.as<uint64_t>() : nullptr, hd ? head->n : 0);
  prof_end(pid, 0, (double)n);
  out.n = read_scalar(0);
  if (trace_)
    fprintf(stderr, "srdl: sort n=%llu full=%llu head=%llu out=%llu\n", (unsigned long long)n,
            (unsigned long long)(full ? full->n : 0), (unsigned long long)(hd ? head->n : 0),
            (unsigned long long)out.n);
  if (pid != (size_t)-1) {
    // Algorithmic bytes: each counting pass reads and writes the packed
    // keys once; packing reads the input; the dedup pass reads the sorted
    // keys and writes the distinct ones (plus one probe word per key into
    // FULL when the delta is fused).
    const double ks = 2 * kb <= 32 ? 4 : 8;
    const double passes = (2 * kb + L_.radix_bits - 1) / L_.radix_bits;
    kev_[pid].bytes = passes * 2 * ks * n + 8.0 * n + ks * n + ks * n + 8.0 * out.n +
                      (diff ? 8.0 * n : 0);
  }
}

void Database::upload_inputs() {
  uint32_t mx = 0;
  for (auto& kv : rels_) {
    if (!kv.second->staged.empty()) mx = std::max(mx, kv.second->staged_max);
    if (kv.second->dstaged_n) mx = std::max(mx, kv.second->dstaged_max);
  }
  dom_max_ = mx;
  bits_ = value_bits(mx);
  for (auto& kv : rels_) {
    Relation& r = *kv.second;
    if (r.arity <= 2) continue;
    const int total = r.arity * bits_;
    r.pack_bits = total <= 64 ? bits_ : 0;
    r.pack_half = total <= 64 ? (total + 1) / 2 : 0;
  }
  for (auto& kv : rels_) {
    Relation& r = *kv.second;
    if (!r.loaded) continue;
    if (r.dstaged_n) {
      SRDL_REQUIRE(r.staged.empty(), kErrState,
                   "relation " + r.name + " has both host and device rows staged");
      Index& ix = r.v[kFull].idx[r.canonical];
      sort_into(ix, r.dstaged.as<uint64_t>(), r.dstaged_n, r.canonical == std::vector<int>{0, 1},
                nullptr);
      continue;
    }
    const uint64_t n = r.staged.size() / r.arity;
    DevBuf raw(std::max<uint64_t>(n, 1) * 8, L_.stream);
    bool swap = false;
    if (r.arity == 2) {
      // Host rows are copied once into page-locked memory so that every run
      // uploads them with one asynchronous DMA.
      // (The page-locked buffer is kept and only grows: cudaFreeHost would
      // synchronise the whole device and stall other handles' streams.)
      if (!r.pinned_valid && n) {
        if (r.staged.size() > r.pinned_cap) {
          if (r.pinned) SRDL_CUDA(cudaFreeHost(r.pinned));
          r.pinned = nullptr;
          r.pinned_cap = std::max(r.staged.size(), r.pinned_cap + r.pinned_cap / 2);
          SRDL_CUDA(cudaMallocHost(&r.pinned, r.pinned_cap * 4));
        }
        memcpy(r.pinned, r.staged.data(), r.staged.size() * 4);
        r.pinned_valid = true;
      }
      // A row-major (c0, c1) pair read as a little-endian uint64 is
      // (c1 << 32) | c0, i.e. the key of permutation (1,0).
      if (n)
        SRDL_CUDA(cudaMemcpyAsync(raw.as<uint64_t>(), r.pinned, n * 8, cudaMemcpyHostToDevice,
                                  L_.stream));
      swap = (r.canonical == std::vector<int>{0, 1});
    } else if (r.arity == 1) {
      std::vector<uint64_t> k(n);
      for (uint64_t i = 0; i < n; i++) k[i] = (uint64_t)r.staged[i] << 32;
      SRDL_CUDA(cudaMemcpyAsync(raw.as<uint64_t>(), k.data(), n * 8, cudaMemcpyHostToDevice,
                                L_.stream));
      SRDL_CUDA(cudaStreamSynchronize(L_.stream));
    } else {
      // arity 3-4: columns in canonical order, packed pack_bits apiece and
      // split at pack_half bits (the layout the joins emit)
      SRDL_REQUIRE(r.pack_half > 0, kErrUnsupported,
                   "relation " + r.name + ": arity x value bits must be <= 64 to load it");
      const int k = r.arity, b = r.pack_bits, h = r.pack_half;
      std::vector<uint64_t> keys(n);
      for (uint64_t i = 0; i < n; i++) {
        const uint32_t* row = &r.staged[i * k];
        uint64_t p = 0;
        for (int j = 0; j < k; j++) p = (p << b) | row[r.canonical[j]];
        keys[i] = ((p >> h) << 32) | (p & ((1ull << h) - 1));
      }
      SRDL_CUDA(cudaMemcpyAsync(raw.as<uint64_t>(), keys.data(), n * 8, cudaMemcpyHostToDevice,
                                L_.stream));
      SRDL_CUDA(cudaStreamSynchronize(L_.stream));
    }
    Index& ix = r.v[kFull].idx[r.canonical];
    sort_into(ix, raw.as<uint64_t>(), n, swap, nullptr, nullptr, r.arity > 2 ? r.pack_half : 0);
  }
}

// ------------------------------------------------------------------ indexes

Index& Database::full_base(Relation& r, const std::vector<int>& perm) {
  auto it = r.v[kFull].idx.find(perm);
  if (it != r.v[kFull].idx.end()) return it->second;
  return ensure_index(r, kFull, perm);
}

void Database::compact_head(Relation& r) {
  if (r.head.n == 0) return;
  Index h = std::move(r.head);
  r.head = Index{};
  Index& f = full_base(r, r.canonical);
  Index m;
  m.n = f.n + h.n;
  m.keys = DevBuf(m.n * 8, L_.stream);
  size_t pid = prof_begin("merge");
  merge_disjoint(L_, f.keys.as<uint64_t>(), f.n, h.keys.as<uint64_t>(), h.n, m.keys.as<uint64_t>());
  prof_end(pid, 16.0 * m.n, (double)m.n);
  m.epoch = r.full_epoch;
  r.v[kFull].idx.clear();
  r.v[kFull].idx[r.canonical] = std::move(m);
}

void Database::subtract_head(Relation& r, const std::vector<int>& perm, Index& d) {
  if (r.head.n == 0 || d.n == 0 || perm != r.canonical) return;
  Index& h = r.head;
  Index out;
  out.keys = DevBuf(d.n * 8, L_.stream);
  DevBuf scratch(diff_scratch_bytes(d.n) + 1024, L_.stream);
  Scratch s{scratch.as<char>(), scratch.bytes(), 0};
  size_t pid = prof_begin("set_difference");
  set_difference(L_, d.keys.as<uint64_t>(), d.n, h.keys.as<uint64_t>(), h.n,
                 out.keys.as<uint64_t>(), d_small_.as<uint64_t>(), s);
  out.n = read_scalar(0);
  prof_end(pid, 8.0 * (d.n + h.n + out.n), (double)d.n);
  d = std::move(out);
}

Index& Database::ensure_index(Relation& r, Ver v, const std::vector<int>& perm) {
  SRDL_REQUIRE((int)perm.size() == r.arity, kErrPlan, "index arity mismatch on " + r.name);
  if (v == kFull && r.head.n) compact_head(r);
  RelVersion& rv = r.v[v];
  auto it = rv.idx.find(perm);
  if (it != rv.idx.end()) {
    if (v != kFull || it->second.epoch >= r.full_epoch) return it->second;
    rv.idx.erase(it);  // a FULL permutation that missed the latest delta
  }
  Index& ix = rv.idx[perm];
  // Build from an existing permutation of the same version (for FULL, one
  // that holds every merged delta).
  const Index* src = nullptr;
  for (auto& kv : rv.idx) {
    if (&kv.second == &ix) continue;
    if (!src || (v == kFull && kv.second.epoch > src->epoch)) src = &kv.second;
  }
  if (src) {
    SRDL_REQUIRE(r.arity == 2, kErrUnsupported, "secondary index on non-binary relation " + r.name);
    sort_into(ix, src->keys.as<uint64_t>(), src->n, true, nullptr);
    ix.epoch = src->epoch;
    return ix;
  }
  ix.n = 0;
  ix.keys = DevBuf(8, L_.stream);
  return ix;
}

void Database::ensure_trie(Relation& r, Index& ix, int64_t hi_max) {
  (void)r;
  if (ix.trie) return;
  const uint64_t hmax = hi_max < 0 ? (uint64_t)dom_max_ : (uint64_t)hi_max;
  const uint64_t n = ix.n;
  size_t pid = prof_begin("trie_build");
  ix.lo = DevBuf(std::max<uint64_t>(n, 1) * 4, L_.stream);
  ix.roots = DevBuf(std::max<uint64_t>(n, 1) * 4, L_.stream);
  build_lo(L_, ix.keys.as<uint64_t>(), n, ix.lo.as<uint32_t>());
  DevBuf scratch(roots_scratch_bytes(n) + 1024, L_.stream);
  Scratch s{scratch.as<char>(), scratch.bytes(), 0};
  // the root count stays on the device: kernels read it, the host never waits for it
  ix.nroots_d = DevBuf(8, L_.stream);
  build_roots(L_, ix.keys.as<uint64_t>(), n, ix.roots.as<uint32_t>(), ix.nroots_d.as<uint64_t>(), s);
  ix.dir_n = 0;
  if (hmax + 2 <= kDenseDirMax) {
    ix.dir_n = (uint32_t)(hmax + 2);
    ix.dir = DevBuf((size_t)ix.dir_n * 4, L_.stream);
    build_dir(L_, ix.keys.as<uint64_t>(), n, ix.dir.as<uint32_t>(), ix.dir_n);
  }
  prof_end(pid, 8.0 * n + 4.0 * n + 8.0 * n + 4.0 * ix.dir_n, (double)n);
  ix.trie = true;
}

// With SRDL_HASH_MIN=L set, child lists longer than L values of an index
// probed by a column join get an open-addressing table.  Off by default: on
// the R-MAT triangle workload the binary search over sorted, co-located
// probes measured faster (47.8 ms vs 53.0 ms per step at L = 32).
static uint32_t hash_min_len() {
  static const uint32_t v = [] {
    const char* e = getenv("SRDL_HASH_MIN");
    return e ? (uint32_t)strtoul(e, nullptr, 10) : 0u;
  }();
  return v;
}

void Database::set_option(const std::string& name, int64_t value) {
  SRDL_REQUIRE(value >= 0, kErrArg, "set_option: negative value for " + name);
  if (name == "bitmap_mb") opt_bitmap_mb_ = value;
  else if (name == "hash_min") opt_hash_min_ = value;
  else if (name == "lsm_compact_pct") opt_lsm_pct_ = value;
  else if (name == "mem_limit_mb") opt_mem_limit_ = (uint64_t)value << 20;
  else if (name == "device_loop") opt_device_loop_ = value ? 1 : 0;
  else if (name == "device_loop_cap_limit") opt_loop_cap_limit_ = (uint64_t)value;
  else if (name == "shard_world") {
    SRDL_REQUIRE(value >= 1 && value <= 65536, kErrArg, "set_option: shard_world out of [1, 65536]");
    shard_world_ = value;
  } else if (name == "shard_rank") shard_rank_ = value;
  else if (name == "radix_bits") {
    SRDL_REQUIRE(value >= 1 && value <= 8, kErrArg, "set_option: radix_bits out of [1, 8]");
    L_.radix_bits = (int)value;
  } else if (name == "join_chunk") {
    SRDL_REQUIRE(value >= 64 && value <= (1 << 20), kErrArg, "set_option: join_chunk out of [64, 2^20]");
    L_.join_chunk = (int)value;
  } else if (name == "join_blocks_per_sm") {
    SRDL_REQUIRE(value >= 1 && value <= 64, kErrArg, "set_option: join_blocks_per_sm out of [1, 64]");
    L_.join_bpsm = (int)value;
  } else if (name == "pivot_min") {
    SRDL_REQUIRE(value >= 0 && value <= (1ll << 32), kErrArg, "set_option: pivot_min out of [0, 2^32]");
    opt_pivot_min_ = value;
  }
  else throw Error{kErrArg, "set_option: unknown option " + name};
}

void Database::ensure_hash(Index& ix) {
  if (ix.hash_done) return;
  ix.hash_done = true;
  const uint32_t min_len = opt_hash_min_ >= 0 ? (uint32_t)opt_hash_min_ : hash_min_len();
  if (min_len == 0 || !ix.dir_n || ix.n == 0 || dom_max_ == 0xffffffffu) return;
  size_t pid = prof_begin("child_hash_build");
  DevBuf scratch(child_hash_scratch_bytes(ix.dir_n), L_.stream);
  Scratch s{scratch.as<char>(), scratch.bytes(), 0};
  const uint32_t nv = ix.dir_n - 1;
  uint64_t* sizes = s.take<uint64_t>(nv);
  uint64_t* offs = s.take<uint64_t>(nv + 1);
  child_hash_plan(L_, ix.dir.as<uint32_t>(), ix.dir_n, min_len, sizes, offs, s);
  SRDL_CUDA(cudaMemcpyAsync(h_small_ + 5, offs + nv, 8, cudaMemcpyDeviceToHost, L_.stream));
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  const uint64_t slots = h_small_[5];
  if (slots == 0 || slots >= 0xffffffffull) {
    prof_end(pid, 0, 0);
    return;
  }
  ix.hdir = DevBuf((size_t)nv * 4, L_.stream);
  ix.hpool = DevBuf(slots * 4, L_.stream);
  SRDL_CUDA(cudaMemsetAsync(ix.hpool.as<void>(), 0xff, slots * 4, L_.stream));
  child_hash_build(L_, ix.keys.as<uint64_t>(), ix.n, ix.dir.as<uint32_t>(), ix.dir_n, sizes, offs,
                   ix.hdir.as<uint32_t>(), ix.hpool.as<uint32_t>());
  prof_end(pid, 8.0 * ix.n + 4.0 * slots + 16.0 * nv, (double)ix.n);
}

// Bitmaps for the longest child lists of an index probed by a column join:
// a membership test becomes one load instead of a binary search of up to 16
// dependent steps.  The threshold is the smallest length kBitmapMinLen * 2^k
// whose bitmaps (one bit per value of the domain each) fit in SRDL_BITMAP_MB
// (default 768 MB; 0 disables); domains above 2^24 values get none.  On the
// R-MAT scale-20 triangle count the default picks lists of 512 or more
// (4,552 bitmaps, 569 MB): 14.1 ms per step, against 14.8 ms at 1,024,
// 16.1 ms at 2,048 and 14.2-14.4 ms at 256 and 128.
static uint64_t bitmap_budget() {
  static const uint64_t v = [] {
    const char* e = getenv("SRDL_BITMAP_MB");
    return (e ? (uint64_t)strtoull(e, nullptr, 10) : 768ull) << 20;
  }();
  return v;
}

void Database::ensure_bitmaps(Index& ix) {
  if (ix.bitmap_done) return;
  ix.bitmap_done = true;
  const uint64_t budget = opt_bitmap_mb_ >= 0 ? (uint64_t)opt_bitmap_mb_ << 20 : bitmap_budget();
  if (budget == 0 || !ix.dir_n || ix.n < kBitmapMinLen || dom_max_ >= (1u << 24)) return;
  const uint32_t bwords = (uint32_t)(((uint64_t)dom_max_ + 1 + 31) / 32);
  size_t pid = prof_begin("trie_build");
  DevBuf cnt(kBitmapLevels * 8 + 8, L_.stream);
  bitmap_plan(L_, ix.dir.as<uint32_t>(), ix.dir_n, cnt.as<unsigned long long>());
  unsigned long long c[kBitmapLevels];
  SRDL_CUDA(cudaMemcpyAsync(c, cnt.as<void>(), sizeof(c), cudaMemcpyDeviceToHost, L_.stream));
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  int level = -1;
  for (int k = 0; k < kBitmapLevels; k++)
    if (c[k] && c[k] * bwords * 4ull <= budget) {
      level = k;
      break;
    }
  if (level < 0) {
    prof_end(pid, 0, 0);
    return;
  }
  const uint64_t slots = c[level];
  ix.bwords = bwords;
  ix.bdir = DevBuf((size_t)(ix.dir_n - 1) * 4, L_.stream);
  ix.bpool = DevBuf(slots * bwords * 4, L_.stream);
  SRDL_CUDA(cudaMemsetAsync(ix.bpool.as<void>(), 0, slots * bwords * 4, L_.stream));
  bitmap_build(L_, ix.keys.as<uint64_t>(), ix.n, ix.dir.as<uint32_t>(), ix.dir_n, kBitmapMinLen << level,
               ix.bdir.as<uint32_t>(), ix.bpool.as<uint32_t>(), bwords,
               reinterpret_cast<unsigned int*>(cnt.as<unsigned long long>() + kBitmapLevels));
  prof_end(pid, 8.0 * ix.n + 4.0 * slots * bwords + 8.0 * ix.dir_n, (double)ix.n);
}

TrieView Database::view2(Index& ix) {
  SRDL_REQUIRE(ix.trie, kErrState, "view of an index without its trie");
  TrieView t;
  t.keys = ix.keys.as<uint64_t>();
  t.lo = ix.lo.as<uint32_t>();
  t.roots = ix.roots.as<uint32_t>();
  t.dir = ix.dir_n ? ix.dir.as<uint32_t>() : nullptr;
  t.hdir = ix.hdir.bytes() ? ix.hdir.as<uint32_t>() : nullptr;
  t.hpool = ix.hpool.bytes() ? ix.hpool.as<uint32_t>() : nullptr;
  t.bdir = ix.bdir.bytes() ? ix.bdir.as<uint32_t>() : nullptr;
  t.bpool = ix.bpool.bytes() ? ix.bpool.as<uint32_t>() : nullptr;
  t.bwords = ix.bwords;
  t.bslots = ix.bwords ? (uint32_t)(ix.bpool.bytes() / ((size_t)ix.bwords * 4)) : 0;
  t.n = ix.n;
  t.n_roots_d = ix.nroots_d.as<uint64_t>();
  t.dir_n = ix.dir_n;
  t.arity = 2;
  return t;
}

// The pair and row views of a ternary relation's packed array `canon` (in the
// relation's canonical column order) for the column order `order`: the
// tuples are re-packed in that order and sorted when it differs, then split.
Split3& Database::ensure_split(Relation& r, Index& canon, const std::vector<int>& order) {
  auto it = canon.split.find(order);
  if (it != canon.split.end()) return *it->second;
  SRDL_REQUIRE(r.arity == 3 && r.pack_half > 0, kErrUnsupported,
               "relation " + r.name + ": ternary reads need arity x value bits <= 64");
  auto sp = std::make_shared<Split3>();
  const int b = r.pack_bits, h = r.pack_half;
  const uint64_t n = canon.n;
  const uint64_t* keys = canon.keys.as<uint64_t>();
  Index sorted;
  if (order != r.canonical && n) {
    int sel[3];
    for (int j = 0; j < 3; j++) {
      sel[j] = -1;
      for (int q = 0; q < 3; q++)
        if (r.canonical[q] == order[j]) sel[j] = q;
      SRDL_REQUIRE(sel[j] >= 0, kErrPlan, "relation " + r.name + ": bad column order");
    }
    DevBuf re(n * 8, L_.stream);
    repack3(L_, keys, n, b, h, sel, re.as<uint64_t>());
    sort_into(sorted, re.as<uint64_t>(), n, false, nullptr, nullptr, h);
    keys = sorted.keys.as<uint64_t>();
  }
  sp->pair.keys = DevBuf(std::max<uint64_t>(n, 1) * 8, L_.stream);
  sp->rows.keys = DevBuf(std::max<uint64_t>(n, 1) * 8, L_.stream);
  DevBuf scratch(split3_scratch_bytes(n), L_.stream);
  Scratch s{scratch.as<char>(), scratch.bytes(), 0};
  size_t pid = prof_begin("split3");
  split3(L_, keys, n, b, h, sp->pair.keys.as<uint64_t>(), sp->rows.keys.as<uint64_t>(),
         d_small_.as<uint64_t>(), s);
  prof_end(pid, 8.0 * n + 3 * 8.0 * n + 8.0 * n, (double)n);
  sp->pair.n = n ? read_scalar(0) : 0;
  sp->rows.n = n;
  ensure_trie(r, sp->pair);
  ensure_trie(r, sp->rows, sp->pair.n ? (int64_t)sp->pair.n - 1 : 0);
  Split3& ref = *sp;
  canon.split[order] = std::move(sp);
  return ref;
}

TrieView Database::view(Relation& r, Index& ix) {
  ensure_trie(r, ix);
  TrieView t;
  t.keys = ix.keys.as<uint64_t>();
  t.lo = ix.lo.as<uint32_t>();
  t.roots = ix.roots.as<uint32_t>();
  t.dir = ix.dir_n ? ix.dir.as<uint32_t>() : nullptr;
  t.hdir = ix.hdir.bytes() ? ix.hdir.as<uint32_t>() : nullptr;
  t.hpool = ix.hpool.bytes() ? ix.hpool.as<uint32_t>() : nullptr;
  t.bdir = ix.bdir.bytes() ? ix.bdir.as<uint32_t>() : nullptr;
  t.bpool = ix.bpool.bytes() ? ix.bpool.as<uint32_t>() : nullptr;
  t.bwords = ix.bwords;
  t.bslots = ix.bwords ? (uint32_t)(ix.bpool.bytes() / ((size_t)ix.bwords * 4)) : 0;
  t.n = ix.n;
  t.n_roots_d = ix.nroots_d.as<uint64_t>();
  t.dir_n = ix.dir_n;
  t.arity = r.arity;
  return t;
}

}  // namespace srdl
