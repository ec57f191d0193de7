// loop.cu -- the device loop: a recursive step's iterations captured in one
// CUDA graph and repeated on the device until the delta is empty.
//
// Replaces, for the steps it accepts, the host-driven iteration of the
// generated fixpoint (step_N of src/srdatalog/codegen/jit/orchestrator_jit.py:
// 600-747: run the pipelines, rebuild NEW, compute DELTA, merge, read the
// delta sizes on the host, repeat) and the small-delta fused path
// (complete_runner.py:302-376), whose speculative output capacity with an
// overflow replay it shares.
//
// How.  Iteration 0 of a recursive step runs on the host path (it reads FULL
// for DELTA, and builds the indexes, tries and bitmaps of the relations the
// step only reads).  From then on, when the step qualifies (loop_eligible),
// every buffer an iteration touches is allocated up front with a capacity
// learned from the sizes seen so far, every count stays on the device, and
// the kernels of one iteration are captured twice -- reading FULL / DELTA
// from buffer set 0 and writing set 1, then the reverse -- into a graph
//
//     WHILE (go) { iteration(0 -> 1); control; IF (go) { iteration(1 -> 0); control } }
//
// whose control kernel counts the iteration, sums the new deltas and sets
// the conditions: the loop stops on an empty delta (the fixpoint), at the
// run's iteration limit, or when a kernel found a capacity too small (the
// overflow flag; kernels never write past a capacity).  One launch, one
// host synchronisation.  On overflow the failed iteration's inputs are
// intact (they are the other buffer set): the host resumes from them on the
// host path, and the next entry sizes the buffers from the larger counts
// that path measures.  Results are those of the host path: the same
// kernels, the same DELTA = unique(NEW) - FULL, FULL |= DELTA.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <set>

#include "runtime.h"

namespace srdl {

namespace {

// Counts of one relation in the loop (device memory).
struct LoopCounts {
  uint64_t n_full[2];
  uint64_t n_delta[2];
  uint64_t n_new;
  uint64_t n_roots[2];
  uint64_t derived;  // NEW keys produced by the loop's complete iterations
};

struct LoopCtl {
  unsigned int overflow;         // a capacity was too small in the current iteration
  unsigned int parity;           // buffer set holding the latest complete iteration
  unsigned long long done;       // complete iterations
  unsigned long long remaining;  // iterations this launch may still do
  unsigned long long bodies;     // iterations started (complete or not)
  double alg_bytes;              // algorithmic bytes of the complete iterations (as the host path counts them)
};

// ks: packed key bytes of the sort, passes: its counting passes.
__global__ void loop_ctrl_kernel(LoopCtl* ctl, LoopCounts* cnt, int nrel, int p, int ks, int passes,
                                 cudaGraphConditionalHandle hw, cudaGraphConditionalHandle hi,
                                 int set_if) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  ctl->bodies++;
  unsigned go = 0;
  if (!ctl->overflow) {
    ctl->done++;
    ctl->parity = 1 - p;
    uint64_t delta = 0;
    for (int r = 0; r < nrel; r++) {
      const double nn = (double)cnt[r].n_new, nd = (double)cnt[r].n_delta[1 - p];
      const double nf = (double)cnt[r].n_full[p];
      delta += cnt[r].n_delta[1 - p];
      cnt[r].derived += cnt[r].n_new;
      // emitted keys, the sort with its fused difference, the merge and
      // the delta's trie view -- the bytes the host path charges for them
      ctl->alg_bytes += 8.0 * nn + passes * 2.0 * ks * nn + 8.0 * nn + 2.0 * ks * nn + 8.0 * nd +
                        8.0 * nn + 16.0 * (nf + nd) + 16.0 * nd;
    }
    go = delta > 0 && ctl->done < ctl->remaining;
  }
  cudaGraphSetConditional(hw, go);
  if (set_if) cudaGraphSetConditional(hi, go);
}

constexpr uint64_t kLoopMaxIters = 20000;  // iterations one graph launch may run

// n rounded up to a quarter step of its power of two (at least 1024).
uint64_t round_cap(uint64_t n) {
  if (n <= 1024) return 1024;
  uint64_t p = 1024;
  while (p * 2 <= n) p <<= 1;
  const uint64_t q = p / 4;
  return (n + q - 1) / q * q;
}

}  // namespace

// Buffers of one relation the step computes.
struct LoopRel {
  Relation* r = nullptr;
  uint64_t cap_new = 0, cap_delta = 0, cap_full = 0;  // raw NEW, DELTA (<= cap_new), FULL
  int producers = 0;  // execute ops inserting into it
  DevBuf newk, sort_scr, trie_scr;
  DevBuf full[2], delta[2], lo[2], roots[2], dir[2];
};

// Buffers of one join level of one pipeline.
struct LoopLevel {
  uint64_t cap_rows = 1, cap_total = 0;
  DevBuf wscr, xscr, count;
  DevBuf cols[kMaxSlots];
};

struct LoopCtx {
  std::vector<LoopRel> rels;
  std::vector<std::vector<LoopLevel>> pipes;  // per execute op
  DevBuf cnt, ctl;
  uint32_t dir_n = 0;
  LoopCounts* cnt_d() { return cnt.as<LoopCounts>(); }
  LoopCtl* ctl_d() { return ctl.as<LoopCtl>(); }
  int rel_index(const std::string& name) const {
    for (size_t i = 0; i < rels.size(); i++)
      if (rels[i].r->name == name) return (int)i;
    return -1;
  }
};

// Relations a step computes (those it takes a delta of).
static std::vector<std::string> computed_rels(const Step& st) {
  std::vector<std::string> out;
  for (auto& op : st.ops)
    if (op.kind == Op::ComputeDelta && std::find(out.begin(), out.end(), op.rel) == out.end())
      out.push_back(op.rel);
  return out;
}

bool Database::loop_eligible(const Step& st, std::string& why) {
  auto no = [&](const std::string& w) {
    why = w;
    return false;
  };
  if (!st.recursive) return no("not a recursive step");
  if (shard_world_ > 1) return no("sharded evaluation");
  if ((uint64_t)dom_max_ + 2 > (1ull << 24)) return no("value domain above 2^24 (no dense directory)");
  const std::vector<std::string> comp = computed_rels(st);
  const std::set<std::string> computed(comp.begin(), comp.end());
  if (computed.empty() || computed.size() > 8) return no("computes no relation, or more than 8");
  bool maintenance = false;
  std::map<std::string, int> rebuilt, merged;
  for (auto& op : st.ops) {
    switch (op.kind) {
      case Op::Execute: {
        if (maintenance) return no("a pipeline after the maintenance ops");
        if (op.count) return no("count-only rule " + op.rule);
        if (op.shard != Op::NoShard) return no("sharded rule " + op.rule);
        for (auto& po : op.pipeline) {
          if (po.kind == PipeOp::Insert) {
            Relation& t = rel(po.rel);
            if (!computed.count(po.rel))
              return no("rule " + op.rule + " inserts into a relation the step does not compute");
            if (t.arity != 2 || po.index != t.canonical)
              return no("rule " + op.rule + " does not insert a binary tuple in canonical order");
            continue;
          }
          for (auto& d : po.sources) {
            Relation& r = rel(d.rel);
            if (r.arity > 2) return no("rule " + op.rule + " reads a relation of arity > 2");
            if (d.ver == kNew) return no("rule " + op.rule + " reads NEW");
            if (!computed.count(d.rel)) continue;
            if (d.ver != kDelta) return no("rule " + op.rule + " reads FULL of a relation the step computes");
            if (d.index != r.canonical) return no("rule " + op.rule + " reads a DELTA in another order");
            if (po.kind == PipeOp::Scan || po.kind == PipeOp::Negation)
              return no("rule " + op.rule + " scans or negates a DELTA");
          }
        }
        break;
      }
      case Op::Rebuild:
        maintenance = true;
        if (op.ver != kNew || !computed.count(op.rel) || op.index != rel(op.rel).canonical)
          return no("rebuild of " + op.rel + " outside NEW in canonical order");
        rebuilt[op.rel]++;
        break;
      case Op::ComputeDelta: {
        maintenance = true;
        Relation& r = rel(op.rel);
        if (r.arity != 2 || op.index != r.canonical) return no("delta of " + op.rel + " not binary canonical");
        break;
      }
      case Op::Merge:
        maintenance = true;
        if (!computed.count(op.rel) || op.index != rel(op.rel).canonical)
          return no("merge into a second permutation of " + op.rel);
        merged[op.rel]++;
        break;
      case Op::Clear:
      case Op::CheckSize:
        maintenance = maintenance || op.kind == Op::CheckSize;
        break;
      default:
        return no("op kind not run by the device loop");
    }
  }
  for (auto& n : computed)
    if (rebuilt[n] != 1 || merged[n] != 1) return no("relation " + n + " not rebuilt and merged once");
  return true;
}

int Database::run_device_loop(const Step& st, uint64_t it0, uint64_t max_iters, uint64_t* done) {
  *done = 0;
  if (max_iters <= it0) return kLoopSkipped;
  const auto t0 = std::chrono::steady_clock::now();
  const std::vector<std::string> comp = computed_rels(st);
  std::vector<const Op*> execs;
  for (auto& op : st.ops)
    if (op.kind == Op::Execute) execs.push_back(&op);

  LoopCtx X;
  X.dir_n = dom_max_ + 2;
  // ---- capacities and buffers (an allocation refused by the run's memory
  //      limit leaves the step to the host path)
  try {
    for (auto& name : comp) {
      LoopRel lr;
      lr.r = &rel(name);
      Relation& r = *lr.r;
      Index& f = ensure_index(r, kFull, r.canonical);  // merges a Device2LevelIndex HEAD
      auto dit = r.v[kDelta].idx.find(r.canonical);
      const uint64_t dn = dit == r.v[kDelta].idx.end() ? 0 : dit->second.n;
      // room: twice the largest NEW (before dedup) and DELTA seen; FULL's
      // final size seen before plus an eighth, or the current FULL plus
      // four DELTA rooms (overflows redo an iteration on the host path and
      // re-enter with the sizes it measured)
      const uint64_t seen_new = std::max(new_max_[name], dn);
      const uint64_t seen_delta = std::max(delta_max_[name], dn);
      lr.cap_new = round_cap(std::max<uint64_t>(2 * seen_new, 1 << 16));
      lr.cap_delta = std::min(lr.cap_new, round_cap(std::max<uint64_t>(2 * seen_delta, 1 << 16)));
      lr.cap_full =
          round_cap(std::max<uint64_t>(full_max_[name] + full_max_[name] / 8, f.n + 4 * lr.cap_delta));
      if (opt_loop_cap_limit_) {
        // smaller capacities than the counts seen (tests of the overflow path)
        lr.cap_new = std::max<uint64_t>(std::min(lr.cap_new, opt_loop_cap_limit_), dn + 1);
        lr.cap_delta = std::min(lr.cap_new, std::max<uint64_t>(std::min(lr.cap_delta, opt_loop_cap_limit_), dn + 1));
        lr.cap_full = std::max<uint64_t>(std::min(lr.cap_full, 16 * opt_loop_cap_limit_), f.n + 1);
      }
      for (const Op* op : execs)
        for (auto& po : op->pipeline)
          if (po.kind == PipeOp::Insert && po.rel == name) lr.producers++;
      {
        // the buffers below; leave the step to the host path rather than
        // take most of the free memory (the host path needs far less)
        const uint64_t need = lr.cap_new * 8 + lr.cap_delta * (16 + 8 + 8) +
                              sort_dev_scratch_bytes(lr.cap_new, lr.cap_full, bits_) + lr.cap_full * 16;
        size_t free_b = 0, total_b = 0;
        SRDL_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const ArenaUse au = arena_use(L_.stream);
        if ((double)need > 0.7 * (double)(free_b + au.cached))
          throw Error{kErrCapacity, "device loop buffers (" + std::to_string(need >> 20) +
                                        " MB) would take most of the free device memory"};
      }
      lr.newk = DevBuf(lr.cap_new * 8, L_.stream);
      lr.sort_scr = DevBuf(sort_dev_scratch_bytes(lr.cap_new, lr.cap_full, bits_), L_.stream);
      lr.trie_scr = DevBuf(roots_scratch_bytes(lr.cap_delta) + 1024, L_.stream);
      for (int q = 0; q < 2; q++) {
        lr.full[q] = DevBuf(lr.cap_full * 8, L_.stream);
        lr.delta[q] = DevBuf(lr.cap_delta * 8, L_.stream);
        lr.lo[q] = DevBuf(lr.cap_delta * 4, L_.stream);
        lr.roots[q] = DevBuf(lr.cap_delta * 4, L_.stream);
        lr.dir[q] = DevBuf((size_t)X.dir_n * 4, L_.stream);
      }
      X.rels.push_back(std::move(lr));
    }
    for (const Op* op : execs) {
      std::vector<LoopLevel> lvls;
      std::vector<uint64_t>& seen = level_max_[op];
      uint64_t rows = 1;
      for (size_t li = 0; li < seen.size(); li++) {
        LoopLevel ll;
        ll.cap_rows = rows;
        ll.cap_total = round_cap(std::max<uint64_t>(2 * seen[li], 4096));
        if (opt_loop_cap_limit_) ll.cap_total = std::min(ll.cap_total, opt_loop_cap_limit_);
        ll.wscr = DevBuf(join_work_scratch_bytes(ll.cap_rows), L_.stream);
        ll.xscr = DevBuf(join_expand_scratch_bytes(L_, ll.cap_total), L_.stream);
        ll.count = DevBuf(8, L_.stream);
        rows = ll.cap_total;
        lvls.push_back(std::move(ll));
      }
      X.pipes.push_back(std::move(lvls));
    }
    X.cnt = DevBuf(X.rels.size() * sizeof(LoopCounts), L_.stream);
    X.ctl = DevBuf(sizeof(LoopCtl), L_.stream);
  } catch (const Error& e) {
    if (e.code != kErrCapacity && e.code != kErrCuda) throw;
    (void)cudaGetLastError();
    loop_stats_.skipped++;
    loop_stats_.last_error = e.msg;
    return kLoopSkipped;
  }

  // ---- initial state: buffer set 0 = the host's FULL and DELTA
  {
    std::vector<LoopCounts> init(X.rels.size());
    memset(init.data(), 0, init.size() * sizeof(LoopCounts));
    for (size_t i = 0; i < X.rels.size(); i++) {
      Relation& r = *X.rels[i].r;
      auto dit = r.v[kDelta].idx.find(r.canonical);
      init[i].n_full[0] = ensure_index(r, kFull, r.canonical).n;
      init[i].n_delta[0] = dit == r.v[kDelta].idx.end() ? 0 : dit->second.n;
    }
    SRDL_CUDA(cudaMemcpyAsync(X.cnt.as<void>(), init.data(), init.size() * sizeof(LoopCounts),
                              cudaMemcpyHostToDevice, L_.stream));
    SRDL_CUDA(cudaStreamSynchronize(L_.stream));  // the host array leaves scope
  }
  for (size_t i = 0; i < X.rels.size(); i++) {
    LoopRel& lr = X.rels[i];
    Relation& r = *lr.r;
    Index& f = ensure_index(r, kFull, r.canonical);
    auto dit = r.v[kDelta].idx.find(r.canonical);
    const uint64_t dn = dit == r.v[kDelta].idx.end() ? 0 : dit->second.n;
    LoopCounts* c = X.cnt_d() + i;
    if (f.n)
      SRDL_CUDA(cudaMemcpyAsync(lr.full[0].as<void>(), f.keys.as<void>(), f.n * 8, cudaMemcpyDeviceToDevice,
                                L_.stream));
    if (dn)
      SRDL_CUDA(cudaMemcpyAsync(lr.delta[0].as<void>(), dit->second.keys.as<void>(), dn * 8,
                                cudaMemcpyDeviceToDevice, L_.stream));
    Scratch ts{lr.trie_scr.as<char>(), lr.trie_scr.bytes(), 0};
    build_lo(L_, lr.delta[0].as<uint64_t>(), lr.cap_delta, lr.lo[0].as<uint32_t>(), &c->n_delta[0]);
    build_roots(L_, lr.delta[0].as<uint64_t>(), lr.cap_delta, lr.roots[0].as<uint32_t>(), &c->n_roots[0], ts,
                &c->n_delta[0]);
    build_dir(L_, lr.delta[0].as<uint64_t>(), lr.cap_delta, lr.dir[0].as<uint32_t>(), X.dir_n,
              &c->n_delta[0]);
  }
  {
    // (a fixpoint always converges; the cap bounds one graph launch should
    // an engine fault keep the delta from emptying -- the host path then
    // continues)
    LoopCtl init{};
    init.remaining = std::min<uint64_t>(max_iters - it0, kLoopMaxIters);
    SRDL_CUDA(cudaMemcpyAsync(X.ctl.as<void>(), &init, sizeof(init), cudaMemcpyHostToDevice, L_.stream));
    SRDL_CUDA(cudaStreamSynchronize(L_.stream));  // the host copy leaves scope
  }

  // DELTA views of buffer set p (the join kernels read counts on the device)
  auto delta_views = [&](int p) {
    LoopCounts* cnt = X.cnt_d();
    std::map<std::string, TrieView> dv;
    for (size_t i = 0; i < X.rels.size(); i++) {
      LoopRel& lr = X.rels[i];
      TrieView t;
      t.keys = lr.delta[p].as<uint64_t>();
      t.lo = lr.lo[p].as<uint32_t>();
      t.roots = lr.roots[p].as<uint32_t>();
      t.dir = lr.dir[p].as<uint32_t>();
      t.dir_n = X.dir_n;
      t.n = lr.cap_delta;
      t.n_roots_d = &cnt[i].n_roots[p];
      t.arity = 2;
      dv[lr.r->name] = t;
    }
    return dv;
  };

  // table columns: a level's output holds the slots the next level reads
  {
    const std::map<std::string, TrieView> dv0 = delta_views(0);
    for (size_t k = 0; k < execs.size(); k++) {
      std::vector<LoopLevel>& lvls = X.pipes[k];
      PipePlan pp = plan_pipeline(*execs[k], true, 1, &dv0);
      if (pp.levels.size() != lvls.size()) {
        loop_stats_.skipped++;
        loop_stats_.last_error = "a pipeline's levels were not all seen on the host path";
        return kLoopSkipped;
      }
      try {
        for (size_t li = 0; li + 1 < pp.levels.size(); li++) {
          const int bound = pp.levels[li + 1].n_in_slots;
          for (int c = 0; c < bound && c < kMaxSlots; c++)
            lvls[li].cols[c] = DevBuf(lvls[li].cap_total * 4, L_.stream);
        }
      } catch (const Error& e) {
        if (e.code != kErrCapacity && e.code != kErrCuda) throw;
        (void)cudaGetLastError();
        loop_stats_.skipped++;
        loop_stats_.last_error = e.msg;
        return kLoopSkipped;
      }
    }
  }

  // ---- one iteration reading buffer set p, writing 1 - p, then the control kernel
  auto body = [&](int p, cudaGraphConditionalHandle hw, cudaGraphConditionalHandle hi, int set_if) {
    LoopCounts* cnt = X.cnt_d();
    unsigned int* ovf = &X.ctl_d()->overflow;
    for (size_t i = 0; i < X.rels.size(); i++) SRDL_CUDA(cudaMemsetAsync(&cnt[i].n_new, 0, 8, L_.stream));
    const std::map<std::string, TrieView> dv = delta_views(p);
    for (size_t k = 0; k < execs.size(); k++) {
      const Op& op = *execs[k];
      PipePlan pp = plan_pipeline(op, true, 1, &dv);
      std::vector<LoopLevel>& lvls = X.pipes[k];
      SRDL_REQUIRE(pp.levels.size() == lvls.size(), kErrState, "device loop: level count changed");
      const int ri = X.rel_index(pp.target->name);
      SRDL_REQUIRE(ri >= 0, kErrState, "device loop: insert into an unknown relation");
      LoopRel& lr = X.rels[ri];
      Table cur;
      cur.n = 1;
      for (size_t li = 0; li < pp.levels.size(); li++) {
        LevelSpec& lv = pp.levels[li];
        LoopLevel& ll = lvls[li];
        const bool last = li + 1 == pp.levels.size();
        Scratch s{ll.wscr.as<char>(), ll.wscr.bytes(), 0};
        JoinWork w = join_count(L_, lv, cur, s);
        Scratch xs{ll.xscr.as<char>(), ll.xscr.bytes(), 0};
        JoinDev jd;
        jd.d_total = w.offs + cur.n;
        jd.d_overflow = ovf;
        if (last) {
          lv.emit = kEmitKeys;
          lv.key_arity = 2;
          for (int c = 0; c < 2; c++) lv.key_slot[c] = pp.key_slot[c];
          jd.out_cap = lr.cap_new;
          jd.exact_ok = lr.producers == 1;
          join_expand(L_, lv, cur, w, ll.cap_total, nullptr, lr.newk.as<uint64_t>(), &cnt[ri].n_new, xs,
                      &jd);
        } else {
          lv.emit = kEmitTable;
          Table next;
          const int bound = pp.levels[li + 1].n_in_slots;
          for (int c = 0; c < bound && c < kMaxSlots; c++) {
            SRDL_REQUIRE(ll.cols[c].bytes() > 0, kErrState, "device loop: table column missing");
            next.col[c] = ll.cols[c].as<uint32_t>();
          }
          SRDL_CUDA(cudaMemsetAsync(ll.count.as<void>(), 0, 8, L_.stream));
          jd.out_cap = ll.cap_total;
          join_expand(L_, lv, cur, w, ll.cap_total, &next, nullptr, ll.count.as<uint64_t>(), xs, &jd);
          next.n = ll.cap_total;
          next.d_n = ll.count.as<uint64_t>();
          cur = next;
        }
      }
    }
    for (size_t i = 0; i < X.rels.size(); i++) {
      LoopRel& lr = X.rels[i];
      LoopCounts* c = cnt + i;
      Scratch ss{lr.sort_scr.as<char>(), lr.sort_scr.bytes(), 0};
      // DELTA = unique(NEW) - FULL, FULL' = FULL U DELTA, DELTA's trie view
      sort_dedup_dev(L_, lr.newk.as<uint64_t>(), lr.cap_new, &c->n_new, bits_, lr.full[p].as<uint64_t>(),
                     lr.cap_full, &c->n_full[p], lr.delta[1 - p].as<uint64_t>(), lr.cap_delta, &c->n_delta[1 - p],
                     ovf, ss);
      merge_disjoint_dev(L_, lr.full[p].as<uint64_t>(), lr.cap_full, &c->n_full[p],
                         lr.delta[1 - p].as<uint64_t>(), lr.cap_delta, &c->n_delta[1 - p],
                         lr.full[1 - p].as<uint64_t>(), lr.cap_full, &c->n_full[1 - p], ovf);
      Scratch ts{lr.trie_scr.as<char>(), lr.trie_scr.bytes(), 0};
      build_lo(L_, lr.delta[1 - p].as<uint64_t>(), lr.cap_delta, lr.lo[1 - p].as<uint32_t>(), &c->n_delta[1 - p]);
      build_roots(L_, lr.delta[1 - p].as<uint64_t>(), lr.cap_delta, lr.roots[1 - p].as<uint32_t>(),
                  &c->n_roots[1 - p], ts, &c->n_delta[1 - p]);
      build_dir(L_, lr.delta[1 - p].as<uint64_t>(), lr.cap_delta, lr.dir[1 - p].as<uint32_t>(), X.dir_n,
                &c->n_delta[1 - p]);
      // batched runs: the instances with a delta row in this iteration
      // (its number is it0 + 1 + the bodies started before it)
      if (loop_marks_)
        instance_mark(L_, lr.delta[1 - p].as<uint64_t>(), lr.cap_delta, &c->n_delta[1 - p],
                      inst_bounds_d_.as<uint32_t>(), (uint32_t)(inst_bounds_.size() - 1), (uint32_t)(it0 + 1),
                      &X.ctl_d()->bodies, loop_marks_);
    }
    const int ks = 2 * bits_ <= 32 ? 4 : 8;
    const int maxw = L_.radix_bits >= 1 && L_.radix_bits <= 8 ? L_.radix_bits : 8;
    const int passes = (2 * bits_ + maxw - 1) / maxw;
    loop_ctrl_kernel<<<1, 32, 0, L_.stream>>>(X.ctl_d(), cnt, (int)X.rels.size(), p, ks, passes, hw, hi,
                                              set_if);
    SRDL_CUDA(cudaGetLastError());
    count_launches(1);
  };

  // ---- capture: WHILE (go) { body(0); IF (go) { body(1) } }, on the loop's
  // own stream, after everything queued on the database's stream
  // (kernel attributes are set before the capture, not inside it)
  warm_device_loop_kernels(bits_);
  if (!loop_stream_) {
    SRDL_CUDA(cudaStreamCreateWithFlags(&loop_stream_, cudaStreamNonBlocking));
    SRDL_CUDA(cudaEventCreateWithFlags(&loop_ev_[0], cudaEventDisableTiming));
    SRDL_CUDA(cudaEventCreateWithFlags(&loop_ev_[1], cudaEventDisableTiming));
  }
  SRDL_CUDA(cudaEventRecord(loop_ev_[0], L_.stream));
  SRDL_CUDA(cudaStreamWaitEvent(loop_stream_, loop_ev_[0], 0));
  const cudaStream_t db_stream = L_.stream;
  struct StreamSwap {
    Launch& L;
    cudaStream_t keep;
    ~StreamSwap() { L.stream = keep; }
  } swap{L_, db_stream};
  L_.stream = loop_stream_;
  const bool prof = profile_;
  profile_ = false;
  const uint64_t l0 = launches_total();
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  struct GraphGuard {
    cudaGraph_t& g;
    cudaGraphExec_t& ge;
    ~GraphGuard() {
      if (ge) cudaGraphExecDestroy(ge);
      if (g) cudaGraphDestroy(g);
    }
  } guard{g, ge};
  uint64_t per_body = 0;
  try {
    SRDL_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle hw, hi;
    SRDL_CUDA(cudaGraphConditionalHandleCreate(&hw, g, 1, cudaGraphCondAssignDefault));
    SRDL_CUDA(cudaGraphConditionalHandleCreate(&hi, g, 0, cudaGraphCondAssignDefault));
    cudaGraphNodeParams wp = {};
    wp.type = cudaGraphNodeTypeConditional;
    wp.conditional.handle = hw;
    wp.conditional.type = cudaGraphCondTypeWhile;
    wp.conditional.size = 1;
    cudaGraphNode_t wnode;
    SRDL_CUDA(cudaGraphAddNode(&wnode, g, nullptr, 0, &wp));
    cudaGraph_t wbody = wp.conditional.phGraph_out[0];
    cudaGraph_t tmp;
    SRDL_CUDA(cudaStreamBeginCaptureToGraph(L_.stream, wbody, nullptr, nullptr, 0,
                                            cudaStreamCaptureModeThreadLocal));
    try {
      body(0, hw, hi, 1);
    } catch (...) {
      cudaStreamEndCapture(L_.stream, &tmp);
      throw;
    }
    per_body = launches_total() - l0;
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    SRDL_CUDA(cudaStreamGetCaptureInfo(L_.stream, &cs, nullptr, nullptr, &deps, &ndeps));
    std::vector<cudaGraphNode_t> tail(deps, deps + ndeps);
    SRDL_CUDA(cudaStreamEndCapture(L_.stream, &tmp));
    cudaGraphNodeParams ip = {};
    ip.type = cudaGraphNodeTypeConditional;
    ip.conditional.handle = hi;
    ip.conditional.type = cudaGraphCondTypeIf;
    ip.conditional.size = 1;
    cudaGraphNode_t inode;
    SRDL_CUDA(cudaGraphAddNode(&inode, wbody, tail.data(), tail.size(), &ip));
    cudaGraph_t ibody = ip.conditional.phGraph_out[0];
    SRDL_CUDA(cudaStreamBeginCaptureToGraph(L_.stream, ibody, nullptr, nullptr, 0,
                                            cudaStreamCaptureModeThreadLocal));
    try {
      body(1, hw, hi, 0);
    } catch (...) {
      cudaStreamEndCapture(L_.stream, &tmp);
      throw;
    }
    SRDL_CUDA(cudaStreamEndCapture(L_.stream, &tmp));
    SRDL_CUDA(cudaGraphInstantiate(&ge, g, 0));
  } catch (const Error& e) {
    // a capture the runtime refuses leaves the step to the host path
    profile_ = prof;
    count_launches(-(int)(launches_total() - l0));
    (void)cudaGetLastError();
    SRDL_CUDA(cudaStreamSynchronize(loop_stream_));
    loop_stats_.skipped++;
    loop_stats_.last_error = e.msg;
    return kLoopSkipped;
  }
  profile_ = prof;
  count_launches(-(int)(launches_total() - l0));  // counted again per executed iteration below
  const auto t1 = std::chrono::steady_clock::now();

  // ---- run (events on the database's stream time the launch)
  L_.stream = db_stream;
  size_t pid = prof_begin("device_loop");
  SRDL_CUDA(cudaGraphLaunch(ge, loop_stream_));
  LoopCtl ctl{};
  std::vector<LoopCounts> cnt(X.rels.size());
  SRDL_CUDA(cudaMemcpyAsync(&ctl, X.ctl.as<void>(), sizeof(ctl), cudaMemcpyDeviceToHost, loop_stream_));
  SRDL_CUDA(cudaMemcpyAsync(cnt.data(), X.cnt.as<void>(), cnt.size() * sizeof(LoopCounts),
                            cudaMemcpyDeviceToHost, loop_stream_));
  SRDL_CUDA(cudaEventRecord(loop_ev_[1], loop_stream_));
  SRDL_CUDA(cudaStreamWaitEvent(db_stream, loop_ev_[1], 0));
  prof_end(pid, 0, (double)X.rels.size());
  SRDL_CUDA(cudaStreamSynchronize(loop_stream_));
  if (pid != (size_t)-1) kev_[pid].bytes = ctl.alg_bytes;
  count_launches((int)(per_body * ctl.bodies));
  const auto t2 = std::chrono::steady_clock::now();

  // ---- the latest complete iteration becomes the host state
  const int q = (int)ctl.parity;
  for (size_t i = 0; i < X.rels.size(); i++) {
    LoopRel& lr = X.rels[i];
    Relation& r = *lr.r;
    const LoopCounts& c = cnt[i];
    r.v[kFull].clear();
    r.head = Index{};
    Index& f = r.v[kFull].idx[r.canonical];
    f.keys = std::move(lr.full[q]);
    f.n = c.n_full[q];
    r.v[kDelta].clear();
    r.v[kNew].clear();
    Index& d = r.v[kDelta].idx[r.canonical];
    d.keys = std::move(lr.delta[q]);
    d.n = c.n_delta[q];
    d.lo = std::move(lr.lo[q]);
    d.roots = std::move(lr.roots[q]);
    d.dir = std::move(lr.dir[q]);
    d.dir_n = X.dir_n;
    d.nroots_d = DevBuf(8, L_.stream);
    SRDL_CUDA(cudaMemcpyAsync(d.nroots_d.as<void>(), &X.cnt_d()[i].n_roots[q], 8, cudaMemcpyDeviceToDevice,
                              L_.stream));
    d.trie = true;
    r.delta_epoch += ctl.done;
    r.base_epoch = r.delta_epoch - 1;
    r.full_epoch = r.delta_epoch;
    f.epoch = r.delta_epoch;
    derived_ += c.derived;
    full_max_[r.name] = std::max<uint64_t>(full_max_[r.name], c.n_full[q]);
    delta_max_[r.name] = std::max<uint64_t>(delta_max_[r.name], c.n_delta[q]);
  }
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  *done = ctl.done;
  loop_stats_.entries++;
  loop_stats_.iterations += ctl.done;
  loop_stats_.capture_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
  loop_stats_.run_ms += std::chrono::duration<double, std::milli>(t2 - t1).count();
  if (ctl.overflow) {
    loop_stats_.overflows++;
    // the host path redoes the failed iteration and measures the counts
    // that were too large; the next entry sizes from at least twice these
    for (auto& lr : X.rels) {
      new_max_[lr.r->name] = std::max(new_max_[lr.r->name], lr.cap_new);
      delta_max_[lr.r->name] = std::max(delta_max_[lr.r->name], lr.cap_delta);
      full_max_[lr.r->name] = std::max(full_max_[lr.r->name], lr.cap_full);
    }
    for (size_t k = 0; k < execs.size(); k++) {
      std::vector<uint64_t>& seen = level_max_[execs[k]];
      for (size_t li = 0; li < seen.size() && li < X.pipes[k].size(); li++)
        seen[li] = std::max(seen[li], X.pipes[k][li].cap_total);
    }
    return kLoopOverflow;
  }
  return kLoopDone;
}

}  // namespace srdl
