// exec.cu -- Database: pipeline execution, maintenance ops, fixpoint loop.
//
// Op semantics follow the reference's MIR helpers:
//   rebuild_index      RT/gpu/runtime/gpu_mir_helpers.h:204-232
//   compute_delta_index gpu_mir_helpers.h:88-122   (DELTA = NEW - FULL)
//   merge_index        gpu_mir_helpers.h:136-159   (FULL |= DELTA)
//   clear_relation     gpu_mir_helpers.h:308
//   iteration-0 DELTA reads go to FULL           gpu_mir_helpers.h:419-426
//   loop: stop when the summed delta is empty, at most max_iters joins
//         (src/srdatalog/codegen/jit/orchestrator_jit.py:600-747).
// When a rebuild of NEW is followed only by check_size / clear(DELTA) before
// the compute_delta_index of the same relation, the sort's dedup pass also
// drops the keys already in FULL, so NEW is never written out separately.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <sstream>

#include "runtime.h"

namespace srdl {

namespace {

struct FilterTerm {
  std::string a, b;
  int op;
};

bool is_uint(const std::string& s) {
  if (s.empty()) return false;
  for (char c : s)
    if (c < '0' || c > '9') return false;
  return true;
}

std::string trim(const std::string& s) {
  size_t b = s.find_first_not_of(" \t\n()"), e = s.find_last_not_of(" \t\n()");
  return b == std::string::npos ? std::string() : s.substr(b, e - b + 1);
}

// Restricted filter grammar: "return a OP b && c OP d ...;" with bound
// variables or unsigned constants.  The reference pastes the C++ body into
// the generated kernel; anything outside this grammar is rejected.
std::vector<FilterTerm> parse_filter(const std::string& code) {
  std::string s = trim(code);
  SRDL_REQUIRE(s.rfind("return", 0) == 0 && !s.empty() && s.back() == ';', kErrUnsupported,
               "filter '" + code + "': expected 'return <expr>;'");
  s = s.substr(6, s.size() - 7);
  std::vector<FilterTerm> out;
  size_t p = 0;
  while (true) {
    size_t q = s.find("&&", p);
    std::string part = trim(s.substr(p, q == std::string::npos ? std::string::npos : q - p));
    static const char* ops[] = {"!=", "==", "<=", ">=", "<", ">"};
    static const int codes[] = {kNe, kEq, kLe, kGe, kLt, kGt};
    bool found = false;
    for (int k = 0; k < 6 && !found; k++) {
      size_t at = part.find(ops[k]);
      if (at == std::string::npos) continue;
      out.push_back({trim(part.substr(0, at)), trim(part.substr(at + strlen(ops[k]))), codes[k]});
      found = true;
    }
    SRDL_REQUIRE(found, kErrUnsupported, "filter '" + code + "': unsupported term '" + part + "'");
    if (q == std::string::npos) break;
    p = q + 2;
  }
  return out;
}

// A message as a JSON string body: quotes and backslashes escaped, control
// characters dropped.
std::string json_escape(const std::string& m) {
  std::string o;
  for (char c : m) {
    if (c == '"' || c == '\\') o += '\\';
    if ((unsigned char)c >= 0x20) o += c;
  }
  return o;
}

// The device loop runs unless SRDL_DEVICE_LOOP=0 (or the device_loop option)
// turns it off.
bool device_loop_default() {
  static const bool on = [] {
    const char* e = std::getenv("SRDL_DEVICE_LOOP");
    return !(e && e[0] == '0');
  }();
  return on;
}

}  // namespace

constexpr uint64_t kSegsPerShard = 256;

PipePlan Database::plan_pipeline(const Op& op, bool recursive, uint64_t iteration,
                                 const std::map<std::string, TrieView>* dviews) {
  std::map<std::string, int> slot;
  int nslots = 0;
  auto bind = [&](const std::string& v) {
    SRDL_REQUIRE(!slot.count(v), kErrUnsupported, "rule " + op.rule + ": variable " + v + " bound twice");
    SRDL_REQUIRE(nslots < kMaxSlots, kErrUnsupported, "rule " + op.rule + ": too many variables");
    slot[v] = nslots++;
    return slot[v];
  };
  auto slot_of = [&](const std::string& v) {
    auto it = slot.find(v);
    SRDL_REQUIRE(it != slot.end(), kErrPlan, "rule " + op.rule + ": unbound variable " + v);
    return it->second;
  };
  // Ternary relations are stored in their canonical column order only; a
  // read in another order goes through that order's pair / row views.
  auto ternary = [&](const SourceDesc& d) -> Split3& {
    Relation& r = rel(d.rel);
    Ver v = (d.ver == kDelta && recursive && iteration == 0) ? kFull : d.ver;
    SRDL_REQUIRE(r.pack_half > 0, kErrUnsupported,
                 "relation " + r.name + ": ternary reads need arity x value bits <= 64");
    return ensure_split(r, ensure_index(r, v, r.canonical), d.index);
  };
  auto rows_src = [&](const SourceDesc& d) {
    SRDL_REQUIRE(d.prefix.size() <= 1, kErrUnsupported,
                 "rule " + op.rule + ": ternary rows read with " + std::to_string(d.prefix.size()) +
                     " bound columns");
    Split3& sp = ternary(d);
    SrcSpec s;
    s.mode = kSrcRows;
    s.t = view2(sp.rows);
    s.pair = view2(sp.pair);
    s.prefix_slot = d.prefix.empty() ? -1 : slot_of(d.prefix[0]);
    return s;
  };
  auto make_src = [&](const SourceDesc& d, bool probed) {
    Relation& r = rel(d.rel);
    Ver v = (d.ver == kDelta && recursive && iteration == 0) ? kFull : d.ver;
    if (r.arity == 3) {
      SRDL_REQUIRE(d.prefix.size() <= 2, kErrPlan, "rule " + op.rule + ": prefix too long on " + r.name);
      Split3& sp = ternary(d);
      SrcSpec s;
      if (d.prefix.size() <= 1) {
        // c0 or c1 as the next value: the pair index read as a binary relation
        if (probed && !d.prefix.empty() && v == kFull) {
          ensure_hash(sp.pair);
          ensure_bitmaps(sp.pair);
        }
        s.t = view2(sp.pair);
        s.prefix_slot = d.prefix.empty() ? -1 : slot_of(d.prefix[0]);
      } else {
        s.mode = kSrcPair;
        s.t = view2(sp.rows);
        s.pair = view2(sp.pair);
        s.prefix_slot = slot_of(d.prefix[0]);
        s.prefix_slot2 = slot_of(d.prefix[1]);
      }
      return s;
    }
    SRDL_REQUIRE(r.arity <= 2, kErrUnsupported, "join over relation " + r.name + " of arity > 2");
    SRDL_REQUIRE(d.prefix.size() < (size_t)std::max(r.arity, 2), kErrUnsupported,
                 "rule " + op.rule + ": prefix too long on " + r.name);
    if (v == kDelta && dviews) {
      // the device loop's DELTA of this relation (its canonical order)
      auto dv = dviews->find(d.rel);
      if (dv != dviews->end()) {
        SrcSpec s;
        s.t = dv->second;
        s.prefix_slot = d.prefix.empty() ? -1 : slot_of(d.prefix[0]);
        return s;
      }
    }
    Index& ix = ensure_index(r, v, d.index);
    // Hash long child lists of probed FULL indexes; a delta is rebuilt every
    // iteration and is usually the short (driving) side anyway.
    if (probed && !d.prefix.empty() && v == kFull) {
      ensure_trie(r, ix);
      ensure_hash(ix);
      ensure_bitmaps(ix);
    }
    SrcSpec s;
    s.t = view(r, ix);
    s.prefix_slot = d.prefix.empty() ? -1 : slot_of(d.prefix[0]);
    return s;
  };

  std::vector<LevelSpec> levels;
  const PipeOp* insert = nullptr;
  for (const PipeOp& po : op.pipeline) {
    if (po.kind == PipeOp::Negation) {
      // anti-join: a filter term that probes the negated relation's index
      SRDL_REQUIRE(!levels.empty(), kErrPlan, "rule " + op.rule + ": negation before any join");
      LevelSpec& lv = levels.back();
      SRDL_REQUIRE(lv.nfilt < kMaxFilt, kErrUnsupported, "too many filter terms");
      const SourceDesc& d = po.sources[0];
      Relation& nr = rel(d.rel);
      SRDL_REQUIRE(nr.arity <= 3, kErrUnsupported, "negation over relation " + nr.name + " of arity > 3");
      // the probed prefix: the constants (their columns lead the index), then the variables
      struct Val {
        int slot;
        uint32_t c;
      };
      std::vector<Val> vals;
      for (uint32_t c : po.const_prefix) vals.push_back({-1, c});
      for (auto& v : d.prefix) vals.push_back({slot_of(v), 0});
      SRDL_REQUIRE(!vals.empty() && vals.size() <= (size_t)std::min(nr.arity, 2), kErrUnsupported,
                   "negation on " + nr.name + ": one or two bound values (constants or variables)");
      FiltSpec f;
      f.negation = true;
      f.neg_n = (int)vals.size();
      f.a_slot = vals[0].slot;
      f.a_const = vals[0].c;
      if (vals.size() > 1) {
        f.b_slot = vals[1].slot;
        f.b_const = vals[1].c;
      }
      if (nr.arity == 3) {
        // the pair view (c0, c1) of the relation in the negation's column order
        f.neg = view2(ternary(d).pair);
      } else {
        f.neg = view(nr, ensure_index(nr, d.ver, d.index));
      }
      lv.filt[lv.nfilt++] = f;
      continue;
    }
    if (po.kind == PipeOp::Filter) {
      SRDL_REQUIRE(!levels.empty(), kErrPlan, "rule " + op.rule + ": filter before any join");
      LevelSpec& lv = levels.back();
      for (auto& t : parse_filter(po.code)) {
        SRDL_REQUIRE(lv.nfilt < kMaxFilt, kErrUnsupported, "too many filter terms");
        FiltSpec f;
        f.op = t.op;
        if (is_uint(t.a)) f.a_const = (uint32_t)std::stoul(t.a); else f.a_slot = slot_of(t.a);
        if (is_uint(t.b)) f.b_const = (uint32_t)std::stoul(t.b); else f.b_slot = slot_of(t.b);
        lv.filt[lv.nfilt++] = f;
      }
      continue;
    }
    if (po.kind == PipeOp::Insert) {
      insert = &po;
      continue;
    }
    LevelSpec lv;
    lv.n_in_slots = nslots;
    if (po.kind == PipeOp::Scan) {
      const SourceDesc& d = po.sources[0];
      lv.kind = kScan;
      lv.nsrc = 1;
      if (rel(d.rel).arity == 3) {
        lv.src[0] = rows_src(d);
        lv.wide = 1;
      } else {
        lv.src[0] = make_src(d, false);
      }
      SRDL_REQUIRE(po.vars.size() == d.index.size(), kErrPlan, "scan arity mismatch");
      for (size_t j = d.prefix.size(); j < po.vars.size(); j++) lv.scan_slot[j] = bind(po.vars[j]);
    } else if (po.kind == PipeOp::ColumnJoin) {
      lv.kind = kColumnJoin;
      SRDL_REQUIRE(po.sources.size() <= (size_t)kMaxSrc && !po.sources.empty(), kErrUnsupported,
                   "column join with too many sources");
      // every list but the per-row shortest is probed: hash the long ones
      for (auto& d : po.sources) {
        lv.src[lv.nsrc] = make_src(d, po.sources.size() > 1);
        if (lv.src[lv.nsrc].mode != kSrcPlain) lv.wide = 1;
        lv.nsrc++;
      }
      lv.cj_slot = bind(po.var);
    } else {
      lv.kind = kCartesian;
      SRDL_REQUIRE(po.sources.size() <= (size_t)kMaxSrc, kErrUnsupported, "cartesian too wide");
      for (size_t i = 0; i < po.sources.size(); i++) {
        const auto& vs = i < po.var_from_source.size() ? po.var_from_source[i]
                                                        : std::vector<std::string>{};
        const SourceDesc& d = po.sources[i];
        if (vs.size() == 2 && rel(d.rel).arity == 3) {
          // a ternary source under one bound column binds the other two
          SRDL_REQUIRE(d.prefix.size() == 1, kErrUnsupported,
                       "rule " + op.rule + ": ternary source binding two variables needs one bound column");
          lv.src[lv.nsrc] = rows_src(d);
          lv.src[lv.nsrc].out_slot = bind(vs[0]);
          lv.src[lv.nsrc].out_slot2 = bind(vs[1]);
        } else {
          SRDL_REQUIRE(vs.size() <= 1, kErrUnsupported, "cartesian source binding several variables");
          lv.src[lv.nsrc] = make_src(d, false);
          lv.src[lv.nsrc].out_slot = vs.empty() ? -1 : bind(vs[0]);
        }
        if (lv.src[lv.nsrc].mode != kSrcPlain) lv.wide = 1;
        lv.nsrc++;
      }
    }
    // the expand kernels hold the values a level binds in kMaxSrc + 1 registers
    SRDL_REQUIRE(nslots - lv.n_in_slots <= kMaxSrc + 1, kErrUnsupported,
                 "rule " + op.rule + ": a join level binds more than " + std::to_string(kMaxSrc + 1) +
                     " variables");
    levels.push_back(lv);
  }
  SRDL_REQUIRE(insert && !levels.empty(), kErrPlan, "rule " + op.rule + ": no insert_into");
  const bool sharded = shard_world_ > 1 && op.shard != Op::NoShard;
  // Work sharding splits the last-but-one level of rules with three or more
  // levels (its items -- e.g. the triangle's (a, b) edges -- carry bounded
  // work each, so interleaved segments balance; the first level's root keys
  // can carry a hub's whole subtree) and otherwise the last level.
  const size_t work_split = levels.size() >= 3 ? levels.size() - 2 : levels.size() - 1;
  if (sharded && op.shard == Op::Key) {
    // keep the bindings whose key value this shard owns, at the level binding it
    const int ks = slot_of(op.shard_var);
    for (size_t li = 0; li < levels.size(); li++) {
      const int bound_after = li + 1 < levels.size() ? levels[li + 1].n_in_slots : nslots;
      if (ks < levels[li].n_in_slots || ks >= bound_after) continue;
      LevelSpec& lv = levels[li];
      SRDL_REQUIRE(lv.nfilt < kMaxFilt, kErrUnsupported, "too many filter terms");
      FiltSpec f;
      f.a_slot = ks;
      f.b_const = (uint32_t)shard_rank_;
      f.shard_world = (uint32_t)shard_world_;
      lv.filt[lv.nfilt++] = f;
      break;
    }
  }

  Relation* target = &rel(insert->rel);
  if (!op.count && target->arity > 2) {
    SRDL_REQUIRE(target->arity <= 4 && target->pack_half > 0, kErrUnsupported,
                 "rule " + op.rule + ": materialising " + target->name + " needs arity <= 4 and " +
                     "arity x value bits <= 64");
    SRDL_REQUIRE(insert->index == target->canonical, kErrUnsupported,
                 "rule " + op.rule + ": " + target->name + " is written in its canonical order only");
  }

  PipePlan pp;
  pp.levels = std::move(levels);
  pp.insert = insert;
  pp.target = target;
  pp.nslots = nslots;
  pp.sharded = sharded;
  pp.work_split = work_split;
  if (!op.count)
    for (int c = 0; c < target->arity && c < 4; c++)
      pp.key_slot[c] = slot_of(insert->vars[insert->index[c]]);
  return pp;
}

void Database::exec_pipeline(const Op& op, bool recursive, uint64_t iteration) {
  PipePlan pp = plan_pipeline(op, recursive, iteration, nullptr);
  std::vector<LevelSpec>& levels = pp.levels;
  Relation* target = pp.target;
  const int nslots = pp.nslots;
  const bool sharded = pp.sharded;
  const size_t work_split = pp.work_split;
  std::vector<uint64_t>& seen = level_max_[&op];
  seen.resize(levels.size(), 0);
  // Walk the levels over a table of partial bindings.
  Table cur;
  cur.n = 1;
  std::vector<DevBuf> cur_cols;
  DevBuf cur_count;
  for (size_t li = 0; li < levels.size(); li++) {
    LevelSpec& lv = levels[li];
    const bool last = li + 1 == levels.size();
    DevBuf wscr(join_work_scratch_bytes(cur.n), L_.stream);
    Scratch s{wscr.as<char>(), wscr.bytes(), 0};
    size_t pid = prof_begin("join_count");
    // the last level of a count-only rule: rows probing a long bitmapped
    // list of the table's first column go to the pivot kernel (join.cu)
    lv.pivot_src = -1;
    if (last && op.count && opt_pivot_min_ > 0 && !(sharded && op.shard == Op::Work) &&
        !group_bounds_.count(op.rule) && lv.kind == kColumnJoin && lv.nsrc == 2 && lv.nfilt == 0 &&
        !lv.wide && cur.n > 0) {
      for (int ps = 0; ps < 2; ps++) {
        const SrcSpec& P = lv.src[ps];
        const SrcSpec& D = lv.src[1 - ps];
        if (P.prefix_slot == 0 && D.prefix_slot != 0 && P.mode == kSrcPlain && D.mode == kSrcPlain &&
            P.t.bdir && P.t.bpool && P.t.bwords && P.t.bslots && P.t.dir_n &&
            join_pivot_smem_bytes(P.t.bwords) <= kPivotSmemMax) {
          lv.pivot_src = ps;
          lv.pivot_min = (uint32_t)std::min<int64_t>(opt_pivot_min_, 0xffffffffll);
          lv.pivot_slots = P.t.bslots;
          break;
        }
      }
    }
    JoinWork w = join_count(L_, lv, cur, s);
    prof_end(pid, 8.0 * cur.n * (lv.n_in_slots + 3), (double)cur.n);
    SRDL_CUDA(cudaMemcpyAsync(h_small_ + 3, w.offs + cur.n, 8, cudaMemcpyDeviceToHost, L_.stream));
    if (w.poffs)
      SRDL_CUDA(cudaMemcpyAsync(h_small_ + 6, w.poffs + cur.n, 8, cudaMemcpyDeviceToHost, L_.stream));
    SRDL_CUDA(cudaMemsetAsync(d_small_.as<uint64_t>() + 2, 0, 8, L_.stream));
    SRDL_CUDA(cudaStreamSynchronize(L_.stream));
    uint64_t total = h_small_[3];
    const uint64_t pivot_total = w.poffs ? h_small_[6] : 0;  // the pivot kernel's candidates
    seen[li] = std::max(seen[li], total);
    if (sharded && op.shard == Op::Work && li == work_split) {
      // Deal this level's work items out in segments, kSegsPerShard per
      // shard, interleaved so every shard gets a share of each key range
      // (skewed keys cluster); later levels see only this shard's rows.
      const uint64_t per = total / ((uint64_t)shard_world_ * kSegsPerShard);
      lv.seg = std::max<uint64_t>(32, (per + 31) & ~uint64_t(31));
      lv.seg_world = (uint32_t)shard_world_;
      lv.seg_rank = (uint32_t)shard_rank_;
      total = seg_owned(total, lv.seg, shard_world_, shard_rank_);
    }
    // the expand pass's own scratch, sized for this level's candidates
    DevBuf xscr(join_expand_scratch_bytes(L_, total) + (w.poffs ? join_pivot_scratch_bytes(lv.pivot_slots) : 0),
                L_.stream);
    Scratch xs{xscr.as<char>(), xscr.bytes(), 0};
    if (last) {
      if (op.count) {
        lv.emit = kEmitCount;
        DevBuf gb, gc;
        auto grp = group_bounds_.find(op.rule);
        if (grp != group_bounds_.end()) {
          SRDL_REQUIRE(lv.kind == kColumnJoin && lv.nsrc == 2 && lv.nfilt == 0, kErrUnsupported,
                       "grouped counts need a two-source column join without filters as the "
                       "last level of rule " + op.rule);
          const uint64_t ng = grp->second.size() - 1;
          gb = DevBuf(grp->second.size() * 4, L_.stream);
          gc = DevBuf(ng * 8, L_.stream);
          SRDL_CUDA(cudaMemcpyAsync(gb.as<void>(), grp->second.data(), grp->second.size() * 4,
                                    cudaMemcpyHostToDevice, L_.stream));
          SRDL_CUDA(cudaMemsetAsync(gc.as<void>(), 0, ng * 8, L_.stream));
          lv.grp_bounds = gb.as<uint32_t>();
          lv.n_groups = (uint32_t)ng;
          lv.grp_counts = gc.as<unsigned long long>();
        }
        pid = prof_begin("join_expand_count");
        join_expand(L_, lv, cur, w, total, nullptr, nullptr, d_small_.as<uint64_t>() + 2, xs);
        if (lv.grp_counts) {
          std::vector<uint64_t> h(lv.n_groups);
          SRDL_CUDA(cudaMemcpyAsync(h.data(), gc.as<void>(), h.size() * 8, cudaMemcpyDeviceToHost,
                                    L_.stream));
          SRDL_CUDA(cudaStreamSynchronize(L_.stream));
          auto& acc = group_counts_[op.rule];
          acc.resize(h.size(), 0);
          for (size_t g = 0; g < h.size(); g++) acc[g] += h[g];
        }
        // per candidate: its value (4 B) and one probed word of each other list (4 B)
        prof_end(pid, 4.0 * (total + pivot_total) * std::max(1, lv.nsrc), (double)(total + pivot_total));
        counts_[op.rule] += read_scalar(2);
      } else {
        lv.emit = kEmitKeys;
        lv.key_arity = target->arity;
        lv.pack_bits = target->pack_bits;
        lv.pack_half = target->pack_half;
        for (int c = 0; c < target->arity; c++) lv.key_slot[c] = pp.key_slot[c];
        Chunk ch;
        ch.order = pp.insert->index;
        if (levels.size() == 1 && lv.kind == kScan && lv.nsrc == 1 && !lv.wide && lv.src[0].prefix_slot < 0 &&
            lv.nfilt == 0 && !sharded && target->arity == 2 && lv.src[0].t.arity == 2 && lv.src[0].t.keys &&
            pp.key_slot[0] == lv.scan_slot[0] && pp.key_slot[1] == lv.scan_slot[1]) {
          // A rule that copies a whole binary index in its own column order
          // (Knows(x,y) <= KnowsInput(x,y)): the keys are that index's,
          // already sorted and unique -- copied, and never sorted again.
          const uint64_t nk = lv.src[0].t.n;
          ch.keys = DevBuf(std::max<uint64_t>(nk, 1) * 8, L_.stream);
          pid = prof_begin("join_expand_keys");
          if (nk)
            SRDL_CUDA(cudaMemcpyAsync(ch.keys.as<void>(), lv.src[0].t.keys, nk * 8, cudaMemcpyDeviceToDevice,
                                      L_.stream));
          prof_end(pid, 16.0 * nk, (double)nk);
          ch.n = nk;
          ch.sorted = true;
          derived_ += ch.n;
          target->v[kNew].chunks.push_back(std::move(ch));
          break;
        }
        ch.keys = DevBuf(std::max<uint64_t>(total, 1) * 8, L_.stream);
        pid = prof_begin("join_expand_keys");
        join_expand(L_, lv, cur, w, total, nullptr, ch.keys.as<uint64_t>(),
                    d_small_.as<uint64_t>() + 2, xs);
        // a filter-free two-source product emits exactly its candidates
        const bool exact = lv.kind == kCartesian && lv.nsrc == 2 && lv.src[0].out_slot >= 0 &&
                           lv.src[1].out_slot >= 0 && lv.nfilt == 0;
        ch.n = total == 0 ? 0 : exact ? total : read_scalar(2);
        prof_end(pid, 4.0 * total * std::max(1, lv.nsrc) + 8.0 * ch.n, (double)total);
        derived_ += ch.n;
        target->v[kNew].chunks.push_back(std::move(ch));
      }
    } else {
      lv.emit = kEmitTable;
      Table next;
      std::vector<DevBuf> cols;
      for (int c = 0; c < nslots && c < kMaxSlots; c++) {
        bool bound_here = c < levels[li + 1].n_in_slots;
        if (!bound_here) break;
        cols.emplace_back(std::max<uint64_t>(total, 1) * 4, L_.stream);
        next.col[c] = cols.back().as<uint32_t>();
      }
      // The table's row count stays on the device; the next level uses the
      // candidate total as capacity and reads the true count itself.
      DevBuf count(8, L_.stream);
      SRDL_CUDA(cudaMemsetAsync(count.as<void>(), 0, 8, L_.stream));
      pid = prof_begin("join_expand_table");
      join_expand(L_, lv, cur, w, total, &next, nullptr, count.as<uint64_t>(), xs);
      prof_end(pid, 4.0 * total * std::max(1, lv.nsrc), (double)total);
      next.n = total;
      next.d_n = count.as<uint64_t>();
      cur = next;
      cur_cols = std::move(cols);
      cur_count = std::move(count);
    }
    if (!last && cur.n == 0) {
      if (op.count) counts_[op.rule] += 0;
      break;
    }
  }
}

void Database::op_rebuild(const Step& st, size_t pos, const Op& op) {
  Relation& r = rel(op.rel);
  RelVersion& rv = r.v[op.ver];
  if (r.arity > 2 && (rv.chunks.empty() || r.pack_half == 0)) {
    // nothing materialised (count-only heads, or no output this time)
    rv.chunks.clear();
    rv.idx[op.index];
    return;
  }
  // packed tuples of arity 3-4 sort as binary keys of pack_half-bit halves
  const int key_bits = r.arity > 2 ? r.pack_half : 0;
  if (r.arity > 2)
    for (auto& c : rv.chunks)
      SRDL_REQUIRE(c.order == op.index, kErrUnsupported,
                   "relation " + r.name + " of arity > 2 rebuilt in another order");
  uint64_t total = 0;
  for (auto& c : rv.chunks) total += c.n;
  if (op.ver == kNew) new_max_[r.name] = std::max(new_max_[r.name], total);
  // Gather the chunks into one buffer packed in the target order.
  DevBuf gathered;
  const uint64_t* in = nullptr;
  if (rv.chunks.size() == 1 && rv.chunks[0].order == op.index) {
    in = rv.chunks[0].keys.as<uint64_t>();
  } else if (total) {
    gathered = DevBuf(total * 8, L_.stream);
    uint64_t off = 0;
    for (auto& c : rv.chunks) {
      if (!c.n) continue;
      if (c.order == op.index)
        SRDL_CUDA(cudaMemcpyAsync(gathered.as<uint64_t>() + off, c.keys.as<uint64_t>(), c.n * 8,
                                  cudaMemcpyDeviceToDevice, L_.stream));
      else
        swap_halves(L_, c.keys.as<uint64_t>(), c.n, gathered.as<uint64_t>() + off);
      off += c.n;
    }
    in = gathered.as<uint64_t>();
  }
  // Fuse with the delta computation when nothing reads NEW in between.
  bool fuse = false;
  if (op.ver == kNew) {
    for (size_t i = pos + 1; i < st.ops.size(); i++) {
      const Op& o = st.ops[i];
      if (o.kind == Op::ComputeDelta && o.rel == op.rel && o.index == op.index) {
        fuse = true;
        break;
      }
      if (o.kind == Op::CheckSize && o.rel == op.rel) continue;
      if (o.kind == Op::Clear && o.rel == op.rel && o.ver == kDelta) continue;
      break;
    }
  }
  if (rv.chunks.size() == 1 && rv.chunks[0].sorted && rv.chunks[0].order == op.index && r.arity <= 2 &&
      !(r.lsm && r.head.n)) {
    // a copied index: sorted and unique already
    Chunk& c = rv.chunks[0];
    Index fresh;
    fresh.n = c.n;
    if (fuse && r.v[kFull].has_index()) {
      const Index& full = r.lsm ? full_base(r, op.index) : ensure_index(r, kFull, op.index);
      fresh.keys = DevBuf(std::max<uint64_t>(c.n, 1) * 8, L_.stream);
      if (full.n && c.n) {
        DevBuf ds(diff_scratch_bytes(c.n) + 1024, L_.stream);
        Scratch s2{ds.as<char>(), ds.bytes(), 0};
        size_t pid = prof_begin("sort_dedup_diff");
        set_difference(L_, c.keys.as<uint64_t>(), c.n, full.keys.as<uint64_t>(), full.n,
                       fresh.keys.as<uint64_t>(), d_small_.as<uint64_t>(), s2);
        fresh.n = read_scalar(0);
        prof_end(pid, 8.0 * (c.n + full.n + fresh.n), (double)c.n);
      } else if (c.n) {
        SRDL_CUDA(cudaMemcpyAsync(fresh.keys.as<void>(), c.keys.as<void>(), c.n * 8, cudaMemcpyDeviceToDevice,
                                  L_.stream));
      }
    } else {
      fresh.keys = std::move(c.keys);
    }
    rv.chunks.clear();
    rv.idx.clear();
    if (fuse) {
      r.pending = std::move(fresh);
      r.pending_delta = true;
    } else {
      rv.idx[op.index] = std::move(fresh);
    }
    return;
  }
  if (fuse) {
    const Index* full = nullptr;
    if (r.v[kFull].has_index())
      full = r.lsm ? &full_base(r, op.index) : &ensure_index(r, kFull, op.index);
    const Index* head = r.lsm && op.index == r.canonical && r.head.n ? &r.head : nullptr;
    sort_into(r.pending, in ? in : nullptr, total, false, full, head, key_bits);
    r.pending_delta = true;
    rv.chunks.clear();
    rv.idx.clear();
  } else {
    Index fresh;
    sort_into(fresh, in, total, false, nullptr, nullptr, key_bits);
    rv.chunks.clear();
    rv.idx.clear();
    rv.idx[op.index] = std::move(fresh);
  }
}

void Database::op_compute_delta(const Op& op) {
  Relation& r = rel(op.rel);
  SRDL_REQUIRE(r.arity <= 2 || op.index == r.canonical, kErrUnsupported,
               "relation " + r.name + " of arity > 2: delta in a non-canonical order");
  r.v[kDelta].clear();
  r.delta_epoch++;
  if (r.pending_delta) {
    delta_max_[r.name] = std::max(delta_max_[r.name], r.pending.n);
    r.v[kDelta].idx[op.index] = std::move(r.pending);
    r.pending = Index{};
    r.pending_delta = false;
    return;
  }
  if (r.arity > 2) {
    auto it = r.v[kNew].idx.find(op.index);
    if (r.pack_half == 0 || it == r.v[kNew].idx.end() || it->second.n == 0) {
      r.v[kDelta].idx[op.index];
      return;
    }
  }
  Index& nw = ensure_index(r, kNew, op.index);
  Index& d = r.v[kDelta].idx[op.index];
  d.keys = DevBuf(std::max<uint64_t>(nw.n, 1) * 8, L_.stream);
  if (!r.v[kFull].has_index() || nw.n == 0) {
    if (nw.n)
      SRDL_CUDA(cudaMemcpyAsync(d.keys.as<uint64_t>(), nw.keys.as<uint64_t>(), nw.n * 8,
                                cudaMemcpyDeviceToDevice, L_.stream));
    d.n = nw.n;
    return;
  }
  Index& f = r.lsm ? full_base(r, op.index) : ensure_index(r, kFull, op.index);
  DevBuf scratch(diff_scratch_bytes(nw.n) + 1024, L_.stream);
  Scratch s{scratch.as<char>(), scratch.bytes(), 0};
  size_t pid = prof_begin("set_difference");
  set_difference(L_, nw.keys.as<uint64_t>(), nw.n, f.keys.as<uint64_t>(), f.n, d.keys.as<uint64_t>(),
                 d_small_.as<uint64_t>(), s);
  d.n = read_scalar(0);
  prof_end(pid, 8.0 * (nw.n + f.n + d.n), (double)nw.n);
  if (r.lsm) subtract_head(r, op.index, d);
  delta_max_[r.name] = std::max(delta_max_[r.name], d.n);
}

void Database::op_merge(const Op& op) {
  Relation& r = rel(op.rel);
  if (r.arity > 2 && op.index != r.canonical) return;  // stored in the canonical order only
  if (r.arity > 2) {
    auto it = r.v[kDelta].idx.find(op.index);
    if (r.pack_half == 0 || it == r.v[kDelta].idx.end() || it->second.n == 0) {
      r.v[kFull].idx[op.index];
      return;
    }
  }
  RelVersion& dv = r.v[kDelta];
  Index* d = nullptr;
  auto it = dv.idx.find(op.index);
  if (it != dv.idx.end()) d = &it->second;
  else if (dv.has_index()) d = &ensure_index(r, kDelta, op.index);
  const uint64_t dn = d ? d->n : 0;
  if (!r.v[kFull].has_index()) {
    Index& f = r.v[kFull].idx[op.index];
    f.keys = DevBuf(std::max<uint64_t>(dn, 1) * 8, L_.stream);
    if (dn)
      SRDL_CUDA(cudaMemcpyAsync(f.keys.as<uint64_t>(), d->keys.as<uint64_t>(), dn * 8,
                                cudaMemcpyDeviceToDevice, L_.stream));
    f.n = dn;
    f.epoch = r.delta_epoch;
    r.base_epoch = r.full_epoch;
    r.full_epoch = r.delta_epoch;
    return;
  }
  if (dn == 0) return;
  if (r.lsm) {
    if (op.index != r.canonical) {
      // Only the canonical permutation has a HEAD; this one is rebuilt from it.
      r.v[kFull].idx.erase(op.index);
      return;
    }
    // DELTA goes into HEAD (O(|HEAD| + |DELTA|)); HEAD is merged into FULL
    // once it holds more than lsm_compact_pct percent of FULL (default 10,
    // device_2level_index.h:291-318).
    Index& f = full_base(r, op.index);
    const uint64_t fn = f.n;
    for (auto it2 = r.v[kFull].idx.begin(); it2 != r.v[kFull].idx.end();)
      it2 = it2->first == r.canonical ? std::next(it2) : r.v[kFull].idx.erase(it2);
    Index& h = r.head;
    r.base_epoch = r.full_epoch;
    r.full_epoch = r.delta_epoch;
    Index m;
    m.n = h.n + dn;
    m.keys = DevBuf(m.n * 8, L_.stream);
    size_t pid = prof_begin("merge");
    if (h.n)
      merge_disjoint(L_, h.keys.as<uint64_t>(), h.n, d->keys.as<uint64_t>(), dn,
                     m.keys.as<uint64_t>());
    else
      SRDL_CUDA(cudaMemcpyAsync(m.keys.as<uint64_t>(), d->keys.as<uint64_t>(), dn * 8,
                                cudaMemcpyDeviceToDevice, L_.stream));
    prof_end(pid, 16.0 * m.n, (double)m.n);
    h = std::move(m);
    if (h.n * 100 > fn * (uint64_t)opt_lsm_pct_) compact_head(r);
    return;
  }
  // The same DELTA is merged into every permutation the plan lists.  The
  // first one takes it on top of an up-to-date FULL; a later one merges it
  // only when it was up to date just before this delta, and is otherwise
  // rebuilt from a permutation that already holds it (never merged twice).
  auto fit = r.v[kFull].idx.find(op.index);
  Index* f = fit == r.v[kFull].idx.end() ? nullptr : &fit->second;
  if (r.full_epoch < r.delta_epoch) {
    if (!f || f->epoch != r.full_epoch) f = &ensure_index(r, kFull, op.index);
    r.base_epoch = r.full_epoch;
  } else {
    if (f && f->epoch == r.delta_epoch) return;
    if (!f || f->epoch != r.base_epoch) {
      ensure_index(r, kFull, op.index);  // rebuilt from one that holds this delta
      return;
    }
  }
  Index m;
  m.n = f->n + dn;
  m.keys = DevBuf(m.n * 8, L_.stream);
  size_t pid = prof_begin("merge");
  merge_disjoint(L_, f->keys.as<uint64_t>(), f->n, d->keys.as<uint64_t>(), dn,
                 m.keys.as<uint64_t>());
  prof_end(pid, 16.0 * m.n, (double)m.n);
  m.epoch = r.delta_epoch;
  r.full_epoch = r.delta_epoch;
  r.v[kFull].idx[op.index] = std::move(m);
}

uint64_t Database::shards_sum(uint64_t local) {
  std::vector<uint64_t> c((size_t)shard_world_, 0);
  c[0] = local;
  SRDL_REQUIRE(xfn_(xuser_, 2, "", c.data(), nullptr, nullptr, (void*)L_.stream) == 0, kErrState,
               "exchange callback failed (convergence vote)");
  return c[0];
}

// Sends the relation's NEW tuples to the shards that own their first
// declared column and keeps the ones received (one NEW chunk, canonical
// order).  Nothing to do on a single shard.
void Database::op_exchange(const Op& op) {
  if (shard_world_ <= 1) return;
  SRDL_REQUIRE(xfn_ != nullptr, kErrState,
               "plan exchanges tuples of " + op.rel + " between shards: set an exchange callback");
  Relation& r = rel(op.rel);
  SRDL_REQUIRE(r.arity <= 2, kErrUnsupported, "exchange of relation " + r.name + " of arity > 2");
  RelVersion& nv = r.v[kNew];
  const std::vector<int>& order = r.canonical;
  uint64_t total = 0;
  for (auto& c : nv.chunks) total += c.n;
  // gather NEW in canonical order
  DevBuf keys(std::max<uint64_t>(total, 1) * 8, L_.stream);
  uint64_t off = 0;
  for (auto& c : nv.chunks) {
    if (!c.n) continue;
    if (c.order == order)
      SRDL_CUDA(cudaMemcpyAsync(keys.as<uint64_t>() + off, c.keys.as<uint64_t>(), c.n * 8,
                                cudaMemcpyDeviceToDevice, L_.stream));
    else
      swap_halves(L_, c.keys.as<uint64_t>(), c.n, keys.as<uint64_t>() + off);
    off += c.n;
  }
  nv.chunks.clear();
  nv.idx.clear();
  const uint32_t world = (uint32_t)shard_world_;
  const bool col0_lo = !order.empty() && order[0] != 0;
  // group the keys by destination shard: one order-preserving selection per shard
  DevBuf send(std::max<uint64_t>(total, 1) * 8, L_.stream);
  std::vector<uint64_t> counts(world, 0);
  if (total) {
    DevBuf scratch(shard_select_scratch_bytes(total) + 1024, L_.stream);
    uint64_t acc = 0;
    for (uint32_t d = 0; d < world; d++) {
      Scratch s{scratch.as<char>(), scratch.bytes(), 0};
      shard_select(L_, keys.as<uint64_t>(), total, col0_lo, world, d, send.as<uint64_t>() + acc,
                   d_small_.as<uint64_t>(), s);
      counts[d] = read_scalar(0);
      acc += counts[d];
    }
    SRDL_REQUIRE(acc == total, kErrState, "exchange: keys lost while grouping by shard");
  }
  std::vector<uint64_t> io = counts;
  SRDL_REQUIRE(xfn_(xuser_, 0, r.name.c_str(), io.data(), nullptr, nullptr, (void*)L_.stream) == 0,
               kErrState, "exchange callback failed (counts of " + r.name + ")");
  uint64_t recv = 0;
  for (uint64_t v : io) recv += v;
  Chunk ch;
  ch.order = order;
  ch.keys = DevBuf(std::max<uint64_t>(recv, 1) * 8, L_.stream);
  ch.n = recv;
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  SRDL_REQUIRE(xfn_(xuser_, 1, r.name.c_str(), io.data(), send.as<uint64_t>(),
                    ch.keys.as<uint64_t>(), (void*)L_.stream) == 0,
               kErrState, "exchange callback failed (tuples of " + r.name + ")");
  nv.chunks.push_back(std::move(ch));
}

static const char* op_kind_name(Op::Kind k) {
  switch (k) {
    case Op::Execute: return "execute_pipeline";
    case Op::Rebuild: return "rebuild_index";
    case Op::Clear: return "clear_relation";
    case Op::CheckSize: return "check_size";
    case Op::ComputeDelta: return "compute_delta";
    case Op::Merge: return "merge_index";
    case Op::RebuildFrom: return "rebuild_index_from";
    case Op::Reconstruct: return "reconstruct";
    case Op::Hook: return "inject_cpp_hook";
    case Op::Exchange: return "exchange";
  }
  return "other";
}

void Database::exec_ops(const Step& st, uint64_t it) {
  for (size_t i = 0; i < st.ops.size(); i++) {
    const Op& op = st.ops[i];
    const auto h0 = std::chrono::steady_clock::now();
    struct OpTimer {
      OpStats& s;
      std::chrono::steady_clock::time_point t0;
      ~OpTimer() {
        const double ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        s.ms += ms;
        s.max_ms = ms > s.max_ms ? ms : s.max_ms;
        s.calls++;
      }
    } timer{opstats_[op_kind_name(op.kind)], h0};
    switch (op.kind) {
      case Op::Execute: exec_pipeline(op, st.recursive, it); break;
      case Op::Rebuild: {
        // NEW: sort + dedup the join output.  FULL / DELTA: make the
        // permutation current.  The planner places RebuildIndex(FULL) after
        // a stratum for the permutations later strata read but the stratum
        // did not merge into (src/srdatalog/mir/passes.py:104-145), so it is
        // rebuilt from a permutation holding every merged delta; relations
        // of arity > 2 keep their canonical order only (other orders are
        // derived views, built when a join reads them).
        Relation& r = rel(op.rel);
        if (op.ver == kNew) op_rebuild(st, i, op);
        else if (r.arity <= 2 && r.v[op.ver].has_index()) ensure_index(r, op.ver, op.index);
        break;
      }
      case Op::Clear:
        // A pending fused delta survives the clear of the old DELTA.
        rel(op.rel).v[op.ver].clear();
        break;
      case Op::CheckSize: break;
      case Op::ComputeDelta: op_compute_delta(op); break;
      case Op::Merge: op_merge(op); break;
      case Op::RebuildFrom: {
        // relations of arity > 2 keep their canonical order only (other
        // orders are derived views, built when a join reads them)
        Relation& r = rel(op.rel);
        if (r.arity <= 2) ensure_index(r, op.ver, op.index);
        break;
      }
      case Op::Reconstruct: break;
      case Op::Hook: break;
      case Op::Exchange: op_exchange(op); break;
    }
  }
}

void Database::run(uint64_t max_iters) {
  try {
    run_steps(max_iters);
  } catch (...) {
    // a failed run keeps none of its relations (their buffers go back to
    // the arena); the staged inputs stay for the next run
    cudaStreamSynchronize(L_.stream);
    reset_device_state();
    throw;
  }
}

void Database::run_steps(uint64_t max_iters) {
  init_device();
  SRDL_REQUIRE(shard_rank_ < shard_world_, kErrArg, "shard_rank must be below shard_world");
  reset_device_state();
  // the run's device-memory limit applies to every buffer the run holds,
  // the staged inputs included; the peak is recorded whether it succeeds
  arena_set_limit(L_.stream, 0);
  arena_reset_peak(L_.stream);
  struct MemRecord {
    Database* db;
    ~MemRecord() { db->mem_run_ = arena_use(db->L_.stream); }
  } mem_record{this};
  if (opt_mem_limit_) {
    const ArenaUse u = arena_use(L_.stream);
    SRDL_REQUIRE(u.in_use <= opt_mem_limit_, kErrCapacity,
                 "device memory limit of the run exceeded: " + std::to_string(u.in_use) +
                     " bytes held before it starts, limit " + std::to_string(opt_mem_limit_) +
                     " (mem_limit_mb)");
    arena_set_limit(L_.stream, opt_mem_limit_);
  }
  const uint64_t launches0 = launches_total();
  auto t0 = std::chrono::steady_clock::now();
  opstats_.clear();
  reset_alloc_max();
  const AllocStats a0 = alloc_stats();
  upload_inputs();
  instances_begin();
  {
    OpStats& u = opstats_["upload_inputs"];
    u.ms = u.max_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    u.calls = 1;
  }
  for (size_t si = 0; si < steps_.size(); si++) {
    const Step& st = steps_[si];
    auto s0 = std::chrono::steady_clock::now();
    if (!st.recursive) {
      exec_ops(st, 0);
      step_stats_[si].iterations = 1;
    } else {
      std::vector<std::string> computed;
      for (auto& op : st.ops)
        if (op.kind == Op::ComputeDelta) computed.push_back(op.rel);
      // From iteration 1 on, a qualifying step runs on the device loop
      // (loop.cu); an overflow hands one iteration back to the host path,
      // after which the loop is entered again (at most three times a step).
      std::string why;
      const bool loop_on =
          (opt_device_loop_ < 0 ? device_loop_default() : opt_device_loop_ != 0) && loop_eligible(st, why);
      int entries = 0;
      for (uint64_t it = 0; it < max_iters; it++) {
        if (it > 0) {
          uint64_t total = 0;
          for (auto& n : computed)
            for (auto& kv : rel(n).v[kDelta].idx) {
              total += kv.second.n;
              break;
            }
          // sharded with exchanges: stop only when every shard's delta is empty
          if (xfn_ && shard_world_ > 1) total = shards_sum(total);
          if (total == 0) break;
          if (loop_on && entries < 3) {
            entries++;
            uint64_t done = 0;
            loop_marks_ = instance_marks(si);
            const int rc = run_device_loop(st, it, max_iters, &done);
            loop_marks_ = nullptr;
            step_stats_[si].iterations += done;
            it += done;
            if (rc == kLoopDone) break;
            if (rc == kLoopSkipped) entries = 3;
            if (it >= max_iters) break;
          }
        }
        exec_ops(st, it);
        mark_instances(si, st, (uint32_t)(it + 1));
        step_stats_[si].iterations++;
      }
      instances_end(si, step_stats_[si].iterations);
      // Post-stratum reconstruct: every LSM relation ends as one FULL array.
      for (auto& kv : rels_)
        if (kv.second->head.n) compact_head(*kv.second);
      // the final FULL sizes size the device loop's buffers in later runs
      for (auto& n : computed) {
        Relation& r = rel(n);
        auto fit = r.v[kFull].idx.find(r.canonical);
        if (fit != r.v[kFull].idx.end()) full_max_[n] = std::max(full_max_[n], fit->second.n);
      }
    }
    SRDL_CUDA(cudaStreamSynchronize(L_.stream));
    step_stats_[si].ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - s0).count();
  }
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  run_ms_ = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  const AllocStats a1 = alloc_stats();
  alloc_ = {a1.ms - a0.ms, a1.max_ms, a1.calls - a0.calls};
  {
    cudaMemPool_t pool;
    uint64_t reserved = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, device_) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess)
      pool_reserved_gb_ = reserved / 1e9;
  }
  launches_ = launches_total() - launches0;
  prof_collect();
}

ArenaUse Database::mem_stats() const {
  ArenaUse u = dev_ready_ ? arena_use(L_.stream) : ArenaUse{};
  u.peak = mem_run_.peak;
  u.limit = opt_mem_limit_;
  return u;
}

uint64_t Database::size(const std::string& name) {
  Relation& r = rel(name);
  if (r.head.n) compact_head(r);
  auto& fv = r.v[kFull];
  auto it = fv.idx.find(r.canonical);
  if (it != fv.idx.end()) return it->second.n;
  for (auto& kv : fv.idx) return kv.second.n;
  return 0;
}

uint64_t Database::count(const std::string& rule) const {
  auto it = counts_.find(rule);
  return it == counts_.end() ? 0 : it->second;
}

int64_t Database::dump(const std::string& name, uint32_t* out, uint64_t cap_rows) {
  Relation& r = rel(name);
  if (!r.v[kFull].has_index()) return 0;
  if (r.arity > 2) {
    // packed tuples: unpack in index order, place in declared column order
    auto it = r.v[kFull].idx.find(r.canonical);
    if (r.pack_half == 0 || it == r.v[kFull].idx.end()) return 0;
    Index& ix = it->second;
    if (!out) return (int64_t)ix.n;
    SRDL_CUDA(cudaSetDevice(device_));
    const uint64_t n = std::min(ix.n, cap_rows);
    std::vector<uint64_t> keys(n);
    if (n)
      SRDL_CUDA(cudaMemcpyAsync(keys.data(), ix.keys.as<uint64_t>(), n * 8, cudaMemcpyDeviceToHost,
                                L_.stream));
    SRDL_CUDA(cudaStreamSynchronize(L_.stream));
    const int k = r.arity, b = r.pack_bits, h = r.pack_half;
    const uint64_t cmask = (1ull << b) - 1, hmask = (1ull << h) - 1;
    for (uint64_t i = 0; i < n; i++) {
      const uint64_t p = ((keys[i] >> 32) << h) | (keys[i] & hmask);
      for (int c = 0; c < k; c++)
        out[i * k + r.canonical[c]] = (uint32_t)((p >> (b * (k - 1 - c))) & cmask);
    }
    bool identity = true;
    for (int c = 0; c < k; c++) identity &= r.canonical[c] == c;
    if (!identity) {  // rows must come sorted in declared column order
      std::vector<std::vector<uint32_t>> rows(n);
      for (uint64_t i = 0; i < n; i++) rows[i].assign(out + i * k, out + (i + 1) * k);
      std::sort(rows.begin(), rows.end());
      for (uint64_t i = 0; i < n; i++) std::copy(rows[i].begin(), rows[i].end(), out + i * k);
    }
    return (int64_t)ix.n;
  }
  SRDL_CUDA(cudaSetDevice(device_));
  Index& ix = ensure_index(r, kFull, identity_perm(r.arity));
  if (!out) return (int64_t)ix.n;
  const uint64_t n = std::min(ix.n, cap_rows);
  std::vector<uint64_t> keys(n);
  if (n)
    SRDL_CUDA(cudaMemcpyAsync(keys.data(), ix.keys.as<uint64_t>(), n * 8, cudaMemcpyDeviceToHost,
                              L_.stream));
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  for (uint64_t i = 0; i < n; i++) {
    if (r.arity == 2) {
      out[2 * i] = (uint32_t)(keys[i] >> 32);
      out[2 * i + 1] = (uint32_t)keys[i];
    } else {
      out[i] = (uint32_t)(keys[i] >> 32);
    }
  }
  return (int64_t)ix.n;
}

std::string Database::stats_json() const {
  std::ostringstream o;
  o << "{\"plan\":\"" << name_ << "\",\"run_ms\":" << run_ms_ << ",\"derived\":" << derived_
    << ",\"value_bits\":" << bits_ << ",\"steps\":[";
  for (size_t i = 0; i < step_stats_.size(); i++) {
    o << (i ? "," : "") << "{\"recursive\":" << (steps_[i].recursive ? "true" : "false")
      << ",\"iterations\":" << step_stats_[i].iterations << ",\"ms\":" << step_stats_[i].ms << "}";
  }
  o << "],\"launches\":" << launches_ << ",\"kernels\":{";
  bool kfirst = true;
  for (auto& kv : kstats_) {
    o << (kfirst ? "" : ",") << "\"" << kv.first << "\":{\"ms\":" << kv.second.ms
      << ",\"bytes\":" << kv.second.bytes << ",\"units\":" << kv.second.units
      << ",\"scopes\":" << kv.second.scopes << "}";
    kfirst = false;
  }
  o << "},\"host_ops\":{";
  bool ofirst = true;
  for (auto& kv : opstats_) {
    o << (ofirst ? "" : ",") << "\"" << kv.first << "\":{\"ms\":" << kv.second.ms
      << ",\"max_ms\":" << kv.second.max_ms << ",\"calls\":" << kv.second.calls << "}";
    ofirst = false;
  }
  o << "},\"device_loop\":{\"entries\":" << loop_stats_.entries << ",\"iterations\":"
    << loop_stats_.iterations << ",\"overflows\":" << loop_stats_.overflows << ",\"skipped\":"
    << loop_stats_.skipped << ",\"capture_ms\":" << loop_stats_.capture_ms << ",\"run_ms\":"
    << loop_stats_.run_ms << ",\"last_error\":\"" << json_escape(loop_stats_.last_error) << "\"";
  o << "},\"mem\":{\"peak_bytes\":" << mem_run_.peak << ",\"limit_bytes\":" << opt_mem_limit_;
  o << "},\"alloc\":{\"ms\":" << alloc_.ms << ",\"max_ms\":" << alloc_.max_ms
    << ",\"calls\":" << alloc_.calls << ",\"pool_reserved_gb\":" << pool_reserved_gb_;
  o << "},\"counts\":{";
  bool first = true;
  for (auto& kv : counts_) {
    o << (first ? "" : ",") << "\"" << kv.first << "\":" << kv.second;
    first = false;
  }
  o << "}}";
  return o.str();
}

}  // namespace srdl
