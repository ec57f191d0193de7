// join.cu -- leapfrog-style WCOJ levels as two-pass count / expand kernels.
//
// Replaces the generated JitRunner_<rule>::kernel_count / kernel_materialize
// (src/srdatalog/codegen/jit/complete_runner.py:163-301) and their search
// primitives (RT/gpu/search.h group_*_bound, RT/gpu/runtime/jit/
// intersect_handles.h).  A pipeline is executed one MIR level at a time over
// a table of partial bindings:
//
//   count  : for every binding row, the size of its candidate list -- for a
//            column join the SHORTEST of the source lists (the leapfrog
//            driver), for a cartesian join the product of the lists, for a
//            scan the scanned range;
//   scan   : exclusive prefix sum of the counts (64-bit);
//   expand : one thread per candidate.  Its row is found by binary search in
//            the prefix sums, so a hub key with millions of candidates is
//            spread over thousands of threads exactly like a leaf key with
//            one (this replaces warp-per-root-key traversal plus the
//            work-stealing / block-group balancing of the reference,
//            ws_infrastructure.h and complete_runner.py:377-737).  A column
//            join candidate is probed in every other source list by binary
//            search; filters run next; survivors are appended with one
//            warp-aggregated atomic per warp (row order does not matter: the
//            next consumer is a sort), or only counted for count-only rules.
#include "kernels.h"

namespace srdl {

constexpr int kJThreads = 256;

// List of source s for input row r: [b, b+len) over roots (no prefix) or
// over child values (prefix bound).
__device__ __forceinline__ void src_list(const SrcSpec& s, const Table& in, uint64_t r,
                                         uint32_t& b, uint32_t& len) {
  if (s.prefix_slot < 0) {
    b = 0;
    len = s.t.n_roots;
  } else {
    uint32_t e;
    trie_range(s.t, in.col[s.prefix_slot][r], b, e);
    len = e - b;
  }
}

__device__ __forceinline__ uint32_t src_value(const SrcSpec& s, uint32_t pos) {
  return s.prefix_slot < 0 ? s.t.roots[pos] : s.t.lo[pos];
}

__device__ __forceinline__ bool src_contains(const SrcSpec& s, const Table& in, uint64_t r,
                                             uint32_t v) {
  if (s.prefix_slot < 0) return trie_has_root(s.t, v);
  uint32_t b, e;
  trie_range(s.t, in.col[s.prefix_slot][r], b, e);
  return child_contains(s.t, b, e, v);
}

__global__ void __launch_bounds__(kJThreads) join_count_kernel(LevelSpec lv, Table in,
                                                               uint64_t* __restrict__ work,
                                                               uint8_t* __restrict__ drv,
                                                               uint32_t* __restrict__ beg) {
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < in.n;
       r += (uint64_t)gridDim.x * blockDim.x) {
    if (lv.kind == kColumnJoin) {
      uint32_t best = 0xffffffffu, bb = 0;
      int bd = 0;
      for (int s = 0; s < lv.nsrc; s++) {
        uint32_t b, len;
        src_list(lv.src[s], in, r, b, len);
        if (len < best) {
          best = len;
          bd = s;
          bb = b;
        }
      }
      work[r] = best;
      drv[r] = (uint8_t)bd;
      beg[r] = bb;
    } else if (lv.kind == kCartesian) {
      uint64_t prod = 1;
      for (int s = 0; s < lv.nsrc; s++) {
        uint32_t b, len;
        src_list(lv.src[s], in, r, b, len);
        if (lv.src[s].out_slot < 0) prod = len ? prod : 0;
        else prod *= len;
      }
      work[r] = prod;
    } else {  // scan
      const SrcSpec& s = lv.src[0];
      if (s.prefix_slot < 0) {
        work[r] = s.t.n;
      } else {
        uint32_t b, e;
        trie_range(s.t, in.col[s.prefix_slot][r], b, e);
        work[r] = e - b;
      }
    }
  }
}

__device__ __forceinline__ uint64_t row_of(const uint64_t* offs, uint64_t lo, uint64_t hi,
                                           uint64_t w) {
  // largest r in [lo, hi) with offs[r] <= w
  uint64_t a = lo, b = hi;
  while (a + 1 < b) {
    uint64_t m = (a + b) >> 1;
    if (offs[m] <= w) a = m;
    else b = m;
  }
  return a;
}

__device__ __forceinline__ bool filt_ok(const FiltSpec& f, uint32_t a, uint32_t b) {
  switch (f.op) {
    case kNe: return a != b;
    case kEq: return a == b;
    case kLt: return a < b;
    case kLe: return a <= b;
    case kGt: return a > b;
    default: return a >= b;
  }
}

template <int EMIT>
__global__ void __launch_bounds__(kJThreads) join_expand_kernel(
    LevelSpec lv, Table in, const uint64_t* __restrict__ offs, const uint8_t* __restrict__ drv,
    const uint32_t* __restrict__ beg, uint64_t total, Table out, uint64_t* __restrict__ out_keys,
    unsigned long long* __restrict__ d_out_n) {
  __shared__ uint64_t rows[2];
  __shared__ unsigned long long red[kJThreads / 32];
  const int lane = threadIdx.x & 31;
  unsigned long long my_count = 0;
  for (uint64_t t0 = (uint64_t)blockIdx.x * kJThreads; t0 < total;
       t0 += (uint64_t)gridDim.x * kJThreads) {
    const uint64_t tlast = t0 + kJThreads - 1 < total ? t0 + kJThreads - 1 : total - 1;
    if (threadIdx.x == 0) rows[0] = row_of(offs, 0, in.n, t0);
    if (threadIdx.x == 32) rows[1] = row_of(offs, 0, in.n, tlast);
    __syncthreads();
    const uint64_t w = t0 + threadIdx.x;
    bool ok = w < total;
    uint64_t r = 0;
    uint32_t nv[kMaxSrc + 1];  // values of the slots this level binds
#pragma unroll
    for (int i = 0; i < kMaxSrc + 1; i++) nv[i] = 0;
    if (ok) {
      r = row_of(offs, rows[0], rows[1] + 1, w);
      const uint64_t local = w - offs[r];
      if (lv.kind == kColumnJoin) {
        const int d = drv[r];
        const uint32_t v = src_value(lv.src[d], beg[r] + (uint32_t)local);
        for (int s = 0; s < lv.nsrc && ok; s++)
          if (s != d) ok = src_contains(lv.src[s], in, r, v);
        nv[lv.cj_slot - lv.n_in_slots] = v;
      } else if (lv.kind == kCartesian) {
        uint64_t rem = local;
        for (int s = lv.nsrc - 1; s >= 0; s--) {
          const SrcSpec& sp = lv.src[s];
          if (sp.out_slot < 0) continue;
          uint32_t b, len;
          src_list(sp, in, r, b, len);
          const uint32_t idx = (uint32_t)(rem % len);
          rem /= len;
          nv[sp.out_slot - lv.n_in_slots] = src_value(sp, b + idx);
        }
      } else {
        const SrcSpec& sp = lv.src[0];
        uint32_t b = 0;
        if (sp.prefix_slot >= 0) {
          uint32_t e;
          trie_range(sp.t, in.col[sp.prefix_slot][r], b, e);
        }
        const uint64_t i = b + local;
        if (lv.scan_slot[0] >= 0) nv[lv.scan_slot[0] - lv.n_in_slots] = (uint32_t)(sp.t.keys[i] >> 32);
        if (lv.scan_slot[1] >= 0) nv[lv.scan_slot[1] - lv.n_in_slots] = (uint32_t)sp.t.keys[i];
      }
    }
    auto val = [&](int slot) -> uint32_t {
      return slot < lv.n_in_slots ? in.col[slot][r] : nv[slot - lv.n_in_slots];
    };
    for (int f = 0; f < lv.nfilt && ok; f++) {
      const FiltSpec& fs = lv.filt[f];
      const uint32_t a = fs.a_slot >= 0 ? val(fs.a_slot) : fs.a_const;
      const uint32_t b = fs.b_slot >= 0 ? val(fs.b_slot) : fs.b_const;
      ok = filt_ok(fs, a, b);
    }
    if (EMIT == kEmitCount) {
      my_count += ok;
    } else {
      const unsigned m = __ballot_sync(kAllLanes, ok);
      if (m) {
        const int leader = __ffs(m) - 1;
        unsigned long long base = 0;
        if (lane == leader) base = atomicAdd(d_out_n, (unsigned long long)__popc(m));
        base = __shfl_sync(kAllLanes, base, leader);
        if (ok) {
          const uint64_t pos = base + __popc(m & lanemask_lt());
          if (EMIT == kEmitKeys) {
            const uint64_t hi = val(lv.key_slot[0]);
            const uint64_t lo = lv.key_arity > 1 ? val(lv.key_slot[1]) : 0;
            out_keys[pos] = (hi << 32) | lo;
          } else {
            for (int c = 0; c < kMaxSlots; c++)
              if (out.col[c]) out.col[c][pos] = val(c);
          }
        }
      }
    }
    __syncthreads();
  }
  if (EMIT == kEmitCount) {
    unsigned long long s = warp_sum(my_count);
    if (lane == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned long long t = 0;
      for (int i = 0; i < kJThreads / 32; i++) t += red[i];
      if (t) atomicAdd(d_out_n, t);
    }
  }
}

size_t join_work_scratch_bytes(uint64_t rows) {
  rows = rows ? rows : 1;
  return ((rows * 8 + 255) & ~size_t(255)) + ((rows + 1) * 8 + 255) + ((rows + 255) & ~size_t(255)) +
         ((rows * 4 + 255) & ~size_t(255)) + scan_scratch_bytes(rows) + 1024;
}

static int jgrid(uint64_t n, int sms) {
  uint64_t g = (n + kJThreads - 1) / kJThreads;
  uint64_t cap = (uint64_t)sms * 16;
  if (g > cap) g = cap;
  return g ? (int)g : 1;
}

JoinWork join_count(const Launch& L, const LevelSpec& lv, const Table& in, Scratch& s) {
  JoinWork w;
  uint64_t* work = s.take<uint64_t>(in.n ? in.n : 1);
  w.offs = s.take<uint64_t>(in.n + 1);
  w.drv = s.take<uint8_t>(in.n ? in.n : 1);
  w.beg = s.take<uint32_t>(in.n ? in.n : 1);
  if (in.n) {
    join_count_kernel<<<jgrid(in.n, L.num_sms), kJThreads, 0, L.stream>>>(lv, in, work, w.drv,
                                                                          w.beg);
    SRDL_CUDA(cudaGetLastError());
    count_launches(1);
  }
  exclusive_scan_u64(L, work, in.n, w.offs, s);
  return w;
}

void join_expand(const Launch& L, const LevelSpec& lv, const Table& in, const JoinWork& w,
                 uint64_t total, Table* out_table, uint64_t* out_keys, uint64_t* d_out_n) {
  if (total == 0) return;
  Table out = out_table ? *out_table : Table{};
  const int g = jgrid(total, L.num_sms);
  auto* cnt = reinterpret_cast<unsigned long long*>(d_out_n);
  if (lv.emit == kEmitCount)
    join_expand_kernel<kEmitCount><<<g, kJThreads, 0, L.stream>>>(lv, in, w.offs, w.drv, w.beg,
                                                                 total, out, out_keys, cnt);
  else if (lv.emit == kEmitKeys)
    join_expand_kernel<kEmitKeys><<<g, kJThreads, 0, L.stream>>>(lv, in, w.offs, w.drv, w.beg,
                                                                total, out, out_keys, cnt);
  else
    join_expand_kernel<kEmitTable><<<g, kJThreads, 0, L.stream>>>(lv, in, w.offs, w.drv, w.beg,
                                                                 total, out, out_keys, cnt);
  SRDL_CUDA(cudaGetLastError());
  count_launches(1);
}

}  // namespace srdl
