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
//   expand : one lane per candidate.  Every warp owns an equal, contiguous
//            slice of the candidates and walks it 32 at a time, finding each
//            lane's row by galloping forward in the prefix sums from the
//            previous row.  A hub key with millions of candidates is thus
//            spread over thousands of warps exactly like a leaf key with one
//            (this replaces warp-per-root-key traversal plus the
//            work-stealing / block-group balancing of the reference,
//            ws_infrastructure.h and complete_runner.py:377-737), and no
//            block ever synchronises.  A column-join candidate is probed in
//            every other source list by binary search; filters run next.
//            Final levels append keys with one warp-aggregated atomic per
//            warp (the consumer sorts them) or only count; intermediate
//            tables are written in input order (count pass + scan + write
//            pass), so every binding table stays lexicographically sorted.

#include <algorithm>

#include "kernels.h"

namespace srdl {

constexpr int kJThreads = 256;
constexpr uint32_t kNoPair = 0xffffffffu;

// Position of the pair (a, b) in a pair index (a binary view whose row
// positions number the pairs), or kNoPair.
__device__ __forceinline__ uint32_t pair_pos(const TrieView& p, uint32_t a, uint32_t b) {
  uint32_t kb, ke;
  trie_range(p, a, kb, ke);
  const uint32_t q = lower_bound_u32(p.lo, kb, ke, b);
  return (q < ke && p.lo[q] == b) ? q : kNoPair;
}

// First row of a row index whose pair position is >= g (g <= pair count).
__device__ __forceinline__ uint32_t rows_from(const TrieView& t, uint32_t g) {
  if (t.dir && g < t.dir_n) return t.dir[g];
  return (uint32_t)lower_bound_u64(t.keys, 0, t.n, (uint64_t)g << 32);
}

// List of source s for input row r: [b, b+len) over roots (no prefix), over
// child values (prefix bound), or, for the ternary modes, over the row
// index's children of a pair (kSrcPair) or its rows under a range of pairs
// (kSrcRows).
__device__ __forceinline__ void src_list(const SrcSpec& s, const Table& in, uint64_t r,
                                         uint32_t& b, uint32_t& len) {
  if (s.mode == kSrcPair) {
    const uint32_t g = pair_pos(s.pair, in.col[s.prefix_slot][r], in.col[s.prefix_slot2][r]);
    uint32_t e = 0;
    b = 0;
    if (g != kNoPair) trie_range(s.t, g, b, e);
    len = e - b;
  } else if (s.mode == kSrcRows) {
    if (s.prefix_slot < 0) {
      b = 0;
      len = (uint32_t)s.t.n;
    } else {
      uint32_t kb, ke;
      trie_range(s.pair, in.col[s.prefix_slot][r], kb, ke);
      b = rows_from(s.t, kb);
      len = rows_from(s.t, ke) - b;
    }
  } else if (s.prefix_slot < 0) {
    b = 0;
    len = (uint32_t)*s.t.n_roots_d;
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
  if (s.mode == kSrcPair) {
    const uint32_t g = pair_pos(s.pair, in.col[s.prefix_slot][r], in.col[s.prefix_slot2][r]);
    return g != kNoPair && trie_child_contains(s.t, g, v);
  }
  if (s.prefix_slot < 0) return trie_has_root(s.t, v);
  return trie_child_contains(s.t, in.col[s.prefix_slot][r], v);
}

__global__ void __launch_bounds__(kJThreads) join_count_kernel(LevelSpec lv, Table in,
                                                               uint64_t* __restrict__ work,
                                                               uint8_t* __restrict__ drv,
                                                               uint32_t* __restrict__ beg,
                                                               uint2* __restrict__ orange,
                                                               uint32_t* __restrict__ obm,
                                                               uint64_t* __restrict__ pwork) {
  // A table written by the previous level may fill only part of its
  // capacity; its true size is on the device and the rest expands to nothing.
  const uint64_t nrows = in.d_n ? min(in.n, *in.d_n) : in.n;
  for (uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; r < in.n;
       r += (uint64_t)gridDim.x * blockDim.x) {
    if (r >= nrows) {
      work[r] = 0;
      if (pwork) pwork[r] = 0;
      continue;
    }
    if (lv.kind == kColumnJoin && lv.nsrc == 2) {
      // Leapfrog seek: the shorter list drives; it is clipped to the other
      // list's value range [first, last] (only that part can intersect),
      // searching only at an end that lies outside it.  The other list's
      // range is probed as it is.
      uint32_t b0, n0, b1, n1;
      src_list(lv.src[0], in, r, b0, n0);
      src_list(lv.src[1], in, r, b1, n1);
      const uint32_t* v0 = lv.src[0].prefix_slot < 0 ? lv.src[0].t.roots : lv.src[0].t.lo;
      const uint32_t* v1 = lv.src[1].prefix_slot < 0 ? lv.src[1].t.roots : lv.src[1].t.lo;
      const int bd = n1 < n0 ? 1 : 0;
      const uint32_t* dv = bd ? v1 : v0;
      const uint32_t* ov = bd ? v0 : v1;
      uint32_t db = bd ? b1 : b0, de = db + (bd ? n1 : n0);
      const uint32_t ob = bd ? b0 : b1, oe = ob + (bd ? n0 : n1);
      if (db < de && ob < oe) {
        const uint32_t lo = ov[ob], hi = ov[oe - 1];
        if (dv[db] < lo) db = lower_bound_u32(dv, db, de, lo);
        if (db < de && dv[de - 1] > hi) de = lower_bound_u32(dv, db, de, hi + 1);
      } else {
        de = db;
      }
      work[r] = de - db;
      drv[r] = (uint8_t)bd;
      beg[r] = db;
      orange[r] = make_uint2(ob, oe);
      if (obm) {
        // the probed (other) list's bitmap, if its parent value has one
        const uint32_t* obd = bd ? lv.src[0].t.bdir : lv.src[1].t.bdir;
        const int ops = bd ? lv.src[0].prefix_slot : lv.src[1].prefix_slot;
        obm[r] = (obd && ops >= 0) ? obd[in.col[ops][r]] : kNoBitmap;
        if (pwork) {
          // a pivot row: the probed list is the pivot source's, bitmapped
          // and long; its candidates move from cj2 to the pivot kernel
          const bool piv = bd != lv.pivot_src && obm[r] != kNoBitmap &&
                           (lv.pivot_src == 0 ? n0 : n1) >= lv.pivot_min;
          pwork[r] = piv ? (uint64_t)(de - db) : 0;
          if (piv) work[r] = 0;
        }
      }
    } else if (lv.kind == kColumnJoin) {
      uint32_t best = 0xffffffffu, bb = 0;
      int bd = 0;
      bool empty = false;
      for (int s = 0; s < lv.nsrc; s++) {
        uint32_t b, len;
        src_list(lv.src[s], in, r, b, len);
        empty |= len == 0;
        if (len < best) {
          best = len;
          bd = s;
          bb = b;
        }
      }
      work[r] = empty ? 0 : best;
      drv[r] = (uint8_t)bd;
      beg[r] = bb;
      if (lv.nsrc == 2) {
        uint32_t ob, olen;
        src_list(lv.src[1 - bd], in, r, ob, olen);
        orange[r] = make_uint2(ob, ob + olen);
      }
    } else if (lv.kind == kCartesian) {
      uint64_t prod = 1;
      for (int s = 0; s < lv.nsrc; s++) {
        uint32_t b, len;
        src_list(lv.src[s], in, r, b, len);
        if (lv.src[s].out_slot < 0) prod = len ? prod : 0;
        else prod *= len;
        // two-source form: list 0 begin in beg, list 1 as [begin, length)
        if (lv.nsrc == 2) {
          if (s == 0) beg[r] = b;
          else orange[r] = make_uint2(b, len);
        }
      }
      work[r] = prod;
    } else {  // scan
      const SrcSpec& s = lv.src[0];
      if (s.mode == kSrcRows) {
        uint32_t b, len;
        src_list(s, in, r, b, len);
        work[r] = len;
      } else if (s.prefix_slot < 0) {
        work[r] = s.t.n;
      } else {
        uint32_t b, e;
        trie_range(s.t, in.col[s.prefix_slot][r], b, e);
        work[r] = e - b;
      }
    }
  }
}

// Largest r in [lo, n) with offs[r] <= w, given offs[lo] <= w: gallop, then bisect.
__device__ __forceinline__ uint64_t gallop_row(const uint64_t* offs, uint64_t lo, uint64_t n,
                                               uint64_t w) {
  uint64_t step = 1;
  while (lo + step < n && offs[lo + step] <= w) {
    lo += step;
    step <<= 1;
  }
  uint64_t hi = lo + step < n ? lo + step : n;  // offs[hi] > w or hi == n
  while (lo + 1 < hi) {
    uint64_t m = (lo + hi) >> 1;
    if (offs[m] <= w) lo = m;
    else hi = m;
  }
  return lo;
}

__device__ __forceinline__ bool filt_ok(const FiltSpec& f, uint32_t a, uint32_t b) {
  if (f.shard_world) return shard_owner(a, f.shard_world) == f.b_const;
  if (f.negation) return f.neg_n == 1 ? !trie_has_root(f.neg, a) : !trie_child_contains(f.neg, a, b);
  switch (f.op) {
    case kNe: return a != b;
    case kEq: return a == b;
    case kLt: return a < b;
    case kLe: return a <= b;
    case kGt: return a > b;
    default: return a >= b;
  }
}

// A shard's work items are the segments seg_rank, seg_rank + seg_world, ...
// of `seg` items each (lv.seg = 0: all items, unsegmented).  The expand
// kernels walk this shard's items as a dense "virtual" range [0, total) in
// warp rounds of 32; SegWalk maps a round's first virtual item to its actual
// item (a round never straddles segments: seg and every warp's start are
// multiples of 32).
// Instantiated with SEG = false for unsharded levels, which keep the plain
// index arithmetic (and register count) of the hot kernels.
template <bool SEG>
struct SegWalk {
  uint64_t seg, stride, rank_off, idx, off;
  __device__ __forceinline__ SegWalk(const LevelSpec& lv, uint64_t v0) {
    if (SEG) {
      seg = lv.seg;
      idx = v0 / seg;
      off = v0 - idx * seg;
      stride = seg * lv.seg_world;
      rank_off = seg * lv.seg_rank;
    } else {
      seg = idx = stride = rank_off = 0;
      off = v0;
    }
  }
  __device__ __forceinline__ uint64_t at() const { return SEG ? idx * stride + rank_off + off : off; }
  __device__ __forceinline__ void next() {
    off += 32;
    if (SEG && off == seg) {
      off = 0;
      idx++;
    }
  }
};

// Key of an emitted binding from its column values c[0..key_arity) in the
// target index order: (c0 << 32) | c1 for two columns (c0 << 32 for one);
// three or four columns packed pack_bits apiece into P and split at
// pack_half bits, (P >> pack_half) << 32 | (P mod 2^pack_half).
__device__ __forceinline__ uint64_t emit_key(const LevelSpec& lv, const uint32_t (&c)[4]) {
  if (lv.key_arity <= 2) return ((uint64_t)c[0] << 32) | (lv.key_arity > 1 ? c[1] : 0u);
  uint64_t p = 0;
#pragma unroll
  for (int i = 0; i < 4; i++)
    if (i < lv.key_arity) p = (p << lv.pack_bits) | c[i];
  return ((p >> lv.pack_half) << 32) | (p & ((1ull << lv.pack_half) - 1));
}

enum ExpandMode : int { kModeCount = 0, kModeKeys = 1, kModeTableCount = 2, kModeTableWrite = 3 };

// Device loop: the true candidate count (clamped to the capacity `total`;
// a larger count raises the overflow flag once, from the first thread).
__device__ __forceinline__ uint64_t dev_total(const JoinDev& jd, uint64_t total) {
  if (!jd.d_total) return total;
  const uint64_t t = *jd.d_total;
  if (t > total) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && jd.d_overflow) atomicExch(jd.d_overflow, 1u);
    return total;
  }
  return t;
}

// A warp's share of the candidates when the count is only known on the
// device: whole rounds of 32, spread evenly over the grid's warps.
__device__ __forceinline__ uint64_t dev_warp_chunk(const JoinDev& jd, uint64_t chunk, uint64_t total) {
  if (!jd.d_total) return chunk;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x / 32);
  return (((total + warps - 1) / warps) + 31) & ~uint64_t(31);
}

// Warp-aggregated append of the m-set lanes' keys at *d_out_n; with an
// output capacity, positions past it are dropped and raise the flag.
__device__ __forceinline__ void append_key(const JoinDev& jd, unsigned m, bool ok, int lane,
                                           unsigned long long* d_out_n, uint64_t* out_keys,
                                           uint64_t key) {
  if (!m) return;
  const int leader = __ffs(m) - 1;
  unsigned long long pos0 = 0;
  if (lane == leader) pos0 = atomicAdd(d_out_n, (unsigned long long)__popc(m));
  pos0 = __shfl_sync(kAllLanes, pos0, leader);
  const uint64_t pos = pos0 + __popc(m & lanemask_lt());
  if (jd.out_cap && pos0 + __popc(m) > jd.out_cap && lane == leader && jd.d_overflow)
    atomicExch(jd.d_overflow, 1u);
  if (ok && (!jd.out_cap || pos < jd.out_cap)) out_keys[pos] = key;
}

// in.col[k][r] with a compile-time slot index, so the Table parameter is
// never copied to local memory for a runtime subscript.
__device__ __forceinline__ uint32_t slot_value(const Table& t, int k, uint64_t r) {
  uint32_t x = 0;
#pragma unroll
  for (int c = 0; c < kMaxSlots; c++)
    if (c == k) x = t.col[c][r];
  return x;
}

__device__ __forceinline__ void slot_store(const Table& t, int k, uint64_t pos, uint32_t x) {
#pragma unroll
  for (int c = 0; c < kMaxSlots; c++)
    if (c == k) t.col[c][pos] = x;
}

// Filters of a level over the input row's slots and up to two new values.
__device__ __forceinline__ bool level_filters(const LevelSpec& lv, const Table& in, uint64_t r,
                                              int s0, uint32_t v0, int s1, uint32_t v1) {
  bool ok = true;
#pragma unroll
  for (int f = 0; f < kMaxFilt; f++) {
    if (f < lv.nfilt) {
      const FiltSpec fs = lv.filt[f];
      uint32_t a = fs.a_const, b = fs.b_const;
      if (fs.a_slot >= 0)
        a = fs.a_slot == s0 ? v0 : fs.a_slot == s1 ? v1 : slot_value(in, fs.a_slot, r);
      if (fs.b_slot >= 0)
        b = fs.b_slot == s0 ? v0 : fs.b_slot == s1 ? v1 : slot_value(in, fs.b_slot, r);
      if (fs.negation || fs.shard_world) {
        ok &= filt_ok(fs, a, b);
        continue;
      }
      switch (fs.op) {
        case kNe: ok &= a != b; break;
        case kEq: ok &= a == b; break;
        case kLt: ok &= a < b; break;
        case kLe: ok &= a <= b; break;
        case kGt: ok &= a > b; break;
        default: ok &= a >= b; break;
      }
    }
  }
  return ok;
}

// First index p in [b, e) with a[p] >= v (e if none); branch-free halving.
__device__ __forceinline__ uint32_t lower_bound_bf(const uint32_t* __restrict__ a, uint32_t b,
                                                   uint32_t e, uint32_t v) {
  uint32_t len = e - b;
  if (len == 0) return b;
  while (len > 1) {
    const uint32_t half = len >> 1;
    b = (a[b + half] < v) ? b + half : b;
    len -= half;
  }
  return b + (a[b] < v ? 1u : 0u);
}

// Two-source column join without filters (the common leapfrog step): the
// count pass stored, per row, the driver list begin and the other list's
// range, so a candidate costs one coalesced load of its value plus a
// branch-free binary search in the other list (or one bitmap word, or a
// directory check when the other list is all roots of a dense index).
//
// Work distribution: the candidates are cut into chunks of `chunk` (a
// multiple of 32) and resident warps take chunks in increasing order from a
// device-wide counter (block-level work stealing).  Rows are sorted by their
// first column, so the warps in flight at any moment all work inside a
// window of about (resident warps x chunk) candidates: the few first-column
// values there, whose child lists and bitmaps the probes of the window reuse,
// stay in L2 instead of every warp's slice touching a different part of the
// index.  A skewed row spans as many chunks as its candidates fill.  The
// table modes record each chunk's surviving count (count pass) and write the
// chunk's survivors at the scanned offset (write pass), so the table stays
// in input order.
template <int MODE, bool SEG>
__global__ void __launch_bounds__(kJThreads) join_cj2_kernel(
    LevelSpec lv, Table in, const uint64_t* __restrict__ offs, const uint8_t* __restrict__ drv,
    const uint32_t* __restrict__ beg, const uint2* __restrict__ orange,
    const uint32_t* __restrict__ obm, uint64_t total, uint64_t chunk,
    unsigned long long* __restrict__ queue, Table out, uint64_t* __restrict__ out_keys,
    unsigned long long* __restrict__ d_out_n, uint64_t* __restrict__ chunk_counts, JoinDev jd) {
  const int lane = threadIdx.x & 31;
  // (count-only rules never run in the device loop: the count instance
  // keeps the registers of the hot triangle level free of it)
  if (MODE != kModeCount) total = dev_total(jd, total);
  const uint32_t* vals0 = lv.src[0].prefix_slot < 0 ? lv.src[0].t.roots : lv.src[0].t.lo;
  const uint32_t* vals1 = lv.src[1].prefix_slot < 0 ? lv.src[1].t.roots : lv.src[1].t.lo;
  // a roots-list side with a dense directory answers membership in O(1)
  const uint32_t* dir0 = lv.src[0].prefix_slot < 0 ? lv.src[0].t.dir : nullptr;
  const uint32_t* dir1 = lv.src[1].prefix_slot < 0 ? lv.src[1].t.dir : nullptr;
  const uint32_t dn0 = lv.src[0].t.dir_n, dn1 = lv.src[1].t.dir_n;
  const uint32_t* bp0 = lv.src[0].t.bpool;
  const uint32_t* bp1 = lv.src[1].t.bpool;
  const uint32_t bw0 = lv.src[0].t.bwords, bw1 = lv.src[1].t.bwords;
  const uint64_t nchunks = (total + chunk - 1) / chunk;
  unsigned long long counted = 0;  // count mode: this warp's survivors over all its chunks
  while (true) {
    unsigned long long k = 0;
    if (lane == 0) k = atomicAdd(queue, 1ull);
    k = __shfl_sync(kAllLanes, k, 0);
    if (k >= nchunks) break;
    const uint64_t c0 = k * chunk;
    const uint64_t c1 = c0 + chunk < total ? c0 + chunk : total;
    unsigned long long running = MODE == kModeTableWrite ? chunk_counts[k] : 0ull;
    SegWalk<SEG> sw(lv, c0);
    // the row holding the chunk's first candidate: the last row whose offset
    // is <= it (a warp-wide search, log32 of the rows in load rounds)
    const uint64_t first = sw.at();
    uint64_t r0 = warp_partition_point(0, in.n, [&](uint64_t i) { return offs[i] <= first; }) - 1;
    // The row of the round's first candidate and its metadata, kept while the
    // warp stays in it (r0 is warp-uniform): most candidates lie in rows
    // longer than a warp round, whose lanes then need no row search and no
    // per-lane metadata loads.
    uint64_t crow = ~0ull, c_off = 0, c_end = 0;
    int cd = 0;
    uint32_t cbeg = 0, cslot = kNoBitmap;
    uint2 crg = make_uint2(0, 0);
    for (uint64_t base = c0; base < c1; base += 32, sw.next()) {
      const uint64_t abase = sw.at();
      const uint64_t w = abase + lane;
      bool ok = base + lane < c1;
      uint64_t r = r0;
      uint32_t v = 0;
      if (r0 != crow) {
        crow = r0;
        c_off = offs[r0];
        c_end = offs[r0 + 1];
        cd = drv[r0];
        cbeg = beg[r0];
        crg = orange[r0];
        cslot = obm ? obm[r0] : kNoBitmap;
      }
      if (MODE == kModeCount && !SEG && abase + 63 < c_end && base + 63 < c1 && !lv.grp_bounds) {
        // count only: two rounds at once while both lie in the cached row,
        // so each lane has two independent loads and probes in flight
        auto probe = [&](uint32_t x) -> bool {
          const uint32_t* odir = cd == 0 ? dir1 : dir0;
          if (odir) {
            const uint32_t odn = cd == 0 ? dn1 : dn0;
            return x + 1u < odn && odir[x] < odir[x + 1];
          }
          if (cslot != kNoBitmap) {
            const uint32_t* bm = cd == 0 ? bp1 : bp0;
            const uint32_t bw = cd == 0 ? bw1 : bw0;
            return (bm[(uint64_t)cslot * bw + (x >> 5)] >> (x & 31)) & 1u;
          }
          const uint32_t* ov = cd == 0 ? vals1 : vals0;
          const uint32_t p = lower_bound_bf(ov, crg.x, crg.y, x);
          return p < crg.y && ov[p] == x;
        };
        const uint32_t* dv = cd == 0 ? vals0 : vals1;
        const uint32_t i0 = cbeg + (uint32_t)(w - c_off);
        const uint32_t va = dv[i0], vb = dv[i0 + 32];
        const bool oa = probe(va), ob = probe(vb);
        running += __popc(__ballot_sync(kAllLanes, oa)) + __popc(__ballot_sync(kAllLanes, ob));
        base += 32;  // (the loop adds the second round's 32)
        sw.next();
        continue;    // r0 stays: both rounds lie in its row
      }
      if (abase + 31 < c_end) {
        if (ok) {
          v = (cd == 0 ? vals0 : vals1)[cbeg + (uint32_t)(w - c_off)];
          const uint32_t* odir = cd == 0 ? dir1 : dir0;
          if (odir) {
            const uint32_t odn = cd == 0 ? dn1 : dn0;
            ok = v + 1u < odn && odir[v] < odir[v + 1];
          } else if (cslot != kNoBitmap) {
            const uint32_t* bm = cd == 0 ? bp1 : bp0;
            const uint32_t bw = cd == 0 ? bw1 : bw0;
            ok = (bm[(uint64_t)cslot * bw + (v >> 5)] >> (v & 31)) & 1u;
          } else {
            const uint32_t* ov = cd == 0 ? vals1 : vals0;
            const uint32_t p = lower_bound_bf(ov, crg.x, crg.y, v);
            ok = p < crg.y && ov[p] == v;
          }
        }
      } else if (ok) {
        r = gallop_row(offs, r0, in.n, w);
        const uint32_t local = (uint32_t)(w - offs[r]);
        const int d = drv[r];
        v = (d == 0 ? vals0 : vals1)[beg[r] + local];
        const uint32_t* odir = d == 0 ? dir1 : dir0;
        const uint32_t slot = obm ? obm[r] : kNoBitmap;
        if (odir) {
          const uint32_t odn = d == 0 ? dn1 : dn0;
          ok = v + 1u < odn && odir[v] < odir[v + 1];
        } else if (slot != kNoBitmap) {
          const uint32_t* bm = d == 0 ? bp1 : bp0;
          const uint32_t bw = d == 0 ? bw1 : bw0;
          ok = (bm[(uint64_t)slot * bw + (v >> 5)] >> (v & 31)) & 1u;
        } else {
          const uint2 rg = orange[r];
          const uint32_t* ov = d == 0 ? vals1 : vals0;
          const uint32_t p = lower_bound_bf(ov, rg.x, rg.y, v);
          ok = p < rg.y && ov[p] == v;
        }
      }
      const unsigned m = __ballot_sync(kAllLanes, ok);
      if (MODE == kModeCount && lv.grp_bounds) {
        // per-group counts (one request of a batch per group): warp-aggregated
        int g = -1;
        if (ok) {
          const uint32_t key = lv.n_in_slots > 0 ? in.col[0][r] : v;
          uint32_t lo = 0, hi = lv.n_groups + 1;  // last bound <= key
          while (lo + 1 < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (lv.grp_bounds[mid] <= key) lo = mid;
            else hi = mid;
          }
          if (key >= lv.grp_bounds[0] && lo < lv.n_groups) g = (int)lo;
        }
        const unsigned peers = __match_any_sync(kAllLanes, g);
        if (g >= 0 && lane == __ffs(peers) - 1)
          atomicAdd(&lv.grp_counts[g], (unsigned long long)__popc(peers));
      }
      if (MODE == kModeCount || MODE == kModeTableCount) {
        running += __popc(m);
      } else if (MODE == kModeKeys) {
        uint64_t key = 0;
        if (ok) {
          uint32_t kc[4];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int ks = lv.key_slot[i];
            kc[i] = i < lv.key_arity ? (ks < lv.n_in_slots ? slot_value(in, ks, r) : v) : 0u;
          }
          key = emit_key(lv, kc);
        }
        append_key(jd, m, ok, lane, d_out_n, out_keys, key);
      } else {
        if (ok) {
          const uint64_t pos = running + __popc(m & lanemask_lt());
#pragma unroll
          for (int c = 0; c < kMaxSlots; c++)
            if (c < lv.n_in_slots) out.col[c][pos] = in.col[c][r];
          slot_store(out, lv.cj_slot, pos, v);
        }
        running += __popc(m);
      }
      r0 = __shfl_sync(kAllLanes, r, 31);
    }
    if (MODE == kModeCount) counted += running;
    else if (MODE == kModeTableCount && lane == 0) chunk_counts[k] = running;
  }
  if (MODE == kModeCount && lane == 0 && counted) atomicAdd(d_out_n, counted);
}

template <int MODE, bool SEG>
__global__ void __launch_bounds__(kJThreads) join_expand_kernel(
    LevelSpec lv, Table in, const uint64_t* __restrict__ offs, const uint8_t* __restrict__ drv,
    const uint32_t* __restrict__ beg, uint64_t total, uint64_t chunk, Table out,
    uint64_t* __restrict__ out_keys, unsigned long long* __restrict__ d_out_n,
    uint64_t* __restrict__ warp_counts, JoinDev jd) {
  const int lane = threadIdx.x & 31;
  total = dev_total(jd, total);
  chunk = dev_warp_chunk(jd, chunk, total);
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t c0 = gw * chunk;
  const uint64_t c1 = c0 + chunk < total ? c0 + chunk : total;
  unsigned long long running = 0;
  if (MODE == kModeTableWrite) running = warp_counts[gw];
  if (c0 < c1) {
    SegWalk<SEG> sw(lv, c0);
    uint64_t r0 = gallop_row(offs, 0, in.n, sw.at());
    for (uint64_t base = c0; base < c1; base += 32, sw.next()) {
      const uint64_t w = sw.at() + lane;
      bool ok = base + lane < c1;
      uint64_t r = r0;
      uint32_t nv[kMaxSrc + 1];  // values of the slots this level binds
#pragma unroll
      for (int i = 0; i < kMaxSrc + 1; i++) nv[i] = 0;
      if (ok) {
        r = gallop_row(offs, r0, in.n, w);
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
            if (sp.mode == kSrcRows) {
              // a ternary row under the bound c0: c1 from the pair index, c2 from the row
              const uint32_t i = b + idx;
              nv[sp.out_slot - lv.n_in_slots] = sp.pair.lo[(uint32_t)(sp.t.keys[i] >> 32)];
              nv[sp.out_slot2 - lv.n_in_slots] = sp.t.lo[i];
            } else {
              nv[sp.out_slot - lv.n_in_slots] = src_value(sp, b + idx);
            }
          }
        } else {
          const SrcSpec& sp = lv.src[0];
          if (sp.mode == kSrcRows) {
            uint32_t b, len;
            src_list(sp, in, r, b, len);
            const uint32_t i = b + (uint32_t)local;
            const uint32_t g = (uint32_t)(sp.t.keys[i] >> 32);
            if (lv.scan_slot[0] >= 0) nv[lv.scan_slot[0] - lv.n_in_slots] = (uint32_t)(sp.pair.keys[g] >> 32);
            if (lv.scan_slot[1] >= 0) nv[lv.scan_slot[1] - lv.n_in_slots] = sp.pair.lo[g];
            if (lv.scan_slot[2] >= 0) nv[lv.scan_slot[2] - lv.n_in_slots] = sp.t.lo[i];
          } else {
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
      const unsigned m = __ballot_sync(kAllLanes, ok);
      if (MODE == kModeCount || MODE == kModeTableCount) {
        running += __popc(m);
      } else if (MODE == kModeKeys) {
        uint64_t key = 0;
        if (ok) {
          uint32_t kc[4];
#pragma unroll
          for (int i = 0; i < 4; i++) kc[i] = i < lv.key_arity ? val(lv.key_slot[i]) : 0u;
          key = emit_key(lv, kc);
        }
        append_key(jd, m, ok, lane, d_out_n, out_keys, key);
      } else {  // ordered table write
        if (ok) {
          const uint64_t pos = running + __popc(m & lanemask_lt());
          for (int c = 0; c < kMaxSlots; c++)
            if (out.col[c]) out.col[c][pos] = val(c);
        }
        running += __popc(m);
      }
      r0 = __shfl_sync(kAllLanes, r, 31);
    }
  }
  if (MODE == kModeCount) {
    if (lane == 0 && running) atomicAdd(d_out_n, running);
  } else if (MODE == kModeTableCount) {
    if (lane == 0) warp_counts[gw] = running;
  }
}

// Two-source cartesian product (both sources bind one variable): per row the
// count pass stored list 0's begin and list 1's [begin, length); candidate
// `local` pairs element local / len1 of list 0 with local % len1 of list 1.
template <int MODE, bool SEG>
__global__ void __launch_bounds__(kJThreads) join_cart2_kernel(
    LevelSpec lv, Table in, const uint64_t* __restrict__ offs, const uint32_t* __restrict__ beg,
    const uint2* __restrict__ orange, uint64_t total, uint64_t chunk, Table out,
    uint64_t* __restrict__ out_keys, unsigned long long* __restrict__ d_out_n,
    uint64_t* __restrict__ warp_counts, JoinDev jd) {
  const int lane = threadIdx.x & 31;
  total = dev_total(jd, total);
  chunk = dev_warp_chunk(jd, chunk, total);
  // every candidate a result (no filter) and the output private to this
  // launch: each is written at its own index
  const bool exact = MODE == kModeKeys && lv.nfilt == 0 && (!jd.d_total || jd.exact_ok);
  const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t c0 = gw * chunk;
  const uint64_t c1 = c0 + chunk < total ? c0 + chunk : total;
  const uint32_t* vals0 = lv.src[0].prefix_slot < 0 ? lv.src[0].t.roots : lv.src[0].t.lo;
  const uint32_t* vals1 = lv.src[1].prefix_slot < 0 ? lv.src[1].t.roots : lv.src[1].t.lo;
  const int s0 = lv.src[0].out_slot, s1 = lv.src[1].out_slot;
  unsigned long long running = 0;
  if (MODE == kModeTableWrite) running = warp_counts[gw];
  if (exact && gw == 0 && lane == 0) {
    *d_out_n = total;
    if (jd.out_cap && total > jd.out_cap && jd.d_overflow) atomicExch(jd.d_overflow, 1u);
  }
  if (c0 < c1) {
    SegWalk<SEG> sw(lv, c0);
    uint64_t r0 = gallop_row(offs, 0, in.n, sw.at());
    for (uint64_t base = c0; base < c1; base += 32, sw.next()) {
      const uint64_t w = sw.at() + lane;
      bool ok = base + lane < c1;
      uint64_t r = r0;
      uint32_t v0 = 0, v1 = 0;
      if (ok) {
        r = gallop_row(offs, r0, in.n, w);
        const uint64_t local = w - offs[r];
        const uint2 rg = orange[r];
        uint32_t i0, i1;
        if (local < (1ull << 32)) {  // 32-bit division whenever it fits
          i0 = (uint32_t)local / rg.y;
          i1 = (uint32_t)local - i0 * rg.y;
        } else {
          i0 = (uint32_t)(local / rg.y);
          i1 = (uint32_t)(local - (uint64_t)i0 * rg.y);
        }
        v0 = vals0[beg[r] + i0];
        v1 = vals1[rg.x + i1];
        if (lv.nfilt) ok = level_filters(lv, in, r, s0, v0, s1, v1);
      }
      if (exact) {
        // every candidate is a result: candidate index = output position
        if (ok) {
          uint32_t kc[4];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int ks = lv.key_slot[i];
            kc[i] = i >= lv.key_arity ? 0u : ks == s0 ? v0 : ks == s1 ? v1 : slot_value(in, ks, r);
          }
          if (!jd.out_cap || base + lane < jd.out_cap) out_keys[base + lane] = emit_key(lv, kc);
        }
        r0 = __shfl_sync(kAllLanes, r, 31);
        continue;
      }
      const unsigned m = __ballot_sync(kAllLanes, ok);
      if (MODE == kModeCount || MODE == kModeTableCount) {
        running += __popc(m);
      } else if (MODE == kModeKeys) {
        uint64_t key = 0;
        if (ok) {
          uint32_t kc[4];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int ks = lv.key_slot[i];
            kc[i] = i >= lv.key_arity ? 0u : ks == s0 ? v0 : ks == s1 ? v1 : slot_value(in, ks, r);
          }
          key = emit_key(lv, kc);
        }
        append_key(jd, m, ok, lane, d_out_n, out_keys, key);
      } else {
        if (ok) {
          const uint64_t pos = running + __popc(m & lanemask_lt());
#pragma unroll
          for (int c = 0; c < kMaxSlots; c++)
            if (c < lv.n_in_slots) out.col[c][pos] = in.col[c][r];
          slot_store(out, s0, pos, v0);
          slot_store(out, s1, pos, v1);
        }
        running += __popc(m);
      }
      r0 = __shfl_sync(kAllLanes, r, 31);
    }
  }
  if (MODE == kModeCount) {
    if (lane == 0 && running) atomicAdd(d_out_n, running);
  } else if (MODE == kModeTableCount) {
    if (lane == 0) warp_counts[gw] = running;
  }
}

size_t join_work_scratch_bytes(uint64_t rows) {
  rows = rows ? rows : 1;
  // (+ the pivot rows' work, offsets and their scan)
  return ((rows * 8 + 255) & ~size_t(255)) + ((rows + 1) * 8 + 255) + ((rows + 255) & ~size_t(255)) +
         2 * ((rows * 4 + 255) & ~size_t(255)) + ((rows * 8 + 255) & ~size_t(255)) +
         scan_scratch_bytes(rows) + 1024 + ((rows * 8 + 255) & ~size_t(255)) + ((rows + 1) * 8 + 511) +
         scan_scratch_bytes(rows) + 512;
}

static int jgrid(uint64_t n, const Launch& L) {
  uint64_t g = (n + kJThreads - 1) / kJThreads;
  uint64_t cap = (uint64_t)L.num_sms * (L.join_bpsm > 0 ? L.join_bpsm : 16);
  if (g > cap) g = cap;
  return g ? (int)g : 1;
}

// Most per-chunk counts the two-source column join keeps in its table modes.
constexpr uint64_t kCj2MaxTableChunks = 1ull << 18;

size_t join_expand_scratch_bytes(const Launch& L, uint64_t total) {
  // per-warp counts of the generic kernels' table modes, or per-chunk counts
  // of the two-source column join's (chunks of at least 64 candidates)
  const uint64_t warps = (uint64_t)jgrid(total, L) * (kJThreads / 32);
  const uint64_t chunks = std::min<uint64_t>(kCj2MaxTableChunks, (total + 63) / 64);
  const uint64_t n = std::max<uint64_t>(warps, chunks);
  return 2 * ((n + 1) * 8 + 255) + scan_scratch_bytes(n) + 4096;
}

// Resident blocks per SM of the two-source column-join kernel for a level
// (its register count differs per mode), asked of the runtime once each.
template <int MODE, bool SEG>
static int cj2_occ() {
  static int occ = [] {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, join_cj2_kernel<MODE, SEG>, kJThreads, 0) !=
            cudaSuccess ||
        b < 1) {
      (void)cudaGetLastError();
      b = 4;
    }
    return b;
  }();
  return occ;
}

static int cj2_blocks_per_sm(bool seg, int emit) {
  if (emit == kEmitCount) return seg ? cj2_occ<kModeCount, true>() : cj2_occ<kModeCount, false>();
  if (emit == kEmitKeys) return seg ? cj2_occ<kModeKeys, true>() : cj2_occ<kModeKeys, false>();
  return std::min(seg ? cj2_occ<kModeTableCount, true>() : cj2_occ<kModeTableCount, false>(),
                  seg ? cj2_occ<kModeTableWrite, true>() : cj2_occ<kModeTableWrite, false>());
}

// ---- pivot count kernel ------------------------------------------------------
//
// Count-only two-source column join, pivot rows only (join_count marks them):
// rows (a, ...) whose driver list is the other source's and whose probed
// list is a's, a long list with a bitmap.  Rows are sorted by a, so the
// pivot rows of one a form a run: pivot_runs_kernel finds every bitmapped
// value's run (two binary searches in the table's first column, one thread
// per value) and splits it into pieces of kPvPiece candidates.  A block (one
// per SM, 1024 threads) takes pieces in order from a device counter, copies
// the piece's bitmap into shared memory (again only when the value changes),
// and its 32 warps walk the piece's candidates as the cj2 kernel does, each
// candidate a bit test in shared memory instead of a probe of the bitmap in
// global memory.
constexpr int kPvThreads = 1024;
constexpr uint64_t kPvPiece = 1u << 19;  // candidates per piece

// First i in [lo, hi) with a[i] >= x (a sorted).
__device__ __forceinline__ uint64_t pv_lower(const uint32_t* a, uint64_t lo, uint64_t hi, uint32_t x) {
  while (lo < hi) {
    const uint64_t m = lo + (hi - lo) / 2;
    if (a[m] < x) lo = m + 1;
    else hi = m;
  }
  return lo;
}

// Per bitmap slot (a bitmapped value v): the rows of v in the table (first
// column pcol, true row count min(cap, *d_n)), their pivot candidates
// [cand_lo, cand_hi) and the number of pieces they make.
__global__ void pivot_runs_kernel(const uint32_t* __restrict__ bdir, uint32_t nv, const uint32_t* __restrict__ pcol,
                                  uint64_t cap, const uint64_t* __restrict__ d_n, const uint64_t* __restrict__ poffs,
                                  uint32_t nslots, uint64_t* __restrict__ run_lo, uint64_t* __restrict__ run_hi,
                                  uint64_t* __restrict__ cand_lo, uint64_t* __restrict__ cand_hi,
                                  uint64_t* __restrict__ pieces) {
  const uint64_t nrows = dev_size(cap, d_n);
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    const uint32_t slot = bdir[v];
    if (slot == kNoBitmap || slot >= nslots) continue;
    const uint64_t lo = pv_lower(pcol, 0, nrows, v);
    const uint64_t hi = pv_lower(pcol, lo, nrows, v + 1);
    const uint64_t cl = poffs[lo], ch = poffs[hi];
    run_lo[slot] = lo;
    run_hi[slot] = hi;
    cand_lo[slot] = cl;
    cand_hi[slot] = ch;
    pieces[slot] = (ch - cl + kPvPiece - 1) / kPvPiece;
  }
}

__global__ void __launch_bounds__(kPvThreads, 1) join_pivot_count_kernel(
    const uint32_t* __restrict__ dvals, const uint64_t* __restrict__ poffs, const uint32_t* __restrict__ beg,
    const uint64_t* __restrict__ run_lo, const uint64_t* __restrict__ run_hi,
    const uint64_t* __restrict__ cand_lo, const uint64_t* __restrict__ cand_hi,
    const uint64_t* __restrict__ piece_offs, uint32_t nslots, const uint32_t* __restrict__ bpool,
    uint32_t bwords, unsigned long long* __restrict__ queue, unsigned long long* __restrict__ d_out_n) {
  extern __shared__ __align__(16) uint32_t bm[];
  __shared__ uint64_t s_c0, s_c1, s_rl, s_rh;
  __shared__ uint32_t s_slot;
  __shared__ int s_done;
  __shared__ unsigned long long s_sum[kPvThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint64_t npieces = piece_offs[nslots];
  uint32_t loaded = kNoBitmap;
  unsigned long long counted = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned long long k = atomicAdd(queue, 1ull);
      s_done = k >= npieces;
      if (k < npieces) {
        // the slot of piece k: the last slot with piece_offs[slot] <= k
        uint32_t lo = 0, hi = nslots;
        while (hi - lo > 1) {
          const uint32_t m = lo + (hi - lo) / 2;
          if (piece_offs[m] <= k) lo = m;
          else hi = m;
        }
        const uint64_t j = k - piece_offs[lo];
        const uint64_t c0 = cand_lo[lo] + j * kPvPiece;
        s_slot = lo;
        s_c0 = c0;
        s_c1 = c0 + kPvPiece < cand_hi[lo] ? c0 + kPvPiece : cand_hi[lo];
        s_rl = run_lo[lo];
        s_rh = run_hi[lo];
      }
    }
    __syncthreads();
    if (s_done) break;
    const uint32_t slot = s_slot;
    const uint64_t c0 = s_c0, c1 = s_c1, rl = s_rl, rh = s_rh;
    if (slot != loaded) {
      // (word loads: a bitmap starts at slot * bwords words, not always on
      // a 16-byte boundary)
      const uint32_t* src = bpool + (uint64_t)slot * bwords;
      for (uint32_t i = threadIdx.x; i < bwords; i += kPvThreads) bm[i] = src[i];
      __syncthreads();
      loaded = slot;
    }
    // warp wid walks its share of the piece in rounds of 32 candidates; the
    // row of the round's first candidate is kept while the warp stays in it
    const uint64_t len = c1 - c0;
    const uint64_t wb = c0 + len * wid / (kPvThreads / 32);
    const uint64_t we = c0 + len * (wid + 1) / (kPvThreads / 32);
    if (wb < we) {
      uint64_t r0 = warp_partition_point(rl, rh, [&](uint64_t i) { return poffs[i] <= wb; }) - 1;
      uint64_t crow = ~0ull, c_off = 0, c_end = 0;
      uint32_t cbeg = 0;
      for (uint64_t base = wb; base < we; base += 32) {
        const uint64_t w = base + lane;
        const bool ok = w < we;
        if (r0 != crow) {
          crow = r0;
          c_off = poffs[r0];
          c_end = poffs[r0 + 1];
          cbeg = beg[r0];
        }
        uint32_t v = 0;
        if (base + 31 < c_end) {
          if (ok) v = dvals[cbeg + (uint32_t)(w - c_off)];
        } else if (ok) {
          const uint64_t r = gallop_row(poffs, r0, rh, w);
          v = dvals[beg[r] + (uint32_t)(w - poffs[r])];
        }
        if (ok) counted += (bm[v >> 5] >> (v & 31)) & 1u;
        // the next round's first row (the row of its first candidate)
        const uint64_t nb = base + 32;
        if (nb < we && nb >= c_end) r0 = gallop_row(poffs, r0, rh, nb);
      }
    }
    __syncthreads();  // (the bitmap and s_* are rewritten by the next piece)
  }
  // block total -> the level's count
  const unsigned long long ws = warp_sum(counted);
  if (lane == 0) s_sum[wid] = ws;
  __syncthreads();
  if (wid == 0) {
    unsigned long long t = lane < kPvThreads / 32 ? s_sum[lane] : 0ull;
    t = warp_sum(t);
    if (lane == 0 && t) atomicAdd(d_out_n, t);
  }
}

JoinWork join_count(const Launch& L, const LevelSpec& lv, const Table& in, Scratch& s) {
  JoinWork w;
  uint64_t* work = s.take<uint64_t>(in.n ? in.n : 1);
  w.offs = s.take<uint64_t>(in.n + 1);
  w.drv = s.take<uint8_t>(in.n ? in.n : 1);
  w.beg = s.take<uint32_t>(in.n ? in.n : 1);
  w.orange = s.take<uint2>(in.n ? in.n : 1);
  if (lv.kind == kColumnJoin && lv.nsrc == 2 && !lv.wide && (lv.src[0].t.bdir || lv.src[1].t.bdir))
    w.obm = s.take<uint32_t>(in.n ? in.n : 1);
  uint64_t* pwork = nullptr;
  if (w.obm && lv.pivot_src >= 0 && in.n) {
    pwork = s.take<uint64_t>(in.n);
    w.poffs = s.take<uint64_t>(in.n + 1);
  }
  if (in.n) {
    join_count_kernel<<<jgrid(in.n, L), kJThreads, 0, L.stream>>>(lv, in, work, w.drv,
                                                                          w.beg, w.orange, w.obm, pwork);
    SRDL_CUDA(cudaGetLastError());
    count_launches(1);
  }
  exclusive_scan_u64(L, work, in.n, w.offs, s);
  if (pwork) exclusive_scan_u64(L, pwork, in.n, w.poffs, s);
  return w;
}

size_t join_pivot_smem_bytes(uint32_t bwords) { return (size_t)bwords * 4; }

size_t join_pivot_scratch_bytes(uint32_t nslots) {
  return 7 * ((size_t)(nslots + 1) * 8 + 511) + scan_scratch_bytes(nslots) + 2048;
}

// The pivot rows' count (count mode; w.poffs set): the runs of the
// bitmapped values, their pieces, then one block per SM over the pieces.
static void join_pivot_count(const Launch& L, const LevelSpec& lv, const Table& in, const JoinWork& w,
                             unsigned long long* d_out_n, Scratch& s) {
  const int ps = lv.pivot_src, ds = 1 - ps;
  const SrcSpec& P = lv.src[ps];
  const SrcSpec& D = lv.src[ds];
  const uint32_t* dvals = D.prefix_slot < 0 ? D.t.roots : D.t.lo;
  const uint32_t nslots = lv.pivot_slots;
  if (!nslots || !P.t.dir_n) return;
  const size_t smem = join_pivot_smem_bytes(P.t.bwords);
  static size_t attr = 0;
  if (smem > attr) {
    SRDL_CUDA(cudaFuncSetAttribute(join_pivot_count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    attr = smem;
  }
  uint64_t* run_lo = s.take<uint64_t>(nslots);
  uint64_t* run_hi = s.take<uint64_t>(nslots);
  uint64_t* cand_lo = s.take<uint64_t>(nslots);
  uint64_t* cand_hi = s.take<uint64_t>(nslots);
  uint64_t* pieces = s.take<uint64_t>(nslots);
  uint64_t* piece_offs = s.take<uint64_t>(nslots + 1);
  unsigned long long* q = s.take<unsigned long long>(1);
  SRDL_CUDA(cudaMemsetAsync(pieces, 0, nslots * 8, L.stream));
  SRDL_CUDA(cudaMemsetAsync(q, 0, sizeof(unsigned long long), L.stream));
  const uint32_t nv = P.t.dir_n - 1;
  pivot_runs_kernel<<<(int)std::min<uint64_t>((nv + 255) / 256, (uint64_t)L.num_sms * 8), 256, 0, L.stream>>>(
      P.t.bdir, nv, in.col[P.prefix_slot], in.n, in.d_n, w.poffs, nslots, run_lo, run_hi, cand_lo, cand_hi,
      pieces);
  exclusive_scan_u64(L, pieces, nslots, piece_offs, s);
  join_pivot_count_kernel<<<L.num_sms, kPvThreads, smem, L.stream>>>(
      dvals, w.poffs, w.beg, run_lo, run_hi, cand_lo, cand_hi, piece_offs, nslots, P.t.bpool, P.t.bwords, q,
      d_out_n);
  SRDL_CUDA(cudaGetLastError());
  count_launches(2);
}

void join_expand(const Launch& L, const LevelSpec& lv, const Table& in, const JoinWork& w,
                 uint64_t total, Table* out_table, uint64_t* out_keys, uint64_t* d_out_n,
                 Scratch& s, const JoinDev* dev) {
  auto* cnt = reinterpret_cast<unsigned long long*>(d_out_n);
  if (w.poffs && lv.emit == kEmitCount) join_pivot_count(L, lv, in, w, cnt, s);
  if (total == 0) return;
  const JoinDev jd = dev ? *dev : JoinDev{};
  const int g = jgrid(total, L);
  const uint64_t warps = (uint64_t)g * (kJThreads / 32);
  const uint64_t chunk = ((total + warps - 1) / warps + 31) & ~uint64_t(31);
  Table out = out_table ? *out_table : Table{};
  if (lv.kind == kColumnJoin && lv.nsrc == 2 && lv.nfilt == 0 && !lv.wide) {
    // Persistent warps over a chunk queue: as many blocks as stay resident
    // (at most join_bpsm per SM), about eight chunks per warp for balance,
    // chunks of 64-4096 candidates (the table modes keep at most
    // kCj2MaxTableChunks per-chunk counts).
    const int occ = cj2_blocks_per_sm(lv.seg != 0, lv.emit);
    const int bpsm = std::max(1, std::min(occ, L.join_bpsm > 0 ? L.join_bpsm : 16));
    const uint64_t resident = (uint64_t)L.num_sms * bpsm * (kJThreads / 32);
    uint64_t chunk = (total + resident * 8 - 1) / (resident * 8);
    chunk = std::min<uint64_t>(std::max<uint64_t>(chunk, 64), (uint64_t)std::max(64, L.join_chunk));
    if (lv.emit == kEmitTable)
      chunk = std::max<uint64_t>(chunk, (total + kCj2MaxTableChunks - 1) / kCj2MaxTableChunks);
    chunk = (chunk + 31) & ~uint64_t(31);
    const uint64_t nchunks = (total + chunk - 1) / chunk;
    const uint64_t blocks = std::min<uint64_t>((uint64_t)L.num_sms * bpsm,
                                               (nchunks + kJThreads / 32 - 1) / (kJThreads / 32));
    const int gq = (int)std::max<uint64_t>(blocks, 1);
    unsigned long long* q = s.take<unsigned long long>(2);
    SRDL_CUDA(cudaMemsetAsync(q, 0, 2 * sizeof(unsigned long long), L.stream));
#define SRDL_CJ2(MODE, Q, CC)                                                                     \
  (lv.seg ? join_cj2_kernel<MODE, true><<<gq, kJThreads, 0, L.stream>>>(                           \
                lv, in, w.offs, w.drv, w.beg, w.orange, w.obm, total, chunk, Q, out, out_keys, cnt, \
                CC, jd)                                                                           \
          : join_cj2_kernel<MODE, false><<<gq, kJThreads, 0, L.stream>>>(                          \
                lv, in, w.offs, w.drv, w.beg, w.orange, w.obm, total, chunk, Q, out, out_keys, cnt, \
                CC, jd))
    if (lv.emit == kEmitCount) {
      SRDL_CJ2(kModeCount, q, nullptr);
      count_launches(1);
    } else if (lv.emit == kEmitKeys) {
      SRDL_CJ2(kModeKeys, q, nullptr);
      count_launches(1);
    } else {
      uint64_t* cc = s.take<uint64_t>(nchunks + 1);
      uint64_t* co = s.take<uint64_t>(nchunks + 1);
      // with the count on the device, chunks past it are never taken: zero
      // their counts so the scan over the capacity's chunks stays exact
      if (jd.d_total) SRDL_CUDA(cudaMemsetAsync(cc, 0, (nchunks + 1) * 8, L.stream));
      SRDL_CJ2(kModeTableCount, q, cc);
      SRDL_CUDA(cudaGetLastError());
      exclusive_scan_u64(L, cc, nchunks, co, s);
      SRDL_CUDA(cudaMemcpyAsync(d_out_n, co + nchunks, 8, cudaMemcpyDeviceToDevice, L.stream));
      SRDL_CJ2(kModeTableWrite, q + 1, co);
      count_launches(2);
    }
#undef SRDL_CJ2
    SRDL_CUDA(cudaGetLastError());
    return;
  }
  if (lv.kind == kCartesian && lv.nsrc == 2 && lv.src[0].out_slot >= 0 && lv.src[1].out_slot >= 0 &&
      !lv.wide) {
#define SRDL_CART2(MODE, WC)                                                                 \
  (lv.seg ? join_cart2_kernel<MODE, true><<<g, kJThreads, 0, L.stream>>>(                     \
                lv, in, w.offs, w.beg, w.orange, total, chunk, out, out_keys, cnt, WC, jd)      \
          : join_cart2_kernel<MODE, false><<<g, kJThreads, 0, L.stream>>>(                    \
                lv, in, w.offs, w.beg, w.orange, total, chunk, out, out_keys, cnt, WC, jd))
    if (lv.emit == kEmitCount) {
      SRDL_CART2(kModeCount, nullptr);
      count_launches(1);
    } else if (lv.emit == kEmitKeys) {
      SRDL_CART2(kModeKeys, nullptr);
      count_launches(1);
    } else {
      uint64_t* wc = s.take<uint64_t>(warps + 1);
      uint64_t* wo = s.take<uint64_t>(warps + 1);
      SRDL_CART2(kModeTableCount, wc);
      SRDL_CUDA(cudaGetLastError());
      exclusive_scan_u64(L, wc, warps, wo, s);
      SRDL_CUDA(cudaMemcpyAsync(d_out_n, wo + warps, 8, cudaMemcpyDeviceToDevice, L.stream));
      SRDL_CART2(kModeTableWrite, wo);
      count_launches(2);
    }
#undef SRDL_CART2
    SRDL_CUDA(cudaGetLastError());
    return;
  }
#define SRDL_EXP(MODE, WC)                                                                    \
  (lv.seg ? join_expand_kernel<MODE, true><<<g, kJThreads, 0, L.stream>>>(                       \
                lv, in, w.offs, w.drv, w.beg, total, chunk, out, out_keys, cnt, WC, jd)          \
          : join_expand_kernel<MODE, false><<<g, kJThreads, 0, L.stream>>>(                      \
                lv, in, w.offs, w.drv, w.beg, total, chunk, out, out_keys, cnt, WC, jd))
  if (lv.emit == kEmitCount) {
    SRDL_EXP(kModeCount, nullptr);
    count_launches(1);
  } else if (lv.emit == kEmitKeys) {
    SRDL_EXP(kModeKeys, nullptr);
    count_launches(1);
  } else {
    uint64_t* wc = s.take<uint64_t>(warps + 1);
    uint64_t* wo = s.take<uint64_t>(warps + 1);
    SRDL_EXP(kModeTableCount, wc);
    SRDL_CUDA(cudaGetLastError());
    exclusive_scan_u64(L, wc, warps, wo, s);
    SRDL_CUDA(cudaMemcpyAsync(d_out_n, wo + warps, 8, cudaMemcpyDeviceToDevice, L.stream));
    SRDL_EXP(kModeTableWrite, wo);
    count_launches(2);
  }
#undef SRDL_EXP
  SRDL_CUDA(cudaGetLastError());
}

}  // namespace srdl
