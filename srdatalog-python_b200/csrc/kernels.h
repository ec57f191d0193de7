// kernels.h -- host-side launch wrappers for the srdl device kernels.
//
// Every wrapper is stream-ordered and allocation-free: temporaries come
// from a caller-provided scratch region whose size the matching
// *_scratch_bytes() function reports.  Sizes that the host must know
// (unique counts, join output counts) are written to device memory; the
// caller decides when to read them back.
#pragma once

#include "common.cuh"

namespace srdl {

struct Launch {
  cudaStream_t stream = 0;
  int num_sms = 148;
  uint32_t* d_err = nullptr;  // device error word (bounded-wait failures etc.)
  int radix_bits = 8;         // widest radix-sort digit (1..8): passes = ceil(key bits / this)
  int join_bpsm = 16;         // join launches: at most this many blocks per SM (work per warp)
  int join_chunk = 4096;      // two-source column join: largest chunk of candidates a warp takes
};

// Bump allocator over a caller-provided scratch region.  Every piece starts
// on a 256-byte boundary of the address space (asynchronous 16-byte copies
// need aligned sources), whatever the alignment of the region itself.
struct Scratch {
  char* base = nullptr;
  size_t cap = 0, used = 0;
  template <typename T>
  T* take(size_t count) {
    const size_t pad = (256 - ((uintptr_t)(base + used) & 255)) & 255;
    size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    SRDL_REQUIRE(used + pad + bytes <= cap, kErrCapacity, "scratch region too small");
    T* p = reinterpret_cast<T*>(base + used + pad);
    used += pad + bytes;
    return p;
  }
};

// Ask for the largest shared-memory carveout for a kernel (once per kernel):
// the default split caps blocks of the shared-memory-heavy kernels per SM.
template <typename K>
inline void prefer_shared(K* kernel) {
  static bool done = false;
  if (!done) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxShared);
    done = true;
  }
}

// Process-wide count of kernels this library has launched (bench evidence).
void count_launches(int k);
uint64_t launches_total();

// Largest value in d[0..n) -> *d_max (uint32; 0 when n == 0).
void max_u32(const Launch& L, const uint32_t* d, uint64_t n, uint32_t* d_max);

// ---------------------------------------------------------------- sort
// Bits needed to hold every value of the active domain (max value < 2^bits).
int value_bits(uint32_t max_value);

// Scratch needed by sort_dedup for n input keys.
size_t sort_scratch_bytes(uint64_t n, int dom_bits);

// Radix-sorts n uint64 keys (both 32-bit halves < 2^dom_bits; halves
// swapped first when `swap` is set) and writes the distinct keys, in
// ascending order, into `out`.  When `full` is given, keys present in the
// sorted unique array full[0..n_full) are dropped as well (fused
// DELTA = unique(NEW) - FULL); so are keys present in head[0..n_head) (the
// HEAD segment of a Device2LevelIndex FULL).  The output count goes to
// *d_nout.  `out` needs room for n keys and may alias `in`.
void sort_dedup(const Launch& L, const uint64_t* in, uint64_t n, int dom_bits, bool swap,
                const uint64_t* full, uint64_t n_full, uint64_t* out, uint64_t* d_nout,
                Scratch& s, const uint64_t* head = nullptr, uint64_t n_head = 0);

// ------------------------------------------------------------- set ops
size_t diff_scratch_bytes(uint64_t n);
// out = a - b for sorted unique arrays; *d_nout = |out|; out needs room for na.
void set_difference(const Launch& L, const uint64_t* a, uint64_t na, const uint64_t* b,
                    uint64_t nb, uint64_t* out, uint64_t* d_nout, Scratch& s);

// out = a U b (sorted unique, disjoint) by merge path; out needs na+nb.
void merge_disjoint(const Launch& L, const uint64_t* a, uint64_t na, const uint64_t* b,
                    uint64_t nb, uint64_t* out);

// Device loop: out = a U b with the counts on the device (*d_na, *d_nb; na_cap
// and nb_cap are capacities); *d_nout = the merged count; a merged count
// above out_cap sets *d_overflow and writes nothing.
void merge_disjoint_dev(const Launch& L, const uint64_t* a, uint64_t na_cap, const uint64_t* d_na,
                        const uint64_t* b, uint64_t nb_cap, const uint64_t* d_nb, uint64_t* out,
                        uint64_t out_cap, uint64_t* d_nout, unsigned int* d_overflow);

// Scratch sort_dedup_dev needs for `cap` keys against a FULL of full_cap.
size_t sort_dev_scratch_bytes(uint64_t cap, uint64_t full_cap, int bits);

// Sets, once, the kernel attributes the device loop's kernels use (a graph
// capture must not be the first to set them).
void warm_device_loop_kernels(int bits);
void warm_merge_kernels();

// sort_dedup with the input count on the device (device loop): `cap` keys of
// room in `in`, *d_n present; FULL (room full_cap, count *d_n_full, may be
// null) is subtracted; `out` has room for out_cap keys (more kept keys
// raise *d_overflow and are not written; *d_nout is still the full count).
// No host decision depends on the counts.
void sort_dedup_dev(const Launch& L, const uint64_t* in, uint64_t cap, const uint64_t* d_n,
                    int bits, const uint64_t* full, uint64_t full_cap, const uint64_t* d_n_full,
                    uint64_t* out, uint64_t out_cap, uint64_t* d_nout, unsigned int* d_overflow,
                    Scratch& s);

// Trie view pieces for a sorted unique key array (with d_n: n is a capacity
// and the count is on the device).
size_t roots_scratch_bytes(uint64_t n);
void build_lo(const Launch& L, const uint64_t* keys, uint64_t n, uint32_t* lo,
              const uint64_t* d_n = nullptr);
void build_dir(const Launch& L, const uint64_t* keys, uint64_t n, uint32_t* dir, uint32_t dir_n,
               const uint64_t* d_n = nullptr);
void build_roots(const Launch& L, const uint64_t* keys, uint64_t n, uint32_t* roots,
                 uint64_t* d_nroots, Scratch& s, const uint64_t* d_n = nullptr);

// Hash tables for the child lists longer than `min_len` of a dense-directory
// trie.  Plan: sizes[v] = slots for value v (0 = no table), offs = exclusive
// scan (dir_n entries, offs[dir_n-1] = total slots).  Build: hdir[v] = first
// slot or kNoHash; every child of a hashed list is inserted into `pool`,
// which the caller pre-fills with 0xff bytes.
// Bitmaps of long child lists.  bitmap_plan: cnt[k] = values whose child
// list has at least (kBitmapMinLen << k) entries, k < kBitmapLevels.  bitmap_build:
// bdir[v] = a fresh slot for lists of at least min_len entries (kNoBitmap
// otherwise); every key (v, c) of such a list sets bit c of v's bitmap
// (pool zeroed by the caller); *d_slots receives the slot count.
constexpr int kBitmapLevels = 10;
constexpr uint32_t kBitmapMinLen = 128;
void bitmap_plan(const Launch& L, const uint32_t* dir, uint32_t dir_n, unsigned long long* cnt);
void bitmap_build(const Launch& L, const uint64_t* keys, uint64_t n, const uint32_t* dir,
                  uint32_t dir_n, uint32_t min_len, uint32_t* bdir, uint32_t* pool, uint32_t bwords,
                  unsigned int* d_slots);

size_t child_hash_scratch_bytes(uint32_t dir_n);
void child_hash_plan(const Launch& L, const uint32_t* dir, uint32_t dir_n, uint32_t min_len,
                     uint64_t* sizes, uint64_t* offs, Scratch& s);
void child_hash_build(const Launch& L, const uint64_t* keys, uint64_t n, const uint32_t* dir,
                      uint32_t dir_n, const uint64_t* sizes, const uint64_t* offs, uint32_t* hdir,
                      uint32_t* pool);

// last[j] = max(last[j], base + *iter_dev) for every instance j (values
// [bounds[j], bounds[j+1]), j < k) with a key in the sorted keys[0..n), n =
// min(*n_dev, cap) when n_dev is given, else cap; iter_dev may be null.
void instance_mark(const Launch& L, const uint64_t* keys, uint64_t cap, const uint64_t* n_dev,
                   const uint32_t* bounds, uint32_t k, uint32_t base, const unsigned long long* iter_dev,
                   uint32_t* last);

// pos[j] = first row of the sorted keys whose high word is >= bounds[j].
void bounds_positions(const Launch& L, const uint64_t* keys, uint64_t n, const uint32_t* bounds,
                      uint64_t n_bounds, uint64_t* pos);

// Keys whose first declared column (the key's low word when `col0_lo`, else
// its high word) is owned by shard `dest` of `world` (shard_owner), in
// order, to out; their count to *d_nout.
size_t shard_select_scratch_bytes(uint64_t n);
void shard_select(const Launch& L, const uint64_t* keys, uint64_t n, bool col0_lo, uint32_t world,
                  uint32_t dest, uint64_t* out, uint64_t* d_nout, Scratch& s);

// Ternary relations: keys pack a tuple (x0, x1, x2) `bits` apiece into P and
// split it at `half` bits, (P >> half) << 32 | (P mod 2^half).
// repack3: the tuples of `in` with their columns reordered, out column j =
// in column sel[j] (out is not sorted).
void repack3(const Launch& L, const uint64_t* in, uint64_t n, int bits, int half, const int sel[3],
             uint64_t* out);
// split3: for sorted unique packed keys, pair_keys = the distinct (x0, x1) as
// x0 << 32 | x1 (room for n; the count goes to *d_npairs) and row_keys[i] =
// (position of row i's pair in pair_keys) << 32 | x2.  Both come out sorted.
size_t split3_scratch_bytes(uint64_t n);
void split3(const Launch& L, const uint64_t* keys, uint64_t n, int bits, int half,
            uint64_t* pair_keys, uint64_t* row_keys, uint64_t* d_npairs, Scratch& s);

// Swap the two 32-bit halves of every key (index permutation (1,0) <-> (0,1)).
void swap_halves(const Launch& L, const uint64_t* in, uint64_t n, uint64_t* out);

// Exclusive scan of n uint64 values; out has n+1 entries (out[n] = total).
size_t scan_scratch_bytes(uint64_t n);
void exclusive_scan_u64(const Launch& L, const uint64_t* in, uint64_t n, uint64_t* out,
                        Scratch& s);

// ---------------------------------------------------------------- join
constexpr int kMaxSlots = 8;
constexpr int kMaxSrc = 4;
constexpr int kMaxFilt = 4;

enum LevelKind : int { kColumnJoin = 0, kCartesian = 1, kScan = 2 };
enum EmitKind : int { kEmitTable = 0, kEmitKeys = 1, kEmitCount = 2 };
enum FiltOp : int { kNe = 0, kEq = 1, kLt = 2, kLe = 3, kGt = 4, kGe = 5 };

// Sources over a ternary relation read two binary views of it, built per
// column order (c0, c1, c2): the pair index P = the distinct (c0, c1) as
// keys, and the row index R = (position of the row's (c0, c1) in P) << 32 | c2.
// With no or one bound column a source reads P like a binary relation
// (kSrcPlain).  kSrcPair: c0 and c1 bound (prefix_slot, prefix_slot2); the
// list is R's children of the pair's position.  kSrcRows: the rows of R under
// P's children of c0 (prefix_slot; all rows when -1), binding c1 from P
// (out_slot) and c2 from R (out_slot2).
enum SrcMode : int { kSrcPlain = 0, kSrcPair = 1, kSrcRows = 2 };

struct SrcSpec {
  TrieView t;
  int prefix_slot = -1;  // binding slot holding the prefix value, -1: no prefix (roots)
  int out_slot = -1;     // cartesian: slot this source binds (-1: existence only)
  int mode = kSrcPlain;
  int prefix_slot2 = -1;  // kSrcPair: slot of the second bound column
  int out_slot2 = -1;     // kSrcRows: slot bound to c2
  TrieView pair;          // kSrcPair / kSrcRows: the pair index P (t is R)
};

struct FiltSpec {
  int a_slot = -1, b_slot = -1;  // -1: use the constant
  uint32_t a_const = 0, b_const = 0;
  int op = kNe;
  // Negation (MIR `negation`, mir/types.py:189): keep the binding iff the
  // tuple (a) -- (a, b) when neg_n is 2 -- is not a key prefix of `neg`
  // (a ternary relation is probed through its pair view in the negation's
  // column order).  Values come from slots or constants (a_const, b_const).
  bool negation = false;
  int neg_n = 1;
  TrieView neg;
  // Shard filter: keep the binding iff shard_owner(a, shard_world) == b_const
  // (0: not a shard filter).
  uint32_t shard_world = 0;
};

struct LevelSpec {
  int kind = kColumnJoin;
  int nsrc = 0;
  SrcSpec src[kMaxSrc];
  int cj_slot = -1;                     // column join: slot of the joined variable
  int scan_slot[3] = {-1, -1, -1};      // scan: slots for index columns 0, 1 (and 2: kSrcRows)
  int wide = 0;                         // a source is kSrcPair / kSrcRows: generic kernels only
  int nfilt = 0;
  FiltSpec filt[kMaxFilt];
  int n_in_slots = 0;                   // slots bound by the input table
  int emit = kEmitTable;
  int key_slot[4] = {-1, -1, -1, -1};   // emit keys: slots of the target index columns
  int key_arity = 2;
  // emit keys of arity 3-4: columns packed pack_bits apiece, split at pack_half
  int pack_bits = 0, pack_half = 0;
  // Count mode only: also add every counted binding to grp_counts[g] for the
  // group g with grp_bounds[g] <= (value of slot 0) < grp_bounds[g+1].
  const uint32_t* grp_bounds = nullptr;  // n_groups + 1 sorted entries
  uint32_t n_groups = 0;
  unsigned long long* grp_counts = nullptr;
  // Count-only two-source column joins: rows whose driver is the other
  // source's list and whose probed list -- source pivot_src's, indexed by
  // the table's first (sorted) column -- has a bitmap and at least
  // pivot_min values are counted by the pivot kernel (the bitmap of the
  // rows' common first value held in shared memory) instead of cj2.
  int pivot_src = -1;
  uint32_t pivot_min = 0;
  uint32_t pivot_slots = 0;  // bitmaps of the pivot source
  // Sharded work: expand only segments seg_rank, seg_rank + seg_world, ...
  // of `seg` work items each (seg a multiple of 32; 0: every item).
  uint64_t seg = 0;
  uint32_t seg_world = 1, seg_rank = 0;
};

struct Table {
  uint32_t* col[kMaxSlots] = {};
  uint64_t n = 0;                 // rows (or row capacity when d_n is set)
  const uint64_t* d_n = nullptr;  // device-resident row count <= n, or null
};

size_t join_work_scratch_bytes(uint64_t rows);
// Pass 1: per input row, the number of work items (candidates) it expands
// to.  Writes offsets[0..rows] (exclusive scan) and the total into
// *d_total (= offsets[rows]).  Scratch keeps per-row driver info that
// join_expand reads, so the same Scratch must be passed to both.
struct JoinWork {
  uint64_t* offs = nullptr;  // rows + 1
  uint8_t* drv = nullptr;    // column join: driver source per row
  uint32_t* beg = nullptr;   // column join: driver list begin per row
  uint2* orange = nullptr;   // two-source column join: the other list [x, y) per row
  uint32_t* obm = nullptr;   // two-source column join: bitmap slot of the other list, or kNoBitmap
  uint64_t* poffs = nullptr; // pivot rows (lv.pivot_src): prefix sums of their candidates, rows + 1
};
JoinWork join_count(const Launch& L, const LevelSpec& lv, const Table& in, Scratch& s);

// Shared memory the pivot kernel needs for one bitmap of `bwords` words;
// levels whose bitmaps need more than kPivotSmemMax keep the cj2 kernel.
size_t join_pivot_smem_bytes(uint32_t bwords);
// Scratch the pivot pass adds to a level's expand scratch.
size_t join_pivot_scratch_bytes(uint32_t nslots);
constexpr size_t kPivotSmemMax = 200 * 1024;

// Pass 2: expands `total` work items (all of the count pass's items, or
// with lv.seg set this shard's segments of them, total = seg_owned(...));
// surviving bindings are appended to `out_table` (emit table, in input
// order: the table stays sorted), to `out_keys` (emit keys, any order) or
// counted (emit count) via *d_out_n, which the caller zeroes.  Output
// capacity = total.  The scratch for a level of `total` candidates comes
// from join_expand_scratch_bytes(L, total).
size_t join_expand_scratch_bytes(const Launch& L, uint64_t total);

// Device loop: the candidate count is on the device (d_total, the count
// pass's offs[rows]); `total` is then its capacity.  A count above the
// capacity, or emitted keys beyond out_cap (emit keys: appended after the
// keys already at *d_out_n), set *d_overflow; nothing is written out of
// bounds.
struct JoinDev {
  const uint64_t* d_total = nullptr;
  uint64_t out_cap = 0;
  unsigned int* d_overflow = nullptr;
  // emit keys: the output buffer is this launch's alone (one rule fills the
  // relation's NEW), so a filter-free product may write each key at its
  // candidate index and set *d_out_n to the count
  bool exact_ok = false;
};

void join_expand(const Launch& L, const LevelSpec& lv, const Table& in, const JoinWork& w,
                 uint64_t total, Table* out_table, uint64_t* out_keys, uint64_t* d_out_n,
                 Scratch& s, const JoinDev* dev = nullptr);

// Work items of shard `rank` among `world` when `total` items are dealt out
// in segments of `seg` (segment i goes to shard i mod world).
inline uint64_t seg_owned(uint64_t total, uint64_t seg, uint64_t world, uint64_t rank) {
  const uint64_t round = seg * world, full = total / round, rem = total - full * round;
  const uint64_t lo = rank * seg;
  return full * seg + (rem > lo ? (rem - lo < seg ? rem - lo : seg) : 0);
}


}  // namespace srdl
