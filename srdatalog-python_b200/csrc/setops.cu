// setops.cu -- merge-path union, set difference, trie views, scans.
//
// merge_disjoint replaces DSAI::merge (thrust::merge + set_union on root
// keys, RT/gpu/device_sorted_array_index.ipp:709-847): FULL and DELTA are
// disjoint sorted arrays, so FULL U DELTA is a plain merge whose output size
// is known up front.  A first launch finds the merge-path split point of
// every 2048-element output tile (one binary search per tile boundary); then
// each block owns one output tile, stages both input slices in shared memory
// with coalesced loads, merges 8 outputs per thread and writes the tile back
// coalesced.
//
// set_difference replaces thrust::set_difference on the zipped columns
// (.ipp:1104-1107) and the binary-probe variant (.ipp:933-1041): every
// element of `a` is probed in the slice of `b` that its block's key range
// can reach, then the survivors are compacted in order.
#include <algorithm>
#include <atomic>

#include "compact.cuh"
#include "kernels.h"

namespace srdl {

static std::atomic<uint64_t> g_launches{0};
void count_launches(int k) { g_launches.fetch_add((uint64_t)k, std::memory_order_relaxed); }
uint64_t launches_total() { return g_launches.load(std::memory_order_relaxed); }

constexpr int kMgThreads = 256;
constexpr int kMgItems = 8;
constexpr int kMgTile = kMgThreads * kMgItems;

// Number of elements taken from `a` among the first `diag` merged outputs
// (ties resolve towards `a`).
__device__ __forceinline__ uint64_t merge_path(const uint64_t* a, uint64_t na, const uint64_t* b,
                                               uint64_t nb, uint64_t diag) {
  uint64_t lo = diag > nb ? diag - nb : 0;
  uint64_t hi = diag < na ? diag : na;
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (a[mid] <= b[diag - 1 - mid]) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Split search for every output tile, one thread per tile boundary.  The
// splits are parked in the output itself: tile t's start split goes to
// out[t*kMgTile] and its end split to out[t*kMgTile + 1] (the last tile's end
// split is na and is not stored).  Only tile t's block reads or writes tile
// t's slots, and it reads them before writing its outputs, so no scratch
// buffer is needed.
// Device loop: na / nb are capacities and the counts are *d_na / *d_nb;
// tiles past the merged count do nothing (the last real tile ends at na).
// A merged count above out_cap raises *d_overflow and merges nothing.
struct MergeDev {
  const uint64_t* d_na = nullptr;
  const uint64_t* d_nb = nullptr;
  uint64_t out_cap = 0;
  uint64_t* d_nout = nullptr;        // receives na + nb
  unsigned int* d_overflow = nullptr;
};

__device__ __forceinline__ bool merge_dev_sizes(const MergeDev& md, uint64_t& na, uint64_t& nb) {
  na = dev_size(na, md.d_na);
  nb = dev_size(nb, md.d_nb);
  return !(md.out_cap && na + nb > md.out_cap);
}

__global__ void merge_split_kernel(const uint64_t* __restrict__ a, uint64_t na,
                                   const uint64_t* __restrict__ b, uint64_t nb, uint64_t tiles,
                                   uint64_t* __restrict__ out, MergeDev md) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (t >= tiles) return;
  if (!merge_dev_sizes(md, na, nb)) {
    if (t == 0 && md.d_overflow) atomicExch(md.d_overflow, 1u);
    return;
  }
  if (t == 0 && md.d_nout) *md.d_nout = na + nb;
  const uint64_t diag = t * kMgTile;
  if (diag >= na + nb) return;
  const uint64_t s = merge_path(a, na, b, nb, diag);
  out[diag] = s;
  if (t > 0) out[diag - kMgTile + 1] = s;
}

// Shared-memory index with one pad word per 16 keys: threads that walk the
// tile 8 (or about 4) keys apart then hit different banks.
__device__ __forceinline__ int mg_pad(int p) { return p + (p >> 4); }
constexpr int kMgPadded = kMgTile + kMgTile / 16;

__global__ void __launch_bounds__(kMgThreads) merge_kernel(const uint64_t* __restrict__ a,
                                                           uint64_t na,
                                                           const uint64_t* __restrict__ b,
                                                           uint64_t nb,
                                                           uint64_t* __restrict__ out, MergeDev md) {
  __shared__ uint64_t sin[kMgPadded];
  __shared__ uint64_t sout[kMgPadded];
  __shared__ uint64_t split[2];
  if (!merge_dev_sizes(md, na, nb)) return;
  const uint64_t total = na + nb;
  // one output tile per block (host sizes); with the counts on the device
  // the capped grid walks the tiles
  for (uint64_t tile = blockIdx.x;; tile += gridDim.x) {
    const uint64_t d0 = tile * kMgTile;
    if (d0 >= total) return;
    const uint64_t d1 = d0 + kMgTile < total ? d0 + kMgTile : total;
    const bool last = d1 == total;
    if (threadIdx.x == 0) split[0] = out[d0];
    if (threadIdx.x == 1) split[1] = last ? na : out[d0 + 1];
    __syncthreads();
    const uint64_t i0 = split[0], i1 = split[1];
    const uint64_t j0 = d0 - i0, j1 = d1 - i1;
    const int la = (int)(i1 - i0), lb = (int)(j1 - j0), lt = la + lb;
    for (int k = threadIdx.x; k < lt; k += kMgThreads)
      sin[mg_pad(k)] = k < la ? a[i0 + k] : b[j0 + k - la];
    __syncthreads();
    const int ld = threadIdx.x * kMgItems;
    if (ld < lt) {
      int lo = ld > lb ? ld - lb : 0, hi = ld < la ? ld : la;
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (sin[mg_pad(mid)] <= sin[mg_pad(la + ld - 1 - mid)]) lo = mid + 1;
        else hi = mid;
      }
      int i = lo, j = ld - lo;
      uint64_t va = i < la ? sin[mg_pad(i)] : 0, vb = j < lb ? sin[mg_pad(la + j)] : 0;
#pragma unroll
      for (int k = 0; k < kMgItems; k++) {
        if (ld + k >= lt) break;
        const bool take_a = (j >= lb) || (i < la && va <= vb);
        sout[mg_pad(ld + k)] = take_a ? va : vb;
        if (take_a) {
          i++;
          va = i < la ? sin[mg_pad(i)] : 0;
        } else {
          j++;
          vb = j < lb ? sin[mg_pad(la + j)] : 0;
        }
      }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < lt; k += kMgThreads) out[d0 + k] = sout[mg_pad(k)];
    __syncthreads();  // the shared tiles are refilled for the next tile
  }
}

void merge_disjoint(const Launch& L, const uint64_t* a, uint64_t na, const uint64_t* b,
                    uint64_t nb, uint64_t* out) {
  const uint64_t total = na + nb;
  if (total == 0) return;
  const uint64_t blocks = (total + kMgTile - 1) / kMgTile;
  SRDL_REQUIRE(blocks < (1ull << 31), kErrCapacity, "merge: too many rows");
  prefer_shared(merge_kernel);
  merge_split_kernel<<<(unsigned)((blocks + 255) / 256), 256, 0, L.stream>>>(a, na, b, nb, blocks,
                                                                             out, MergeDev{});
  merge_kernel<<<(unsigned)blocks, kMgThreads, 0, L.stream>>>(a, na, b, nb, out, MergeDev{});
  SRDL_CUDA(cudaGetLastError());
  count_launches(2);
}

void warm_merge_kernels() { prefer_shared(merge_kernel); }

void merge_disjoint_dev(const Launch& L, const uint64_t* a, uint64_t na_cap, const uint64_t* d_na,
                        const uint64_t* b, uint64_t nb_cap, const uint64_t* d_nb, uint64_t* out,
                        uint64_t out_cap, uint64_t* d_nout, unsigned int* d_overflow) {
  const uint64_t blocks = std::max<uint64_t>(1, (na_cap + nb_cap + kMgTile - 1) / kMgTile);
  SRDL_REQUIRE(blocks < (1ull << 31), kErrCapacity, "merge: too many rows");
  MergeDev md{d_na, d_nb, out_cap, d_nout, d_overflow};
  prefer_shared(merge_kernel);
  merge_split_kernel<<<(unsigned)((blocks + 255) / 256), 256, 0, L.stream>>>(a, na_cap, b, nb_cap,
                                                                             blocks, out, md);
  // a capped grid (the tiles are walked): blocks beyond the true count would
  // only be scheduled to exit
  const uint64_t mgrid = std::min<uint64_t>(blocks, (uint64_t)L.num_sms * 8);
  merge_kernel<<<(unsigned)mgrid, kMgThreads, 0, L.stream>>>(a, na_cap, b, nb_cap, out, md);
  SRDL_CUDA(cudaGetLastError());
  count_launches(2);
}

size_t diff_scratch_bytes(uint64_t n) { return cp_scratch_bytes(n); }

void set_difference(const Launch& L, const uint64_t* a, uint64_t na, const uint64_t* b,
                    uint64_t nb, uint64_t* out, uint64_t* d_nout, Scratch& s) {
  DedupDiffSel<uint64_t> sel{a, 32, false, b, nb, out};
  compact_diff(L, sel, na, d_nout, s);
}

__global__ void lo_kernel(const uint64_t* __restrict__ keys, uint64_t n, uint32_t* __restrict__ lo,
                          const uint64_t* d_n) {
  n = dev_size(n, d_n);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    lo[i] = (uint32_t)keys[i];
}

__global__ void dir_kernel(const uint64_t* __restrict__ keys, uint64_t n, uint32_t* __restrict__ dir,
                           uint32_t dir_n, const uint64_t* d_n) {
  n = dev_size(n, d_n);
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < dir_n;
       v += (uint64_t)gridDim.x * blockDim.x)
    dir[v] = (uint32_t)lower_bound_u64(keys, 0, n, v << 32);
}

__global__ void swap_kernel(const uint64_t* __restrict__ in, uint64_t n, uint64_t* __restrict__ out) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t k = in[i];
    out[i] = (k << 32) | (k >> 32);
  }
}

static int grid_for(uint64_t n, int sms) {
  uint64_t g = (n + 255) / 256;
  uint64_t cap = (uint64_t)sms * 16;
  if (g > cap) g = cap;
  return g ? (int)g : 1;
}

void build_lo(const Launch& L, const uint64_t* keys, uint64_t n, uint32_t* lo, const uint64_t* d_n) {
  if (!n) return;
  lo_kernel<<<grid_for(n, L.num_sms), 256, 0, L.stream>>>(keys, n, lo, d_n);
  SRDL_CUDA(cudaGetLastError());
  count_launches(1);
}

void build_dir(const Launch& L, const uint64_t* keys, uint64_t n, uint32_t* dir, uint32_t dir_n,
               const uint64_t* d_n) {
  if (!dir_n) return;
  dir_kernel<<<grid_for(dir_n, L.num_sms), 256, 0, L.stream>>>(keys, n, dir, dir_n, d_n);
  SRDL_CUDA(cudaGetLastError());
  count_launches(1);
}

size_t roots_scratch_bytes(uint64_t n) { return cp_scratch_bytes(n); }

void build_roots(const Launch& L, const uint64_t* keys, uint64_t n, uint32_t* roots,
                 uint64_t* d_nroots, Scratch& s, const uint64_t* d_n) {
  RootSel sel{keys, roots};
  compact(L, sel, n, d_nroots, s, d_n);
}

void swap_halves(const Launch& L, const uint64_t* in, uint64_t n, uint64_t* out) {
  if (!n) return;
  swap_kernel<<<grid_for(n, L.num_sms), 256, 0, L.stream>>>(in, n, out);
  SRDL_CUDA(cudaGetLastError());
  count_launches(1);
}

// ---- ternary relations: column orders and the pair / row views ---------------
// A ternary tuple (x0, x1, x2) in some column order is one uint64 key: P =
// x0 << 2b | x1 << b | x2, stored split at `half` bits as
// (P >> half) << 32 | (P mod 2^half), so key order is tuple order.

__device__ __forceinline__ uint64_t tern_unsplit(uint64_t k, int half) {
  return ((k >> 32) << half) | (k & ((1ull << half) - 1));
}

__device__ __forceinline__ uint64_t tern_split(uint64_t p, int half) {
  return ((p >> half) << 32) | (p & ((1ull << half) - 1));
}

__global__ void repack3_kernel(const uint64_t* __restrict__ in, uint64_t n, int bits, int half,
                               int s0, int s1, int s2, uint64_t* __restrict__ out) {
  const uint64_t mb = (1ull << bits) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = tern_unsplit(in[i], half);
    const uint64_t x[3] = {p >> (2 * bits), (p >> bits) & mb, p & mb};
    out[i] = tern_split((x[s0] << (2 * bits)) | (x[s1] << bits) | x[s2], half);
  }
}

// flag[i] = 1 where row i starts a new (x0, x1) pair
__global__ void split3_flag_kernel(const uint64_t* __restrict__ keys, uint64_t n, int bits, int half,
                                   uint64_t* __restrict__ flag) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t pr = tern_unsplit(keys[i], half) >> bits;
    flag[i] = (i == 0 || (tern_unsplit(keys[i - 1], half) >> bits) != pr) ? 1 : 0;
  }
}

// row i's pair number = pairs started before it (excl[i]) + flag[i] - 1
__global__ void split3_write_kernel(const uint64_t* __restrict__ keys, uint64_t n, int bits,
                                    int half, const uint64_t* __restrict__ flag,
                                    const uint64_t* __restrict__ excl, uint64_t* __restrict__ pair_keys,
                                    uint64_t* __restrict__ row_keys) {
  const uint64_t mb = (1ull << bits) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t p = tern_unsplit(keys[i], half);
    const uint64_t g = excl[i] + flag[i] - 1;
    row_keys[i] = (g << 32) | (p & mb);
    if (flag[i]) pair_keys[g] = ((p >> (2 * bits)) << 32) | ((p >> bits) & mb);
  }
}

void repack3(const Launch& L, const uint64_t* in, uint64_t n, int bits, int half, const int sel[3],
             uint64_t* out) {
  if (!n) return;
  SRDL_REQUIRE(bits >= 1 && 3 * bits <= 64 && half >= 1 && half <= 32, kErrArg, "repack3: bad packing");
  for (int j = 0; j < 3; j++) SRDL_REQUIRE(sel[j] >= 0 && sel[j] < 3, kErrArg, "repack3: bad order");
  repack3_kernel<<<grid_for(n, L.num_sms), 256, 0, L.stream>>>(in, n, bits, half, sel[0], sel[1],
                                                               sel[2], out);
  SRDL_CUDA(cudaGetLastError());
  count_launches(1);
}

size_t split3_scratch_bytes(uint64_t n) {
  return 2 * (((n + 1) * 8 + 255) & ~size_t(255)) + scan_scratch_bytes(n) + 1024;
}

void split3(const Launch& L, const uint64_t* keys, uint64_t n, int bits, int half,
            uint64_t* pair_keys, uint64_t* row_keys, uint64_t* d_npairs, Scratch& s) {
  if (!n) {
    SRDL_CUDA(cudaMemsetAsync(d_npairs, 0, 8, L.stream));
    return;
  }
  SRDL_REQUIRE(bits >= 1 && 3 * bits <= 64 && half >= 1 && half <= 32, kErrArg, "split3: bad packing");
  uint64_t* flag = s.take<uint64_t>(n + 1);
  uint64_t* excl = s.take<uint64_t>(n + 1);
  split3_flag_kernel<<<grid_for(n, L.num_sms), 256, 0, L.stream>>>(keys, n, bits, half, flag);
  SRDL_CUDA(cudaGetLastError());
  exclusive_scan_u64(L, flag, n, excl, s);
  split3_write_kernel<<<grid_for(n, L.num_sms), 256, 0, L.stream>>>(keys, n, bits, half, flag, excl,
                                                                    pair_keys, row_keys);
  SRDL_CUDA(cudaGetLastError());
  SRDL_CUDA(cudaMemcpyAsync(d_npairs, excl + n, 8, cudaMemcpyDeviceToDevice, L.stream));
  count_launches(2);
}

// ---- partition by owning shard (exchange ops) --------------------------------

// Keeps the keys whose first declared column (the key's low word when
// `col0_lo`, else its high word) belongs to shard `dest`; order-preserving.
struct OwnerSel {
  const uint64_t* keys;
  uint64_t* out;
  bool col0_lo;
  uint32_t world, dest;
  __device__ void block_setup(uint64_t, uint64_t) {}
  __device__ bool select(uint64_t i) const {
    const uint64_t k = keys[i];
    return shard_owner(col0_lo ? (uint32_t)k : (uint32_t)(k >> 32), world) == dest;
  }
  using value_type = uint64_t;
  __device__ uint64_t value(uint64_t i) const { return keys[i]; }
  __device__ void store(uint64_t pos, uint64_t v) const { out[pos] = v; }
};

size_t shard_select_scratch_bytes(uint64_t n) { return cp_scratch_bytes(n); }

void shard_select(const Launch& L, const uint64_t* keys, uint64_t n, bool col0_lo, uint32_t world,
                  uint32_t dest, uint64_t* out, uint64_t* d_nout, Scratch& s) {
  SRDL_REQUIRE(world >= 1 && dest < world, kErrArg, "shard_select: destination out of range");
  OwnerSel sel{keys, out, col0_lo, world, dest};
  compact(L, sel, n, d_nout, s);
}

__global__ void hash_size_kernel(const uint32_t* __restrict__ dir, uint32_t nv, uint32_t min_len,
                                 uint64_t* __restrict__ sizes) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < nv;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t len = dir[v + 1] - dir[v];
    sizes[v] = len > min_len ? (1ull << hash_log2(len)) : 0;
  }
}

__global__ void hash_dir_kernel(const uint64_t* __restrict__ sizes, const uint64_t* __restrict__ offs,
                                uint32_t nv, uint32_t* __restrict__ hdir) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < nv;
       v += (uint64_t)gridDim.x * blockDim.x)
    hdir[v] = sizes[v] ? (uint32_t)offs[v] : kNoHash;
}

__global__ void hash_insert_kernel(const uint64_t* __restrict__ keys, uint64_t n,
                                   const uint32_t* __restrict__ dir, const uint32_t* __restrict__ hdir,
                                   uint32_t* __restrict__ pool) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = (uint32_t)(keys[i] >> 32), x = (uint32_t)keys[i];
    const uint32_t off = hdir[v];
    if (off == kNoHash) continue;
    const int k = hash_log2(dir[v + 1] - dir[v]);
    const uint32_t mask = (1u << k) - 1;
    uint32_t h = hash_slot(x, k);
    // at most `mask + 1` probes; the table is at most half full
    for (uint32_t probe = 0; probe <= mask; probe++) {
      const uint32_t old = atomicCAS(&pool[off + h], kHashEmpty, x);
      if (old == kHashEmpty || old == x) break;
      h = (h + 1) & mask;
    }
  }
}

size_t child_hash_scratch_bytes(uint32_t dir_n) {
  return 2 * ((size_t)dir_n * 8 + 512) + scan_scratch_bytes(dir_n) + 1024;
}

void child_hash_plan(const Launch& L, const uint32_t* dir, uint32_t dir_n, uint32_t min_len,
                     uint64_t* sizes, uint64_t* offs, Scratch& s) {
  const uint32_t nv = dir_n - 1;
  hash_size_kernel<<<grid_for(nv, L.num_sms), 256, 0, L.stream>>>(dir, nv, min_len, sizes);
  SRDL_CUDA(cudaGetLastError());
  count_launches(1);
  exclusive_scan_u64(L, sizes, nv, offs, s);
}

void child_hash_build(const Launch& L, const uint64_t* keys, uint64_t n, const uint32_t* dir,
                      uint32_t dir_n, const uint64_t* sizes, const uint64_t* offs, uint32_t* hdir,
                      uint32_t* pool) {
  const uint32_t nv = dir_n - 1;
  hash_dir_kernel<<<grid_for(nv, L.num_sms), 256, 0, L.stream>>>(sizes, offs, nv, hdir);
  SRDL_CUDA(cudaGetLastError());
  if (n) hash_insert_kernel<<<grid_for(n, L.num_sms), 256, 0, L.stream>>>(keys, n, dir, hdir, pool);
  SRDL_CUDA(cudaGetLastError());
  count_launches(n ? 2 : 1);
}

// ---- bitmaps of long child lists ---------------------------------------

__global__ void bitmap_plan_kernel(const uint32_t* __restrict__ dir, uint32_t nv,
                                   unsigned long long* __restrict__ cnt) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x) {
    const uint32_t len = dir[v + 1] - dir[v];
#pragma unroll
    for (int k = 0; k < kBitmapLevels; k++)
      if (len >= (kBitmapMinLen << k)) atomicAdd(&cnt[k], 1ull);
  }
}

__global__ void bitmap_assign_kernel(const uint32_t* __restrict__ dir, uint32_t nv,
                                     uint32_t min_len, uint32_t* __restrict__ bdir,
                                     unsigned int* __restrict__ d_slots) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nv; v += gridDim.x * blockDim.x)
    bdir[v] = dir[v + 1] - dir[v] >= min_len ? atomicAdd(d_slots, 1u) : kNoBitmap;
}

__global__ void bitmap_fill_kernel(const uint64_t* __restrict__ keys, uint64_t n,
                                   const uint32_t* __restrict__ bdir, uint32_t* __restrict__ pool,
                                   uint32_t bwords) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    const uint32_t s = bdir[k >> 32], c = (uint32_t)k;
    if (s != kNoBitmap) atomicOr(&pool[(uint64_t)s * bwords + (c >> 5)], 1u << (c & 31));
  }
}

void bitmap_plan(const Launch& L, const uint32_t* dir, uint32_t dir_n, unsigned long long* cnt) {
  const uint32_t nv = dir_n - 1;
  SRDL_CUDA(cudaMemsetAsync(cnt, 0, kBitmapLevels * sizeof(unsigned long long), L.stream));
  bitmap_plan_kernel<<<grid_for(nv, L.num_sms), 256, 0, L.stream>>>(dir, nv, cnt);
  SRDL_CUDA(cudaGetLastError());
  count_launches(1);
}

void bitmap_build(const Launch& L, const uint64_t* keys, uint64_t n, const uint32_t* dir,
                  uint32_t dir_n, uint32_t min_len, uint32_t* bdir, uint32_t* pool, uint32_t bwords,
                  unsigned int* d_slots) {
  const uint32_t nv = dir_n - 1;
  SRDL_CUDA(cudaMemsetAsync(d_slots, 0, sizeof(unsigned int), L.stream));
  bitmap_assign_kernel<<<grid_for(nv, L.num_sms), 256, 0, L.stream>>>(dir, nv, min_len, bdir,
                                                                       d_slots);
  if (n)
    bitmap_fill_kernel<<<grid_for(n, L.num_sms), 256, 0, L.stream>>>(keys, n, bdir, pool, bwords);
  SRDL_CUDA(cudaGetLastError());
  count_launches(n ? 2 : 1);
}

__global__ void bounds_kernel(const uint64_t* __restrict__ keys, uint64_t n,
                              const uint32_t* __restrict__ bounds, uint64_t nb,
                              uint64_t* __restrict__ pos) {
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < nb;
       j += (uint64_t)gridDim.x * blockDim.x)
    pos[j] = lower_bound_u64(keys, 0, n, (uint64_t)bounds[j] << 32);
}

void bounds_positions(const Launch& L, const uint64_t* keys, uint64_t n, const uint32_t* bounds,
                      uint64_t n_bounds, uint64_t* pos) {
  if (!n_bounds) return;
  bounds_kernel<<<grid_for(n_bounds, L.num_sms), 256, 0, L.stream>>>(keys, n, bounds, n_bounds, pos);
  SRDL_CUDA(cudaGetLastError());
  count_launches(1);
}

__global__ void max_kernel(const uint32_t* __restrict__ d, uint64_t n, uint32_t* __restrict__ out) {
  uint32_t m = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    m = max(m, d[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(kAllLanes, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

void max_u32(const Launch& L, const uint32_t* d, uint64_t n, uint32_t* d_max) {
  SRDL_CUDA(cudaMemsetAsync(d_max, 0, sizeof(uint32_t), L.stream));
  if (!n) return;
  max_kernel<<<grid_for(n, L.num_sms), 256, 0, L.stream>>>(d, n, d_max);
  SRDL_CUDA(cudaGetLastError());
  count_launches(1);
}

// ------------------------------------------------------------------ scan

constexpr int kScThreads = 256;
constexpr int kScItems = 8;
constexpr int kScTile = kScThreads * kScItems;

__global__ void __launch_bounds__(kScThreads) scan_sum_kernel(const uint64_t* __restrict__ in,
                                                              uint64_t n, uint64_t chunk,
                                                              uint64_t* __restrict__ bsum) {
  __shared__ uint64_t sh[kScThreads / 32 + 1];
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = begin + chunk < n ? begin + chunk : n;
  uint64_t s = 0;
  for (uint64_t i = begin + threadIdx.x; i < end; i += kScThreads) s += in[i];
  uint64_t tot;
  block_excl_scan(s, sh, &tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void scan_blocks_kernel(uint64_t* bsum, int nb) {
  __shared__ uint64_t sh[1024 / 32 + 1];
  const int per = (nb + blockDim.x - 1) / blockDim.x;
  const int s = threadIdx.x * per, e = min(nb, s + per);
  uint64_t sum = 0;
  for (int i = s; i < e; i++) sum += bsum[i];
  uint64_t tot;
  uint64_t run = block_excl_scan(sum, sh, &tot);
  for (int i = s; i < e; i++) {
    uint64_t v = bsum[i];
    bsum[i] = run;
    run += v;
  }
  if (threadIdx.x == 0) bsum[nb] = tot;
}

__global__ void __launch_bounds__(kScThreads) scan_write_kernel(const uint64_t* __restrict__ in,
                                                                uint64_t n, uint64_t chunk,
                                                                const uint64_t* __restrict__ boff,
                                                                uint64_t* __restrict__ out) {
  __shared__ uint64_t sh[kScThreads / 32 + 1];
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = begin + chunk < n ? begin + chunk : n;
  uint64_t base = boff[blockIdx.x];
  for (uint64_t tile = begin; tile < end; tile += kScTile) {
    const uint64_t i0 = tile + (uint64_t)threadIdx.x * kScItems;
    uint64_t v[kScItems];
    uint64_t s = 0;
#pragma unroll
    for (int j = 0; j < kScItems; j++) {
      v[j] = (i0 + j < end) ? in[i0 + j] : 0;
      s += v[j];
    }
    uint64_t tot;
    uint64_t run = base + block_excl_scan(s, sh, &tot);
#pragma unroll
    for (int j = 0; j < kScItems; j++) {
      if (i0 + j < end) out[i0 + j] = run;
      run += v[j];
    }
    base += tot;
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = boff[gridDim.x];
}

size_t scan_scratch_bytes(uint64_t) { return (size_t)(256 * 8 + 2) * 8 + 512; }

void exclusive_scan_u64(const Launch& L, const uint64_t* in, uint64_t n, uint64_t* out,
                        Scratch& s) {
  if (n == 0) {
    SRDL_CUDA(cudaMemsetAsync(out, 0, sizeof(uint64_t), L.stream));
    return;
  }
  const uint64_t tiles = (n + kScTile - 1) / kScTile;
  const uint64_t cap = (uint64_t)L.num_sms * 8;
  const uint64_t per = (tiles + cap - 1) / cap;
  const uint64_t chunk = (per ? per : 1) * kScTile;
  const int nb = (int)((n + chunk - 1) / chunk);
  uint64_t* bsum = s.take<uint64_t>(nb + 1);
  scan_sum_kernel<<<nb, kScThreads, 0, L.stream>>>(in, n, chunk, bsum);
  scan_blocks_kernel<<<1, 1024, 0, L.stream>>>(bsum, nb);
  scan_write_kernel<<<nb, kScThreads, 0, L.stream>>>(in, n, chunk, bsum, out);
  SRDL_CUDA(cudaGetLastError());
  count_launches(3);
}

}  // namespace srdl
