// compact.cuh -- order-preserving stream compaction in three launches.
//
//   1. flag   : each block owns a contiguous chunk; every warp evaluates the
//               selector on 32 consecutive elements at a time and stores the
//               ballot as one flag word (bit l = element 32w + l); the block's
//               selected count goes to blk_counts;
//   2. scan   : one block turns the per-block counts into offsets + total;
//   3. write  : each block walks its chunk a 2048-element tile at a time;
//               warp w takes the tile's elements [256w, 256w + 256) in eight
//               rounds of 32, so a round's output positions are the running
//               count plus the popcount of the lower lanes of its flag word:
//               loads and stores are coalesced.
// No block waits on another, so nothing can spin.  Selectors provide
//   __device__ void block_setup(uint64_t begin, uint64_t end);  (all threads)
//   __device__ bool select(uint64_t i);
//   using value_type = ...;
//   __device__ value_type value(uint64_t i);        (what element i emits)
//   __device__ void store(uint64_t pos, value_type v);
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace srdl {

constexpr int kCpThreads = 256;
constexpr int kCpWarps = kCpThreads / 32;
constexpr int kCpItems = 8;
constexpr int kCpTile = kCpThreads * kCpItems;

// Grid shape for n elements: every block owns `chunk` elements (a multiple
// of the tile), at most 8 blocks per SM, no empty blocks.
inline uint64_t cp_chunk(uint64_t n, int sms) {
  uint64_t tiles = (n + kCpTile - 1) / kCpTile;
  uint64_t cap = (uint64_t)sms * 8;
  uint64_t per = (tiles + cap - 1) / cap;
  return (per ? per : 1) * (uint64_t)kCpTile;
}
inline int cp_blocks(uint64_t n, uint64_t chunk) {
  uint64_t nb = (n + chunk - 1) / chunk;
  return nb ? (int)nb : 1;
}
inline uint64_t cp_words(uint64_t n) { return (n + 31) / 32; }
inline size_t cp_scratch_bytes(uint64_t n) {
  // flag words + per-block counts and offsets (blocks <= 8 per SM; 256 SMs
  // bound) + the FULL and HEAD positions of every tile boundary (set
  // difference), each piece padded to 256 bytes, plus alignment slack for the
  // region itself
  // (+ the merge-path cuts: FULL at most 16 times the keys on that path)
  const uint64_t tiles = (n + kCpTile - 1) / kCpTile + 1;
  const uint64_t mtiles = (17 * n + kCpTile - 1) / kCpTile + 2;
  return ((cp_words(n) * 4 + 255) & ~uint64_t(255)) + (size_t)(256 * 8 + 1) * 12 + 3 * 256 +
         2 * ((tiles * 8 + 255) & ~uint64_t(255)) + 2 * ((mtiles * 8 + 255) & ~uint64_t(255)) + 256;
}

// With d_n (device loop), n is a capacity and the count is *d_n; chunk 0
// then means the even split of the true count over the grid.
template <class Sel>
__global__ void __launch_bounds__(kCpThreads) cp_flag_kernel(Sel sel, uint64_t n, uint64_t chunk,
                                                             uint32_t* flags, uint32_t* blk_counts,
                                                             const uint64_t* d_n) {
  __shared__ uint32_t sh[kCpThreads / 32 + 1];
  n = dev_size(n, d_n);
  chunk = dev_chunk(chunk, n, kCpTile);
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = begin + chunk < n ? begin + chunk : n;
  const int lane = threadIdx.x & 31;
  sel.block_setup(begin, end);
  uint32_t cnt = 0;
  // chunk starts are multiples of 32, so each round of a warp is one flag word
  for (uint64_t w0 = begin + (threadIdx.x & ~31u); w0 < end; w0 += kCpThreads) {
    const uint64_t i = w0 + lane;
    const bool f = i < end && sel.select(i);
    const uint32_t m = __ballot_sync(kAllLanes, f);
    if (lane == 0) flags[w0 / 32] = m;
    cnt += f;
  }
  uint32_t tot;
  block_excl_scan(cnt, sh, &tot);
  if (threadIdx.x == 0) blk_counts[blockIdx.x] = tot;
}

// One block; exclusive scan of nb block counts into offs[0..nb], total -> *d_total.
__global__ void cp_scan_kernel(const uint32_t* blk_counts, int nb, uint64_t* offs,
                               uint64_t* d_total);

template <class Sel>
__global__ void __launch_bounds__(kCpThreads) cp_write_kernel(Sel sel, uint64_t n, uint64_t chunk,
                                                              const uint32_t* __restrict__ flags,
                                                              const uint64_t* offs,
                                                              const uint64_t* d_n) {
  __shared__ uint32_t wtot[2][kCpWarps];
  n = dev_size(n, d_n);
  chunk = dev_chunk(chunk, n, kCpTile);
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = begin + chunk < n ? begin + chunk : n;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned lt = lanemask_lt();
  uint64_t base = offs[blockIdx.x];
  int par = 0;
  for (uint64_t tile = begin; tile < end; tile += kCpTile, par ^= 1) {
    // lane r < 8 fetches the flag word of round r of this warp's 256 elements
    const uint64_t w0 = tile + (uint64_t)wid * (kCpItems * 32);
    const uint64_t wi = w0 + (uint64_t)lane * 32;
    const uint32_t my_word = (lane < kCpItems && wi < end) ? flags[wi / 32] : 0u;
    // the eight rounds' element loads are all issued before the first
    // store (coalesced either way; this keeps eight loads in flight)
    typename Sel::value_type v[kCpItems];
#pragma unroll
    for (int r = 0; r < kCpItems; r++) {
      const uint64_t i = w0 + (uint64_t)r * 32 + lane;
      if (i < end) v[r] = sel.value(i);
    }
    const uint32_t wcount = warp_sum((uint32_t)__popc(my_word));
    if (lane == 0) wtot[par][wid] = wcount;
    __syncthreads();
    uint64_t pos = base;
    uint32_t tile_total = 0;
#pragma unroll
    for (int w = 0; w < kCpWarps; w++) {
      const uint32_t c = wtot[par][w];
      pos += w < wid ? c : 0;
      tile_total += c;
    }
#pragma unroll
    for (int r = 0; r < kCpItems; r++) {
      const uint32_t m = __shfl_sync(kAllLanes, my_word, r);
      if ((m >> lane) & 1u) sel.store(pos + __popc(m & lt), v[r]);
      pos += __popc(m);
    }
    base += tile_total;
  }
}

// Runs the three launches; the selected count lands in *d_total.  With d_n,
// n is a capacity and the element count is *d_n (device loop).
template <class Sel>
void compact(const Launch& L, Sel sel, uint64_t n, uint64_t* d_total, Scratch& s,
             const uint64_t* d_n = nullptr) {
  if (n == 0) {
    SRDL_CUDA(cudaMemsetAsync(d_total, 0, sizeof(uint64_t), L.stream));
    return;
  }
  const uint64_t chunk = cp_chunk(n, L.num_sms);
  const int nb = cp_blocks(n, chunk);
  const uint64_t kchunk = d_n ? 0 : chunk;
  uint32_t* flags = s.take<uint32_t>(cp_words(n));
  uint32_t* counts = s.take<uint32_t>(nb);
  uint64_t* offs = s.take<uint64_t>(nb + 1);
  cp_flag_kernel<Sel><<<nb, kCpThreads, 0, L.stream>>>(sel, n, kchunk, flags, counts, d_n);
  cp_scan_kernel<<<1, 1024, 0, L.stream>>>(counts, nb, offs, d_total);
  cp_write_kernel<Sel><<<nb, kCpThreads, 0, L.stream>>>(sel, n, kchunk, flags, offs, d_n);
  SRDL_CUDA(cudaGetLastError());
  count_launches(3);
}

// Keeps a[i] when it differs from a[i-1] (optional) and is absent from the
// sorted unique arrays full[0..n_full) and head[0..n_head) (a Device2Level
// relation's two segments; head may be empty).  Keys are stored compressed
// as (hi << bits) | lo and are expanded to (hi << 32) | lo on output.
template <typename K>
struct DedupDiffSel {
  const K* a;
  int bits;
  bool dedup;
  const uint64_t* full;
  uint64_t n_full;
  uint64_t* out;
  const uint64_t* head = nullptr;
  uint64_t n_head = 0;
  const uint64_t* d_n_full = nullptr;  // device loop: FULL's count on the device (n_full = capacity)
  uint64_t out_cap = ~0ull;             // device loop: room in `out`; a key past it raises *d_overflow
  unsigned int* d_overflow = nullptr;

  __device__ __forceinline__ uint64_t expand(K c) const {
    if (sizeof(K) == 8 && bits == 32) return (uint64_t)c;
    const uint64_t m = (1ull << bits) - 1;
    return (((uint64_t)c >> bits) << 32) | ((uint64_t)c & m);
  }
  __device__ void block_setup(uint64_t begin, uint64_t end) {
    __shared__ uint64_t range[2];
    if (full && n_full) {
      if (threadIdx.x == 0 && begin < end) {
        range[0] = lower_bound_u64(full, 0, n_full, expand(a[begin]));
        uint64_t last = expand(a[end - 1]);
        uint64_t hi = lower_bound_u64(full, range[0], n_full, last);
        range[1] = (hi < n_full && full[hi] == last) ? hi + 1 : hi;
      }
      __syncthreads();
      lo_ = range[0];
      hi_ = range[1];
    }
  }
  uint64_t lo_ = 0, hi_ = 0;
  __device__ bool select(uint64_t i) const {
    K c = a[i];
    if (dedup && i > 0 && a[i - 1] == c) return false;
    if (full && hi_ > lo_) {
      uint64_t k = expand(c);
      uint64_t p = lower_bound_u64(full, lo_, hi_, k);
      if (p < hi_ && full[p] == k) return false;
    }
    return true;
  }
  using value_type = uint64_t;
  __device__ uint64_t value(uint64_t i) const { return expand(a[i]); }
  __device__ void store(uint64_t pos, uint64_t v) const {
    if (pos < out_cap) out[pos] = v;
    else if (d_overflow) *d_overflow = 1u;
  }
};

// FULL position of every tile boundary: fpos[t] = lower_bound(FULL, first key
// of tile t) for t < tiles, fpos[tiles] = n_full.  One warp per boundary
// (32-ary search), all boundaries in parallel.  Tile t's keys can only match
// FULL[fpos[t], fpos[t+1] + 1): its last key is <= the next tile's first.
// hpos (when a HEAD is given) holds the same positions in HEAD.
template <typename K>
__global__ void dd_bounds_kernel(DedupDiffSel<K> sel, uint64_t n, uint64_t tiles,
                                 uint64_t* __restrict__ fpos, uint64_t* __restrict__ hpos,
                                 const uint64_t* d_n, int path) {
  sel.n_full = dev_size(sel.n_full, sel.d_n_full);
  n = dev_size(n, d_n);
  if (!diff_path_runs(path, sel, n)) return;
  const uint64_t real = (n + kCpTile - 1) / kCpTile;  // tiles holding keys
  // one warp per boundary; warps walk the boundaries when the grid is capped
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) / 32;
  for (uint64_t t = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) / 32; t <= tiles; t += warps) {
    uint64_t p = sel.n_full, q = sel.n_head;
    if (t < real) {
      const uint64_t first = sel.expand(sel.a[t * kCpTile]);
      p = warp_partition_point(0, sel.n_full, [&](uint64_t i) { return sel.full[i] < first; });
      if (hpos)
        q = warp_partition_point(0, sel.n_head, [&](uint64_t i) { return sel.head[i] < first; });
    }
    if ((threadIdx.x & 31) == 0) {
      fpos[t] = p;
      if (hpos) hpos[t] = q;
    }
    if (d_n && t > real) break;  // past the true tiles every entry is n_full
  }
}

// Flag pass of DedupDiffSel with FULL: the block walks its chunk one tile at
// a time and stages the tile's keys and, when it fits, the tile's slice of
// FULL in shared memory.  Thread t owns the tile's keys [8t, 8t + 8): it
// binary-searches the slice for its first key only and walks forward from
// there for the other seven (both runs are sorted), so a key costs about one
// comparison instead of a dozen.  The eight flag bits of four neighbouring
// threads form one 32-key flag word.  Slices that do not fit are searched in
// global memory, each key galloping forward from the previous key's
// position; the HEAD segment is probed by binary search within the tile's
// range.
constexpr int kDdStage = 4000;  // FULL keys staged per tile (31.25 KB: with 64-bit tile keys under 48 KB)

template <typename K>
__global__ void __launch_bounds__(kCpThreads) dd_flag_kernel(DedupDiffSel<K> sel, uint64_t n,
                                                             uint64_t chunk,
                                                             const uint64_t* __restrict__ fpos,
                                                             const uint64_t* __restrict__ hpos,
                                                             uint32_t* flags,
                                                             uint32_t* blk_counts,
                                                             const uint64_t* d_n, int path) {
  __shared__ uint64_t stage[kDdStage];
  __shared__ K skey[kCpTile + 1];  // skey[j + 1] = tile key j, skey[0] = the key before the tile
  __shared__ uint32_t sh[kCpThreads / 32 + 1];
  sel.n_full = dev_size(sel.n_full, sel.d_n_full);
  n = dev_size(n, d_n);
  if (!diff_path_runs(path, sel, n)) return;
  chunk = dev_chunk(chunk, n, kCpTile);
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = begin + chunk < n ? begin + chunk : n;
  const int lane = threadIdx.x & 31;
  const uint32_t j0 = threadIdx.x * kCpItems;
  uint32_t cnt = 0;
  for (uint64_t tile = begin; tile < end; tile += kCpTile) {
    const uint32_t tn = (uint32_t)(end - tile < kCpTile ? end - tile : kCpTile);
    const uint64_t t = tile / kCpTile;
    const uint64_t f0 = fpos[t];
    uint64_t f1 = fpos[t + 1] + 1;
    f1 = f1 < sel.n_full ? f1 : sel.n_full;
    const uint32_t len = (uint32_t)(f1 > f0 ? (f1 - f0 < 0xffffffffull ? f1 - f0 : 0xffffffffull) : 0);
    const bool staged = len <= (uint32_t)kDdStage;
    uint64_t h0 = 0, h1 = 0;
    if (hpos) {
      h0 = hpos[t];
      h1 = hpos[t + 1] + 1;
      h1 = h1 < sel.n_head ? h1 : sel.n_head;
    }
    // Staging: every thread issues all of its loads before its first shared
    // store, so a tile costs one or two memory round trips, not one per load.
    {
      K kr[kCpItems];
#pragma unroll
      for (int q = 0; q < kCpItems; q++) {
        const uint32_t j = threadIdx.x + q * kCpThreads;
        kr[q] = j < tn ? sel.a[tile + j] : K(0);
      }
      const K prev = (threadIdx.x == 0 && tile > 0) ? sel.a[tile - 1] : K(0);
      if (staged) {
        for (uint32_t b0 = 0; b0 < len; b0 += kCpThreads * kCpItems) {
          uint64_t fr[kCpItems];
#pragma unroll
          for (int q = 0; q < kCpItems; q++) {
            const uint32_t j = b0 + threadIdx.x + q * kCpThreads;
            fr[q] = j < len ? sel.full[f0 + j] : 0;
          }
#pragma unroll
          for (int q = 0; q < kCpItems; q++) {
            const uint32_t j = b0 + threadIdx.x + q * kCpThreads;
            if (j < len) stage[j] = fr[q];
          }
        }
      }
#pragma unroll
      for (int q = 0; q < kCpItems; q++) {
        const uint32_t j = threadIdx.x + q * kCpThreads;
        if (j < tn) skey[j + 1] = kr[q];
      }
      if (threadIdx.x == 0) skey[0] = prev;
    }
    __syncthreads();
    uint32_t bits = 0;
    if (j0 < tn) {
      uint32_t p = 0;
      uint64_t g = f0;  // unstaged slice: this thread's position in FULL
      if (staged && len) {
        const uint64_t k0 = sel.expand(skey[j0 + 1]);
        uint32_t lo = 0, hi = len;
        while (lo < hi) {
          const uint32_t mid = (lo + hi) >> 1;
          if (stage[mid] < k0) lo = mid + 1;
          else hi = mid;
        }
        p = lo;
      }
#pragma unroll
      for (int q = 0; q < kCpItems; q++) {
        const uint32_t j = j0 + q;
        if (j >= tn) break;
        const K c = skey[j + 1];
        bool keep = !(sel.dedup && (tile + j) > 0 && skey[j] == c);
        if (keep && len) {
          const uint64_t k = sel.expand(c);
          if (staged) {
            while (p < len && stage[p] < k) p++;
            keep = !(p < len && stage[p] == k);
          } else {
            g = q == 0 ? lower_bound_u64(sel.full, f0, f1, k)
                       : gallop_lower_bound_u64(sel.full, g, f1, k);
            keep = !(g < f1 && sel.full[g] == k);
          }
        }
        if (keep && h1 > h0) {
          const uint64_t k = sel.expand(c);
          const uint64_t g = lower_bound_u64(sel.head, h0, h1, k);
          keep = !(g < h1 && sel.head[g] == k);
        }
        bits |= (keep ? 1u : 0u) << q;
      }
    }
    // lanes 4w..4w+3 hold the bytes of flag word w of this warp's 128 keys
    uint32_t word = bits << (8 * (lane & 3));
    word |= __shfl_down_sync(kAllLanes, word, 1);
    word |= __shfl_down_sync(kAllLanes, word, 2);
    if ((lane & 3) == 0 && j0 < tn) flags[(tile + j0) / 32] = word;
    cnt += __popc(bits);
    __syncthreads();
  }
  uint32_t tot;
  block_excl_scan(cnt, sh, &tot);
  if (threadIdx.x == 0) blk_counts[blockIdx.x] = tot;
}

// ---- merge-path flag pass (FULL streamed once) ------------------------------
//
// The keys a (sorted, possibly repeating) and FULL (sorted, unique) are
// merged, FULL first on equal values, and the merged sequence is cut into
// tiles of kCpTile elements (one thread per tile boundary finds the cut by
// merge-path binary search, and the tile's start in HEAD).  Persistent blocks
// walk the tiles; the next tile's two slices are copied into the second
// shared buffer with cp.async while the current tile is merged, 8 merged
// elements per thread.  An a-key is kept iff it differs from the last FULL
// key taken at or before it (so it is not in FULL) and from the a-key before
// it (dedup); HEAD, when present, is probed per kept key within the tile's
// HEAD range.  Bits are OR-ed into the flag words (a tile's a-range does not
// start on a word boundary).

// Number of a-keys among the first `diag` merged elements.
template <typename K>
__device__ __forceinline__ uint64_t dm_path(const DedupDiffSel<K>& sel, uint64_t na,
                                            uint64_t diag) {
  uint64_t lo = diag > sel.n_full ? diag - sel.n_full : 0;
  uint64_t hi = diag < na ? diag : na;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (sel.expand(sel.a[mid]) < sel.full[diag - 1 - mid]) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// split[t] = a-keys among the first t*kCpTile merged elements; hpos[t] = the
// HEAD position of a[split[t]] (n_head past the last key).
// Device loop (d_n set): the merge path and the probe path are both in the
// graph and each kernel runs only when the counts on the device select its
// path (FULL at most kDmMaxFullRatio times the keys: merge path).
constexpr uint64_t kDmMaxFullRatio = 16;
enum DiffPath : int { kPathAny = 0, kPathMerge = 1, kPathProbe = 2 };

template <typename K>
__device__ __forceinline__ bool diff_path_runs(int path, const DedupDiffSel<K>& sel, uint64_t n) {
  if (path == kPathAny) return true;
  const bool merge = sel.n_full <= kDmMaxFullRatio * n;
  return (path == kPathMerge) == merge;
}

template <typename K>
__global__ void dm_split_kernel(DedupDiffSel<K> sel, uint64_t na, uint64_t tiles,
                                uint64_t* __restrict__ split, uint64_t* __restrict__ hpos,
                                const uint64_t* d_n, int path) {
  const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  sel.n_full = dev_size(sel.n_full, sel.d_n_full);
  na = dev_size(na, d_n);
  if (!diff_path_runs(path, sel, na)) return;
  if (d_n) tiles = (na + sel.n_full + kCpTile - 1) / kCpTile;
  if (t > tiles) return;
  const uint64_t total = na + sel.n_full;
  const uint64_t diag = t * kCpTile < total ? t * kCpTile : total;
  const uint64_t i = dm_path(sel, na, diag);
  split[t] = i;
  if (hpos)
    hpos[t] = i < na ? lower_bound_u64(sel.head, 0, sel.n_head, sel.expand(sel.a[i])) : sel.n_head;
}

template <int BYTES>
__device__ __forceinline__ void cp_async_small(void* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(BYTES)
               : "memory");
}

// One merged tile's slices: la a-keys (K) at the start of the buffer, lf FULL
// keys after them at an 8-byte boundary; returns nothing, commits one group.
template <typename K>
__device__ __forceinline__ void dm_fetch(const DedupDiffSel<K>& sel, unsigned char* buf,
                                         uint64_t i0, uint32_t la, uint64_t j0, uint32_t lf) {
  K* da = reinterpret_cast<K*>(buf);
  uint64_t* df = reinterpret_cast<uint64_t*>(buf + ((la * sizeof(K) + 7) & ~size_t(7)));
  for (uint32_t k = threadIdx.x; k < la; k += kCpThreads) cp_async_small<sizeof(K)>(da + k, sel.a + i0 + k);
  for (uint32_t k = threadIdx.x; k < lf; k += kCpThreads) cp_async_small<8>(df + k, sel.full + j0 + k);
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <typename K>
__global__ void __launch_bounds__(kCpThreads) dm_mark_kernel(DedupDiffSel<K> sel, uint64_t na,
                                                             uint64_t tiles,
                                                             const uint64_t* __restrict__ split,
                                                             const uint64_t* __restrict__ hpos,
                                                             uint32_t* __restrict__ flags,
                                                             const uint64_t* d_n, int path) {
  __shared__ __align__(16) unsigned char buf[2][kCpTile * 8];
  __shared__ uint32_t sbits[kCpTile / 32 + 2];
  sel.n_full = dev_size(sel.n_full, sel.d_n_full);
  na = dev_size(na, d_n);
  if (!diff_path_runs(path, sel, na)) return;
  if (d_n) tiles = (na + sel.n_full + kCpTile - 1) / kCpTile;
  const uint64_t total = na + sel.n_full;
  auto bounds = [&](uint64_t t, uint64_t& i0, uint64_t& i1, uint64_t& j0, uint64_t& j1) {
    const uint64_t d0 = t * kCpTile;
    const uint64_t d1 = d0 + kCpTile < total ? d0 + kCpTile : total;
    i0 = split[t];
    i1 = split[t + 1];
    j0 = d0 - i0;
    j1 = d1 - i1;
  };
  uint64_t t = blockIdx.x;
  if (t >= tiles) return;
  uint64_t i0, i1, j0, j1;
  bounds(t, i0, i1, j0, j1);
  dm_fetch(sel, buf[0], i0, (uint32_t)(i1 - i0), j0, (uint32_t)(j1 - j0));
  int cur = 0;
  for (;;) {
    const uint64_t tn = t + gridDim.x;
    uint64_t ni0 = 0, ni1 = 0, nj0 = 0, nj1 = 0;
    if (tn < tiles) {
      bounds(tn, ni0, ni1, nj0, nj1);
      dm_fetch(sel, buf[cur ^ 1], ni0, (uint32_t)(ni1 - ni0), nj0, (uint32_t)(nj1 - nj0));
    }
    const uint32_t la = (uint32_t)(i1 - i0), lf = (uint32_t)(j1 - j0);
    const uint64_t w0 = i0 / 32;
    const uint32_t nwords = la ? (uint32_t)((i1 - 1) / 32 - w0 + 1) : 0;
    for (uint32_t k = threadIdx.x; k < nwords; k += kCpThreads) sbits[k] = 0;
    // values just before the tile (for the first element of thread 0's run)
    const uint64_t edge_a = i0 > 0 ? sel.expand(sel.a[i0 - 1]) : 0;
    const uint64_t edge_f = j0 > 0 ? sel.full[j0 - 1] : 0;
    uint64_t h0 = 0, h1 = 0;
    if (hpos) {
      h0 = hpos[t];
      h1 = hpos[t + 1] + 1;
      h1 = h1 < sel.n_head ? h1 : sel.n_head;
    }
    if (tn < tiles) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
    else asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    const K* sa = reinterpret_cast<const K*>(buf[cur]);
    const uint64_t* sf =
        reinterpret_cast<const uint64_t*>(buf[cur] + ((la * sizeof(K) + 7) & ~size_t(7)));
    const uint32_t diag = threadIdx.x * kCpItems;
    if (diag < la + lf && la) {
      uint32_t lo = diag > lf ? diag - lf : 0, hi = diag < la ? diag : la;
      while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (sel.expand(sa[mid]) < sf[diag - 1 - mid]) lo = mid + 1;
        else hi = mid;
      }
      uint32_t ia = lo, jf = diag - lo;
      bool has_f = jf > 0 || j0 > 0;
      uint64_t last_f = jf > 0 ? sf[jf - 1] : edge_f;
      bool has_p = ia > 0 || i0 > 0;
      uint64_t prev = ia > 0 ? sel.expand(sa[ia - 1]) : edge_a;
      // this thread's a-keys are consecutive: their bits fit two flag words
      const uint64_t wbase = (i0 + ia) / 32;
      uint64_t mask = 0;
#pragma unroll
      for (int q = 0; q < kCpItems; q++) {
        if (ia + jf >= la + lf) break;
        const uint64_t x = ia < la ? sel.expand(sa[ia]) : 0;
        const bool take_a = jf >= lf || (ia < la && x < sf[jf]);
        if (!take_a) {
          last_f = sf[jf++];
          has_f = true;
          continue;
        }
        bool keep = !(has_f && last_f == x) && !(sel.dedup && has_p && prev == x);
        if (keep && h1 > h0) {
          const uint64_t g = lower_bound_u64(sel.head, h0, h1, x);
          keep = !(g < h1 && sel.head[g] == x);
        }
        if (keep) mask |= 1ull << (i0 + ia - wbase * 32);
        prev = x;
        has_p = true;
        ia++;
      }
      if ((uint32_t)mask) atomicOr(&sbits[wbase - w0], (uint32_t)mask);
      if (mask >> 32) atomicOr(&sbits[wbase + 1 - w0], (uint32_t)(mask >> 32));
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < nwords; k += kCpThreads)
      if (sbits[k]) atomicOr(&flags[w0 + k], sbits[k]);
    __syncthreads();
    if (tn >= tiles) break;
    t = tn;
    i0 = ni0;
    i1 = ni1;
    j0 = nj0;
    j1 = nj1;
    cur ^= 1;
  }
}

// Per-block selected counts of a flag-word array (blocks own `chunk` keys).
template <typename K>
static __global__ void __launch_bounds__(kCpThreads) cp_count_kernel(const uint32_t* __restrict__ flags,
                                                              uint64_t n, uint64_t chunk,
                                                              uint32_t* blk_counts,
                                                              DedupDiffSel<K> sel,
                                                              const uint64_t* d_n, int path) {
  __shared__ uint32_t sh[kCpThreads / 32 + 1];
  sel.n_full = dev_size(sel.n_full, sel.d_n_full);
  n = dev_size(n, d_n);
  if (!diff_path_runs(path, sel, n)) return;
  chunk = dev_chunk(chunk, n, kCpTile);
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = begin + chunk < n ? begin + chunk : n;
  uint32_t c = 0;
  for (uint64_t w = begin / 32 + threadIdx.x; w < (end + 31) / 32; w += kCpThreads)
    c += __popc(flags[w]);
  uint32_t tot;
  block_excl_scan(c, sh, &tot);
  if (threadIdx.x == 0) blk_counts[blockIdx.x] = tot;
}

// The merge-path pass streams all of FULL; past kDmMaxFullRatio the per-tile
// probes of dd_flag_kernel read less.

// compact() for DedupDiffSel with a FULL array: merge path when FULL is not
// much larger than the keys, tiled shared-memory probes otherwise.
template <typename K>
void compact_diff(const Launch& L, DedupDiffSel<K> sel, uint64_t n, uint64_t* d_total, Scratch& s) {
  if (!sel.head || sel.n_head == 0) {
    sel.head = nullptr;
    sel.n_head = 0;
  }
  if ((!sel.full || sel.n_full == 0) && !sel.head) {
    compact(L, sel, n, d_total, s);
    return;
  }
  if (!sel.full) sel.n_full = 0;
  if (n == 0) {
    SRDL_CUDA(cudaMemsetAsync(d_total, 0, sizeof(uint64_t), L.stream));
    return;
  }
  const uint64_t chunk = cp_chunk(n, L.num_sms);
  const int nb = cp_blocks(n, chunk);
  const uint64_t tiles = (n + kCpTile - 1) / kCpTile;
  uint32_t* flags = s.take<uint32_t>(cp_words(n));
  uint32_t* counts = s.take<uint32_t>(nb);
  uint64_t* offs = s.take<uint64_t>(nb + 1);
  if (sel.n_full <= kDmMaxFullRatio * n) {
    const uint64_t mtiles = (n + sel.n_full + kCpTile - 1) / kCpTile;
    SRDL_REQUIRE(mtiles < (1ull << 31), kErrCapacity, "set difference: too many rows");
    uint64_t* split = s.take<uint64_t>(mtiles + 1);
    uint64_t* mhpos = sel.head ? s.take<uint64_t>(mtiles + 1) : nullptr;
    SRDL_CUDA(cudaMemsetAsync(flags, 0, cp_words(n) * 4, L.stream));
    dm_split_kernel<K><<<(unsigned)((mtiles + 1 + 255) / 256), 256, 0, L.stream>>>(sel, n, mtiles,
                                                                                  split, mhpos, nullptr,
                                                                                  kPathAny);
    const unsigned mgrid = (unsigned)std::min<uint64_t>(mtiles, (uint64_t)L.num_sms * 4);
    dm_mark_kernel<K><<<mgrid, kCpThreads, 0, L.stream>>>(sel, n, mtiles, split, mhpos, flags, nullptr,
                                                          kPathAny);
    cp_count_kernel<K><<<nb, kCpThreads, 0, L.stream>>>(flags, n, chunk, counts, sel, nullptr, kPathAny);
    cp_scan_kernel<<<1, 1024, 0, L.stream>>>(counts, nb, offs, d_total);
    cp_write_kernel<DedupDiffSel<K>><<<nb, kCpThreads, 0, L.stream>>>(sel, n, chunk, flags, offs,
                                                                       nullptr);
    SRDL_CUDA(cudaGetLastError());
    count_launches(5);
    return;
  }
  uint64_t* fpos = s.take<uint64_t>(tiles + 1);
  uint64_t* hpos = sel.head ? s.take<uint64_t>(tiles + 1) : nullptr;
  prefer_shared(dd_flag_kernel<K>);
  const uint64_t bthreads = (tiles + 1) * 32;
  dd_bounds_kernel<K><<<(unsigned)((bthreads + 255) / 256), 256, 0, L.stream>>>(sel, n, tiles, fpos,
                                                                                hpos, nullptr, kPathAny);
  dd_flag_kernel<K><<<nb, kCpThreads, 0, L.stream>>>(sel, n, chunk, fpos, hpos, flags, counts,
                                                     nullptr, kPathAny);
  cp_scan_kernel<<<1, 1024, 0, L.stream>>>(counts, nb, offs, d_total);
  cp_write_kernel<DedupDiffSel<K>><<<nb, kCpThreads, 0, L.stream>>>(sel, n, chunk, flags, offs,
                                                                     nullptr);
  SRDL_CUDA(cudaGetLastError());
  count_launches(4);
}

// compact_diff with the key count on the device (device loop): `cap` keys
// of room, *d_n of them present, FULL's count at sel.d_n_full (n_full its
// capacity).  Both the merge path and the per-tile probe path are launched;
// each kernel runs only when the counts on the device select its path (the
// host's rule: merge while FULL is at most kDmMaxFullRatio times the keys),
// so no host decision depends on the counts.  Grids are sized for the
// capacities and each block derives its share of the true counts.
inline size_t diff_dev_extra_bytes(uint64_t cap, uint64_t full_cap) {
  return ((cap + full_cap) / kCpTile + 2) * 8 + 512;
}

template <typename K>
void compact_diff_dev(const Launch& L, DedupDiffSel<K> sel, uint64_t cap, const uint64_t* d_n,
                      uint64_t* d_total, Scratch& s) {
  sel.head = nullptr;
  sel.n_head = 0;
  if (!sel.full || !sel.d_n_full) {
    sel.full = nullptr;
    sel.n_full = 0;
    sel.d_n_full = nullptr;
    compact(L, sel, cap, d_total, s, d_n);
    return;
  }
  const uint64_t chunk = cp_chunk(cap, L.num_sms);
  const int nb = cp_blocks(cap, chunk);
  const uint64_t tiles = (cap + kCpTile - 1) / kCpTile;
  const uint64_t mtiles = (cap + sel.n_full + kCpTile - 1) / kCpTile;
  uint32_t* flags = s.take<uint32_t>(cp_words(cap));
  uint32_t* counts = s.take<uint32_t>(nb);
  uint64_t* offs = s.take<uint64_t>(nb + 1);
  uint64_t* fpos = s.take<uint64_t>(tiles + 1);
  uint64_t* split = s.take<uint64_t>(mtiles + 1);
  prefer_shared(dd_flag_kernel<K>);
  // merge path: the mark pass ORs its bits into zeroed flag words
  SRDL_CUDA(cudaMemsetAsync(flags, 0, cp_words(cap) * 4, L.stream));
  dm_split_kernel<K><<<(unsigned)((mtiles + 1 + 255) / 256), 256, 0, L.stream>>>(sel, cap, mtiles, split,
                                                                                nullptr, d_n, kPathMerge);
  const unsigned mgrid = (unsigned)std::min<uint64_t>(mtiles, (uint64_t)L.num_sms * 4);
  dm_mark_kernel<K><<<mgrid, kCpThreads, 0, L.stream>>>(sel, cap, mtiles, split, nullptr, flags, d_n,
                                                        kPathMerge);
  cp_count_kernel<K><<<nb, kCpThreads, 0, L.stream>>>(flags, cap, 0, counts, sel, d_n, kPathMerge);
  // probe path (a capped grid of warps walks the tile boundaries)
  const uint64_t bthreads = (tiles + 1) * 32;
  const uint64_t bblocks = std::min<uint64_t>((bthreads + 255) / 256, (uint64_t)L.num_sms * 8);
  dd_bounds_kernel<K><<<(unsigned)bblocks, 256, 0, L.stream>>>(sel, cap, tiles, fpos, nullptr, d_n,
                                                              kPathProbe);
  dd_flag_kernel<K><<<nb, kCpThreads, 0, L.stream>>>(sel, cap, 0, fpos, nullptr, flags, counts, d_n,
                                                     kPathProbe);
  // either way: offsets and the ordered write of the kept keys
  cp_scan_kernel<<<1, 1024, 0, L.stream>>>(counts, nb, offs, d_total);
  cp_write_kernel<DedupDiffSel<K>><<<nb, kCpThreads, 0, L.stream>>>(sel, cap, 0, flags, offs, d_n);
  SRDL_CUDA(cudaGetLastError());
  count_launches(7);
}

// Distinct first-column values of a sorted key array.
struct RootSel {
  const uint64_t* keys;
  uint32_t* roots;
  __device__ void block_setup(uint64_t, uint64_t) {}
  __device__ bool select(uint64_t i) const {
    return i == 0 || (keys[i] >> 32) != (keys[i - 1] >> 32);
  }
  using value_type = uint32_t;
  __device__ uint32_t value(uint64_t i) const { return (uint32_t)(keys[i] >> 32); }
  __device__ void store(uint64_t pos, uint32_t v) const { roots[pos] = v; }
};

}  // namespace srdl
