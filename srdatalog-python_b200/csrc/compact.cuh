// compact.cuh -- order-preserving stream compaction in three launches.
//
//   1. flag   : each block owns a contiguous chunk, evaluates the selector per
//               element, stores a flag byte and the block's selected count;
//   2. scan   : one block turns the per-block counts into offsets + total;
//   3. write  : each block re-reads its flags tile by tile, block-scans them
//               and hands every selected element its output position.
// No block waits on another, so nothing can spin.  Selectors provide
//   __device__ void block_setup(uint64_t begin, uint64_t end);  (all threads)
//   __device__ bool select(uint64_t i);
//   __device__ void emit(uint64_t i, uint64_t pos);
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace srdl {

constexpr int kCpThreads = 256;
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
inline size_t cp_scratch_bytes(uint64_t n) {
  // flags + per-block counts and offsets (blocks <= 8 per SM; 256 SMs bound)
  return ((n + 255) & ~uint64_t(255)) + (size_t)(256 * 8 + 1) * 12 + 3 * 256;
}

template <class Sel>
__global__ void __launch_bounds__(kCpThreads) cp_flag_kernel(Sel sel, uint64_t n, uint64_t chunk,
                                                             uint8_t* flags, uint32_t* blk_counts) {
  __shared__ uint32_t sh[kCpThreads / 32 + 1];
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = begin + chunk < n ? begin + chunk : n;
  sel.block_setup(begin, end);
  uint32_t cnt = 0;
  for (uint64_t i = begin + threadIdx.x; i < end; i += kCpThreads) {
    bool f = sel.select(i);
    flags[i] = f ? 1 : 0;
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
                                                              const uint8_t* flags,
                                                              const uint64_t* offs) {
  __shared__ uint64_t sh[kCpThreads / 32 + 1];
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = begin + chunk < n ? begin + chunk : n;
  uint64_t base = offs[blockIdx.x];
  for (uint64_t tile = begin; tile < end; tile += kCpTile) {
    const uint64_t i0 = tile + (uint64_t)threadIdx.x * kCpItems;
    uint8_t f[kCpItems];
    if (i0 + kCpItems <= end) {
      uint2 v = *reinterpret_cast<const uint2*>(flags + i0);
#pragma unroll
      for (int j = 0; j < 4; j++) f[j] = (v.x >> (8 * j)) & 0xff;
#pragma unroll
      for (int j = 0; j < 4; j++) f[4 + j] = (v.y >> (8 * j)) & 0xff;
    } else {
#pragma unroll
      for (int j = 0; j < kCpItems; j++) f[j] = (i0 + j < end) ? flags[i0 + j] : 0;
    }
    uint64_t c = 0;
#pragma unroll
    for (int j = 0; j < kCpItems; j++) c += f[j];
    uint64_t tot;
    uint64_t pos = base + block_excl_scan(c, sh, &tot);
#pragma unroll
    for (int j = 0; j < kCpItems; j++)
      if (f[j]) sel.emit(i0 + j, pos++);
    base += tot;
  }
}

// Runs the three launches; the selected count lands in *d_total.
template <class Sel>
void compact(const Launch& L, Sel sel, uint64_t n, uint64_t* d_total, Scratch& s) {
  if (n == 0) {
    SRDL_CUDA(cudaMemsetAsync(d_total, 0, sizeof(uint64_t), L.stream));
    return;
  }
  const uint64_t chunk = cp_chunk(n, L.num_sms);
  const int nb = cp_blocks(n, chunk);
  uint8_t* flags = s.take<uint8_t>(n);
  uint32_t* counts = s.take<uint32_t>(nb);
  uint64_t* offs = s.take<uint64_t>(nb + 1);
  cp_flag_kernel<Sel><<<nb, kCpThreads, 0, L.stream>>>(sel, n, chunk, flags, counts);
  cp_scan_kernel<<<1, 1024, 0, L.stream>>>(counts, nb, offs, d_total);
  cp_write_kernel<Sel><<<nb, kCpThreads, 0, L.stream>>>(sel, n, chunk, flags, offs);
  SRDL_CUDA(cudaGetLastError());
  count_launches(3);
}

// Keeps a[i] when it differs from a[i-1] (optional) and is absent from the
// sorted unique array full[0..n_full).  Keys are stored compressed as
// (hi << bits) | lo and are expanded to (hi << 32) | lo on output.
template <typename K>
struct DedupDiffSel {
  const K* a;
  int bits;
  bool dedup;
  const uint64_t* full;
  uint64_t n_full;
  uint64_t* out;

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
  __device__ void emit(uint64_t i, uint64_t pos) const { out[pos] = expand(a[i]); }
};

// Flag pass of DedupDiffSel with FULL: the block walks its chunk one tile at
// a time; two warps locate the tile's slice of FULL (32-ary searches), the
// block stages the slice in shared memory when it fits, and every key is then
// probed by binary search in shared memory instead of global memory.
constexpr int kDdStage = 4096;  // FULL keys staged per tile (32 KB)

template <typename K>
__global__ void __launch_bounds__(kCpThreads) dd_flag_kernel(DedupDiffSel<K> sel, uint64_t n,
                                                             uint64_t chunk, uint8_t* flags,
                                                             uint32_t* blk_counts) {
  __shared__ uint64_t stage[kDdStage];
  __shared__ uint64_t rng[2];
  __shared__ uint32_t sh[kCpThreads / 32 + 1];
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = begin + chunk < n ? begin + chunk : n;
  const int wid = threadIdx.x >> 5;
  uint32_t cnt = 0;
  for (uint64_t tile = begin; tile < end; tile += kCpTile) {
    const uint64_t tend = tile + kCpTile < end ? tile + kCpTile : end;
    if (wid == 0) {
      const uint64_t first = sel.expand(sel.a[tile]);
      const uint64_t f0 = warp_partition_point(0, sel.n_full,
                                               [&](uint64_t i) { return sel.full[i] < first; });
      if ((threadIdx.x & 31) == 0) rng[0] = f0;
    } else if (wid == 1) {
      const uint64_t last = sel.expand(sel.a[tend - 1]);
      const uint64_t f1 = warp_partition_point(0, sel.n_full,
                                               [&](uint64_t i) { return sel.full[i] <= last; });
      if ((threadIdx.x & 31) == 0) rng[1] = f1;
    }
    __syncthreads();
    const uint64_t f0 = rng[0], f1 = rng[1];
    const uint64_t len = f1 > f0 ? f1 - f0 : 0;
    const bool staged = len <= (uint64_t)kDdStage;
    if (staged)
      for (uint64_t j = threadIdx.x; j < len; j += kCpThreads) stage[j] = sel.full[f0 + j];
    __syncthreads();
    for (uint64_t i = tile + threadIdx.x; i < tend; i += kCpThreads) {
      const K c = sel.a[i];
      bool keep = !(sel.dedup && i > 0 && sel.a[i - 1] == c);
      if (keep && len) {
        const uint64_t k = sel.expand(c);
        if (staged) {
          uint32_t lo = 0, hi = (uint32_t)len;
          while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (stage[mid] < k) lo = mid + 1;
            else hi = mid;
          }
          keep = !(lo < len && stage[lo] == k);
        } else {
          const uint64_t p = lower_bound_u64(sel.full, f0, f1, k);
          keep = !(p < f1 && sel.full[p] == k);
        }
      }
      flags[i] = keep ? 1 : 0;
      cnt += keep;
    }
    __syncthreads();
  }
  uint32_t tot;
  block_excl_scan(cnt, sh, &tot);
  if (threadIdx.x == 0) blk_counts[blockIdx.x] = tot;
}

// compact() for DedupDiffSel with a FULL array: tiled, shared-memory probes.
template <typename K>
void compact_diff(const Launch& L, DedupDiffSel<K> sel, uint64_t n, uint64_t* d_total, Scratch& s) {
  if (!sel.full || sel.n_full == 0) {
    compact(L, sel, n, d_total, s);
    return;
  }
  if (n == 0) {
    SRDL_CUDA(cudaMemsetAsync(d_total, 0, sizeof(uint64_t), L.stream));
    return;
  }
  const uint64_t chunk = cp_chunk(n, L.num_sms);
  const int nb = cp_blocks(n, chunk);
  uint8_t* flags = s.take<uint8_t>(n);
  uint32_t* counts = s.take<uint32_t>(nb);
  uint64_t* offs = s.take<uint64_t>(nb + 1);
  prefer_shared(dd_flag_kernel<K>);
  dd_flag_kernel<K><<<nb, kCpThreads, 0, L.stream>>>(sel, n, chunk, flags, counts);
  cp_scan_kernel<<<1, 1024, 0, L.stream>>>(counts, nb, offs, d_total);
  cp_write_kernel<DedupDiffSel<K>><<<nb, kCpThreads, 0, L.stream>>>(sel, n, chunk, flags, offs);
  SRDL_CUDA(cudaGetLastError());
  count_launches(3);
}

// Distinct first-column values of a sorted key array.
struct RootSel {
  const uint64_t* keys;
  uint32_t* roots;
  __device__ void block_setup(uint64_t, uint64_t) {}
  __device__ bool select(uint64_t i) const {
    return i == 0 || (keys[i] >> 32) != (keys[i - 1] >> 32);
  }
  __device__ void emit(uint64_t i, uint64_t pos) const { roots[pos] = (uint32_t)(keys[i] >> 32); }
};

}  // namespace srdl
