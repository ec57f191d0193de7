// sort.cu -- index build: LSD radix sort of packed keys + fused dedup / difference.
//
// Replaces rebuild_index_fn -> zip_sort_columns (thrust::sort on a zip
// iterator, a CUB merge sort: RT/gpu/sort.h:297-302) followed by
// deduplicate_aggregate_and_unique (RT/gpu/deduplication.h:178-258) and, for
// ComputeDeltaIndex, DSAI::set_difference_update
// (RT/gpu/device_sorted_array_index.ipp:966-1130).
//
// Design.  Datalog creates no values: every value of every relation comes
// from the loaded inputs (and rule constants), so the runtime knows a bound
// 2^bits on all values.  A two-column key (hi, lo) is compressed to
// (hi << bits) | lo -- 32 bits when 2*bits <= 32 -- and sorted with
// ceil(2*bits / 8) stable counting passes (digits of at most Launch::radix_bits).  Each pass is a histogram launch
// (shared-memory counters per block), a per-digit scan over the blocks, and a
// scatter launch in which every warp ranks its keys with one ballot per digit
// bit, the tile is staged in shared memory in digit order and written out
// coalesced.  No
// block ever waits on another.  The dedup (and optional "not in FULL" test)
// runs as one order-preserving compaction over the sorted keys that also
// expands them back to (hi << 32) | lo.
#include "compact.cuh"
#include "kernels.h"

namespace srdl {

constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsPerWarp = 256;                  // keys per warp per tile
constexpr int kRsTile = kRsWarps * kRsPerWarp;   // 2048 keys per tile
constexpr int kRsBins = 256;
static_assert(kRsThreads == kRsBins, "one thread per digit in the per-tile digit loops");

int value_bits(uint32_t max_value) {
  int b = 0;
  while (b < 32 && (uint64_t(max_value) >> b) != 0) b++;
  return b ? b : 1;
}

__global__ void cp_scan_kernel(const uint32_t* blk_counts, int nb, uint64_t* offs,
                               uint64_t* d_total) {
  __shared__ uint64_t sh[1024 / 32 + 1];
  const int per = (nb + blockDim.x - 1) / blockDim.x;
  const int s = threadIdx.x * per, e = min(nb, s + per);
  uint64_t sum = 0;
  for (int i = s; i < e; i++) sum += blk_counts[i];
  uint64_t tot;
  uint64_t run = block_excl_scan(sum, sh, &tot);
  for (int i = s; i < e; i++) {
    offs[i] = run;
    run += blk_counts[i];
  }
  if (threadIdx.x == 0) {
    offs[nb] = tot;
    *d_total = tot;
  }
}

template <typename K>
__global__ void rs_pack(const uint64_t* __restrict__ in, uint64_t n, int bits, bool swap,
                        K* __restrict__ out, const uint64_t* d_n) {
  n = dev_size(n, d_n);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t k = in[i];
    uint64_t hi = k >> 32, lo = k & 0xffffffffull;
    if (swap) {
      uint64_t t = hi;
      hi = lo;
      lo = t;
    }
    out[i] = (K)((hi << bits) | lo);
  }
}

template <typename K>
__global__ void __launch_bounds__(kRsThreads) rs_hist(const K* __restrict__ keys, uint64_t n,
                                                      uint64_t chunk, int shift, int nbins,
                                                      uint32_t* __restrict__ counts,
                                                      const uint64_t* d_n) {
  __shared__ uint32_t h[kRsBins];
  n = dev_size(n, d_n);
  chunk = dev_chunk(chunk, n, kRsTile);
  for (int d = threadIdx.x; d < nbins; d += kRsThreads) h[d] = 0;
  __syncthreads();
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = begin + chunk < n ? begin + chunk : n;
  const uint32_t mask = nbins - 1;
  // 16-byte loads: the chunk starts a multiple of kRsTile keys into a
  // 256-byte aligned array; a ragged tail is read key by key.
  constexpr uint64_t kPer = 16 / sizeof(K);
  const uint64_t vend = begin < end ? begin + (end - begin) / kPer * kPer : begin;
  const uint4* vec = reinterpret_cast<const uint4*>(keys + begin);
  for (uint64_t q = threadIdx.x; begin + q * kPer < vend; q += kRsThreads) {
    const uint4 v = __ldg(vec + q);
    if constexpr (sizeof(K) == 8) {
      const uint64_t k0 = ((uint64_t)v.y << 32) | v.x, k1 = ((uint64_t)v.w << 32) | v.z;
      atomicAdd(&h[(uint32_t)(k0 >> shift) & mask], 1u);
      atomicAdd(&h[(uint32_t)(k1 >> shift) & mask], 1u);
    } else {
      atomicAdd(&h[(v.x >> shift) & mask], 1u);
      atomicAdd(&h[(v.y >> shift) & mask], 1u);
      atomicAdd(&h[(v.z >> shift) & mask], 1u);
      atomicAdd(&h[(v.w >> shift) & mask], 1u);
    }
  }
  for (uint64_t i = vend + threadIdx.x; i < end; i += kRsThreads)
    atomicAdd(&h[(uint32_t)(keys[i] >> shift) & mask], 1u);
  __syncthreads();
  for (int d = threadIdx.x; d < nbins; d += kRsThreads) counts[(uint64_t)d * gridDim.x + blockIdx.x] = h[d];
}

// Block d turns row d of the digit-major counters (one counter per
// histogram block) into exclusive offsets within the digit, in place, and
// writes the digit's total to digit_tot[d].
__global__ void __launch_bounds__(kRsThreads) rs_rowscan(uint32_t* c, int nb,
                                                         uint32_t* __restrict__ digit_tot) {
  __shared__ uint32_t sh[kRsThreads / 32 + 1];
  uint32_t* row = c + (uint64_t)blockIdx.x * nb;
  const int per = (nb + kRsThreads - 1) / kRsThreads;
  const int s = threadIdx.x * per, e = min(nb, s + per);
  uint32_t sum = 0;
  for (int i = s; i < e; i++) sum += row[i];
  uint32_t tot;
  uint32_t run = block_excl_scan(sum, sh, &tot);
  for (int i = s; i < e; i++) {
    uint32_t v = row[i];
    row[i] = run;
    run += v;
  }
  if (threadIdx.x == 0) digit_tot[blockIdx.x] = tot;
}

// Asynchronous 16-byte global -> shared copy (cp.async, no registers held);
// bytes past `src_bytes` (< 16 on a ragged tail) are zero-filled.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, uint32_t src_bytes) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Issue the copy of keys [tile, min(tile + kRsTile, end)) into `buf`.  Tile
// starts are multiples of kRsTile keys from a 256-byte aligned buffer, so
// every 16-byte piece is aligned; a piece that straddles `end` copies only
// the valid bytes, and pieces past it copy nothing.
template <typename K>
__device__ __forceinline__ void rs_prefetch(K* buf, const K* in, uint64_t tile, uint64_t end) {
  constexpr int kPieces = kRsTile * (int)sizeof(K) / 16;
  const uint64_t valid_bytes = (end > tile ? end - tile : 0) * sizeof(K);
  const char* src = reinterpret_cast<const char*>(in + tile);
  char* dst = reinterpret_cast<char*>(buf);
  for (int p = threadIdx.x; p < kPieces; p += kRsThreads) {
    const uint64_t off = (uint64_t)p * 16;
    const uint64_t left = off >= valid_bytes ? 0 : valid_bytes - off;
    const uint32_t nb = left < 16 ? (uint32_t)left : 16u;
    cp_async16(dst + off, nb ? src + off : src, nb);
  }
  cp_async_commit();
}

// One counting pass over this block's chunk, a tile of kRsTile keys at a
// time, for digits of DB bits.  The next tile is copied into the other shared
// buffer while the current one is ranked and written, so every block keeps a
// tile of loads in flight.  Within a warp, the lanes holding the same digit
// are found with DB ballots (one per digit bit), which is cheaper than a
// match instruction; the lowest such lane adds the group's size to the warp's
// counter for the digit and passes the old value on.  The staged
// (digit-ordered) tile reuses the buffer the current keys were read from.
// Five resident blocks per SM (their shared memory fits; the register cap
// that needs costs no spills).
template <typename K, int DB>
__global__ void __launch_bounds__(kRsThreads, 5) rs_scatter(const K* __restrict__ in,
                                                         K* __restrict__ out, uint64_t n,
                                                         uint64_t chunk, int shift,
                                                         const uint32_t* __restrict__ offs,
                                                         const uint32_t* __restrict__ digit_tot,
                                                         const uint64_t* d_n) {
  constexpr int nbins = 1 << DB;
  constexpr uint32_t mask = nbins - 1;
  __shared__ uint32_t base[kRsBins];             // next global output position per digit
  __shared__ uint32_t gofs[kRsBins];             // base[d] minus the digit's start in the staged tile
  __shared__ uint32_t wofs[kRsWarps][kRsBins];   // per-warp digit counts -> staged positions
  __shared__ uint32_t scan_sh[kRsThreads / 32 + 1];
  __shared__ __align__(16) K buf[2][kRsTile];

  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  n = dev_size(n, d_n);
  chunk = dev_chunk(chunk, n, kRsTile);
  const uint64_t begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t end = begin + chunk < n ? begin + chunk : n;
  if (begin < end) rs_prefetch(buf[0], in, begin, end);
  {
    // digit base = keys with a smaller digit; plus this block's offset in the digit
    const int d = threadIdx.x;  // kRsThreads == kRsBins
    const uint32_t t = d < nbins ? digit_tot[d] : 0;
    uint32_t all;
    const uint32_t dbase = block_excl_scan(t, scan_sh, &all);
    base[d] = d < nbins ? dbase + offs[(uint64_t)d * gridDim.x + blockIdx.x] : 0;
  }

  const unsigned lt = lanemask_lt();
  int cur = 0;
  for (uint64_t tile = begin; tile < end; tile += kRsTile, cur ^= 1) {
#pragma unroll
    for (int w = 0; w < kRsWarps; w++) wofs[w][threadIdx.x] = 0;
    const uint64_t next = tile + kRsTile;
    if (next < end) {
      rs_prefetch(buf[cur ^ 1], in, next, end);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const uint32_t cnt = (uint32_t)((end - tile) < kRsTile ? (end - tile) : kRsTile);
    K key[kRsPerWarp / 32];
    uint32_t rank[kRsPerWarp / 32];  // rank in the warp's digit run | digit << 16
    // Warp `wid` owns keys [wid*256, +256) of the tile in rounds of 32, so the
    // (round, lane) order is the input order.  Each round's counter update
    // precedes the next round's (__syncwarp orders them): ranks are stable.
#pragma unroll
    for (int r = 0; r < kRsPerWarp / 32; r++) {
      const uint32_t j = (uint32_t)wid * kRsPerWarp + r * 32 + lane;
      const bool valid = j < cnt;
      key[r] = buf[cur][j];
      const uint32_t d = (uint32_t)(key[r] >> shift) & mask;
      unsigned peers = __ballot_sync(kAllLanes, valid);
#pragma unroll
      for (int b = 0; b < DB; b++) {
        const bool bit = (d >> b) & 1u;
        const unsigned m = __ballot_sync(kAllLanes, bit);
        peers &= bit ? m : ~m;
      }
      // invalid lanes (a ragged last tile) get an empty group and lane 0 as leader
      peers = valid ? peers : 0u;
      const int leader = valid ? __ffs(peers) - 1 : 0;
      uint32_t old = 0;
      if (valid && lane == leader) old = atomicAdd(&wofs[wid][d], (uint32_t)__popc(peers));
      old = __shfl_sync(kAllLanes, old, leader);
      rank[r] = valid ? (old + __popc(peers & lt)) | (d << 16) : 0xffffffffu;
      __syncwarp();
    }
    __syncthreads();
    // Per digit: staged start of each warp's run (tile start of the digit plus
    // the earlier warps' counts), and the global offset of the digit's run.
    {
      const int d = threadIdx.x;  // kRsThreads == kRsBins
      uint32_t c[kRsWarps], run = 0;
#pragma unroll
      for (int w = 0; w < kRsWarps; w++) {
        c[w] = wofs[w][d];
        run += c[w];
      }
      uint32_t all;
      uint32_t start = block_excl_scan(run, scan_sh, &all);
      gofs[d] = base[d] - start;
      base[d] += run;
#pragma unroll
      for (int w = 0; w < kRsWarps; w++) {
        wofs[w][d] = start;
        start += c[w];
      }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRsPerWarp / 32; r++) {
      if (rank[r] != 0xffffffffu) buf[cur][wofs[wid][rank[r] >> 16] + (rank[r] & 0xffffu)] = key[r];
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < cnt; j += kRsThreads) {
      const K k = buf[cur][j];
      out[gofs[(uint32_t)(k >> shift) & mask] + j] = k;
    }
    __syncthreads();
  }
}

template <typename K>
static void launch_scatter(const Launch& L, int nb, int w, const K* in, K* out, uint64_t n,
                           uint64_t chunk, int shift, const uint32_t* offs,
                           const uint32_t* digit_tot, const uint64_t* d_n) {
#define SRDL_SCATTER_CASE(DB)                                                          \
  case DB:                                                                             \
    prefer_shared(rs_scatter<K, DB>);                                                  \
    rs_scatter<K, DB><<<nb, kRsThreads, 0, L.stream>>>(in, out, n, chunk, shift, offs, \
                                                       digit_tot, d_n);                \
    break;
  switch (w) {
    SRDL_SCATTER_CASE(1)
    SRDL_SCATTER_CASE(2)
    SRDL_SCATTER_CASE(3)
    SRDL_SCATTER_CASE(4)
    SRDL_SCATTER_CASE(5)
    SRDL_SCATTER_CASE(6)
    SRDL_SCATTER_CASE(7)
    SRDL_SCATTER_CASE(8)
    default:
      throw Error{kErrState, "radix sort: digit width out of range"};
  }
#undef SRDL_SCATTER_CASE
}

static inline bool use32(int bits) { return 2 * bits <= 32; }

size_t sort_dev_scratch_bytes(uint64_t cap, uint64_t full_cap, int bits) {
  return sort_scratch_bytes(cap, bits) + diff_dev_extra_bytes(cap, full_cap);
}

size_t sort_scratch_bytes(uint64_t n, int bits) {
  const size_t ks = use32(bits) ? 4 : 8;
  const size_t counts = (size_t)kRsBins * 256 * 8 * 4;  // <= 8 blocks per SM, 256 SMs
  return 2 * (((n * ks) + 255) & ~size_t(255)) + counts + 2048 + cp_scratch_bytes(n) + 1024;
}

template <typename K>
static void sort_dedup_t(const Launch& L, const uint64_t* in, uint64_t n, int bits, bool swap,
                         const uint64_t* full, uint64_t n_full, uint64_t* out,
                         uint64_t* d_nout, Scratch& s, const uint64_t* head, uint64_t n_head,
                         const uint64_t* d_n, const uint64_t* d_n_full, uint64_t out_cap = ~0ull,
                         unsigned int* d_overflow = nullptr) {
  SRDL_REQUIRE(n < (1ull << 32), kErrCapacity, "sort: more than 2^32-1 rows in one index");
  K* a = s.take<K>(n);
  K* b = s.take<K>(n);
  const int pgrid = (int)std::min<uint64_t>((n + 255) / 256, (uint64_t)L.num_sms * 16);
  rs_pack<K><<<pgrid ? pgrid : 1, 256, 0, L.stream>>>(in, n, bits, swap, a, d_n);
  SRDL_CUDA(cudaGetLastError());
  count_launches(1);

  // Tile partition shared by the histogram and scatter launches (with the
  // count on the device, the blocks derive the same even split from it).
  const uint64_t tiles = (n + kRsTile - 1) / kRsTile;
  const uint64_t cap = (uint64_t)L.num_sms * 8;
  const uint64_t per = (tiles + cap - 1) / cap;
  const uint64_t chunk = (per ? per : 1) * kRsTile;
  const int nb = (int)((n + chunk - 1) / chunk);
  const uint64_t kchunk = d_n ? 0 : chunk;
  uint32_t* counts = s.take<uint32_t>((size_t)kRsBins * nb);
  uint32_t* digit_tot = s.take<uint32_t>(kRsBins);

  const int total_bits = 2 * bits;
  const int maxw = L.radix_bits >= 1 && L.radix_bits <= 8 ? L.radix_bits : 8;
  const int passes = (total_bits + maxw - 1) / maxw;
  int shift = 0;
  for (int p = 0; p < passes && (n > 1 || d_n); p++) {
    const int w = total_bits / passes + (p < total_bits % passes ? 1 : 0);
    const int nbins = 1 << w;
    rs_hist<K><<<nb, kRsThreads, 0, L.stream>>>(a, n, kchunk, shift, nbins, counts, d_n);
    rs_rowscan<<<nbins, kRsThreads, 0, L.stream>>>(counts, nb, digit_tot);
    launch_scatter<K>(L, nb, w, a, b, n, kchunk, shift, counts, digit_tot, d_n);
    SRDL_CUDA(cudaGetLastError());
    count_launches(3);
    std::swap(a, b);
    shift += w;
  }
  DedupDiffSel<K> sel{a, bits, true, full, n_full, out, head, n_head};
  sel.d_n_full = d_n_full;
  sel.out_cap = out_cap;
  sel.d_overflow = d_overflow;
  if (d_n) compact_diff_dev(L, sel, n, d_n, d_nout, s);
  else compact_diff(L, sel, n, d_nout, s);
}

void sort_dedup(const Launch& L, const uint64_t* in, uint64_t n, int bits, bool swap,
                const uint64_t* full, uint64_t n_full, uint64_t* out, uint64_t* d_nout,
                Scratch& s, const uint64_t* head, uint64_t n_head) {
  if (n == 0) {
    SRDL_CUDA(cudaMemsetAsync(d_nout, 0, sizeof(uint64_t), L.stream));
    return;
  }
  if (use32(bits))
    sort_dedup_t<uint32_t>(L, in, n, bits, swap, full, n_full, out, d_nout, s, head, n_head,
                           nullptr, nullptr);
  else sort_dedup_t<uint64_t>(L, in, n, bits, swap, full, n_full, out, d_nout, s, head, n_head,
                              nullptr, nullptr);
}

template <typename K>
static void warm_sort_kernels() {
  prefer_shared(rs_scatter<K, 1>);
  prefer_shared(rs_scatter<K, 2>);
  prefer_shared(rs_scatter<K, 3>);
  prefer_shared(rs_scatter<K, 4>);
  prefer_shared(rs_scatter<K, 5>);
  prefer_shared(rs_scatter<K, 6>);
  prefer_shared(rs_scatter<K, 7>);
  prefer_shared(rs_scatter<K, 8>);
  prefer_shared(dd_flag_kernel<K>);
}

void warm_device_loop_kernels(int bits) {
  if (use32(bits)) warm_sort_kernels<uint32_t>();
  else warm_sort_kernels<uint64_t>();
  warm_merge_kernels();
}

void sort_dedup_dev(const Launch& L, const uint64_t* in, uint64_t cap, const uint64_t* d_n,
                    int bits, const uint64_t* full, uint64_t full_cap, const uint64_t* d_n_full,
                    uint64_t* out, uint64_t out_cap, uint64_t* d_nout, unsigned int* d_overflow,
                    Scratch& s) {
  cap = cap ? cap : 1;
  if (use32(bits))
    sort_dedup_t<uint32_t>(L, in, cap, bits, false, full, full_cap, out, d_nout, s, nullptr, 0, d_n,
                           d_n_full, out_cap, d_overflow);
  else sort_dedup_t<uint64_t>(L, in, cap, bits, false, full, full_cap, out, d_nout, s, nullptr, 0,
                              d_n, d_n_full, out_cap, d_overflow);
}

}  // namespace srdl
