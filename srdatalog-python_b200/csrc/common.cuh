// common.cuh -- shared definitions for the srdl sm_100a runtime.
//
// Data layout in HBM.  Every materialised relation version holds ONE
// sorted, duplicate-free array of uint64 keys per index permutation:
//     key = (value of index column 0) << 32 | (value of index column 1)
// which is the lexicographic order of the reference's column-major sorted
// arrays (src/srdatalog/runtime/generalized_datalog/gpu/device_sorted_array_index.h:337).
// Joins additionally read a "trie view" of an index: the child column as a
// dense uint32 array, the distinct first-column values (roots) and, when the
// value domain is small, a dense directory dir[v] = first row whose first
// column is >= v, so that the rows with prefix v are [dir[v], dir[v+1]).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace srdl {

constexpr int kWarp = 32;
constexpr unsigned kAllLanes = 0xffffffffu;

// Status codes returned through the C ABI.
enum Status : int {
  kOk = 0,
  kErrArg = 1,
  kErrState = 2,
  kErrCuda = 3,
  kErrPlan = 4,
  kErrCapacity = 5,
  kErrIo = 6,
  kErrUnsupported = 7,
  kErrTimeout = 8,
};

void set_error(const std::string& msg);
const char* last_error();

struct Error {
  int code;
  std::string msg;
};

#define SRDL_CUDA(call)                                                             \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess)                                                          \
      throw ::srdl::Error{::srdl::kErrCuda, std::string(#call) + ": " +             \
                                                cudaGetErrorString(e_) + " at " +   \
                                                __FILE__ + ":" + std::to_string(__LINE__)}; \
  } while (0)

#define SRDL_REQUIRE(cond, code, msg)                                 \
  do {                                                                \
    if (!(cond)) throw ::srdl::Error{(code), std::string(msg)};       \
  } while (0)

// Read-only view of one sorted index used by the join kernels.
struct TrieView {
  const uint64_t* keys = nullptr;   // n sorted unique keys
  const uint32_t* lo = nullptr;     // n child values (low words of keys)
  const uint32_t* roots = nullptr;  // n_roots distinct first-column values
  const uint32_t* dir = nullptr;    // dense directory, dir_n = domain + 2 entries, or null
  // Hashed child lists (dense directory only): hdir[v] = first slot of the
  // open-addressing table holding the children of v, or kNoHash; the table
  // has hash_cap(len) slots for a list of len children.
  const uint32_t* hdir = nullptr;
  const uint32_t* hpool = nullptr;
  // Bitmaps of long child lists (dense directory only): bdir[v] = bitmap slot
  // of v's children or kNoBitmap; bitmap s is bpool[s*bwords .. +bwords), bit
  // c set iff (v, c) is a key.
  const uint32_t* bdir = nullptr;
  const uint32_t* bpool = nullptr;
  uint32_t bwords = 0;
  uint32_t bslots = 0;  // bitmaps in bpool
  uint64_t n = 0;
  const uint64_t* n_roots_d = nullptr;  // device-resident root count
  uint32_t dir_n = 0;
  int arity = 2;
};

__device__ __forceinline__ uint64_t lower_bound_u64(const uint64_t* a, uint64_t lo,
                                                    uint64_t hi, uint64_t key) {
  while (lo < hi) {
    uint64_t mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// lower_bound in [lo, hi) for a key known to be >= a[lo - 1]'s key: gallop
// forward from lo (1, 2, 4, ... steps), then binary-search the last gap.
__device__ __forceinline__ uint64_t gallop_lower_bound_u64(const uint64_t* a, uint64_t lo,
                                                           uint64_t hi, uint64_t key) {
  uint64_t step = 1, prev = lo;
  while (lo < hi && a[lo] < key) {
    prev = lo + 1;
    lo = lo + step < hi ? lo + step : hi;
    step <<= 1;
  }
  return lower_bound_u64(a, prev, lo, key);
}

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* a, uint32_t lo,
                                                    uint32_t hi, uint32_t key) {
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Rows whose first index column equals v: [b, e).  Same contract as
// NodeHandle::prefix (RT/gpu/device_sorted_array_index.ipp:67-157) for a
// two-column index.
__device__ __forceinline__ void trie_range(const TrieView& t, uint32_t v, uint32_t& b,
                                           uint32_t& e) {
  if (t.dir) {
    if (v + 1u < t.dir_n) {
      b = t.dir[v];
      e = t.dir[v + 1];
    } else {
      b = e = 0;
    }
  } else {
    uint64_t k0 = (uint64_t)v << 32;
    b = (uint32_t)lower_bound_u64(t.keys, 0, t.n, k0);
    e = (v == 0xffffffffu) ? (uint32_t)t.n
                           : (uint32_t)lower_bound_u64(t.keys, b, t.n, k0 + (1ull << 32));
  }
}

constexpr uint32_t kNoHash = 0xffffffffu;
constexpr uint32_t kNoBitmap = 0xffffffffu;
constexpr uint32_t kHashEmpty = 0xffffffffu;

// log2 of the table size for a list of len children: load factor <= 1/2.
__host__ __device__ __forceinline__ int hash_log2(uint32_t len) {
  int k = 1;
  while ((1u << k) < 2u * len) k++;
  return k;
}

__host__ __device__ __forceinline__ uint32_t hash_slot(uint32_t x, int k) {
  return (uint32_t)(((uint64_t)x * 0x9E3779B97F4A7C15ull) >> (64 - k));
}

// Owner of key value v among `world` shards: a multiplicative hash scaled to
// [0, world), so consecutive ids spread evenly.  The Python host layer
// (shard.owner) computes the same function.
__host__ __device__ __forceinline__ uint32_t shard_owner(uint32_t v, uint32_t world) {
  return (uint32_t)(((uint64_t)(v * 0x9E3779B1u) * world) >> 32);
}

__device__ __forceinline__ bool trie_has_root(const TrieView& t, uint32_t v) {
  uint32_t b, e;
  trie_range(t, v, b, e);
  return b < e;
}

// Is v among child values lo[b..e)?
__device__ __forceinline__ bool child_contains(const TrieView& t, uint32_t b, uint32_t e,
                                               uint32_t v) {
  uint32_t p = lower_bound_u32(t.lo, b, e, v);
  return p < e && t.lo[p] == v;
}

// Is v a child of prefix value pv?  Long lists answer from their hash table
// (about two dependent loads), short ones by binary search.
__device__ __forceinline__ bool trie_child_contains(const TrieView& t, uint32_t pv, uint32_t v) {
  uint32_t b, e;
  trie_range(t, pv, b, e);
  if (b == e) return false;
  if (t.hdir) {
    const uint32_t off = t.hdir[pv];
    if (off != kNoHash) {
      const int k = hash_log2(e - b);
      const uint32_t mask = (1u << k) - 1;
      uint32_t h = hash_slot(v, k);
      for (uint32_t probe = 0; probe <= mask; probe++) {
        const uint32_t s = t.hpool[off + h];
        if (s == v) return true;
        if (s == kHashEmpty) return false;
        h = (h + 1) & mask;
      }
      return false;
    }
  }
  return child_contains(t, b, e, v);
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T y = __shfl_up_sync(kAllLanes, v, d);
    if (lane >= d) v += y;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(kAllLanes, v, d);
  return v;
}

// Exclusive block scan; `sh` must hold blockDim.x/32 + 1 elements.  Returns
// the exclusive prefix of v and writes the block total into *total.
template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* sh, T* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  T inc = warp_incl_scan(v);
  if (lane == 31) sh[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    T s = lane < nw ? sh[lane] : T(0);
    T si = warp_incl_scan(s);
    if (lane < nw) sh[lane] = si - s;
    if (lane == nw - 1) sh[nw] = si;
  }
  __syncthreads();
  T r = sh[wid] + inc - v;
  *total = sh[nw];
  __syncthreads();
  return r;
}

// First i in [lo, hi) where pred(i) is false, for a predicate that is true
// on a prefix; called by all 32 lanes of a warp.  Each round tests 32 evenly
// spaced positions, so the number of dependent load rounds is log32(hi-lo).
template <class Pred>
__device__ __forceinline__ uint64_t warp_partition_point(uint64_t lo, uint64_t hi, Pred pred) {
  const int lane = threadIdx.x & 31;
  while (hi - lo > 32) {
    const uint64_t step = (hi - lo + 31) / 32;
    const uint64_t i = lo + lane * step;
    const bool p = i < hi && pred(i);
    const int k = __popc(__ballot_sync(kAllLanes, p));
    const uint64_t nlo = k > 0 ? lo + (uint64_t)(k - 1) * step + 1 : lo;
    const uint64_t cand = lo + (uint64_t)k * step;
    hi = cand < hi ? cand : hi;
    lo = nlo;
  }
  const uint64_t i = lo + lane;
  const bool p = i < hi && pred(i);
  return lo + __popc(__ballot_sync(kAllLanes, p));
}

inline int div_up(uint64_t a, uint64_t b) { return (int)((a + b - 1) / b); }

// Device-resident sizes (the device loop): a kernel given a capacity `cap`
// and a count d_n on the device works on min(cap, *d_n) items; without d_n,
// on cap.  Grids are sized for the capacity on the host.
__device__ __forceinline__ uint64_t dev_size(uint64_t cap, const uint64_t* d_n) {
  if (!d_n) return cap;
  const uint64_t n = *d_n;
  return n < cap ? n : cap;
}

// Items per block when `gridDim.x` blocks share n items in whole tiles: the
// host's value, or, when it passes 0 (n known on the device only), the same
// even split derived on the device.
__device__ __forceinline__ uint64_t dev_chunk(uint64_t chunk, uint64_t n, uint64_t tile) {
  if (chunk) return chunk;
  const uint64_t tiles = (n + tile - 1) / tile;
  const uint64_t per = (tiles + gridDim.x - 1) / gridDim.x;
  return (per ? per : 1) * tile;
}

}  // namespace srdl
