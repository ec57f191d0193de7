// instances.cu -- per-instance state of a batched run.
//
// A batched run evaluates many independent instances of one program as one
// database whose instance j owns the values [bounds[j], bounds[j+1]) (the
// host shifts each instance's values into its own range; no rule can join
// two ranges, so every tuple stays in the range of its first column).  All
// instances share every launch of an iteration; these kernels keep, on the
// device, what a one-instance-at-a-time run would report per instance:
//
//  * convergence -- after each iteration of a recursive step, the instances
//    that still have a delta row record the iteration (instance_mark_kernel,
//    one binary search per instance in each sorted delta).  The iterations
//    instance j's own run takes are min(T, last_j + 1) for a step that ran T
//    iterations: its run stops after the first iteration whose delta is
//    empty (the loop of step_N in src/srdatalog/codegen/jit/
//    orchestrator_jit.py:600-747), and an instance whose delta emptied
//    gains nothing from later iterations of the union.
//  * fingerprints -- per instance, the sum over its rows (x, y) of
//    mix_a(x - b_j) * mix_b(y - b_j) mod 2^64 (instance-local values), an
//    order-free digest of the row set that a checker can compute from any
//    representation of the expected relation (the product form lets it sum
//    per source over a reachability set without listing the pairs).
#include <algorithm>

#include "runtime.h"

namespace srdl {

namespace {

// SplitMix64 output function (Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014; the constants of Vigna's
// splitmix64.c): a bijective 64-bit mixer.
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ uint64_t row_fingerprint(uint32_t x, uint32_t y) {
  return splitmix64((uint64_t)x ^ 0x243F6A8885A308D3ull) * splitmix64((uint64_t)y ^ 0x13198A2E03707344ull);
}

// last[j] = max(last[j], iteration) for every instance j with a key of the
// sorted keys[0..n) (n = min(*n_dev, cap) when n_dev is given) whose high
// word lies in [bounds[j], bounds[j+1]).  iteration = base + *iter_dev.
__global__ void instance_mark_kernel(const uint64_t* __restrict__ keys, uint64_t cap,
                                     const uint64_t* __restrict__ n_dev, const uint32_t* __restrict__ bounds,
                                     uint32_t k, uint32_t base, const unsigned long long* __restrict__ iter_dev,
                                     uint32_t* __restrict__ last) {
  const uint64_t n = n_dev ? min(*n_dev, cap) : cap;
  if (!n) return;
  const uint32_t it = base + (iter_dev ? (uint32_t)*iter_dev : 0u);
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < k; j += gridDim.x * blockDim.x) {
    const uint64_t p = lower_bound_u64(keys, 0, n, (uint64_t)bounds[j] << 32);
    if (p < n && (uint32_t)(keys[p] >> 32) < bounds[j + 1] && last[j] < it) last[j] = it;
  }
}

// Rows per warp of the fingerprint kernel (contiguous, so that a lane's
// instance changes only at range boundaries).
constexpr uint64_t kFpChunk = 32 * 128;

// sums[j] += fingerprints of the rows in [pos[0], pos[k]) whose high word is
// in instance j's range (keys packed (y, x) when `swapped`).  Warps take chunks of consecutive rows; each lane
// keeps one running sum and adds it to its instance's total when the
// instance changes (once per range a chunk crosses).
__global__ void range_fingerprint_kernel(const uint64_t* __restrict__ keys, const uint64_t* __restrict__ pos,
                                         const uint32_t* __restrict__ bounds, uint32_t k, bool swapped,
                                         unsigned long long* __restrict__ sums) {
  const uint64_t lo = pos[0], hi = pos[k];
  if (hi <= lo) return;
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t c0 = lo + warp * kFpChunk; c0 < hi; c0 += warps * kFpChunk) {
    const uint64_t c1 = min(hi, c0 + kFpChunk);
    uint32_t cur = 0xFFFFFFFFu;
    uint64_t acc = 0;
    for (uint64_t i = c0 + lane; i < c1; i += 32) {
      const uint64_t key = keys[i];
      const uint32_t hw = (uint32_t)(key >> 32), lw = (uint32_t)key;
      const uint32_t x = swapped ? lw : hw, y = swapped ? hw : lw;
      // (both columns lie in the range of the instance; the sorted high
      // word finds it)
      if (cur == 0xFFFFFFFFu || hw >= bounds[cur + 1]) {
        if (cur != 0xFFFFFFFFu && acc) atomicAdd(&sums[cur], (unsigned long long)acc);
        // the instance owning x: the last j with bounds[j] <= x (rows lie in
        // [bounds[0], bounds[k]), so one exists; empty ranges are skipped)
        uint32_t a = cur == 0xFFFFFFFFu ? 0 : cur + 1, b = k;
        while (b - a > 1) {
          const uint32_t m = a + (b - a) / 2;
          if (bounds[m] <= hw) a = m;
          else b = m;
        }
        cur = a;
        acc = 0;
      }
      acc += row_fingerprint(x - bounds[cur], y - bounds[cur]);
    }
    if (cur != 0xFFFFFFFFu && acc) atomicAdd(&sums[cur], (unsigned long long)acc);
  }
}

int grid_of(uint64_t n, int per_block, int sms) {
  const uint64_t g = (n + per_block - 1) / per_block;
  const uint64_t cap = (uint64_t)sms * 16;
  return (int)std::max<uint64_t>(1, std::min(g, cap));
}

}  // namespace

void instance_mark(const Launch& L, const uint64_t* keys, uint64_t cap, const uint64_t* n_dev,
                   const uint32_t* bounds, uint32_t k, uint32_t base, const unsigned long long* iter_dev,
                   uint32_t* last) {
  if (!k || !cap) return;
  instance_mark_kernel<<<grid_of(k, 256, L.num_sms), 256, 0, L.stream>>>(keys, cap, n_dev, bounds, k, base,
                                                                         iter_dev, last);
  SRDL_CUDA(cudaGetLastError());
  count_launches(1);
}

void Database::set_instances(const uint32_t* bounds, uint64_t n_bounds) {
  inst_iters_.clear();
  inst_last_.clear();
  if (n_bounds == 0) {
    inst_bounds_.clear();
    return;
  }
  SRDL_REQUIRE(bounds && n_bounds >= 2 && n_bounds <= (1ull << 31), kErrArg,
               "set_instances: need 2 or more bounds");
  for (uint64_t j = 0; j + 1 < n_bounds; j++)
    SRDL_REQUIRE(bounds[j] <= bounds[j + 1], kErrArg, "set_instances: bounds must be non-decreasing");
  inst_bounds_.assign(bounds, bounds + n_bounds);
}

// Called at the start of a run: the bounds on the device and, for every
// recursive step whose computed relations are all binary, a zeroed array
// of last iterations.
void Database::instances_begin() {
  inst_iters_.clear();
  inst_last_.clear();
  inst_bounds_d_ = DevBuf();
  if (inst_bounds_.empty()) return;
  const uint64_t nb = inst_bounds_.size();
  inst_bounds_d_ = DevBuf(nb * 4, L_.stream);
  SRDL_CUDA(cudaMemcpyAsync(inst_bounds_d_.as<void>(), inst_bounds_.data(), nb * 4, cudaMemcpyHostToDevice,
                            L_.stream));
  for (size_t si = 0; si < steps_.size(); si++) {
    const Step& st = steps_[si];
    if (!st.recursive) continue;
    bool binary = true;
    for (auto& op : st.ops)
      if (op.kind == Op::ComputeDelta && rel(op.rel).arity != 2) binary = false;
    if (!binary) continue;
    DevBuf& last = inst_last_[si];
    last = DevBuf((nb - 1) * 4, L_.stream);
    SRDL_CUDA(cudaMemsetAsync(last.as<void>(), 0, (nb - 1) * 4, L_.stream));
  }
  // the host copy of the bounds stays alive (member); no sync needed
}

uint32_t* Database::instance_marks(size_t si) {
  auto it = inst_last_.find(si);
  return it == inst_last_.end() ? nullptr : it->second.as<uint32_t>();
}

// Host path: after iteration `iter` (1-based) of step si, mark the instances
// with a delta row in any relation the step computes.
void Database::mark_instances(size_t si, const Step& st, uint32_t iter) {
  uint32_t* last = instance_marks(si);
  if (!last) return;
  const uint32_t k = (uint32_t)(inst_bounds_.size() - 1);
  for (auto& op : st.ops) {
    if (op.kind != Op::ComputeDelta) continue;
    Relation& r = rel(op.rel);
    auto it = r.v[kDelta].idx.find(r.canonical);
    if (it == r.v[kDelta].idx.end() || !it->second.n) continue;
    instance_mark(L_, it->second.keys.as<uint64_t>(), it->second.n, nullptr, inst_bounds_d_.as<uint32_t>(), k,
                  iter, nullptr, last);
  }
}

// After step si ran T iterations: every instance's own iteration count.
void Database::instances_end(size_t si, uint64_t T) {
  uint32_t* last = instance_marks(si);
  if (!last) return;
  const uint64_t k = inst_bounds_.size() - 1;
  std::vector<uint32_t>& out = inst_iters_[si];
  out.assign(k, 0);
  SRDL_CUDA(cudaMemcpyAsync(out.data(), last, k * 4, cudaMemcpyDeviceToHost, L_.stream));
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
  for (auto& v : out) v = (uint32_t)std::min<uint64_t>(T, (uint64_t)v + 1);
}

void Database::instance_iterations(uint64_t step, uint32_t* out, uint64_t n_instances) const {
  SRDL_REQUIRE(!inst_bounds_.empty(), kErrArg, "instance_iterations: no instances set");
  SRDL_REQUIRE(n_instances == inst_bounds_.size() - 1, kErrArg, "instance_iterations: wrong instance count");
  SRDL_REQUIRE(step < steps_.size(), kErrArg, "instance_iterations: no such step");
  if (!steps_[step].recursive) {
    for (uint64_t j = 0; j < n_instances; j++) out[j] = step_stats_[step].iterations ? 1 : 0;
    return;
  }
  auto it = inst_iters_.find(step);
  SRDL_REQUIRE(it != inst_iters_.end(), kErrUnsupported,
               "instance_iterations: not recorded for this step (not run since the instances were set, or a "
               "relation it computes is not binary)");
  std::copy(it->second.begin(), it->second.end(), out);
}

// A FULL index of binary relation r (the canonical permutation when it
// exists, else the first built; identity built when there is none);
// *swapped: its keys are packed (column 1, column 0).
Index& Database::binary_full_index(Relation& r, bool* swapped) {
  auto& fv = r.v[kFull];
  auto it = fv.idx.find(r.canonical);
  if (it == fv.idx.end()) it = fv.idx.begin();
  if (it == fv.idx.end()) {
    if (swapped) *swapped = false;
    return ensure_index(r, kFull, identity_perm(2));
  }
  if (swapped) *swapped = it->first.size() == 2 && it->first[0] == 1;
  return it->second;
}

void Database::range_checksums(const std::string& name, const uint32_t* bounds, uint64_t n_bounds,
                               uint64_t* sums) {
  Relation& r = rel(name);
  SRDL_REQUIRE(bounds || n_bounds == 0, kErrArg, "range_checksums: null bounds");
  if (n_bounds < 2) return;
  SRDL_REQUIRE(n_bounds <= (1ull << 31), kErrArg, "range_checksums: too many bounds");
  for (uint64_t j = 0; j + 1 < n_bounds; j++)
    SRDL_REQUIRE(bounds[j] <= bounds[j + 1], kErrArg, "range_checksums: bounds must be non-decreasing");
  SRDL_REQUIRE(r.arity == 2, kErrUnsupported, "range_checksums: binary relations only");
  const uint64_t k = n_bounds - 1;
  if (r.head.n) compact_head(r);
  if (!r.v[kFull].has_index()) {
    for (uint64_t j = 0; j < k; j++) sums[j] = 0;
    return;
  }
  SRDL_CUDA(cudaSetDevice(device_));
  bool swapped = false;
  Index& ix = binary_full_index(r, &swapped);
  DevBuf d_bounds(n_bounds * 4, L_.stream);
  DevBuf d_pos(n_bounds * 8, L_.stream);
  DevBuf d_sums(k * 8, L_.stream);
  SRDL_CUDA(cudaMemcpyAsync(d_bounds.as<void>(), bounds, n_bounds * 4, cudaMemcpyHostToDevice, L_.stream));
  SRDL_CUDA(cudaMemsetAsync(d_sums.as<void>(), 0, k * 8, L_.stream));
  bounds_positions(L_, ix.keys.as<uint64_t>(), ix.n, d_bounds.as<uint32_t>(), n_bounds, d_pos.as<uint64_t>());
  if (ix.n) {
    range_fingerprint_kernel<<<grid_of(ix.n, (int)(8 * kFpChunk), L_.num_sms), 256, 0,
                               L_.stream>>>(ix.keys.as<uint64_t>(), d_pos.as<uint64_t>(),
                                            d_bounds.as<uint32_t>(), (uint32_t)k, swapped,
                                            d_sums.as<unsigned long long>());
    SRDL_CUDA(cudaGetLastError());
    count_launches(1);
  }
  SRDL_CUDA(cudaMemcpyAsync(sums, d_sums.as<void>(), k * 8, cudaMemcpyDeviceToHost, L_.stream));
  SRDL_CUDA(cudaStreamSynchronize(L_.stream));
}

}  // namespace srdl
