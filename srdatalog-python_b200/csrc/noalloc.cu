// noalloc.cu -- index build (sort + dedup) without any device allocation.
//
// Some callers may not allocate device memory on their call path: a host
// engine whose memory manager owns every device allocation and has planned
// the budget up front, or a latency-critical caller for which cudaMalloc's
// implicit synchronisation and fragmentation are unacceptable.  For them,
// srdl_sort_unique_u64_noalloc runs the same kernels as srdl_sort_unique_u64
// but takes its temporaries from one file-scope device array of fixed size,
// which every GPU that loads this library holds until the process exits.
//
// Host code cannot use the array's name as a device address (on the host it
// names a stand-in), so the first call on each device, with that device
// current, resolves the address with cudaGetSymbolAddress and caches it.
// That first call should therefore come before any stream capture.  The
// cached address belongs to the device's current context: it does not
// survive cudaDeviceReset (or any other teardown of the primary context), so
// a process that resets a device must not call this entry point on that
// device afterwards.  Calls that overlap on the GPU share the array and
// race; serialise them (one stream, or events).  Every scratch word is
// written before it is read, so nothing needs clearing between calls.
#include <mutex>

#include "../../include/srdl.h"
#include "kernels.h"

namespace {

constexpr uint64_t kNoAllocMaxKeys = 1ull << 20;             // 1,048,576 keys
constexpr size_t kNoAllocScratchBytes = 20ull << 20;         // 20 MiB
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_sort_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {};

}  // namespace

extern "C" {

uint64_t srdl_sort_unique_noalloc_max_keys(void) { return kNoAllocMaxKeys; }

int srdl_sort_unique_u64_noalloc(const uint64_t* d_in, uint64_t n, int value_bits,
                                 uint64_t* d_out, uint64_t* d_n_out, void* stream) {
  using namespace srdl;
  if ((!d_in && n) || !d_out || !d_n_out || value_bits < 1 || value_bits > 32) {
    set_error("srdl_sort_unique_u64_noalloc: bad argument");
    return kErrArg;
  }
  if (n > kNoAllocMaxKeys) {
    set_error("srdl_sort_unique_u64_noalloc: " + std::to_string(n) +
              " keys exceed the static scratch limit of " + std::to_string(kNoAllocMaxKeys) +
              " keys; use srdl_sort_unique_u64 with caller scratch");
    return kErrCapacity;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_error(std::string("srdl_sort_unique_u64_noalloc: no usable current device: ") +
              cudaGetErrorString(e));
    return kErrCuda;
  }
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_sort_scratch);
      if (e != cudaSuccess || !p) {
        set_error(std::string("srdl_sort_unique_u64_noalloc: cudaGetSymbolAddress failed: ") +
                  cudaGetErrorString(e));
        return kErrCuda;
      }
      g_scratch_addr[dev] = p;
    }
    base = g_scratch_addr[dev];
  }
  try {
    if (sort_scratch_bytes(n, value_bits) > kNoAllocScratchBytes)
      throw Error{kErrCapacity, "srdl_sort_unique_u64_noalloc: scratch estimate exceeds the array"};
    Launch L;
    L.stream = (cudaStream_t)stream;
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 148;
    L.num_sms = sms;
    Scratch s{static_cast<char*>(base), kNoAllocScratchBytes, 0};
    sort_dedup(L, d_in, n, value_bits, false, nullptr, 0, d_out, d_n_out, s);
    return 0;
  } catch (const Error& err) {
    set_error(err.msg);
    return err.code;
  } catch (const std::exception& err) {
    set_error(std::string("srdl_sort_unique_u64_noalloc: ") + err.what());
    return kErrState;
  }
}

}  // extern "C"
