// capi.cu -- extern "C" boundary of libsrdl and the CSV input path.
//
// The reference's generated shim (src/srdatalog/codegen/jit/main_file.py:
// 656-780) exports srdatalog_init/load_csv/load_all/run/size/shutdown over
// one process-global host DB.  libsrdl exposes the same operations on an
// explicit handle (srdl_*); the per-program shim that build_project emits
// keeps the srdatalog_* names and forwards to these.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cmath>
#include <cstring>
#include <fstream>
#include <vector>
#include <sstream>

#include "../../include/srdl.h"
#include "runtime.h"

using namespace srdl;

struct srdl_db {
  std::unique_ptr<Database> db;
};

namespace srdl {

// CSV reader with the reference's delimiter detection (RT/runtime/io.h:
// 200-245): a tab in the first line selects tab, else a comma selects comma,
// else a run of >= 2 spaces selects "multi-space", else single space.
// Values parse as signed 64-bit integers and are stored as uint32 (the
// reference casts through size_t to its uint32 value type, io.h:351).
static void parse_csv(const std::string& path, int arity, std::vector<uint32_t>& out) {
  int fd = ::open(path.c_str(), O_RDONLY);
  SRDL_REQUIRE(fd >= 0, kErrIo, "cannot open " + path);
  struct stat stt;
  if (fstat(fd, &stt) != 0) {
    ::close(fd);
    throw Error{kErrIo, "cannot stat " + path};
  }
  const size_t size = (size_t)stt.st_size;
  if (size == 0) {
    ::close(fd);
    return;
  }
  const char* base = (const char*)mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
  ::close(fd);
  SRDL_REQUIRE(base != MAP_FAILED, kErrIo, "cannot map " + path);
  const char* p = base;
  const char* end = base + size;
  const char* le = p;
  while (le < end && *le != '\n') le++;
  size_t tabs = 0, commas = 0, run = 0, max_run = 0;
  for (const char* c = p; c < le; c++) {
    if (*c == '\t') tabs++;
    if (*c == ',') commas++;
    if (*c == ' ') max_run = std::max(max_run, ++run);
    else run = 0;
  }
  const char delim = tabs ? '\t' : (commas ? ',' : ' ');
  (void)max_run;  // multi-space and single-space files both split on runs of blanks
  std::string err;
  while (p < end && err.empty()) {
    const char* le2 = p;
    while (le2 < end && *le2 != '\n') le2++;
    const char* q = p;
    const char* qe = le2;
    if (qe > q && qe[-1] == '\r') qe--;
    int got = 0;
    while (q < qe) {
      while (q < qe && (*q == ' ' || (*q == '\t' && delim != '\t'))) q++;
      if (q >= qe) break;
      bool neg = false;
      if (*q == '-' || *q == '+') neg = *q++ == '-';
      if (q >= qe || *q < '0' || *q > '9') {
        err = "non-integer field in " + path;
        break;
      }
      unsigned long long v = 0;
      while (q < qe && *q >= '0' && *q <= '9') v = v * 10 + (unsigned)(*q++ - '0');
      const long long sv = neg ? -(long long)v : (long long)v;
      if (got < arity) out.push_back((uint32_t)(uint64_t)sv);
      got++;
      while (q < qe && (*q == ' ' || (*q == '\t' && delim != '\t'))) q++;
      if (q < qe && delim != ' ') {
        if (*q != delim) {
          err = "unexpected character in " + path;
          break;
        }
        q++;
      }
    }
    if (err.empty() && got > 0 && got < arity)
      err = "row with " + std::to_string(got) + " fields in " + path;
    p = le2 < end ? le2 + 1 : end;
  }
  munmap((void*)base, size);
  SRDL_REQUIRE(err.empty(), kErrIo, err);
}

void Database::load_csv(const std::string& name, const std::string& path) {
  Relation& r = rel(name);
  SRDL_REQUIRE(!r.input_file.empty(), kErrArg, "relation " + name + " is not an input relation");
  std::vector<uint32_t> rows;
  parse_csv(path, r.arity, rows);
  load_rows(name, rows.data(), rows.size() / r.arity);
}

void Database::load_all(const std::string& dir) {
  for (auto& n : inputs_) load_csv(n, dir + "/" + rel(n).input_file);
}

}  // namespace srdl

#define SRDL_GUARD(ret_on_error, ...)                                   \
  try {                                                                  \
    __VA_ARGS__                                                          \
  } catch (const srdl::Error& e) {                                       \
    srdl::set_error(e.msg);                                              \
    return (ret_on_error) ? (ret_on_error) : e.code;                     \
  } catch (const std::exception& e) {                                    \
    srdl::set_error(e.what());                                           \
    return (ret_on_error) ? (ret_on_error) : (int)srdl::kErrState;       \
  }

static int guard_code(const srdl::Error& e) { return e.code; }

extern "C" {

const char* srdl_last_error(void) { return srdl::last_error(); }

int srdl_version(void) { return SRDL_ABI_VERSION; }

int srdl_open(const char* plan_json, int device, srdl_db** out) {
  if (!plan_json || !out) return kErrArg;
  try {
    auto* h = new srdl_db;
    h->db = std::make_unique<Database>(std::string(plan_json), device);
    *out = h;
    return 0;
  } catch (const srdl::Error& e) {
    set_error(e.msg);
    return guard_code(e);
  } catch (const std::exception& e) {
    set_error(e.what());
    return kErrState;
  }
}

int srdl_close(srdl_db* h) {
  delete h;
  return 0;
}

int srdl_init_device(srdl_db* h) {
  if (!h) return kErrArg;
  SRDL_GUARD(0, h->db->init_device(); return 0;)
}

int srdl_load_rows(srdl_db* h, const char* rel, const uint32_t* rows, uint64_t n_rows) {
  if (!h || !rel) return kErrArg;
  SRDL_GUARD(0, h->db->load_rows(rel, rows, n_rows); return 0;)
}

int srdl_load_csv(srdl_db* h, const char* rel, const char* path) {
  if (!h || !rel || !path) return kErrArg;
  SRDL_GUARD(0, h->db->load_csv(rel, path); return 0;)
}

int srdl_load_all(srdl_db* h, const char* dir) {
  if (!h || !dir) return kErrArg;
  SRDL_GUARD(0, h->db->load_all(dir); return 0;)
}

int srdl_set_stream(srdl_db* h, void* stream) {
  if (!h) return kErrArg;
  SRDL_GUARD(0, h->db->set_stream((cudaStream_t)stream); return 0;)
}

int srdl_set_profiling(srdl_db* h, int enable) {
  if (!h) return kErrArg;
  h->db->set_profiling(enable != 0);
  return 0;
}

int srdl_load_device_rows(srdl_db* h, const char* rel, const uint32_t* d_rows, uint64_t n_rows) {
  if (!h || !rel) return kErrArg;
  SRDL_GUARD(0, h->db->load_device_rows(rel, d_rows, n_rows); return 0;)
}

uint64_t srdl_launch_count(void) { return srdl::launches_total(); }

int srdl_set_option(srdl_db* h, const char* name, int64_t value) {
  if (!h || !name) return kErrArg;
  SRDL_GUARD(0, h->db->set_option(name, value); return 0;)
}

int srdl_set_exchange(srdl_db* h, srdl_exchange_fn fn, void* user) {
  if (!h) return kErrArg;
  SRDL_GUARD(0, h->db->set_exchange(fn, user); return 0;)
}

int srdl_copy_device(void* dst, const void* src, uint64_t bytes, void* stream) {
  if ((!dst || !src) && bytes) return kErrArg;
  SRDL_GUARD(0, {
    if (bytes) {
      SRDL_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, (cudaStream_t)stream));
      SRDL_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    }
    return 0;
  })
}

int srdl_set_count_groups(srdl_db* h, const char* rule, const uint32_t* bounds,
                          uint64_t n_bounds) {
  if (!h || !rule) return kErrArg;
  SRDL_GUARD(0, h->db->set_count_groups(rule, bounds, n_bounds); return 0;)
}

int srdl_group_counts(srdl_db* h, const char* rule, uint64_t* out, uint64_t n_groups) {
  if (!h || !rule || (n_groups && !out)) return kErrArg;
  SRDL_GUARD(0, h->db->group_counts(rule, out, n_groups); return 0;)
}

int srdl_clear_inputs(srdl_db* h) {
  if (!h) return kErrArg;
  SRDL_GUARD(0, h->db->clear_inputs(); return 0;)
}

int srdl_range_counts(srdl_db* h, const char* rel, const uint32_t* bounds, uint64_t n_bounds,
                      uint64_t* counts) {
  if (!h || !rel || (n_bounds > 1 && !counts)) return kErrArg;
  SRDL_GUARD(0, h->db->range_counts(rel, bounds, n_bounds, counts); return 0;)
}

int srdl_set_instances(srdl_db* h, const uint32_t* bounds, uint64_t n_bounds) {
  if (!h || (n_bounds && !bounds)) return kErrArg;
  SRDL_GUARD(0, h->db->set_instances(bounds, n_bounds); return 0;)
}

int srdl_instance_iterations(srdl_db* h, uint64_t step, uint32_t* out, uint64_t n_instances) {
  if (!h || (n_instances && !out)) return kErrArg;
  SRDL_GUARD(0, h->db->instance_iterations(step, out, n_instances); return 0;)
}

int srdl_range_checksums(srdl_db* h, const char* rel, const uint32_t* bounds, uint64_t n_bounds,
                         uint64_t* sums) {
  if (!h || !rel || (n_bounds > 1 && !sums)) return kErrArg;
  SRDL_GUARD(0, h->db->range_checksums(rel, bounds, n_bounds, sums); return 0;)
}

uint64_t srdl_staged_rows(srdl_db* h, const char* rel) {
  if (!h || !rel || !h->db->has_rel(rel)) return 0;
  return h->db->staged_rows(rel);
}

int srdl_run(srdl_db* h, uint64_t max_iters) {
  if (!h) return kErrArg;
  SRDL_GUARD(0, h->db->run(max_iters ? max_iters : (uint64_t)0x7fffffff); return 0;)
}

uint64_t srdl_size(srdl_db* h, const char* rel) {
  if (!h || !rel) return 0;
  try {
    if (!h->db->has_rel(rel)) return 0;
    return h->db->size(rel);
  } catch (const srdl::Error& e) {
    set_error(e.msg);
    return 0;
  }
}

uint64_t srdl_count(srdl_db* h, const char* rule) {
  if (!h || !rule) return 0;
  return h->db->count(rule);
}

int64_t srdl_dump(srdl_db* h, const char* rel, uint32_t* out_rows, uint64_t cap_rows) {
  if (!h || !rel) return -kErrArg;
  try {
    return h->db->dump(rel, out_rows, cap_rows);
  } catch (const srdl::Error& e) {
    set_error(e.msg);
    return -(int64_t)e.code;
  }
}

// SHA-256 (FIPS 180-4).  The round constants are the first 32 bits of the
// fractional parts of the cube roots of the first 64 primes, the initial
// hash the same of the square roots of the first 8; both are derived here
// in extended precision.
namespace {
struct Sha256 {
  uint32_t k[64], h0[8];
  Sha256() {
    int primes[64], np = 0;
    for (int c = 2; np < 64; c++) {
      bool prime = true;
      for (int d = 2; d * d <= c; d++) prime &= c % d != 0;
      if (prime) primes[np++] = c;
    }
    for (int i = 0; i < 64; i++) {
      const long double r = cbrtl((long double)primes[i]);
      k[i] = (uint32_t)((r - floorl(r)) * 4294967296.0L);
    }
    for (int i = 0; i < 8; i++) {
      const long double r = sqrtl((long double)primes[i]);
      h0[i] = (uint32_t)((r - floorl(r)) * 4294967296.0L);
    }
  }
  static uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
  void block(uint32_t* h, const unsigned char* p) const {
    uint32_t w[64];
    for (int i = 0; i < 16; i++)
      w[i] = (uint32_t)p[4 * i] << 24 | (uint32_t)p[4 * i + 1] << 16 | (uint32_t)p[4 * i + 2] << 8 | p[4 * i + 3];
    for (int i = 16; i < 64; i++) {
      const uint32_t s0 = rotr(w[i - 15], 7) ^ rotr(w[i - 15], 18) ^ (w[i - 15] >> 3);
      const uint32_t s1 = rotr(w[i - 2], 17) ^ rotr(w[i - 2], 19) ^ (w[i - 2] >> 10);
      w[i] = w[i - 16] + s0 + w[i - 7] + s1;
    }
    uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
    for (int i = 0; i < 64; i++) {
      const uint32_t t1 = hh + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + k[i] + w[i];
      const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
      hh = g;
      g = f;
      f = e;
      e = d + t1;
      d = c;
      c = b;
      b = a;
      a = t1 + t2;
    }
    h[0] += a; h[1] += b; h[2] += c; h[3] += d; h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
  }
  void digest(const unsigned char* data, uint64_t n, unsigned char out[32]) const {
    uint32_t h[8];
    for (int i = 0; i < 8; i++) h[i] = h0[i];
    uint64_t i = 0;
    for (; i + 64 <= n; i += 64) block(h, data + i);
    unsigned char tail[128] = {0};
    const uint64_t rem = n - i;
    for (uint64_t j = 0; j < rem; j++) tail[j] = data[i + j];
    tail[rem] = 0x80;
    const uint64_t tl = rem + 1 + 8 <= 64 ? 64 : 128;
    const uint64_t bits = n * 8;
    for (int j = 0; j < 8; j++) tail[tl - 1 - j] = (unsigned char)(bits >> (8 * j));
    for (uint64_t j = 0; j < tl; j += 64) block(h, tail + j);
    for (int j = 0; j < 8; j++)
      for (int b = 0; b < 4; b++) out[4 * j + b] = (unsigned char)(h[j] >> (24 - 8 * b));
  }
};
const Sha256& sha256() {
  static const Sha256 s;
  return s;
}
}  // namespace

int srdl_sha256(const void* data, uint64_t n_bytes, unsigned char* out32) {
  if ((!data && n_bytes) || !out32) return kErrArg;
  sha256().digest(static_cast<const unsigned char*>(data), n_bytes, out32);
  return 0;
}

int srdl_hash(srdl_db* h, const char* rel, unsigned char* out32) {
  if (!h || !rel || !out32) return kErrArg;
  SRDL_GUARD(0, {
    const int64_t rows = h->db->dump(rel, nullptr, 0);
    const int arity = h->db->rel(rel).arity;
    std::vector<uint32_t> buf((size_t)rows * arity + 1);
    h->db->dump(rel, buf.data(), (uint64_t)rows);
    sha256().digest(reinterpret_cast<const unsigned char*>(buf.data()),
                    (uint64_t)rows * arity * 4, out32);
    return 0;
  })
}

int srdl_stats_json(srdl_db* h, char* buf, uint64_t cap) {
  if (!h || !buf || cap == 0) return kErrArg;
  std::string s = h->db->stats_json();
  if (s.size() + 1 > cap) {
    set_error("stats buffer too small");
    return kErrCapacity;
  }
  memcpy(buf, s.c_str(), s.size() + 1);
  return 0;
}

int srdl_mem_stats(srdl_db* h, uint64_t* out4) {
  if (!h || !out4) return kErrArg;
  SRDL_GUARD(0, {
    const srdl::ArenaUse u = h->db->mem_stats();
    out4[0] = u.in_use;
    out4[1] = u.peak;
    out4[2] = u.cached;
    out4[3] = u.limit;
    return 0;
  })
}

int srdl_trim_cache(srdl_db* h) {
  if (!h) return kErrArg;
  SRDL_GUARD(0, h->db->trim_cache(); return 0;)
}

// ------------------------------------------------------ kernel primitives

static Launch launch_for(void* stream) {
  Launch L;
  L.stream = (cudaStream_t)stream;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  L.num_sms = sms;
  return L;
}

uint64_t srdl_sort_unique_scratch_bytes(uint64_t n, int value_bits) {
  if (value_bits < 1 || value_bits > 32) return 0;
  return sort_scratch_bytes(n, value_bits);
}

int srdl_sort_unique_u64(const uint64_t* d_in, uint64_t n, int value_bits, uint64_t* d_out,
                         uint64_t* d_n_out, void* d_scratch, uint64_t scratch_bytes,
                         void* stream) {
  if ((!d_in && n) || !d_out || !d_n_out || value_bits < 1 || value_bits > 32) {
    srdl::set_error("srdl_sort_unique_u64: bad argument");
    return kErrArg;
  }
  SRDL_GUARD(0, {
    Launch L = launch_for(stream);
    Scratch s{(char*)d_scratch, (size_t)scratch_bytes, 0};
    sort_dedup(L, d_in, n, value_bits, false, nullptr, 0, d_out, d_n_out, s);
    return 0;
  })
}

uint64_t srdl_set_difference_scratch_bytes(uint64_t na) { return diff_scratch_bytes(na) + 1024; }

int srdl_set_difference_u64(const uint64_t* d_a, uint64_t na, const uint64_t* d_b, uint64_t nb,
                            uint64_t* d_out, uint64_t* d_n_out, void* d_scratch,
                            uint64_t scratch_bytes, void* stream) {
  if ((!d_a && na) || (!d_b && nb) || !d_out || !d_n_out) {
    srdl::set_error("srdl_set_difference_u64: bad argument");
    return kErrArg;
  }
  SRDL_GUARD(0, {
    Launch L = launch_for(stream);
    Scratch s{(char*)d_scratch, (size_t)scratch_bytes, 0};
    set_difference(L, d_a, na, d_b, nb, d_out, d_n_out, s);
    return 0;
  })
}

int srdl_merge_u64(const uint64_t* d_a, uint64_t na, const uint64_t* d_b, uint64_t nb,
                   uint64_t* d_out, void* stream) {
  if ((!d_a && na) || (!d_b && nb) || !d_out) {
    srdl::set_error("srdl_merge_u64: bad argument");
    return kErrArg;
  }
  SRDL_GUARD(0, {
    Launch L = launch_for(stream);
    merge_disjoint(L, d_a, na, d_b, nb, d_out);
    return 0;
  })
}

}  // extern "C"
