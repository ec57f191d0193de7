/*
 * oracle.c -- CPU restatement of the reference's semi-naive evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this
 * file; tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
 * reference arm use it as the checker and as the timed CPU baseline.
 *
 * Parity status: UNPINNED against the reference's own outputs.  The
 * reference has no tuple-level golden vectors and its GPU runtime cannot
 * be built here (needs clang >= 20, boost, highway).  The restatement is
 * pinned instead by known-answer graphs (chains, cycles, complete graphs,
 * stars) and by an independent numpy/scipy restatement in the tests.
 *
 * Representation: a binary relation index is an array of uint64 keys,
 * key = (first index column << 32) | second index column, sorted
 * ascending and unique.  That is the lexicographic uint32 order of the
 * reference's column-major sorted arrays
 * (src/srdatalog/runtime/generalized_datalog/gpu/device_sorted_array_index.h:337).
 *
 * Build: see oracle/Makefile (gcc -O3 -fopenmp, C11).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  uint64_t* keys; /* malloc'd, canonical-index key order */
  uint64_t n;
  uint64_t iterations; /* recursive-step iterations executed */
  uint64_t derived;    /* rows materialised by the joins (before dedup) */
} orc_result;

void orc_free(void* p) { free(p); }

/* ---------------------------------------------------------------- sort */

/* LSD radix sort (8-bit digits) of uint64 keys, skipping digits that are
 * constant over the input.  Follows the contract of zip_sort_columns
 * (RT/gpu/sort.h:297-302): lexicographic order of the index columns. */
static void radix_sort_u64(uint64_t* a, uint64_t n) {
  if (n < 2) return;
  uint64_t* tmp = (uint64_t*)malloc(n * sizeof(uint64_t));
  uint64_t all_or = 0, all_and = ~0ull;
  for (uint64_t i = 0; i < n; i++) { all_or |= a[i]; all_and &= a[i]; }
  uint64_t varying = all_or ^ all_and;
  uint64_t* src = a; uint64_t* dst = tmp;
  for (int shift = 0; shift < 64; shift += 8) {
    if (((varying >> shift) & 0xffu) == 0) continue;
    uint64_t cnt[256];
    memset(cnt, 0, sizeof(cnt));
    for (uint64_t i = 0; i < n; i++) cnt[(src[i] >> shift) & 0xffu]++;
    uint64_t s = 0;
    for (int d = 0; d < 256; d++) { uint64_t c = cnt[d]; cnt[d] = s; s += c; }
    for (uint64_t i = 0; i < n; i++) dst[cnt[(src[i] >> shift) & 0xffu]++] = src[i];
    uint64_t* t = src; src = dst; dst = t;
  }
  if (src != a) memcpy(a, src, n * sizeof(uint64_t));
  free(tmp);
}

/* sort + unique in place; returns the unique count.
 * Reference: rebuild_index_fn (RT/gpu/runtime/gpu_mir_helpers.h:204-232)
 * -> zip sort (RT/gpu/sort.h:297) -> deduplicate_aggregate_and_unique
 * (RT/gpu/deduplication.h:178-258, NoProvenance branch). */
uint64_t orc_sort_unique_u64(uint64_t* a, uint64_t n) {
  radix_sort_u64(a, n);
  if (n == 0) return 0;
  uint64_t w = 1;
  for (uint64_t i = 1; i < n; i++)
    if (a[i] != a[w - 1]) a[w++] = a[i];
  return w;
}

/* out = a - b (both sorted unique).  Reference: DSAI::set_difference_update
 * (RT/gpu/device_sorted_array_index.ipp:966-1130), thrust::set_difference
 * on the zipped columns. */
uint64_t orc_set_difference_u64(const uint64_t* a, uint64_t na, const uint64_t* b,
                                uint64_t nb, uint64_t* out) {
  uint64_t i = 0, j = 0, w = 0;
  while (i < na) {
    if (j >= nb || a[i] < b[j]) out[w++] = a[i++];
    else if (a[i] > b[j]) j++;
    else { i++; j++; }
  }
  return w;
}

/* out = a U b for sorted unique disjoint-or-not inputs (set union keeps one
 * copy).  Reference: DSAI::merge (RT/gpu/device_sorted_array_index.ipp:709-847). */
uint64_t orc_merge_u64(const uint64_t* a, uint64_t na, const uint64_t* b, uint64_t nb,
                       uint64_t* out) {
  uint64_t i = 0, j = 0, w = 0;
  while (i < na || j < nb) {
    if (j >= nb || (i < na && a[i] < b[j])) out[w++] = a[i++];
    else if (i >= na || b[j] < a[i]) out[w++] = b[j++];
    else { out[w++] = a[i++]; j++; }
  }
  return w;
}

/* --------------------------------------------------------- index access */

static uint64_t lower_bound_u64(const uint64_t* a, uint64_t n, uint64_t key) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    uint64_t mid = lo + (hi - lo) / 2;
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

/* rows whose first column == v: [*b, *e).  Mirrors NodeHandle::prefix
 * (RT/gpu/device_sorted_array_index.ipp:67-157) on a 2-column index. */
static void prefix_range(const uint64_t* a, uint64_t n, uint32_t v, uint64_t* b, uint64_t* e) {
  *b = lower_bound_u64(a, n, (uint64_t)v << 32);
  *e = (v == 0xffffffffu) ? n : lower_bound_u64(a, n, ((uint64_t)v + 1) << 32);
}

/* distinct first-column values (root_unique_values) */
static uint32_t* roots_of(const uint64_t* a, uint64_t n, uint64_t* nr) {
  uint32_t* r = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
  uint64_t w = 0;
  for (uint64_t i = 0; i < n; i++) {
    uint32_t h = (uint32_t)(a[i] >> 32);
    if (w == 0 || r[w - 1] != h) r[w++] = h;
  }
  *nr = w;
  return r;
}

/* growable per-thread output buffer */
typedef struct { uint64_t* p; uint64_t n, cap; } vec64;
static void vpush(vec64* v, uint64_t x) {
  if (v->n == v->cap) {
    v->cap = v->cap ? v->cap * 2 : 1024;
    v->p = (uint64_t*)realloc(v->p, v->cap * sizeof(uint64_t));
  }
  v->p[v->n++] = x;
}

static uint64_t* concat_threads(vec64* vs, int nt, uint64_t* total) {
  uint64_t t = 0;
  for (int i = 0; i < nt; i++) t += vs[i].n;
  uint64_t* out = (uint64_t*)malloc((t ? t : 1) * sizeof(uint64_t));
  uint64_t w = 0;
  for (int i = 0; i < nt; i++) {
    if (vs[i].n) memcpy(out + w, vs[i].p, vs[i].n * sizeof(uint64_t));
    w += vs[i].n;
    free(vs[i].p);
  }
  *total = t;
  return out;
}

static int nthreads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
static int tid(void) {
#ifdef _OPENMP
  return omp_get_thread_num();
#else
  return 0;
#endif
}

/* One semi-naive maintenance round for a relation: NEW is sorted+deduped,
 * DELTA = NEW - FULL, FULL = FULL U DELTA.  Order of
 * RebuildIndex/ComputeDeltaIndex/MergeIndex from hir/lower.py:519-589. */
static void maintain(uint64_t* newk, uint64_t nnew, uint64_t** full, uint64_t* nfull,
                     uint64_t** delta, uint64_t* ndelta) {
  nnew = orc_sort_unique_u64(newk, nnew);
  uint64_t* d = (uint64_t*)malloc((nnew ? nnew : 1) * sizeof(uint64_t));
  uint64_t nd = orc_set_difference_u64(newk, nnew, *full, *nfull, d);
  uint64_t* f = (uint64_t*)malloc(((*nfull + nd) ? (*nfull + nd) : 1) * sizeof(uint64_t));
  uint64_t nf = orc_merge_u64(*full, *nfull, d, nd, f);
  free(*full);
  free(*delta);
  *full = f; *nfull = nf;
  *delta = d; *ndelta = nd;
}

/* ------------------------------------------------------------------ TC */

/* Transitive closure exactly as the TC plan runs it (tests/fixtures/tc.mir.sexpr):
 *   EdgeLoad : Edge(0,1)  <- sort_unique(ArcInput)
 *   TCBase   : Path(1,0)  <- {(y,x) : Edge(x,y)}
 *   TCRec_D0 : column-join y over Path(1,0)^DELTA and Edge(0,1);
 *              cartesian x in DeltaPath[y], z in Edge[y]; insert (z,x) in (1,0) order.
 * Iteration 0 of the recursive step reads FULL for DELTA
 * (RT/gpu/runtime/gpu_mir_helpers.h:419-426).  The loop stops when the
 * delta is empty or after max_iters joins (orchestrator_jit.py:600-747).
 * `edges` are (x<<32|y) keys, any order, duplicates allowed. */
int orc_tc(const uint64_t* edges, uint64_t m, uint64_t max_iters, orc_result* res) {
  uint64_t* E = (uint64_t*)malloc((m ? m : 1) * sizeof(uint64_t));
  memcpy(E, edges, m * sizeof(uint64_t));
  uint64_t ne = orc_sort_unique_u64(E, m);
  uint64_t* full = (uint64_t*)malloc(8); uint64_t nfull = 0;
  uint64_t* delta = (uint64_t*)malloc(8); uint64_t ndelta = 0;
  uint64_t* newk = (uint64_t*)malloc((ne ? ne : 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < ne; i++) newk[i] = (E[i] << 32) | (E[i] >> 32);
  maintain(newk, ne, &full, &nfull, &delta, &ndelta);
  free(newk);
  uint64_t derived = ne;
  uint64_t iters = 0;
  int nt = nthreads();
  for (uint64_t it = 0; it < max_iters; it++) {
    if (it > 0 && ndelta == 0) break;
    const uint64_t* D = (it == 0) ? full : delta;
    uint64_t nd = (it == 0) ? nfull : ndelta;
    uint64_t nroots;
    uint32_t* roots = roots_of(D, nd, &nroots);
    vec64* outs = (vec64*)calloc(nt, sizeof(vec64));
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t r = 0; r < (int64_t)nroots; r++) {
      uint32_t y = roots[r];
      uint64_t eb, ee, db, de;
      prefix_range(E, ne, y, &eb, &ee);
      if (eb == ee) continue;
      prefix_range(D, nd, y, &db, &de);
      vec64* o = &outs[tid()];
      for (uint64_t i = db; i < de; i++) {
        uint32_t x = (uint32_t)D[i];
        for (uint64_t j = eb; j < ee; j++) {
          uint32_t z = (uint32_t)E[j];
          vpush(o, ((uint64_t)z << 32) | x);
        }
      }
    }
    free(roots);
    uint64_t nn;
    newk = concat_threads(outs, nt, &nn);
    free(outs);
    derived += nn;
    maintain(newk, nn, &full, &nfull, &delta, &ndelta);
    free(newk);
    iters++;
  }
  free(E);
  free(delta);
  res->keys = full; res->n = nfull; res->iterations = iters; res->derived = derived;
  return 0;
}

/* ------------------------------------------------------------------ SG */

/* Same generation as the SG plan runs it (tests/fixtures/integration/sg.mir.sexpr):
 *   SGBase  : column-join p over Arc(0,1) x2; cartesian x,y in Arc[p]; filter x != y
 *   SGRec_D1: column-join p over Sg(0,1)^DELTA, Arc(0,1);
 *             column-join q over DeltaSg[p], Arc roots;
 *             cartesian x in Arc[p], y in Arc[q]; insert (x,y). */
int orc_sg(const uint64_t* arcs, uint64_t m, uint64_t max_iters, orc_result* res) {
  uint64_t* A = (uint64_t*)malloc((m ? m : 1) * sizeof(uint64_t));
  memcpy(A, arcs, m * sizeof(uint64_t));
  uint64_t na = orc_sort_unique_u64(A, m);
  uint64_t nroots_a;
  uint32_t* aroots = roots_of(A, na, &nroots_a);
  int nt = nthreads();
  uint64_t* full = (uint64_t*)malloc(8); uint64_t nfull = 0;
  uint64_t* delta = (uint64_t*)malloc(8); uint64_t ndelta = 0;
  vec64* outs = (vec64*)calloc(nt, sizeof(vec64));
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t r = 0; r < (int64_t)nroots_a; r++) {
    uint64_t b, e;
    prefix_range(A, na, aroots[r], &b, &e);
    vec64* o = &outs[tid()];
    for (uint64_t i = b; i < e; i++)
      for (uint64_t j = b; j < e; j++) {
        uint32_t x = (uint32_t)A[i], y = (uint32_t)A[j];
        if (x != y) vpush(o, ((uint64_t)x << 32) | y);
      }
  }
  uint64_t nn;
  uint64_t* newk = concat_threads(outs, nt, &nn);
  free(outs);
  uint64_t derived = nn;
  maintain(newk, nn, &full, &nfull, &delta, &ndelta);
  free(newk);
  uint64_t iters = 0;
  for (uint64_t it = 0; it < max_iters; it++) {
    if (it > 0 && ndelta == 0) break;
    const uint64_t* D = (it == 0) ? full : delta;
    uint64_t nd = (it == 0) ? nfull : ndelta;
    uint64_t nroots;
    uint32_t* roots = roots_of(D, nd, &nroots);
    outs = (vec64*)calloc(nt, sizeof(vec64));
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t r = 0; r < (int64_t)nroots; r++) {
      uint32_t p = roots[r];
      uint64_t pb, pe, db, de;
      prefix_range(A, na, p, &pb, &pe);
      if (pb == pe) continue;
      prefix_range(D, nd, p, &db, &de);
      vec64* o = &outs[tid()];
      for (uint64_t k = db; k < de; k++) {
        uint32_t q = (uint32_t)D[k];
        uint64_t qb, qe;
        prefix_range(A, na, q, &qb, &qe);
        for (uint64_t i = pb; i < pe; i++)
          for (uint64_t j = qb; j < qe; j++)
            vpush(o, ((uint64_t)(uint32_t)A[i] << 32) | (uint32_t)A[j]);
      }
    }
    free(roots);
    newk = concat_threads(outs, nt, &nn);
    free(outs);
    derived += nn;
    maintain(newk, nn, &full, &nfull, &delta, &ndelta);
    free(newk);
    iters++;
  }
  free(A);
  free(aroots);
  free(delta);
  res->keys = full; res->n = nfull; res->iterations = iters; res->derived = derived;
  return 0;
}

/* ------------------------------------------------------------ triangle */

/* Count-only triangle join (tests/fixtures/integration/lsqb_triangle_count.mir.sexpr):
 *   a in roots(K); b in K[a] n roots(K); c in K[b] n K[a]; count bindings.
 * The reference counts per thread in uint32 and reduces in uint64
 * (lsqb_triangle_count orchestrator.cpp:40-47); the count here is uint64
 * throughout.  `edges` are (a<<32|b) keys, any order, duplicates allowed. */
uint64_t orc_triangle_count(const uint64_t* edges, uint64_t m) {
  uint64_t* K = (uint64_t*)malloc((m ? m : 1) * sizeof(uint64_t));
  memcpy(K, edges, m * sizeof(uint64_t));
  uint64_t nk = orc_sort_unique_u64(K, m);
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : total)
  for (int64_t e = 0; e < (int64_t)nk; e++) {
    uint32_t a = (uint32_t)(K[e] >> 32), b = (uint32_t)K[e];
    uint64_t ab, ae, bb, be;
    prefix_range(K, nk, b, &bb, &be);
    if (bb == be) continue; /* b not a root: contributes nothing */
    prefix_range(K, nk, a, &ab, &ae);
    uint64_t i = ab, j = bb, c = 0;
    while (i < ae && j < be) {
      uint32_t x = (uint32_t)K[i], y = (uint32_t)K[j];
      if (x < y) i++;
      else if (y < x) j++;
      else { c++; i++; j++; }
    }
    total += c;
  }
  free(K);
  return total;
}

/* Bounded sample of the triangle join for CPU timing: only edges whose
 * position in the sorted index is = phase (mod stride) are expanded.  The
 * index build is timed separately (t_sort) from the sampled join (t_join). */
static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

uint64_t orc_triangle_count_sample(const uint64_t* edges, uint64_t m, uint64_t stride,
                                   uint64_t phase, double* t_sort, double* t_join) {
  double t0 = now_s();
  uint64_t* K = (uint64_t*)malloc((m ? m : 1) * sizeof(uint64_t));
  memcpy(K, edges, m * sizeof(uint64_t));
  uint64_t nk = orc_sort_unique_u64(K, m);
  double t1 = now_s();
  uint64_t total = 0;
  if (stride == 0) stride = 1;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : total)
  for (int64_t e = (int64_t)phase; e < (int64_t)nk; e += (int64_t)stride) {
    uint32_t a = (uint32_t)(K[e] >> 32), b = (uint32_t)K[e];
    uint64_t ab, ae, bb, be;
    prefix_range(K, nk, b, &bb, &be);
    if (bb == be) continue;
    prefix_range(K, nk, a, &ab, &ae);
    uint64_t i = ab, j = bb, c = 0;
    while (i < ae && j < be) {
      uint32_t x = (uint32_t)K[i], y = (uint32_t)K[j];
      if (x < y) i++;
      else if (y < x) j++;
      else { c++; i++; j++; }
    }
    total += c;
  }
  double t2 = now_s();
  free(K);
  *t_sort = t1 - t0;
  *t_join = t2 - t1;
  return total;
}

int orc_num_threads(void) { return nthreads(); }
