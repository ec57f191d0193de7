'''Python side of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline /
reference arm import this module.  The product never routes through it.

Parity status: UNPINNED against the reference's own outputs (the
reference ships no tuple-level golden vectors and its runtime cannot be
built here).  Pins used instead: known-answer graphs and an independent
linear-algebra restatement (tests/test_oracle.py).

Two restatements of the reference's semi-naive evaluation live here:

* `liboracle.so` (oracle.c): fast C/OpenMP evaluators for the TC, SG and
  triangle plans, plus sort+unique / set difference / merge.
* `run_plan`: a small pure-Python interpreter for ANY plan this runtime
  accepts, for tiny inputs; it walks the MIR op sequence literally
  (src/srdatalog/hir/lower.py:442-789) with Python sets.
'''

from __future__ import annotations

import ctypes
import hashlib
import itertools
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class _Result(ctypes.Structure):
  _fields_ = [('keys', ctypes.POINTER(ctypes.c_uint64)), ('n', ctypes.c_uint64),
              ('iterations', ctypes.c_uint64), ('derived', ctypes.c_uint64)]


def build() -> str:
  path = os.path.join(HERE, 'liboracle.so')
  src = os.path.join(HERE, 'oracle.c')
  if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
    subprocess.run(['make', '-s', '-C', HERE], check=True)
  return path


def lib():
  global _LIB
  if _LIB is None:
    L = ctypes.CDLL(build())
    u64, p64 = ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)
    L.orc_sort_unique_u64.argtypes = [p64, u64]
    L.orc_sort_unique_u64.restype = u64
    L.orc_set_difference_u64.argtypes = [p64, u64, p64, u64, p64]
    L.orc_set_difference_u64.restype = u64
    L.orc_merge_u64.argtypes = [p64, u64, p64, u64, p64]
    L.orc_merge_u64.restype = u64
    for f in (L.orc_tc, L.orc_sg):
      f.argtypes = [p64, u64, u64, ctypes.POINTER(_Result)]
      f.restype = ctypes.c_int
    L.orc_triangle_count.argtypes = [p64, u64]
    L.orc_triangle_count.restype = u64
    L.orc_triangle_count_sample.argtypes = [p64, u64, u64, u64, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double)]
    L.orc_triangle_count_sample.restype = u64
    L.orc_free.argtypes = [ctypes.c_void_p]
    L.orc_num_threads.restype = ctypes.c_int
    _LIB = L
  return _LIB


def _p64(a: np.ndarray):
  return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def pack(edges: np.ndarray, order=(0, 1)) -> np.ndarray:
  '''(m,2) uint32 rows -> uint64 keys in the given index column order.'''
  e = np.asarray(edges, dtype=np.uint32)
  return (e[:, order[0]].astype(np.uint64) << np.uint64(32)) | e[:, order[1]].astype(np.uint64)


def unpack(keys: np.ndarray, order=(0, 1)) -> np.ndarray:
  '''uint64 keys in index order -> (n,2) uint32 rows in declared column order.'''
  k = np.asarray(keys, dtype=np.uint64)
  out = np.empty((k.shape[0], 2), np.uint32)
  out[:, order[0]] = (k >> np.uint64(32)).astype(np.uint32)
  out[:, order[1]] = (k & np.uint64(0xffffffff)).astype(np.uint32)
  return out


def sort_unique(keys: np.ndarray) -> np.ndarray:
  a = np.array(keys, dtype=np.uint64, copy=True)
  n = lib().orc_sort_unique_u64(_p64(a), a.shape[0])
  return a[:n]


def set_difference(a: np.ndarray, b: np.ndarray) -> np.ndarray:
  a = np.ascontiguousarray(a, np.uint64)
  b = np.ascontiguousarray(b, np.uint64)
  out = np.empty(max(1, a.shape[0]), np.uint64)
  n = lib().orc_set_difference_u64(_p64(a), a.shape[0], _p64(b), b.shape[0], _p64(out))
  return out[:n]


def merge(a: np.ndarray, b: np.ndarray) -> np.ndarray:
  a = np.ascontiguousarray(a, np.uint64)
  b = np.ascontiguousarray(b, np.uint64)
  out = np.empty(max(1, a.shape[0] + b.shape[0]), np.uint64)
  n = lib().orc_merge_u64(_p64(a), a.shape[0], _p64(b), b.shape[0], _p64(out))
  return out[:n]


def _run(fn, edges: np.ndarray, max_iters: int):
  keys = np.ascontiguousarray(pack(edges), np.uint64)
  r = _Result()
  rc = fn(_p64(keys), keys.shape[0], max_iters or (2**31 - 1), ctypes.byref(r))
  if rc != 0:
    raise RuntimeError(f'oracle failed: {rc}')
  out = np.ctypeslib.as_array(r.keys, shape=(r.n,)).copy() if r.n else np.zeros(0, np.uint64)
  lib().orc_free(ctypes.cast(r.keys, ctypes.c_void_p))
  return out, int(r.iterations), int(r.derived)


def tc(edges: np.ndarray, max_iters: int = 0):
  '''Path relation keys in canonical index order (1,0), iterations, derived rows.'''
  return _run(lib().orc_tc, edges, max_iters)


def sg(edges: np.ndarray, max_iters: int = 0):
  '''Sg relation keys in canonical index order (0,1), iterations, derived rows.'''
  return _run(lib().orc_sg, edges, max_iters)


def triangle_count(edges: np.ndarray) -> int:
  keys = np.ascontiguousarray(pack(edges), np.uint64)
  return int(lib().orc_triangle_count(_p64(keys), keys.shape[0]))


def triangle_count_sample(edges: np.ndarray, stride: int, phase: int = 0):
  '''(sampled count, sort seconds, sampled-join seconds) over every stride-th edge.'''
  keys = np.ascontiguousarray(pack(edges), np.uint64)
  ts, tj = ctypes.c_double(), ctypes.c_double()
  c = lib().orc_triangle_count_sample(_p64(keys), keys.shape[0], stride, phase, ctypes.byref(ts),
                                      ctypes.byref(tj))
  return int(c), ts.value, tj.value


def num_threads() -> int:
  return int(lib().orc_num_threads())


def dump_hash(rows: np.ndarray) -> str:
  '''SHA-256 of a relation dump: rows sorted lexicographically in declared
  column order, serialised row-major as little-endian uint32.'''
  r = np.ascontiguousarray(rows, dtype='<u4')
  if r.shape[0]:
    order = np.lexsort(tuple(r[:, c] for c in reversed(range(r.shape[1]))))
    r = np.ascontiguousarray(r[order])
  return hashlib.sha256(r.tobytes()).hexdigest()


# ---------------------------------------------------------------------------
# Order-free fingerprints of binary relations (batched runs)
# ---------------------------------------------------------------------------
#
# The library reports, per instance of a batched run, the sum mod 2^64 of
# fx(x) * fy(y) over the instance's rows (x, y) in its own values
# (srdl_range_checksums), fx(v) = m(v ^ 0x243F6A8885A308D3), fy(v) = m(v ^
# 0x13198A2E03707344), m the SplitMix64 output function.  Because the sum is
# bilinear, a transitive closure's fingerprint is the sum over sources x of
# fx(x) * (sum of fy over x's reachability set), which
# `tc_closure_fingerprint` computes from strongly connected components
# without listing the |Path| pairs (up to ~4*10^9 for one instance of the
# batched config) -- an exact check of instances the semi-naive
# restatement above is too slow for.

def _splitmix64(v: np.ndarray) -> np.ndarray:
  '''SplitMix64 output function (Steele, Lea and Flood, OOPSLA 2014;
  Vigna's splitmix64.c constants), elementwise on uint64 (wrapping).'''
  z = np.asarray(v, np.uint64).copy()
  with np.errstate(over='ignore'):
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def fp_x(v) -> np.ndarray:
  return _splitmix64(np.asarray(v, np.uint64) ^ np.uint64(0x243F6A8885A308D3))


def fp_y(v) -> np.ndarray:
  return _splitmix64(np.asarray(v, np.uint64) ^ np.uint64(0x13198A2E03707344))


def _wsum(a: np.ndarray) -> int:
  '''Sum of uint64 values mod 2^64.'''
  with np.errstate(over='ignore'):
    return int(np.sum(np.asarray(a, np.uint64), dtype=np.uint64))


def row_fingerprint(rows: np.ndarray) -> int:
  '''Fingerprint of a set of (x, y) rows (uint32, declared column order).'''
  r = np.asarray(rows, np.uint32).reshape(-1, 2)
  if not r.shape[0]:
    return 0
  with np.errstate(over='ignore'):
    return _wsum(fp_x(r[:, 0]) * fp_y(r[:, 1]))


def tc_closure_fingerprint(edges: np.ndarray, n: int | None = None) -> tuple:
  '''(|Path|, fingerprint of Path) for Path = the pairs (x, y) joined by a
  path of one or more edges -- the least fixpoint of the TC program
  (Path(x,y) <= Edge(x,y); Path(x,z) <= Path(x,y), Edge(y,z)) -- by
  strongly connected components (Tarjan 1972 via scipy) and their
  condensation in reverse topological order.  R(S), the nodes reachable in
  one or more steps from a component S, is S itself when S has a cycle,
  plus (T u R(T)) for every successor T.  The largest component C is kept
  implicit: R(S) = [R(C) if S reaches C] + an explicit set of the other
  nodes, which stays small on graphs with one giant component.'''
  import scipy.sparse as sp
  from scipy.sparse.csgraph import breadth_first_order, connected_components
  e = np.asarray(edges, np.int64).reshape(-1, 2)
  if n is None:
    n = int(e.max()) + 1 if e.shape[0] else 0
  if not e.shape[0]:
    return 0, 0
  g = sp.csr_matrix((np.ones(e.shape[0], np.int8), (e[:, 0], e[:, 1])), shape=(n, n))
  ncomp, lab = connected_components(g, directed=True, connection='strong')
  lab = lab.astype(np.int64)
  size = np.bincount(lab, minlength=ncomp)
  selfloop = np.zeros(ncomp, bool)
  sl = e[:, 0] == e[:, 1]
  selfloop[lab[e[sl, 0]]] = True
  cyclic = (size > 1) | selfloop
  members = [[] for _ in range(ncomp)]
  order = np.argsort(lab, kind='stable')
  cuts = np.searchsorted(lab[order], np.arange(ncomp + 1))
  for c in range(ncomp):
    members[c] = order[cuts[c]:cuts[c + 1]]
  # condensation edges, deduplicated
  cs, cd = lab[e[:, 0]], lab[e[:, 1]]
  keep = cs != cd
  dag = np.unique(cs[keep] * ncomp + cd[keep])
  ds, dd = dag // ncomp, dag % ncomp
  succ_cut = np.searchsorted(ds, np.arange(ncomp + 1))
  # reverse topological order (Kahn on the reversed condensation)
  outdeg = np.diff(succ_cut).astype(np.int64)
  pred_order = np.argsort(dd, kind='stable')
  pred_src = ds[pred_order]
  pred_cut = np.searchsorted(dd[pred_order], np.arange(ncomp + 1))
  stack = list(np.nonzero(outdeg == 0)[0])
  rev_topo = []
  while stack:
    c = stack.pop()
    rev_topo.append(c)
    for p in pred_src[pred_cut[c]:pred_cut[c + 1]]:
      outdeg[p] -= 1
      if outdeg[p] == 0:
        stack.append(p)
  hub = int(np.argmax(size))
  fy_all = fp_y(np.arange(n, dtype=np.uint64))
  if cyclic[hub]:
    reach_hub = breadth_first_order(g, int(members[hub][0]), directed=True, return_predecessors=False)
    in_hub = np.zeros(n, bool)
    in_hub[reach_hub] = True
    hub_size, hub_g = int(reach_hub.shape[0]), _wsum(fy_all[reach_hub])
  else:
    in_hub = np.zeros(n, bool)
    hub_size, hub_g = 0, 0
  flag = np.zeros(ncomp, bool)        # R(S) includes R(hub)
  explicit = [None] * ncomp           # the rest of R(S)
  comp_size = np.zeros(ncomp, np.int64)
  comp_g = np.zeros(ncomp, np.uint64)
  empty = frozenset()
  for c in rev_topo:
    if c == hub and cyclic[hub]:
      flag[c], explicit[c] = True, empty
    else:
      f = False
      parts = []
      for t in dd[succ_cut[c]:succ_cut[c + 1]]:
        f = f or bool(flag[t]) or (t == hub and cyclic[hub])
        parts.append(members[t])
        if explicit[t]:
          parts.append(np.fromiter(explicit[t], np.int64, len(explicit[t])))
      if cyclic[c]:
        parts.append(members[c])
      if parts:
        s = np.unique(np.concatenate(parts))
        if f:
          s = s[~in_hub[s]]
        ex = frozenset(s.tolist())
      else:
        ex = empty
      flag[c], explicit[c] = f, ex
    ex = explicit[c]
    comp_size[c] = (hub_size if flag[c] else 0) + len(ex)
    g_ex = _wsum(fy_all[np.fromiter(ex, np.int64, len(ex))]) if ex else 0
    comp_g[c] = np.uint64(((hub_g if flag[c] else 0) + g_ex) & 0xFFFFFFFFFFFFFFFF)
  total = int(np.sum(comp_size[lab]))
  with np.errstate(over='ignore'):
    fpr = _wsum(fp_x(np.arange(n, dtype=np.uint64)) * comp_g[lab])
  return total, fpr


def _tc_fp_job(job):
  return tc_closure_fingerprint(*job)


def tc_closure_fingerprints(jobs: list, workers: int = 0) -> list:
  """tc_closure_fingerprint over [(edges, n), ...] in a pool of processes
  started with spawn (safe after the caller has used a GPU)."""
  import concurrent.futures as cf
  import multiprocessing as mp
  workers = workers or min(16, os.cpu_count() or 1)
  if workers <= 1 or len(jobs) < 8:
    return [tc_closure_fingerprint(*j) for j in jobs]
  with cf.ProcessPoolExecutor(workers, mp_context=mp.get_context('spawn')) as ex:
    return list(ex.map(_tc_fp_job, jobs, chunksize=16))


# ---------------------------------------------------------------------------
# Generic pure-Python plan interpreter (tiny inputs only)
# ---------------------------------------------------------------------------

def _filter_fn(code: str):
  import re
  body = code.strip()[len('return'):-1].strip()
  terms = []
  for part in body.split('&&'):
    m = re.match(r'^\(?\s*(\w+)\s*(!=|==|<=|>=|<|>)\s*(\w+)\s*\)?$', part.strip())
    if not m:
      raise ValueError(f'unsupported filter {code!r}')
    terms.append(m.groups())
  ops = {'!=': lambda a, b: a != b, '==': lambda a, b: a == b, '<': lambda a, b: a < b,
         '<=': lambda a, b: a <= b, '>': lambda a, b: a > b, '>=': lambda a, b: a >= b}

  def ev(bind):
    def val(t):
      return int(t) if t.isdigit() else bind[t]
    return all(ops[o](val(a), val(b)) for a, o, b in terms)
  return ev


def run_plan(plan: dict, inputs: dict, max_iters: int = 0):
  '''Evaluate `plan` over `inputs` ({relation: (m,k) uint32 rows}).

  Returns ({relation: sorted list of tuples in declared column order},
  {rule: count} for count-only rules).  Semantics:
  insert_into adds to NEW; rebuild_index dedups NEW; compute_delta_index
  sets DELTA = NEW - FULL (gpu_mir_helpers.h:88-122); merge_index sets
  FULL |= DELTA (gpu_mir_helpers.h:136-159); recursive steps loop until
  the delta of every relation the step computes is empty, iteration 0
  reading FULL for DELTA (gpu_mir_helpers.h:419-426).
  '''
  rels = {r['name']: r for r in plan['relations']}
  db = {(n, v): set() for n in rels for v in ('FULL', 'DELTA', 'NEW')}
  for name, rows in inputs.items():
    db[(name, 'FULL')] = {tuple(int(x) for x in r) for r in np.asarray(rows).reshape(-1, rels[name]['arity'])}
  for name, r in rels.items():
    # rows the plan carries (the one-tuple relations of head constants)
    db[(name, 'FULL')] |= {tuple(int(x) for x in row) for row in r.get('facts', ())}
  counts: dict[str, int] = {}
  cap = max_iters or (2**31 - 1)

  def values(src, bind, iteration):
    ver = src['ver']
    if ver == 'DELTA' and iteration == 0:
      ver = 'FULL'
    idx = src['index']
    pre = [bind[v] for v in src['prefix']]
    col = idx[len(pre)]
    out = set()
    for t in db[(src['rel'], ver)]:
      if all(t[idx[i]] == pre[i] for i in range(len(pre))):
        out.add(t[col])
    return out

  def tuples(src, bind, iteration, k):
    # distinct values of the k index columns after the prefix
    ver = src['ver']
    if ver == 'DELTA' and iteration == 0:
      ver = 'FULL'
    idx = src['index']
    pre = [bind[v] for v in src['prefix']]
    cols = idx[len(pre):len(pre) + k]
    return {tuple(t[c] for c in cols) for t in db[(src['rel'], ver)]
            if all(t[idx[i]] == pre[i] for i in range(len(pre)))}

  def execute(op, iteration):
    binds = [dict()]
    for p in op['pipeline']:
      k = p['op']
      nb = []
      if k == 'scan':
        for b in binds:
          ver = 'FULL' if (p['ver'] == 'DELTA' and iteration == 0) else p['ver']
          for t in db[(p['rel'], ver)]:
            c = dict(b)
            ok = True
            # Scan vars follow the index's access order (generate_scan,
            # src/srdatalog/hir/lower.py:46-60): vars[j] <-> column index[j].
            for j, v in enumerate(p['vars']):
              val = t[p['index'][j]]
              if v in c and c[v] != val:
                ok = False
              c[v] = val
            if ok:
              nb.append(c)
      elif k == 'column_join':
        for b in binds:
          vs = None
          for s in p['sources']:
            x = values(s, b, iteration)
            vs = x if vs is None else (vs & x)
          for v in sorted(vs):
            c = dict(b)
            c[p['var']] = v
            nb.append(c)
      elif k == 'cartesian_join':
        # a source binds the len(vars) columns after its prefix, in index
        # order (a ternary source under one bound column binds two); an
        # empty var list only requires the prefix to be present
        for b in binds:
          lists = []
          empty = False
          for s, vars_ in zip(p['sources'], p['var_from_source']):
            vs = tuples(s, b, iteration, max(1, len(vars_)))
            empty |= not vs
            if vars_:
              lists.append((vars_, sorted(vs)))
          if empty:
            continue
          for combo in itertools.product(*[lst for _, lst in lists]):
            c = dict(b)
            for (vars_, _), vals in zip(lists, combo):
              for v, val in zip(vars_, vals):
                c[v] = val
            nb.append(c)
      elif k == 'filter':
        ev = _filter_fn(p['code'])
        nb = [b for b in binds if ev(b)]
      elif k == 'negation':
        # keep a binding iff no tuple of the relation starts (in index order)
        # with the prefix values
        # (constant arguments first: their columns lead the index,
        # src/srdatalog/hir/plan.py:284-286)
        idx, pre, cp = p['index'], p['prefix'], tuple(p.get('const_prefix', []))
        k = len(cp) + len(pre)
        present = {tuple(t[idx[i]] for i in range(k)) for t in db[(p['rel'], p['ver'])]}
        nb = [b for b in binds if cp + tuple(b[v] for v in pre) not in present]
      elif k == 'insert_into':
        if op['count']:
          counts[op['rule']] = counts.get(op['rule'], 0) + len(binds)
        else:
          tgt = db[(p['rel'], 'NEW')]
          for b in binds:
            tgt.add(tuple(b[v] for v in p['vars']))
        nb = binds
      binds = nb

  def run_ops(ops, iteration):
    for op in ops:
      k = op['op']
      if k == 'execute_pipeline':
        execute(op, iteration)
      elif k == 'compute_delta_index':
        db[(op['rel'], 'DELTA')] = db[(op['rel'], 'NEW')] - db[(op['rel'], 'FULL')]
      elif k == 'merge_index':
        db[(op['rel'], 'FULL')] = db[(op['rel'], 'FULL')] | db[(op['rel'], 'DELTA')]
      elif k == 'clear_relation':
        if op['ver'] == 'NEW':
          db[(op['rel'], 'NEW')] = set()
        # DELTA is cleared right before compute_delta_index overwrites it
        # (lower.py: ClearRelation(DELTA) precedes ComputeDeltaIndex).

  for step in plan['steps']:
    ops = step['ops']
    if not step['recursive']:
      run_ops(ops, 0)
      continue
    computed = {op['rel'] for op in ops if op['op'] == 'compute_delta_index'}
    for it in range(cap):
      if it > 0 and sum(len(db[(r, 'DELTA')]) for r in computed) == 0:
        break
      run_ops(ops, it)
  out = {n: sorted(db[(n, 'FULL')]) for n in rels}
  return out, counts


def _by_first(rel: set) -> dict:
  out: dict = {}
  for a, b in rel:
    out.setdefault(a, set()).add(b)
  return out


def andersen(inputs: dict) -> list:
  '''PointsTo of examples/andersen.py:60-97 by naive iteration over Python
  sets (rules Base, Assign, Load, Store), independent of any plan.'''
  pts = set(map(tuple, np.asarray(inputs['AddressOf']).tolist()))
  assign = list(map(tuple, np.asarray(inputs['Assign']).tolist()))
  load = list(map(tuple, np.asarray(inputs['Load']).tolist()))
  store = list(map(tuple, np.asarray(inputs['Store']).tolist()))
  while True:
    by = _by_first(pts)
    new = set()
    for y, z in assign:                       # PointsTo(y,x) <= PointsTo(z,x), Assign(y,z)
      for x in by.get(z, ()):
        new.add((y, x))
    for y, x in load:                         # PointsTo(y,w) <= PointsTo(x,z), Load(y,x), PointsTo(z,w)
      for z in by.get(x, ()):
        for w in by.get(z, ()):
          new.add((y, w))
    for y, x in store:                        # PointsTo(z,w) <= PointsTo(y,z), Store(y,x), PointsTo(x,w)
      for z in by.get(y, ()):
        for w in by.get(x, ()):
          new.add((z, w))
    if new <= pts:
      return sorted(pts)
    pts |= new


def cspa(inputs: dict) -> dict:
  '''ValueFlow / ValueAlias / MemoryAlias of examples/cspa.py:75-108 by naive
  iteration over Python sets, independent of any plan.'''
  assign = set(map(tuple, np.asarray(inputs['AssignInput']).tolist()))
  deref = set(map(tuple, np.asarray(inputs['DerefInput']).tolist()))
  vf = set(assign)                                              # VF_Assign
  vf |= {(x, x) for x, _ in assign} | {(x, x) for _, x in assign}   # VF_Refl1/2
  ma = {(x, x) for _, x in assign} | {(x, x) for x, _ in assign}    # MA_Refl1/2
  va: set = set()
  while True:
    vf_by, ma_by, va_by, de_by = _by_first(vf), _by_first(ma), _by_first(va), _by_first(deref)
    n_vf = {(x, y) for x, z in vf for y in vf_by.get(z, ())}            # VF_Trans
    n_vf |= {(x, y) for x, z in assign for y in ma_by.get(z, ())}       # VF_Assign_MA
    n_va = {(x, y) for z, xs in vf_by.items() for x in xs for y in xs}  # VA_VF
    n_va |= {(x, y) for z, xs in vf_by.items() for w in ma_by.get(z, ())
             for x in xs for y in vf_by.get(w, ())}                      # VA_VF_MA_VF
    n_ma = {(x, w) for y, xs in de_by.items() for z in va_by.get(y, ())
            for x in xs for w in de_by.get(z, ())}                       # MA_Deref_VA
    if n_vf <= vf and n_va <= va and n_ma <= ma:
      return {'ValueFlow': sorted(vf), 'ValueAlias': sorted(va), 'MemoryAlias': sorted(ma)}
    vf |= n_vf
    va |= n_va
    ma |= n_ma


def lsqb_q7(inputs: dict) -> dict:
  '''Counts of examples/lsqb_q7_optional.py:106-131 in closed form: with T, C,
  R, L the numbers of distinct tags, creators, replying comments and likers
  of a message, Case1 = sum T*C*R*L, Case2 = sum over messages without likers
  of T*C*R, Case3 = sum over messages without replies of T*C*L, Case4 = sum
  over messages with neither of T*C.'''
  def per_msg(rows, col):
    a = np.unique(np.asarray(rows, np.int64), axis=0)
    keys, cnt = np.unique(a[:, col], return_counts=True)
    return dict(zip(keys.tolist(), cnt.tolist()))
  t = per_msg(inputs['HasTag'], 0)
  c = per_msg(inputs['HasCreator'], 0)
  r = per_msg(inputs['ReplyOf'], 1)
  lk = per_msg(inputs['Likes'], 1)
  out = {'Case1Both': 0, 'Case2ReplyOnly': 0, 'Case3LikeOnly': 0, 'Case4Neither': 0}
  for m, nt in t.items():
    nc = c.get(m, 0)
    nr, nl = r.get(m, 0), lk.get(m, 0)
    out['Case1Both'] += nt * nc * nr * nl
    if nl == 0:
      out['Case2ReplyOnly'] += nt * nc * nr
    if nr == 0:
      out['Case3LikeOnly'] += nt * nc * nl
    if nr == 0 and nl == 0:
      out['Case4Neither'] += nt * nc
  return out


def lsqb_q6(inputs: dict) -> int:
  '''Count of examples/lsqb_q6_count.py:70-91 in closed form: Knows is the
  symmetric closure of the input, N(p) its neighbours and I(p) the distinct
  interests of p; the bindings (p1, p2, p3, t) with p1 != p3 number
  sum over p2 of (|N(p2)| - 1) * sum over p3 in N(p2) of I(p3).'''
  e = np.asarray(inputs['KnowsInput'], np.int64)
  k = np.unique(np.concatenate([e, e[:, ::-1]]), axis=0)
  hi = np.unique(np.asarray(inputs['HasInterestInput'], np.int64), axis=0)
  n = int(max(k.max(initial=0), hi[:, 0].max(initial=0))) + 1
  interests = np.bincount(hi[:, 0], minlength=n)
  deg = np.bincount(k[:, 0], minlength=n)
  s = np.bincount(k[:, 0], weights=interests[k[:, 1]], minlength=n)
  return int(np.sum((deg - 1) * s))


def _adj(rows) -> dict:
  out: dict = {}
  for a, b in np.unique(np.asarray(rows, np.int64).reshape(-1, 2), axis=0).tolist():
    out.setdefault(a, set()).add(b)
  return out


def lsqb_q3(inputs: dict) -> list:
  '''Triangle of examples/lsqb_q3_triangle.py:66-85, by Python sets:
  (p1, p2, p3) with Knows(p1,p2), Knows(p2,p3), Knows(p3,p1) whose three
  people are located in cities of one country.'''
  knows = _adj(inputs['KnowsInput'])
  city = {p: c for p, c in np.asarray(inputs['IsLocatedInInput']).tolist()}
  country = {c: k for c, k in np.asarray(inputs['IsPartOfInput']).tolist()}
  loc = _adj(inputs['IsLocatedInInput'])
  part = _adj(inputs['IsPartOfInput'])
  del city, country
  out = set()
  for p1, n1 in knows.items():
    for p2 in n1:
      for p3 in knows.get(p2, ()):
        if p1 not in knows.get(p3, ()):
          continue
        cos = [set().union(*(part.get(c, set()) for c in loc.get(p, ()))) for p in (p1, p2, p3)]
        if cos[0] & cos[1] & cos[2]:
          out.add((p1, p2, p3))
  return sorted(out)


def triangle3(a, b, c) -> list:
  '''Z(x,y,z) <= A(x,y), B(y,z), C(z,x) (examples/debug_triangle.py:55-59;
  examples/gen_jit_code.py:39-43 with A = B = C = Edge), by Python sets.'''
  ab, bb, cb = _adj(a), _adj(b), _adj(c)
  out = []
  for x, ys in ab.items():
    for y in ys:
      for z in bb.get(y, ()):
        if x in cb.get(z, ()):
          out.append((x, y, z))
  return sorted(out)


def lsqb_two_hop(inputs: dict, second: str | None = None, negate: bool = False,
                 as_planned: bool = True) -> set:
  '''Path of examples/lsqb_q6_2hop.py:66-85 (second hop over a second Knows
  copy: lsqb_q6_nosj.py; ends that do not know each other: lsqb_q9_neg2hop.py
  :66-90), by Python sets: (p1, p2, p3, t) with Knows(p1,p2),
  Knows'(p2,p3), HasInterest(p3,t), p1 != p3 (and not Knows(p1,p3)).

  as_planned: the reference's planner lowers the first atom of the 2hop and
  nosj rules to a join on Knows' column 0 for p2 (fixtures
  tests/fixtures/integration/lsqb_q6_2hop.mir.sexpr, lsqb_q6_nosj.mir.sexpr:
  both p2 sources use index (0 1) with an empty prefix, p1 then comes from
  Knows[p2]), i.e. it evaluates Knows(p2,p1); the reference executes that
  plan, so its output is this reading.  Q9's plan reads Knows(p1,p2) through
  index (1 0), the rule as written.'''
  k1 = _adj(inputs['KnowsInput'])
  k2 = _adj(inputs[second]) if second else k1
  hi = _adj(inputs['HasInterestInput'])
  first = k1
  if as_planned and not negate:
    rev: dict = {}
    for a, bs in k1.items():
      for b in bs:
        rev.setdefault(b, set()).add(a)
    first = rev  # first[p1] = {p2 : Knows(p2, p1)}
  out = set()
  for p1, n1 in first.items():
    for p2 in n1:
      for p3 in k2.get(p2, ()):
        if p1 == p3 or (negate and p3 in k1.get(p1, ())):
          continue
        for t in hi.get(p3, ()):
          out.add((p1, p2, p3, t))
  return out


def reach_avoid(edges: np.ndarray, blocked: np.ndarray) -> dict:
  '''Reach = transitive closure of Edge minus Blocked edges; Cut = Blocked
  pairs not in Reach (the reach_avoid test program), by Python sets.'''
  blk = set(map(tuple, np.asarray(blocked).tolist()))
  ok = [tuple(e) for e in np.asarray(edges).tolist() if tuple(e) not in blk]
  succ: dict = {}
  for a, b in ok:
    succ.setdefault(a, set()).add(b)
  reach = set(ok)
  frontier = set(ok)
  while frontier:
    new = {(x, z) for x, y in frontier for z in succ.get(y, ())} - reach
    reach |= new
    frontier = new
  return {'Reach': sorted(reach), 'Cut': sorted(p for p in blk if p not in reach)}


def head_const(edges: np.ndarray, sources: np.ndarray) -> list:
  '''Mark of the head_const test program, by Python sets: (r, 7) for every
  node r reachable from a source (sources included), (x, 9) for every edge
  (x, y) whose target y is such a node.'''
  succ: dict = {}
  pairs = [tuple(e) for e in np.asarray(edges).reshape(-1, 2).tolist()]
  for a, b in pairs:
    succ.setdefault(a, set()).add(b)
  reach = set(np.asarray(sources).reshape(-1).tolist())
  frontier = set(reach)
  while frontier:
    frontier = {z for y in frontier for z in succ.get(y, ())} - reach
    reach |= frontier
  return sorted({(r, 7) for r in reach} | {(x, 9) for x, y in pairs if y in reach})


def rewrite_consts(in3: np.ndarray, in2: np.ndarray) -> dict:
  '''P and Q of the reference's rewrite_consts program
  (tests/test_rule_rewrite.py:99): P = {x | (x, 42, 99) in In},
  Q = {(x, 7) | x in In2}.'''
  p = {(int(r[0]),) for r in np.asarray(in3).reshape(-1, 3) if r[1] == 42 and r[2] == 99}
  q = {(int(x), 7) for x in np.asarray(in2).reshape(-1)}
  return {'P': sorted(p), 'Q': sorted(q)}


def galen(inputs: dict) -> dict:
  '''OutP and OutQ of the Galen program (examples/galen.py rules LoadP ..
  Join3c), by naive iteration over Python sets until nothing changes.'''
  def rows(name, k):
    return {tuple(int(x) for x in r) for r in np.asarray(inputs[name]).reshape(-1, k).tolist()}
  p_in, s_in = rows('PInput', 2), rows('SInput', 2)
  q_in, r_in, c_in, u_in = (rows(n, 3) for n in ('QInput', 'RInput', 'CInput', 'UInput'))
  out_p, out_q = set(p_in), set(q_in)
  s_by, r_by, u_by = {}, {}, {}
  for r, q in s_in:
    s_by.setdefault(r, set()).add(q)
  for y, u, e in r_in:
    r_by.setdefault(y, set()).add((u, e))
  for w, r, z in u_in:
    u_by.setdefault(w, set()).add((r, z))
  while True:
    p_from, q_from, q_xry = {}, {}, {}
    for x, y in out_p:
      p_from.setdefault(x, set()).add(y)
    for x, r, z in out_q:
      q_from.setdefault(x, set()).add((r, z))
      q_xry.setdefault((r, z), set()).add(x)
    new_p, new_q = set(), set()
    for x, y in out_p:
      for z in p_from.get(y, ()):                        # TC
        new_p.add((x, z))
      for r, z in q_from.get(y, ()):                     # PropQ
        new_q.add((x, r, z))
    for y, w in out_p:                                   # Join3a: OutQ(x, r, y)
      for r, z in u_by.get(w, ()):
        for x in q_xry.get((r, y), ()):
          new_p.add((x, z))
    for y, w, z in c_in:                                 # Join3b
      for x, ys in p_from.items():
        if w in ys and y in ys:
          new_p.add((x, z))
    for x, r, z in out_q:
      for q in s_by.get(r, ()):                          # PropQS
        new_q.add((x, q, z))
      for u, e in r_by.get(r, ()):                       # Join3c, y = r
        for uu, o in q_from.get(z, ()):
          if uu == u:
            new_q.add((x, e, o))
    if new_p <= out_p and new_q <= out_q:
      return {'OutP': sorted(out_p), 'OutQ': sorted(out_q)}
    out_p |= new_p
    out_q |= new_q


def live(inputs: dict) -> dict:
  '''Live and Out of the live test program, by Python sets: Live(v, p) for
  every (v, q) in Used with p reaching q over Cfg edges (p -> q), zero or
  more steps; Out(o, p) for Live(v, p) and Derefs(v, o).'''
  def rows(name):
    return {tuple(int(x) for x in r) for r in np.asarray(inputs[name]).reshape(-1, 2).tolist()}
  used, cfg, derefs = rows('Used'), rows('Cfg'), rows('Derefs')
  pred: dict = {}
  for p, q in cfg:
    pred.setdefault(q, set()).add(p)
  lv = set(used)
  frontier = set(used)
  while frontier:
    new = {(v, p) for v, q in frontier for p in pred.get(q, ())} - lv
    lv |= new
    frontier = new
  by_v: dict = {}
  for v, o in derefs:
    by_v.setdefault(v, set()).add(o)
  out = {(o, p) for v, p in lv for o in by_v.get(v, ())}
  return {'Live': sorted(lv), 'Out': sorted(out)}
