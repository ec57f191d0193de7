'''Seeded synthetic inputs for the benchmark programs (uint32 edge lists).

Every generator returns an (m, 2) uint32 numpy array of directed edges
(column 0 = source, column 1 = target) in draw order, duplicates and
self-loops already removed where the workload says so.  numpy's
`Generator(PCG64(seed))` is the only randomness source, so a seed fully
determines the input on every machine.

These stand in for the reference's CSV inputs (examples/tc.py `Arc.csv`,
examples/sg.py `Arc.csv`, examples/lsqb_triangle_count.py
`Person_knows_Person.csv`); no public dataset is used.
'''

from __future__ import annotations

import math

import numpy as np


def _rng(seed: int) -> np.random.Generator:
  return np.random.Generator(np.random.PCG64(seed))


def _dedup_in_order(src: np.ndarray, dst: np.ndarray) -> np.ndarray:
  key = (src.astype(np.uint64) << np.uint64(32)) | dst.astype(np.uint64)
  _, first = np.unique(key, return_index=True)
  first.sort()
  return np.stack([src[first], dst[first]], axis=1).astype(np.uint32)


def uniform_edges(n_nodes: int, n_edges: int, seed: int = 1) -> np.ndarray:
  '''TC input: draw (src,dst) uniformly in [0,n_nodes), drop self-loops,
  keep the first `n_edges` distinct pairs in draw order.'''
  if n_edges > n_nodes * (n_nodes - 1):
    raise ValueError('more distinct edges requested than the graph can hold')
  rng = _rng(seed)
  out = np.zeros((0, 2), np.uint32)
  batch = max(1024, int(n_edges * 1.3))
  src_all = np.zeros(0, np.uint32)
  dst_all = np.zeros(0, np.uint32)
  while out.shape[0] < n_edges:
    s = rng.integers(0, n_nodes, batch, dtype=np.uint32)
    d = rng.integers(0, n_nodes, batch, dtype=np.uint32)
    keep = s != d
    src_all = np.concatenate([src_all, s[keep]])
    dst_all = np.concatenate([dst_all, d[keep]])
    out = _dedup_in_order(src_all, dst_all)
  return np.ascontiguousarray(out[:n_edges])


def tc_small(seed: int = 1) -> np.ndarray:
  '''Transitive-closure config: 20,000 distinct directed edges over 5,000 nodes.'''
  return uniform_edges(5000, 20000, seed)


def sg_forest(n_nodes: int = 200_000, window: int = 1000, cross_frac: float = 0.1,
              seed: int = 2) -> np.ndarray:
  '''Same-generation config: node i>0 takes a parent uniform in
  [max(0,i-window), i-1]; round(cross_frac*(n-1)) extra cross edges (u,v)
  with u<v after ordering, self-pairs dropped; all edges deduplicated.
  Edges point parent -> child (Arc(p, x)).'''
  rng = _rng(seed)
  i = np.arange(1, n_nodes, dtype=np.int64)
  lo = np.maximum(0, i - window)
  par = lo + (rng.random(i.shape[0]) * (i - lo)).astype(np.int64)
  par = np.minimum(par, i - 1)
  n_cross = int(round(cross_frac * (n_nodes - 1)))
  u = rng.integers(0, n_nodes, n_cross, dtype=np.int64)
  v = rng.integers(0, n_nodes, n_cross, dtype=np.int64)
  a, b = np.minimum(u, v), np.maximum(u, v)
  keep = a != b
  src = np.concatenate([par, a[keep]]).astype(np.uint32)
  dst = np.concatenate([i, b[keep]]).astype(np.uint32)
  return _dedup_in_order(src, dst)


def rmat_edges(scale: int = 20, n_draws: int = 1 << 24, abcd=(0.57, 0.19, 0.19, 0.05),
               seed: int = 3, chunk: int = 1 << 22) -> np.ndarray:
  '''Triangle config: R-MAT with 2^scale nodes and n_draws draws; each
  edge oriented as (min, max); self-loops and duplicates removed.'''
  a, b, c, _ = abcd
  rng = _rng(seed)
  srcs, dsts = [], []
  left = n_draws
  while left > 0:
    k = min(chunk, left)
    s = np.zeros(k, np.uint32)
    d = np.zeros(k, np.uint32)
    for level in range(scale):
      r = rng.random(k)
      bit = np.uint32(1 << (scale - 1 - level))
      down = r >= a + b            # quadrant c or d: source bit set
      right = ((r >= a) & (r < a + b)) | (r >= a + b + c)  # b or d: target bit set
      s |= np.where(down, bit, np.uint32(0))
      d |= np.where(right, bit, np.uint32(0))
    srcs.append(s)
    dsts.append(d)
    left -= k
  s = np.concatenate(srcs)
  d = np.concatenate(dsts)
  lo, hi = np.minimum(s, d), np.maximum(s, d)
  keep = lo != hi
  return _dedup_in_order(lo[keep], hi[keep])


def er_instance(n_nodes: int, mean_deg: float, seed: int) -> np.ndarray:
  '''Batched-TC instance: round(mean_deg*n) directed Erdos-Renyi draws,
  self-loops and duplicates removed.'''
  rng = _rng(seed)
  m = int(round(mean_deg * n_nodes))
  s = rng.integers(0, n_nodes, m, dtype=np.uint32)
  d = rng.integers(0, n_nodes, m, dtype=np.uint32)
  keep = s != d
  return _dedup_in_order(s[keep], d[keep])


def batched_shapes(count: int = 4096, n_lo: int = 64, n_hi: int = 65536,
                   deg_lo: float = 2.0, deg_hi: float = 8.0, seed0: int = 1000):
  '''(n_j, c_j) of the batched-fixpoint config: n_j = round(exp(U[ln n_lo,
  ln n_hi])) nodes and mean out-degree c_j = U[deg_lo, deg_hi], drawn with
  seed seed0+j.'''
  out = []
  for j in range(count):
    rng = _rng(seed0 + j)
    n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
    c = float(rng.uniform(deg_lo, deg_hi))
    out.append((n, c))
  return out


def batched_instances(count: int = 4096, n_lo: int = 64, n_hi: int = 65536,
                      deg_lo: float = 2.0, deg_hi: float = 8.0, seed0: int = 1000,
                      n_max: int | None = None, only=None):
  '''Batched-fixpoint config: instance j is a directed Erdos-Renyi graph
  (er_instance, seed seed0 + j + 10^6) of the shape batched_shapes draws.
  n_max keeps the instances with n_j <= n_max, `only` the listed j (the
  config's own draws either way).'''
  out = []
  keep = None if only is None else set(only)
  for j, (n, c) in enumerate(batched_shapes(count, n_lo, n_hi, deg_lo, deg_hi, seed0)):
    if (n_max is not None and n > n_max) or (keep is not None and j not in keep):
      continue
    out.append(er_instance(n, c, seed0 + j + 1_000_000))
  return out


def served_request_input(program: str, m: int, seed: int) -> dict:
  '''Input of one served request with about m input edges, generated as in
  the corresponding config but kept small enough for its closure to fit:
  TC on a subcritical Erdos-Renyi graph (n = 2m nodes, mean out-degree 1/2),
  SG on the windowed forest with n = m/1.1 nodes (m capped at 5,500), and
  the triangle count on an R-MAT graph with m draws (edge factor ~8).'''
  if program == 'tc':
    return {'ArcInput': er_instance(max(2, 2 * m), 0.5, seed)}
  if program == 'sg':
    n = max(16, int(round(min(m, 5_500) / 1.1)))
    return {'Arc': sg_forest(n, window=min(1000, n - 1), seed=seed)}
  if program == 'triangle':
    scale = max(6, int(math.ceil(math.log2(max(m, 64) / 8))))
    return {'KnowsInput': rmat_edges(scale, m, seed=seed, chunk=1 << 20)}
  raise ValueError(program)


def write_csv(edges: np.ndarray, path: str, delimiter: str = '\t') -> None:
  '''Write an edge list as the reference's loader reads it (one row per line).'''
  np.savetxt(path, edges.astype(np.int64), fmt='%d', delimiter=delimiter)


def _pairs(rng: np.random.Generator, n_vars: int, m: int) -> np.ndarray:
  s = rng.integers(0, n_vars, m, dtype=np.uint32)
  d = rng.integers(0, n_vars, m, dtype=np.uint32)
  return _dedup_in_order(s, d)


def andersen_inputs(n_vars: int, m: int, seed: int) -> dict:
  '''Inputs of the Andersen program (examples/andersen.py): AddressOf,
  Assign, Load and Store facts over `n_vars` variables, about m/4 each,
  drawn uniformly and deduplicated.'''
  rng = _rng(seed)
  q = max(1, m // 4)
  return {'AddressOf': _pairs(rng, n_vars, q), 'Assign': _pairs(rng, n_vars, q),
          'Load': _pairs(rng, n_vars, q), 'Store': _pairs(rng, n_vars, q)}


def cspa_inputs(n_vars: int, m: int, seed: int) -> dict:
  '''Inputs of the CSPA program (examples/cspa.py): AssignInput (3/4 of m)
  and DerefInput (1/4) over `n_vars` variables, uniform, deduplicated.'''
  rng = _rng(seed)
  return {'AssignInput': _pairs(rng, n_vars, max(1, 3 * m // 4)),
          'DerefInput': _pairs(rng, n_vars, max(1, m // 4))}


def lsqb_q7_inputs(n_msgs: int, seed: int, tags: int = 64, persons: int = 5000,
                   reply_frac: float = 0.5, like_frac: float = 0.5) -> dict:
  '''Inputs of LSQB Q7 (examples/lsqb_q7_optional.py) over n_msgs messages:
  every message gets 1-3 tags and 1 creator; a `reply_frac` share of the
  messages gets 1-4 replying comments (comment ids above the messages) and a
  `like_frac` share 1-6 likers; uniform draws, deduplicated.'''
  rng = _rng(seed)
  m = np.arange(n_msgs, dtype=np.uint32)

  def fan(msgs, lo, hi, vals):
    k = rng.integers(lo, hi + 1, msgs.shape[0])
    mm = np.repeat(msgs, k)
    return mm, rng.integers(0, vals, mm.shape[0], dtype=np.uint32)

  tm, tv = fan(m, 1, 3, tags)
  cm, cv = fan(m, 1, 1, persons)
  rmsg = m[rng.random(n_msgs) < reply_frac]
  rm, rc = fan(rmsg, 1, 4, 4 * n_msgs)
  lmsg = m[rng.random(n_msgs) < like_frac]
  lm, lp = fan(lmsg, 1, 6, persons)
  return {'HasTag': _dedup_in_order(tm, tv), 'HasCreator': _dedup_in_order(cm, cv),
          'ReplyOf': _dedup_in_order((rc + n_msgs).astype(np.uint32), rm),
          'Likes': _dedup_in_order(lp, lm)}


def lsqb_q6_inputs(n_persons: int, m_knows: int, seed: int, tags: int = 200) -> dict:
  '''Inputs of LSQB Q6 (examples/lsqb_q6_count.py): uniform Knows pairs
  (no self-loops, deduplicated) and 0-4 interests per person.'''
  rng = _rng(seed)
  knows = uniform_edges(n_persons, m_knows, seed)
  k = rng.integers(0, 5, n_persons)
  p = np.repeat(np.arange(n_persons, dtype=np.uint32), k)
  t = rng.integers(0, tags, p.shape[0], dtype=np.uint32)
  return {'KnowsInput': knows, 'HasInterestInput': _dedup_in_order(p, t)}


def lsqb_q3_inputs(n_persons: int, m_knows: int, seed: int, cities: int = 40,
                   countries: int = 4) -> dict:
  '''Inputs of LSQB Q3 (examples/lsqb_q3_triangle.py): uniform Knows pairs,
  every person in one city, every city in one country (ids of cities and
  countries start after the persons', as one id space).'''
  rng = _rng(seed)
  knows = uniform_edges(n_persons, m_knows, seed)
  person = np.arange(n_persons, dtype=np.uint32)
  city = (n_persons + rng.integers(0, cities, n_persons)).astype(np.uint32)
  cid = np.arange(n_persons, n_persons + cities, dtype=np.uint32)
  country = (n_persons + cities + rng.integers(0, countries, cities)).astype(np.uint32)
  return {'KnowsInput': knows, 'IsLocatedInInput': np.stack([person, city], 1),
          'IsPartOfInput': np.stack([cid, country], 1)}


def lsqb_q6_nosj_inputs(n_persons: int, m_knows: int, seed: int, tags: int = 200) -> dict:
  '''Inputs of the Q6 variant without self-join (examples/lsqb_q6_nosj.py):
  Q6's inputs plus a second, independent Knows.'''
  inp = lsqb_q6_inputs(n_persons, m_knows, seed, tags)
  inp['KnowsInput2'] = uniform_edges(n_persons, m_knows, seed + 1000)
  return inp


def galen_inputs(n_vals: int, m: int, seed: int) -> dict:
  '''Inputs of the Galen program (examples/galen.py) over values
  [0, n_vals): binary P and S, ternary Q, R, C and U, about m/6 rows each,
  uniform and deduplicated.'''
  rng = _rng(seed)
  q = max(1, m // 6)

  def triples() -> np.ndarray:
    t = rng.integers(0, n_vals, (q, 3), dtype=np.uint32)
    key = (t[:, 0].astype(np.uint64) * n_vals + t[:, 1]) * n_vals + t[:, 2]
    _, first = np.unique(key, return_index=True)
    first.sort()
    return np.ascontiguousarray(t[first])

  return {'PInput': _pairs(rng, n_vals, q), 'SInput': _pairs(rng, n_vals, q),
          'QInput': triples(), 'RInput': triples(), 'CInput': triples(), 'UInput': triples()}


def plan_inputs(plan: dict, n_vals: int, m: int, seed: int) -> dict:
  '''Uniform facts for every input relation of a plan (those with an input
  file): about m distinct rows each over values [0, n_vals), drawn in the
  plan's relation order from one seeded generator.'''
  rng = _rng(seed)
  out = {}
  for r in plan['relations']:
    if not r['input_file']:
      continue
    k = r['arity']
    t = rng.integers(0, n_vals, (m, k), dtype=np.uint32)
    key = np.zeros(m, np.uint64)
    for j in range(k):
      key = key * np.uint64(n_vals) + t[:, j].astype(np.uint64)
    _, first = np.unique(key, return_index=True)
    first.sort()
    out[r['name']] = np.ascontiguousarray(t[first])
  return out
