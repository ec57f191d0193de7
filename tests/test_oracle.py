'''Pins for the CPU oracle (no GPU).

The reference ships no tuple-level golden vectors, so the oracle is pinned
by (1) closed-form answers on hand-checkable graphs, (2) an independent
linear-algebra / graph-search restatement (scipy), (3) the generic
pure-Python plan interpreter walking the reference's MIR plans, and (4) the
committed expected values for the smaller golden workloads.
'''

import math

import numpy as np
import oracle
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import breadth_first_order
from srdatalog_b200 import workloads as W


def tc_rows(edges):
  keys, iters, _ = oracle.tc(np.asarray(edges, np.uint32).reshape(-1, 2))
  return {tuple(map(int, r)) for r in oracle.unpack(keys, order=(1, 0))}, iters


def scipy_tc(edges, n):
  e = np.asarray(edges, np.int64).reshape(-1, 2)
  A = sp.csr_matrix((np.ones(len(e)), (e[:, 0], e[:, 1])), shape=(n, n))
  out = set()
  for s in range(n):
    order = breadth_first_order(A, s, directed=True, return_predecessors=False)
    # nodes reachable by a path of length >= 1: successors' closure
    succ = A.indices[A.indptr[s]:A.indptr[s + 1]]
    reach = set()
    for t in succ:
      reach.update(breadth_first_order(A, int(t), directed=True, return_predecessors=False).tolist())
    del order
    out.update((s, t) for t in reach)
  return out


def test_tc_chain():
  n = 40
  rows, iters = tc_rows([(i, i + 1) for i in range(n - 1)])
  assert len(rows) == n * (n - 1) // 2
  assert iters == n - 1  # one join per path length, last one finds nothing new


def test_tc_cycle_and_complete():
  n = 25
  rows, _ = tc_rows([(i, (i + 1) % n) for i in range(n)])
  assert len(rows) == n * n
  m = 12
  rows, _ = tc_rows([(i, j) for i in range(m) for j in range(m) if i != j])
  assert len(rows) == m * m


def test_tc_star_and_empty():
  rows, _ = tc_rows([(0, i) for i in range(1, 30)])
  assert rows == {(0, i) for i in range(1, 30)}
  keys, iters, _ = oracle.tc(np.zeros((0, 2), np.uint32))
  assert keys.shape[0] == 0


@pytest.mark.parametrize('seed', [3, 4, 5])
def test_tc_matches_scipy(seed):
  e = W.uniform_edges(60, 150, seed)
  rows, _ = tc_rows(e)
  assert rows == scipy_tc(e, 60)


def sg_brute(edges):
  '''SG(x,y): x,y reachable from one node by paths of equal length >= 1,
  excluding x == y at length 1 (the base rule's filter).'''
  e = [tuple(map(int, r)) for r in edges]
  nodes = sorted({v for r in e for v in r})
  ch = {v: set() for v in nodes}
  for a, b in e:
    ch[a].add(b)
  out = set()
  for a in nodes:
    level = {a}
    depth = 0
    while level and depth < len(nodes) + 1:
      level = set().union(*[ch[v] for v in level]) if level else set()
      depth += 1
      for x in level:
        for y in level:
          if depth == 1 and x == y:
            continue
          out.add((x, y))
  # recursive SG rows can also come from different ancestors at equal depth
  # along SG itself; iterate to the least fixpoint of the two rules.
  changed = True
  sgs = {(x, y) for a in nodes for x in ch[a] for y in ch[a] if x != y}
  while changed:
    new = {(x, y) for (p, q) in sgs for x in ch.get(p, ()) for y in ch.get(q, ())}
    changed = not new <= sgs
    sgs |= new
  return sgs


def test_sg_matches_fixpoint_definition():
  e = W.sg_forest(300, window=20, seed=9)
  keys, _, _ = oracle.sg(e)
  got = {tuple(map(int, r)) for r in oracle.unpack(keys, order=(0, 1))}
  assert got == sg_brute(e)


def test_triangle_known_answers():
  for n in (3, 4, 7, 12):
    e = np.array([(i, j) for i in range(n) for j in range(i + 1, n)], np.uint32)
    assert oracle.triangle_count(e) == math.comb(n, 3)
  assert oracle.triangle_count(np.zeros((0, 2), np.uint32)) == 0


def test_triangle_matches_scipy():
  e = W.rmat_edges(10, 20000, seed=11)
  n = 1 << 10
  A = sp.csr_matrix((np.ones(len(e)), (e[:, 0].astype(np.int64), e[:, 1].astype(np.int64))),
                    shape=(n, n))
  want = int((A @ A).multiply(A).sum())
  assert oracle.triangle_count(e) == want


def test_primitives_match_numpy():
  rng = np.random.default_rng(0)
  a = rng.integers(0, 1 << 40, 5000, dtype=np.uint64)
  a = np.concatenate([a, a[:700]])
  su = oracle.sort_unique(a)
  assert np.array_equal(su, np.unique(a))
  b = np.unique(rng.integers(0, 1 << 40, 3000, dtype=np.uint64))
  b = np.union1d(b, su[::3])
  d = oracle.set_difference(su, b)
  assert np.array_equal(d, np.setdiff1d(su, b))
  m = oracle.merge(b, d)
  assert np.array_equal(m, np.union1d(b, d))


@pytest.mark.parametrize('name', ['tc', 'tc_left'])
def test_plan_interpreter_tc(plans, name):
  e = W.uniform_edges(25, 50, seed=2)
  out, _ = oracle.run_plan(plans[name], {'ArcInput': e})
  rows, _ = tc_rows(e)
  assert set(out['Path']) == rows


def test_plan_interpreter_sg_and_triangle(plans):
  e = W.sg_forest(120, window=10, seed=3)
  out, _ = oracle.run_plan(plans['sg'], {'Arc': e})
  keys, _, _ = oracle.sg(e)
  assert set(out['Sg']) == {tuple(map(int, r)) for r in oracle.unpack(keys)}
  t = W.rmat_edges(7, 600, seed=4)
  _, counts = oracle.run_plan(plans['triangle'], {'KnowsInput': t})
  assert counts['TriangleJoin'] == oracle.triangle_count(t)


def test_plan_interpreter_max_iters(plans):
  e = [(i, i + 1) for i in range(10)]
  out, _ = oracle.run_plan(plans['tc'], {'ArcInput': np.array(e, np.uint32)}, max_iters=2)
  # base (length 1) + two joins (lengths 2 and 3)
  assert len(out['Path']) == 10 + 9 + 8
  keys, iters, _ = oracle.tc(np.array(e, np.uint32), max_iters=2)
  assert keys.shape[0] == 27 and iters == 2


@pytest.mark.parametrize('name', ['tc_mid', 'sg_2k', 'triangle_rmat14'])
def test_golden_expected(expected, name):
  import gen_expected
  got = gen_expected.compute(name)
  assert got == expected[name]


def test_generators_deterministic():
  a = W.uniform_edges(100, 300, seed=1)
  b = W.uniform_edges(100, 300, seed=1)
  assert np.array_equal(a, b)
  assert len({tuple(r) for r in a}) == 300 and not np.any(a[:, 0] == a[:, 1])
  f = W.sg_forest(500, seed=2)
  assert np.all(f[:499, 0] < f[:499, 1])
  r = W.rmat_edges(8, 4000, seed=3)
  assert np.all(r[:, 0] < r[:, 1])
  insts = W.batched_instances(count=3)
  assert all(x.shape[1] == 2 for x in insts)


@pytest.mark.parametrize('n,m,seed', [(5, 8, 0), (40, 30, 1), (40, 90, 2), (300, 280, 3),
                                      (300, 900, 4), (2000, 1900, 5), (2000, 6000, 6)])
def test_closure_fingerprint_matches_semi_naive(n, m, seed):
  '''The SCC restatement of TC's fixpoint (used on instances too large for
  the semi-naive evaluator) gives the semi-naive oracle's size and row
  fingerprint, on graphs with self-loops, duplicate edges, cycles and
  isolated parts.'''
  e = np.random.default_rng(seed).integers(0, n, (m, 2)).astype(np.uint32)
  keys, _, _ = oracle.tc(np.unique(e, axis=0))
  rows = oracle.unpack(keys, (1, 0))
  assert oracle.tc_closure_fingerprint(e, n) == (rows.shape[0], oracle.row_fingerprint(rows))


def test_closure_fingerprint_shapes():
  chain = np.array([[i, i + 1] for i in range(50)], np.uint32)
  assert oracle.tc_closure_fingerprint(chain)[0] == 50 * 51 // 2
  loops = np.array([[0, 0], [1, 2], [2, 1], [3, 3], [3, 4]], np.uint32)
  rows = np.array([[0, 0], [1, 1], [1, 2], [2, 1], [2, 2], [3, 3], [3, 4]], np.uint32)
  assert oracle.tc_closure_fingerprint(loops) == (7, oracle.row_fingerprint(rows))
  assert oracle.tc_closure_fingerprint(np.zeros((0, 2), np.uint32)) == (0, 0)
  # the fingerprint is order-free and sensitive to one row
  assert oracle.row_fingerprint(rows[::-1]) == oracle.row_fingerprint(rows)
  assert oracle.row_fingerprint(rows[1:]) != oracle.row_fingerprint(rows)


def test_closure_fingerprints_pool():
  jobs = [(np.random.default_rng(s).integers(0, 200, (400, 2)).astype(np.uint32), 200)
          for s in range(12)]
  assert oracle.tc_closure_fingerprints(jobs, workers=2) == [oracle.tc_closure_fingerprint(*j)
                                                              for j in jobs]
