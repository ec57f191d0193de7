'''Sharded evaluation: a program split over `world` shards (run here by
threads of one process on one GPU; shards meet only at host-side barriers
of the exchange callback, no kernel waits on another shard's) gives, once
combined, exactly the unsharded result: partitioned relations are disjoint
and their union is the relation, counts add up, replicated relations are
equal on every shard.'''

import numpy as np
import oracle
import pytest
from conftest import load_plan
from srdatalog_b200 import workloads as W
from srdatalog_b200.shard import combine_dumps, combine_sizes, owner, run_local_shards, shard_plan

pytestmark = pytest.mark.gpu


def run_shards(plan_name, inputs, world, rels=(), rules=()):
  spec = shard_plan(load_plan(plan_name))
  sizes, counts, dumps = [], [], {r: [] for r in rels}
  shards = run_local_shards(spec, world, inputs)
  for rank, sd in enumerate(shards):
    with sd:
      sizes.append({r: sd.local_size(r) for r in rels})
      counts.append({r: sd.local_count(r) for r in rules})
      for r in rels:
        d = sd.local_dump(r)
        if r in spec.partitioned and d.shape[0]:
          # a shard holds only keys it owns
          assert np.all(owner(d[:, 0], world) == rank), r
        dumps[r].append(d)
  total = combine_sizes(spec, sizes)
  cnt = {r: sum(c[r] for c in counts) for r in rules}
  return spec, total, cnt, {r: combine_dumps(spec, r, dumps[r]) for r in rels}


@pytest.mark.parametrize('world', [2, 3, 8])
@pytest.mark.parametrize('plan_name', ['tc', 'tc_lsm'])
def test_tc_sharded_by_source(plan_name, world):
  e = W.uniform_edges(2000, 6000, 7)
  spec, sizes, _, dumps = run_shards(plan_name, {'ArcInput': e}, world, rels=('Path',))
  assert spec.partitioned == ['Path'] and spec.modes['TCBase'] == 'key'
  keys, _, _ = oracle.tc(e)
  want = oracle.unpack(keys, order=(1, 0))
  assert sizes['Path'] == want.shape[0]
  assert oracle.dump_hash(dumps['Path']) == oracle.dump_hash(want)


@pytest.mark.parametrize('world', [2, 5])
def test_triangle_sharded_by_work(world, expected):
  e = W.rmat_edges(14, 1 << 18, seed=5)
  spec, sizes, cnt, _ = run_shards('triangle', {'KnowsInput': e}, world, rels=('Knows',),
                                   rules=('TriangleJoin',))
  assert spec.modes['TriangleJoin'] == 'work' and spec.partitioned == []
  assert cnt['TriangleJoin'] == expected['triangle_rmat14']['count']
  assert sizes['Knows'] == e.shape[0]  # replicated: every shard loads all edges


def test_triangle_shards_small_and_empty():
  import math
  e = np.array([(i, j) for i in range(9) for j in range(i + 1, 9)], np.uint32)
  for world in (2, 7, 200):  # more shards than work items: empty windows
    _, _, cnt, _ = run_shards('triangle', {'KnowsInput': e}, world, rules=('TriangleJoin',))
    assert cnt['TriangleJoin'] == math.comb(9, 3)
  _, _, cnt, _ = run_shards('triangle', {'KnowsInput': np.zeros((0, 2), np.uint32)}, 3,
                            rules=('TriangleJoin',))
  assert cnt['TriangleJoin'] == 0


def test_triangle_rmat20_sharded(expected):
  e = W.rmat_edges(20, 1 << 24, seed=3)
  _, sizes, cnt, _ = run_shards('triangle', {'KnowsInput': e}, 4, rels=('Knows',),
                                rules=('TriangleJoin',))
  assert cnt['TriangleJoin'] == expected['triangle_rmat20']['count']
  assert sizes['Knows'] == expected['triangle_rmat20']['edges']


@pytest.mark.parametrize('world', [2, 4])
def test_reach_avoid_sharded(world):
  '''Partitioned relations under negation: the later stratum's rule reads
  the partitioned Reach only negated, so it is cut to its own keys.'''
  n, m, seed = 400, 1500, 1
  e = W.uniform_edges(n, m, seed)
  blocked = np.concatenate([e[::3], W.uniform_edges(n, m // 4, seed + 10)])
  spec, sizes, _, dumps = run_shards('reach_avoid', {'Edge': e, 'Blocked': blocked}, world,
                                     rels=('Reach', 'Cut'))
  assert spec.modes['CutPairs'] == 'key'
  want = oracle.reach_avoid(e, blocked)
  for rel in ('Reach', 'Cut'):
    w = np.array(want[rel], np.uint32).reshape(-1, 2)
    assert sizes[rel] == w.shape[0], rel
    assert oracle.dump_hash(dumps[rel]) == oracle.dump_hash(w), rel


def test_lsqb_counts_sharded():
  inp6 = W.lsqb_q6_inputs(20_000, 200_000, 1)
  _, _, cnt, _ = run_shards('lsqb_q6', inp6, 3, rules=('TwoHopPath',))
  assert cnt['TwoHopPath'] == oracle.lsqb_q6(inp6)
  inp7 = W.lsqb_q7_inputs(5000, 1)
  want = oracle.lsqb_q7(inp7)
  _, _, cnt, _ = run_shards('lsqb_q7', inp7, 3, rules=tuple(want))
  assert cnt == want


@pytest.mark.parametrize('world', [2, 3, 5])
def test_sg_sharded_with_exchange(expected, world):
  '''Same generation moves the key in its recursive rule: each iteration's
  derived tuples go to the shards owning them, and the fixpoint stops when
  every shard's delta is empty.'''
  exp = expected['sg_2k']
  spec, sizes, _, dumps = run_shards('sg', {'Arc': W.sg_forest(2000, seed=4)}, world, rels=('Sg',))
  assert spec.partitioned == ['Sg'] and spec.exchanged == ['Sg']
  assert sizes['Sg'] == exp['size']
  assert oracle.dump_hash(dumps['Sg']) == exp['sha256']


@pytest.mark.parametrize('world', [2, 4])
def test_left_recursive_tc_sharded_with_exchange(expected, world):
  exp = expected['tc_mid']
  e = W.uniform_edges(2000, 6000, 7)
  spec, sizes, _, dumps = run_shards('tc_left', {'ArcInput': e}, world, rels=('Path',))
  assert spec.exchanged == ['Path']
  assert sizes['Path'] == exp['size']
  assert oracle.dump_hash(dumps['Path']) == exp['sha256']


def test_sg_shards_small_and_empty():
  '''Shards that own no tuple still take part in every exchange and vote.'''
  e = np.array([[0, 1], [0, 2], [1, 3], [2, 4]], np.uint32)
  want, _ = oracle.run_plan(load_plan('sg'), {'Arc': e})
  _, sizes, _, dumps = run_shards('sg', {'Arc': e}, 7, rels=('Sg',))
  assert sizes['Sg'] == len(want['Sg'])
  assert {tuple(map(int, r)) for r in dumps['Sg']} == set(want['Sg'])
  _, sizes, _, _ = run_shards('sg', {'Arc': np.zeros((0, 2), np.uint32)}, 3, rels=('Sg',))
  assert sizes['Sg'] == 0
