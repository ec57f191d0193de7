'''The device loop: the iterations of a recursive step after the first run
as one CUDA graph that loops on the device (convergence decided there), and
give the host path's results -- bit-exact against the oracle and the golden
fixtures -- including when too-small capacities send iterations back to the
host path (overflow), under max_iters, and on repeated runs.'''

import numpy as np
import oracle
import pytest
from conftest import load_plan
from srdatalog_b200 import native
from srdatalog_b200 import workloads as W

pytestmark = pytest.mark.gpu


def run(plan, inputs, loop=True, cap=0, max_iters=0, repeat=1):
  db = native.Database(load_plan(plan))
  db.set_option('device_loop', 1 if loop else 0)
  if cap:
    db.set_option('device_loop_cap_limit', cap)
  for rel, rows in inputs.items():
    db.load_rows(rel, rows)
  for _ in range(repeat):
    db.run(max_iters)
  return db


def loop_stats(db):
  return db.stats()['device_loop']


def rec_iterations(db):
  return [s['iterations'] for s in db.stats()['steps'] if s['recursive']]


def same(a, b, rel):
  assert a.size(rel) == b.size(rel), rel
  assert a.hash(rel) == b.hash(rel), rel


def test_tc_small_config_runs_on_the_device(expected):
  '''TC on 20,000 edges: iterations 1.. run in one graph launch (the second
  run sizes its buffers from the first and never overflows); size, hash and
  iteration count equal the golden ones.'''
  db = run('tc', {'ArcInput': W.tc_small(1)}, repeat=2)
  st = loop_stats(db)
  assert st['entries'] == 1 and st['overflows'] == 0, st
  assert st['iterations'] == expected['tc_small']['iterations'] - 1, st
  assert db.size('Path') == expected['tc_small']['size']
  assert oracle.dump_hash(db.dump('Path')) == expected['tc_small']['sha256']
  assert rec_iterations(db)[0] == expected['tc_small']['iterations']


@pytest.mark.parametrize('name', ['sg_2k', 'sg_10k'])
def test_sg_runs_on_the_device(expected, name):
  n, seed = (2000, 4) if name == 'sg_2k' else (10000, 2)
  db = run('sg', {'Arc': W.sg_forest(n, seed=seed)}, repeat=2)
  st = loop_stats(db)
  assert st['entries'] >= 1 and st['iterations'] > 0, st
  assert db.size('Sg') == expected[name]['size']
  assert db.hash('Sg') == expected[name]['sha256']
  assert rec_iterations(db)[-1] == expected[name]['iterations']


@pytest.mark.parametrize('plan', ['tc', 'tc_lsm', 'tc_left', 'tc_2level_bg'])
@pytest.mark.parametrize('n,m,seed', [(40, 90, 0), (300, 900, 1), (3000, 7000, 2)])
def test_tc_variants_equal_host_path_and_oracle(plan, n, m, seed):
  e = W.uniform_edges(n, m, seed)
  dev = run(plan, {'ArcInput': e})
  host = run(plan, {'ArcInput': e}, loop=False)
  assert loop_stats(host)['entries'] == 0
  same(dev, host, 'Path')
  assert rec_iterations(dev) == rec_iterations(host)
  keys, _, _ = oracle.tc(e)
  assert dev.size('Path') == keys.shape[0]


@pytest.mark.parametrize('cap', [1024, 4096, 20_000])
def test_overflow_hands_iterations_back_to_the_host(cap, expected):
  '''Capacities far below the counts: kernels raise the overflow flag
  instead of writing past a buffer, the loop stops, the failed iteration is
  redone on the host path from the intact buffer set, and the loop is
  entered again; the result is still the golden one.'''
  db = run('tc', {'ArcInput': W.tc_small(1)}, cap=cap)
  st = loop_stats(db)
  assert st['overflows'] >= 1, st
  assert db.size('Path') == expected['tc_small']['size']
  assert oracle.dump_hash(db.dump('Path')) == expected['tc_small']['sha256']
  assert rec_iterations(db)[0] == expected['tc_small']['iterations']


@pytest.mark.parametrize('max_iters', [1, 2, 3, 5, 9])
def test_max_iters_on_the_device_loop(max_iters):
  e = W.uniform_edges(2000, 6000, 7)
  dev = run('tc', {'ArcInput': e}, max_iters=max_iters)
  host = run('tc', {'ArcInput': e}, loop=False, max_iters=max_iters)
  same(dev, host, 'Path')
  assert rec_iterations(dev) == rec_iterations(host) == [max_iters]


@pytest.mark.parametrize('n,m,seed', [(400, 1500, 1), (20_000, 24_000, 2)])
def test_reach_avoid_negation_on_the_device(n, m, seed):
  e = W.uniform_edges(n, m, seed)
  blocked = np.concatenate([e[::3], W.uniform_edges(n, m // 4, seed + 10)])
  db = run('reach_avoid', {'Edge': e, 'Blocked': blocked})
  want = oracle.reach_avoid(e, blocked)
  for rel in ('Reach', 'Cut'):
    w = np.array(want[rel], np.uint32).reshape(-1, 2)
    assert db.size(rel) == w.shape[0], rel
    assert oracle.dump_hash(db.dump(rel)) == oracle.dump_hash(w), rel


@pytest.mark.parametrize('name', ['live', 'live_lsm'])
def test_live_on_the_device(name):
  plan = load_plan(name)
  inp = W.plan_inputs(plan, 3000, 9000, 3)
  want = oracle.live(inp)
  db = run(name, inp)
  assert loop_stats(db)['entries'] >= 1
  for rel in ('Live', 'Out'):
    w = np.array(want[rel], np.uint32).reshape(-1, 2)
    assert db.size(rel) == w.shape[0], rel
    assert oracle.dump_hash(db.dump(rel)) == oracle.dump_hash(w), rel


def test_head_constants_on_the_device():
  e = W.uniform_edges(3000, 7000, 3)
  src = np.array([[3], [14]], np.uint32)
  want = np.array(oracle.head_const(e, src), np.uint32).reshape(-1, 2)
  db = run('head_const', {'ArcInput': e, 'SourceInput': src})
  assert db.size('Mark') == want.shape[0]
  assert oracle.dump_hash(db.dump('Mark')) == oracle.dump_hash(want)


def test_polonius_steps_on_the_device():
  '''The linear recursive strata of Polonius run on the device loop; every
  relation equals the plan interpreter's.'''
  plan = load_plan('polonius')
  inp = W.plan_inputs(plan, 32, 30, 3)
  want, _ = oracle.run_plan(plan, inp)
  db = run('polonius', inp)
  arity = {r['name']: r['arity'] for r in plan['relations']}
  for rel, rows in want.items():
    w = np.array(rows, np.uint32).reshape(-1, arity[rel])
    assert db.size(rel) == w.shape[0], rel
    assert oracle.dump_hash(db.dump(rel)) == oracle.dump_hash(w), rel
