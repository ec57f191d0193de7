'''Batched fixpoints on the GPU: per-instance results of disjoint-union runs
(sizes, row fingerprints, and each instance's own iteration count recorded
on the device) equal one-instance-at-a-time runs and the oracle -- on the
host path and on the device loop -- and the batched config's own instances
run in waves under a device-memory budget: every instance with n <= 8,192
(2,899 instances, about 1.9e10 Path tuples) and a seeded sample of larger
ones, each checked against the SCC restatement of its closure.'''

import math

import numpy as np
import oracle
import pytest
from conftest import load_plan
from srdatalog_b200 import native
from srdatalog_b200 import workloads as W
from srdatalog_b200.batch import BatchRun, WaveRun

pytestmark = pytest.mark.gpu

TC_STEP = 4  # the recursive step of the TC plan


def small_instances(count, seed, n_lo=16, n_hi=600):
  rng = np.random.default_rng(seed)
  out = []
  for j in range(count):
    n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
    out.append({'ArcInput': W.er_instance(n, float(rng.uniform(0.6, 4.0)), seed * 1000 + j)})
  # a long chain (many iterations), a single edge, a 2-cycle
  out.append({'ArcInput': np.array([[i, i + 1] for i in range(60)], np.uint32)})
  out.append({'ArcInput': np.array([[0, 1]], np.uint32)})
  out.append({'ArcInput': np.array([[0, 1], [1, 0]], np.uint32)})
  return out


def alone(plan, inst, max_iters=0, loop=None):
  db = native.Database(plan)
  if loop is not None:
    db.set_option('device_loop', loop)
  for rel, rows in inst.items():
    db.load_rows(rel, rows)
  db.run(max_iters)
  it = [s['iterations'] for s in db.stats()['steps'] if s['recursive']]
  return db, it


@pytest.mark.parametrize('loop', [0, 1])
@pytest.mark.parametrize('plan_name', ['tc', 'tc_lsm'])
def test_tc_instances_equal_single_runs(plan_name, loop):
  '''Per instance: size, fingerprint and rows equal its own run; its
  recorded iterations equal its own run's; on the device loop the union's
  iterations run in one graph.'''
  plan = load_plan(plan_name)
  insts = small_instances(45, 1)
  db = native.Database(plan)
  db.set_option('device_loop', loop)
  br = BatchRun(plan, insts, db=db)
  if loop:
    assert db.stats()['device_loop']['entries'] >= 1
  sizes, sums, its = br.sizes('Path'), br.checksums('Path'), br.iterations()[TC_STEP]
  rows = br.split_rows('Path')
  for j, inst in enumerate(insts):
    one, it = alone(plan, inst, loop=0)
    got = one.dump('Path')
    assert sizes[j] == got.shape[0], j
    assert int(sums[j]) == oracle.row_fingerprint(got), j
    assert oracle.dump_hash(rows[j]) == oracle.dump_hash(got), j
    assert [int(its[j])] == it, j
    keys, iters, _ = oracle.tc(inst['ArcInput'])
    assert keys.shape[0] == got.shape[0] and iters == it[0], j


@pytest.mark.parametrize('max_iters', [1, 2, 5])
@pytest.mark.parametrize('loop', [0, 1])
def test_iterations_under_max_iters(max_iters, loop):
  plan = load_plan('tc')
  insts = small_instances(20, 2)
  db = native.Database(plan)
  db.set_option('device_loop', loop)
  br = BatchRun(plan, insts, db=db, max_iters=max_iters)
  its, sizes = br.iterations()[TC_STEP], br.sizes('Path')
  for j, inst in enumerate(insts):
    one, it = alone(plan, inst, max_iters=max_iters)
    assert [int(its[j])] == it and sizes[j] == one.size('Path'), j


def test_sg_instances_equal_oracle():
  plan = load_plan('sg')
  insts = [{'Arc': W.sg_forest(n, window=min(50, n - 1), seed=s)}
           for s, n in enumerate([30, 200, 800, 64, 1500, 17, 400])]
  br = BatchRun(plan, insts)
  sizes, sums = br.sizes('Sg'), br.checksums('Sg')
  step = [i for i, st in enumerate(plan['steps']) if st.get('recursive')][0]
  its = br.iterations()[step]
  for j, inst in enumerate(insts):
    keys, iters, _ = oracle.sg(inst['Arc'])
    rows = oracle.unpack(keys, (0, 1))
    assert sizes[j] == rows.shape[0] and int(sums[j]) == oracle.row_fingerprint(rows), j
    assert its[j] == alone(plan, inst)[1][0], j


def test_range_checksums_of_empty_ranges_and_unbatched_runs():
  db = native.Database(load_plan('tc'))
  e = W.uniform_edges(500, 1500, 4)
  db.load_rows('ArcInput', e)
  db.run()
  rows = db.dump('Path')
  b = np.array([0, 0, 500, 500, 501], np.uint32)
  sums = db.range_checksums('Path', b)
  assert sums.tolist() == [0, oracle.row_fingerprint(rows), 0, 0]
  with pytest.raises(native.SrdlError):
    db.instance_iterations(4)  # no instances set


def config_waves(insts, budget=120e9):
  plan = load_plan('tc')
  wr = WaveRun(plan, insts, budget_bytes=int(budget), sizes=['Path'], checksums=['Path'])
  wr.run()
  assert not wr.errors, wr.errors
  return plan, wr


def test_config_instances_up_to_8192_nodes():
  '''Every instance of the batched config's own draws with n <= 8,192
  (2,899 of 4,096) in budgeted waves: size and fingerprint against the SCC
  oracle for every instance, iterations against its own run for every
  16th.'''
  shapes = [s for s in W.batched_shapes() if s[0] <= 8192]
  insts = [{'ArcInput': e} for e in W.batched_instances(n_max=8192)]
  assert len(insts) == len(shapes) == 2899
  plan, wr = config_waves(insts)
  want = oracle.tc_closure_fingerprints([(i['ArcInput'], n) for i, (n, _) in zip(insts, shapes)])
  got = list(zip(wr.sizes['Path'].tolist(), wr.checksums['Path'].tolist()))
  bad = [j for j in range(len(insts)) if got[j] != want[j]]
  assert not bad, bad[:10]
  assert sum(s for s, _ in want) > 1.9e10
  for j in range(0, len(insts), 16):
    assert [int(wr.iterations[TC_STEP][j])] == alone(plan, insts[j])[1], j


def test_config_sample_of_larger_instances():
  '''A seeded sample of the config's instances with 8,192 < n <= 32,768
  (each up to ~10^9 Path tuples), in budgeted waves, against the SCC
  oracle and their own runs.'''
  shapes = W.batched_shapes()
  cand = [j for j, (n, _) in enumerate(shapes) if 8192 < n <= 32768]
  pick = sorted(np.random.default_rng(2024).choice(cand, 6, replace=False).tolist())
  insts = [{'ArcInput': e} for e in W.batched_instances(only=pick)]
  plan, wr = config_waves(insts)
  want = oracle.tc_closure_fingerprints([(i['ArcInput'], shapes[j][0]) for i, j in zip(insts, pick)])
  for k, j in enumerate(pick):
    assert (int(wr.sizes['Path'][k]), int(wr.checksums['Path'][k])) == want[k], j
    assert [int(wr.iterations[TC_STEP][k])] == alone(plan, insts[k])[1], j
