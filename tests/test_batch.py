'''Disjoint-union batching: host-side logic (no GPU).'''

import numpy as np
import pytest
from conftest import load_plan
from srdatalog_b200.batch import BatchError, check_batchable, make_union


def test_union_offsets_and_relabel():
  a = {'ArcInput': np.array([[0, 1], [1, 2]], np.uint32)}
  b = {'ArcInput': np.array([[0, 3]], np.uint32)}
  c = {'ArcInput': np.zeros((0, 2), np.uint32)}
  u = make_union([a, b, c])
  assert u.offsets.tolist() == [0, 3, 7, 8]
  assert u.inputs['ArcInput'].tolist() == [[0, 1], [1, 2], [3, 6]]


def test_plans_with_variable_filters_batch():
  for name in ('tc', 'sg', 'triangle', 'tc_left', 'tc_lsm'):
    check_batchable(load_plan(name))


def test_constant_filter_rejected():
  plan = load_plan('sg')
  for st in plan['steps']:
    for op in st['ops']:
      if op['op'] == 'execute_pipeline':
        for p in op['pipeline']:
          if p['op'] == 'filter':
            p['code'] = 'return x != 3;'
  with pytest.raises(BatchError):
    check_batchable(plan)


def test_union_overflow_rejected():
  big = {'ArcInput': np.array([[0, 0xFFFFFFF0]], np.uint32)}
  with pytest.raises(BatchError):
    make_union([big, big])


# ---------------------------------------------------------------- waves

from srdatalog_b200.batch import WaveRun, derived_arities, instance_bound, plan_waves  # noqa: E402
from srdatalog_b200.native import SrdlError  # noqa: E402


def test_bounds_and_wave_plan():
  assert derived_arities(load_plan('tc')) == [2, 2]  # Arc (copied from ArcInput) and Path
  inst = {'ArcInput': np.array([[0, 9], [3, 4]], np.uint32)}
  assert instance_bound(inst, [2]) == 100
  assert instance_bound({'ArcInput': np.zeros((0, 2), np.uint32)}, [2]) == 1
  assert plan_waves([5, 5, 5, 20, 1, 1], 10) == [[0, 1], [2], [3], [4, 5]]
  assert plan_waves([], 10) == []


class FakeDb:
  '''Stands in for a Database: a run "needs" 30 bytes per bound tuple of
  its instances and fails with status 5 above the memory limit.'''

  def __init__(self):
    self.limit = 0
    self.runs = []

  def set_option(self, name, value):
    if name == 'mem_limit_mb':
      self.limit = value << 20

  def clear_inputs(self):
    self.rows = None

  def load_rows(self, rel, rows):
    self.rows = np.asarray(rows)

  def set_count_groups(self, rule, bounds):
    pass

  def set_instances(self, bounds):
    self.bounds = np.asarray(bounds, np.int64)

  def run(self, max_iters=0):
    spans = np.diff(self.bounds)
    self.peak = int(30 * (spans ** 2).sum())
    self.runs.append(len(spans))
    if self.peak > self.limit:
      raise SrdlError('srdl_run', 5, 'device memory limit of the run exceeded')

  def mem_stats(self):
    return {'peak': self.peak}

  def range_counts(self, rel, bounds):
    b = np.asarray(bounds, np.int64)
    x = self.rows[:, 0].astype(np.int64)
    return np.array([((x >= b[j]) & (x < b[j + 1])).sum() for j in range(len(b) - 1)], np.uint64)

  def instance_iterations(self, step):
    return (np.diff(self.bounds) % 7 + 1).astype(np.uint32)


def test_wave_run_splits_outgrown_waves_and_keeps_the_partition():
  rng = np.random.default_rng(3)
  insts = []
  for j in range(40):
    n = int(rng.integers(4, 400))
    e = rng.integers(0, n, (2 * n, 2)).astype(np.uint32)
    e[0] = [n - 1, 0]  # span n
    insts.append({'ArcInput': e})
  db = FakeDb()
  budget = 6 << 20
  # bytes_per_bound far too low: every planned wave outgrows the budget
  wr = WaveRun(load_plan('tc'), insts, db=db, budget_bytes=budget, bytes_per_bound=1.0,
               sizes=['Path'])
  wr.run()
  assert not wr.errors and wr.splits > 0
  assert sorted(j for w in wr.waves for j in w) == list(range(40))
  # every instance's result sits at its own index
  want = [int((i['ArcInput'][:, 0] >= 0).sum()) for i in insts]
  assert wr.sizes['Path'].tolist() == want
  spans = np.array([int(i['ArcInput'].max()) + 1 for i in insts])
  assert wr.iterations[4].tolist() == (spans % 7 + 1).tolist()  # the recursive step
  assert wr.bytes_per_bound >= 15  # 30 B per span^2, bound = 2 span^2
  # a second run reuses the partition: no split, no failed run
  runs = len(db.runs)
  wr.run()
  splits = wr.splits
  wr.run()
  assert wr.splits == splits and len(db.runs) - runs == 2 * len(wr.waves)
  assert all(30 * float(wr.bounds[w].sum()) / 2 <= budget for w in wr.waves)


def test_wave_run_reports_an_instance_beyond_the_budget():
  small = {'ArcInput': np.array([[0, 1], [1, 2]], np.uint32)}
  huge = {'ArcInput': np.array([[0, 999]], np.uint32)}
  wr = WaveRun(load_plan('tc'), [small, huge, small], db=FakeDb(), budget_bytes=1 << 20,
               sizes=['Path'])
  wr.run()
  assert list(wr.errors) == [1] and 'limit' in wr.errors[1]
  assert wr.sizes['Path'].tolist() == [2, 0, 2]
