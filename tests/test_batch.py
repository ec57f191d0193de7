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
