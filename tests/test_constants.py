'''Head constants (MIR constant-bind, mir/types.py:99-109) and body
constants: the plan lowering (a column join over a one-tuple relation the
plan carries as facts), the oracle interpreter on the lowered plans against
set restatements, and the plan checks.'''

import copy

import numpy as np
import oracle
import pytest
from conftest import load_plan
from srdatalog_b200 import workloads as W
from srdatalog_b200.batch import BatchError, check_batchable
from srdatalog_b200.plan import CONST_PREFIX, PlanError, _const_literal, validate_plan
from srdatalog_b200.shard import shard_plan


def _pipelines(plan):
  return {op['rule']: op['pipeline'] for st in plan['steps'] for op in st['ops']
          if op['op'] == 'execute_pipeline'}


def test_rewrite_consts_lowering():
  plan = load_plan('rewrite_consts')
  rels = {r['name']: r for r in plan['relations']}
  assert rels['__const_7']['facts'] == [[7]] and rels['__const_7']['arity'] == 1
  assert 'facts' not in rels['Q']
  head = _pipelines(plan)['HeadConst']
  assert [p['op'] for p in head] == ['scan', 'column_join', 'insert_into']
  assert head[1]['var'] == '_hc0'
  assert head[1]['sources'] == [{'rel': '__const_7', 'ver': 'FULL', 'index': [0], 'prefix': []}]
  body = _pipelines(plan)['BodyConst']
  assert body[1] == {'op': 'filter', 'vars': ['_c0', '_c1'], 'code': 'return _c0 == 42 && _c1 == 99;'}


def test_head_const_plan_shares_constant_relations():
  plan = load_plan('head_const')
  consts = sorted(r['name'] for r in plan['relations'] if r['name'].startswith(CONST_PREFIX))
  assert consts == ['__const_7', '__const_9']   # MarkSource and MarkStep share __const_7


@pytest.mark.parametrize('seed', range(4))
def test_rewrite_consts_interpreter_vs_sets(seed):
  rng = np.random.default_rng(seed)
  in3 = rng.integers(0, 4, (60, 3)).astype(np.uint32)
  in3[:, 1] = np.where(rng.random(60) < 0.5, 42, in3[:, 1])
  in3[:, 2] = np.where(rng.random(60) < 0.5, 99, in3[:, 2])
  in2 = rng.integers(0, 50, 20).astype(np.uint32).reshape(-1, 1)
  got, _ = oracle.run_plan(load_plan('rewrite_consts'), {'In': in3, 'In2': in2})
  want = oracle.rewrite_consts(in3, in2)
  assert got['P'] == want['P'] and got['Q'] == want['Q']
  assert want['P'] and want['Q']


@pytest.mark.parametrize('seed', range(5))
def test_head_const_interpreter_vs_sets(seed):
  e = W.uniform_edges(60, 70 + 10 * seed, seed)
  src = np.array([[seed], [seed + 11]], np.uint32)
  got, _ = oracle.run_plan(load_plan('head_const'), {'ArcInput': e, 'SourceInput': src})
  assert got['Mark'] == oracle.head_const(e, src)
  assert {t for _, t in got['Mark']} <= {7, 9}


def test_constant_literals():
  from types import SimpleNamespace as NS
  for code, v in [('7', 7), (' 42 ', 42), ('return 5;', 5), ('(3)', 3), ('4294967295u', 2**32 - 1)]:
    assert _const_literal(NS(var_name='v', code=code)) == v
  for code in ['x + 1', '-1', '4294967296', '"abc"', '1.5', '']:
    with pytest.raises(PlanError, match='not an unsigned'):
      _const_literal(NS(var_name='v', code=code))


def test_plan_checks_facts():
  plan = load_plan('head_const')
  bad = copy.deepcopy(plan)
  next(r for r in bad['relations'] if r['name'] == '__const_7')['facts'] = [[7, 1]]
  with pytest.raises(PlanError, match='facts of __const_7'):
    validate_plan(bad)
  bad = copy.deepcopy(plan)
  next(r for r in bad['relations'] if r['name'] == '__const_9')['facts'] = [[2**32]]
  with pytest.raises(PlanError, match='facts of __const_9'):
    validate_plan(bad)


def test_reserved_constant_relation_name():
  from srdatalog_b200 import plan as P
  steps = load_plan('rewrite_consts')['steps']
  with pytest.raises(PlanError, match='reserved'):
    P._const_relations(steps, {'__const_7'})
  assert [r['name'] for r in P._const_relations(steps, {'Q'})] == ['__const_7']


def test_batch_refuses_constants():
  with pytest.raises(BatchError, match='constant'):
    check_batchable(load_plan('head_const'))


def test_shard_plan_accepts_constants():
  spec = shard_plan(load_plan('head_const'))
  assert '__const_7' in spec.replicated


@pytest.mark.parametrize('name', ['live', 'live_lsm'])
@pytest.mark.parametrize('seed', range(3))
def test_live_interpreter_vs_sets(name, seed):
  '''The live program (a relation stored in order (1, 0) by its recursive
  stratum, read in order (0, 1) by a later one after a RebuildIndex(FULL)):
  the plan interpreter agrees with the rules restated on sets.'''
  plan = load_plan(name)
  steps = [o for s in plan['steps'] for o in s['ops']]
  assert {'op': 'rebuild_index', 'rel': 'Live', 'ver': 'FULL', 'index': [0, 1]}.items() <= \
      next(o for o in steps if o['op'] == 'rebuild_index' and o['ver'] == 'FULL').items()
  inp = W.plan_inputs(plan, 30, 60, seed)
  got, _ = oracle.run_plan(plan, inp)
  want = oracle.live(inp)
  assert got['Live'] == want['Live'] and got['Out'] == want['Out']
  assert len(want['Out']) > 0
