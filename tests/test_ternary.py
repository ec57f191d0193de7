'''Joins over ternary relations (the Galen program, examples/galen.py, MIR
pinned by tests/fixtures/integration/galen.mir.sexpr): the oracle
interpreter, which binds several columns of one cartesian source, against
a set-based restatement of the rules, and the access patterns the plan asks
the runtime for.'''

import oracle
import pytest
from conftest import load_plan
from srdatalog_b200 import workloads as W

CASES = [(12, 40, 0), (20, 120, 1), (30, 150, 2)]


@pytest.mark.parametrize('n,m,seed', CASES)
def test_galen_interpreter_vs_rules(n, m, seed):
  inp = W.galen_inputs(n, m, seed)
  got, _ = oracle.run_plan(load_plan('galen'), inp)
  want = oracle.galen(inp)
  assert got['OutP'] == want['OutP'] and got['OutQ'] == want['OutQ']


def test_galen_access_patterns():
  '''Ternary sources appear with 0, 1 and 2 bound columns, in three column
  orders, and cartesian sources bind two columns of OutQ under one.'''
  plan = load_plan('galen')
  arity = {r['name']: r['arity'] for r in plan['relations']}
  bound, orders, two_var = set(), set(), 0
  for st in plan['steps']:
    for op in st['ops']:
      for p in op.get('pipeline', ()):
        for i, s in enumerate(p.get('sources', ())):
          if arity[s['rel']] == 3:
            bound.add(len(s['prefix']))
            orders.add(tuple(s['index']))
            if p['op'] == 'cartesian_join' and len(p['var_from_source'][i]) == 2:
              two_var += 1
        if p['op'] == 'scan' and arity[p['rel']] == 3:
          bound.add('scan')
  assert bound == {0, 1, 2, 'scan'}
  assert orders == {(0, 1, 2), (1, 0, 2), (2, 1, 0)}
  assert two_var >= 2


def test_polonius_interpreter_derives():
  '''The Polonius plan (MIR pinned to the reference fixture) derives the
  relations its rules define from uniform facts; the GPU parity test checks
  the engine against these interpreter results.'''
  plan = load_plan('polonius')
  got, _ = oracle.run_plan(plan, W.plan_inputs(plan, 24, 20, 2))
  for rel in ('subset', 'origin_live_on_entry', 'loan_live_at', 'errors', 'move_error'):
    assert got[rel], rel


def test_ternary_programs_shard_as_replicas():
  '''Exchanges move binary tuples only: programs whose joins need other
  shards' ternary tuples fall back to replicas, with the reason.'''
  from srdatalog_b200.shard import shard_plan
  for name in ('galen', 'polonius'):
    spec = shard_plan(load_plan(name))
    assert spec.fallback and not spec.partitioned and not spec.exchanged


@pytest.mark.parametrize('n,m,seed', [(10, 8, 0), (24, 20, 2)])
def test_polonius_liveness_rules_restated(n, m, seed):
  '''Two Polonius relations of the interpreter against the rules restated on
  sets: var_live_on_entry (vle_used, vle_cfg with its negation) and
  origin_live_on_entry (ole_universal, ole_drop, ole_use).'''
  plan = load_plan('polonius')
  inp = W.plan_inputs(plan, n, m, seed)
  got, _ = oracle.run_plan(plan, inp)
  facts = {k: set(map(tuple, v.tolist())) for k, v in inp.items()}
  vle = set(facts['var_used_at'])
  while True:
    new = {(v, p1) for (v, p2) in vle for (p1, q) in facts['cfg_edge']
           if q == p2 and (v, p1) not in facts['var_defined_at']} - vle
    if not new:
      break
    vle |= new
  assert vle == set(got['var_live_on_entry'])
  live = {(o, p) for (p,) in got['cfg_node'] for (o,) in facts['universal_region']}
  live |= {(o, p) for (v, p) in got['var_drop_live_on_entry']
           for (w, o) in facts['drop_of_var_derefs_origin'] if v == w}
  live |= {(o, p) for (v, p) in vle for (w, o) in facts['use_of_var_derefs_origin'] if v == w}
  assert live == set(got['origin_live_on_entry'])
