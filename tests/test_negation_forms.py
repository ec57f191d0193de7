'''Negation with constant arguments and over ternary relations: the plan
lowering (constants lead the probed prefix, in the index order the
reference's planner gives, src/srdatalog/hir/plan.py:284-286) and the plan
interpreter, against a direct restatement of each rule (no GPU).'''

import numpy as np
import oracle
import pytest
from conftest import load_plan


def negations(plan):
  out = {}
  for st in plan['steps']:
    for op in st['ops']:
      if op['op'] == 'execute_pipeline':
        for p in op['pipeline']:
          if p['op'] == 'negation':
            out[op['rule']] = (p['rel'], p['index'], p['prefix'], p.get('const_prefix', []))
  return out


def test_lowered_forms():
  neg = negations(load_plan('neg_forms'))
  assert neg['NegConst'] == ('Blocked', [1, 0], ['x'], [3])
  assert neg['NegTern2'] == ('Tern', [0, 2, 1], ['x', 'y'], [])
  assert neg['NegTernConst'] == ('Tern', [0, 1, 2], ['y'], [5])
  assert neg['NegTern1'] == ('Tern', [2, 0, 1], ['x'], [])


def inputs(n, m, seed):
  rng = np.random.default_rng(seed)
  e = np.unique(rng.integers(0, n, (m, 2)), axis=0).astype(np.uint32)
  b = rng.integers(0, n, (m // 2, 2)).astype(np.uint32)
  b[: m // 8, 1] = 3
  t = rng.integers(0, n, (m // 4, 3)).astype(np.uint32)
  t[: m // 16, 0] = 5
  return {'Edge': e, 'Blocked': b, 'Tern': t}


def expected(inp):
  e = [tuple(r) for r in inp['Edge'].tolist()]
  blocked = {tuple(r) for r in inp['Blocked'].tolist()}
  tern = [tuple(r) for r in inp['Tern'].tolist()]
  t02 = {(a, c) for a, _, c in tern}
  t01_5 = {b for a, b, _ in tern if a == 5}
  t2 = {c for _, _, c in tern}
  return {
    'OutConst': {(x, y) for x, y in e if (x, 3) not in blocked},
    'OutTern2': {(x, y) for x, y in e if (x, y) not in t02},
    'OutTernConst': {(x, y) for x, y in e if y not in t01_5},
    'OutTern1': {(x, y) for x, y in e if x not in t2},
  }


@pytest.mark.parametrize('n,m,seed', [(20, 60, 0), (60, 400, 1)])
def test_interpreter_matches_rules(n, m, seed):
  inp = inputs(n, m, seed)
  got, _ = oracle.run_plan(load_plan('neg_forms'), inp)
  want = expected(inp)
  for rel, rows in want.items():
    assert set(got[rel]) == rows and len(got[rel]) == len(rows), rel
    assert 0 < len(rows) < inp['Edge'].shape[0], rel  # every form filters something, not everything
