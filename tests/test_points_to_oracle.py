'''Beyond TC/SG/triangle: the points-to programs (examples/andersen.py,
examples/cspa.py) and LSQB Q7 with negation (examples/lsqb_q7_optional.py): the plan
interpreter (oracle.run_plan, which walks the MIR op sequence) agrees with
independent naive restatements of the programs' rules, so either can check
the GPU path.'''

import numpy as np
import oracle
import pytest
from conftest import load_plan
from srdatalog_b200 import workloads as W


@pytest.mark.parametrize('seed', [0, 1])
def test_andersen_interpreter_vs_rules(seed):
  inp = W.andersen_inputs(50, 140, seed)
  got, _ = oracle.run_plan(load_plan('andersen'), inp)
  assert sorted(got['PointsTo']) == oracle.andersen(inp)


@pytest.mark.parametrize('seed', [0, 1])
def test_cspa_interpreter_vs_rules(seed):
  inp = W.cspa_inputs(40, 90, seed)
  got, _ = oracle.run_plan(load_plan('cspa'), inp)
  want = oracle.cspa(inp)
  for rel in ('ValueFlow', 'ValueAlias', 'MemoryAlias'):
    assert sorted(got[rel]) == want[rel]


def test_points_to_plans_shape():
  an = load_plan('andersen')
  ops = [o['op'] for s in an['steps'] for o in s['ops']]
  assert ops.count('inject_cpp_hook') == 2            # Store_D0 / Store_D2 hooks, skipped
  rec = [s for s in an['steps'] if s['recursive']][0]
  assert sum(o['op'] == 'execute_pipeline' for o in rec['ops']) == 5   # the parallel group
  cs = load_plan('cspa')
  assert {r['name'] for r in cs['relations']} >= {'ValueFlow', 'ValueAlias', 'MemoryAlias'}


@pytest.mark.parametrize('seed', [0, 1])
def test_lsqb_q7_interpreter_vs_closed_form(seed):
  '''Negation: the plan interpreter's counts of LSQB Q7 equal the closed form.'''
  inp = W.lsqb_q7_inputs(60, seed, tags=8, persons=30)
  _, counts = oracle.run_plan(load_plan('lsqb_q7'), inp)
  assert counts == oracle.lsqb_q7(inp)


@pytest.mark.parametrize('seed', [0, 1])
def test_lsqb_q6_interpreter_vs_closed_form(seed):
  inp = W.lsqb_q6_inputs(40, 90, seed, tags=6)
  _, counts = oracle.run_plan(load_plan('lsqb_q6'), inp)
  assert counts['TwoHopPath'] == oracle.lsqb_q6(inp)


@pytest.mark.parametrize('seed', [0, 1, 2])
def test_lsqb_q3_interpreter_vs_sets(seed):
  '''LSQB Q3: the materialised arity-3 Triangle of the plan interpreter equals
  the set restatement.'''
  inp = W.lsqb_q3_inputs(50, 400, seed, cities=8, countries=2)
  got, _ = oracle.run_plan(load_plan('lsqb_q3'), inp)
  assert sorted(got['Triangle']) == oracle.lsqb_q3(inp)


@pytest.mark.parametrize('seed', [0, 1])
def test_lsqb_two_hop_variants_interpreter_vs_sets(seed):
  '''LSQB Q6 two-hop and no-self-join (materialised arity-4 Path) and Q9
  (count with a negated binary relation): interpreter == set restatement of
  the plans the reference's planner emits.'''
  inp = W.lsqb_q6_inputs(40, 150, seed, tags=6)
  got, _ = oracle.run_plan(load_plan('lsqb_q6_2hop'), inp)
  assert set(got['Path']) == oracle.lsqb_two_hop(inp)
  nosj = W.lsqb_q6_nosj_inputs(40, 150, seed, tags=6)
  got, _ = oracle.run_plan(load_plan('lsqb_q6_nosj'), nosj)
  assert set(got['Path']) == oracle.lsqb_two_hop(nosj, 'KnowsInput2')
  _, counts = oracle.run_plan(load_plan('lsqb_q9'), inp)
  assert counts['NegPath'] == len(oracle.lsqb_two_hop(inp, negate=True))


@pytest.mark.parametrize('seed', [0, 1])
def test_more_reference_programs_interpreter_vs_sets(seed):
  '''debug_triangle / gen_jit_code (arity-3 Z), tc_2level_bg, lsqb_q6_bg_test
  and print_mir (the Andersen rules with other plans): the plan interpreter
  equals the set restatements.'''
  r, s, t = (W.uniform_edges(30, 200, seed + k) for k in (1, 2, 3))
  got, _ = oracle.run_plan(load_plan('debug_triangle'), {'RRel': r, 'SRel': s, 'TRel': t})
  assert sorted(got['ZRel']) == oracle.triangle3(r, s, t)
  e = W.uniform_edges(30, 250, seed + 4)
  got, _ = oracle.run_plan(load_plan('gen_jit_triangle'), {'Edge': e})
  assert sorted(got['Z']) == oracle.triangle3(e, e, e)
  e = W.uniform_edges(50, 120, seed + 6)
  got, _ = oracle.run_plan(load_plan('tc_2level_bg'), {'ArcInput': e})
  keys, _, _ = oracle.tc(e)
  assert len(got['Path']) == keys.shape[0]
  inp = W.lsqb_q6_nosj_inputs(40, 150, seed + 5, tags=6)
  got, _ = oracle.run_plan(load_plan('lsqb_q6_bg'), inp)
  assert set(got['PathBG']) == oracle.lsqb_two_hop(inp, 'KnowsInput2', as_planned=False)
  inp = W.andersen_inputs(40, 120, seed + 7)
  got, _ = oracle.run_plan(load_plan('print_mir'), inp)
  assert sorted(got['PointsTo']) == sorted(oracle.andersen(inp))


@pytest.mark.parametrize('seed', [0, 1, 2])
def test_reach_avoid_interpreter_vs_sets(seed):
  '''Negation on two bound variables (inside a recursive join and in a later
  stratum): interpreter == set restatement.'''
  e = W.uniform_edges(30, 70, seed)
  blocked = np.ascontiguousarray(e[::3])
  extra = W.uniform_edges(30, 20, seed + 10)
  blocked = np.concatenate([blocked, extra])
  got, _ = oracle.run_plan(load_plan('reach_avoid'), {'Edge': e, 'Blocked': blocked})
  want = oracle.reach_avoid(e, blocked)
  assert sorted(got['Reach']) == want['Reach']
  assert sorted(got['Cut']) == want['Cut']


def test_set_option_rejects_unknown_names():
  from srdatalog_b200 import native
  db = native.Database(load_plan('tc'))
  with pytest.raises(Exception):
    db.set_option('no_such_option', 1)
  with pytest.raises(Exception):
    db.set_option('bitmap_mb', -1)
  db.set_option('bitmap_mb', 0)
  db.set_option('radix_bits', 7)
  db.set_option('join_blocks_per_sm', 32)
  for name, bad in (('radix_bits', 0), ('radix_bits', 9), ('join_blocks_per_sm', 0),
                    ('join_blocks_per_sm', 65)):
    with pytest.raises(Exception):
      db.set_option(name, bad)
  db.close()
