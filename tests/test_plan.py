'''Plan format: committed plans are valid and, when the srdatalog front end
is importable, identical to what the reference's HIR/MIR lowering produces
for the benchmark programs (whose MIR is pinned by the reference fixtures).'''

import os
import subprocess
import sys

import pytest
from conftest import GOLDEN, REPO, load_plan
from srdatalog_b200.plan import PlanError, parse_filter, validate_plan

# A checkout of the reference (its src/ holds the srdatalog front end), named
# by the environment; the front-end checks are skipped without one.
REF = os.environ.get('SRDATALOG_REF', '')


@pytest.mark.parametrize('name', ['tc', 'sg', 'triangle', 'tc_left'])
def test_committed_plans_validate(name):
  validate_plan(load_plan(name))


def test_plan_shapes(plans):
  tc = plans['tc']
  canon = {r['name']: r['canonical'] for r in tc['relations']}
  assert canon['Path'] == [1, 0] and canon['Edge'] == [0, 1]
  rec = [s for s in tc['steps'] if s['recursive']]
  assert len(rec) == 1
  kinds = [o['op'] for o in rec[0]['ops']]
  assert kinds == ['execute_pipeline', 'rebuild_index', 'clear_relation', 'check_size',
                   'compute_delta_index', 'clear_relation', 'merge_index']
  tri = [o for s in plans['triangle']['steps'] for o in s['ops'] if o['op'] == 'execute_pipeline']
  assert tri[-1]['count'] is True


def test_filter_grammar():
  assert parse_filter('return x != y;', ['x', 'y']) == [('x', '!=', 'y')]
  assert parse_filter('return (x < y) && (y != 3);', ['x', 'y']) == [('x', '<', 'y'), ('y', '!=', '3')]
  with pytest.raises(PlanError):
    parse_filter('return foo(x);', ['x'])
  with pytest.raises(PlanError):
    parse_filter('return x != z;', ['x'])


def test_validate_rejects_unbound():
  plan = load_plan('tc')
  ep = plan['steps'][4]['ops'][0]
  ep['pipeline'][-1]['vars'] = ['x', 'q']
  with pytest.raises(PlanError):
    validate_plan(plan)


@pytest.mark.skipif(not REF or not os.path.isdir(os.path.join(REF, 'src', 'srdatalog')),
                    reason='srdatalog front end not available (set SRDATALOG_REF)')
def test_plans_regenerate_identically():
  r = subprocess.run([sys.executable, os.path.join(GOLDEN, 'gen_plans.py'), '--ref', REF, '--check'],
                     capture_output=True, text=True, cwd=REPO)
  assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.skipif(not REF or not os.path.isdir(os.path.join(REF, 'src', 'srdatalog')),
                    reason='srdatalog front end not available (set SRDATALOG_REF)')
def test_build_project_from_dsl(tmp_path):
  sys.path.insert(0, os.path.join(REF, 'src'))
  try:
    import programs
    from srdatalog_b200 import build_project
    proj = build_project(programs.tc_program(), 'TcPlan', cache_base=str(tmp_path))
    assert proj['plan'] == load_plan('tc')
    assert os.path.exists(proj['main']) and os.path.exists(proj['plan_path'])
  finally:
    sys.path.remove(os.path.join(REF, 'src'))
