'''Autotuner search logic with a synthetic timer (no GPU).'''

import json

import pytest
from conftest import load_plan
from srdatalog_b200.autotune import LSM, autotune, recursive_relations, with_index_types


def fake_timer(costs, sig=(('Path', 7),)):
  calls = []

  def timer(plan, options):
    idx = {r['name']: r['index_type'] for r in plan['relations']}
    ms = 100.0
    ms -= 30 if idx.get('Path') == LSM else 0
    ms -= costs.get(('bitmap_mb', options.get('bitmap_mb')), 0)
    for k in ('radix_bits', 'join_blocks_per_sm'):
      ms -= costs.get((k, options.get(k)), 0)
    if idx.get('Path') == LSM:
      ms -= costs.get(('lsm_compact_pct', options.get('lsm_compact_pct')), 0)
    calls.append((idx.get('Path'), dict(options)))
    return ms, sig

  timer.calls = calls
  return timer


def test_recursive_relations():
  assert recursive_relations(load_plan('tc')) == ['Path']
  assert recursive_relations(load_plan('triangle')) == []


def test_finds_the_fastest_setting():
  t = fake_timer({('bitmap_mb', 64): 5, ('lsm_compact_pct', 25): 3, ('radix_bits', 7): 2,
                  ('join_blocks_per_sm', 32): 1})
  r = autotune(load_plan('tc'), {'ArcInput': [[0, 1]]}, timer=t)
  assert r.index_types == {'Path': LSM}
  assert r.options == {'bitmap_mb': 64, 'lsm_compact_pct': 25, 'radix_bits': 7,
                       'join_blocks_per_sm': 32}
  assert r.ms == 100 - 30 - 5 - 3 - 2 - 1
  # the compaction knob is only tried with the LSM policy on
  assert all('lsm_compact_pct' not in o for p, o in t.calls if p != LSM)


def test_plain_policy_drops_lsm_knob():
  def timer(plan, options):
    idx = {r['name']: r['index_type'] for r in plan['relations']}
    return (50.0 if idx['Path'] == '' else 60.0), (('Path', 1),)
  r = autotune(load_plan('tc'), {'ArcInput': [[0, 1]]}, timer=timer, space={'bitmap_mb': [0, 256]})
  assert r.index_types == {'Path': ''} and 'lsm_compact_pct' not in r.options


def test_result_change_raises():
  state = {'n': 0}

  def timer(plan, options):
    state['n'] += 1
    return 10.0, (('Path', state['n']),)
  with pytest.raises(AssertionError):
    autotune(load_plan('tc'), {'ArcInput': [[0, 1]]}, timer=timer)


def test_cache_round_trip(tmp_path):
  path = str(tmp_path / 'tune.json')
  t = fake_timer({})
  r1 = autotune(load_plan('tc'), {'ArcInput': [[0, 1]] * 5}, timer=t, cache_path=path)
  n = len(t.calls)
  r2 = autotune(load_plan('tc'), {'ArcInput': [[0, 1]] * 6}, timer=t, cache_path=path)
  assert len(t.calls) == n                       # same shape class: answered from the cache
  assert r2.to_json() == r1.to_json()
  assert list(json.load(open(path)))


def test_with_index_types_copies():
  p = load_plan('tc')
  q = with_index_types(p, {'Path': LSM})
  assert [r['index_type'] for r in p['relations'] if r['name'] == 'Path'] == ['']
  assert [r['index_type'] for r in q['relations'] if r['name'] == 'Path'] == [LSM]
