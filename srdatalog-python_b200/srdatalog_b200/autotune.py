'''Autotuner: picks a program's runtime settings by timing runs on the
caller's own input.

None of the knobs changes a result; they trade memory and work:

* ``index_type`` of every relation a recursive step merges into: ``''`` (one
  sorted array per permutation) or ``Device2LevelIndex`` (FULL + HEAD, the
  reference's LSM policy, device_2level_index.h:35-321);
* ``bitmap_mb``: budget for bitmaps of the longest child lists of probed FULL
  indexes (0 turns them off);
* ``lsm_compact_pct``: HEAD is merged into FULL once it exceeds this
  percentage of FULL (only tried when some relation uses the LSM policy);
* ``radix_bits``: widest radix-sort digit (passes = key bits / this);
* ``join_blocks_per_sm``: grid cap of the join launches, i.e. the
  candidates each warp walks (the work-splitting chunk).

Search: coordinate descent from the defaults -- each knob in turn takes every
value of its range with the others fixed, and the fastest (median of ``reps``
timed runs after one warm-up run) is kept; at most two sweeps.  Every run's
output signature (sizes of the relations the program prints, counts of its
count-only rules) must equal the first run's, else the tuner raises.  Results
can be cached in a JSON file keyed by the plan's name and the input's shape
(row counts rounded up to powers of two).
'''

from __future__ import annotations

import copy
import json
import os
import statistics
import time
from dataclasses import dataclass, field

import numpy as np

LSM = 'SRDatalog::GPU::Device2LevelIndex'

DEFAULT_SPACE = {
  'bitmap_mb': [0, 64, 256, 768, 2048],
  'lsm_compact_pct': [5, 10, 25],
  'radix_bits': [6, 7, 8],
  'join_blocks_per_sm': [8, 16, 32],
}

# library defaults: the tuner's starting point
DEFAULTS = {'bitmap_mb': 768, 'lsm_compact_pct': 10, 'radix_bits': 8, 'join_blocks_per_sm': 16}


@dataclass
class TuneResult:
  index_types: dict                 # relation -> index_type
  options: dict                     # srdl_set_option name -> value
  ms: float                         # median run time of the chosen setting
  trials: list = field(default_factory=list)   # [(setting, ms)] in the order tried

  def apply(self, plan: dict) -> dict:
    '''A copy of `plan` with the chosen index types.'''
    return with_index_types(plan, self.index_types)

  def configure(self, db) -> None:
    '''Set the chosen options on a native.Database.'''
    for k, v in self.options.items():
      db.set_option(k, v)

  def to_json(self) -> dict:
    return {'index_types': self.index_types, 'options': self.options, 'ms': self.ms}


def recursive_relations(plan: dict) -> list:
  '''Relations that a recursive step merges deltas into (the LSM candidates).'''
  out = []
  for st in plan['steps']:
    if not st['recursive']:
      continue
    for op in st['ops']:
      if op['op'] == 'merge_index' and op['rel'] not in out:
        out.append(op['rel'])
  return out


def with_index_types(plan: dict, index_types: dict) -> dict:
  p = copy.deepcopy(plan)
  for r in p['relations']:
    if r['name'] in index_types:
      r['index_type'] = index_types[r['name']]
  return p


def input_signature(inputs: dict) -> str:
  parts = []
  for name in sorted(inputs):
    n = int(np.asarray(inputs[name]).shape[0])
    parts.append(f'{name}:{1 << max(n - 1, 0).bit_length()}')
  return ','.join(parts)


def _output_signature(db, plan: dict) -> tuple:
  sig = []
  for r in plan['relations']:
    if r.get('print_size') and r['arity'] <= 2:
      sig.append((r['name'], db.size(r['name'])))
  for st in plan['steps']:
    for op in st['ops']:
      if op['op'] == 'execute_pipeline' and op.get('count'):
        sig.append((op['rule'], db.count(op['rule'])))
  return tuple(sig)


def native_timer(inputs: dict, device: int = 0, reps: int = 3):
  '''timer(plan, options) -> (median ms, output signature): one database per
  plan variant (index types change the plan), the inputs loaded once.'''
  from .native import Database

  dbs: dict = {}

  def timer(plan: dict, options: dict):
    key = json.dumps([r['index_type'] for r in plan['relations']])
    db = dbs.get(key)
    if db is None:
      db = dbs[key] = Database(plan, device=device)
      for rel, rows in inputs.items():
        db.load_rows(rel, rows)
    for k, v in options.items():
      db.set_option(k, v)
    db.run()
    times = []
    for _ in range(reps):
      t0 = time.perf_counter()
      db.run()
      times.append((time.perf_counter() - t0) * 1e3)
    return statistics.median(times), _output_signature(db, plan)

  timer.close = lambda: [db.close() for db in dbs.values()]  # type: ignore[attr-defined]
  return timer


def autotune(plan: dict, inputs: dict, device: int = 0, reps: int = 3, space: dict | None = None,
             cache_path: str | None = None, timer=None) -> TuneResult:
  '''Tune `plan` on `inputs` (see the module doc).  `timer(plan, options)`
  may replace the native timer (tests use a synthetic one).'''
  space = dict(DEFAULT_SPACE if space is None else space)
  key = f'{plan.get("name", "plan")}|{input_signature(inputs)}'
  if cache_path and os.path.exists(cache_path):
    cached = json.load(open(cache_path)).get(key)
    if cached:
      return TuneResult(cached['index_types'], cached['options'], cached['ms'])
  own = timer is None
  if own:
    timer = native_timer(inputs, device, reps)
  rec = recursive_relations(plan)
  knobs = [(f'index_type:{r}', ['', LSM]) for r in rec]
  knobs += [(k, list(v)) for k, v in space.items()]
  setting = {f'index_type:{r}': next(x['index_type'] for x in plan['relations'] if x['name'] == r)
             for r in rec}
  setting.update(DEFAULTS)
  setting = {k: v for k, v in setting.items() if any(k == kk for kk, _ in knobs)}
  trials: list = []
  seen: dict = {}
  ref_sig = None

  def run(s: dict) -> float:
    nonlocal ref_sig
    frozen = json.dumps(s, sort_keys=True)
    if frozen in seen:
      return seen[frozen]
    idx = {k.split(':', 1)[1]: v for k, v in s.items() if k.startswith('index_type:')}
    opts = {k: v for k, v in s.items() if not k.startswith('index_type:')}
    if not any(v == LSM for v in idx.values()) and 'lsm_compact_pct' in opts:
      opts = {k: v for k, v in opts.items() if k != 'lsm_compact_pct'}
    ms, sig = timer(with_index_types(plan, idx), opts)
    if ref_sig is None:
      ref_sig = sig
    elif sig != ref_sig:
      raise AssertionError(f'autotune: setting {s} changed the result {sig} != {ref_sig}')
    seen[frozen] = ms
    trials.append((dict(s), ms))
    return ms

  try:
    best = run(setting)
    for _ in range(2):
      improved = False
      for name, values in knobs:
        for v in values:
          if setting.get(name) == v:
            continue
          if name == 'lsm_compact_pct' and not any(
              setting.get(k) == LSM for k in setting if k.startswith('index_type:')):
            continue
          cand = dict(setting)
          cand[name] = v
          ms = run(cand)
          if ms < best:
            best, setting, improved = ms, cand, True
      if not improved:
        break
  finally:
    if own:
      timer.close()
  idx = {k.split(':', 1)[1]: v for k, v in setting.items() if k.startswith('index_type:')}
  opts = {k: v for k, v in setting.items() if not k.startswith('index_type:')}
  if not any(v == LSM for v in idx.values()):
    opts.pop('lsm_compact_pct', None)
  result = TuneResult(idx, opts, best, trials)
  if cache_path:
    data = json.load(open(cache_path)) if os.path.exists(cache_path) else {}
    data[key] = result.to_json()
    with open(cache_path, 'w') as f:
      json.dump(data, f, indent=1, sort_keys=True)
  return result


__all__ = ['TuneResult', 'autotune', 'recursive_relations', 'with_index_types', 'native_timer',
           'input_signature', 'LSM']
