'''Batched fixpoints: many independent instances of one program in one run.

Instance j's values are shifted by an offset o_j = sum over k < j of
(largest value of instance k + 1), and all instances are loaded together.
Datalog never creates values, and a rule can only join tuples through
shared values, so no tuple of the union can mix two instances: the union's
least fixpoint is the disjoint union of the instances' fixpoints, each
living in its own value range [o_j, o_j + span_j).  One srdl_run then
evaluates every instance in the same launches -- each iteration's kernels
cover all instances that still have a delta; instances that converged early
simply contribute nothing -- and instance j's result is read back as the
rows whose first column lies in its range.

Requirements checked here: the plan's filters and rule heads use no
constants (a constant would have to be shifted per instance), and the union's values fit in
uint32.  Count-only rules are counted per instance too: the count of every
binding is also added to the group of its first variable's value
(srdl_set_count_groups), and each instance is one group.
'''

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .native import Database
from .plan import parse_filter


class BatchError(ValueError):
  pass


def count_rules(plan: dict) -> list:
  return [op['rule'] for st in plan['steps'] for op in st['ops']
          if op['op'] == 'execute_pipeline' and op.get('count')]


def check_batchable(plan: dict) -> None:
  '''Reject plans whose filters compare with constants or whose rule
  heads hold constants (relations with facts).'''
  for r in plan['relations']:
    if r.get('facts'):
      raise BatchError(f'relation {r["name"]}: a head constant prevents value shifting')
  for step in plan['steps']:
    for op in step['ops']:
      if op['op'] != 'execute_pipeline':
        continue
      bound: list[str] = []
      for p in op['pipeline']:
        if p['op'] in ('scan', 'cartesian_join'):
          bound += p['vars']
        elif p['op'] == 'column_join':
          bound.append(p['var'])
        elif p['op'] == 'filter':
          for a, _, b in parse_filter(p['code'], bound):
            if a.isdigit() or b.isdigit():
              raise BatchError(f'rule {op["rule"]}: a filter constant prevents value shifting')


@dataclass
class Union:
  inputs: dict           # relation -> (m, arity) uint32 rows of the union
  offsets: np.ndarray    # (k+1,) uint64 range starts; offsets[k] = end of the last range


def make_union(instances: list[dict]) -> Union:
  '''instances: list of {relation: (m, arity) uint32 rows}.'''
  spans = []
  for inst in instances:
    mx = -1
    for rows in inst.values():
      a = np.asarray(rows)
      if a.size:
        mx = max(mx, int(a.max()))
    spans.append(mx + 1 if mx >= 0 else 1)
  offsets = np.zeros(len(instances) + 1, np.uint64)
  offsets[1:] = np.cumsum(np.asarray(spans, np.uint64))
  if int(offsets[-1]) > 0xFFFFFFFF:
    raise BatchError('the union of the instances needs more than 2^32 values')
  parts: dict = {}
  for j, inst in enumerate(instances):
    for rel, rows in inst.items():
      a = np.asarray(rows, np.uint64)
      parts.setdefault(rel, []).append((a + offsets[j]).astype(np.uint32))
  inputs = {rel: np.ascontiguousarray(np.concatenate(p, axis=0)) for rel, p in parts.items()}
  return Union(inputs, offsets)


class BatchRun:
  '''One disjoint-union evaluation; per-instance sizes and rows on demand.'''

  def __init__(self, plan: dict, instances: list[dict], device: int = 0, max_iters: int = 0,
               db: Database | None = None, union: Union | None = None):
    check_batchable(plan)
    self.union = union or make_union(instances)
    self.k = len(self.union.offsets) - 1
    self.db = db or Database(plan, device=device)
    self.db.clear_inputs()
    for rel, rows in self.union.inputs.items():
      self.db.load_rows(rel, rows)
    bounds = self.union.offsets.astype(np.uint32)
    for rule in count_rules(plan):
      self.db.set_count_groups(rule, bounds)
    self.db.run(max_iters)

  def counts(self, rule: str) -> np.ndarray:
    '''Per-instance counts of a count-only rule.'''
    return self.db.group_counts(rule)

  def sizes(self, rel: str) -> np.ndarray:
    '''Per-instance row counts of FULL(rel), computed on the device.'''
    return self.db.range_counts(rel, self.union.offsets.astype(np.uint32))

  def split_rows(self, rel: str) -> list[np.ndarray]:
    '''Every instance's rows of FULL(rel), shifted back to its own values.'''
    all_rows = self.db.dump(rel)
    cuts = np.searchsorted(all_rows[:, 0], self.union.offsets.astype(np.int64), side='left')
    return [(all_rows[cuts[j]:cuts[j + 1]].astype(np.uint64) - self.union.offsets[j])
            .astype(np.uint32) for j in range(self.k)]
