'''Serving on the GPU: every request's result is the same alone and in the
mix (concurrent workers, continuous batching), and equals the oracle.'''

import numpy as np
import oracle
import pytest
from conftest import load_plan
from srdatalog_b200 import native
from srdatalog_b200 import workloads as W
from srdatalog_b200.serve import ProgramSpec, Request, Server, log_uniform_sizes, poisson_arrivals, replay

pytestmark = pytest.mark.gpu

OUT = {'tc': 'Path', 'sg': 'Sg', 'triangle': 'TriangleJoin'}


def programs():
  return {'tc': ProgramSpec(load_plan('tc'), 'Path'), 'sg': ProgramSpec(load_plan('sg'), 'Sg'),
          'triangle': ProgramSpec(load_plan('triangle'), 'TriangleJoin', count_only=True)}


def make_requests(n, seed):
  rng = np.random.default_rng(seed)
  progs = rng.choice(['tc', 'sg', 'triangle'], size=n, p=[0.5, 0.3, 0.2])
  sizes = log_uniform_sizes(n, 100, 4000, seed)
  return [Request(i, str(p), W.served_request_input(str(p), int(m), 10_000 + i))
          for i, (p, m) in enumerate(zip(progs, sizes))]


def alone(req):
  db = native.Database(load_plan(req.program))
  for rel, rows in req.inputs.items():
    db.load_rows(rel, rows)
  db.run()
  if req.program == 'triangle':
    return db.count('TriangleJoin'), None
  return db.size(OUT[req.program]), db.dump(OUT[req.program])


def test_mixed_requests_same_alone_and_in_the_mix():
  reqs = make_requests(60, seed=3)
  with Server(programs(), workers=3, keep_rows=True, max_batch=16) as srv:
    stats = replay(srv, reqs, poisson_arrivals(len(reqs), 2000.0, seed=4))
  assert stats.summary()['mean_batch'] > 1.0      # batching did happen
  for r in reqs:
    want, rows = alone(r)
    assert r.result == want, (r.rid, r.program)
    if rows is not None:
      assert oracle.dump_hash(r.rows) == oracle.dump_hash(rows)
  for r in reqs[:12]:
    e = list(r.inputs.values())[0]
    if r.program == 'tc':
      keys, _, _ = oracle.tc(e)
      assert r.result == keys.shape[0]
    elif r.program == 'sg':
      keys, _, _ = oracle.sg(e)
      assert r.result == keys.shape[0]
    else:
      assert r.result == oracle.triangle_count(e)


def test_budget_is_never_exceeded():
  reqs = make_requests(24, seed=8)
  fps = [max(1 << 20, 512 * sum(v.shape[0] for v in r.inputs.values())) for r in reqs]
  budget = max(fps)
  with Server(programs(), workers=3, budget_bytes=budget) as srv:
    replay(srv, reqs, np.zeros(len(reqs)))
    assert srv.peak_in_use <= budget
  for r in reqs:
    assert r.result == alone(r)[0]
