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


def peak_alone(req, loop=True):
  '''Device bytes a fresh handle holds at the peak of the request's run
  (loop=False: on the host path, the least a run needs -- under a tighter
  memory limit the device loop declines its buffers and runs there).'''
  db = native.Database(load_plan(req.program))
  db.set_option('device_loop', 1 if loop else 0)
  for rel, rows in req.inputs.items():
    db.load_rows(rel, rows)
  db.run()
  return db.mem_stats()['peak']


def test_budget_is_never_exceeded():
  '''Runs are held to their reservations and admitted within the budget;
  the peak is the device bytes the library measured, not an estimate.'''
  reqs = make_requests(24, seed=8)
  budget = 4 * max(peak_alone(r) for r in reqs)
  with Server(programs(), workers=3, budget_bytes=budget) as srv:
    replay(srv, reqs, np.zeros(len(reqs)))
    assert 0 < srv.peak_in_use <= budget
    assert srv.peak_reserved <= budget
  for r in reqs:
    assert not r.error
    assert r.result == alone(r)[0]
    assert 0 < r.peak_bytes <= budget


def test_outgrown_reservation_is_requeued_and_held_back():
  '''Estimates far below the real need (1 MB): every run that outgrows its
  reservation stops with status 5 and goes back to the queue with twice the
  reservation; once reservations are large, only one run fits the budget at
  a time and the others wait.  Every result still equals the request run
  alone, and the measured device bytes never pass the budget.'''
  progs = {'tc': ProgramSpec(load_plan('tc'), 'Path', bytes_per_edge=1)}
  reqs = [Request(i, 'tc', {'ArcInput': W.uniform_edges(2000, 6000, 40 + i)}) for i in range(3)]
  peak = max(peak_alone(r, loop=False) for r in reqs)
  mb = 1 << 20
  grown = mb << max(0, (peak - 1) // mb).bit_length()    # the doubling's first reservation >= peak
  budget = grown + grown // 2                            # room for one such run at a time
  with Server(progs, workers=3, budget_bytes=budget, learn=False) as srv:
    replay(srv, reqs, np.zeros(len(reqs)))
    assert srv.retried >= len(reqs)
    assert srv.held_back                                 # a grown request waited for the budget
    assert 0 < srv.peak_in_use <= budget
  for r in reqs:
    assert not r.error and r.retries > 0
    assert r.footprint <= budget and r.peak_bytes <= r.footprint
    assert r.result == alone(r)[0]


def test_request_beyond_the_budget_fails_cleanly():
  '''A request whose run outgrows the whole budget fails (error set, result
  -1) without stopping the server; the other request is answered.'''
  progs = {'tc': ProgramSpec(load_plan('tc'), 'Path', bytes_per_edge=1)}
  big = Request(0, 'tc', {'ArcInput': W.uniform_edges(2000, 6000, 40)})
  small = Request(1, 'tc', {'ArcInput': W.uniform_edges(50, 80, 41)})
  budget = max(8 << 20, 4 * peak_alone(small))
  assert peak_alone(big) > budget
  with Server(progs, workers=2, budget_bytes=budget, learn=False) as srv:
    replay(srv, [big, small], np.zeros(2))
  assert big.result == -1 and 'memory limit' in big.error
  assert not small.error and small.result == alone(small)[0]
