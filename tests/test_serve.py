'''Serving: admission and batch formation on the host (no GPU; no workers).'''

import numpy as np
from conftest import load_plan
from srdatalog_b200.serve import ProgramSpec, Request, Server, poisson_arrivals


def programs():
  return {'tc': ProgramSpec(load_plan('tc'), 'Path'),
          'triangle': ProgramSpec(load_plan('triangle'), 'TriangleJoin', count_only=True)}


def req(i, prog, fp, n=4):
  rel = 'ArcInput' if prog == 'tc' else 'KnowsInput'
  return Request(i, prog, {rel: np.array([[0, i % n + 1]], np.uint32)}, footprint=fp)


def test_admission_respects_budget_in_arrival_order():
  s = Server(programs(), workers=0, budget_bytes=100)
  for i, fp in enumerate([40, 40, 40, 10]):
    s.submit(req(i, 'tc', fp))
  assert [r.rid for r in s.ready] == [0, 1]       # 120 > 100: request 2 waits
  assert [r.rid for r in s.pending] == [2, 3]     # and 3 does not overtake it
  assert s.peak_reserved == 80
  assert s.held_back == {2}


def test_oversized_request_runs_alone():
  s = Server(programs(), workers=0, budget_bytes=100)
  s.submit(req(0, 'tc', 500))
  assert [r.rid for r in s.ready] == [0]
  assert s.ready[0].footprint == 100              # reserved: the whole budget, no more
  s.submit(req(1, 'tc', 10))
  assert [r.rid for r in s.pending] == [1]


def test_batches_group_one_program():
  s = Server(programs(), workers=0, budget_bytes=1 << 40, max_batch=3)
  for i, p in enumerate(['tc', 'triangle', 'tc', 'tc', 'tc', 'triangle']):
    s.submit(req(i, p, 1))
  b1 = s._take_batch()
  assert [r.rid for r in b1] == [0, 2, 3]         # oldest program, max_batch of it
  b2 = s._take_batch()
  assert [r.rid for r in b2] == [1, 5]            # count-only rules batch too (grouped counts)
  assert [r.rid for r in s.ready] == [4]
  plain = Server(programs(), workers=0, batching=False)
  for i in range(3):
    plain.submit(req(i, 'tc', 1))
  assert len(plain._take_batch()) == 1


def test_poisson_arrivals_seeded():
  a = poisson_arrivals(1000, 500.0, seed=5)
  assert np.all(np.diff(a) >= 0)
  assert abs(a[-1] - 2.0) < 0.3
  assert np.array_equal(a, poisson_arrivals(1000, 500.0, seed=5))


def test_large_requests_run_alone_and_span_is_capped():
  s = Server(programs(), workers=0, budget_bytes=1 << 40, batch_max_edges=10, batch_max_span=20)
  big = Request(0, 'tc', {'ArcInput': np.zeros((11, 2), np.uint32)}, footprint=1)
  s.submit(big)
  for i in range(1, 6):
    s.submit(Request(i, 'tc', {'ArcInput': np.array([[0, 7]], np.uint32)}, footprint=1))
  assert [r.rid for r in s._take_batch()] == [0]          # over the edge limit: alone
  assert [r.rid for r in s._take_batch()] == [1, 2]       # spans 8 + 8 <= 20 < 24
  assert [r.rid for r in s._take_batch()] == [3, 4]


def test_requeue_keeps_arrival_order():
  s = Server(programs(), workers=0, budget_bytes=10)
  for i in range(4):
    r = req(i, 'tc', 10)
    r.arrival = float(i)
    s.submit(r)
  assert [r.rid for r in s.ready] == [0] and [r.rid for r in s.pending] == [1, 2, 3]
  back = s.ready.pop(0)                           # its run outgrew the reservation
  s.in_use -= back.footprint
  s._requeue(back)
  assert [r.rid for r in s.pending] == [0, 1, 2, 3]
  s._admit()
  assert [r.rid for r in s.ready] == [0]


class FakeHandle:
  def __init__(self):
    self.trimmed = 0

  def trim_cache(self):
    self.trimmed += 1


def test_idle_caches_count_against_the_budget_and_are_trimmed():
  s = Server(programs(), workers=0, budget_bytes=100)
  h = FakeHandle()
  s.idle_cache[id(h)] = (h, 70)                   # an idle handle caches 70 bytes
  s.submit(req(0, 'tc', 50))                      # 70 + 50 > 100: its cache is given back
  assert h.trimmed == 1 and s.idle_cache[id(h)] == (h, 0)
  assert [r.rid for r in s.ready] == [0]


def test_estimates_learn_from_measured_peaks():
  s = Server(programs(), workers=0, budget_bytes=1 << 40)
  small = req(0, 'tc', 0)                                      # 1 edge
  assert s._estimate(s.programs['tc'], small) == 1 << 20       # spec default before any run
  s._observe([small], 5 << 20)                                 # a 1-edge run peaked at 5 MB
  assert s._estimate(s.programs['tc'], small) == int((5 << 20) * 1.25)
  big = Request(1, 'tc', {'ArcInput': np.zeros((1 << 17, 2), np.uint32)})
  assert s._estimate(s.programs['tc'], big) == int((1 << 17) * (5 << 20) * 1.25)  # nearest class
  s._observe([big], 300 << 20)                                 # 2400 B per edge in its class
  assert s._estimate(s.programs['tc'], big) == int((300 << 20) * 1.25)
  assert s._estimate(s.programs['tc'], small) == int((5 << 20) * 1.25)
  off = Server(programs(), workers=0, learn=False)
  off._observe([small], 5 << 20)
  assert off._estimate(off.programs['tc'], small) == 1 << 20


def test_outgrown_runs_raise_their_size_class():
  s = Server(programs(), workers=0, budget_bytes=1 << 40)
  r = Request(0, 'tc', {'ArcInput': np.zeros((1 << 12, 2), np.uint32)}, footprint=8 << 20)
  s._observe_outgrown([r])                     # 8 MB was not enough for 4,096 edges
  assert s._estimate(s.programs['tc'], r) == int(2 * (8 << 20) * 1.25)
