'''Serving: a request loop that admits Datalog queries of mixed programs and
sizes against a device-memory budget and batches them continuously.

* Admission: every request holds a reservation of device memory
  (`footprint`, first an estimate from its input size); it is admitted when
  the reservations of the admitted, unfinished requests plus the blocks idle
  handles cache stay within the budget, in arrival order (a large request
  waits; later small ones do not overtake it).
* Estimates: a request's first reservation comes from its program's measured
  runs: the largest peak per input edge of runs in its size class (input
  edges to a power of two; the nearest class seen), times 1.25, with a 1 MB
  floor; before any run, from the spec's bytes_per_edge.  A run that
  outgrows its reservation raises its class to twice that reservation.
* Enforcement: a run may hold at most its batch's reservations on the device
  (libsrdl's per-run limit, option mem_limit_mb, measured by the handle's
  caching arena).  A run that outgrows it stops with status 5; its requests
  go back to the head of the queue with twice the reservation and are
  admitted again when memory frees up.  A request that outgrows the whole
  budget fails cleanly (`error` set, result -1) while the others proceed.
* Continuous batching: a dispatcher hands work to whichever of the `workers`
  is idle.  A worker takes the oldest admitted request and, with it, every
  admitted request of the same program (up to `max_batch`), and evaluates
  them as one disjoint-union run (srdatalog_b200.batch): their iterations share
  launches; count-only programs (the triangle count) get per-request counts
  from grouped counting.  Only small requests are unioned (see Server).
* Workers own their database handles, so each has its own CUDA stream and
  the runs of different workers overlap on the GPU; relations stay on the
  device until the request's result (its size or count) has been read.
* Measured memory: after every run the server reads, from the library, the
  device bytes every handle holds and caches (srdl_mem_stats); `peak_in_use`
  is the largest such total seen, `peak_reserved` the largest sum of
  reservations.

A request's result is identical alone and in any mix: instances of a union
cannot interact (see batch.py), and runs on different handles share nothing.
'''

from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from .batch import make_union
from .native import Database, SrdlError

_MB = 1 << 20


@dataclass
class Request:
  rid: int
  program: str                 # key into the server's plans
  inputs: dict                 # relation -> (m, 2) uint32 rows
  arrival: float = 0.0         # seconds (perf_counter clock)
  footprint: int = 0           # reserved device bytes (estimate; doubled when outgrown)
  retries: int = 0             # runs that outgrew the reservation
  peak_bytes: int = 0          # measured peak of the run that answered it (its union's)
  error: str = ''              # set when the request failed (result stays -1)
  admitted: float = -1.0
  started: float = -1.0
  finished: float = -1.0
  result: int = -1             # size of the output relation, or the count
  rows: np.ndarray | None = None
  batch_size: int = 0

  @property
  def latency(self) -> float:
    return self.finished - self.arrival


@dataclass
class ProgramSpec:
  plan: dict
  out: str                     # output relation (size) or rule (count)
  count_only: bool = False
  bytes_per_edge: int = 512    # footprint estimate per input edge


def default_footprint(spec: ProgramSpec, req: Request) -> int:
  m = sum(int(np.asarray(r).shape[0]) for r in req.inputs.values())
  return max(1 << 20, m * spec.bytes_per_edge)


@dataclass
class ServeStats:
  requests: list = field(default_factory=list)
  wall_s: float = 0.0

  def summary(self) -> dict:
    lat = np.array([r.latency for r in self.requests]) * 1e3
    bs = np.array([r.batch_size for r in self.requests])
    return {
      'requests': len(self.requests),
      'queries_per_s': len(self.requests) / self.wall_s if self.wall_s else 0.0,
      'p50_ms': float(np.percentile(lat, 50)) if lat.size else None,
      'p99_ms': float(np.percentile(lat, 99)) if lat.size else None,
      'mean_batch': float(bs.mean()) if bs.size else None,
      'wall_s': self.wall_s,
    }


class Server:
  '''Admission-controlled, continuously batching request loop (see module doc).'''

  def __init__(self, programs: dict, device: int = 0, workers: int = 8,
               budget_bytes: int = 120 << 30, max_batch: int = 16, batching: bool = True,
               keep_rows: bool = False, batch_max_edges: int = 1 << 20,
               batch_max_span: int = 1 << 23, learn: bool = True, device_loop: bool = False):
    self.programs = programs
    self.device_loop = device_loop
    # Reservation estimates learned from measured peaks: per program and
    # size class (input edges to a power of two), the largest peak per input
    # edge seen.  Without learning (or before the program's first run) the
    # spec's bytes_per_edge with a 1 MB floor.
    self.learn = learn
    self.est_ratio: dict = {}
    self.device = device
    self.budget = budget_bytes
    self.max_batch = max_batch if batching else 1
    self.keep_rows = keep_rows
    # Only small requests are unioned: their runs are dominated by per-launch
    # and per-iteration overhead, which a union shares.  A large request runs
    # alone (other workers proceed in parallel), and a union's value span stays
    # small enough for the dense per-value directory.
    self.batch_max_edges = batch_max_edges
    self.batch_max_span = batch_max_span
    self.cv = threading.Condition()
    self.pending: list[Request] = []   # arrived, waiting for admission (FIFO)
    self.ready: list[Request] = []     # admitted, not started
    self.in_use = 0                    # reservations of admitted, unfinished requests
    self.peak_reserved = 0
    self.idle_cache: dict = {}         # handle id -> (handle, bytes it caches while idle)
    self.handles: list = []            # every handle of every worker (measured usage)
    self.peak_in_use = 0               # largest measured device bytes of all handles
    self.retried = 0                   # runs that outgrew their reservation
    self.held_back: set = set()        # ids of requests that waited for the budget
    self.submitted = 0
    self.done: list[Request] = []
    self.errors: list[BaseException] = []
    self.stopping = False
    self.threads = [threading.Thread(target=self._worker, args=(w,), daemon=True)
                    for w in range(workers)]
    for t in self.threads:
      t.start()

  # ------------------------------------------------------------ client side
  def submit(self, req: Request) -> None:
    spec = self.programs[req.program]
    with self.cv:
      if not req.footprint:
        req.footprint = self._estimate(spec, req)
      req.footprint = min(req.footprint, self.budget)
      self.pending.append(req)
      self.submitted += 1
      self._admit()
      self.cv.notify_all()

  def drain(self, timeout_s: float = 3600.0) -> None:
    '''Wait until every submitted request has finished (or raise).'''
    deadline = time.perf_counter() + timeout_s
    with self.cv:
      while len(self.done) < self.submitted and not self.errors:
        left = deadline - time.perf_counter()
        if left <= 0:
          raise TimeoutError('serving did not drain in time')
        self.cv.wait(min(left, 1.0))
      if self.errors:
        raise RuntimeError(f'worker failed: {self.errors[0]!r}')

  def close(self) -> None:
    with self.cv:
      self.stopping = True
      self.cv.notify_all()
    for t in self.threads:
      t.join(timeout=60)

  def __enter__(self):
    return self

  def __exit__(self, *exc):
    self.close()

  # ------------------------------------------------------------ scheduling
  def _admit(self) -> None:
    now = time.perf_counter()
    while self.pending:
      r = self.pending[0]
      cached = sum(b for _, b in self.idle_cache.values())
      # a request as large as the whole budget runs alone
      if self.in_use + cached + r.footprint > self.budget and self.in_use + cached > 0:
        if cached:
          self._trim_idle()
          continue
        self.held_back.add(r.rid)
        break
      self.pending.pop(0)
      self.in_use += r.footprint
      self.peak_reserved = max(self.peak_reserved, self.in_use)
      r.admitted = now
      self.ready.append(r)

  def _trim_idle(self) -> None:
    '''Idle handles give their cached blocks back (called with cv held: a
    worker takes its handle out of idle_cache under cv before running it).'''
    for key, (db, _) in list(self.idle_cache.items()):
      db.trim_cache()
      self.idle_cache[key] = (db, 0)

  def _estimate(self, spec: ProgramSpec, req: Request) -> int:
    m = _edges(req)
    known = self.est_ratio.get(req.program)
    if not known:
      return default_footprint(spec, req)
    b = m.bit_length()
    nearest = min(known, key=lambda k: (abs(k - b), -k))   # ties: the larger size class
    return max(1 << 20, int(m * known[nearest] * 1.25))

  def _observe(self, batch: list, peak: int) -> None:
    '''Learn from a successful run's measured peak (cv held): the largest
    peak per input edge of the program's runs with as many edges, to a
    power of two.'''
    if not self.learn or peak <= 0:
      return
    m = max(1, sum(_edges(r) for r in batch))
    ratios = self.est_ratio.setdefault(batch[0].program, {})
    b = m.bit_length()
    ratios[b] = max(ratios.get(b, 0.0), peak / m)

  def _observe_outgrown(self, batch: list) -> None:
    '''A run that outgrew its reservation needs more than it: its size
    class starts at twice that from now on (cv held).'''
    if not self.learn:
      return
    m = max(1, sum(_edges(r) for r in batch))
    ratios = self.est_ratio.setdefault(batch[0].program, {})
    b = m.bit_length()
    ratios[b] = max(ratios.get(b, 0.0), 2.0 * sum(r.footprint for r in batch) / m)

  def _requeue(self, r: Request) -> None:
    '''Back into the pending queue in arrival order (ahead of later arrivals).'''
    i = 0
    while i < len(self.pending) and (self.pending[i].arrival, self.pending[i].rid) <= (r.arrival, r.rid):
      i += 1
    self.pending.insert(i, r)

  def _take_batch(self) -> list:
    first = self.ready[0]
    if self.max_batch == 1 or _edges(first) > self.batch_max_edges:
      batch = [first]
    else:
      batch, span = [], 0
      for r in self.ready:
        if r.program != first.program or _edges(r) > self.batch_max_edges:
          continue
        s = _span(r)
        if batch and (len(batch) >= self.max_batch or span + s > self.batch_max_span):
          break
        batch.append(r)
        span += s
    ids = {id(r) for r in batch}
    self.ready = [r for r in self.ready if id(r) not in ids]
    return batch

  def _measure(self) -> None:
    '''Device bytes all handles hold and cache now, read from the library.'''
    total = 0
    for db in list(self.handles):
      m = db.mem_stats()
      total += m['in_use'] + m['cached']
    self.peak_in_use = max(self.peak_in_use, total)

  def _worker(self, wid: int) -> None:
    dbs: dict = {}
    try:
      while True:
        with self.cv:
          while not self.ready and not self.stopping:
            self.cv.wait()
          if not self.ready:
            return
          batch = self._take_batch()
        t0 = time.perf_counter()
        for r in batch:
          r.started = t0
          r.batch_size = len(batch)
        db = self._handle(dbs, batch[0].program)
        with self.cv:
          self.idle_cache.pop(id(db), None)
        # the run may hold at most its requests' reservations
        db.set_option('mem_limit_mb', max(1, sum(r.footprint for r in batch) // _MB))
        outgrown = ''
        try:
          self._run(db, batch)
        except SrdlError as e:
          if e.code != 5:
            raise
          outgrown = str(e)
        mem = db.mem_stats()
        t1 = time.perf_counter()
        with self.cv:
          self._measure()
          for r in batch:
            self.in_use -= r.footprint
            r.peak_bytes = mem['peak']
          if outgrown:
            self.retried += 1
            self._observe_outgrown(batch)
            for r in batch:
              if r.footprint >= self.budget:
                r.error = outgrown
                r.result = -1
                r.finished = t1
                self.done.append(r)
              else:
                r.retries += 1
                r.footprint = min(self.budget, 2 * r.footprint)
                self._requeue(r)
          else:
            self._observe(batch, mem['peak'])
            for r in batch:
              r.finished = t1
            self.done.extend(batch)
          self.idle_cache[id(db)] = (db, mem['cached'])
          self._admit()
          self.cv.notify_all()
    except BaseException as e:  # surface to drain()
      with self.cv:
        self.errors.append(e)
        self.cv.notify_all()
    finally:
      with self.cv:
        for db in dbs.values():
          self.idle_cache.pop(id(db), None)
          if db in self.handles:
            self.handles.remove(db)
      for db in dbs.values():
        db.close()

  def _handle(self, dbs: dict, program: str) -> Database:
    db = dbs.get(program)
    if db is None:
      db = dbs[program] = Database(self.programs[program].plan, device=self.device)
      db.init_device()
      # The served requests are small and their unions short-lived: the
      # device loop's graph capture and capacity buffers cost them more than
      # its saved host round trips (and inflate the learned reservations).
      db.set_option('device_loop', 1 if self.device_loop else 0)
      with self.cv:
        self.handles.append(db)
    return db

  def _run(self, db: Database, batch: list) -> None:
    spec = self.programs[batch[0].program]
    db.clear_inputs()
    if spec.count_only:
      db.set_count_groups(spec.out, [])
    if len(batch) == 1:
      r = batch[0]
      for rel, rows in r.inputs.items():
        db.load_rows(rel, rows)
      db.run()
      r.result = db.count(spec.out) if spec.count_only else db.size(spec.out)
      if self.keep_rows and not spec.count_only:
        r.rows = db.dump(spec.out)
      return
    union = make_union([r.inputs for r in batch])
    for rel, rows in union.inputs.items():
      db.load_rows(rel, rows)
    bounds = union.offsets.astype(np.uint32)
    if spec.count_only:
      db.set_count_groups(spec.out, bounds)
    db.run()
    sizes = db.group_counts(spec.out) if spec.count_only else db.range_counts(spec.out, bounds)
    all_rows = db.dump(spec.out) if self.keep_rows and not spec.count_only else None
    if all_rows is not None:
      cuts = np.searchsorted(all_rows[:, 0], union.offsets.astype(np.int64), side='left')
    for j, r in enumerate(batch):
      r.result = int(sizes[j])
      if all_rows is not None:
        r.rows = (all_rows[cuts[j]:cuts[j + 1]].astype(np.uint64) - union.offsets[j]).astype(np.uint32)


def _edges(r: Request) -> int:
  return sum(int(np.asarray(a).shape[0]) for a in r.inputs.values())


def _span(r: Request) -> int:
  mx = -1
  for rows in r.inputs.values():
    a = np.asarray(rows)
    if a.size:
      mx = max(mx, int(a.max()))
  return mx + 1 if mx >= 0 else 1


def poisson_arrivals(n: int, rate: float, seed: int) -> np.ndarray:
  '''n arrival offsets (seconds) of a Poisson process with the given rate.'''
  rng = np.random.Generator(np.random.PCG64(seed))
  return np.cumsum(rng.exponential(1.0 / rate, n))


def replay(server: Server, requests: list, offsets: np.ndarray) -> ServeStats:
  '''Open-loop client: submits request i at t0 + offsets[i] (its latency is
  measured from that scheduled time), then waits for all to finish.'''
  order = np.argsort(offsets, kind='stable')
  t0 = time.perf_counter()
  for i in order:
    due = t0 + float(offsets[i])
    d = due - time.perf_counter()
    if d > 0:
      time.sleep(d)
    requests[i].arrival = due
    server.submit(requests[i])
  server.drain()
  end = max(r.finished for r in requests)
  return ServeStats(requests=list(requests), wall_s=end - t0)


def log_uniform_sizes(n: int, lo: float, hi: float, seed: int) -> np.ndarray:
  rng = np.random.Generator(np.random.PCG64(seed))
  return np.round(np.exp(rng.uniform(math.log(lo), math.log(hi), n))).astype(np.int64)


__all__ = ['Request', 'ProgramSpec', 'Server', 'ServeStats', 'replay', 'poisson_arrivals',
           'log_uniform_sizes', 'default_footprint']
