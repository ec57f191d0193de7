'''Benchmark: semi-naive Datalog on B200 through libsrdl.

Default workload (one step = one srdl_run of the plan over one input):
  triangle  -- count-only 3-way WCOJ over an R-MAT graph, scale 20,
               16,777,216 draws, (a,b,c,d) = (0.57,0.19,0.19,0.05), seed 3,
               oriented x<y, deduplicated (15,701,388 edges).
Others (--workload): tc (20k edges over 5k nodes, seed 1) and sg (windowed
forest, n = 10,000, seed 2; the stated 200k-node forest outgrows HBM).

value : tuples/s with the input already in HBM (srdl_load_device_rows),
        CUDA events on the database stream, L2 flushed between steps.
e2e   : same metric through the C ABI from pinned host rows (srdl_load_rows
        + srdl_run, which uploads them), result read back to the host.
Multi-GPU (torchrun): one program sharded over the GPUs
(srdatalog_b200.shard: the triangle count splits a join level's work
items, TC partitions Path by source, SG partitions Sg and sends each
iteration's derived tuples to their owners with one all-to-all; inputs
replicated, one final all-reduce of the result), value = the job's tuples
over the max per-rank time (strong scaling); plans the analysis cannot
shard run as independent replicas (weak scaling).
SRDL_BENCH_BACKEND=gloo runs the collectives on the host (ranks may then
share a GPU, which exercises the N>1 path but times nothing meaningful).
--workload served: the request server (8 workers, unions of at most 16
requests: --serve-workers, --serve-max-batch) against the plain loop at
--rate offered requests/s.
--workload primitives: the sort / merge / set-difference primitives alone
(--keys, --bits), one JSON line each.
--impl reference: the CPU restatement of the reference's evaluation on
the host cores, one full run of the same workload per step (the batched
and served workloads: a seeded sample of their queries).
'''

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(REPO, 'srdatalog-python_b200'), os.path.join(REPO, 'oracle')]

import numpy as np  # noqa: E402

PEAKS_PATH = os.path.join(REPO, 'MEASURED_PEAKS.json')
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
  'triangle': dict(plan='triangle', rel='KnowsInput', out='TriangleJoin', kind='count',
                   desc='triangle count, R-MAT scale 20, 16,777,216 draws, '
                        '(a,b,c,d)=(0.57,0.19,0.19,0.05), seed 3, oriented x<y, dedup'),
  'tc': dict(plan='tc', rel='ArcInput', out='Path', kind='size',
             desc='transitive closure, 20,000 distinct uniform edges over 5,000 nodes, seed 1'),
  'sg': dict(plan='sg', rel='Arc', out='Sg', kind='size',
             desc='same generation, windowed forest n=10,000 (parent in [i-1000,i-1]) '
                  '+ 10% cross edges, seed 2'),
  'batched': dict(plan='tc', rel='ArcInput', out='Path', kind='batched', tune=True,
                  desc='4,096 independent TC instances, directed Erdos-Renyi, n log-uniform in '
                       '[64, 1024], mean out-degree U[2,8], seed 1000+j; evaluated as one '
                       'disjoint union; index policy and options picked by the autotuner'),
  'batched-wide': dict(plan='tc', rel='ArcInput', out='Path', kind='batched', tune=True,
                       desc='the batched config\'s own 4,096 draws (n log-uniform in [64, 65,536], '
                            'mean out-degree U[2,8], seed 1000+j), the instances with n <= '
                            '{n_max}; evaluated in disjoint-union waves under a device-memory '
                            'budget; options picked by the autotuner'),
}

BATCH_COUNT = 4096
BATCH_N_HI = 1024
PLAIN_SAMPLE_STRIDE = 16
WIDE_N_MAX = 8192


_BATCH = None


def make_batch(name: str = 'batched', n_max: int = WIDE_N_MAX) -> list:
  """Instances of a batched workload (generated once per process)."""
  global _BATCH
  if _BATCH is None or _BATCH[0] != (name, n_max):
    from srdatalog_b200 import workloads as W
    if name == 'batched':
      es = W.batched_instances(count=BATCH_COUNT, n_hi=BATCH_N_HI)
    else:
      es = W.batched_instances(count=BATCH_COUNT, n_hi=65536, n_max=n_max)
    _BATCH = ((name, n_max), [{'ArcInput': e} for e in es])
  return _BATCH[1]


def make_edges(name: str) -> np.ndarray:
  from srdatalog_b200 import workloads as W
  cache = os.path.join('/tmp', f'srdl_bench_{name}.npy')
  if os.path.exists(cache):
    return np.load(cache)
  e = {'triangle': lambda: W.rmat_edges(20, 1 << 24, seed=3),
       'tc': lambda: W.tc_small(1),
       'sg': lambda: W.sg_forest(10000, seed=2)}[name]()
  try:
    np.save(cache, e)
  except OSError:
    pass
  return e


def load_plan(name: str) -> dict:
  with open(os.path.join(REPO, 'tests', 'golden', 'plans', f'{name}.json')) as f:
    return json.load(f)


def result_units(db, wl) -> int:
  return db.count(wl['out']) if wl['kind'] == 'count' else db.size(wl['out'])


def plain_loop(plan, insts, stride, stream_ptr, device):
  """The one-query-at-a-time loop: every sampled instance through its own
  srdl_run on one handle (host rows, result size read back).  Returns the
  rate, and per sampled instance its Path size and recursive iterations."""
  import torch
  from srdatalog_b200 import Database
  db = Database(plan, device=device)
  db.set_stream(stream_ptr)
  sample = insts[::stride]
  for inst in sample[:4]:  # warm-up
    db.clear_inputs()
    db.load_rows('ArcInput', inst['ArcInput'])
    db.run()
  torch.cuda.synchronize()
  t0 = time.perf_counter()
  sizes, iters = [], []
  for inst in sample:
    db.clear_inputs()
    db.load_rows('ArcInput', inst['ArcInput'])
    db.run()
    sizes.append(db.size('Path'))
    iters.append([st['iterations'] for st in db.stats()['steps'] if st['recursive']])
  dt = time.perf_counter() - t0
  db.close()
  return {'queries_per_s': len(sample) / dt, 'ms_per_query': 1e3 * dt / len(sample),
          'sample': f'every {stride}th of {len(insts)} instances ({len(sample)})'}, sizes, iters


class ClockSampler:
  '''nvidia-smi clocks + throttle reasons sampled during the timed region.'''

  FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
            'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
            'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

  def __init__(self, gpu_index: int):
    self.gpu = gpu_index
    self.proc = None
    self.lines: list[str] = []

  def start(self):
    try:
      self.proc = subprocess.Popen(['nvidia-smi', f'--query-gpu={self.FIELDS}', '--format=csv,noheader,nounits',
                                    '-i', str(self.gpu), '-lms', '200'], stdout=subprocess.PIPE,
                                   stderr=subprocess.DEVNULL, text=True)
      self.t = threading.Thread(target=self._read, daemon=True)
      self.t.start()
    except (OSError, FileNotFoundError):
      self.proc = None

  def _read(self):
    for line in self.proc.stdout:
      self.lines.append(line.strip())

  def stop(self) -> dict:
    if not self.proc:
      return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
    time.sleep(0.25)
    self.proc.terminate()
    try:
      self.proc.wait(timeout=5)
    except subprocess.TimeoutExpired:
      self.proc.kill()
    sm, mx, reasons = [], None, set()
    names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
    for ln in self.lines:
      f = [x.strip() for x in ln.split(',')]
      if len(f) < 9:
        continue
      try:
        sm.append(float(f[1]))
        mx = float(f[2])
      except ValueError:
        continue
      for nm, v in zip(names, f[5:9]):
        if v.lower() == 'active':
          reasons.add(nm)
    return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': mx,
            'samples': len(sm), 'reasons': sorted(reasons)}


def max_over_ranks(x: float, dist, device) -> float:
  '''The largest x over all ranks (every rank gets it); x itself on one rank.'''
  if dist is None:
    return x
  import torch
  t = torch.tensor([x], dtype=torch.float64, device=device)
  dist.all_reduce(t, op=dist.ReduceOp.MAX)
  return float(t.item())


def sum_over_ranks(x: int, dist, device) -> int:
  '''The sum of an integer over all ranks (every rank gets it); x itself on one rank.'''
  if dist is None:
    return x
  import torch
  t = torch.tensor([x], dtype=torch.int64, device=device)
  dist.all_reduce(t, op=dist.ReduceOp.SUM)
  return int(t.item())


def replica_throughput(units_per_step: float, steps: int, world: int, max_ms: float) -> float:
  '''Whole-job rate of `world` independent replicas, each doing units_per_step
  per step for `steps` steps, timed by the slowest rank (max_ms in total).'''
  return units_per_step * steps * world / (max_ms / 1e3)


def hbm_peak():
  try:
    with open(PEAKS_PATH) as f:
      return float(json.load(f)['hbm_gbs']), 'measured'
  except (OSError, KeyError, ValueError):
    return FALLBACK_HBM_GBS, 'fallback'


def cpu_baseline(wl_name: str, edges, n_max: int = WIDE_N_MAX) -> dict:
  '''The oracle (CPU restatement of the reference's evaluation) on the host
  cores, on a bounded sample; returns tuples/s for the same metric.'''
  import oracle
  cores = oracle.num_threads()
  if wl_name == 'served':
    reqs = serve_requests(serve_pool(), 64, seed=11)
    fn = {'tc': oracle.tc, 'sg': oracle.sg}
    t0 = time.perf_counter()
    for r in reqs:
      e = list(r.inputs.values())[0]
      if r.program == 'triangle':
        oracle.triangle_count(e)
      else:
        fn[r.program](e)
    dt = time.perf_counter() - t0
    return {'value': len(reqs) / dt, 'unit': 'queries/s', 'cores': cores, 'kind': 'port',
            'sample': f'first 64 requests of the served stream, one at a time ({dt:.2f} s)'}
  if wl_name in ('batched', 'batched-wide'):
    # every 16th instance in order (sizes are drawn independently of the
    # order), stopped after 20 s of CPU work
    insts = make_batch(wl_name, n_max)
    sample = insts[::PLAIN_SAMPLE_STRIDE]
    t0 = time.perf_counter()
    done = 0
    for inst in sample:
      oracle.tc(inst['ArcInput'])
      done += 1
      if time.perf_counter() - t0 > 20.0:
        break
    dt = time.perf_counter() - t0
    return {'value': done / dt, 'unit': 'queries/s', 'cores': cores, 'kind': 'port',
            'sample': f'TC of the first {done} of every {PLAIN_SAMPLE_STRIDE}th instance '
                      f'({len(sample)}), {dt:.2f} s'}
  if wl_name == 'triangle':
    t0 = time.perf_counter()
    c = oracle.triangle_count(edges)
    dt = time.perf_counter() - t0
    value = c / dt
    sample = (f'full workload: index build + join over all {edges.shape[0]} edges '
              f'({dt:.2f} s, {c} triangles)')
  else:
    t0 = time.perf_counter()
    if wl_name == 'tc':
      keys, _, _ = oracle.tc(edges)
    else:
      keys, _, _ = oracle.sg(edges)
    dt = time.perf_counter() - t0
    value = keys.shape[0] / dt
    sample = f'full fixpoint ({dt:.2f} s, {keys.shape[0]} tuples)'
  return {'value': value, 'unit': 'tuples/s', 'cores': cores, 'kind': 'port', 'sample': sample,
          'seconds': dt}


def run_reference(args, rank, world):
  wl = WORKLOADS.get(args.workload, {'desc': SERVE_DESC})
  if rank != 0:
    return
  if args.workload == 'batched-wide':
    wl = dict(wl, desc=wl['desc'].format(n_max=args.batch_n_max))
  edges = None if args.workload in ('served', 'batched', 'batched-wide') else make_edges(args.workload)
  vals, secs = [], []
  for i in range(args.warmup + args.steps):
    cb = cpu_baseline(args.workload, edges, args.batch_n_max)
    if i >= args.warmup:
      vals.append(cb['value'])
      if 'seconds' in cb:  # a step is one whole run (triangle, tc, sg)
        secs.append(cb.pop('seconds'))
  v = statistics.median(vals)
  cb['value'] = v
  cb.pop('seconds', None)
  unit = cb['unit']
  line = {'impl': 'reference', 'metric': f'{unit} ({args.workload})', 'value': v,
          'unit': unit, 'n_gpus': world, 'steps': args.steps, 'warmup': args.warmup,
          'ms_per_step': statistics.median(secs) * 1e3 if secs else None,
          'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
          'dtype': 'u32', 'data': 'synthetic',
          'config': {'workload': wl['desc']}, 'cpu_baseline': cb,
          'e2e': {'value': v, 'unit': unit, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
  print(json.dumps(line), flush=True)


SERVE_MIX = (('tc', 0.5), ('sg', 0.3), ('triangle', 0.2))
SERVE_POOL = 48          # distinct inputs per program; requests draw from them
SERVE_REQUESTS = 512
SERVE_DESC = ('served queries: Poisson arrivals, 50% TC / 30% SG / 20% triangle count, input '
              'edges log-uniform in [1e3, 4e6] (TC subcritical n=2m, SG forest n<=5,000, '
              'triangle R-MAT), 120 GB admission budget (runs held to their reservations), '
              '8 workers, continuous batching')


def serve_pool():
  '''SERVE_POOL seeded inputs per program with log-uniform sizes (cached).'''
  from srdatalog_b200 import workloads as W
  from srdatalog_b200.serve import log_uniform_sizes
  pool = {}
  for k, (prog, _) in enumerate(SERVE_MIX):
    cache = os.path.join('/tmp', f'srdl_serve_{prog}.npz')
    if os.path.exists(cache):
      z = np.load(cache)
      pool[prog] = [z[f'a{i}'] for i in range(SERVE_POOL)]
      continue
    sizes = log_uniform_sizes(SERVE_POOL, 1e3, 4e6, seed=50 + k)
    pool[prog] = [list(W.served_request_input(prog, int(m), 700 + 97 * k + i).values())[0]
                  for i, m in enumerate(sizes)]
    try:
      np.savez(cache, **{f'a{i}': a for i, a in enumerate(pool[prog])})
    except OSError:
      pass
  return pool


def serve_requests(pool, n, seed):
  from srdatalog_b200.serve import Request
  rel = {'tc': 'ArcInput', 'sg': 'Arc', 'triangle': 'KnowsInput'}
  rng = np.random.Generator(np.random.PCG64(seed))
  progs = rng.choice([p for p, _ in SERVE_MIX], size=n, p=[w for _, w in SERVE_MIX])
  picks = rng.integers(0, SERVE_POOL, n)
  return [Request(i, str(p), {rel[str(p)]: pool[str(p)][int(j)]}) for i, (p, j) in
          enumerate(zip(progs, picks))]


def run_served(args, rank, world):
  '''Served queries: the batching server vs the plain one-at-a-time loop on
  the same seeded request stream.  One step = one replay of the stream.'''
  import torch
  from srdatalog_b200.serve import ProgramSpec, Server, poisson_arrivals, replay
  if world > 1 and rank != 0:
    return
  progs = {'tc': ProgramSpec(load_plan('tc_lsm'), 'Path'), 'sg': ProgramSpec(load_plan('sg'), 'Sg'),
           'triangle': ProgramSpec(load_plan('triangle'), 'TriangleJoin', count_only=True)}
  pool = serve_pool()
  rate = args.rate
  offs = poisson_arrivals(SERVE_REQUESTS, rate, seed=5)
  torch.cuda.init()
  with Server(progs, workers=args.serve_workers, budget_bytes=120 << 30,
              batch_max_edges=args.batch_max_edges, max_batch=args.serve_max_batch) as srv:
    for w in range(args.warmup):  # warm-up replays (handles, pools, caches)
      replay(srv, serve_requests(pool, 64, seed=900 + w), poisson_arrivals(64, rate, seed=w))
    results, sums = None, []
    for s in range(args.steps):
      reqs = serve_requests(pool, SERVE_REQUESTS, seed=11)
      st = replay(srv, reqs, offs)
      got = [r.result for r in reqs]
      assert results is None or got == results  # same answers every replay
      assert not any(r.error for r in reqs)
      results = got
      sums.append(st.summary())
    memory = {'budget_bytes': srv.budget, 'peak_in_use_bytes': srv.peak_in_use,
              'peak_reserved_bytes': srv.peak_reserved, 'runs_outgrowing_reservation': srv.retried,
              'requests_held_back': len(srv.held_back),
              'note': 'peak_in_use: device bytes all handles held and cached (libsrdl '
                      'srdl_mem_stats), sampled after every run'}
  h2d = sum(int(list(r.inputs.values())[0].nbytes) for r in serve_requests(pool, SERVE_REQUESTS, 11))
  with Server(progs, workers=1, batching=False) as plain_srv:
    reqs = serve_requests(pool, SERVE_REQUESTS, seed=11)
    pst = replay(plain_srv, reqs, offs).summary()
    assert [r.result for r in reqs] == results
  qps = statistics.median(s['queries_per_s'] for s in sums)
  line = {
    'metric': 'queries/s (served)', 'value': qps, 'unit': 'queries/s', 'n_gpus': 1,
    'steps': args.steps, 'warmup': args.warmup,
    'ms_per_step': statistics.median(s['wall_s'] for s in sums) * 1e3,
    'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'u32',
    'data': 'synthetic',
    'config': {'workload': SERVE_DESC, 'offered_rate': rate, 'requests_per_step': SERVE_REQUESTS,
               'workers': args.serve_workers, 'batch_max_edges': args.batch_max_edges,
               'max_batch': args.serve_max_batch},
    'latency_ms': {'p50': statistics.median(s['p50_ms'] for s in sums),
                   'p99': statistics.median(s['p99_ms'] for s in sums)},
    'mean_batch': statistics.median(s['mean_batch'] for s in sums),
    'plain_loop': pst, 'speedup_vs_plain_loop': qps / pst['queries_per_s'],
    'memory': memory,
    'e2e': {'value': qps, 'unit': 'queries/s', 'h2d_bytes_per_step': h2d,
            'd2h_bytes_per_step': 8 * SERVE_REQUESTS,
            'note': 'every request is end to end: host rows in, its size/count read back'},
    'roofline': None,
  }
  print(json.dumps(line), flush=True)


def run_primitives(args, rank, world):
  '''The sort + unique, merge and set-difference primitives of libsrdl on
  --keys random (hi, lo) pairs with --bits-bit halves, built on the device.
  Each primitive runs --warmup times untimed, then --steps times between
  CUDA events on the current stream (median reported); one JSON line per
  primitive gives its time and algorithmic bandwidth (the bytes the
  operation must move at least) against the measured HBM peak:
    sort + unique of n keys: read the input, write the packed keys, read and
      write them once per counting pass, read them for the dedup and write
      the distinct keys;
    merge of two disjoint sorted arrays: 16 B per output key;
    set difference a - b: 8 B per key of a, b and the result.
  torch provides device buffers and the stream only.'''
  import ctypes

  import torch
  from srdatalog_b200 import native
  if rank != 0:
    return
  lib = native.lib()
  n, bits = args.keys, args.bits
  peak, peak_kind = hbm_peak()
  st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
  g = torch.Generator(device='cuda').manual_seed(1)
  hi = torch.randint(0, 1 << bits, (n,), device='cuda', dtype=torch.int64, generator=g)
  lo = torch.randint(0, 1 << bits, (n,), device='cuda', dtype=torch.int64, generator=g)
  keys = (hi << 32) | lo
  del hi, lo
  flush = torch.empty(64 << 20, dtype=torch.int32, device='cuda')  # 256 MB > 126 MB L2

  def timed(fn):
    for _ in range(args.warmup):
      fn()
    ms = []
    for i in range(args.steps):
      flush.fill_(i)
      e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
      e0.record()
      fn()
      e1.record()
      e1.synchronize()
      ms.append(e0.elapsed_time(e1))
    return statistics.median(ms)

  def report(name, ms, alg_bytes, **extra):
    gbs = alg_bytes / ms / 1e6
    print(json.dumps({'primitive': name, 'ms': round(ms, 4), 'alg_gbs': round(gbs, 1),
                      'frac_of_peak': round(gbs / peak, 3), 'peak_gbs': peak,
                      'peak_source': peak_kind, 'steps': args.steps, **extra}), flush=True)

  out = torch.empty_like(keys)
  dn = torch.zeros(1, dtype=torch.int64, device='cuda')
  sb = lib.srdl_sort_unique_scratch_bytes(n, bits)
  scratch = torch.empty(sb, dtype=torch.uint8, device='cuda')

  def sort():
    rc = lib.srdl_sort_unique_u64(keys.data_ptr(), n, bits, out.data_ptr(), dn.data_ptr(),
                                  scratch.data_ptr(), sb, st)
    assert rc == 0, native.last_error()

  ms = timed(sort)
  u = int(dn.item())
  # packed key width k and the passes the library runs: read the input
  # (8 B), write packed keys (k), P passes reading and writing k each, read
  # the sorted keys once more (k) and write the distinct ones (8 B)
  k = 4 if 2 * bits <= 32 else 8
  passes = (2 * bits + 7) // 8  # the library's default widest digit is 8 bits
  alg = n * (8 + k + passes * 2 * k + k) + 8 * u
  report('sort_unique', ms, alg, keys=n, unique=u, value_bits=bits, passes=passes,
         io_gbs=round(16 * n / ms / 1e6, 1))
  del scratch

  a = out[0:u:2].contiguous()
  b = out[1:u:2].contiguous()
  m = torch.empty(a.numel() + b.numel(), dtype=torch.int64, device='cuda')

  def merge():
    rc = lib.srdl_merge_u64(a.data_ptr(), a.numel(), b.data_ptr(), b.numel(), m.data_ptr(), st)
    assert rc == 0, native.last_error()

  report('merge', timed(merge), 16 * m.numel(), keys=m.numel())
  del a, b, m

  sub = out[0:u:3].contiguous()
  d = torch.empty(u, dtype=torch.int64, device='cuda')
  dn2 = torch.zeros(1, dtype=torch.int64, device='cuda')
  sb2 = lib.srdl_set_difference_scratch_bytes(u)
  scratch2 = torch.empty(sb2, dtype=torch.uint8, device='cuda')

  def diff():
    rc = lib.srdl_set_difference_u64(out.data_ptr(), u, sub.data_ptr(), sub.numel(), d.data_ptr(),
                                     dn2.data_ptr(), scratch2.data_ptr(), sb2, st)
    assert rc == 0, native.last_error()

  ms = timed(diff)
  nd = int(dn2.item())
  report('set_difference', ms, 8 * (u + sub.numel() + nd), a=u, b=sub.numel(), result=nd)


def run_batched(args, rank, world):
  """Batched fixpoints: every instance of the workload per step, in
  disjoint-union waves (srdatalog_b200.batch.WaveRun) under a device-memory
  budget; queries/s against the one-query-at-a-time loop.  Every step
  reads back each instance's Path size (checked against the plain loop on
  a sample, iterations too).  N > 1: independent replicas (the instances
  of a batch share nothing; no collective on the data path)."""
  import torch
  dist = None
  if world > 1:
    import datetime

    import torch.distributed as dist
    torch.cuda.set_device(local_of(world))
    dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300))
  local = local_of(world)
  dev = torch.device('cuda', local)
  torch.cuda.set_device(dev)
  from srdatalog_b200 import Database, native
  from srdatalog_b200.batch import WaveRun, make_union
  wl = dict(WORKLOADS[args.workload])
  if args.workload == 'batched-wide':
    wl['desc'] = wl['desc'].format(n_max=args.batch_n_max)
  plan = load_plan(wl['plan'])
  plain_plan = plan  # the one-query-at-a-time loop runs the plan as given
  insts = make_batch(args.workload, args.batch_n_max)
  k = len(insts)
  stream = torch.cuda.current_stream(dev)
  budget = int(args.batch_budget_gb * 1e9)
  tuned = None
  if wl.get('tune'):
    # untimed: the autotuner times candidate settings on the union of all
    # instances when they fit one run, else of the first instances whose
    # closures (at most n^2 tuples each) add up to 1e9 (about one wave)
    from srdatalog_b200.autotune import autotune
    sample, tot = [], 0
    for inst in insts:
      n = int(inst[wl['rel']].max()) + 1
      if args.workload != 'batched' and sample and tot + n * n > 1e9:
        break
      sample.append(inst)
      tot += n * n
    tuned = autotune(plan, {wl['rel']: make_union(sample).inputs[wl['rel']]}, device=local, reps=2)
    plan = tuned.apply(plan)
  db = Database(plan, device=local)
  if tuned:
    tuned.configure(db)
  db.set_stream(stream.cuda_stream)
  db.set_profiling(True)
  wr = WaveRun(plan, insts, db=db, budget_bytes=budget, sizes=[wl['out']])
  kernels: dict = {}
  collect = [False]

  def on_wave(d):
    if collect[0]:
      for name, st in d.stats()['kernels'].items():
        agg = kernels.setdefault(name, {'ms': 0.0, 'bytes': 0.0, 'units': 0.0, 'scopes': 0})
        for f in agg:
          agg[f] += st[f]

  # first run from host rows settles the wave partition (splits if a wave
  # outgrows the budget); then every wave's union is staged on the device
  wr.run(on_wave=on_wave)
  assert not wr.errors, wr.errors
  unions = {tuple(w): make_union([insts[j] for j in w]) for w in wr.waves}
  d_rows = {key: torch.from_numpy(u.inputs[wl['rel']].view(np.int32).reshape(-1)).to(dev)
            for key, u in unions.items()}
  rows_of = {id(u): d_rows[key] for key, u in unions.items()}

  def union_of(wave):
    return unions[tuple(wave)]

  def load_dev(d, u):
    t = rows_of[id(u)]
    d.load_device_rows(wl['rel'], t.data_ptr(), t.numel() // 2)

  flush = torch.empty(64 << 20, dtype=torch.int32, device=dev)  # 256 MB > 126 MB L2
  for _ in range(args.warmup):
    wr.run(union_of=union_of, load=load_dev, on_wave=on_wave)
  want = wr.sizes[wl['out']].copy()
  want_iters = {s: v.copy() for s, v in wr.iterations.items()}
  waves_before = len(wr.waves)

  def timed(load, tag):
    ms = []
    l0 = native.lib().srdl_launch_count()
    for i in range(args.steps):
      flush.fill_(i)
      e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
      e0.record(stream)
      wr.run(union_of=union_of, load=load, on_wave=on_wave)
      e1.record(stream)
      e1.synchronize()
      ms.append(e0.elapsed_time(e1))
      assert not wr.errors and len(wr.waves) == waves_before, tag
      assert np.array_equal(wr.sizes[wl['out']], want), tag
    return ms, native.lib().srdl_launch_count() - l0

  if dist:
    dist.barrier()
  torch.cuda.synchronize(dev)
  sampler = ClockSampler(local)
  sampler.start()
  collect[0] = True
  step_ms, launches = timed(load_dev, 'device rows')
  collect[0] = False
  torch.cuda.synchronize(dev)
  clocks = sampler.stop()
  total_ms = max_over_ranks(sum(step_ms), dist, dev)
  value = replica_throughput(k, args.steps, world, total_ms)
  tuples = float(want.astype(np.float64).sum())

  # e2e: the same waves from host rows (copied in every step), sizes read back
  if dist:
    dist.barrier()
  e2e_ms, _ = timed(None, 'host rows')
  e2e_total = max_over_ranks(sum(e2e_ms), dist, dev)
  h2d = int(sum(u.inputs[wl['rel']].nbytes for u in unions.values()))
  plain = None
  if not args.no_cpu_baseline:
    plain, sizes, iters = plain_loop(plain_plan, insts, PLAIN_SAMPLE_STRIDE, stream.cuda_stream, local)
    assert [int(x) for x in want[::PLAIN_SAMPLE_STRIDE]] == sizes
    rec = sorted(want_iters)
    assert all([int(want_iters[s][j]) for s in rec] == it
               for j, it in zip(range(0, k, PLAIN_SAMPLE_STRIDE), iters)), 'iterations differ'
  stats = db.stats()
  db.close()
  if dist:
    dist.barrier()
    dist.destroy_process_group()
  if rank != 0:
    return
  top = max(kernels.items(), key=lambda kv: kv[1]['ms'])
  name, kk = top
  peak, peak_kind = hbm_peak()
  achieved = (kk['bytes'] / (kk['ms'] / 1e3)) / 1e9 if kk['ms'] else 0.0
  roof = {'bound': 'hbm', 'kernel': name, 'achieved': achieved, 'peak': peak,
          'peak_source': peak_kind, 'unit': 'GB/s', 'frac': achieved / peak,
          'traffic': None, 'traffic_source': None,
          'bytes_per_launch': kk['bytes'] / max(1, kk['scopes']),
          'ms_per_launch': kk['ms'] / max(1, kk['scopes']),
          'share_of_step': kk['ms'] / total_ms if world == 1 else None}
  line = {
    'metric': f'queries/s ({args.workload})', 'value': value, 'unit': 'queries/s', 'n_gpus': world,
    'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': total_ms / args.steps,
    'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'u32',
    'data': 'synthetic',
    'config': {'workload': wl['desc'], 'instances': k,
               'edges': int(sum(i['ArcInput'].shape[0] for i in insts)),
               'path_tuples_per_step': int(tuples),
               'tuples_per_s': tuples * args.steps * world / (total_ms / 1e3),
               'waves': len(wr.waves), 'wave_splits': wr.splits,
               'budget_bytes': budget, 'peak_bytes': wr.peak_bytes,
               'bytes_per_bound_tuple': wr.bytes_per_bound,
               'device_loop': stats.get('device_loop'),
               'parallelism': f'replicas{world}',
               'l2': 'flushed between steps (256 MB write)',
               'inputs': 'HBM-resident for value; host rows for e2e'},
    'e2e': {'value': replica_throughput(k, args.steps, world, e2e_total), 'unit': 'queries/s',
            'ms_per_step': e2e_total / args.steps, 'h2d_bytes_per_step': h2d,
            'd2h_bytes_per_step': 8 * k, 'step_ms': [round(x, 3) for x in e2e_ms]},
    'step_ms': [round(x, 3) for x in step_ms],
    'gpu_launches': int(launches),
    'roofline': roof,
    'kernels': {k2: {'ms_per_step': v['ms'] / args.steps,
                     'gbs': (v['bytes'] / (v['ms'] / 1e3) / 1e9) if v['ms'] else 0.0}
                for k2, v in sorted(kernels.items(), key=lambda kv: -kv[1]['ms'])},
    'clocks': clocks,
  }
  if tuned:
    line['config']['autotuned'] = dict(tuned.to_json(), trials=len(tuned.trials))
  if plain:
    line['plain_loop'] = plain
    line['speedup_vs_plain_loop'] = value / plain['queries_per_s']
  if world == 1 and not args.no_cpu_baseline:
    line['cpu_baseline'] = cpu_baseline(args.workload, None, args.batch_n_max)
  print(json.dumps(line), flush=True)


def local_of(world: int) -> int:
  import torch
  return int(os.environ.get('LOCAL_RANK', '0')) % max(1, torch.cuda.device_count())


def main():
  ap = argparse.ArgumentParser()
  ap.add_argument('--gpus', type=int, default=1)
  ap.add_argument('--steps', type=int, default=10)
  ap.add_argument('--warmup', type=int, default=3)
  ap.add_argument('--impl', default='srdl', choices=['srdl', 'reference'])
  ap.add_argument('--workload', default='triangle',
                  choices=sorted(WORKLOADS) + ['served', 'primitives'])
  ap.add_argument('--keys', type=int, default=200_000_000, help='primitives: keys')
  ap.add_argument('--bits', type=int, default=21, help='primitives: bits per key half')
  ap.add_argument('--rate', type=float, default=2000.0, help='served: offered load (req/s)')
  ap.add_argument('--serve-workers', type=int, default=8, help='served: concurrent workers')
  ap.add_argument('--batch-max-edges', type=int, default=1 << 20,
                  help='served: largest request (input edges) that is unioned with others')
  ap.add_argument('--serve-max-batch', type=int, default=16,
                  help='served: most requests evaluated as one union')
  ap.add_argument('--batch-n-max', type=int, default=WIDE_N_MAX,
                  help='batched-wide: the config instances with at most this many nodes')
  ap.add_argument('--batch-budget-gb', type=float, default=120.0,
                  help='batched: device memory one wave may hold')
  ap.add_argument('--no-cpu-baseline', action='store_true')
  ap.add_argument('--quick', action='store_true',
                  help='kernel-resident path only (no e2e, no CPU baseline): for profiler runs')
  args = ap.parse_args()
  args.warmup = max(args.warmup, 3)

  rank = int(os.environ.get('RANK', '0'))
  world = int(os.environ.get('WORLD_SIZE', '1'))
  local = int(os.environ.get('LOCAL_RANK', '0'))
  if args.impl == 'reference':
    return run_reference(args, rank, world)
  if args.workload == 'served':
    return run_served(args, rank, world)
  if args.workload == 'primitives':
    return run_primitives(args, rank, world)
  if WORKLOADS[args.workload]['kind'] == 'batched':
    return run_batched(args, rank, world)

  import torch
  dist = None
  # SRDL_BENCH_BACKEND=gloo runs the collectives on the host (several ranks
  # can then share one GPU to exercise the N > 1 path; their kernels never
  # wait on one another); timings are only meaningful with nccl.
  backend = os.environ.get('SRDL_BENCH_BACKEND', 'nccl')
  local = local % max(1, torch.cuda.device_count())
  if world > 1:
    import datetime

    import torch.distributed as dist
    torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
  dev = torch.device('cuda', local)
  coll = dev if backend == 'nccl' else torch.device('cpu')  # where collective tensors live
  torch.cuda.set_device(dev)

  from srdatalog_b200 import Database, native
  from srdatalog_b200.shard import TorchExchange, shard_plan
  wl = WORKLOADS[args.workload]
  plan = load_plan(wl['plan'])
  edges = make_edges(args.workload)
  n = edges.shape[0]
  tuned = None
  if wl.get('tune'):
    # untimed: the autotuner times candidate settings on this very input
    from srdatalog_b200.autotune import autotune
    tuned = autotune(plan, {wl['rel']: edges}, device=local, reps=2)
    plan = tuned.apply(plan)
  # N > 1: shard the one program over the ranks when its plan allows it
  spec = shard_plan(plan) if world > 1 else None
  sharded = bool(spec and spec.useful)
  if sharded:
    plan = spec.plan
  # plans whose recursive rules derive other shards' tuples send them there
  # every iteration (all_to_all over the process group)
  xch = TorchExchange() if sharded and spec.exchanged else None
  stream = torch.cuda.current_stream(dev)

  def open_db():
    d = Database(plan, device=local)
    if tuned:
      tuned.configure(d)
    if sharded:
      d.set_option('shard_world', world)
      d.set_option('shard_rank', rank)
      if xch:
        d.set_exchange(xch.callback(rank))
    d.set_stream(stream.cuda_stream)
    return d

  def job_units(d) -> int:
    # the job's result: a sharded relation's or count's parts add up
    u = result_units(d, wl)
    return sum_over_ranks(u, dist, coll) if sharded else u

  # ---------------- kernel-resident path (value)
  d_edges = torch.from_numpy(edges.view(np.int32).reshape(-1)).to(dev)
  db = open_db()
  db.load_device_rows(wl['rel'], d_edges.data_ptr(), n)
  db.set_profiling(True)
  flush = torch.empty(64 << 20, dtype=torch.int32, device=dev)  # 256 MB > 126 MB L2
  for _ in range(args.warmup):
    db.run()
    job_units(db)
  units = job_units(db)
  per_step = units
  metric_name = f'tuples/s ({args.workload})'
  unit_name = 'tuples/s'
  kernels: dict = {}
  step_ms = []
  launches = 0
  sampler = ClockSampler(local)
  if dist:
    dist.barrier()
  torch.cuda.synchronize(dev)
  sampler.start()
  for i in range(args.steps):
    flush.fill_(i)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = native.lib().srdl_launch_count()
    ev0.record(stream)
    db.run()
    got = job_units(db) if sharded else units  # sharded: the final all-reduce is timed
    ev1.record(stream)
    ev1.synchronize()
    launches += native.lib().srdl_launch_count() - l0
    step_ms.append(ev0.elapsed_time(ev1))
    for k, s in db.stats()['kernels'].items():
      agg = kernels.setdefault(k, {'ms': 0.0, 'bytes': 0.0, 'units': 0.0, 'scopes': 0})
      for f in agg:
        agg[f] += s[f]
    assert got == units and (sharded or result_units(db, wl) == units)
  torch.cuda.synchronize(dev)
  clocks = sampler.stop()
  if dist:
    dist.barrier()
  total_ms = sum(step_ms)
  total_ms = max_over_ranks(total_ms, dist, coll)
  # sharded: per_step is already the whole job's; replicas: one per rank
  copies = 1 if sharded else world
  value = replica_throughput(per_step, args.steps, copies, total_ms)
  stats = db.stats()
  db.close()
  del d_edges

  # ---------------- end-to-end path through the C ABI with host inputs (e2e)
  if args.quick:
    if dist:
      dist.destroy_process_group()
    if rank == 0:
      print(json.dumps({'metric': metric_name, 'value': value,
                        'ms_per_step': total_ms / args.steps, 'quick': True,
                        'step_ms': [round(x, 3) for x in step_ms]}), flush=True)
    return
  db2 = open_db()
  db2.load_rows(wl['rel'], edges)
  for _ in range(args.warmup):
    db2.run()
    job_units(db2)
  e2e_ms = []
  if dist:
    dist.barrier()
  torch.cuda.synchronize(dev)
  for i in range(args.steps):
    flush.fill_(i)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    db2.run()
    got = job_units(db2)  # result read back to the host (summed over shards)
    ev1.record(stream)
    ev1.synchronize()
    e2e_ms.append(ev0.elapsed_time(ev1))
    assert got == units
  e2e_total = sum(e2e_ms)
  e2e_total = max_over_ranks(e2e_total, dist, coll)
  db2.close()
  if dist:
    dist.barrier()
    dist.destroy_process_group()
  if rank != 0:
    return

  # ---------------- roofline of the dominant kernel family
  top = max(kernels.items(), key=lambda kv: kv[1]['ms'])
  name, k = top
  peak, peak_kind = hbm_peak()
  achieved = (k['bytes'] / (k['ms'] / 1e3)) / 1e9 if k['ms'] else 0.0
  # DRAM bytes per launch from an ncu capture of this workload's dominant
  # kernel (profiles/traffic.json: read + write bytes and the units that
  # capture processed, scaled to this run's units per launch)
  traffic, traffic_src = None, None
  prof = os.path.join(REPO, 'profiles', 'traffic.json')
  if os.path.exists(prof):
    with open(prof) as f:
      tr = json.load(f).get(args.workload, {}).get(name)
    if tr:
      traffic = tr['dram_bytes'] / tr['units'] * k['units'] / max(1, k['scopes'])
      traffic_src = tr['source']
  roof = {'bound': 'hbm', 'kernel': name, 'achieved': achieved, 'peak': peak,
          'peak_source': peak_kind, 'unit': 'GB/s', 'frac': achieved / peak,
          'traffic': traffic, 'traffic_source': traffic_src,
          'bytes_per_launch': k['bytes'] / max(1, k['scopes']),
          'ms_per_launch': k['ms'] / max(1, k['scopes']),
          'share_of_step': k['ms'] / total_ms if world == 1 else None}
  line = {
    'metric': metric_name, 'value': value, 'unit': unit_name, 'n_gpus': world,
    'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': total_ms / args.steps,
    'higher_is_better': True, 'scaling': 'strong' if sharded else 'weak', 'vs_baseline': None,
    'dtype': 'u32',
    'data': 'synthetic',
    'config': {'workload': wl['desc'], 'edges': int(n), 'tuples_per_step': int(units),
               'parallelism': f'shards{world}' if sharded else f'replicas{world}',
               'l2': 'flushed between steps (256 MB write)',
               'inputs': 'HBM-resident for value; pinned host rows for e2e'},
    'e2e': {'value': replica_throughput(per_step, args.steps, copies, e2e_total), 'unit': unit_name,
            'ms_per_step': e2e_total / args.steps, 'h2d_bytes_per_step': int(n) * 8,
            'd2h_bytes_per_step': 8,
            'step_ms': [round(x, 3) for x in e2e_ms]},
    'step_ms': [round(x, 3) for x in step_ms],
    'gpu_launches': int(launches),
    'roofline': roof,
    'kernels': {k2: {'ms_per_step': v['ms'] / args.steps,
                     'gbs': (v['bytes'] / (v['ms'] / 1e3) / 1e9) if v['ms'] else 0.0}
                for k2, v in sorted(kernels.items(), key=lambda kv: -kv[1]['ms'])},
    'iterations': [s['iterations'] for s in stats['steps']],
    'clocks': clocks,
  }
  if sharded:
    line['config']['sharding'] = {'partitioned': spec.partitioned,
                                  'rules': {r: m for r, m in spec.modes.items() if m},
                                  'inputs': 'replicated on every rank'}
  elif world > 1 and spec is not None:
    line['config']['sharding'] = {'replicas': spec.fallback or 'nothing to split'}
  if tuned:
    line['config']['autotuned'] = dict(tuned.to_json(), trials=len(tuned.trials))
  if world == 1 and not args.no_cpu_baseline:
    line['cpu_baseline'] = cpu_baseline(args.workload, edges)
    line['cpu_baseline'].pop('seconds', None)
  print(json.dumps(line), flush=True)


if __name__ == '__main__':
  main()
