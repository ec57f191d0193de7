'''Sharding host logic on CPU: the ownership function, the plan analysis
that marks rules for sharded evaluation, result combination, and the final
sum over two gloo ranks.'''

import ctypes
import os
import socket

import numpy as np
import pytest
from conftest import load_plan
from srdatalog_b200.shard import (ShardError, ShardSpec, allreduce_results, combine_dumps,
                                  combine_sizes, owner, shard_plan, shard_rows)

PLANS = ['andersen', 'cspa', 'lsqb_q6', 'lsqb_q7', 'reach_avoid', 'sg', 'tc', 'tc_left',
         'tc_lsm', 'triangle']

# plan -> (partitioned relations, {rule: mode} for the marked rules, falls back,
#          relations exchanged between shards)
EXPECTED = {
  'andersen': ([], {}, True, []),
  'cspa': ([], {}, True, []),
  'lsqb_q6': ([], {'TwoHopPath': 'work'}, False, []),
  'lsqb_q7': ([], {'Case1Both': 'work', 'Case2ReplyOnly': 'work', 'Case3LikeOnly': 'work',
                   'Case4Neither': 'work'}, False, []),
  'reach_avoid': (['Reach', 'Cut'], {'ReachBase': 'key', 'CutPairs': 'key'}, False, []),
  'sg': (['Sg'], {'SGBase': 'key', 'SGRec_D1': 'exchange'}, False, ['Sg']),
  'tc': (['Path'], {'TCBase': 'key'}, False, []),
  'tc_left': (['Path'], {'TCBase': 'key', 'TCRecL_D1': 'exchange'}, False, ['Path']),
  'tc_lsm': (['Path'], {'TCBase': 'key'}, False, []),
  'triangle': ([], {'TriangleJoin': 'work'}, False, []),
}


def test_owner_matches_formula_and_spreads_keys():
  v = np.array([0, 1, 2, 12345, 0xFFFFFFFF], np.uint32)
  for world in (1, 2, 3, 8):
    want = [((int(x) * 0x9E3779B1) % (1 << 32)) * world >> 32 for x in v]
    assert owner(v, world).tolist() == want
  ids = np.arange(200_000, dtype=np.uint32)
  for world in (2, 3, 8):
    counts = np.bincount(owner(ids, world), minlength=world)
    assert counts.min() > 0.97 * ids.size / world and counts.max() < 1.03 * ids.size / world
  assert owner(ids, 1).max() == 0


@pytest.mark.parametrize('name', PLANS)
def test_shard_plan_marks(name):
  plan = load_plan(name)
  spec = shard_plan(plan)
  part, marks, falls_back, sent = EXPECTED[name]
  assert spec.partitioned == part
  assert {r: m for r, m in spec.modes.items() if m} == marks
  assert bool(spec.fallback) == falls_back
  assert spec.exchanged == sent
  assert sorted(spec.partitioned + spec.replicated) == sorted(r['name'] for r in plan['relations'])
  # the marks sit on the plan's rules; the input plan is left alone
  for st in spec.plan['steps']:
    for op in st['ops']:
      if op['op'] == 'execute_pipeline':
        assert op.get('shard', '') == marks.get(op['rule'], '')
        assert ('shard_var' in op) == (op.get('shard') == 'key')
  # an exchange op right before every rebuild of a relation an exchange rule derives
  for st in spec.plan['steps']:
    ops = st['ops']
    for i, op in enumerate(ops):
      if op['op'] == 'exchange':
        assert op['rel'] in sent
        assert ops[i + 1]['op'] == 'rebuild_index' and ops[i + 1]['rel'] == op['rel']
        assert any(o.get('shard') == 'exchange' for o in ops[:i] if o['op'] == 'execute_pipeline')
  assert 'shard' not in str(plan) and 'exchange' not in str(plan)


def test_key_mode_uses_head_key():
  spec = shard_plan(load_plan('tc'))
  op = next(op for st in spec.plan['steps'] for op in st['ops'] if op.get('rule') == 'TCBase')
  assert op['shard_var'] == 'x'


def test_join_across_keys_is_reported():
  spec = shard_plan(load_plan('andersen'))
  assert 'other shards' in spec.fallback and not spec.useful


def _host_copy(dst, src, nbytes, stream):
  ctypes.memmove(dst, src, nbytes)


def _exchange_round(ex, world, sends):
  '''Drives one exchange (phases 0, 1, 2) of `world` threads over host
  buffers: sends[r][d] = keys shard r sends to shard d.'''
  import threading
  out = [None] * world

  def work(r):
    fn = ex.callback(r)
    counts = (ctypes.c_uint64 * world)(*[len(sends[r][d]) for d in range(world)])
    fn(0, 'R', counts, 0, 0, 0)
    got = [counts[i] for i in range(world)]
    flat = [k for d in range(world) for k in sends[r][d]]
    sbuf = (ctypes.c_uint64 * max(1, len(flat)))(*flat)
    rbuf = (ctypes.c_uint64 * max(1, sum(got)))()
    fn(1, 'R', counts, ctypes.addressof(sbuf), ctypes.addressof(rbuf), 0)
    vote = (ctypes.c_uint64 * world)(len(flat))
    fn(2, '', vote, 0, 0, 0)
    out[r] = (got, list(rbuf)[:sum(got)], vote[0])

  ths = [threading.Thread(target=work, args=(r,)) for r in range(world)]
  for t in ths:
    t.start()
  for t in ths:
    t.join(timeout=60)
  return out


def test_local_exchange_moves_keys_to_owners():
  from srdatalog_b200.shard import LocalExchange
  world = 3
  sends = [[[100 * r + 10 * d + k for k in range(r + d)] for d in range(world)]
           for r in range(world)]
  out = _exchange_round(LocalExchange(world, timeout=30, copy=_host_copy), world, sends)
  total = sum(len(sends[r][d]) for r in range(world) for d in range(world))
  for d in range(world):
    got, keys, vote = out[d]
    assert got == [len(sends[s][d]) for s in range(world)]
    assert keys == [k for s in range(world) for k in sends[s][d]]  # grouped by source
    assert vote == total


def test_local_exchange_abort_releases_the_other_shards():
  '''A shard whose run fails aborts the exchange: the shards waiting in the
  barrier get an error at once instead of waiting for it.'''
  import threading
  import time
  from srdatalog_b200.shard import LocalExchange
  ex = LocalExchange(3, timeout=60, copy=_host_copy)
  errors = []

  def waiting(r):
    counts = (ctypes.c_uint64 * 3)(1, 1, 1)
    try:
      ex.callback(r)(0, 'R', counts, 0, 0, 0)
    except threading.BrokenBarrierError as e:
      errors.append(e)

  ths = [threading.Thread(target=waiting, args=(r,)) for r in (0, 1)]
  t0 = time.monotonic()
  for t in ths:
    t.start()
  time.sleep(0.2)
  ex.abort()  # shard 2 failed before reaching the exchange
  for t in ths:
    t.join(timeout=30)
  assert len(errors) == 2 and time.monotonic() - t0 < 30


def test_marked_plans_load_in_native_library():
  from srdatalog_b200 import native
  for name in PLANS:
    db = native.Database(shard_plan(load_plan(name)).plan)
    db.set_option('shard_world', 4)
    db.set_option('shard_rank', 3)
    with pytest.raises(Exception):
      db.set_option('shard_world', 0)
    db.close()
  bad = shard_plan(load_plan('triangle')).plan
  for st in bad['steps']:
    for op in st['ops']:
      if op['op'] == 'execute_pipeline':
        op['shard'] = 'bogus'
  with pytest.raises(Exception):
    native.Database(bad)


def test_shard_rows_partitions_rows():
  rows = np.array([[i, i + 1] for i in range(1000)], np.uint32)
  parts = [shard_rows(rows, 3, r) for r in range(3)]
  assert sum(p.shape[0] for p in parts) == 1000
  got = np.concatenate(parts)
  assert sorted(map(tuple, got.tolist())) == sorted(map(tuple, rows.tolist()))
  for r, p in enumerate(parts):
    assert np.all(owner(p[:, 0], 3) == r)
  assert shard_rows(np.zeros((0, 2), np.uint32), 3, 1).shape == (0, 2)


def test_combine_sizes_and_dumps():
  spec = ShardSpec(plan={}, partitioned=['P'], replicated=['E'])
  assert combine_sizes(spec, [{'P': 3, 'E': 7}, {'P': 4, 'E': 7}]) == {'P': 7, 'E': 7}
  with pytest.raises(AssertionError):
    combine_sizes(spec, [{'E': 7}, {'E': 8}])
  a = np.array([[5, 1], [9, 0]], np.uint32)
  b = np.array([[1, 2], [5, 0]], np.uint32)
  got = combine_dumps(spec, 'P', [a, b])
  assert got.tolist() == [[1, 2], [5, 0], [5, 1], [9, 0]]
  assert combine_dumps(spec, 'E', [a, a]) is a
  with pytest.raises(ShardError):
    raise ShardError('x')


def _free_port():
  with socket.socket() as s:
    s.bind(('127.0.0.1', 0))
    return s.getsockname()[1]


def _rank_main(rank, world, port, out):
  import sys
  repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
  sys.path[:0] = [os.path.join(repo, 'srdatalog-python_b200'), os.path.join(repo, 'tests')]
  import torch.distributed as dist
  from srdatalog_b200.shard import allreduce_results as ar
  os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
  dist.init_process_group('gloo', rank=rank, world_size=world)
  try:
    spec = ShardSpec(plan={}, partitioned=['Path'], replicated=['Edge'])
    sizes, counts = ar(spec, {'Path': 10 + rank, 'Edge': 99}, {'Tri': 1000 * (rank + 1)})
    out.put((rank, sizes, counts))
  finally:
    dist.destroy_process_group()


def _torch_exchange_rank(rank, world, port, out):
  import sys
  repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
  sys.path[:0] = [os.path.join(repo, 'srdatalog-python_b200'), os.path.join(repo, 'tests')]
  import torch.distributed as dist
  from srdatalog_b200.shard import TorchExchange
  os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
  dist.init_process_group('gloo', rank=rank, world_size=world)
  try:
    fn = TorchExchange(copy=lambda dst, src, n, s: ctypes.memmove(dst, src, n)).callback(rank)
    sends = [[7 * rank + d] * (rank + d + 1) for d in range(world)]
    counts = (ctypes.c_uint64 * world)(*[len(s) for s in sends])
    fn(0, 'R', counts, 0, 0, 0)
    got = [counts[i] for i in range(world)]
    flat = [k for s in sends for k in s]
    sbuf = (ctypes.c_uint64 * len(flat))(*flat)
    rbuf = (ctypes.c_uint64 * sum(got))()
    fn(1, 'R', counts, ctypes.addressof(sbuf), ctypes.addressof(rbuf), 0)
    vote = (ctypes.c_uint64 * world)(len(flat))
    fn(2, '', vote, 0, 0, 0)
    out.put((rank, got, list(rbuf), vote[0]))
  finally:
    dist.destroy_process_group()


def test_two_rank_torch_exchange():
  import torch.multiprocessing as mp
  ctx = mp.get_context('spawn')
  q = ctx.Queue()
  port = _free_port()
  world = 2
  procs = [ctx.Process(target=_torch_exchange_rank, args=(r, world, port, q)) for r in range(world)]
  for p in procs:
    p.start()
  res = sorted(q.get(timeout=120) for _ in procs)
  for p in procs:
    p.join(timeout=60)
    assert p.exitcode == 0
  total = sum(r + d + 1 for r in range(world) for d in range(world))
  for d, got, keys, vote in res:
    assert got == [s + d + 1 for s in range(world)]
    assert keys == [k for s in range(world) for k in [7 * s + d] * (s + d + 1)]
    assert vote == total


def test_two_rank_allreduce_of_results():
  import torch.multiprocessing as mp
  ctx = mp.get_context('spawn')
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
  for p in procs:
    p.start()
  res = sorted(q.get(timeout=120) for _ in procs)
  for p in procs:
    p.join(timeout=60)
    assert p.exitcode == 0
  for _, sizes, counts in res:
    assert sizes == {'Path': 21, 'Edge': 99}
    assert counts == {'Tri': 3000}
  assert allreduce_results is not None
