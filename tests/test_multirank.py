'''The bench's N>1 path on CPU: two gloo ranks, the job is timed by the
slowest rank, the whole-job rate counts every rank's units (replicas) and a
sharded job's result is the sum of its parts.'''

import os
import socket

import pytest

torch = pytest.importorskip('torch')
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
  with socket.socket() as s:
    s.bind(('127.0.0.1', 0))
    return s.getsockname()[1]


def _rank_main(rank, world, port, out):
  import sys
  repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
  sys.path.insert(0, repo)
  import bench
  os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
  dist.init_process_group('gloo', rank=rank, world_size=world)
  try:
    dist.barrier()
    my_ms = 100.0 + 50.0 * rank           # rank 1 is the slow one
    total = bench.max_over_ranks(my_ms, dist, 'cpu')
    rate = bench.replica_throughput(1000, 4, world, total)
    units = bench.sum_over_ranks(1000 + rank, dist, 'cpu')   # a sharded job's parts
    dist.barrier()
    out.put((rank, total, rate, units))
  finally:
    dist.destroy_process_group()


def test_two_rank_replicas_max_timing():
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
  assert [r[1] for r in res] == [150.0, 150.0]          # every rank sees the max
  assert res[0][2] == res[1][2] == pytest.approx(1000 * 4 * 2 / 0.150)
  assert [r[3] for r in res] == [2001, 2001]            # and the sum of the parts


def test_single_rank_is_identity():
  import bench
  assert bench.max_over_ranks(12.5, None, 'cpu') == 12.5
  assert bench.sum_over_ranks(7, None, 'cpu') == 7
  assert bench.replica_throughput(10, 2, 1, 1000.0) == pytest.approx(20.0)
