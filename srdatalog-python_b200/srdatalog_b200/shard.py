'''Sharding one program's evaluation over several databases, one per GPU.

Every shard holds the same input relations (replicated) and evaluates the
same plan; the derived relations of recursive strata are *partitioned* by
their first column: shard r keeps the tuples whose column-0 value v has
``owner(v, world) == r`` (a multiplicative hash; libsrdl's shard_owner is
the same function).  No tuple moves between shards during the fixpoint, so
the only collective is the final sum of sizes and counts.  This works when
every rule keeps the partition key in place:

* a rule whose head is partitioned and that reads partitioned relations must
  read all of them with the head's column-0 variable in their column 0 (TC:
  ``Path(x,z) <= Path(x,y), Edge(y,z)``) -- nothing to restrict, the delta
  it reads is already this shard's part;
* a rule whose head is partitioned and that reads only replicated relations
  keeps only the bindings whose key variable it owns (plan mark
  ``"shard": "key"``; TC's base rule);
* a count-only rule over replicated relations splits the work items of its
  last join level evenly over the shards (``"shard": "work"``: the triangle
  count); one over partitioned relations read on one shared column-0
  variable needs no restriction;
* a relation derived only from replicated relations, outside recursion,
  stays replicated (every shard computes it; cheap loads like TC's Edge).

* a rule whose positive partitioned atoms share one key variable other
  than the head's (same generation: ``SG(x,y) <= Edge(a,x), SG(a,b),
  Edge(b,y)`` reads SG keyed by a, derives keys x; left-recursive TC) has its
  bindings confined to this shard's keys but derives tuples for any shard:
  the plan gets an ``exchange`` op for the head relation before its NEW
  version is indexed, which sends every derived tuple to its owner (one
  all-to-all per iteration), and the fixpoint stops when every shard's
  delta is empty (one sum per iteration).  The exchange itself is a
  callback: ``LocalExchange`` for shards run by threads of one process,
  ``TorchExchange`` for one process per GPU under torch.distributed.

Plans in which one rule reads partitioned relations on two different keys
(Andersen's ``PointsTo(x,z), PointsTo(z,w)``) would need more than an
exchange of derived tuples; for those ``shard_plan`` falls back to
replicating every relation, and only count-only rules are split.  The
reference evaluates on one GPU (its multi-node MPI code is unused), so this
layer has no counterpart there; each shard's evaluation is the single-GPU
one.
'''

from __future__ import annotations

import copy
import ctypes
import threading
from dataclasses import dataclass, field

import numpy as np


class ShardError(ValueError):
  pass


def owner(values, world: int) -> np.ndarray:
  '''Shard owning each uint32 key value: (v * 0x9E3779B1 mod 2^32) * world >> 32.'''
  v = np.asarray(values, dtype=np.uint32).astype(np.uint64)
  h = (v * np.uint64(0x9E3779B1)) & np.uint64(0xFFFFFFFF)
  return ((h * np.uint64(world)) >> np.uint64(32)).astype(np.int64)


@dataclass
class ShardSpec:
  plan: dict                                  # the plan with per-rule shard marks
  partitioned: list = field(default_factory=list)  # relations split by column 0
  replicated: list = field(default_factory=list)
  modes: dict = field(default_factory=dict)   # rule -> 'work' | 'key' | 'exchange' | ''
  fallback: str = ''                          # why partitioning was given up, if it was
  exchanged: list = field(default_factory=list)  # relations sent between shards each iteration

  @property
  def useful(self) -> bool:
    '''True when some rule's work is divided among the shards.'''
    return any(self.modes.values()) or bool(self.partitioned)


def _rules(plan: dict):
  for si, st in enumerate(plan['steps']):
    for op in st['ops']:
      if op['op'] == 'execute_pipeline':
        yield si, st, op


def _insert(op: dict) -> dict:
  return next(p for p in op['pipeline'] if p['op'] == 'insert_into')


def _atoms(pipeline: list) -> list:
  '''The atom occurrences a pipeline reads: (rel, {column: var}, negated).
  The planner splits an atom over levels as source descriptors whose
  prefixes extend one another; those are chained back into one atom here.'''
  descs = []
  for p in pipeline:
    k = p['op']
    if k == 'scan':
      pre = list(p['prefix'])
      descs.append((p, pre + list(p['vars'][len(pre):]), False))
    elif k == 'column_join':
      for s in p['sources']:
        descs.append((s, list(s['prefix']) + [p['var']], False))
    elif k == 'cartesian_join':
      for i, s in enumerate(p['sources']):
        got = p['var_from_source'][i] if i < len(p['var_from_source']) else []
        descs.append((s, list(s['prefix']) + list(got), False))
    elif k == 'negation':
      descs.append((p, list(p['prefix']), True))
  chains: list = []  # [rel, ver, index, positions, negated]
  for s, pos, neg in descs:
    key = (s['rel'], s['ver'], tuple(s['index']))
    pre = list(s['prefix'])
    for c in chains:
      if not neg and not c[4] and (c[0], c[1], c[2]) == key and pre and c[3] == pre:
        c[3] = pos
        break
    else:
      chains.append([s['rel'], s['ver'], tuple(s['index']), pos, neg])
  return [(rel, {index[j]: v for j, v in enumerate(pos)}, neg)
          for rel, _, index, pos, neg in chains]


def _recursive_relations(plan: dict) -> set:
  out = set()
  for st in plan['steps']:
    if st['recursive']:
      for op in st['ops']:
        if op['op'] == 'merge_index':
          out.add(op['rel'])
  return out


def _closure(plan: dict, seed: set) -> set:
  part = set(seed)
  changed = True
  while changed:
    changed = False
    for _, _, op in _rules(plan):
      if op.get('count'):
        continue
      head = _insert(op)['rel']
      if head not in part and any(rel in part for rel, _, _ in _atoms(op['pipeline'])):
        part.add(head)
        changed = True
  return part


def _modes(plan: dict, part: set) -> dict:
  # A positive atom over a partitioned relation confines a rule's bindings to
  # this shard's keys; a negated one does not (a tuple absent here may live
  # on another shard), so a rule whose partitioned atoms are all negated is
  # cut to its own keys explicitly.
  modes = {}
  for _, _, op in _rules(plan):
    atoms = [(cols.get(0), neg) for rel, cols, neg in _atoms(op['pipeline']) if rel in part]
    keys = {k for k, _ in atoms}
    positive = any(not neg for _, neg in atoms)
    if op.get('count'):
      if not atoms:
        modes[op['rule']] = 'work'
      elif len(keys) == 1 and None not in keys:
        modes[op['rule']] = '' if positive else ('key', next(iter(keys)))
      else:
        raise ShardError(f'count rule {op["rule"]} reads partitioned relations on different keys')
      continue
    ins = _insert(op)
    if ins['rel'] not in part:
      modes[op['rule']] = ''
      continue
    k = ins['vars'][0]
    if not atoms or keys == {k}:
      modes[op['rule']] = '' if positive else ('key', k)
    elif len(keys) == 1 and None not in keys and positive:
      # bindings confined to this shard's keys; derived tuples go to their owners
      modes[op['rule']] = 'exchange'
    else:
      bad = sorted(str(x) for x in keys - {k})
      raise ShardError(f'rule {op["rule"]} derives {ins["rel"]} keyed by {k} from partitioned '
                       f'relations keyed by {", ".join(bad)}: the join itself needs tuples of '
                       f'other shards')
  return modes


def _insert_exchanges(plan: dict, modes: dict) -> list:
  '''Adds an exchange op for every relation an 'exchange' rule of a step
  derives, before the step's first rebuild of its NEW version.'''
  sent = []
  for st in plan['steps']:
    rels = []
    for op in st['ops']:
      if op['op'] == 'execute_pipeline' and modes.get(op['rule']) == 'exchange':
        r = _insert(op)['rel']
        if r not in rels:
          rels.append(r)
    for r in rels:
      pos = next((i for i, op in enumerate(st['ops']) if op['op'] == 'rebuild_index' and
                  op['rel'] == r and op.get('ver') == 'NEW'), None)
      if pos is None:
        raise ShardError(f'no rebuild of NEW {r} to exchange before')
      st['ops'].insert(pos, {'op': 'exchange', 'rel': r})
      if r not in sent:
        sent.append(r)
  return sent


def shard_plan(plan: dict) -> ShardSpec:
  '''Mark `plan` for evaluation as one of several shards (see module doc).'''
  names = [r['name'] for r in plan['relations']]
  fallback = ''
  part = _closure(plan, _recursive_relations(plan))
  try:
    modes = _modes(plan, part)
  except ShardError as e:
    fallback = str(e)
    part = set()
    modes = _modes(plan, part)
  p = copy.deepcopy(plan)
  sent = _insert_exchanges(p, modes)
  flat = {}
  for _, _, op in _rules(p):
    m = modes[op['rule']]
    op.pop('shard', None)
    op.pop('shard_var', None)
    if isinstance(m, tuple):
      op['shard'], op['shard_var'] = m
      flat[op['rule']] = 'key'
    elif m:
      op['shard'] = m
      flat[op['rule']] = m
    else:
      flat[op['rule']] = ''
  return ShardSpec(plan=p, partitioned=[n for n in names if n in part],
                   replicated=[n for n in names if n not in part], modes=flat, fallback=fallback,
                   exchanged=sent)


def shard_rows(rows, world: int, rank: int) -> np.ndarray:
  '''The rows of a partitioned relation that shard `rank` owns (by column 0).'''
  a = np.ascontiguousarray(np.asarray(rows, dtype=np.uint32))
  if a.ndim != 2 or a.shape[0] == 0:
    return a
  return a[owner(a[:, 0], world) == rank]


class ShardedDatabase:
  '''One shard of a program: a native.Database evaluating `spec.plan` as
  shard `rank` of `world`.  Inputs are loaded in full (replicated); rows
  loaded into a partitioned relation are cut to this shard's part.'''

  def __init__(self, spec: ShardSpec, rank: int, world: int, device: int = 0, exchange=None):
    from .native import Database
    if not 0 <= rank < world:
      raise ValueError(f'rank {rank} outside [0, {world})')
    if spec.exchanged and world > 1 and exchange is None:
      raise ValueError(f'plan exchanges {spec.exchanged} between shards: pass exchange=')
    self.spec, self.rank, self.world = spec, rank, world
    self.db = Database(spec.plan, device=device)
    self.db.set_option('shard_world', world)
    self.db.set_option('shard_rank', rank)
    if exchange is not None:
      self.db.set_exchange(exchange.callback(rank))

  def load_rows(self, rel: str, rows) -> None:
    if rel in self.spec.partitioned:
      rows = shard_rows(rows, self.world, self.rank)
    self.db.load_rows(rel, rows)

  def run(self, max_iters: int = 0) -> None:
    self.db.run(max_iters)

  def local_size(self, rel: str) -> int:
    return self.db.size(rel)

  def local_count(self, rule: str) -> int:
    return self.db.count(rule)

  def local_dump(self, rel: str) -> np.ndarray:
    return self.db.dump(rel)

  def close(self) -> None:
    self.db.close()

  def __enter__(self):
    return self

  def __exit__(self, *exc):
    self.close()


def _device_copy(dst: int, src: int, nbytes: int, stream: int) -> None:
  from . import native
  native.check(native.lib().srdl_copy_device(ctypes.c_void_p(dst), ctypes.c_void_p(src), nbytes,
                                              ctypes.c_void_p(stream)), 'srdl_copy_device')


class LocalExchange:
  '''Exchange among `world` shards that are run by threads of one process
  (ShardedDatabase(..., exchange=ex) per thread).  Shards meet at a barrier
  in every phase; a receiver copies its slices straight out of the senders'
  buffers (peer copies when the shards sit on different GPUs of the
  process).  `copy(dst, src, nbytes, stream)` may replace the device copy;
  it must have finished the copy when it returns (the default one
  synchronises), because a sender's buffer goes back to its stream's arena
  as soon as the exchange's last barrier is passed.  A shard whose run fails
  should call abort(), so the others stop waiting.'''

  def __init__(self, world: int, timeout: float = 600.0, copy=None):
    self.world = world
    self.barrier = threading.Barrier(world, timeout=timeout)
    self.slots: list = [None] * world
    self.sent: list = [None] * world  # each shard's send counts of the current exchange
    self.copy = copy or _device_copy

  def abort(self) -> None:
    self.barrier.abort()

  def callback(self, rank: int):
    w = self.world

    def fn(phase, rel, counts, send, recv, stream):
      if phase == 0:    # counts: sent to each shard -> received from each shard
        self.sent[rank] = [int(counts[i]) for i in range(w)]
        self.barrier.wait()
        for src in range(w):
          counts[src] = self.sent[src][rank]
        self.barrier.wait()
      elif phase == 1:  # move the keys: my slice of every sender's buffer, in sender order
        self.slots[rank] = (send, list(self.sent[rank]))
        self.barrier.wait()
        pos = 0
        for src in range(w):
          sptr, scounts = self.slots[src]
          n = scounts[rank]
          if n:
            self.copy(recv + 8 * pos, sptr + 8 * sum(scounts[:rank]), 8 * n, stream)
          pos += n
        self.barrier.wait()  # senders keep their buffers until every slice is copied
      elif phase == 2:  # convergence vote
        self.slots[rank] = int(counts[0])
        self.barrier.wait()
        counts[0] = sum(self.slots)
        self.barrier.wait()
      else:
        raise ValueError(f'unknown exchange phase {phase}')

    return fn


class TorchExchange:
  '''Exchange for one process per GPU under torch.distributed: counts and
  keys move with all_to_all_single (NCCL moves device tensors, gloo host
  ones), the vote is an all_reduce.  The engine's buffers are copied into
  and out of torch tensors on the database's stream.'''

  def __init__(self, group=None, copy=None):
    import torch.distributed as dist
    self.dist = dist
    self.group = group
    self.copy = copy or _device_copy

  def _device(self):
    import torch
    if self.dist.get_backend(self.group) == 'nccl':
      return torch.device('cuda', torch.cuda.current_device())
    return torch.device('cpu')

  def callback(self, rank: int):
    import torch
    dist = self.dist
    w = dist.get_world_size(self.group)
    state = {}

    def fn(phase, rel, counts, send, recv, stream):
      dev = self._device()
      if phase == 0:
        sent = torch.tensor([int(counts[i]) for i in range(w)], dtype=torch.int64, device=dev)
        got = torch.empty_like(sent)
        dist.all_to_all_single(got, sent, group=self.group)
        state['sent'] = [int(x) for x in sent.tolist()]
        state['got'] = [int(x) for x in got.tolist()]
        for i in range(w):
          counts[i] = state['got'][i]
      elif phase == 1:
        ns, nr = sum(state['sent']), sum(state['got'])
        src = torch.empty(max(ns, 1), dtype=torch.int64, device=dev)
        dst = torch.empty(max(nr, 1), dtype=torch.int64, device=dev)
        if ns:
          self.copy(src.data_ptr(), send, 8 * ns, stream)
        dist.all_to_all_single(dst[:nr], src[:ns], output_split_sizes=state['got'],
                               input_split_sizes=state['sent'], group=self.group)
        if dev.type == 'cuda':
          torch.cuda.current_stream(dev).synchronize()
        if nr:
          self.copy(recv, dst.data_ptr(), 8 * nr, stream)
      elif phase == 2:
        t = torch.tensor([int(counts[0])], dtype=torch.int64, device=dev)
        dist.all_reduce(t, group=self.group)
        counts[0] = int(t.item())
      else:
        raise ValueError(f'unknown exchange phase {phase}')

    return fn


def run_local_shards(spec: ShardSpec, world: int, inputs: dict, device=0, max_iters: int = 0,
                     exchange: LocalExchange | None = None) -> list:
  '''Runs the `world` shards of `spec` in threads of this process (shard r
  on device[r] when `device` is a list, else all on one device) and returns
  the open ShardedDatabase of every shard (the caller reads and closes
  them).  Exchanges, if the plan has any, go through a LocalExchange.'''
  ex = exchange or (LocalExchange(world) if spec.exchanged and world > 1 else None)
  devs = device if isinstance(device, (list, tuple)) else [device] * world
  shards = [ShardedDatabase(spec, r, world, device=devs[r], exchange=ex) for r in range(world)]
  for sd in shards:
    for rel, rows in inputs.items():
      sd.load_rows(rel, rows)
  errors: list = [None] * world

  def work(r):
    try:
      shards[r].run(max_iters)
    except BaseException as e:  # noqa: BLE001 -- reported after the join
      errors[r] = e
      if ex is not None:
        ex.abort()

  threads = [threading.Thread(target=work, args=(r,)) for r in range(world)]
  for th in threads:
    th.start()
  for th in threads:
    th.join()
  failed = [e for e in errors if e is not None]
  if failed:
    for sd in shards:
      sd.close()
    raise failed[0]
  return shards


def combine_sizes(spec: ShardSpec, per_shard: list) -> dict:
  '''Whole-program sizes from per-shard {relation: size}: partitioned
  relations add up, replicated ones are equal on every shard.'''
  out = {}
  for rel in per_shard[0]:
    vals = [d[rel] for d in per_shard]
    if rel in spec.partitioned:
      out[rel] = int(sum(vals))
    else:
      if len(set(vals)) != 1:
        raise AssertionError(f'replicated relation {rel} differs across shards: {vals}')
      out[rel] = int(vals[0])
  return out


def combine_dumps(spec: ShardSpec, rel: str, dumps: list) -> np.ndarray:
  '''Whole-relation dump (sorted rows) from per-shard dumps.'''
  if rel not in spec.partitioned:
    return dumps[0]
  a = np.concatenate([np.asarray(d, dtype=np.uint32) for d in dumps])
  if a.shape[0] == 0:
    return a
  order = np.lexsort(tuple(a[:, c] for c in reversed(range(a.shape[1]))))
  return a[order]


def allreduce_results(spec: ShardSpec, sizes: dict, counts: dict, group=None) -> tuple:
  '''Sum this shard's sizes of partitioned relations and its counts over
  all shards of the torch.distributed group (replicated sizes stay as they
  are).  Every shard must pass the same keys.'''
  import torch
  import torch.distributed as dist

  srels = sorted(r for r in sizes if r in spec.partitioned)
  crules = sorted(counts)
  vals = [sizes[r] for r in srels] + [counts[r] for r in crules]
  dev = torch.device('cpu')
  if dist.get_backend(group) == 'nccl':
    dev = torch.device('cuda', torch.cuda.current_device())
  t = torch.tensor(vals, dtype=torch.int64, device=dev)
  if t.numel():
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
  got = [int(x) for x in t.cpu().tolist()]
  out_sizes = dict(sizes)
  for i, r in enumerate(srels):
    out_sizes[r] = got[i]
  out_counts = {r: got[len(srels) + i] for i, r in enumerate(crules)}
  return out_sizes, out_counts


__all__ = ['ShardError', 'ShardSpec', 'ShardedDatabase', 'LocalExchange', 'TorchExchange',
           'run_local_shards', 'owner', 'shard_plan', 'shard_rows', 'combine_sizes',
           'combine_dumps', 'allreduce_results']
