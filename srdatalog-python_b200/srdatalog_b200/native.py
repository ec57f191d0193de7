'''ctypes binding of libsrdl (include/srdl.h) and a Python handle wrapper.

There is no fallback: if libsrdl.so is missing or fails to load, every
entry point raises.  Build it with `make -C srdatalog-python_b200/csrc`
or `python -c "import __graft_entry__; __graft_entry__.build()"`.
'''

from __future__ import annotations

import ctypes
import json
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, 'lib', 'libsrdl.so')

_u64 = ctypes.c_uint64
_i64 = ctypes.c_int64
_vp = ctypes.c_void_p
_cp = ctypes.c_char_p
_u32p = ctypes.POINTER(ctypes.c_uint32)

# srdl_exchange_fn: (user, phase, rel, counts, d_send, d_recv, stream) -> int
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, _vp, ctypes.c_int, _cp, ctypes.POINTER(_u64), _vp, _vp,
                               _vp)

# name -> (restype, argtypes); mirrors include/srdl.h
SIGNATURES = {
  'srdl_last_error': (_cp, []),
  'srdl_version': (ctypes.c_int, []),
  'srdl_open': (ctypes.c_int, [_cp, ctypes.c_int, ctypes.POINTER(_vp)]),
  'srdl_close': (ctypes.c_int, [_vp]),
  'srdl_init_device': (ctypes.c_int, [_vp]),
  'srdl_load_rows': (ctypes.c_int, [_vp, _cp, _u32p, _u64]),
  'srdl_load_csv': (ctypes.c_int, [_vp, _cp, _cp]),
  'srdl_load_all': (ctypes.c_int, [_vp, _cp]),
  'srdl_staged_rows': (_u64, [_vp, _cp]),
  'srdl_load_device_rows': (ctypes.c_int, [_vp, _cp, _vp, _u64]),
  'srdl_set_stream': (ctypes.c_int, [_vp, _vp]),
  'srdl_set_profiling': (ctypes.c_int, [_vp, ctypes.c_int]),
  'srdl_launch_count': (_u64, []),
  'srdl_clear_inputs': (ctypes.c_int, [_vp]),
  'srdl_set_count_groups': (ctypes.c_int, [_vp, _cp, _u32p, _u64]),
  'srdl_group_counts': (ctypes.c_int, [_vp, _cp, ctypes.POINTER(_u64), _u64]),
  'srdl_range_counts': (ctypes.c_int, [_vp, _cp, _u32p, _u64, ctypes.POINTER(_u64)]),
  'srdl_set_instances': (ctypes.c_int, [_vp, _u32p, _u64]),
  'srdl_instance_iterations': (ctypes.c_int, [_vp, _u64, _u32p, _u64]),
  'srdl_range_checksums': (ctypes.c_int, [_vp, _cp, _u32p, _u64, ctypes.POINTER(_u64)]),
  'srdl_run': (ctypes.c_int, [_vp, _u64]),
  'srdl_size': (_u64, [_vp, _cp]),
  'srdl_count': (_u64, [_vp, _cp]),
  'srdl_dump': (_i64, [_vp, _cp, _u32p, _u64]),
  'srdl_stats_json': (ctypes.c_int, [_vp, ctypes.c_char_p, _u64]),
  'srdl_mem_stats': (ctypes.c_int, [_vp, ctypes.POINTER(_u64)]),
  'srdl_trim_cache': (ctypes.c_int, [_vp]),
  'srdl_sort_unique_scratch_bytes': (_u64, [_u64, ctypes.c_int]),
  'srdl_sort_unique_u64': (ctypes.c_int, [_vp, _u64, ctypes.c_int, _vp, _vp, _vp, _u64, _vp]),
  'srdl_set_difference_scratch_bytes': (_u64, [_u64]),
  'srdl_set_difference_u64': (ctypes.c_int, [_vp, _u64, _vp, _u64, _vp, _vp, _vp, _u64, _vp]),
  'srdl_merge_u64': (ctypes.c_int, [_vp, _u64, _vp, _u64, _vp, _vp]),
  'srdl_sort_unique_u64_noalloc': (ctypes.c_int, [_vp, _u64, ctypes.c_int, _vp, _vp, _vp]),
  'srdl_sort_unique_noalloc_max_keys': (_u64, []),
  'srdl_set_option': (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_int64]),
  'srdl_set_exchange': (ctypes.c_int, [_vp, EXCHANGE_FN, _vp]),
  'srdl_copy_device': (ctypes.c_int, [_vp, _vp, _u64, _vp]),
  'srdl_hash': (ctypes.c_int, [_vp, _cp, ctypes.c_char_p]),
  'srdl_sha256': (ctypes.c_int, [_vp, _u64, ctypes.c_char_p]),
}


def sha256(data: bytes) -> str:
  '''SHA-256 (hex) computed by libsrdl.'''
  out = ctypes.create_string_buffer(32)
  buf = ctypes.create_string_buffer(bytes(data), max(1, len(data)))
  check(lib().srdl_sha256(buf, len(data), out), 'srdl_sha256')
  return out.raw.hex()

_LIB = None


class SrdlError(RuntimeError):
  def __init__(self, what: str, code: int, msg: str):
    super().__init__(f'{what} failed with status {code}: {msg}')
    self.code = code


def lib() -> ctypes.CDLL:
  '''Load libsrdl.so once; raises if it is absent (no CPU fallback exists).'''
  global _LIB
  if _LIB is None:
    if not os.path.exists(LIB_PATH):
      raise OSError(f'libsrdl.so not built ({LIB_PATH}); run make -C srdatalog-python_b200/csrc')
    L = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)
    for name, (res, args) in SIGNATURES.items():
      f = getattr(L, name)
      f.restype = res
      f.argtypes = args
    _LIB = L
  return _LIB


def last_error() -> str:
  return lib().srdl_last_error().decode()


def check(rc: int, what: str) -> None:
  if rc != 0:
    raise SrdlError(what, rc, last_error())


class Database:
  '''One plan bound to one GPU (handle API of libsrdl).'''

  def __init__(self, plan, device: int = 0):
    text = plan if isinstance(plan, str) else json.dumps(plan)
    self.plan = json.loads(text)
    h = _vp()
    check(lib().srdl_open(text.encode(), device, ctypes.byref(h)), 'srdl_open')
    self._h = h
    self._arity = {r['name']: r['arity'] for r in self.plan['relations']}

  def close(self) -> None:
    if getattr(self, '_h', None):
      lib().srdl_close(self._h)
      self._h = None

  def __del__(self):
    try:
      self.close()
    except Exception:
      pass

  def __enter__(self):
    return self

  def __exit__(self, *exc):
    self.close()

  def init_device(self) -> None:
    check(lib().srdl_init_device(self._h), 'srdl_init_device')

  def load_rows(self, rel: str, rows) -> None:
    a = np.ascontiguousarray(rows, dtype=np.uint32)
    n = a.shape[0] if a.ndim > 1 else (a.shape[0] // max(1, self._arity.get(rel, 1)))
    check(lib().srdl_load_rows(self._h, rel.encode(), a.ctypes.data_as(_u32p), n),
          f'srdl_load_rows({rel})')

  def load_csv(self, rel: str, path: str) -> None:
    check(lib().srdl_load_csv(self._h, rel.encode(), path.encode()), f'srdl_load_csv({rel})')

  def load_all(self, directory: str) -> None:
    check(lib().srdl_load_all(self._h, directory.encode()), 'srdl_load_all')

  def load_device_rows(self, rel: str, ptr: int, n_rows: int) -> None:
    '''Stage n_rows uint32 pairs already in device memory at `ptr`.'''
    check(lib().srdl_load_device_rows(self._h, rel.encode(), ptr, n_rows),
          f'srdl_load_device_rows({rel})')

  def set_stream(self, stream_ptr: int) -> None:
    check(lib().srdl_set_stream(self._h, stream_ptr), 'srdl_set_stream')

  def set_profiling(self, on: bool = True) -> None:
    check(lib().srdl_set_profiling(self._h, 1 if on else 0), 'srdl_set_profiling')

  def set_exchange(self, fn) -> None:
    '''fn(phase, rel, counts, send_ptr, recv_ptr, stream_ptr) moves tuples
    between shards (see srdl_set_exchange); counts is a ctypes uint64 array
    of shard_world entries, updated in place.  An exception inside fn fails
    the run.  None removes it.'''
    if fn is None:
      self._xfn = None
      check(lib().srdl_set_exchange(self._h, EXCHANGE_FN(), None), 'srdl_set_exchange')
      return

    def tramp(_user, phase, rel, counts, send, recv, stream):
      try:
        fn(int(phase), rel.decode() if rel else '', counts, send or 0, recv or 0, stream or 0)
        return 0
      except Exception as e:  # reported through the run's error
        self._xerr = e
        return 1

    self._xerr = None
    self._xfn = EXCHANGE_FN(tramp)  # kept alive with the handle
    check(lib().srdl_set_exchange(self._h, self._xfn, None), 'srdl_set_exchange')

  def set_option(self, name: str, value: int) -> None:
    '''Option (srdl_set_option): bitmap_mb, hash_min, lsm_compact_pct,
    radix_bits, join_blocks_per_sm, shard_world, shard_rank, mem_limit_mb.'''
    check(lib().srdl_set_option(self._h, name.encode(), int(value)), 'srdl_set_option')

  def set_count_groups(self, rule: str, bounds) -> None:
    b = np.ascontiguousarray(bounds, dtype=np.uint32)
    self._groups = {**getattr(self, '_groups', {}), rule: b.shape[0] - 1}
    check(lib().srdl_set_count_groups(self._h, rule.encode(), b.ctypes.data_as(_u32p), b.shape[0]),
          f'srdl_set_count_groups({rule})')

  def group_counts(self, rule: str) -> np.ndarray:
    n = self._groups[rule]
    out = np.zeros(n, np.uint64)
    check(lib().srdl_group_counts(self._h, rule.encode(), out.ctypes.data_as(ctypes.POINTER(_u64)), n),
          f'srdl_group_counts({rule})')
    return out

  def clear_inputs(self) -> None:
    check(lib().srdl_clear_inputs(self._h), 'srdl_clear_inputs')

  def range_counts(self, rel: str, bounds) -> np.ndarray:
    '''Rows of FULL(rel) per first-column range [bounds[j], bounds[j+1]).'''
    b = np.ascontiguousarray(bounds, dtype=np.uint32)
    out = np.zeros(max(0, b.shape[0] - 1), np.uint64)
    check(lib().srdl_range_counts(self._h, rel.encode(), b.ctypes.data_as(_u32p), b.shape[0],
                                  out.ctypes.data_as(ctypes.POINTER(_u64))),
          f'srdl_range_counts({rel})')
    return out

  def set_instances(self, bounds) -> None:
    '''Instance j of a batched run owns the values [bounds[j], bounds[j+1]);
    later runs record every instance's own iteration count per recursive
    step (None or an empty array clears).'''
    b = np.ascontiguousarray([] if bounds is None else bounds, dtype=np.uint32)
    self._n_instances = max(0, b.shape[0] - 1)
    check(lib().srdl_set_instances(self._h, b.ctypes.data_as(_u32p) if b.size else None, b.shape[0]),
          'srdl_set_instances')

  def instance_iterations(self, step: int) -> np.ndarray:
    '''Iterations each instance's own run takes in plan step `step` (last run).'''
    out = np.zeros(getattr(self, '_n_instances', 0), np.uint32)
    check(lib().srdl_instance_iterations(self._h, step, out.ctypes.data_as(_u32p), out.shape[0]),
          f'srdl_instance_iterations({step})')
    return out

  def range_checksums(self, rel: str, bounds) -> np.ndarray:
    '''Per-range fingerprints of FULL(rel) (binary): the sum mod 2^64 of
    row_fingerprint(x - bounds[j], y - bounds[j]) over the rows whose first
    column is in [bounds[j], bounds[j+1]).'''
    b = np.ascontiguousarray(bounds, dtype=np.uint32)
    out = np.zeros(max(0, b.shape[0] - 1), np.uint64)
    check(lib().srdl_range_checksums(self._h, rel.encode(), b.ctypes.data_as(_u32p), b.shape[0],
                                     out.ctypes.data_as(ctypes.POINTER(_u64))),
          f'srdl_range_checksums({rel})')
    return out

  def staged_rows(self, rel: str) -> int:
    return int(lib().srdl_staged_rows(self._h, rel.encode()))

  def run(self, max_iters: int = 0) -> None:
    rc = lib().srdl_run(self._h, max_iters)
    xerr = getattr(self, '_xerr', None)
    if rc and xerr is not None:
      self._xerr = None
      raise SrdlError('srdl_run', rc, f'exchange callback raised {xerr!r}') from xerr
    check(rc, 'srdl_run')

  def hash(self, rel: str) -> str:
    '''SHA-256 (hex) of FULL(rel) as dump() returns it (sorted rows,
    little-endian uint32, row-major), computed in libsrdl.'''
    out = ctypes.create_string_buffer(32)
    check(lib().srdl_hash(self._h, rel.encode(), out), 'srdl_hash')
    return out.raw.hex()

  def size(self, rel: str) -> int:
    return int(lib().srdl_size(self._h, rel.encode()))

  def count(self, rule: str) -> int:
    return int(lib().srdl_count(self._h, rule.encode()))

  def dump(self, rel: str) -> np.ndarray:
    '''FULL(rel) as an (n, arity) uint32 array, sorted in declared column order.'''
    n = lib().srdl_dump(self._h, rel.encode(), None, 0)
    if n < 0:
      raise SrdlError(f'srdl_dump({rel})', -n, last_error())
    k = self._arity[rel]
    out = np.empty((n, k), np.uint32)
    if n:
      m = lib().srdl_dump(self._h, rel.encode(), out.ctypes.data_as(_u32p), n)
      if m != n:
        raise SrdlError(f'srdl_dump({rel})', -1, 'size changed')
    return out

  def mem_stats(self) -> dict:
    '''Device bytes of this handle's stream (srdl_mem_stats): held now, the
    last run's peak, cached for reuse, and the run limit (0: none).'''
    out = (_u64 * 4)()
    check(lib().srdl_mem_stats(self._h, out), 'srdl_mem_stats')
    return {'in_use': int(out[0]), 'peak': int(out[1]), 'cached': int(out[2]),
            'limit': int(out[3])}

  def trim_cache(self) -> None:
    '''Return the blocks this handle's stream caches to the device.'''
    check(lib().srdl_trim_cache(self._h), 'srdl_trim_cache')

  def stats(self) -> dict:
    buf = ctypes.create_string_buffer(1 << 16)
    check(lib().srdl_stats_json(self._h, buf, len(buf)), 'srdl_stats_json')
    return json.loads(buf.value.decode())
