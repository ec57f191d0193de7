'''The allocation-free sort entry point, through the C ABI, against the
scratch-taking one.

Callers such as a host engine whose memory manager pre-plans every device
allocation cannot let the library call cudaMalloc; they use
srdl_sort_unique_u64_noalloc, whose temporaries live in a fixed file-scope
device array.  Two calls in a row must each give exactly (integer keys: bit
for bit) what srdl_sort_unique_u64 gives with caller-provided scratch, and
what numpy's np.unique gives, and a request above the array's limit must be
refused with status 5.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test.
'''

import ctypes

import numpy as np
import pytest
from srdatalog_b200 import native

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


def _stream():
  return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _dev(keys):
  return torch.from_numpy(np.ascontiguousarray(keys, np.uint64).view(np.int64).copy()).cuda()


def _with_scratch(keys, bits):
  lib = native.lib()
  n = len(keys)
  d_in = _dev(keys)
  d_out = torch.empty(n, dtype=torch.int64, device='cuda')
  d_n = torch.full((1,), -1, dtype=torch.int64, device='cuda')
  sb = lib.srdl_sort_unique_scratch_bytes(n, bits)
  scratch = torch.empty(sb, dtype=torch.uint8, device='cuda')
  assert lib.srdl_sort_unique_u64(d_in.data_ptr(), n, bits, d_out.data_ptr(), d_n.data_ptr(),
                                  scratch.data_ptr(), sb, _stream()) == 0, native.last_error()
  torch.cuda.synchronize()
  return d_out[:int(d_n.item())].cpu().numpy().view(np.uint64)


def _no_alloc(keys, bits):
  lib = native.lib()
  n = len(keys)
  d_in = _dev(keys)
  d_out = torch.empty(n, dtype=torch.int64, device='cuda')
  d_n = torch.full((1,), -1, dtype=torch.int64, device='cuda')
  assert lib.srdl_sort_unique_u64_noalloc(d_in.data_ptr(), n, bits, d_out.data_ptr(),
                                          d_n.data_ptr(), _stream()) == 0, native.last_error()
  torch.cuda.synchronize()
  return d_out[:int(d_n.item())].cpu().numpy().view(np.uint64)


def test_no_alloc_sort_matches_scratch_entry_point_twice():
  lib = native.lib()
  limit = lib.srdl_sort_unique_noalloc_max_keys()
  assert limit == 1 << 20
  rng = np.random.default_rng(20261203)
  cases = [(20, limit), (13, 300_001)]   # two calls in a row, different shapes
  for bits, n in cases:
    hi = rng.integers(0, 1 << bits, n, dtype=np.uint64)
    lo = rng.integers(0, 1 << bits, n, dtype=np.uint64)
    keys = (hi << np.uint64(32)) | lo
    keys[: n // 4] = keys[rng.integers(0, n, n // 4)]   # duplicates
    want = _with_scratch(keys, bits)
    got = _no_alloc(keys, bits)
    assert got.shape == want.shape
    assert np.array_equal(got, want)
    assert np.array_equal(got, np.unique(keys))   # the sorted distinct keys themselves


def test_no_alloc_sort_rejects_oversize():
  lib = native.lib()
  n = lib.srdl_sort_unique_noalloc_max_keys() + 1
  d_in = torch.zeros(n, dtype=torch.int64, device='cuda')
  d_out = torch.empty(n, dtype=torch.int64, device='cuda')
  d_n = torch.zeros(1, dtype=torch.int64, device='cuda')
  rc = lib.srdl_sort_unique_u64_noalloc(d_in.data_ptr(), n, 8, d_out.data_ptr(), d_n.data_ptr(),
                                        _stream())
  assert rc == 5
  assert 'static scratch limit' in native.last_error()
