'''Kernel primitives through the C ABI on the GPU, bit-exact against the oracle.

torch supplies device buffers and the stream only; every computation runs in
libsrdl's kernels.'''

import ctypes

import numpy as np
import oracle
import pytest
from srdatalog_b200 import native

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


def dev(a: np.ndarray):
  a = np.ascontiguousarray(a, np.uint64)
  if a.shape[0] == 0:
    return torch.zeros(1, dtype=torch.int64, device='cuda')
  return torch.from_numpy(a.view(np.int64).copy()).cuda()


def host(t, n):
  return t[:n].cpu().numpy().view(np.uint64) if n else np.zeros(0, np.uint64)


def stream():
  return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def gpu_sort_unique(keys, bits, alias=False):
  lib = native.lib()
  n = len(keys)
  d_in = dev(keys)
  d_out = d_in if alias else torch.empty(max(n, 1), dtype=torch.int64, device='cuda')
  d_n = torch.full((1,), -1, dtype=torch.int64, device='cuda')
  sb = lib.srdl_sort_unique_scratch_bytes(n, bits)
  scratch = torch.empty(max(sb, 1), dtype=torch.uint8, device='cuda')
  rc = lib.srdl_sort_unique_u64(d_in.data_ptr(), n, bits, d_out.data_ptr(), d_n.data_ptr(),
                                scratch.data_ptr(), sb, stream())
  assert rc == 0, native.last_error()
  torch.cuda.synchronize()
  return host(d_out, int(d_n.item()))


def keys_with_bits(rng, n, bits, dup_frac=0.0):
  hi = rng.integers(0, 1 << bits, n, dtype=np.uint64)
  lo = rng.integers(0, 1 << bits, n, dtype=np.uint64)
  k = (hi << np.uint64(32)) | lo
  if dup_frac:
    m = int(n * dup_frac)
    k[:m] = k[rng.integers(0, n, m)]
  return k


@pytest.mark.parametrize('bits', [1, 5, 13, 16, 17, 20, 24, 32])
@pytest.mark.parametrize('n', [1, 7, 2048, 100_003])
def test_sort_unique_random(bits, n):
  rng = np.random.default_rng(bits * 1000 + n)
  k = keys_with_bits(rng, n, bits, dup_frac=0.3)
  assert np.array_equal(gpu_sort_unique(k, bits), oracle.sort_unique(k))


def test_sort_unique_edge_cases():
  assert gpu_sort_unique(np.zeros(0, np.uint64), 8).shape[0] == 0
  same = np.full(50_000, (3 << 32) | 9, np.uint64)
  assert np.array_equal(gpu_sort_unique(same, 4), np.array([(3 << 32) | 9], np.uint64))
  top = np.uint64(0xFFFFFFFF)
  k = np.array([(top << np.uint64(32)) | top, 0, (top << np.uint64(32)), top, 0], np.uint64)
  assert np.array_equal(gpu_sort_unique(k, 32), np.unique(k))
  rng = np.random.default_rng(1)
  s = np.unique(keys_with_bits(rng, 300_000, 20))
  assert np.array_equal(gpu_sort_unique(s, 20), s)
  assert np.array_equal(gpu_sort_unique(s[::-1].copy(), 20), s)
  assert np.array_equal(gpu_sort_unique(s[::-1].copy(), 20, alias=True), s)


def test_sort_unique_large_skewed():
  rng = np.random.default_rng(7)
  n = 6_000_000
  hi = np.minimum(rng.zipf(1.3, n), (1 << 20) - 1).astype(np.uint64)
  lo = rng.integers(0, 1 << 20, n, dtype=np.uint64)
  k = (hi << np.uint64(32)) | lo
  assert np.array_equal(gpu_sort_unique(k, 20), oracle.sort_unique(k))


def gpu_diff(a, b):
  lib = native.lib()
  da, db = dev(a), dev(b)
  out = torch.empty(max(len(a), 1), dtype=torch.int64, device='cuda')
  d_n = torch.full((1,), -1, dtype=torch.int64, device='cuda')
  sb = lib.srdl_set_difference_scratch_bytes(len(a))
  scratch = torch.empty(sb, dtype=torch.uint8, device='cuda')
  rc = lib.srdl_set_difference_u64(da.data_ptr(), len(a), db.data_ptr(), len(b), out.data_ptr(),
                                   d_n.data_ptr(), scratch.data_ptr(), sb, stream())
  assert rc == 0, native.last_error()
  torch.cuda.synchronize()
  return host(out, int(d_n.item()))


def gpu_merge(a, b):
  lib = native.lib()
  da, db = dev(a), dev(b)
  out = torch.empty(max(len(a) + len(b), 1), dtype=torch.int64, device='cuda')
  rc = lib.srdl_merge_u64(da.data_ptr(), len(a), db.data_ptr(), len(b), out.data_ptr(), stream())
  assert rc == 0, native.last_error()
  torch.cuda.synchronize()
  return host(out, len(a) + len(b))


@pytest.mark.parametrize('na,nb', [(0, 0), (0, 100), (100, 0), (1, 1), (5000, 200_000),
                                   (300_000, 2000), (1_000_000, 1_000_000)])
def test_set_difference(na, nb):
  rng = np.random.default_rng(na + 3 * nb)
  a = np.unique(keys_with_bits(rng, na, 18)) if na else np.zeros(0, np.uint64)
  b = np.unique(np.concatenate([keys_with_bits(rng, nb, 18), a[::2]])) if nb else np.zeros(0, np.uint64)
  assert np.array_equal(gpu_diff(a, b), oracle.set_difference(a, b))


def test_set_difference_many_tiles():
  '''40M - 24M keys built on the device: ~31K merged tiles whose output
  offsets chain through the look-back of every block of the grid; checked
  against torch.isin on the device.'''
  lib = native.lib()
  g = torch.Generator(device='cuda').manual_seed(5)
  a = torch.unique(torch.randint(0, 1 << 40, (40_000_000,), device='cuda', generator=g))
  extra = torch.randint(0, 1 << 40, (8_000_000,), device='cuda', generator=g)
  b = torch.unique(torch.cat([a[::3], extra]))
  out = torch.empty_like(a)
  d_n = torch.full((1,), -1, dtype=torch.int64, device='cuda')
  sb = lib.srdl_set_difference_scratch_bytes(a.numel())
  scratch = torch.empty(sb, dtype=torch.uint8, device='cuda')
  rc = lib.srdl_set_difference_u64(a.data_ptr(), a.numel(), b.data_ptr(), b.numel(), out.data_ptr(),
                                   d_n.data_ptr(), scratch.data_ptr(), sb, stream())
  assert rc == 0, native.last_error()
  torch.cuda.synchronize()
  want = a[~torch.isin(a, b)]
  n = int(d_n.item())
  assert n == want.numel()
  assert torch.equal(out[:n], want)


@pytest.mark.parametrize('na,nb', [(0, 0), (0, 10), (10, 0), (1, 1), (2047, 1), (3_000_000, 1000),
                                   (123_457, 98_765)])
def test_merge_disjoint(na, nb):
  rng = np.random.default_rng(na * 7 + nb)
  u = np.unique(keys_with_bits(rng, na + nb + 10, 24))
  rng.shuffle(u)
  a, b = np.sort(u[:na]), np.sort(u[na:na + nb])
  assert np.array_equal(gpu_merge(a, b), oracle.merge(a, b))


def test_sort_unique_many_tiles():
  '''20M keys of 2 x 21 bits: six 7-bit passes over ~10K tiles spread over
  every block of the grid.'''
  rng = np.random.default_rng(11)
  k = keys_with_bits(rng, 20_000_000, 21, dup_frac=0.1)
  assert np.array_equal(gpu_sort_unique(k, 21), oracle.sort_unique(k))


@pytest.mark.parametrize('bits', [15, 17])
def test_sort_unique_multi_portion(bits):
  '''More than 2^29 keys (32-bit and 64-bit packed forms).  The input is a
  scrambled multiset over the values 0..m-1 (each at least once), built on
  the device; the output must be exactly enc(0..m-1) in order, where enc
  splits a value into (hi, lo) halves of at most `bits` bits.'''
  lib = native.lib()
  n = (1 << 29) + 3 * 2048 + 77
  m = n - 1000
  i = torch.arange(n, dtype=torch.int64, device='cuda')
  v = (i * 2654435761) % n
  v = torch.where(v >= m, v - m, v)              # values m..n-1 fold onto 0..999
  lo_bits = 30 - bits                           # values < 2^30 -> both halves < 2^bits
  enc = lambda x: ((x >> lo_bits) << 32) | (x & ((1 << lo_bits) - 1))
  keys = enc(v)
  del v, i
  out = torch.empty_like(keys)
  d_n = torch.full((1,), -1, dtype=torch.int64, device='cuda')
  sb = lib.srdl_sort_unique_scratch_bytes(n, bits)
  scratch = torch.empty(sb, dtype=torch.uint8, device='cuda')
  rc = lib.srdl_sort_unique_u64(keys.data_ptr(), n, bits, out.data_ptr(), d_n.data_ptr(),
                                scratch.data_ptr(), sb, stream())
  assert rc == 0, native.last_error()
  torch.cuda.synchronize()
  assert int(d_n.item()) == m
  assert torch.equal(out[:m], enc(torch.arange(m, dtype=torch.int64, device='cuda')))
