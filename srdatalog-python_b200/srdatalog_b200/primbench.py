'''Timing of libsrdl's sort / merge / set-difference primitives on one GPU.

    python -m srdatalog_b200.primbench --keys 200000000 [--bits 21] [--peak-gbs 6553]

Keys are random (hi, lo) pairs with `bits`-bit halves, built on the device.
Each primitive runs twice untimed, then once between CUDA events on the
current stream; one JSON line per primitive gives the time and the
algorithmic bandwidth (the bytes the operation must move at least):

* sort + unique of n keys: the passes the library runs -- read the input,
  write the packed keys, read and write them once per counting pass, read
  them for the dedup and write the distinct keys (io_gbs: 16 B per key);
* merge of two disjoint sorted halves: 16 B per output key;
* set difference a - b: 8 B per key of a, b and the result.

torch provides device buffers and the stream only.
'''

from __future__ import annotations

import argparse
import ctypes
import json

from . import native


def main(argv=None) -> int:
  import torch

  ap = argparse.ArgumentParser()
  ap.add_argument('--keys', type=int, default=200_000_000)
  ap.add_argument('--bits', type=int, default=21)
  ap.add_argument('--peak-gbs', type=float, default=0.0,
                  help='HBM peak for the fraction (omit to leave it out)')
  args = ap.parse_args(argv)
  lib = native.lib()
  n, bits = args.keys, args.bits
  st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
  g = torch.Generator(device='cuda').manual_seed(1)
  hi = torch.randint(0, 1 << bits, (n,), device='cuda', dtype=torch.int64, generator=g)
  lo = torch.randint(0, 1 << bits, (n,), device='cuda', dtype=torch.int64, generator=g)
  keys = (hi << 32) | lo
  del hi, lo
  e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)

  def timed(fn):
    for _ in range(2):
      fn()
    torch.cuda.synchronize()
    e0.record()
    fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)

  def report(name, ms, alg_bytes, **extra):
    gbs = alg_bytes / ms / 1e6
    line = {'primitive': name, 'ms': round(ms, 4), 'alg_gbs': round(gbs, 1), **extra}
    if args.peak_gbs:
      line['frac_of_peak'] = round(gbs / args.peak_gbs, 3)
    print(json.dumps(line), flush=True)

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
  # packed key width k and counting passes as the library runs them: read the
  # input (8 B), write packed keys (k), P passes reading and writing k each,
  # read the sorted keys once more (k) and write the distinct ones (8 B)
  k = 4 if 2 * bits <= 32 else 8
  passes = (2 * bits + 7) // 8
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
  return 0


if __name__ == '__main__':
  raise SystemExit(main())
