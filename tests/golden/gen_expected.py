'''Regenerate tests/golden/expected.json with the CPU oracle.

Each entry records the seeded workload, the output size, the SHA-256 of the
sorted dump (declared column order, little-endian uint32 rows) and the
number of recursive iterations, so GPU tests can check full-size runs
without re-running the oracle.

  python tests/golden/gen_expected.py
'''

from __future__ import annotations

import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(REPO, 'oracle'), os.path.join(REPO, 'srdatalog-python_b200')]

import oracle  # noqa: E402
from srdatalog_b200 import workloads as W  # noqa: E402

# name -> (program, generator description, generator callable)
CASES = {
  'tc_small': ('tc', 'uniform_edges(5000, 20000, seed=1)', lambda: W.tc_small(1)),
  'tc_mid': ('tc', 'uniform_edges(2000, 6000, seed=7)', lambda: W.uniform_edges(2000, 6000, 7)),
  'sg_10k': ('sg', 'sg_forest(10000, seed=2)', lambda: W.sg_forest(10000, seed=2)),
  'sg_2k': ('sg', 'sg_forest(2000, seed=4)', lambda: W.sg_forest(2000, seed=4)),
  'triangle_rmat20': ('triangle', 'rmat_edges(20, 1<<24, seed=3)', lambda: W.rmat_edges(20, 1 << 24, seed=3)),
  'triangle_rmat14': ('triangle', 'rmat_edges(14, 1<<18, seed=5)', lambda: W.rmat_edges(14, 1 << 18, seed=5)),
}


def compute(name: str) -> dict:
  prog, desc, gen = CASES[name]
  e = gen()
  out = {'program': prog, 'input': desc, 'edges': int(e.shape[0])}
  if prog == 'tc':
    keys, iters, derived = oracle.tc(e)
    rows = oracle.unpack(keys, order=(1, 0))
    out.update(relation='Path', size=int(rows.shape[0]), sha256=oracle.dump_hash(rows),
               iterations=iters, derived=derived)
  elif prog == 'sg':
    keys, iters, derived = oracle.sg(e)
    rows = oracle.unpack(keys, order=(0, 1))
    out.update(relation='Sg', size=int(rows.shape[0]), sha256=oracle.dump_hash(rows),
               iterations=iters, derived=derived)
  else:
    out.update(rule='TriangleJoin', count=oracle.triangle_count(e))
  return out


def main() -> int:
  names = sys.argv[1:] or list(CASES)
  path = os.path.join(HERE, 'expected.json')
  data = json.load(open(path)) if os.path.exists(path) else {}
  for n in names:
    data[n] = compute(n)
    print(n, data[n], flush=True)
  with open(path, 'w') as f:
    json.dump(data, f, indent=1, sort_keys=True)
    f.write('\n')
  return 0


if __name__ == '__main__':
  raise SystemExit(main())
