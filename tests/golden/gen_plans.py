'''Regenerate tests/golden/plans/*.json from the DSL programs.

Needs the srdatalog front end: --ref names a checkout of the reference
(default: the SRDATALOG_REF environment variable); its src/ directory goes
on sys.path.  For every program that has a
reference MIR fixture, the MIR printed by the front end is first compared
byte-for-byte with that fixture, so the committed plans are the plans the
reference itself would execute.

  SRDATALOG_REF=/root/reference python tests/golden/gen_plans.py
'''

from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def main() -> int:
  ap = argparse.ArgumentParser()
  ap.add_argument('--ref', default=os.environ.get('SRDATALOG_REF', ''))
  ap.add_argument('--check', action='store_true', help='compare instead of writing')
  args = ap.parse_args()
  if not args.ref:
    ap.error('name the reference checkout with --ref or SRDATALOG_REF')
  sys.path.insert(0, os.path.join(args.ref, 'src'))
  sys.path.insert(0, os.path.join(REPO, 'srdatalog-python_b200'))
  sys.path.insert(0, HERE)
  from programs import PROGRAMS
  from srdatalog.hir import compile_to_mir
  from srdatalog.mir.emit import print_mir_sexpr

  from srdatalog_b200.plan import dumps, plan_from_program

  bad = 0
  for key, (builder, project, fixture) in PROGRAMS.items():
    prog = builder()
    if fixture:
      want = open(os.path.join(args.ref, 'tests', 'fixtures', fixture)).read()
      got = print_mir_sexpr(compile_to_mir(prog))
      if want.strip() != got.strip():
        print(f'{key}: MIR differs from reference fixture {fixture}')
        bad += 1
        continue
    plan = plan_from_program(prog, project)
    path = os.path.join(HERE, 'plans', f'{key}.json')
    text = json.dumps(json.loads(dumps(plan)), indent=1, sort_keys=True) + '\n'
    if args.check:
      if open(path).read() != text:
        print(f'{key}: committed plan is stale')
        bad += 1
    else:
      with open(path, 'w') as f:
        f.write(text)
      print(f'wrote {path}')
  return 1 if bad else 0


if __name__ == '__main__':
  raise SystemExit(main())
