'''C-ABI boundary checks that need no GPU: exports, plan loading, CSV input
path, error codes, and the generated srdatalog_* shim.'''

import ctypes
import json
import os
import re

import numpy as np
import pytest
from conftest import REPO, load_plan
from srdatalog_b200 import native
from srdatalog_b200.build import CompilerConfig, compile_jit_project, write_project
from srdatalog_b200.loader import SHIM_ENTRY_POINTS, JitRuntime


def header_functions():
  text = open(os.path.join(REPO, 'include', 'srdl.h')).read()
  text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
  return sorted(set(re.findall(r'\b(srdl_\w+)\s*\(', text)))


def test_library_exports_every_header_symbol():
  lib = native.lib()
  names = header_functions()
  assert len(names) >= 18
  for n in names:
    assert hasattr(lib, n), n
  assert set(names) <= set(native.SIGNATURES), set(names) - set(native.SIGNATURES)
  assert lib.srdl_version() == 1


@pytest.mark.parametrize('name', ['tc', 'sg', 'triangle', 'tc_left', 'tc_lsm', 'head_const',
                                  'rewrite_consts', 'galen', 'polonius'])
def test_open_committed_plans(name):
  db = native.Database(load_plan(name))
  db.close()


def test_plan_facts_checked_by_the_loader():
  h = ctypes.c_void_p()
  lib = native.lib()
  for facts, msg in ([[7, 1]], 'wrong arity'), ([[-1]], 'out of range'), ([[2**32]], 'out of range'):
    plan = load_plan('head_const')
    next(r for r in plan['relations'] if r['name'] == '__const_7')['facts'] = facts
    assert lib.srdl_open(json.dumps(plan).encode(), 0, ctypes.byref(h)) == 4
    assert msg in native.last_error()


def test_plan_errors():
  h = ctypes.c_void_p()
  lib = native.lib()
  assert lib.srdl_open(b'{not json', 0, ctypes.byref(h)) == 4
  assert 'plan' in native.last_error()
  plan = load_plan('tc')
  plan['steps'][0]['ops'][0]['pipeline'][0]['op'] = 'negation'
  assert lib.srdl_open(json.dumps(plan).encode(), 0, ctypes.byref(h)) == 7
  plan = load_plan('tc')
  plan['version'] = 9
  assert lib.srdl_open(json.dumps(plan).encode(), 0, ctypes.byref(h)) == 4
  assert lib.srdl_open(None, 0, ctypes.byref(h)) == 1


def write(tmp_path, name, text):
  p = tmp_path / name
  p.write_text(text)
  return str(p)


@pytest.mark.parametrize('text,rows', [
  ('1\t2\n3\t4\n', [(1, 2), (3, 4)]),
  ('1,2\n3,4\n\n5,6', [(1, 2), (3, 4), (5, 6)]),
  ('1 2\n3 4\r\n', [(1, 2), (3, 4)]),
  ('10   20\n30   40\n', [(10, 20), (30, 40)]),
  ('-1\t7\n', [(0xffffffff, 7)]),
  ('1\t2\t9\n', [(1, 2)]),
  ('', []),
])
def test_csv_parsing(tmp_path, text, rows):
  db = native.Database(load_plan('tc'))
  db.load_csv('ArcInput', write(tmp_path, 'a.csv', text))
  assert db.staged_rows('ArcInput') == len(rows)


def test_csv_errors(tmp_path):
  db = native.Database(load_plan('tc'))
  with pytest.raises(native.SrdlError) as e:
    db.load_csv('ArcInput', str(tmp_path / 'missing.csv'))
  assert e.value.code == 6
  with pytest.raises(native.SrdlError) as e:
    db.load_csv('ArcInput', write(tmp_path, 'b.csv', '1\tx\n'))
  assert e.value.code == 6
  with pytest.raises(native.SrdlError) as e:
    db.load_csv('ArcInput', write(tmp_path, 'c.csv', '1\n'))
  assert e.value.code == 6
  with pytest.raises(native.SrdlError) as e:
    db.load_csv('Nope', write(tmp_path, 'd.csv', '1\t2\n'))
  assert e.value.code == 1
  with pytest.raises(native.SrdlError) as e:
    db.load_csv('Path', write(tmp_path, 'e.csv', '1\t2\n'))
  assert e.value.code == 1


def test_load_all_and_rows(tmp_path):
  db = native.Database(load_plan('triangle'))
  (tmp_path / 'Person_knows_Person.csv').write_text('0|1\n'.replace('|', '\t') * 3)
  db.load_all(str(tmp_path))
  assert db.staged_rows('KnowsInput') == 3
  db.load_rows('KnowsInput', np.array([[5, 6], [7, 8]], np.uint32))
  assert db.staged_rows('KnowsInput') == 5
  with pytest.raises(native.SrdlError):
    db.load_all(str(tmp_path / 'nodir'))


def test_generated_shim_abi(tmp_path):
  proj = write_project(load_plan('tc'), 'TcPlan', cache_base=str(tmp_path))
  br = compile_jit_project(proj, CompilerConfig())
  assert br.ok(), br.compile_results[0].stderr
  rt = JitRuntime(br.artifact, [ep for ep in SHIM_ENTRY_POINTS if ep.name not in
                                ('srdatalog_load_csv', 'srdatalog_run', 'srdatalog_load_all')])
  lib = ctypes.CDLL(br.artifact)
  lib.srdatalog_load_csv.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
  lib.srdatalog_run.argtypes = [ctypes.c_ulonglong]
  lib.srdatalog_load_all.argtypes = [ctypes.c_char_p]
  lib.srdatalog_size.restype = ctypes.c_ulonglong
  # reference status codes (main_file.py:690-753)
  assert lib.srdatalog_run(0) == 1              # nothing loaded yet
  lib.srdatalog_init()                           # 0 on a GPU box, 1 without a device
  assert lib.srdatalog_run(0) == 1              # init alone loads nothing
  assert lib.srdatalog_load_csv(None, b'x') == 1
  assert lib.srdatalog_run(0) == 1              # a rejected (null) load loads nothing
  csv = write(tmp_path, 'Arc.csv', '0\t1\n1\t2\n')
  assert lib.srdatalog_load_csv(b'Nope', csv.encode()) == 2
  assert lib.srdatalog_load_csv(b'ArcInput', b'/nonexistent.csv') == 3
  assert lib.srdatalog_load_csv(b'ArcInput', csv.encode()) == 0
  assert lib.srdatalog_load_all(None) == 1
  assert lib.srdatalog_load_all(str(tmp_path).encode()) == 0
  assert lib.srdatalog_size(b'Unknown') == 0
  assert rt.srdatalog_shutdown() == 0
  assert lib.srdatalog_size(b'Path') == 0
  assert lib.srdatalog_run(0) == 1              # shutdown drops the loaded state


@pytest.mark.parametrize('n', [0, 1, 3, 55, 56, 63, 64, 65, 119, 120, 1000, 1 << 20])
def test_library_sha256_matches_hashlib(n):
  import hashlib
  data = np.random.default_rng(n).integers(0, 256, n, dtype=np.uint8).tobytes()
  assert native.sha256(data) == hashlib.sha256(data).hexdigest()
