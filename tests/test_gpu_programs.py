'''Whole programs on the GPU, bit-exact against the oracle (size + SHA-256 of
the sorted dump, or the count for count-only rules).'''

import ctypes

import numpy as np
import oracle
import pytest
from conftest import load_plan
from srdatalog_b200 import native
from srdatalog_b200 import workloads as W

pytestmark = pytest.mark.gpu


def run(plan_name, inputs, max_iters=0):
  db = native.Database(load_plan(plan_name))
  for rel, rows in inputs.items():
    db.load_rows(rel, rows)
  db.run(max_iters)
  return db


def rows_set(a):
  return {tuple(map(int, r)) for r in a}


def test_tc_small_config(expected):
  exp = expected['tc_small']
  db = run('tc', {'ArcInput': W.tc_small(1)})
  assert db.size('Path') == exp['size']
  rows = db.dump('Path')
  assert oracle.dump_hash(rows) == exp['sha256']
  rec = [s for s in db.stats()['steps'] if s['recursive']]
  assert rec[0]['iterations'] == exp['iterations']


@pytest.mark.parametrize('seed', range(6))
def test_tc_random_small_vs_interpreter(seed):
  e = W.uniform_edges(40 + 10 * seed, 90 + 30 * seed, seed)
  db = run('tc', {'ArcInput': e})
  want, _ = oracle.run_plan(load_plan('tc'), {'ArcInput': e})
  assert rows_set(db.dump('Path')) == set(want['Path'])


def test_tc_mid_and_left_recursive(expected):
  exp = expected['tc_mid']
  e = W.uniform_edges(2000, 6000, 7)
  for plan in ('tc', 'tc_left'):
    db = run(plan, {'ArcInput': e})
    assert db.size('Path') == exp['size']
    assert oracle.dump_hash(db.dump('Path')) == exp['sha256']


def test_tc_edge_cases():
  db = run('tc', {'ArcInput': np.zeros((0, 2), np.uint32)})
  assert db.size('Path') == 0 and db.dump('Path').shape == (0, 2)
  e = np.array([[1, 1], [1, 2], [1, 2], [2, 1]], np.uint32)   # self-loop + duplicate row
  db = run('tc', {'ArcInput': e})
  assert rows_set(db.dump('Path')) == {(1, 1), (1, 2), (2, 1), (2, 2)}
  chain = np.array([(i, i + 1) for i in range(30)], np.uint32)
  for k in (1, 2, 5):
    db = run('tc', {'ArcInput': chain}, max_iters=k)
    keys, _, _ = oracle.tc(chain, max_iters=k)
    assert db.size('Path') == keys.shape[0]
  top = 0xFFFFFFFF
  big = np.array([[top, 5], [5, top - 1], [top - 1, top], [7, 0]], np.uint32)
  db = run('tc', {'ArcInput': big})
  keys, _, _ = oracle.tc(big)
  assert rows_set(db.dump('Path')) == rows_set(oracle.unpack(keys, order=(1, 0)))


def test_repeat_run_same_result():
  e = W.uniform_edges(500, 1500, 3)
  db = run('tc', {'ArcInput': e})
  h1 = oracle.dump_hash(db.dump('Path'))
  db.run()
  assert oracle.dump_hash(db.dump('Path')) == h1


@pytest.mark.parametrize('name', ['sg_2k', 'sg_10k'])
def test_sg_configs(expected, name):
  exp = expected[name]
  n, seed = (2000, 4) if name == 'sg_2k' else (10000, 2)
  db = run('sg', {'Arc': W.sg_forest(n, seed=seed)})
  assert db.size('Sg') == exp['size']
  assert oracle.dump_hash(db.dump('Sg')) == exp['sha256']


def test_sg_small_vs_interpreter():
  e = W.sg_forest(150, window=12, seed=5)
  db = run('sg', {'Arc': e})
  want, _ = oracle.run_plan(load_plan('sg'), {'Arc': e})
  assert rows_set(db.dump('Sg')) == set(want['Sg'])


def test_triangle_known_answers():
  import math
  for n in (3, 5, 40):
    e = np.array([(i, j) for i in range(n) for j in range(i + 1, n)], np.uint32)
    db = run('triangle', {'KnowsInput': e})
    assert db.count('TriangleJoin') == math.comb(n, 3)
  db = run('triangle', {'KnowsInput': np.zeros((0, 2), np.uint32)})
  assert db.count('TriangleJoin') == 0


@pytest.mark.parametrize('name,scale,draws,seed', [('triangle_rmat14', 14, 1 << 18, 5),
                                                    ('triangle_rmat20', 20, 1 << 24, 3)])
def test_triangle_configs(expected, name, scale, draws, seed):
  e = W.rmat_edges(scale, draws, seed=seed)
  db = run('triangle', {'KnowsInput': e})
  assert db.count('TriangleJoin') == expected[name]['count']
  assert db.size('Knows') == expected[name]['edges']


def test_shim_end_to_end(tmp_path, expected):
  from srdatalog_b200.build import CompilerConfig, compile_jit_project, write_project
  proj = write_project(load_plan('tc'), 'TcPlan', cache_base=str(tmp_path))
  br = compile_jit_project(proj, CompilerConfig())
  assert br.ok()
  lib = ctypes.CDLL(br.artifact)
  lib.srdatalog_load_all.argtypes = [ctypes.c_char_p]
  lib.srdatalog_run.argtypes = [ctypes.c_ulonglong]
  lib.srdatalog_size.argtypes = [ctypes.c_char_p]
  lib.srdatalog_size.restype = ctypes.c_ulonglong
  lib.srdatalog_dump.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_uint32), ctypes.c_ulonglong]
  lib.srdatalog_dump.restype = ctypes.c_longlong
  W.write_csv(W.uniform_edges(2000, 6000, 7), str(tmp_path / 'Arc.csv'))
  assert lib.srdatalog_init() == 0
  assert lib.srdatalog_load_all(str(tmp_path).encode()) == 0
  assert lib.srdatalog_run(0) == 0
  n = lib.srdatalog_size(b'Path')
  assert n == expected['tc_mid']['size']
  buf = np.empty((n, 2), np.uint32)
  assert lib.srdatalog_dump(b'Path', buf.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), n) == n
  assert oracle.dump_hash(buf) == expected['tc_mid']['sha256']
  digest = ctypes.create_string_buffer(32)
  assert lib.srdatalog_hash(b'Path', digest) == 0   # computed in the library
  assert digest.raw.hex() == expected['tc_mid']['sha256']
  assert lib.srdatalog_shutdown() == 0


def test_library_hash_matches_oracle(expected):
  db = run('sg', {'Arc': W.sg_forest(2000, seed=4)})
  assert db.hash('Sg') == expected['sg_2k']['sha256'] == oracle.dump_hash(db.dump('Sg'))
  t = run('triangle', {'KnowsInput': W.rmat_edges(12, 40000, seed=5)})
  assert t.hash('Knows') == oracle.dump_hash(t.dump('Knows'))


@pytest.mark.parametrize('pivot_min', [512, 4096])
def test_triangle_pivot_kernel(expected, pivot_min):
  '''The pivot kernel (option pivot_min: rows probing a long bitmapped list
  of the table's first column counted with that bitmap in shared memory)
  gives the same counts as the default path, on R-MAT scale 14 and 20.'''
  for name, scale, draws, seed in (('triangle_rmat14', 14, 1 << 18, 5), ('triangle_rmat20', 20, 1 << 24, 3)):
    e = W.rmat_edges(scale, draws, seed=seed)
    db = native.Database(load_plan('triangle'))
    db.set_option('pivot_min', pivot_min)
    db.load_rows('KnowsInput', e)
    db.run()
    assert db.count('TriangleJoin') == expected[name]['count'], name


def test_triangle_large_ids_sparse_path():
  '''Ids spread over the whole uint32 range leave the dense directory (and the
  hashed child lists) unused: lookups binary-search the keys.  Relabelling
  the graph injectively leaves the count unchanged.'''
  e = W.rmat_edges(14, 1 << 18, seed=5).astype(np.uint64)
  relabel = ((e * np.uint64(2654435761)) % np.uint64(4294967291)).astype(np.uint32)
  db = run('triangle', {'KnowsInput': relabel})
  assert db.count('TriangleJoin') == oracle.triangle_count(relabel)
  db2 = run('triangle', {'KnowsInput': e.astype(np.uint32)})
  assert db2.count('TriangleJoin') == db.count('TriangleJoin')


@pytest.mark.parametrize('plan_name', ['tc', 'tc_lsm'])
def test_batched_union_matches_each_instance(plan_name):
  '''Independent TC instances evaluated as one disjoint union give each
  instance exactly its own closure (checked against the oracle per instance,
  and against the one-at-a-time loop through the same library).'''
  from srdatalog_b200.batch import BatchRun
  insts = [{'ArcInput': W.er_instance(n, c, seed=500 + j)}
           for j, (n, c) in enumerate([(16, 2.0), (40, 3.5), (120, 1.5), (200, 2.5), (64, 8.0),
                                       (3, 1.0), (90, 2.2), (150, 4.0)] * 6)]
  br = BatchRun(load_plan(plan_name), insts)
  per = br.split_rows('Path')
  sizes = br.sizes('Path')
  plain = native.Database(load_plan('tc'))
  for j, inst in enumerate(insts):
    keys, _, _ = oracle.tc(inst['ArcInput'])
    want = oracle.unpack(keys, order=(1, 0))
    assert sizes[j] == want.shape[0]
    assert oracle.dump_hash(per[j]) == oracle.dump_hash(want)
    if j < 8:
      plain.clear_inputs()
      plain.load_rows('ArcInput', inst['ArcInput'])
      plain.run()
      assert plain.size('Path') == want.shape[0]


def test_batched_triangle_counts_per_instance():
  '''Count-only rules over a disjoint union report each instance's count
  through grouped counting (srdl_set_count_groups).'''
  from srdatalog_b200.batch import BatchRun
  insts = [{'KnowsInput': W.rmat_edges(s, d, seed=40 + j)}
           for j, (s, d) in enumerate([(8, 3000), (10, 20000), (6, 500), (12, 60000), (9, 7000)] * 4)]
  insts.append({'KnowsInput': np.array([(i, j) for i in range(30) for j in range(i + 1, 30)],
                                       np.uint32)})
  br = BatchRun(load_plan('triangle'), insts)
  counts = br.counts('TriangleJoin')
  want = [oracle.triangle_count(i['KnowsInput']) for i in insts]
  assert [int(c) for c in counts] == want
  assert br.db.count('TriangleJoin') == sum(want)


def with_index_type(plan: dict, rel: str, index_type: str) -> dict:
  import copy
  p = copy.deepcopy(plan)
  for r in p['relations']:
    if r['name'] == rel:
      r['index_type'] = index_type
  return p


@pytest.mark.parametrize('plan_name,rel,make', [
  ('tc', 'Path', lambda: W.uniform_edges(2000, 6000, 7)),
  ('tc_left', 'Path', lambda: W.uniform_edges(1500, 4000, 9)),
  ('tc', 'Path', lambda: np.array([(i, i + 1) for i in range(300)], np.uint32)),
])
def test_two_level_index_matches_single_array(plan_name, rel, make):
  '''Device2LevelIndex (HEAD + FULL, merged at a tenth of FULL and at the end
  of the stratum) gives the same relation as the single sorted array, also
  when a run stops after a few iterations with a non-empty HEAD.'''
  e = make()
  base = load_plan(plan_name)
  lsm = with_index_type(base, rel, 'SRDatalog::GPU::Device2LevelIndex')
  inp = 'ArcInput'
  for max_iters in (0, 3, 17):
    a = native.Database(base)
    a.load_rows(inp, e)
    a.run(max_iters)
    b = native.Database(lsm)
    b.load_rows(inp, e)
    b.run(max_iters)
    assert b.size(rel) == a.size(rel)
    assert oracle.dump_hash(b.dump(rel)) == oracle.dump_hash(a.dump(rel))


def test_sg_two_level_vs_single_array(expected):
  '''The SG plan declares Sg as Device2LevelIndex; the single-array policy
  gives the same relation.'''
  e = W.sg_forest(2000, seed=4)
  plain = with_index_type(load_plan('sg'), 'Sg', '')
  a = native.Database(plain)
  a.load_rows('Arc', e)
  a.run()
  assert a.size('Sg') == expected['sg_2k']['size']
  assert oracle.dump_hash(a.dump('Sg')) == expected['sg_2k']['sha256']


@pytest.mark.parametrize('n,m,seed', [(50, 140, 0), (300, 700, 1), (1000, 1600, 2)])
def test_andersen_vs_rules(n, m, seed):
  '''Andersen points-to (non-linear Load/Store rules with per-delta orders, a
  parallel group, an injected hook) against the naive rule restatement.'''
  inp = W.andersen_inputs(n, m, seed)
  db = native.Database(load_plan('andersen'))
  for rel, rows in inp.items():
    db.load_rows(rel, rows)
  db.run()
  want = np.array(oracle.andersen(inp), np.uint32).reshape(-1, 2)
  assert db.size('PointsTo') == want.shape[0]
  assert oracle.dump_hash(db.dump('PointsTo')) == oracle.dump_hash(want)


@pytest.mark.parametrize('n,m,seed', [(40, 90, 0), (150, 260, 1), (300, 380, 2)])
def test_cspa_vs_rules(n, m, seed):
  '''CSPA (five mutually recursive relations, anonymous variables) against the
  naive rule restatement.'''
  inp = W.cspa_inputs(n, m, seed)
  db = native.Database(load_plan('cspa'))
  for rel, rows in inp.items():
    db.load_rows(rel, rows)
  db.run()
  want = oracle.cspa(inp)
  for rel in ('ValueFlow', 'ValueAlias', 'MemoryAlias'):
    w = np.array(want[rel], np.uint32).reshape(-1, 2)
    assert db.size(rel) == w.shape[0], rel
    assert oracle.dump_hash(db.dump(rel)) == oracle.dump_hash(w), rel


@pytest.mark.parametrize('n_msgs,seed', [(60, 0), (5000, 1), (400_000, 2)])
def test_lsqb_q7_negation_counts(n_msgs, seed):
  '''LSQB Q7: four-source column join, wide count-only heads and negations of
  unary relations, against the closed-form counts.'''
  inp = W.lsqb_q7_inputs(n_msgs, seed)
  db = native.Database(load_plan('lsqb_q7'))
  for rel, rows in inp.items():
    db.load_rows(rel, rows)
  db.run()
  want = oracle.lsqb_q7(inp)
  got = {rule: db.count(rule) for rule in want}
  assert got == want
  assert db.size('HasReply') == len(set(inp['ReplyOf'][:, 1].tolist()))


@pytest.mark.parametrize('n,m,seed', [(40, 90, 0), (20_000, 200_000, 1), (300_000, 2_400_000, 2)])
def test_lsqb_q6_two_hop_counts(n, m, seed):
  '''LSQB Q6: Knows loaded by two rules (both directions), a filtered
  count-only 2-hop, against the closed form.'''
  inp = W.lsqb_q6_inputs(n, m, seed)
  db = native.Database(load_plan('lsqb_q6'))
  for rel, rows in inp.items():
    db.load_rows(rel, rows)
  db.run()
  assert db.count('TwoHopPath') == oracle.lsqb_q6(inp)


def test_autotune_on_device():
  '''The tuner's runs on the GPU agree on the result, and the tuned setting
  reproduces it.'''
  from srdatalog_b200.autotune import autotune
  e = W.uniform_edges(1500, 5000, 3)
  plan = load_plan('tc')
  res = autotune(plan, {'ArcInput': e}, reps=1, space={'bitmap_mb': [0, 256], 'lsm_compact_pct': [10]})
  db = native.Database(res.apply(plan))
  res.configure(db)
  db.load_rows('ArcInput', e)
  db.run()
  keys, _, _ = oracle.tc(e)
  assert db.size('Path') == keys.shape[0]
  assert len(res.trials) >= 2


@pytest.mark.parametrize('n,m,seed', [(30, 70, 0), (400, 1500, 1), (20_000, 24_000, 2)])
def test_reach_avoid_negation(n, m, seed):
  '''Negation of a binary relation on two bound variables, inside the
  recursive step and in a later stratum over the recursive result.'''
  e = W.uniform_edges(n, m, seed)
  blocked = np.concatenate([e[::3], W.uniform_edges(n, m // 4, seed + 10)])
  db = native.Database(load_plan('reach_avoid'))
  db.load_rows('Edge', e)
  db.load_rows('Blocked', blocked)
  db.run()
  want = oracle.reach_avoid(e, blocked)
  for rel in ('Reach', 'Cut'):
    w = np.array(want[rel], np.uint32).reshape(-1, 2)
    assert db.size(rel) == w.shape[0], rel
    assert oracle.dump_hash(db.dump(rel)) == oracle.dump_hash(w), rel


@pytest.mark.parametrize('n,m,seed', [(60, 90, 0), (3000, 7000, 3)])
def test_head_constants(n, m, seed):
  '''Head constants (constant-bind joins over the plan's one-tuple
  relations) and body constants, inside a recursive stratum; a second run
  after clear_inputs still sees the plan's facts.'''
  e = W.uniform_edges(n, m, seed)
  src = np.array([[seed], [seed + 11]], np.uint32)
  want = np.array(oracle.head_const(e, src), np.uint32).reshape(-1, 2)
  db = native.Database(load_plan('head_const'))
  for _ in range(2):
    db.clear_inputs()
    db.load_rows('ArcInput', e)
    db.load_rows('SourceInput', src)
    db.run()
    assert db.size('Mark') == want.shape[0]
    assert oracle.dump_hash(db.dump('Mark')) == oracle.dump_hash(want)


@pytest.mark.parametrize('n,m,seed', [(12, 40, 0), (20, 120, 1), (30, 150, 2), (40, 180, 6)])
def test_galen_ternary_joins(n, m, seed):
  '''Galen: ternary inputs and the recursive ternary OutQ read in three
  column orders with 0, 1 and 2 bound columns, and cartesian sources
  binding two of its columns; bit-exact against the rules restated on sets.'''
  inp = W.galen_inputs(n, m, seed)
  want = oracle.galen(inp)
  db = run('galen', inp)
  for rel, k in (('OutP', 2), ('OutQ', 3)):
    w = np.array(want[rel], np.uint32).reshape(-1, k)
    assert db.size(rel) == w.shape[0], rel
    assert oracle.dump_hash(db.dump(rel)) == oracle.dump_hash(w), rel


@pytest.mark.parametrize('name', ['live', 'live_lsm'])
@pytest.mark.parametrize('n,m,seed', [(30, 60, 0), (30, 60, 1), (400, 1500, 2), (3000, 9000, 3)])
def test_live_rebuilt_full_permutation(name, n, m, seed):
  '''A relation stored in order (1, 0), merged only in that order by its
  recursive stratum, then read in order (0, 1) by a later stratum after the
  plan's RebuildIndex(FULL, (0, 1)): that permutation is rebuilt from the
  up-to-date one (single array and Device2LevelIndex), bit-exact against the
  rules restated on sets.'''
  plan = load_plan(name)
  inp = W.plan_inputs(plan, n, m, seed)
  want = oracle.live(inp)
  db = run(name, inp)
  for rel in ('Live', 'Out'):
    w = np.array(want[rel], np.uint32).reshape(-1, 2)
    assert db.size(rel) == w.shape[0], rel
    assert oracle.dump_hash(db.dump(rel)) == oracle.dump_hash(w), rel


@pytest.mark.parametrize('n,m,seed', [(10, 8, 0), (24, 20, 2), (32, 30, 3)])
def test_polonius_vs_interpreter(n, m, seed):
  '''Polonius (the reference's examples/polonius_test.py): every relation
  equal to the oracle's plan interpreter on uniform facts.'''
  plan = load_plan('polonius')
  inp = W.plan_inputs(plan, n, m, seed)
  want, _ = oracle.run_plan(plan, inp)
  db = run('polonius', inp)
  arity = {r['name']: r['arity'] for r in plan['relations']}
  assert sum(len(v) for v in want.values()) > sum(len(v) for v in inp.values())
  for rel, rows in want.items():
    w = np.array(rows, np.uint32).reshape(-1, arity[rel])
    assert db.size(rel) == w.shape[0], rel
    assert oracle.dump_hash(db.dump(rel)) == oracle.dump_hash(w), rel


@pytest.mark.parametrize('radix_bits,jbpsm', [(5, 8), (6, 32), (7, 16), (8, 1)])
def test_tuning_options_keep_results(expected, radix_bits, jbpsm):
  '''The autotuner's sort-digit and join-grid knobs change no result.'''
  e = W.uniform_edges(2000, 6000, 7)
  db = native.Database(load_plan('tc'))
  db.set_option('radix_bits', radix_bits)
  db.set_option('join_blocks_per_sm', jbpsm)
  db.load_rows('ArcInput', e)
  db.run()
  assert db.size('Path') == expected['tc_mid']['size']
  assert oracle.dump_hash(db.dump('Path')) == expected['tc_mid']['sha256']
  t = native.Database(load_plan('triangle'))
  t.set_option('radix_bits', radix_bits)
  t.set_option('join_blocks_per_sm', jbpsm)
  t.load_rows('KnowsInput', W.rmat_edges(14, 1 << 18, seed=5))
  t.run()
  assert t.count('TriangleJoin') == expected['triangle_rmat14']['count']


@pytest.mark.parametrize('n,m,seed', [(60, 400, 0), (3000, 60_000, 1)])
def test_lsqb_q3_materialised_arity3(n, m, seed):
  '''LSQB Q3: a materialised arity-3 relation (packed keys), nine atoms, a
  three-source column join; bit-exact against the set restatement.'''
  inp = W.lsqb_q3_inputs(n, m, seed)
  db = run('lsqb_q3', inp)
  want = np.array(oracle.lsqb_q3(inp), np.uint32).reshape(-1, 3)
  assert db.size('Triangle') == want.shape[0]
  assert oracle.dump_hash(db.dump('Triangle')) == oracle.dump_hash(want)
  assert db.hash('Triangle') == oracle.dump_hash(want)


@pytest.mark.parametrize('plan_name,second', [('lsqb_q6_2hop', None), ('lsqb_q6_nosj', 'KnowsInput2')])
@pytest.mark.parametrize('n,m,seed', [(40, 150, 0), (3000, 30_000, 1)])
def test_lsqb_two_hop_materialised_arity4(plan_name, second, n, m, seed):
  inp = (W.lsqb_q6_nosj_inputs if second else W.lsqb_q6_inputs)(n, m, seed)
  db = run(plan_name, inp)
  want = np.array(sorted(oracle.lsqb_two_hop(inp, second)), np.uint32).reshape(-1, 4)
  assert db.size('Path') == want.shape[0]
  assert oracle.dump_hash(db.dump('Path')) == oracle.dump_hash(want)


@pytest.mark.parametrize('n,m,seed', [(40, 150, 0), (5000, 40_000, 2)])
def test_lsqb_q9_negated_two_hop_count(n, m, seed):
  inp = W.lsqb_q6_inputs(n, m, seed)
  db = run('lsqb_q9', inp)
  assert db.count('NegPath') == len(oracle.lsqb_two_hop(inp, negate=True))


def test_arity4_beyond_64_bits_is_refused():
  '''Four columns of 20-bit values do not pack into 64 bits: the run fails
  with a clear status instead of truncating.'''
  inp = W.lsqb_q6_inputs(40, 150, 0)
  inp['HasInterestInput'] = np.concatenate([inp['HasInterestInput'],
                                            np.array([[3, 1_000_000]], np.uint32)])
  db = native.Database(load_plan('lsqb_q6_2hop'))
  for rel, rows in inp.items():
    db.load_rows(rel, rows)
  with pytest.raises(native.SrdlError, match='arity x value bits'):
    db.run()


@pytest.mark.parametrize('n,m,seed', [(30, 200, 0), (2000, 40_000, 1)])
def test_arity3_triangle_programs(n, m, seed):
  '''examples/debug_triangle.py and gen_jit_code.py: directed triangles
  materialised into arity-3 relations, from rows loaded straight into
  relations without input files.'''
  r, s, t = (W.uniform_edges(n, m, seed + k) for k in (1, 2, 3))
  db = run('debug_triangle', {'RRel': r, 'SRel': s, 'TRel': t})
  want = np.array(oracle.triangle3(r, s, t), np.uint32).reshape(-1, 3)
  assert db.size('ZRel') == want.shape[0]
  assert oracle.dump_hash(db.dump('ZRel')) == oracle.dump_hash(want)
  db = run('gen_jit_triangle', {'Edge': r})
  want = np.array(oracle.triangle3(r, r, r), np.uint32).reshape(-1, 3)
  assert db.size('Z') == want.shape[0]
  assert oracle.dump_hash(db.dump('Z')) == oracle.dump_hash(want)


@pytest.mark.parametrize('n,m,seed', [(40, 150, 0), (300, 2500, 1), (2000, 12000, 2)])
def test_triangle_db_program(n, m, seed):
  '''examples/triangle.py: ZRel(x,y,z) <= RRel(x,y), SRel(y,z,h), TRel(z,x,f)
  (the ternary relations' third columns projected away), against the plan
  interpreter.'''
  rng = np.random.default_rng(seed)
  r = W.uniform_edges(n, m, seed + 1)
  s = rng.integers(0, n, (m, 3)).astype(np.uint32)
  t = rng.integers(0, n, (m, 3)).astype(np.uint32)
  inp = {'RRel': r, 'SRel': s, 'TRel': t}
  # the directed-triangle oracle over the projections (y,z) of SRel and
  # (z,x) of TRel; the plan interpreter agrees on the smallest input
  w = np.array(oracle.triangle3(r, np.unique(s[:, :2], axis=0), np.unique(t[:, :2], axis=0)),
               np.uint32).reshape(-1, 3)
  if n <= 40:
    want, _ = oracle.run_plan(load_plan('triangle_db'), inp)
    assert oracle.dump_hash(np.array(sorted(want['ZRel']), np.uint32).reshape(-1, 3)) == oracle.dump_hash(w)
  db = run('triangle_db', inp)
  assert db.size('ZRel') == w.shape[0] > 0
  assert oracle.dump_hash(db.dump('ZRel')) == oracle.dump_hash(w)


@pytest.mark.parametrize('n,m,seed', [(20, 60, 0), (60, 400, 1), (3000, 40000, 2)])
def test_negation_forms_program(n, m, seed):
  '''Negation with a constant argument and over a ternary relation (one or
  two bound columns, around a wildcard, with a constant): every output
  equals the plan interpreter's.'''
  from test_negation_forms import expected, inputs
  inp = inputs(n, m, seed)
  want = expected(inp)
  if n <= 60:
    got, _ = oracle.run_plan(load_plan('neg_forms'), inp)
    for rel, rows in want.items():
      assert set(got[rel]) == rows, rel
  db = run('neg_forms', inp)
  for rel, rows in want.items():
    w = np.array(sorted(rows), np.uint32).reshape(-1, 2)
    assert db.size(rel) == w.shape[0], rel
    assert oracle.dump_hash(db.dump(rel)) == oracle.dump_hash(w), rel


def test_tc_2level_bg_program(expected):
  exp = expected['tc_mid']
  db = run('tc_2level_bg', {'ArcInput': W.uniform_edges(2000, 6000, 7)})
  assert db.size('Path') == exp['size']
  assert oracle.dump_hash(db.dump('Path')) == exp['sha256']


def test_lsqb_q6_bg_program():
  inp = W.lsqb_q6_nosj_inputs(3000, 30_000, 3)
  db = run('lsqb_q6_bg', inp)
  want = np.array(sorted(oracle.lsqb_two_hop(inp, 'KnowsInput2', as_planned=False)),
                  np.uint32).reshape(-1, 4)
  assert db.size('PathBG') == want.shape[0]
  assert oracle.dump_hash(db.dump('PathBG')) == oracle.dump_hash(want)


@pytest.mark.parametrize('n,m,seed', [(50, 140, 0), (1000, 1600, 2)])
def test_print_mir_program(n, m, seed):
  '''examples/print_mir.py: the Andersen rules with another plan for Load's
  second delta, against the naive restatement.'''
  inp = W.andersen_inputs(n, m, seed)
  db = run('print_mir', inp)
  want = np.array(oracle.andersen(inp), np.uint32).reshape(-1, 2)
  assert db.size('PointsTo') == want.shape[0]
  assert oracle.dump_hash(db.dump('PointsTo')) == oracle.dump_hash(want)
