'''The Datalog programs exercised by the tests and the bench, written in the
srdatalog DSL (src/srdatalog/dsl.py: Var 48, Relation 449, Program 507).

Relation and rule names follow the reference's benchmark programs
(examples/tc.py, examples/sg.py, examples/lsqb_triangle_count.py) so that
the MIR they lower to is the one pinned by the reference's fixtures
(tests/fixtures/tc.mir.sexpr, tests/fixtures/integration/sg.mir.sexpr,
tests/fixtures/integration/lsqb_triangle_count.mir.sexpr).

Importing this module needs the srdatalog front end; the committed plan
JSON files next to it are what the GPU tests and the bench load.
'''

from __future__ import annotations

from srdatalog.dsl import Filter, Program, Relation, Var


def tc_program() -> Program:
  '''Transitive closure: Path(x,y) <= Edge(x,y); Path(x,z) <= Path(x,y), Edge(y,z).'''
  arc = Relation('ArcInput', 2, column_types=(int, int), input_file='Arc.csv')
  edge = Relation('Edge', 2, column_types=(int, int))
  path = Relation('Path', 2, column_types=(int, int), print_size=True)
  x, y, z = Var('x'), Var('y'), Var('z')
  return Program(rules=[
    (edge(x, y) <= arc(x, y)).named('EdgeLoad'),
    (path(x, y) <= edge(x, y)).named('TCBase'),
    (path(x, z) <= path(x, y) & edge(y, z)).named('TCRec'),
  ])


def sg_program() -> Program:
  '''Same generation, with the reference's variable orders and LSM index hint.'''
  arc = Relation('Arc', 2, column_types=(int, int), input_file='Arc.csv')
  sg = Relation('Sg', 2, column_types=(int, int), print_size=True,
                index_type='SRDatalog::GPU::Device2LevelIndex')
  p, q, x, y = Var('p'), Var('q'), Var('x'), Var('y')
  return Program(rules=[
    (sg(x, y) <= arc(p, x) & arc(p, y) & Filter(('x', 'y'), 'return x != y;'))
    .named('SGBase').with_plan(var_order=['p', 'x', 'y']),
    (sg(x, y) <= arc(p, x) & sg(p, q) & arc(q, y))
    .named('SGRec').with_plan(var_order=['p', 'q', 'x', 'y']),
  ])


def triangle_program() -> Program:
  '''Count-only 3-way WCOJ: Triangle(a,b,c) <= Knows(a,b), Knows(b,c), Knows(a,c).'''
  kin = Relation('KnowsInput', 2, column_types=(int, int),
                 input_file='Person_knows_Person.csv')
  knows = Relation('Knows', 2, column_types=(int, int))
  tri = Relation('Triangle', 3, column_types=(int, int, int))
  a, b, c, x, y = Var('a'), Var('b'), Var('c'), Var('x'), Var('y')
  return Program(rules=[
    (knows(x, y) <= kin(x, y)).named('KnowsLoad'),
    (tri(a, b, c) <= knows(a, b) & knows(b, c) & knows(a, c))
    .named('TriangleJoin').with_plan(var_order=['a', 'b', 'c']).with_count(),
  ])


def tc_lsm_program() -> Program:
  '''TC with the Device2LevelIndex hint on Path (the index-policy hook of
  the DSL, examples/sg.py:30): same MIR as tc, FULL kept as HEAD + FULL.'''
  arc = Relation('ArcInput', 2, column_types=(int, int), input_file='Arc.csv')
  edge = Relation('Edge', 2, column_types=(int, int))
  path = Relation('Path', 2, column_types=(int, int), print_size=True,
                  index_type='SRDatalog::GPU::Device2LevelIndex')
  x, y, z = Var('x'), Var('y'), Var('z')
  return Program(rules=[
    (edge(x, y) <= arc(x, y)).named('EdgeLoad'),
    (path(x, y) <= edge(x, y)).named('TCBase'),
    (path(x, z) <= path(x, y) & edge(y, z)).named('TCRec'),
  ])


def tc_left_program() -> Program:
  '''Left-recursive TC variant (Path(x,z) <= Edge(x,y), Path(y,z)): a second
  join shape whose delta index is (0,1); no reference fixture pins it.'''
  arc = Relation('ArcInput', 2, column_types=(int, int), input_file='Arc.csv')
  edge = Relation('Edge', 2, column_types=(int, int))
  path = Relation('Path', 2, column_types=(int, int), print_size=True)
  x, y, z = Var('x'), Var('y'), Var('z')
  return Program(rules=[
    (edge(x, y) <= arc(x, y)).named('EdgeLoad'),
    (path(x, y) <= edge(x, y)).named('TCBase'),
    (path(x, z) <= edge(x, y) & path(y, z)).named('TCRecL'),
  ])


def _bin(name: str, input_file: str | None = None, print_size: bool = False) -> Relation:
  kw = {'column_types': (int, int), 'print_size': print_size}
  if input_file:
    kw['input_file'] = input_file
  return Relation(name, 2, **kw)


def andersen_program() -> Program:
  '''Andersen points-to analysis (examples/andersen.py): two non-linear
  rules (Load, Store) with per-delta variable orders, a parallel group of
  five pipelines per iteration, and an injected C++ hook on Store.'''
  address_of = _bin('AddressOf', 'addressOf.csv')
  assign = _bin('Assign', 'assign.csv')
  load = _bin('Load', 'load.csv')
  store = _bin('Store', 'store.csv')
  points_to = _bin('PointsTo', print_size=True)
  w, x, y, z = Var('w'), Var('x'), Var('y'), Var('z')
  return Program(rules=[
    (points_to(y, x) <= address_of(y, x)).named('Base').with_plan(var_order=['y', 'x']),
    (points_to(y, x) <= points_to(z, x) & assign(y, z))
    .named('Assign').with_plan(var_order=['z', 'x', 'y']),
    (points_to(y, w) <= points_to(x, z) & load(y, x) & points_to(z, w))
    .named('Load')
    .with_plan(delta=0, var_order=['x', 'z', 'y', 'w'])
    .with_plan(delta=2, var_order=['z', 'x', 'y', 'w']),
    (points_to(z, w) <= points_to(y, z) & store(y, x) & points_to(x, w))
    .named('Store')
    .with_plan(delta=0, var_order=['y', 'x', 'z', 'w'])
    .with_plan(delta=2, var_order=['x', 'y', 'w', 'z'])
    .with_inject_cpp('// report PointsTo delta / full sizes'),
  ])


def cspa_program() -> Program:
  '''Context-sensitive points-to (examples/cspa.py): five mutually recursive
  binary relations, anonymous variables, three-atom joins.'''
  assign_in = Relation('AssignInput', 2, input_file='Assign.csv')
  deref_in = Relation('DerefInput', 2, input_file='Dereference.csv')
  assign, deref = Relation('Assign', 2), Relation('Deref', 2)
  vf = Relation('ValueFlow', 2, print_size=True)
  va = Relation('ValueAlias', 2, print_size=True)
  ma = Relation('MemoryAlias', 2, print_size=True)
  w, x, y, z = Var('w'), Var('x'), Var('y'), Var('z')
  return Program(rules=[
    (assign(x, y) <= assign_in(x, y)).named('LoadAssign'),
    (deref(x, y) <= deref_in(x, y)).named('LoadDeref'),
    (vf(y, x) <= assign(y, x)).named('VF_Assign'),
    (vf(x, x) <= assign(x, Var('_'))).named('VF_Refl1'),
    (vf(x, x) <= assign(Var('_'), x)).named('VF_Refl2'),
    (ma(x, x) <= assign(Var('_'), x)).named('MA_Refl1'),
    (ma(x, x) <= assign(x, Var('_'))).named('MA_Refl2'),
    (vf(x, y) <= vf(x, z) & vf(z, y)).named('VF_Trans').with_plan(var_order=['z', 'x', 'y']),
    (vf(x, y) <= assign(x, z) & ma(z, y))
    .named('VF_Assign_MA').with_plan(var_order=['z', 'x', 'y']),
    (va(x, y) <= vf(z, x) & vf(z, y)).named('VA_VF').with_plan(var_order=['z', 'x', 'y']),
    (va(x, y) <= vf(z, x) & ma(z, w) & vf(w, y))
    .named('VA_VF_MA_VF').with_plan(var_order=['z', 'w', 'x', 'y']),
    (ma(x, w) <= deref(y, x) & va(y, z) & deref(z, w))
    .named('MA_Deref_VA').with_plan(var_order=['y', 'z', 'x', 'w']),
  ])


def lsqb_q7_program() -> Program:
  '''LSQB Q7 "optional" (examples/lsqb_q7_optional.py): messages with tags and
  creators, counted by whether they have replies and likes; the two
  "without" cases are negations of unary relations.'''
  has_tag = Relation('HasTag', 2, input_file='Message_hasTag_Tag.csv')
  has_creator = Relation('HasCreator', 2, input_file='Message_hasCreator_Person.csv')
  reply_of = Relation('ReplyOf', 2, input_file='ReplyOf_Comment_Message.csv')
  likes = Relation('Likes', 2, input_file='Person_likes_Message.csv')
  has_reply = Relation('HasReply', 1, column_types=(int,))
  has_liker = Relation('HasLiker', 1, column_types=(int,))
  case1 = Relation('Case1', 5, print_size=True)
  case2 = Relation('Case2', 4, print_size=True)
  case3 = Relation('Case3', 4, print_size=True)
  case4 = Relation('Case4', 3, print_size=True)
  c, comment, liker, m, t = Var('c'), Var('comment'), Var('liker'), Var('m'), Var('t')
  return Program(rules=[
    (has_reply(m) <= reply_of(Var('_'), m)).named('MarkHasReply'),
    (has_liker(m) <= likes(Var('_'), m)).named('MarkHasLiker'),
    (case1(m, t, c, comment, liker)
     <= has_tag(m, t) & has_creator(m, c) & reply_of(comment, m) & likes(liker, m))
    .named('Case1Both').with_plan(var_order=['m', 'comment', 'liker', 't', 'c']).with_count(),
    (case2(m, t, c, comment)
     <= has_tag(m, t) & has_creator(m, c) & reply_of(comment, m) & ~has_liker(m))
    .named('Case2ReplyOnly').with_plan(var_order=['m', 'comment', 't', 'c']).with_count(),
    (case3(m, t, c, liker) <= has_tag(m, t) & has_creator(m, c) & likes(liker, m) & ~has_reply(m))
    .named('Case3LikeOnly').with_plan(var_order=['m', 'liker', 't', 'c']).with_count(),
    (case4(m, t, c) <= has_tag(m, t) & has_creator(m, c) & ~has_reply(m) & ~has_liker(m))
    .named('Case4Neither').with_plan(var_order=['m', 't', 'c']).with_count(),
  ])


def lsqb_q6_program() -> Program:
  '''LSQB Q6 2-hop count (examples/lsqb_q6_count.py): Knows loaded in both
  directions by two rules, a count-only arity-4 head with a filter.'''
  knows_in = Relation('KnowsInput', 2, input_file='Person_knows_Person.csv')
  interest_in = Relation('HasInterestInput', 2, input_file='Person_hasInterest_Tag.csv')
  knows = Relation('Knows', 2)
  has_interest = Relation('HasInterest', 2)
  path = Relation('Path', 4)
  p, p1, p2, p3, t, x, y = (Var(n) for n in ('p', 'p1', 'p2', 'p3', 't', 'x', 'y'))
  return Program(rules=[
    (knows(x, y) <= knows_in(x, y)).named('KnowsLoad'),
    (knows(y, x) <= knows_in(x, y)).named('KnowsLoadRev'),
    (has_interest(p, t) <= interest_in(p, t)).named('InterestLoad'),
    (path(p1, p2, p3, t)
     <= knows(p1, p2) & knows(p2, p3) & has_interest(p3, t)
     & Filter(('p1', 'p3'), 'return p1 != p3;'))
    .named('TwoHopPath').with_plan(var_order=['p2', 'p3', 'p1', 't']).with_count(),
  ])


def lsqb_q3_program() -> Program:
  '''LSQB Q3 (examples/lsqb_q3_triangle.py): triangles of Knows whose three
  people live in cities of one country; the arity-3 Triangle is
  materialised (nine atoms, a three-source column join on the country).'''
  knows_in = Relation('KnowsInput', 2, column_types=(int, int), input_file='Person_knows_Person.csv')
  loc_in = Relation('IsLocatedInInput', 2, column_types=(int, int),
                    input_file='Person_isLocatedIn_City.csv')
  part_in = Relation('IsPartOfInput', 2, column_types=(int, int), input_file='City_isPartOf_Country.csv')
  knows = Relation('Knows', 2, column_types=(int, int))
  loc = Relation('IsLocatedIn', 2, column_types=(int, int))
  part = Relation('IsPartOf', 2, column_types=(int, int))
  tri = Relation('Triangle', 3, column_types=(int, int, int), print_size=True)
  c, c1, c2, c3, co = Var('c'), Var('c1'), Var('c2'), Var('c3'), Var('co')
  p, p1, p2, p3, x, y = Var('p'), Var('p1'), Var('p2'), Var('p3'), Var('x'), Var('y')
  return Program(rules=[
    (knows(x, y) <= knows_in(x, y)).named('KnowsLoad'),
    (loc(p, c) <= loc_in(p, c)).named('LocLoad'),
    (part(c, co) <= part_in(c, co)).named('PartOfLoad'),
    (tri(p1, p2, p3)
     <= knows(p1, p2) & knows(p2, p3) & knows(p3, p1)
     & loc(p1, c1) & loc(p2, c2) & loc(p3, c3)
     & part(c1, co) & part(c2, co) & part(c3, co))
    .named('LabeledTriangle').with_plan(var_order=['p1', 'p2', 'p3', 'c1', 'c2', 'c3', 'co']),
  ])


def _two_hop(second: str | None, count: bool, negate: bool = False, path_name: str = 'Path',
             print_size: bool = True):
  knows_in = Relation('KnowsInput', 2, column_types=(int, int), input_file='Person_knows_Person.csv')
  interest_in = Relation('HasInterestInput', 2, column_types=(int, int),
                         input_file='Person_hasInterest_Tag.csv')
  knows = Relation('Knows', 2, column_types=(int, int))
  has_interest = Relation('HasInterest', 2, column_types=(int, int))
  path = Relation(path_name, 4, column_types=(int, int, int, int), print_size=print_size)
  p, p1, p2, p3, t, x, y = (Var(n) for n in ('p', 'p1', 'p2', 'p3', 't', 'x', 'y'))
  rules = [(knows(x, y) <= knows_in(x, y)).named('KnowsLoad')]
  hop2 = knows
  if second:
    knows2_in = Relation('KnowsInput2', 2, column_types=(int, int), input_file='Person_knows_Person.csv')
    hop2 = Relation(second, 2, column_types=(int, int))
    rules.append((hop2(x, y) <= knows2_in(x, y)).named(second + 'Load'))
  rules.append((has_interest(p, t) <= interest_in(p, t)).named('InterestLoad'))
  body = knows(p1, p2) & hop2(p2, p3) & has_interest(p3, t)
  if negate:
    body = body & ~knows(p1, p3)
  body = body & Filter(('p1', 'p3'), 'return p1 != p3;')
  return path, p1, p2, p3, t, body, rules


def lsqb_q6_2hop_program() -> Program:
  '''LSQB Q6 two-hop (examples/lsqb_q6_2hop.py): the arity-4 Path of
  people two Knows hops apart with an interest of the last one, p1 != p3,
  materialised.'''
  path, p1, p2, p3, t, body, rules = _two_hop(None, False)
  return Program(rules=rules + [
    (path(p1, p2, p3, t) <= body).named('TwoHopPath').with_plan(var_order=['p1', 'p2', 'p3', 't'])])


def lsqb_q6_nosj_program() -> Program:
  '''LSQB Q6 without self-join (examples/lsqb_q6_nosj.py): the second hop
  over a second copy of Knows.'''
  path, p1, p2, p3, t, body, rules = _two_hop('Knows2', False)
  return Program(rules=rules + [
    (path(p1, p2, p3, t) <= body).named('TwoHopPath').with_plan(var_order=['p1', 'p2', 'p3', 't'])])


def lsqb_q9_program() -> Program:
  '''LSQB Q9 (examples/lsqb_q9_neg2hop.py): two-hop paths whose ends do not
  know each other, counted: a negation of a binary relation on two bound
  variables in a count-only arity-4 rule.'''
  path, p1, p2, p3, t, body, rules = _two_hop(None, True, negate=True)
  return Program(rules=rules + [
    (path(p1, p2, p3, t) <= body).named('NegPath')
    .with_plan(var_order=['p2', 'p3', 'p1', 't']).with_count()])


def lsqb_q6_bg_program() -> Program:
  '''LSQB Q6 with the block-group plan hint (examples/lsqb_q6_bg_test.py):
  the no-self-join two-hop into an arity-4 PathBG, variables ordered p2
  first.'''
  path, p1, p2, p3, t, body, rules = _two_hop('Knows2', False, path_name='PathBG', print_size=False)
  return Program(rules=rules + [
    (path(p1, p2, p3, t) <= body).named('TwoHopBG')
    .with_plan(var_order=['p2', 'p3', 'p1', 't'], block_group=True)])


def _triangle3(names, rule_name: str) -> Program:
  '''A directed triangle materialised into an arity-3 relation:
  Z(x,y,z) <= A(x,y), B(y,z), C(z,x) over binary relations without input
  files (loaded as rows).'''
  rels = {n: Relation(n, 2, column_types=(int, int)) for n in dict.fromkeys(names[:3])}
  z_rel = Relation(names[3], 3, column_types=(int, int, int))
  a, b, c = (rels[n] for n in names[:3])
  x, y, z = Var('x'), Var('y'), Var('z')
  return Program(rules=[
    (z_rel(x, y, z) <= a(x, y) & b(y, z) & c(z, x)).named(rule_name)
    .with_plan(var_order=['x', 'y', 'z'])])


def debug_triangle_program() -> Program:
  '''examples/debug_triangle.py: ZRel(x,y,z) <= RRel(x,y), SRel(y,z), TRel(z,x).'''
  return _triangle3(('RRel', 'SRel', 'TRel', 'ZRel'), 'TriangleDebug')


def gen_jit_triangle_program() -> Program:
  '''examples/gen_jit_code.py: Z(x,y,z) <= Edge(x,y), Edge(y,z), Edge(z,x).'''
  return _triangle3(('Edge', 'Edge', 'Edge', 'Z'), 'Triangle')


def triangle_db_program() -> Program:
  '''examples/triangle.py: ZRel(x,y,z) <= RRel(x,y), SRel(y,z,h), TRel(z,x,f)
  -- the third columns of the ternary SRel and TRel are projected away.'''
  r_rel = Relation('RRel', 2, column_types=(int, int))
  s_rel = Relation('SRel', 3, column_types=(int, int, int))
  t_rel = Relation('TRel', 3, column_types=(int, int, int))
  z_rel = Relation('ZRel', 3, column_types=(int, int, int))
  f, h, x, y, z = Var('f'), Var('h'), Var('x'), Var('y'), Var('z')
  return Program(rules=[
    (z_rel(x, y, z) <= r_rel(x, y) & s_rel(y, z, h) & t_rel(z, x, f)).named('Triangle')
    .with_plan(var_order=['x', 'y', 'z'])])


def neg_forms_program() -> Program:
  '''Negation with constant arguments and over a ternary relation (the
  forms of examples/reg_scc.py and crdt.py on relations of arity <= 3):
  a constant in a binary negation, two bound columns of a ternary one
  around a wildcard, a constant plus a variable, one bound column.'''
  e = Relation('Edge', 2, column_types=(int, int))
  b = Relation('Blocked', 2, column_types=(int, int))
  t = Relation('Tern', 3, column_types=(int, int, int))
  outs = [Relation(n, 2, column_types=(int, int)) for n in
          ('OutConst', 'OutTern2', 'OutTernConst', 'OutTern1')]
  x, y, w1, w2 = Var('x'), Var('y'), Var('_'), Var('_')
  return Program(rules=[
    (outs[0](x, y) <= e(x, y) & ~b(x, 3)).named('NegConst'),
    (outs[1](x, y) <= e(x, y) & ~t(x, w1, y)).named('NegTern2'),
    (outs[2](x, y) <= e(x, y) & ~t(5, y, w1)).named('NegTernConst'),
    (outs[3](x, y) <= e(x, y) & ~t(w1, w2, x)).named('NegTern1'),
  ])


def tc_2level_bg_program() -> Program:
  '''examples/tc_2level_bg.py: TC with Path as a Device2LevelIndex and the
  recursive rule planned y, x, z with the block-group hint.'''
  arc = Relation('ArcInput', 2, column_types=(int, int), input_file='Arc.csv')
  edge = Relation('Edge', 2, column_types=(int, int))
  path = Relation('Path', 2, column_types=(int, int), print_size=True,
                  index_type='SRDatalog::GPU::Device2LevelIndex')
  x, y, z = Var('x'), Var('y'), Var('z')
  return Program(rules=[
    (edge(x, y) <= arc(x, y)).named('EdgeLoad'),
    (path(x, y) <= edge(x, y)).named('TCBase'),
    (path(x, z) <= path(x, y) & edge(y, z)).named('TCRec')
    .with_plan(delta=0, var_order=['y', 'x', 'z'], block_group=True),
  ])


def print_mir_program() -> Program:
  '''examples/print_mir.py: the Andersen rules over relations without input
  files, the Load rule's second delta planned z, w, x, y.'''
  address_of, assign, load, store = (_bin(n) for n in ('AddressOf', 'Assign', 'Load', 'Store'))
  points_to = _bin('PointsTo')
  w, x, y, z = Var('w'), Var('x'), Var('y'), Var('z')
  return Program(rules=[
    (points_to(y, x) <= address_of(y, x)).named('Base').with_plan(var_order=['y', 'x']),
    (points_to(y, x) <= points_to(z, x) & assign(y, z))
    .named('Assign').with_plan(var_order=['z', 'x', 'y']),
    (points_to(y, w) <= points_to(x, z) & load(y, x) & points_to(z, w))
    .named('Load')
    .with_plan(delta=0, var_order=['x', 'z', 'y', 'w'])
    .with_plan(delta=2, var_order=['z', 'w', 'x', 'y']),
    (points_to(z, w) <= points_to(y, z) & store(y, x) & points_to(x, w))
    .named('Store')
    .with_plan(delta=0, var_order=['y', 'x', 'z', 'w'])
    .with_plan(delta=2, var_order=['x', 'y', 'w', 'z']),
  ])


def reach_avoid_program() -> Program:
  '''Reachability that avoids blocked edges, and the blocked pairs that are
  not reachable: negation of a binary relation on two bound variables, once
  inside a recursive stratum's join and once in a later stratum.  No
  reference fixture pins it (stratified negation exercised here only).'''
  edge = Relation('Edge', 2, column_types=(int, int), input_file='Edge.csv')
  blocked = Relation('Blocked', 2, column_types=(int, int), input_file='Blocked.csv')
  reach = Relation('Reach', 2, column_types=(int, int), print_size=True)
  cut = Relation('Cut', 2, column_types=(int, int), print_size=True)
  x, y, z = Var('x'), Var('y'), Var('z')
  return Program(rules=[
    (reach(x, y) <= edge(x, y) & ~blocked(x, y)).named('ReachBase'),
    (reach(x, z) <= reach(x, y) & edge(y, z) & ~blocked(y, z)).named('ReachStep'),
    (cut(x, y) <= blocked(x, y) & ~reach(x, y)).named('CutPairs'),
  ])


def rewrite_consts_program() -> Program:
  '''Body and head constants (the reference's tests/test_rule_rewrite.py:99,
  MIR pinned by tests/fixtures/rewrite_consts.mir.sexpr): P(x) <= In(x, 42, 99)
  lowers to a filter, Q(x, 7) <= In2(x) to a constant-bind.'''
  x = Var('x')
  inp = Relation('In', 3)
  in2 = Relation('In2', 1)
  p = Relation('P', 1)
  q = Relation('Q', 2)
  return Program(rules=[
    (p(x) <= inp(x, 42, 99)).named('BodyConst'),
    (q(x, 7) <= in2(x)).named('HeadConst'),
  ])


def head_const_program() -> Program:
  '''Head and body constants inside a recursive stratum: nodes reachable
  from the sources are tagged 7, their predecessors 9.  No reference fixture
  pins it (its constant-binds have the shape of rewrite_consts' HeadConst).'''
  arc = Relation('ArcInput', 2, column_types=(int, int), input_file='Arc.csv')
  src = Relation('SourceInput', 1, column_types=(int,), input_file='Source.csv')
  edge = Relation('Edge', 2, column_types=(int, int))
  mark = Relation('Mark', 2, column_types=(int, int), print_size=True)
  x, y = Var('x'), Var('y')
  return Program(rules=[
    (edge(x, y) <= arc(x, y)).named('EdgeLoad'),
    (mark(x, 7) <= src(x)).named('MarkSource'),
    (mark(y, 7) <= mark(x, 7) & edge(x, y)).named('MarkStep'),
    (mark(x, 9) <= edge(x, y) & mark(y, 7)).named('MarkPred'),
  ])


def galen_program() -> Program:
  '''examples/galen.py: the Galen ontology closure over the binary OutP and
  the ternary OutQ, with the reference's variable orders for Join3a and
  Join3c (MIR pinned by tests/fixtures/integration/galen.mir.sexpr).'''
  def rel(name, k, input_file=None, print_size=False):
    return Relation(name, k, column_types=(int,) * k, input_file=input_file,
                    print_size=print_size)
  p_in, s_in = rel('PInput', 2, 'P.csv'), rel('SInput', 2, 'S.csv')
  q_in, r_in = rel('QInput', 3, 'Q.csv'), rel('RInput', 3, 'R.csv')
  c_in, u_in = rel('CInput', 3, 'C.csv'), rel('UInput', 3, 'U.csv')
  out_p, out_q = rel('OutP', 2, print_size=True), rel('OutQ', 3, print_size=True)
  e, o, q, r, u, w, x, y, z = (Var(n) for n in 'eoqruwxyz')
  return Program(rules=[
    (out_p(x, z) <= p_in(x, z)).named('LoadP'),
    (out_q(x, r, z) <= q_in(x, r, z)).named('LoadQ'),
    (out_p(x, z) <= out_p(x, y) & out_p(y, z)).named('TC'),
    (out_q(x, r, z) <= out_p(x, y) & out_q(y, r, z)).named('PropQ'),
    (out_p(x, z) <= out_p(y, w) & u_in(w, r, z) & out_q(x, r, y))
    .named('Join3a').with_plan(delta=2, var_order=['y', 'w', 'r', 'x', 'z']),
    (out_p(x, z) <= c_in(y, w, z) & out_p(x, w) & out_p(x, y)).named('Join3b'),
    (out_q(x, q, z) <= out_q(x, r, z) & s_in(r, q)).named('PropQS'),
    (out_q(x, e, o) <= out_q(x, y, z) & r_in(y, u, e) & out_q(z, u, o))
    .named('Join3c').with_plan(delta=0, var_order=['z', 'y', 'u', 'x', 'e', 'o']),
  ])


def _live(index_type: str | None) -> Program:
  '''Backward liveness and a later read of it in the other column order:
  Live is stored in order (1, 0) (its recursive rule joins on column 1), so
  the later stratum's read Live(v, p) & Derefs(v, o) needs FULL (0, 1),
  which the recursive stratum never merges into: the planner inserts a
  RebuildIndex(FULL) for it after the stratum (src/srdatalog/mir/passes.py:
  104-145).  The shape of Polonius' var_live_on_entry and its ole_use read.'''
  used = _bin('Used', 'Used.csv')
  cfg = _bin('Cfg', 'Cfg.csv')
  derefs = _bin('Derefs', 'Derefs.csv')
  kw = {'column_types': (int, int), 'print_size': True}
  if index_type:
    kw['index_type'] = index_type
  live = Relation('Live', 2, **kw)
  out = Relation('Out', 2, column_types=(int, int), print_size=True)
  v, p, q, o = Var('v'), Var('p'), Var('q'), Var('o')
  return Program(rules=[
    (live(v, p) <= used(v, p)).named('LiveUsed'),
    (live(v, p) <= live(v, q) & cfg(p, q)).named('LiveStep'),
    (out(o, p) <= live(v, p) & derefs(v, o)).named('OutUse'),
  ])


def live_program() -> Program:
  return _live(None)


def live_lsm_program() -> Program:
  return _live('SRDatalog::GPU::Device2LevelIndex')


def polonius_program() -> Program:
  '''examples/polonius_test.py (Polonius borrow checking: 38 relations,
  five of them ternary, binary negations, two-column filters).  The program
  is the reference's own DSL module, loaded from the checkout that provides
  the srdatalog front end (its examples/ directory); its MIR is pinned by
  tests/fixtures/integration/polonius_test.mir.sexpr.'''
  import importlib.util
  import os

  import srdatalog
  root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(srdatalog.__file__))))
  spec = importlib.util.spec_from_file_location(
    'polonius_test', os.path.join(root, 'examples', 'polonius_test.py'))
  mod = importlib.util.module_from_spec(spec)
  spec.loader.exec_module(mod)
  return mod.build_poloniusdb_program()


# name -> (builder, project name, reference MIR fixture or None)
PROGRAMS = {
  'tc': (tc_program, 'TcPlan', 'tc.mir.sexpr'),
  'sg': (sg_program, 'SgPlan', 'integration/sg.mir.sexpr'),
  'triangle': (triangle_program, 'TrianglePlan', 'integration/lsqb_triangle_count.mir.sexpr'),
  'tc_left': (tc_left_program, 'TcLeftPlan', None),
  'tc_lsm': (tc_lsm_program, 'TcPlan', 'tc.mir.sexpr'),
  'andersen': (andersen_program, 'AndersenPlan', 'integration/andersen.mir.sexpr'),
  'cspa': (cspa_program, 'CspaPlan', 'integration/cspa.mir.sexpr'),
  'lsqb_q7': (lsqb_q7_program, 'LsqbQ7Plan', 'integration/lsqb_q7_optional.mir.sexpr'),
  'lsqb_q6': (lsqb_q6_program, 'LsqbQ6Plan', 'integration/lsqb_q6_count.mir.sexpr'),
  'reach_avoid': (reach_avoid_program, 'ReachAvoidPlan', None),
  'lsqb_q3': (lsqb_q3_program, 'LsqbQ3Plan', 'integration/lsqb_q3_triangle.mir.sexpr'),
  'lsqb_q6_2hop': (lsqb_q6_2hop_program, 'LsqbQ62HopPlan', 'integration/lsqb_q6_2hop.mir.sexpr'),
  'lsqb_q6_nosj': (lsqb_q6_nosj_program, 'LsqbQ6NosjPlan', 'integration/lsqb_q6_nosj.mir.sexpr'),
  'lsqb_q9': (lsqb_q9_program, 'LsqbQ9Plan', 'integration/lsqb_q9_neg2hop.mir.sexpr'),
  'lsqb_q6_bg': (lsqb_q6_bg_program, 'LsqbQ6BgPlan', 'integration/lsqb_q6_bg_test.mir.sexpr'),
  'debug_triangle': (debug_triangle_program, 'DebugTrianglePlan',
                     'integration/debug_triangle.mir.sexpr'),
  'gen_jit_triangle': (gen_jit_triangle_program, 'GenJitPlan', 'integration/gen_jit_code.mir.sexpr'),
  'triangle_db': (triangle_db_program, 'TriangleDBPlan', 'integration/triangle.mir.sexpr'),
  'neg_forms': (neg_forms_program, 'NegFormsPlan', None),
  'tc_2level_bg': (tc_2level_bg_program, 'Tc2LevelBgPlan', 'integration/tc_2level_bg.mir.sexpr'),
  'print_mir': (print_mir_program, 'PrintMirPlan', 'integration/print_mir.mir.sexpr'),
  'rewrite_consts': (rewrite_consts_program, 'RewriteConstsPlan', 'rewrite_consts.mir.sexpr'),
  'head_const': (head_const_program, 'HeadConstPlan', None),
  'galen': (galen_program, 'GalenPlan', 'integration/galen.mir.sexpr'),
  'polonius': (polonius_program, 'PoloniusPlan', 'integration/polonius_test.mir.sexpr'),
  'live': (live_program, 'LivePlan', None),
  'live_lsm': (live_lsm_program, 'LivePlan', None),
}
