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


# name -> (builder, project name, reference MIR fixture or None)
PROGRAMS = {
  'tc': (tc_program, 'TcPlan', 'tc.mir.sexpr'),
  'sg': (sg_program, 'SgPlan', 'integration/sg.mir.sexpr'),
  'triangle': (triangle_program, 'TrianglePlan', 'integration/lsqb_triangle_count.mir.sexpr'),
  'tc_left': (tc_left_program, 'TcLeftPlan', None),
  'tc_lsm': (tc_lsm_program, 'TcPlan', 'tc.mir.sexpr'),
}
