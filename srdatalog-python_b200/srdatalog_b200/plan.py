'''MIR program -> flat JSON plan consumed by the native runtime (libsrdl).

The reference lowers a DSL program to MIR (`srdatalog.hir.compile_to_mir`,
src/srdatalog/hir/__init__.py:56) and then *emits C++ text* per rule
(src/srdatalog/codegen/jit/complete_runner.py:1569) and per step
(src/srdatalog/codegen/jit/orchestrator_jit.py:863).  This build keeps the
front end and replaces the emitter: the MIR tree is serialised as data and
a fixed CUDA library interprets it.  Node shapes follow
src/srdatalog/mir/types.py:48-386; only the op kinds that Python lowering
produces for stratified positive programs with filters are accepted.

Plan layout (version 1)::

  {"version": 1, "name": <project>,
   "relations": [{"name", "arity", "input_file", "print_size",
                  "index_type", "canonical": [cols], ["facts": [[v, ...], ...]]}],
   "steps": [{"recursive": bool, "ops": [op, ...]}]}

op kinds: execute_pipeline, rebuild_index, clear_relation, check_size,
compute_delta_index, merge_index, rebuild_index_from_index,
post_stratum_reconstruct, inject_cpp_hook (kept, not executed).  Pipeline
ops: scan, column_join, cartesian_join, filter, negation, insert_into.

A MIR `constant-bind` (a head constant, mir/types.py:99-109) becomes a
column join over a one-tuple relation `__const_<value>` whose tuple the plan
carries in "facts"; the runtime loads facts when it reads the plan.
'''

from __future__ import annotations

import json
import warnings
from typing import Any

from .plugin import runtime_index_type

PLAN_VERSION = 1
CONST_PREFIX = '__const_'


class PlanError(ValueError):
  '''Raised when a MIR construct has no runtime counterpart here.'''


def _ver(v: Any) -> str:
  # Version enum (src/srdatalog/hir/types.py:20): .value is "FULL"/"DELTA"/"NEW".
  s = getattr(v, 'value', v)
  if s not in ('FULL', 'DELTA', 'NEW'):
    raise PlanError(f'unknown relation version {v!r}')
  return s


def _source(node: Any) -> dict:
  kind = type(node).__name__
  if kind not in ('ColumnSource', 'Scan'):
    raise PlanError(f'unsupported join source {kind}')
  return {
    'rel': node.rel_name,
    'ver': _ver(node.version),
    'index': [int(c) for c in node.index],
    'prefix': list(node.prefix_vars),
  }


def _pipeline_op(node: Any) -> dict:
  kind = type(node).__name__
  if kind == 'Scan':
    d = _source(node)
    d.update(op='scan', vars=list(node.vars))
    return d
  if kind == 'ColumnJoin':
    return {'op': 'column_join', 'var': node.var_name,
            'sources': [_source(s) for s in node.sources]}
  if kind == 'CartesianJoin':
    return {'op': 'cartesian_join', 'vars': list(node.vars),
            'var_from_source': [list(v) for v in node.var_from_source],
            'sources': [_source(s) for s in node.sources]}
  if kind == 'Filter':
    return {'op': 'filter', 'vars': list(node.vars), 'code': node.code}
  if kind == 'Negation':
    # anti-join (mir/types.py:189): the probed prefix is the constant
    # arguments' values (their columns lead the index, hir/plan.py:284-286)
    # followed by the bound variables
    d = {'op': 'negation', 'rel': node.rel_name, 'ver': _ver(node.version),
         'index': [int(c) for c in node.index], 'prefix': list(node.prefix_vars)}
    consts = [int(v) for _, v in (getattr(node, 'const_args', None) or [])]
    for v in consts:
      if not 0 <= v <= 0xFFFFFFFF:
        raise PlanError(f'negation on {node.rel_name}: constant {v} is not a uint32 value')
    if consts:
      d['const_prefix'] = consts
    return d
  if kind == 'ConstantBind':
    # binding v to a literal = joining with the one-tuple relation {(value)}
    value = _const_literal(node)
    return {'op': 'column_join', 'var': node.var_name,
            'sources': [{'rel': f'{CONST_PREFIX}{value}', 'ver': 'FULL', 'index': [0],
                         'prefix': []}]}
  if kind == 'InsertInto':
    return {'op': 'insert_into', 'rel': node.rel_name, 'ver': _ver(node.version),
            'vars': list(node.vars), 'index': [int(c) for c in node.index]}
  raise PlanError(f'pipeline op {kind} is not supported by this runtime')


def _const_literal(node: Any) -> int:
  '''Value of a constant-bind whose code is an unsigned 32-bit literal
  (optionally `return <n>;` or parenthesised); other code is rejected.'''
  code = node.code.strip()
  if code.startswith('return') and code.endswith(';'):
    code = code[len('return'):-1].strip()
  code = code.strip('()').strip()
  if code[-1:] in ('u', 'U'):
    code = code[:-1]
  if not code.isdigit() or int(code) >= 2**32:
    raise PlanError(f'constant-bind of {node.var_name}: code {node.code!r} is not an unsigned '
                    '32-bit literal')
  return int(code)


def _const_relations(steps: list, declared: set) -> list:
  '''The one-tuple relations that lowered constant-binds read.'''
  values = set()
  for st in steps:
    for op in st['ops']:
      for p in op.get('pipeline', ()):
        for s in p.get('sources', ()):
          if s['rel'].startswith(CONST_PREFIX):
            values.add(int(s['rel'][len(CONST_PREFIX):]))
  out = []
  for v in sorted(values):
    name = f'{CONST_PREFIX}{v}'
    if name in declared:
      raise PlanError(f'relation name {name} is reserved for head constants')
    out.append({'name': name, 'arity': 1, 'input_file': '', 'print_size': False,
                'index_type': '', 'canonical': [0], 'facts': [[v]]})
  return out


def _instr(node: Any) -> dict:
  kind = type(node).__name__
  if kind == 'ExecutePipeline':
    return {'op': 'execute_pipeline', 'rule': node.rule_name,
            'count': bool(getattr(node, 'count', False)),
            'pipeline': [_pipeline_op(p) for p in node.pipeline]}
  if kind == 'RebuildIndex':
    return {'op': 'rebuild_index', 'rel': node.rel_name, 'ver': _ver(node.version),
            'index': [int(c) for c in node.index]}
  if kind == 'ClearRelation':
    return {'op': 'clear_relation', 'rel': node.rel_name, 'ver': _ver(node.version)}
  if kind == 'CheckSize':
    return {'op': 'check_size', 'rel': node.rel_name, 'ver': _ver(node.version)}
  if kind == 'ComputeDeltaIndex':
    return {'op': 'compute_delta_index', 'rel': node.rel_name,
            'index': [int(c) for c in node.canonical_index]}
  if kind == 'MergeIndex':
    return {'op': 'merge_index', 'rel': node.rel_name, 'index': [int(c) for c in node.index]}
  if kind == 'RebuildIndexFromIndex':
    return {'op': 'rebuild_index_from_index', 'rel': node.rel_name, 'ver': _ver(node.version),
            'source_index': [int(c) for c in node.source_index],
            'index': [int(c) for c in node.target_index]}
  if kind == 'PostStratumReconstructInternCols':
    return {'op': 'post_stratum_reconstruct', 'rel': node.rel_name,
            'index': [int(c) for c in node.canonical_index]}
  if kind == 'InjectCppHook':
    # Raw C++ pasted into the generated step (mir/types.py:358).  There is no
    # C++ code generation here, so the hook is kept in the plan for the record
    # and skipped by the runtime; the reference's own hooks only print sizes.
    warnings.warn(f'rule {node.rule_name}: injected C++ hook is not executed by this runtime',
                  stacklevel=3)
    return {'op': 'inject_cpp_hook', 'rule': node.rule_name, 'code': node.code}
  raise PlanError(f'MIR instruction {kind} is not supported by this runtime')


def _instrs(nodes: Any) -> list:
  '''Instructions in order; a ParallelGroup's independent ops (mir/types.py:351)
  run one after the other, which is one of the orders they may run in.'''
  out = []
  for n in nodes:
    if type(n).__name__ == 'ParallelGroup':
      out += _instrs(n.ops)
    else:
      out.append(_instr(n))
  return out


def _step(plan: Any, recursive: bool) -> dict:
  kind = type(plan).__name__
  if kind in ('FixpointPlan', 'Block'):
    ops = _instrs(plan.instructions)
  else:
    ops = _instrs([plan])
  return {'recursive': bool(recursive), 'ops': ops}


def plan_from_mir(mir_program: Any, relation_decls: list, name: str,
                  canonical: dict[str, list[int]] | None = None) -> dict:
  '''Serialise a `srdatalog.mir.types.Program` plus its relation decls.

  `canonical` maps relation -> canonical index (the reference merges the
  per-stratum maps, later strata winning: src/srdatalog/pipeline.py:112-116).
  Each relation's `index_type` is resolved through the index-plugin
  registry (`srdatalog_b200.plugin`) to the runtime policy's string.
  '''
  canonical = dict(canonical or {})
  rels = []
  for d in relation_decls:
    arity = len(d.types)
    rels.append({
      'name': d.rel_name,
      'arity': arity,
      'input_file': d.input_file or '',
      'print_size': bool(d.print_size),
      'index_type': runtime_index_type(d.index_type or ''),
      'canonical': list(canonical.get(d.rel_name, list(range(arity)))),
    })
  steps = [_step(p, rec) for (p, rec) in mir_program.steps]
  rels += _const_relations(steps, {r['name'] for r in rels})
  plan = {'version': PLAN_VERSION, 'name': name, 'relations': rels, 'steps': steps}
  validate_plan(plan)
  return plan


def plan_from_program(program: Any, name: str) -> dict:
  '''DSL `Program` -> plan, via the srdatalog front end (HIR/MIR passes).'''
  try:
    from srdatalog.hir import compile_to_hir, compile_to_mir
  except ImportError as e:  # pragma: no cover - depends on the environment
    raise ImportError(
      'srdatalog_b200.build_project needs the srdatalog front end '
      '(pip install srdatalog) for DSL -> HIR -> MIR planning') from e
  hir = compile_to_hir(program)
  mir = compile_to_mir(program)
  canonical: dict[str, list[int]] = {}
  for s in hir.strata:
    for rel, cols in s.canonical_index.items():
      canonical[rel] = list(cols)
  return plan_from_mir(mir, hir.relation_decls, name, canonical)


_FILTER_OPS = ('!=', '==', '<=', '>=', '<', '>')


def parse_filter(code: str, vars_: list[str]) -> list[tuple[str, str, str]]:
  '''Restricted filter grammar: `return a OP b [&& c OP d]...;`.

  Operands are bound variable names or unsigned integer constants.  The
  reference pastes the C++ body verbatim into the kernel
  (src/srdatalog/codegen/jit/instructions.py filter emission); here the
  expression is parsed and evaluated on the device, and anything outside
  this grammar is rejected at plan time.
  '''
  s = code.strip()
  if not s.startswith('return') or not s.endswith(';'):
    raise PlanError(f'filter {code!r}: expected "return <expr>;"')
  body = s[len('return'):-1].strip()
  terms = []
  for part in body.split('&&'):
    part = part.strip().strip('()').strip()
    for op in _FILTER_OPS:
      if op in part:
        a, b = (t.strip() for t in part.split(op, 1))
        for t in (a, b):
          if not (t in vars_ or t.isdigit()):
            raise PlanError(f'filter {code!r}: operand {t!r} is not a bound var or constant')
        terms.append((a, op, b))
        break
    else:
      raise PlanError(f'filter {code!r}: unsupported term {part!r}')
  return terms


def validate_plan(plan: dict) -> None:
  '''Host-side checks mirrored by the native plan loader.'''
  if plan.get('version') != PLAN_VERSION:
    raise PlanError('plan version mismatch')
  arity = {r['name']: r['arity'] for r in plan['relations']}
  for r in plan['relations']:
    for row in r.get('facts', ()):
      if len(row) != r['arity'] or not all(isinstance(x, int) and 0 <= x < 2**32 for x in row):
        raise PlanError(f'facts of {r["name"]}: {row!r} is not a row of {r["arity"]} uint32 values')
  for st in plan['steps']:
    for op in st['ops']:
      if op['op'] == 'inject_cpp_hook':
        continue
      if op['op'] != 'execute_pipeline':
        if op['rel'] not in arity:
          raise PlanError(f'unknown relation {op["rel"]}')
        continue
      bound: list[str] = []
      for p in op['pipeline']:
        k = p['op']
        if k in ('scan', 'column_join', 'cartesian_join'):
          srcs = [p] if k == 'scan' else p['sources']
          for s in srcs:
            if s['rel'] not in arity:
              raise PlanError(f'unknown relation {s["rel"]}')
            if sorted(s['index']) != list(range(arity[s['rel']])):
              raise PlanError(f'bad index {s["index"]} for {s["rel"]}')
            for v in s['prefix']:
              if v not in bound:
                raise PlanError(f'prefix var {v} unbound in {op["rule"]}')
          bound += p['vars'] if k in ('scan', 'cartesian_join') else [p['var']]
        elif k == 'filter':
          parse_filter(p['code'], bound)
        elif k == 'negation':
          if p['rel'] not in arity:
            raise PlanError(f'unknown relation {p["rel"]}')
          ar = arity[p['rel']]
          nb = len(p.get('const_prefix', [])) + len(p['prefix'])
          if ar > 3 or not 1 <= nb <= min(ar, 2):
            raise PlanError(f'negation on {p["rel"]}: needs 1..2 bound values (constants or '
                            f'variables) of a relation of arity <= 3')
          for v in p['prefix']:
            if v not in bound:
              raise PlanError(f'negation on {p["rel"]}: unbound var {v} in {op["rule"]}')
        elif k == 'insert_into':
          if p['rel'] not in arity or len(p['vars']) != arity[p['rel']]:
            raise PlanError(f'insert_into {p["rel"]}: arity mismatch')
          for v in p['vars']:
            if v not in bound:
              raise PlanError(f'insert_into {p["rel"]}: unbound var {v}')


def dumps(plan: dict) -> str:
  return json.dumps(plan, sort_keys=True, separators=(',', ':'))
