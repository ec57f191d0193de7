'''Index plugins: the reference's `IndexPlugin` registry, mapped to the
runtime index policies of `libsrdl.so`.

The reference's plugins are codegen hooks (src/srdatalog/codegen/jit/
plugin.py:30-58): each field emits a C++ expression for one index family,
and `resolve_plugin` (plugin.py:158-170) picks the family for a relation's
`index_type` string.  This backend emits no per-program C++; an index family
is a storage policy the native runtime applies to a relation's FULL version:

* ``'sorted'`` — one sorted array per version (the reference's default DSAI
  family, `new_default_plugin`, plugin.py:122-140).
* ``'two_level'`` — FULL kept as FULL + HEAD (the reference's
  Device2LevelIndex, codegen/jit/indexes/two_level.py:30-60): deltas merge
  into HEAD, HEAD into FULL once it passes a tenth of FULL; FULL reads see
  two sorted arrays (`view_count("FULL_VER") == 2`).

`IndexPlugin` keeps the reference's fields so that a plugin module written
for the reference constructs and registers here unchanged; the
expression-level hooks are stored but never called (there is no generated
C++ to put them in).  A family's policy is what its `view_count` hook says
it stores (one array per version: 'sorted'; two for FULL: 'two_level'), or
its explicit ``policy`` field, which must then agree with `view_count`.
Registration and resolution follow the reference: by `cpp_type`, exact
match first, then a substring match in either direction, else the default.
`plan_from_mir` resolves every relation's `index_type` through
`resolve_plugin` and writes the policy's runtime string into the plan, so
the native loader sees only strings it knows.
'''

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

POLICIES = ('sorted', 'two_level')

TWO_LEVEL_CPP_TYPE = 'SRDatalog::GPU::Device2LevelIndex'

# What the native plan loader reads in a relation's "index_type" for each
# policy (runtime.cu: a string naming Device2LevelIndex selects HEAD + FULL).
RUNTIME_INDEX_TYPE = {'sorted': '', 'two_level': TWO_LEVEL_CPP_TYPE}

_VERSIONS = ('FULL_VER', 'DELTA_VER', 'NEW_VER')
_SHAPES = {(1, 1, 1): 'sorted', (2, 1, 1): 'two_level'}


def _no_expr(*_args) -> str:
  return ''


def _one_view(_version: str) -> int:
  return 1


@dataclass
class IndexPlugin:
  '''One index family (reference: codegen/jit/plugin.py:30-58).

  The ``gen_*`` fields are accepted for source compatibility with the
  reference's plugin modules and ignored.  `view_count(version)` is the
  number of sorted arrays a read of FULL_VER / DELTA_VER / NEW_VER sees;
  `policy` (one of `POLICIES`, or None to derive it from `view_count`)
  names the runtime storage policy.
  '''

  name: str
  cpp_type: str
  cpp_headers: list[str] = field(default_factory=list)
  policy: str | None = None

  gen_root_handle: Callable = _no_expr
  gen_prefix: Callable = _no_expr
  gen_prefix_lower_bound: Callable = _no_expr
  gen_degree: Callable = _no_expr
  gen_valid: Callable = _no_expr
  gen_get_value_at: Callable = _no_expr
  gen_get_value: Callable = _no_expr
  gen_child: Callable = _no_expr
  gen_child_range: Callable = _no_expr
  gen_iterators: Callable = _no_expr

  view_count: Callable[[str], int] | None = None
  gen_host_view_setup: Callable = _no_expr

  def __post_init__(self):
    if self.view_count is None:
      self.view_count = _policy_view_count(self.policy or 'sorted')

  @property
  def runtime_index_type(self) -> str:
    '''The plan's "index_type" string for this family.'''
    return RUNTIME_INDEX_TYPE[plugin_policy(self)]


def _policy_view_count(policy: str) -> Callable[[str], int]:
  if policy == 'two_level':
    return lambda version: 2 if version == 'FULL_VER' else 1
  return _one_view


class PluginError(ValueError):
  pass


def new_default_plugin() -> IndexPlugin:
  '''The default family (DSAI; reference plugin.py:122-140): one sorted array.'''
  return IndexPlugin(name='DSAI', cpp_type='')


def new_two_level_plugin() -> IndexPlugin:
  '''Device2LevelIndex (reference codegen/jit/indexes/two_level.py:43-60).'''
  return IndexPlugin(name='Device2LevelIndex', cpp_type=TWO_LEVEL_CPP_TYPE,
                     cpp_headers=['gpu/device_2level_index.h'], policy='two_level')


_PLUGIN_REGISTRY: dict[str, IndexPlugin] = {}
_DEFAULT_PLUGIN: IndexPlugin = new_default_plugin()


def plugin_policy(plugin: IndexPlugin) -> str:
  '''The runtime policy a family maps to: derived from its `view_count`
  (FULL, DELTA, NEW arrays: 1,1,1 -> 'sorted'; 2,1,1 -> 'two_level'), and
  checked against an explicit `policy`.  Raises `PluginError` for a shape
  no runtime policy stores or a disagreeing `policy`.'''
  shape = tuple(plugin.view_count(v) for v in _VERSIONS)
  derived = _SHAPES.get(shape)
  if derived is None:
    raise PluginError(f'index plugin {plugin.name!r}: view counts {dict(zip(_VERSIONS, shape))} '
                      f'match no runtime policy ({POLICIES})')
  if plugin.policy is not None and plugin.policy != derived:
    if plugin.policy not in POLICIES:
      raise PluginError(f'index plugin {plugin.name!r}: policy {plugin.policy!r} '
                        f'is not one of {POLICIES}')
    raise PluginError(f'index plugin {plugin.name!r}: policy {plugin.policy!r} but view '
                      f'counts {dict(zip(_VERSIONS, shape))} are those of {derived!r}')
  return derived


def register_index_plugin(plugin: IndexPlugin) -> None:
  '''Register a family by its `cpp_type` (reference plugin.py:151-155).

  Raises `PluginError` for an empty `cpp_type` or a family no runtime
  policy stores (`plugin_policy`).'''
  if not plugin.cpp_type:
    raise PluginError(f'index plugin {plugin.name!r}: empty cpp_type')
  plugin_policy(plugin)
  _PLUGIN_REGISTRY[plugin.cpp_type] = plugin


def unregister_index_plugin(cpp_type: str) -> None:
  '''Remove a registered family (no-op if absent).'''
  _PLUGIN_REGISTRY.pop(cpp_type, None)


def resolve_plugin(index_type: str) -> IndexPlugin:
  '''Family for an `index_type` string (reference plugin.py:158-170): empty
  -> default; exact `cpp_type` match; else the first registered type that
  contains it or is contained in it; else the default.'''
  if not index_type:
    return _DEFAULT_PLUGIN
  if index_type in _PLUGIN_REGISTRY:
    return _PLUGIN_REGISTRY[index_type]
  for key, plugin in _PLUGIN_REGISTRY.items():
    if key in index_type or index_type in key:
      return plugin
  return _DEFAULT_PLUGIN


def runtime_index_type(index_type: str) -> str:
  '''The plan string the native loader gets for a declared `index_type`.'''
  return resolve_plugin(index_type or '').runtime_index_type


def plugin_view_count(version: str, index_type: str = '') -> int:
  '''Sorted arrays a read of `version` sees (reference plugin.py:256-257).'''
  return resolve_plugin(index_type).view_count(version)


def get_extra_headers_for_types(index_types: list[str]) -> list[str]:
  '''Unique `cpp_headers` of the families the types resolve to
  (reference plugin.py:173-184); empty strings are skipped.'''
  out: list[str] = []
  for t in index_types:
    if not t:
      continue
    for h in resolve_plugin(t).cpp_headers:
      if h not in out:
        out.append(h)
  return out


two_level_plugin = new_two_level_plugin()
register_index_plugin(two_level_plugin)

__all__ = ['IndexPlugin', 'PluginError', 'POLICIES', 'TWO_LEVEL_CPP_TYPE', 'new_default_plugin',
           'new_two_level_plugin', 'plugin_policy', 'register_index_plugin', 'unregister_index_plugin',
           'resolve_plugin', 'runtime_index_type', 'plugin_view_count',
           'get_extra_headers_for_types', 'two_level_plugin']
