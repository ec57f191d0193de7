'''Index-plugin registry: the reference's registration and resolution rules
(src/srdatalog/codegen/jit/plugin.py:151-170, tests/test_jit_multiview.py
plugin-registration cases), and the mapping of each family to the runtime
index policy the plan carries.'''

from types import SimpleNamespace

import pytest
from srdatalog_b200 import plugin as P
from srdatalog_b200.plan import plan_from_mir

TWO_LEVEL = 'SRDatalog::GPU::Device2LevelIndex'


@pytest.fixture
def scratch_type():
  names = []
  yield names
  for n in names:
    P.unregister_index_plugin(n)


def test_two_level_plugin_registered():
  p = P.resolve_plugin(TWO_LEVEL)
  assert p.name == 'Device2LevelIndex' and p.cpp_type == TWO_LEVEL
  assert 'gpu/device_2level_index.h' in p.cpp_headers
  assert P.plugin_policy(p) == 'two_level'


def test_two_level_view_counts():
  assert P.plugin_view_count('FULL_VER', TWO_LEVEL) == 2
  assert P.plugin_view_count('DELTA_VER', TWO_LEVEL) == 1
  assert P.plugin_view_count('NEW_VER', TWO_LEVEL) == 1


def test_default_plugin_unchanged():
  assert P.plugin_view_count('FULL_VER') == 1
  assert P.plugin_view_count('FULL_VER', '') == 1
  assert P.resolve_plugin('').name == 'DSAI'
  assert P.resolve_plugin('SRDatalog::GPU::SomethingUnregistered').name == 'DSAI'


def test_substring_resolution_both_directions():
  # the declared type is a part of a registered one, and contains one
  assert P.resolve_plugin('Device2LevelIndex').cpp_type == TWO_LEVEL
  assert P.resolve_plugin(TWO_LEVEL + '<uint32_t>').cpp_type == TWO_LEVEL


def test_runtime_index_type_strings():
  assert P.runtime_index_type('') == ''
  assert P.runtime_index_type('Device2LevelIndex') == TWO_LEVEL
  assert P.runtime_index_type('Other::Index') == ''


def test_extra_headers():
  assert P.get_extra_headers_for_types(['', TWO_LEVEL, 'Device2LevelIndex']) == \
    ['gpu/device_2level_index.h']
  assert P.get_extra_headers_for_types(['', 'Unknown']) == []


def test_reference_style_plugin_module(scratch_type):
  # a plugin module written the reference's way (start from the default,
  # override the view hooks, register) maps to the two-level policy
  p = P.new_default_plugin()
  p.name, p.cpp_type = 'MyLsm', 'Acme::GPU::MyLsmIndex'
  p.view_count = lambda v: 2 if v == 'FULL_VER' else 1
  p.gen_host_view_setup = lambda e, v: [f'{e}.a()', f'{e}.b()'] if v == 'FULL_VER' else [f'{e}.view()']
  P.register_index_plugin(p)
  scratch_type.append(p.cpp_type)
  assert P.resolve_plugin('Acme::GPU::MyLsmIndex') is p
  assert P.runtime_index_type('Acme::GPU::MyLsmIndex') == TWO_LEVEL


def test_sorted_family_with_misleading_name(scratch_type):
  # a one-array family maps to the default policy whatever its name says
  p = P.IndexPlugin(name='Flat', cpp_type='Acme::FlatNotDevice2LevelIndex')
  P.register_index_plugin(p)
  scratch_type.append(p.cpp_type)
  assert P.runtime_index_type('Acme::FlatNotDevice2LevelIndex') == ''


def test_rejected_plugins():
  with pytest.raises(P.PluginError, match='empty cpp_type'):
    P.register_index_plugin(P.IndexPlugin(name='x', cpp_type=''))
  three = P.IndexPlugin(name='three', cpp_type='Acme::Three', view_count=lambda v: 3)
  with pytest.raises(P.PluginError, match='match no runtime policy'):
    P.register_index_plugin(three)
  liar = P.IndexPlugin(name='liar', cpp_type='Acme::Liar', policy='two_level',
                       view_count=lambda v: 1)
  with pytest.raises(P.PluginError, match='are those of'):
    P.register_index_plugin(liar)
  bad = P.IndexPlugin(name='bad', cpp_type='Acme::Bad', policy='hashed',
                      view_count=lambda v: 1)
  with pytest.raises(P.PluginError, match='not one of'):
    P.register_index_plugin(bad)
  assert P.resolve_plugin('Acme::Three').name == 'DSAI'


def _decl(name, arity, index_type=None):
  return SimpleNamespace(rel_name=name, types=[int] * arity, input_file=None,
                         print_size=False, index_type=index_type)


def test_plan_carries_the_runtime_policy(scratch_type):
  p = P.new_default_plugin()
  p.name, p.cpp_type = 'MyLsm', 'Acme::GPU::MyLsmIndex'
  p.view_count = lambda v: 2 if v == 'FULL_VER' else 1
  P.register_index_plugin(p)
  scratch_type.append(p.cpp_type)
  decls = [_decl('A', 2), _decl('B', 2, TWO_LEVEL), _decl('C', 2, 'Device2LevelIndex'),
           _decl('D', 2, 'Acme::GPU::MyLsmIndex'), _decl('E', 2, 'Unregistered::Index')]
  plan = plan_from_mir(SimpleNamespace(steps=[]), decls, 'p')
  got = {r['name']: r['index_type'] for r in plan['relations']}
  assert got == {'A': '', 'B': TWO_LEVEL, 'C': TWO_LEVEL, 'D': TWO_LEVEL, 'E': ''}
