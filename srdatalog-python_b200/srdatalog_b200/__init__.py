'''srdatalog_b200 -- B200-native semi-naive Datalog backend for srdatalog programs.

The DSL, HIR and MIR come from the srdatalog front end; this package turns
the MIR into a plan that libsrdl.so (hand-written CUDA for sm_100a)
executes on one GPU, and keeps the reference's build/load surface:

    from srdatalog.dsl import Program, Relation, Var
    from srdatalog_b200 import build_project, compile_jit_project, CompilerConfig
    project = build_project(prog, project_name="TcPlan", cache_base="./build")
    br = compile_jit_project(project, CompilerConfig())
    lib = ctypes.CDLL(br.artifact)      # srdatalog_init/load_all/run/size/shutdown

`Database` is the direct handle API (no per-program shim).
'''

from .build import (BuildResult, CompileResult, CompilerConfig, build_project,
                    compile_jit_project, write_project)
from .loader import (SHIM_ENTRY_POINTS, EntryPoint, JitRuntime, build_and_load,
                     gen_runtime_shim_template)
from .native import Database, SrdlError
from .plan import PlanError, plan_from_mir, plan_from_program, validate_plan
from .plugin import IndexPlugin, PluginError, register_index_plugin, resolve_plugin

__version__ = '0.1.0'

__all__ = [
  'BuildResult', 'CompileResult', 'CompilerConfig', 'build_project', 'compile_jit_project',
  'write_project', 'EntryPoint', 'JitRuntime', 'build_and_load', 'gen_runtime_shim_template',
  'SHIM_ENTRY_POINTS', 'Database', 'SrdlError', 'PlanError', 'plan_from_mir',
  'plan_from_program', 'validate_plan', 'IndexPlugin', 'PluginError', 'register_index_plugin',
  'resolve_plugin',
]
