"""Executes ott-jax's own source files for the Sinkhorn path over the NumPy
stand-in for jax (TEST INFRASTRUCTURE ONLY; runs only where the reference
source tree is present, never on the GPU machine or in the product).

Only the modules on the path are executed, in dependency order, from the
reference tree:
  ott/utils.py, math/utils.py, math/fixed_point_loop.py,
  math/unbalanced_functions.py, geometry/epsilon_scheduler.py,
  geometry/costs.py, geometry/geometry.py, geometry/low_rank.py,
  geometry/pointcloud.py, problems/linear/linear_problem.py,
  initializers/linear/initializers.py, solvers/linear/acceleration.py,
  solvers/linear/sinkhorn.py, solvers/linear/_solve.py, and on request
  geometry/segment.py, tools/sinkhorn_divergence.py and
  tools/segment_sinkhorn.py (load_tools).
Modules the path imports but never calls for a balanced dense solve
(regularizers, matrix square roots, implicit differentiation, low-rank and
semidiscrete solvers, dual potentials, jaxopt) are empty placeholders.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types

from oracle import jaxshim

# The reference's source root: $OTT_REFERENCE_SRC, else the ott-jax tree
# checked out beside this repository (<parent>/reference/src).
DEFAULT_ROOT = os.environ.get(
    "OTT_REFERENCE_SRC",
    os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
                 "reference", "src"))


class _Anything:
  """Placeholder class for names only used in annotations or defaults."""

  def __init__(self, *a, **k):
    pass


def _placeholder(name: str, **attrs) -> types.ModuleType:
  """Module whose every attribute is a do-nothing class (names only used in
  annotations, defaults and class bodies off the path)."""
  m = types.ModuleType(name)
  m.__dict__.update(attrs)
  m.__getattr__ = lambda attr: _Anything
  sys.modules[name] = m
  return m


def _package(name: str) -> types.ModuleType:
  m = sys.modules.get(name)
  if m is None:
    m = types.ModuleType(name)
    m.__path__ = []
    sys.modules[name] = m
    parent, _, leaf = name.rpartition(".")
    if parent:
      setattr(_package(parent), leaf, m)
  return m


def _exec(root: str, dotted: str) -> types.ModuleType:
  path = os.path.join(root, *dotted.split(".")) + ".py"
  spec = importlib.util.spec_from_file_location(dotted, path)
  mod = importlib.util.module_from_spec(spec)
  sys.modules[dotted] = mod
  parent, _, leaf = dotted.rpartition(".")
  setattr(_package(parent), leaf, mod)
  spec.loader.exec_module(mod)
  return mod


def load(root: str = DEFAULT_ROOT, x64: bool = True) -> types.SimpleNamespace:
  if not os.path.isdir(os.path.join(root, "ott")):
    raise FileNotFoundError(f"reference source not found under {root}")
  for name in [n for n in sys.modules if n == "ott" or n.startswith("ott.")]:
    del sys.modules[name]
  jaxshim.install(x64=x64)
  _placeholder("jaxopt")
  for pkg in ("ott", "ott.math", "ott.geometry", "ott.problems", "ott.problems.linear",
              "ott.solvers", "ott.solvers.linear", "ott.initializers",
              "ott.initializers.linear"):
    _package(pkg)
  _placeholder("ott.geometry.regularizers")
  sys.modules["ott.geometry"].regularizers = sys.modules["ott.geometry.regularizers"]
  _placeholder("ott.math.matrix_square_root")
  sys.modules["ott.math"].matrix_square_root = sys.modules["ott.math.matrix_square_root"]
  utils = _exec(root, "ott.utils")
  _exec(root, "ott.math.utils")
  _exec(root, "ott.math.fixed_point_loop")
  _exec(root, "ott.math.unbalanced_functions")
  _exec(root, "ott.geometry.epsilon_scheduler")
  costs = _exec(root, "ott.geometry.costs")
  geometry = _exec(root, "ott.geometry.geometry")
  _exec(root, "ott.geometry.low_rank")
  pointcloud = _exec(root, "ott.geometry.pointcloud")
  _placeholder("ott.geometry.semidiscrete_pointcloud")
  sys.modules["ott.geometry"].semidiscrete_pointcloud = sys.modules[
      "ott.geometry.semidiscrete_pointcloud"]
  _placeholder("ott.problems.linear.potentials", DualPotentials=_Anything,
               EntropicPotentials=_Anything)
  sys.modules["ott.problems.linear"].potentials = sys.modules["ott.problems.linear.potentials"]
  linear_problem = _exec(root, "ott.problems.linear.linear_problem")
  _placeholder("ott.problems.linear.semidiscrete_linear_problem")
  sys.modules["ott.problems.linear"].semidiscrete_linear_problem = sys.modules[
      "ott.problems.linear.semidiscrete_linear_problem"]
  initializers = _exec(root, "ott.initializers.linear.initializers")
  _exec(root, "ott.solvers.linear.acceleration")
  _placeholder("ott.solvers.linear.implicit_differentiation", ImplicitDiff=_Anything)
  sys.modules["ott.solvers.linear"].implicit_differentiation = sys.modules[
      "ott.solvers.linear.implicit_differentiation"]
  sinkhorn = _exec(root, "ott.solvers.linear.sinkhorn")
  for name in ("semidiscrete", "sinkhorn_lr", "univariate"):
    _placeholder(f"ott.solvers.linear.{name}")
    setattr(sys.modules["ott.solvers.linear"], name,
            sys.modules[f"ott.solvers.linear.{name}"])
  solve_mod = _exec(root, "ott.solvers.linear._solve")
  sys.modules["ott.solvers.linear"].solve = solve_mod.solve
  acceleration = sys.modules["ott.solvers.linear.acceleration"]
  return types.SimpleNamespace(utils=utils, costs=costs, geometry=geometry,
                               pointcloud=pointcloud, linear_problem=linear_problem,
                               initializers=initializers, sinkhorn=sinkhorn,
                               acceleration=acceleration, solve=solve_mod.solve)


def load_implicit(linear_solver, root: str = DEFAULT_ROOT) -> types.ModuleType:
  """solvers/linear/implicit_differentiation.py from the reference tree,
  after load(). Its default linear solver (``lineax_implicit.solve_lineax``:
  lineax is not installed) is replaced by ``linear_solver``, called with the
  same ``(lin, b, lin_t, symmetric, **kwargs)`` arguments."""
  _placeholder("ott.solvers.linear.lineax_implicit", solve_lineax=linear_solver)
  sys.modules["ott.solvers.linear"].lineax_implicit = sys.modules[
      "ott.solvers.linear.lineax_implicit"]
  return _exec(root, "ott.solvers.linear.implicit_differentiation")


def load_tools(root: str = DEFAULT_ROOT) -> types.SimpleNamespace:
  """geometry/segment.py, tools/sinkhorn_divergence.py and
  tools/segment_sinkhorn.py from the reference tree, after load()."""
  _package("ott.tools")
  segment = _exec(root, "ott.geometry.segment")
  divergence = _exec(root, "ott.tools.sinkhorn_divergence")
  segment_sinkhorn = _exec(root, "ott.tools.segment_sinkhorn")
  return types.SimpleNamespace(segment=segment, sinkhorn_divergence=divergence,
                               segment_sinkhorn=segment_sinkhorn)
