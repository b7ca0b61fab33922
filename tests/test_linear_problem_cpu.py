"""LinearProblem's defaults on the CPU (a stub geometry: only x's device
and the shape are read)."""
import types

import torch

from ott_b200.problems.linear import linear_problem


def _geom(n, m):
  return types.SimpleNamespace(x=torch.zeros(n, 2), shape=(n, m))


def test_uniform_defaults_do_not_change_is_uniform():
  """linear_problem.py:66-99: reading the default weights leaves the
  problem uniform (an assignment when n == m and balanced)."""
  prob = linear_problem.LinearProblem(_geom(4, 4))
  assert prob.is_uniform and prob.is_assignment
  assert torch.allclose(prob.a, torch.full((4,), 0.25)) and prob.b.shape == (4,)
  assert prob.a is prob.a  # made once
  assert prob.is_uniform and prob.is_assignment
  assert not linear_problem.LinearProblem(_geom(4, 5)).is_assignment
  assert not linear_problem.LinearProblem(_geom(4, 4), tau_a=0.9).is_assignment
