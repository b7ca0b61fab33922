"""Linear OT entry point (ott/solvers/linear/_solve.py:29-64)."""
from __future__ import annotations

from typing import Any, List, Optional, Sequence

import torch

from ott_b200.problems.linear import linear_problem
from ott_b200.solvers.linear import sinkhorn

__all__ = ["reg_ot_cost", "solve", "solve_batch"]


def solve(geom, a: Optional[Any] = None, b: Optional[Any] = None,
          tau_a: float = 1.0, tau_b: float = 1.0, rank: int = -1,
          **kwargs: Any) -> sinkhorn.SinkhornOutput:
  """Builds a ``LinearProblem`` and runs ``Sinkhorn(**kwargs)`` on it."""
  if rank > 0:
    raise NotImplementedError("low-rank Sinkhorn (rank > 0) is not on this path")
  prob = linear_problem.LinearProblem(geom, a=a, b=b, tau_a=tau_a, tau_b=tau_b)
  solver = sinkhorn.Sinkhorn(**kwargs)
  return solver(prob)


def solve_batch(geoms: Sequence[Any], a: Optional[Sequence[Any]] = None,
                b: Optional[Sequence[Any]] = None,
                init: Optional[Sequence[Any]] = None,
                **kwargs: Any) -> List[sinkhorn.SinkhornOutput]:
  """Solves many independent problems (uneven n, m; same d) in one launch.

  The reference's route to this is ``jax.vmap`` over padded problems
  (geometry/segment.py:133-184); here each problem keeps its own size and
  its own stopping iteration, and a device work queue balances the units.
  """
  k = len(geoms)
  a = [None] * k if a is None else list(a)
  b = [None] * k if b is None else list(b)
  probs = [linear_problem.LinearProblem(g, a=ai, b=bi)
           for g, ai, bi in zip(geoms, a, b)]
  f_from_g = kwargs.pop("f_from_g", None)
  solver = sinkhorn.Sinkhorn(**kwargs)
  return sinkhorn.run_batch(probs, solver, init, f_from_g=f_from_g)


_RegOTCost = sinkhorn._RegOTCost


def reg_ot_cost(geom, a: Optional[Any] = None, b: Optional[Any] = None,
                **kwargs: Any) -> torch.Tensor:
  """``solve(geom, a, b, **kwargs).reg_ot_cost`` as a differentiable 0-dim
  tensor: ``jax.grad`` of the reference's ``reg_ot_cost`` corresponds to
  ``torch.autograd`` here (gradients w.r.t. ``geom.x``, ``geom.y``, ``a``,
  ``b``): with the default ``use_danskin=True`` the potentials are held
  fixed (``SinkhornOutput.reg_ot_cost_grads``); ``use_danskin=False``
  also differentiates them implicitly."""
  prob = linear_problem.LinearProblem(geom, a=a, b=b)
  out = sinkhorn.Sinkhorn(**kwargs)(prob)
  return sinkhorn._reg_ot_cost_tensor(out)
