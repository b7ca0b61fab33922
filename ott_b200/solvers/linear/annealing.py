"""Epsilon annealing over stages: solve at geometrically decreasing epsilon,
each stage warm-started from the previous stage's potentials.

The reference decays epsilon inside one loop with
``Epsilon(target, init, decay)`` (geometry/epsilon_scheduler.py:22-60, run
here by the persistent kernel through ``eps_init`` / ``eps_decay``), and a
user chains stages by passing ``init=(f, g)`` to ``Sinkhorn.__call__``
(solvers/linear/sinkhorn.py:782-801). This driver is that chain, with every
pair of a batch solved in one launch per stage; each stage runs to its own
threshold. Potentials are in cost units, so a stage's (f, g) is a valid
starting point for the next, smaller epsilon.
"""
from __future__ import annotations

from typing import Any, List, NamedTuple, Optional, Sequence

import numpy as np

from ott_b200.geometry import pointcloud
from ott_b200.problems.linear import linear_problem
from ott_b200.solvers.linear import sinkhorn

__all__ = ["stage_multipliers", "AnnealedOutput", "solve_annealed"]


def stage_multipliers(stages: int, start: float = 1.0, final: float = 1e-3) -> np.ndarray:
  """Geometric multipliers of mean(C): start, ..., final (``stages`` values)."""
  if stages < 1:
    raise ValueError("stages must be >= 1")
  if stages == 1:
    return np.array([final], np.float64)
  k = np.arange(stages, dtype=np.float64) / (stages - 1)
  return start * (final / start) ** k


class AnnealedOutput(NamedTuple):
  """Final-stage outputs of every pair, per-stage iteration counts
  [stages, pairs], the per-stage epsilons [stages, pairs] and which
  (stage, pair) solves were redone by the fallback solver."""

  outputs: List[sinkhorn.SinkhornOutput]
  stage_iters: np.ndarray
  stage_epsilons: np.ndarray
  fallbacks: List[tuple]


def solve_annealed(xs: Sequence[Any], ys: Sequence[Any], a: Optional[Sequence[Any]] = None,
                   b: Optional[Sequence[Any]] = None, *, stages: int = 10, start: float = 1.0,
                   final: float = 1e-3, threshold: float = 1e-3, max_iterations: int = 2000,
                   precision: str = "auto", fallback_precision: Optional[str] = "fp32",
                   **solver_kwargs: Any) -> AnnealedOutput:
  """Anneals every pair (xs[k], ys[k]) from epsilon = start * mean(C_k) to
  final * mean(C_k) over ``stages`` geometric stages, threshold per stage.

  A stage solve that does not converge in the chosen precision is redone
  in ``fallback_precision`` from the same starting potentials.
  """
  K = len(xs)
  a = [None] * K if a is None else list(a)
  b = [None] * K if b is None else list(b)
  base = [pointcloud.PointCloud(x, y, epsilon=1.0, relative_epsilon="mean")
          for x, y in zip(xs, ys)]
  mean_c = np.array([g.epsilon for g in base], np.float64)   # 1.0 * mean(C_k)
  mults = stage_multipliers(stages, start, final)
  solver = sinkhorn.Sinkhorn(threshold=threshold, max_iterations=max_iterations,
                             precision=precision, **solver_kwargs)
  backup = (None if fallback_precision is None else
            sinkhorn.Sinkhorn(threshold=threshold, max_iterations=max_iterations,
                              precision=fallback_precision, **solver_kwargs))
  inits: List[Any] = [None] * K
  iters = np.zeros((stages, K), np.int64)
  epss = np.zeros((stages, K), np.float64)
  redone: List[tuple] = []
  outs: List[sinkhorn.SinkhornOutput] = []
  for s, mult in enumerate(mults):
    probs = []
    for k in range(K):
      geom = pointcloud.PointCloud(base[k].x, base[k].y, epsilon=float(mult * mean_c[k]))
      probs.append(linear_problem.LinearProblem(geom, a[k], b[k]))
      epss[s, k] = geom.epsilon
    outs = sinkhorn.run_batch(probs, solver, inits)
    bad = [k for k, o in enumerate(outs) if not o.converged]
    if bad and backup is not None:
      again = sinkhorn.run_batch([probs[k] for k in bad], backup, [inits[k] for k in bad])
      for k, o in zip(bad, again):
        outs[k] = o
        redone.append((s, k))
    iters[s] = [o.n_iters for o in outs]
    inits = [(o.f, o.g) for o in outs]
  return AnnealedOutput(outs, iters, epss, redone)
