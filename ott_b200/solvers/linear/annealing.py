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

A learned warm start (``StagePredictor``) can replace the previous stage's
f by a prediction of the next stage's f: the reference's learned
initializer fills the f slot (``init_fu``,
initializers/neural/meta_initializer.py:137-158); g is then overwritten by
the first g-update of the loop, which reads only f. The predictor is a
small per-point MLP on this library's tcgen05 bf16 kernels, trained on the
potentials of annealed chains solved by the plain FP32 kernel; a stage it
starts that does not converge is solved again from the previous stage's
potentials by the fallback solver.
"""
from __future__ import annotations

import math
from typing import Any, List, NamedTuple, Optional, Sequence

import numpy as np

from ott_b200.geometry import pointcloud
from ott_b200.problems.linear import linear_problem
from ott_b200.solvers.linear import sinkhorn

__all__ = ["stage_multipliers", "AnnealedOutput", "solve_annealed", "StagePredictor",
           "stage_features"]


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
  [stages, pairs] (a stage redone by the fallback counts both solves), the
  per-stage epsilons [stages, pairs], which (stage, pair) solves were redone
  by the fallback solver, and, when asked for, every stage's f per pair
  (``f_history[k][s]``)."""

  outputs: List[sinkhorn.SinkhornOutput]
  stage_iters: np.ndarray
  stage_epsilons: np.ndarray
  fallbacks: List[tuple]
  f_history: Optional[List[List[Any]]] = None


# Per-point features of the stage predictor (columns of a 128-wide row;
# the rest are zero). For stage s with epsilon e_s, from the f of the stages
# before it (centred: potentials are defined up to a constant), in units of
# e_s: the last change d1 = f_{s-1} - f_{s-2}, the one before it d2, their
# linear extrapolation in epsilon d1 (e_s - e_{s-1}) / (e_{s-1} - e_{s-2}),
# and the epsilon ratios of the steps.
FEATURES = 128


def stage_features(f_hist: Sequence[Any], eps_hist: Sequence[float], eps: float):
  """[n, FEATURES] float32 features of the next stage (needs >= 2 stages)."""
  import torch
  if len(f_hist) < 2:
    raise ValueError("the stage predictor needs the f of two earlier stages")
  c = lambda v: v - v.mean()
  f1, f2 = f_hist[-1].float(), f_hist[-2].float()
  e1, e2 = float(eps_hist[-1]), float(eps_hist[-2])
  d1 = c(f1 - f2) / eps
  d2 = c(f2 - f_hist[-3].float()) / eps if len(f_hist) >= 3 else torch.zeros_like(d1)
  lin = d1 * (eps - e1) / (e1 - e2)
  x = torch.zeros((f1.shape[0], FEATURES), dtype=torch.float32, device=f1.device)
  x[:, 0] = lin
  x[:, 1] = d1
  x[:, 2] = d2
  x[:, 3] = eps / e1
  x[:, 4] = (e1 - e2) / eps
  x[:, 5] = 1.0
  return x


class StagePredictor:
  """Predicts the next annealing stage's f from the earlier stages' f, per
  point: a [FEATURES -> widths -> FEATURES] MLP (tanh-GELU, bf16 weights,
  FP32 accumulation) whose output column 0 minus column 1 is the predicted
  change of f in units of the new epsilon. The library's MLP loss is a
  squared error centred per sample over the weighted outputs; with weight 1
  on columns 0 and 1, target t on column 0 and 0 on column 1 it is
  ((y0 - y1) - t)^2 / 4, the per-point regression.
  """

  def __init__(self, widths: Sequence[int] = (128, 128), lr: float = 1e-3, seed: int = 0,
               device=None):
    from ott_b200.initializers.neural import meta_initializer
    self.mlp = meta_initializer.MLP([FEATURES, *widths, FEATURES], seed=seed, device=device)
    self.lr = lr

  def predict_delta(self, f_hist, eps_hist, eps) -> Any:
    """Predicted (f_next - f_last) / eps_next for every point."""
    import torch
    x = stage_features(f_hist, eps_hist, eps)
    n = x.shape[0]
    pad = (n + 127) // 128 * 128
    if pad != n:
      x = torch.cat([x, torch.zeros((pad - n, FEATURES), device=x.device)], dim=0)
    y = self.mlp.forward(x)[:n]
    return y[:, 0] - y[:, 1]

  def predict_f(self, f_hist, eps_hist, eps) -> Any:
    return f_hist[-1].float() + float(eps) * self.predict_delta(f_hist, eps_hist, eps)

  def fit(self, chains, steps: int = 2000, batch_size: int = 1024, points: int = 8192,
          seed: int = 0):
    """Adam on rows (features, change of f) of solved chains: ``chains`` is a
    list of (f_history, epsilons) per pair, f_history[s] the converged f of
    stage s. Uses stages >= 2, up to ``points`` random points per stage.
    Returns the per-step losses (device)."""
    import torch
    gen = torch.Generator(device="cpu").manual_seed(seed)
    xs, ts = [], []
    for f_hist, epss in chains:
      for s in range(2, len(f_hist)):
        x = stage_features(f_hist[:s], epss[:s], float(epss[s]))
        t = (f_hist[s].float() - f_hist[s - 1].float())
        t = (t - t.mean()) / float(epss[s])
        n = x.shape[0]
        if n > points:
          idx = torch.randperm(n, generator=gen)[:points].to(x.device)
          x, t = x[idx], t[idx]
        xs.append(x)
        ts.append(t)
    X = torch.cat(xs)
    T = torch.zeros((X.shape[0], FEATURES), dtype=torch.float32, device=X.device)
    T[:, 0] = torch.cat(ts)
    W = torch.zeros_like(T)
    W[:, :2] = 1.0
    num = X.shape[0]
    idx_all = torch.randint(0, num, (steps, batch_size), generator=gen).to(X.device)
    losses = []
    for step in range(steps):
      lr = self.lr * 0.5 * (1.0 + math.cos(math.pi * step / steps))
      i = idx_all[step]
      losses.append(self.mlp.gradients(X[i], T[i], W[i]).mean())
      self.mlp.adam(lr=lr)
    self.mlp.check_status()
    return torch.stack(losses)


def solve_annealed(xs: Sequence[Any], ys: Sequence[Any], a: Optional[Sequence[Any]] = None,
                   b: Optional[Sequence[Any]] = None, *, stages: int = 10, start: float = 1.0,
                   final: float = 1e-3, threshold: float = 1e-3, max_iterations: int = 2000,
                   precision: str = "auto", fallback_precision: Optional[str] = "fp32",
                   warm_start: Optional[StagePredictor] = None,
                   warm_budget: Optional[int] = None, record_f: bool = False,
                   **solver_kwargs: Any) -> AnnealedOutput:
  """Anneals every pair (xs[k], ys[k]) from epsilon = start * mean(C_k) to
  final * mean(C_k) over ``stages`` geometric stages, threshold per stage.

  A stage solve that does not converge in the chosen precision is redone
  in ``fallback_precision`` from the same starting potentials. With
  ``warm_start``, stages from the third on start from the predicted f
  (``StagePredictor.predict_f``) within ``warm_budget`` iterations
  (default ``max_iterations``); a pair whose warm-started stage does not
  converge is solved again from the previous stage's potentials by the
  fallback solver (the chosen one when ``fallback_precision`` is None).
  ``record_f`` keeps every stage's f (``f_history``).
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
  warm_solver = None
  if warm_start is not None:
    warm_solver = sinkhorn.Sinkhorn(threshold=threshold,
                                    max_iterations=warm_budget or max_iterations,
                                    precision=precision, **solver_kwargs)
  inits: List[Any] = [None] * K
  iters = np.zeros((stages, K), np.int64)
  epss = np.zeros((stages, K), np.float64)
  redone: List[tuple] = []
  outs: List[sinkhorn.SinkhornOutput] = []
  f_hist: List[List[Any]] = [[] for _ in range(K)]
  for s, mult in enumerate(mults):
    probs = []
    for k in range(K):
      geom = pointcloud.PointCloud(base[k].x, base[k].y, epsilon=float(mult * mean_c[k]))
      probs.append(linear_problem.LinearProblem(geom, a[k], b[k]))
      epss[s, k] = geom.epsilon
    if warm_solver is not None and s >= 2:
      starts = [(warm_start.predict_f(f_hist[k], epss[:s, k], epss[s, k]), inits[k][1])
                for k in range(K)]
      outs = sinkhorn.run_batch(probs, warm_solver, starts)
      bad = [k for k, o in enumerate(outs) if not o.converged]
      redo = backup or solver
      if bad:
        warm_iters = {k: outs[k].n_iters for k in bad}
        again = sinkhorn.run_batch([probs[k] for k in bad], redo, [inits[k] for k in bad])
        for k, o in zip(bad, again):
          outs[k] = o
          redone.append((s, k))
      iters[s] = [o.n_iters for o in outs]
      for k in bad:
        iters[s, k] += warm_iters[k]
    else:
      outs = sinkhorn.run_batch(probs, solver, inits)
      bad = [k for k, o in enumerate(outs) if not o.converged]
      if bad and backup is not None:
        again = sinkhorn.run_batch([probs[k] for k in bad], backup, [inits[k] for k in bad])
        for k, o in zip(bad, again):
          outs[k] = o
          redone.append((s, k))
      iters[s] = [o.n_iters for o in outs]
    inits = [(o.f, o.g) for o in outs]
    for k, o in enumerate(outs):
      f_hist[k].append(o.f.detach().clone())
  return AnnealedOutput(outs, iters, epss, redone, f_hist if record_f else None)
