"""Sinkhorn divergence (ott/tools/sinkhorn_divergence.py:178-352).

``div = reg_ot_cost(x, y) - (reg_ot_cost(x, x) + reg_ot_cost(y, y)) / 2
+ eps (sum(a) - sum(b))^2 / 2`` with the x/x and y/y terms solved by the
symmetric update (parallel updates, momentum 1/2: :318-336) unless
``symmetric_sinkhorn=False``. The two or three solves run in ONE
persistent launch (the batched work queue), and the divergence is a
differentiable tensor (each term's gradient with its potentials held fixed,
the reference's default).
"""
from __future__ import annotations

from types import MappingProxyType
from typing import Any, Mapping, NamedTuple, Optional, Tuple, Type

import torch

from ott_b200 import _arrays
from ott_b200.problems.linear import linear_problem
from ott_b200.solvers.linear import _solve, sinkhorn

__all__ = ["SinkhornDivergenceOutput", "sinkhorn_divergence"]


class SinkhornDivergenceOutput(NamedTuple):
  """sinkhorn_divergence.py:35-175 (the fields on this path)."""
  divergence: torch.Tensor
  potentials: Tuple[Tuple[torch.Tensor, torch.Tensor], ...]
  geoms: Tuple[Any, ...]
  errors: Tuple[Optional[torch.Tensor], ...]
  converged: Tuple[bool, ...]
  a: torch.Tensor
  b: torch.Tensor
  n_iters: Tuple[int, ...]
  outputs: Tuple[sinkhorn.SinkhornOutput, ...]


def sinkhorn_divergence(
    geom: Type[Any],
    *args: Any,
    a: Optional[Any] = None,
    b: Optional[Any] = None,
    solve_kwargs: Mapping[str, Any] = MappingProxyType({}),
    static_b: bool = False,
    offset_static_b: Optional[float] = None,
    share_epsilon: bool = True,
    symmetric_sinkhorn: bool = True,
    **kwargs: Any,
) -> Tuple[torch.Tensor, SinkhornDivergenceOutput]:
  """sinkhorn_divergence.py:178-267: ``geom`` is the geometry class
  (``PointCloud``), ``args`` and ``kwargs`` go to its
  ``prepare_divergences``; returns ``(divergence, output)``."""
  geoms = geom.prepare_divergences(*args, static_b=static_b, **kwargs)
  geom_xy, geom_x, geom_y, *_ = tuple(geoms) + (None,) * 3
  n, m = geom_xy.shape
  if share_epsilon:
    geom_x = geom_x.copy_epsilon(geom_xy)
    if geom_y is not None:
      geom_y = geom_y.copy_epsilon(geom_xy)
  dev = geom_xy.x.device
  a = torch.full((n,), 1.0 / n, device=dev) if a is None else _arrays.as_f32(a, dev)
  b = torch.full((m,), 1.0 / m, device=dev) if b is None else _arrays.as_f32(b, dev)
  kw = dict(solve_kwargs)
  for k in ("parallel_dual_updates", "momentum", "anderson", "rank"):
    if kw.get(k) not in (None, False, -1):
      raise NotImplementedError(f"solve_kwargs[{k!r}] is not on this path")
  solver = sinkhorn.Sinkhorn(**kw)
  probs = [linear_problem.LinearProblem(geom_xy, a, b),
           linear_problem.LinearProblem(geom_x, a, a)]
  if geom_y is not None:
    probs.append(linear_problem.LinearProblem(geom_y, b, b))
  sym = [False] + [bool(symmetric_sinkhorn)] * (len(probs) - 1)
  outs = sinkhorn.run_batch(probs, solver, symmetric=sym)

  def term(p, out):
    return _solve._RegOTCost.apply(p.geom.x, p.geom.y, p.a, p.b, out)

  c_xy, c_xx = term(probs[0], outs[0]), term(probs[1], outs[1])
  if geom_y is not None:
    c_yy = term(probs[2], outs[2])
  else:
    c_yy = torch.tensor(0.0 if offset_static_b is None else float(offset_static_b),
                        dtype=torch.float64, device=dev)
  eps = float(geom_xy.epsilon)
  div = c_xy - 0.5 * (c_xx + c_yy) + 0.5 * eps * (a.double().sum() - b.double().sum()) ** 2
  out = SinkhornDivergenceOutput(
      divergence=div,
      potentials=tuple((o.f, o.g) for o in outs),
      geoms=(geom_xy, geom_x, geom_y),
      errors=tuple(o.errors for o in outs) + ((None,) if geom_y is None else ()),
      converged=tuple(o.converged for o in outs),
      a=a, b=b,
      n_iters=tuple(o.n_iters for o in outs),
      outputs=tuple(outs))
  return div, out
