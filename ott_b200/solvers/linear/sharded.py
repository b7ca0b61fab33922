"""One Sinkhorn problem row-sharded over ranks (one process per GPU).

Each rank holds a contiguous shard of the rows: its points x_r, weights a_r
and potential f_r, and all of y, b and g. One iteration is the reference's
sequential log-domain update (sinkhorn.py:803-857; geometry.py:376-398):

- g-update: each rank computes its shard's column log-sum-exp
  ``L_r[j] = eps log sum_{i in r} exp((f_i - C_ij) / eps)`` on its GPU
  (``ottb_apply_lse_kernel``, axis 0: geometry.py:259-299 with vec = None);
  the ranks all-gather the ``L_r`` (m floats each) and every rank combines
  them, ``L[j] = eps logsumexp_r(L_r[j] / eps)``, then
  ``g = eps log b - where(isfinite(L), L, 0)``;
- f-update: local to the rank, the row log-sum-exp of its rows against all
  of y with the new g (axis 1).

The marginal error (sinkhorn.py:127-221, the column marginal
``exp((g + L) / eps)`` of the state after the f-update) needs the next
g-update's combined ``L``, so an error iteration computes it once and the
next g-update reuses it. Blocks of ``inner_iterations``, the stop test and
the errors buffer follow fixed_point_loop.py:23-93 and sinkhorn.py:914-953;
``reg_ot_cost`` (sinkhorn.py:224-277) all-reduces the shards' sums. The only
exchanges are the column log-sum-exps and scalars; the cost is never formed.
"""
from __future__ import annotations

import ctypes
import math
from typing import Any, Callable, NamedTuple, Optional

import torch
import torch.distributed as dist

from ott_b200 import _arrays, _lib
from ott_b200 import distributed as odist

__all__ = ["ShardedSinkhornOutput", "solve_sharded"]

_PREC = {"auto": _lib.PRECISION_AUTO, "fp32": _lib.PRECISION_FP32,
         "bf16_split3": _lib.PRECISION_BF16_SPLIT3}

LseFn = Callable[[torch.Tensor, int], torch.Tensor]


class ShardedSinkhornOutput(NamedTuple):
  f: torch.Tensor          # this rank's rows
  g: torch.Tensor          # all columns (identical on every rank)
  errors: torch.Tensor     # [ceil(max_iterations / inner_iterations)]
  reg_ot_cost: float
  n_iters: int
  converged: bool
  epsilon: float
  row_offset: int          # first global row of this rank's shard


def _gpu_lse(x: torch.Tensor, y: torch.Tensor, eps: float, inv: float,
             precision: str) -> LseFn:
  """``ottb_apply_lse_kernel`` on this rank's rows and all columns."""
  lib = _lib.load()
  n, m, d = x.shape[0], y.shape[0], x.shape[1]
  if n == 0:  # a rank without rows (more ranks than rows): nothing to sum
    return lambda pot, axis: (torch.full((m,), -math.inf, dtype=torch.float64,
                                         device=x.device) if axis == 0
                              else torch.empty(0, dtype=torch.float64, device=x.device))
  code = _PREC[precision]
  sizes = [lib.ottb_apply_lse_kernel_workspace_size(n, m, d, ax, code) for ax in (0, 1)]
  if min(sizes) == 0:
    raise NotImplementedError("problem sizes not supported")
  ws = torch.empty(max(sizes), dtype=torch.uint8, device=x.device)

  def lse(pot: torch.Tensor, axis: int) -> torch.Tensor:
    p32 = pot.to(torch.float32).contiguous()
    out = torch.empty(m if axis == 0 else n, dtype=torch.float32, device=x.device)
    st = lib.ottb_apply_lse_kernel(x.data_ptr(), y.data_ptr(), n, m, d, p32.data_ptr(),
                                   ctypes.c_float(eps), ctypes.c_float(inv), axis, code,
                                   out.data_ptr(), ws.data_ptr(), ws.numel(),
                                   _arrays.stream_handle())
    _lib.check(st, "ottb_apply_lse_kernel")
    return out.double()

  return lse


def _all_gather_rows(t: torch.Tensor, group: Optional[Any]) -> torch.Tensor:
  """[world, len(t)] of every rank's ``t`` (equal lengths)."""
  _, world = odist.rank_and_world(group)
  if world == 1:
    return t[None]
  dev = t.device
  if dist.get_backend(group) != "nccl":
    t = t.cpu()
  parts = [torch.empty_like(t) for _ in range(world)]
  dist.all_gather(parts, t.contiguous(), group=group)
  return torch.stack(parts).to(dev)


def _sum_ranks(v: torch.Tensor, group: Optional[Any]) -> torch.Tensor:
  _, world = odist.rank_and_world(group)
  if world == 1:
    return v
  dev = v.device
  if dist.get_backend(group) != "nccl":
    v = v.cpu()
  v = v.clone()
  dist.all_reduce(v, op=dist.ReduceOp.SUM, group=group)
  return v.to(dev)


def solve_sharded(x: Any, y: Any, a: Optional[Any] = None, b: Optional[Any] = None, *,
                  epsilon: Optional[float] = None, relative_epsilon: Optional[str] = None,
                  scale_cost: float = 1.0, threshold: float = 1e-3, norm_error: int = 1,
                  inner_iterations: int = 10, min_iterations: int = 0,
                  max_iterations: int = 2000, precision: str = "auto",
                  group: Optional[Any] = None,
                  lse: Optional[LseFn] = None) -> ShardedSinkhornOutput:
  """``linear.solve(PointCloud(X, y, ...), A, b)`` with the rows of X and A
  split over the ranks of ``group`` in rank order: ``x``/``a`` are this
  rank's rows, ``y``/``b`` the whole second measure on every rank.

  ``epsilon`` is absolute, or a multiplier of mean(C) with
  ``relative_epsilon="mean"`` (geometry.py:113-117, 148-176: the closed
  form with uniform weights, from all-reduced sums of the shards);
  ``scale_cost`` a float. ``lse(pot, axis)`` replaces the GPU kernel
  (float64 in and out); the default is ``ottb_apply_lse_kernel`` with the
  given ``precision``.
  """
  if not isinstance(scale_cost, (int, float)):
    raise NotImplementedError("scale_cost must be a float for a sharded solve")
  if relative_epsilon not in (None, "mean"):
    raise NotImplementedError("relative_epsilon must be None or 'mean' for a sharded solve")
  if epsilon is None:
    raise NotImplementedError("pass epsilon (absolute, or with relative_epsilon='mean')")
  rank, world = odist.rank_and_world(group)
  if lse is None:
    dev = _arrays.device()
    x_t, y_t = _arrays.as_f32(x, dev), _arrays.as_f32(y, dev)
  else:
    x_t, y_t = torch.as_tensor(x), torch.as_tensor(y)
    dev = x_t.device
  n_r, m = x_t.shape[0], y_t.shape[0]
  inv = 1.0 / float(scale_cost)
  counts = _all_gather_rows(torch.tensor([float(n_r)], dtype=torch.float64, device=dev),
                            group).reshape(-1)
  n = int(counts.sum())
  offset = int(counts[:rank].sum())
  xd, yd = x_t.double(), y_t.double()
  if relative_epsilon == "mean":
    sums = _sum_ranks(torch.cat([(xd * xd).sum().reshape(1), xd.sum(0)]), group)
    mean_c = inv * (float(sums[0]) / n + float((yd * yd).sum()) / m
                    - 2.0 * float(torch.dot(sums[1:] / n, yd.mean(0))))
    eps = float(epsilon) * mean_c
  else:
    eps = float(epsilon)
  a_t = (torch.full((n_r,), 1.0 / n, dtype=torch.float64, device=dev) if a is None
         else torch.as_tensor(a, device=dev).double())
  b_t = (torch.full((m,), 1.0 / m, dtype=torch.float64, device=dev) if b is None
         else torch.as_tensor(b, device=dev).double())
  if lse is None:
    lse = _gpu_lse(x_t, y_t, eps, inv, precision)
  ninf = torch.tensor(-math.inf, dtype=torch.float64, device=dev)
  zero = torch.zeros((), dtype=torch.float64, device=dev)
  # DefaultInitializer (initializers.py:70-131)
  f = torch.where(a_t > 0, zero, ninf)
  g = torch.where(b_t > 0, zero, ninf)
  log_a = torch.log(a_t)
  log_b = torch.log(b_t)
  outer = int(math.ceil(max_iterations / inner_iterations))
  errors = -torch.ones(max(outer, 1), dtype=torch.float64)[:outer]
  cache = {"L": None}

  def col_lse() -> torch.Tensor:
    parts = _all_gather_rows(lse(f, 0), group) / eps        # [world, m]
    top = parts.max(0).values
    shift = torch.where(torch.isfinite(top), top, zero)
    return eps * (torch.log(torch.exp(parts - shift).sum(0)) + shift)

  def finite(v):
    return torch.where(torch.isfinite(v), v, zero)

  def one_iteration(it: int, compute_error: bool) -> None:
    nonlocal f, g
    L = cache["L"] if cache["L"] is not None else col_lse()
    g = eps * log_b - finite(L)
    f = eps * log_a - finite(lse(g, 1))
    cache["L"] = None
    if it == max_iterations - 1 or (compute_error and it >= min_iterations):
      cache["L"] = col_lse()
      marg = torch.exp((g + cache["L"]) / eps)
      err = float((torch.abs(marg - b_t) ** norm_error).sum() ** (1.0 / norm_error))
    else:
      err = math.inf
    errors[it // inner_iterations] = err

  def cond(it: int) -> bool:
    err = float(errors[it // inner_iterations - 1])
    return math.isfinite(err) and not (it > 0 and err < threshold)

  it = 0
  if min_iterations == max_iterations:
    for _ in range(max_iterations // inner_iterations):
      for k in range(inner_iterations):
        one_iteration(it, k == inner_iterations - 1)
        it += 1
  else:
    while it < max_iterations and (it < min_iterations or cond(it)):
      for k in range(inner_iterations):
        one_iteration(it, k == inner_iterations - 1)
        it += 1
  L = cache["L"] if cache["L"] is not None else col_lse()
  total = float(torch.exp((g + L) / eps).sum())
  div_a = _sum_ranks(torch.where(a_t > 0, a_t * (f - eps * torch.log(
      torch.where(a_t > 0, a_t, torch.ones_like(a_t)))), zero).sum().reshape(1), group)
  div_b = torch.where(b_t > 0, b_t * (g - eps * torch.log(
      torch.where(b_t > 0, b_t, torch.ones_like(b_t)))), zero).sum()
  sum_a = _sum_ranks(a_t.sum().reshape(1), group)
  cost = float(div_a[0] + div_b + eps * (sum_a[0] * b_t.sum() - total))
  converged = bool((not torch.isnan(errors).any()) and (outer == 0 or errors[-1] < threshold))
  n_iters = int((errors != -1).sum()) * inner_iterations
  return ShardedSinkhornOutput(f=f, g=g, errors=errors, reg_ot_cost=cost, n_iters=n_iters,
                               converged=converged, epsilon=eps, row_offset=offset)
