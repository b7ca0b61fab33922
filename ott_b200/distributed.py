"""One process per GPU (``torch.distributed``: NCCL between GPUs, gloo in the
CPU tests): independent problems are partitioned across ranks, each rank
solves its share in ONE persistent launch, and only per-problem scalars and
timings cross ranks. No collective sits on the data path.

The reference maps a function over independent problems with ``jax.vmap``
(geometry/segment.py:133-184); across devices that is a partition of the
problem list, which is what ``shard_bounds`` computes.
"""
from __future__ import annotations

from typing import Any, List, NamedTuple, Optional, Sequence, Tuple

import torch
import torch.distributed as dist

__all__ = ["ShardedBatch", "all_gather_values", "max_over_ranks", "rank_and_world",
           "shard_bounds", "solve_batch_sharded", "sum_over_ranks"]


def rank_and_world(group: Optional[Any] = None) -> Tuple[int, int]:
  if dist.is_available() and dist.is_initialized():
    return dist.get_rank(group), dist.get_world_size(group)
  return 0, 1


def shard_bounds(work: Sequence[float], world_size: int) -> List[Tuple[int, int]]:
  """Contiguous ``[lo, hi)`` ranges of the problem list, one per rank, that
  balance the summed ``work`` (e.g. ``n_k * m_k``): rank r takes the
  problems whose cumulative work midpoint falls in its share
  ``[r W / R, (r + 1) W / R)``. Every problem lands on exactly one rank;
  ranges may be empty when there are fewer problems than ranks."""
  if world_size < 1:
    raise ValueError("world_size must be >= 1")
  total = float(sum(work))
  k = len(work)
  if k == 0:
    return [(0, 0)] * world_size
  if total <= 0.0:
    work, total = [1.0] * k, float(k)
  owner = []
  acc = 0.0
  for w in work:
    mid = acc + 0.5 * float(w)
    owner.append(min(int(mid * world_size / total), world_size - 1))
    acc += float(w)
  bounds = []
  lo = 0
  for r in range(world_size):
    hi = lo
    while hi < k and owner[hi] == r:
      hi += 1
    bounds.append((lo, hi))
    lo = hi
  return bounds


def _scalar_device(group: Optional[Any]) -> torch.device:
  if dist.get_backend(group) == "nccl":
    return torch.device("cuda", torch.cuda.current_device())
  return torch.device("cpu")


def _reduce(value: float, op, group: Optional[Any]) -> float:
  _, world = rank_and_world(group)
  if world == 1:
    return float(value)
  t = torch.tensor([float(value)], dtype=torch.float64, device=_scalar_device(group))
  dist.all_reduce(t, op=op, group=group)
  return float(t.item())


def max_over_ranks(value: float, group: Optional[Any] = None) -> float:
  """The largest of the ranks' values (a job's time is its slowest rank's)."""
  return _reduce(value, dist.ReduceOp.MAX, group)


def sum_over_ranks(value: float, group: Optional[Any] = None) -> float:
  return _reduce(value, dist.ReduceOp.SUM, group)


def all_gather_values(values: Sequence[float], group: Optional[Any] = None) -> List[float]:
  """Every rank's list of scalars, concatenated in rank order (lists may
  differ in length)."""
  _, world = rank_and_world(group)
  if world == 1:
    return [float(v) for v in values]
  gathered: List[Optional[List[float]]] = [None] * world
  dist.all_gather_object(gathered, [float(v) for v in values], group=group)
  return [v for part in gathered for v in part]


class ShardedBatch(NamedTuple):
  """This rank's outputs and the whole job's per-problem scalars."""
  outputs: List[Any]        # SinkhornOutput of problems [lo, hi)
  bounds: Tuple[int, int]   # this rank's range of the problem list
  reg_ot_cost: List[float]  # every problem's, in problem order
  n_iters: List[int]
  converged: List[bool]


def solve_batch_sharded(geoms: Sequence[Any], a: Optional[Sequence[Any]] = None,
                        b: Optional[Sequence[Any]] = None, group: Optional[Any] = None,
                        shapes: Optional[Sequence[Tuple[int, int]]] = None,
                        **kwargs: Any) -> ShardedBatch:
  """``solve_batch`` over all ranks: each rank builds only the geometries of
  its own range (``geoms[k]`` may be a callable returning the geometry, so
  that no rank materialises another's points; ``shapes`` then gives every
  problem's ``(n, m)``), solves them in one launch and the scalars are
  gathered."""
  from ott_b200.solvers.linear import _solve  # local: keeps this module importable on CPU
  rank, world = rank_and_world(group)
  if shapes is None:
    shapes = [g.shape for g in geoms]
  bounds = shard_bounds([float(n) * float(m) for n, m in shapes], world)
  lo, hi = bounds[rank]
  mine = [g() if callable(g) else g for g in geoms[lo:hi]]
  a_mine = None if a is None else list(a)[lo:hi]
  b_mine = None if b is None else list(b)[lo:hi]
  outs = _solve.solve_batch(mine, a_mine, b_mine, **kwargs) if mine else []
  costs = all_gather_values([float(o.reg_ot_cost) for o in outs], group)
  iters = [int(v) for v in all_gather_values([o.n_iters for o in outs], group)]
  conv = [bool(v) for v in all_gather_values([float(o.converged) for o in outs], group)]
  return ShardedBatch(outs, (lo, hi), costs, iters, conv)
