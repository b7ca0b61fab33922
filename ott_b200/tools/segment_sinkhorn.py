"""Regularised OT costs between segments of two point clouds
(ott/tools/segment_sinkhorn.py:24-138 over geometry/segment.py:23-184).

The reference pads every segment to ``max_measure_size`` points (padding
vector 0, weight 0) and ``jax.vmap``s one solve per segment. Padding points
carry no mass, so they change neither the potentials of the real points nor
the cost; they do enter the cost statistics behind a relative or default
epsilon and ``scale_cost="mean"``. Here each segment's epsilon and cost
scale are taken from its padded clouds exactly as the reference computes
them, and the real points alone are solved, all segments in ONE persistent
launch (uneven sizes, no padding work). The result is differentiable
w.r.t. ``x``, ``y`` and the weights (each cost with its potentials held
fixed, the reference's default).
"""
from __future__ import annotations

from types import MappingProxyType
from typing import Any, List, Mapping, Optional, Sequence, Tuple

import numpy as np
import torch

from ott_b200 import _arrays
from ott_b200.geometry import costs, pointcloud
from ott_b200.problems.linear import linear_problem
from ott_b200.solvers.linear import _solve, sinkhorn

__all__ = ["segment_sinkhorn"]


def _segments(num: int, num_segments: Optional[int], max_measure_size: Optional[int],
              segment_ids: Optional[Any], num_per_segment: Optional[Sequence[int]]
              ) -> Tuple[List[np.ndarray], int]:
  """Point indices of every segment (sorted, truncated to the padded size)
  and the padded size (segment.py:80-128)."""
  if segment_ids is not None:
    assert num_segments is not None, "Please specify `num_segments`."
    assert max_measure_size is not None, "Please specify `max_measure_size`."
    ids = np.asarray(torch.as_tensor(segment_ids).cpu()).reshape(-1)
  else:
    assert num_per_segment is not None, "Please specify `num_per_segment`."
    counts = [int(c) for c in num_per_segment]
    if max_measure_size is None:
      max_measure_size = max(counts)
    if num_segments is None:
      num_segments = len(counts)
    else:
      assert num_segments == len(counts)
    ids = np.repeat(np.arange(num_segments), counts)[:num]
    ids = np.concatenate([ids, np.full(num - len(ids), num_segments)])
  size = min(int(max_measure_size), num)
  idx = [np.flatnonzero(ids == s)[:size] for s in range(num_segments)]
  return idx, size


def segment_sinkhorn(
    x: Any,
    y: Any,
    num_segments: Optional[int] = None,
    max_measure_size: Optional[int] = None,
    cost_fn: Optional[costs.CostFn] = None,
    segment_ids_x: Optional[Any] = None,
    segment_ids_y: Optional[Any] = None,
    indices_are_sorted: bool = False,
    num_per_segment_x: Optional[Sequence[int]] = None,
    num_per_segment_y: Optional[Sequence[int]] = None,
    weights_x: Optional[Any] = None,
    weights_y: Optional[Any] = None,
    sinkhorn_kwargs: Mapping[str, Any] = MappingProxyType({}),
    **kwargs: Any,
) -> torch.Tensor:
  """segment_sinkhorn.py:24-138: ``reg_ot_cost`` of every segment pair
  (``[num_segments]`` tensor). Two interfaces as the reference: segment
  ids (with ``num_segments`` and ``max_measure_size``) or contiguous
  segment sizes."""
  del indices_are_sorted  # sorting is explicit here
  if cost_fn is not None and not isinstance(cost_fn, costs.SqEuclidean):
    raise NotImplementedError("ott_b200 implements the squared Euclidean cost only")
  xt = _arrays.as_f32(x)
  dev = xt.device
  yt = _arrays.as_f32(y, dev)
  use_ids = segment_ids_x is not None
  if use_ids:
    assert segment_ids_y is not None
  else:
    assert num_per_segment_x is not None and num_per_segment_y is not None
  nx, ny = xt.shape[0], yt.shape[0]
  idx_x, size_x = _segments(nx, num_segments, max_measure_size, segment_ids_x,
                            num_per_segment_x)
  idx_y, size_y = _segments(ny, num_segments, max_measure_size, segment_ids_y,
                            num_per_segment_y)
  nseg = len(idx_x)
  assert len(idx_y) == nseg, "x and y must hold the same number of segments"
  d = xt.shape[1]
  wx = None if weights_x is None else _arrays.as_f32(weights_x, dev)
  wy = None if weights_y is None else _arrays.as_f32(weights_y, dev)

  probs = []
  for s in range(nseg):
    ix = torch.as_tensor(idx_x[s], device=dev, dtype=torch.long)
    iy = torch.as_tensor(idx_y[s], device=dev, dtype=torch.long)
    xs, ys = xt[ix], yt[iy]
    if wx is None:
      cnt = int((np.asarray(torch.as_tensor(segment_ids_x).cpu()) == s).sum()) if use_ids \
          else int(num_per_segment_x[s])
      a = torch.full((len(idx_x[s]),), 1.0 / cnt, dtype=torch.float32, device=dev)
    else:
      a = wx[ix]
    if wy is None:
      cnt = int((np.asarray(torch.as_tensor(segment_ids_y).cpu()) == s).sum()) if use_ids \
          else int(num_per_segment_y[s])
      b = torch.full((len(idx_y[s]),), 1.0 / cnt, dtype=torch.float32, device=dev)
    else:
      b = wy[iy]
    # epsilon and cost scale of the padded clouds, as the reference sees them
    px = torch.cat([xs.detach(), torch.zeros(size_x - len(idx_x[s]), d, device=dev)])
    py = torch.cat([ys.detach(), torch.zeros(size_y - len(idx_y[s]), d, device=dev)])
    padded = pointcloud.PointCloud(px, py, **kwargs)
    geom = pointcloud.PointCloud(xs, ys, epsilon=padded.epsilon_scheduler,
                                 scale_cost=1.0 / padded.inv_scale_cost)
    probs.append(linear_problem.LinearProblem(geom, a, b))
  outs = sinkhorn.run_batch(probs, sinkhorn.Sinkhorn(**dict(sinkhorn_kwargs)))
  return torch.stack([_solve._RegOTCost.apply(p.geom.x, p.geom.y, p.a, p.b, o)
                      for p, o in zip(probs, outs)])
