"""Point-cloud geometry with squared-Euclidean cost (ott/geometry/pointcloud.py).

The cost is never materialised: every sweep recomputes it tile by tile in
the fused kernels, which is the reference's online mode
(pointcloud.py:85-103) whatever ``batch_size`` is.
"""
from __future__ import annotations

import ctypes
from typing import Any, Optional, Tuple, Union

import torch

from ott_b200 import _arrays, _lib
from ott_b200.geometry import costs, geometry


class PointCloud(geometry.Geometry):
  """Two point clouds ``x [n, d]`` and ``y [m, d]`` (``y=None`` uses ``x``).

  Args mirror pointcloud.py:54-72. ``cost_fn`` must be
  :class:`~ott_b200.geometry.costs.SqEuclidean` (the default);
  ``scale_cost`` may be a float or ``"mean"``.
  """

  def __init__(
      self,
      x: Any,
      y: Optional[Any] = None,
      cost_fn: Optional[costs.CostFn] = None,
      batch_size: Optional[int] = None,
      scale_cost: Union[float, str] = 1.0,
      **kwargs: Any,
  ):
    super().__init__(**kwargs)
    if cost_fn is not None and not isinstance(cost_fn, costs.SqEuclidean):
      raise NotImplementedError(
          f"ott_b200 implements the squared Euclidean cost only, got {cost_fn!r}")
    if batch_size is not None:
      assert batch_size > 0, f"`batch_size={batch_size}` must be positive."
    self.x = _arrays.as_f32(x)
    self.y = self.x if y is None else _arrays.as_f32(y, self.x.device)
    if self.x.ndim != 2 or self.y.ndim != 2 or self.x.shape[1] != self.y.shape[1]:
      raise ValueError(f"x and y must be [n, d] and [m, d], got "
                       f"{tuple(self.x.shape)} and {tuple(self.y.shape)}")
    self.cost_fn = costs.SqEuclidean()
    self._batch_size = batch_size
    self._scale_cost = scale_cost
    self._stats: Optional[Tuple[float, float]] = None
    self._stats_unscaled: Optional[Tuple[float, float]] = None

  # -- shape ---------------------------------------------------------------
  @property
  def shape(self) -> Tuple[int, int]:
    return int(self.x.shape[0]), int(self.y.shape[0])

  @property
  def dim(self) -> int:
    return int(self.x.shape[1])

  @property
  def dtype(self) -> torch.dtype:
    return self.x.dtype

  @property
  def batch_size(self) -> Optional[int]:
    """pointcloud.py:438-444."""
    if self._batch_size is None:
      return None
    n, m = self.shape
    return min(n, m, self._batch_size)

  @property
  def is_online(self) -> bool:
    return self.batch_size is not None

  @property
  def is_squared_euclidean(self) -> bool:
    return True

  @property
  def is_square(self) -> bool:
    n, m = self.shape
    return n == m

  # -- cost statistics (geometry.py:113-135 via pointcloud.py:170-186) -----
  def _cost_stats(self, inv_scale: float, second: bool) -> Tuple[float, float]:
    lib = _lib.load()
    n, m = self.shape
    d = self.dim
    ws_bytes = lib.ottb_cost_stats_workspace_size(n, m, d)
    if ws_bytes == 0:
      raise NotImplementedError(f"cost statistics unsupported for d={d}")
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=self.x.device)
    out = torch.empty(2, dtype=torch.float64, device=self.x.device)
    st = lib.ottb_cost_stats(self.x.data_ptr(), self.y.data_ptr(), n, m, d,
                             ctypes.c_float(inv_scale), 1 if second else 0, out.data_ptr(),
                             ws.data_ptr(), ws_bytes, _arrays.stream_handle())
    _lib.check(st, "ottb_cost_stats")
    mean, msq = out.tolist()
    return mean, msq

  @property
  def inv_scale_cost(self) -> float:
    """pointcloud.py:343-383 for the scalings on this path."""
    sc = self._scale_cost
    if isinstance(sc, (int, float)):
      return 1.0 / float(sc)
    if sc == "mean":
      if self._stats_unscaled is None:
        self._stats_unscaled = self._cost_stats(1.0, second=False)
      return 1.0 / self._stats_unscaled[0]
    raise NotImplementedError(f"scale_cost={sc!r} is not on this path")

  def _scaled_stats(self, second: bool) -> Tuple[float, float]:
    if self._stats is None or (second and self._stats[1] != self._stats[1]):
      self._stats = self._cost_stats(self.inv_scale_cost, second)
    return self._stats

  @property
  def mean_cost_matrix(self) -> float:
    return self._scaled_stats(second=False)[0]

  @property
  def std_cost_matrix(self) -> float:
    """``sqrt(relu(mean(C^2) - mean(C)^2))`` (geometry.py:120-135)."""
    mean, msq = self._scaled_stats(second=True)
    return max(msq - mean * mean, 0.0) ** 0.5

  def __repr__(self) -> str:
    n, m = self.shape
    return f"PointCloud(n={n}, m={m}, d={self.dim}, epsilon={self._epsilon_init})"
