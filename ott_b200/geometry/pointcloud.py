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
    self.y = self.x if (y is None or y is x) else _arrays.as_f32(y, self.x.device)
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

  # -- transport from potentials (geometry.py:361-365, 444-486) ------------
  def apply_transport_from_potentials(self, f: torch.Tensor, g: torch.Tensor, vec: Any,
                                      axis: int = 0) -> torch.Tensor:
    """Applies ``P_ij = exp((f_i + g_j - C_ij) / eps)`` to ``vec`` without
    forming P (geometry.py:444-486): ``axis=0`` sums over rows
    (``vec [..., n] -> [..., m]``), ``axis=1`` over columns
    (``vec [..., m] -> [..., n]``). ``vec`` may be 1-D or a batch."""
    if axis not in (0, 1):
      raise ValueError("axis must be 0 or 1")
    lib = _lib.load()
    n, m = self.shape
    dev = self.x.device
    v = _arrays.as_f32(vec, dev)
    one = v.ndim == 1
    v2 = v.reshape(1, -1) if one else v.reshape(-1, v.shape[-1]).contiguous()
    if v2.shape[1] != (n if axis == 0 else m):
      raise ValueError(f"vec has length {v2.shape[1]}, expected {n if axis == 0 else m}")
    fd = _arrays.as_f32(f, dev).detach()
    gd = _arrays.as_f32(g, dev).detach()
    out = torch.empty((v2.shape[0], m if axis == 0 else n), dtype=torch.float32, device=dev)
    ws_bytes = lib.ottb_apply_transport_workspace_size(n, m, self.dim, v2.shape[0], axis)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    st = lib.ottb_apply_transport(self.x.data_ptr(), self.y.data_ptr(), n, m, self.dim,
                                  fd.data_ptr(), gd.data_ptr(), ctypes.c_float(self.epsilon),
                                  ctypes.c_float(self.inv_scale_cost), v2.data_ptr(),
                                  v2.shape[0], axis, out.data_ptr(), ws.data_ptr(), ws_bytes,
                                  _arrays.stream_handle())
    _lib.check(st, "ottb_apply_transport")
    return out[0] if one else out.reshape(*v.shape[:-1], out.shape[-1])

  def transport_from_potentials(self, f: torch.Tensor, g: torch.Tensor) -> torch.Tensor:
    """The plan ``[n, m]`` (geometry.py:361-365)."""
    lib = _lib.load()
    n, m = self.shape
    dev = self.x.device
    fd = _arrays.as_f32(f, dev).detach()
    gd = _arrays.as_f32(g, dev).detach()
    out = torch.empty((n, m), dtype=torch.float32, device=dev)
    st = lib.ottb_transport_matrix(self.x.data_ptr(), self.y.data_ptr(), n, m, self.dim,
                                   fd.data_ptr(), gd.data_ptr(), ctypes.c_float(self.epsilon),
                                   ctypes.c_float(self.inv_scale_cost), out.data_ptr(),
                                   _arrays.stream_handle())
    _lib.check(st, "ottb_transport_matrix")
    return out

  def marginal_from_potentials(self, f: torch.Tensor, g: torch.Tensor,
                               axis: int = 0) -> torch.Tensor:
    """geometry.py:326-349: column (``axis=0``) or row (``axis=1``)
    marginal of the plan."""
    n, m = self.shape
    ones = torch.ones(n if axis == 0 else m, dtype=torch.float32, device=self.x.device)
    return self.apply_transport_from_potentials(f, g, ones, axis=axis)

  # -- divergences (pointcloud.py:226-237, geometry.py:248-254) -------------
  @classmethod
  def prepare_divergences(cls, x: Any, y: Any, static_b: bool = False,
                          **kwargs: Any) -> Tuple["PointCloud", ...]:
    """The geometries (x, y), (x, x) and, unless ``static_b``, (y, y)."""
    couples = [(x, y), (x, x)]
    if not static_b:
      couples += [(y, y)]
    return tuple(cls(u, v, **kwargs) for (u, v) in couples)

  def copy_epsilon(self, other: geometry.Geometry) -> "PointCloud":
    """This geometry with ``other``'s epsilon schedule."""
    new = PointCloud(self.x, self.y, batch_size=self._batch_size, scale_cost=self._scale_cost,
                     epsilon=other.epsilon_scheduler,
                     relative_epsilon=other._relative_epsilon)
    return new

  def __repr__(self) -> str:
    n, m = self.shape
    return f"PointCloud(n={n}, m={m}, d={self.dim}, epsilon={self._epsilon_init})"
