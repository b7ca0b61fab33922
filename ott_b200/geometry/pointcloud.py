"""Point-cloud geometry with squared-Euclidean cost (ott/geometry/pointcloud.py).

The cost is never materialised: every sweep recomputes it tile by tile in
the fused kernels, which is the reference's online mode
(pointcloud.py:85-103) whatever ``batch_size`` is.
"""
from __future__ import annotations

import ctypes
import functools
from typing import Any, Optional, Tuple, Union

import torch

from ott_b200 import _arrays, _lib
from ott_b200.geometry import costs, geometry

# Below these the tensor-core application's fixed cost (its log-sum-exp
# pass and operand preparation) outweighs its faster products.
TC_PRODUCT_MIN_VECTORS = 8
TC_PRODUCT_MIN_ENTRIES = 1 << 22


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
  def _apply_raw(self, f: torch.Tensor, g: torch.Tensor, v2: torch.Tensor,
                 axis: int, precision: str = "fp32") -> torch.Tensor:
    """The plan applied to ``v2 [k, n or m]`` (no autograd):
    ``ottb_apply_transport`` (FP32), or with ``precision`` "auto" (d >= 32)
    or "bf16_split3" ``ottb_apply_transport_sweep`` on the solver's
    tensor-core sweep ("sweep_fp32": that entry point on the FP32 sweep)."""
    lib = _lib.load()
    n, m = self.shape
    dev = self.x.device
    v2 = _arrays.as_f32(v2, dev).detach().contiguous()
    fd = _arrays.as_f32(f, dev).detach()
    gd = _arrays.as_f32(g, dev).detach()
    out = torch.empty((v2.shape[0], m if axis == 0 else n), dtype=torch.float32, device=dev)
    if v2.shape[0] == 0:
      return out
    sweep = {"bf16_split3": _lib.PRECISION_BF16_SPLIT3, "sweep_fp32": _lib.PRECISION_FP32}
    if precision == "auto" and self.dim >= 32:
      precision = "bf16_split3"
    if precision == "bf16_split3_tc":
      return self._apply_tc(fd, gd, v2, axis, out)
    if precision in sweep:
      code = sweep[precision]
      ws_bytes = _sweep_ws_bytes(n, m, self.dim, v2.shape[0], axis, code)
      if ws_bytes == 0:
        raise NotImplementedError("problem sizes not supported by the sweep engine")
      ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
      st = lib.ottb_apply_transport_sweep(
          self.x.data_ptr(), self.y.data_ptr(), n, m, self.dim, fd.data_ptr(), gd.data_ptr(),
          ctypes.c_float(self.epsilon), ctypes.c_float(self.inv_scale_cost), v2.data_ptr(),
          v2.shape[0], axis, code, out.data_ptr(), ws.data_ptr(), ws_bytes,
          _arrays.stream_handle())
      _lib.check(st, "ottb_apply_transport_sweep")
      return out
    ws_bytes = _apply_ws_bytes(n, m, self.dim, v2.shape[0], axis)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    st = lib.ottb_apply_transport(self.x.data_ptr(), self.y.data_ptr(), n, m, self.dim,
                                  fd.data_ptr(), gd.data_ptr(), ctypes.c_float(self.epsilon),
                                  ctypes.c_float(self.inv_scale_cost), v2.data_ptr(),
                                  v2.shape[0], axis, out.data_ptr(), ws.data_ptr(), ws_bytes,
                                  _arrays.stream_handle())
    _lib.check(st, "ottb_apply_transport")
    return out

  def _apply_tc(self, fd: torch.Tensor, gd: torch.Tensor, v2: torch.Tensor, axis: int,
                out: torch.Tensor) -> torch.Tensor:
    """``ottb_apply_transport_tc``: both products of the application on the
    tensor cores (BF16 split-3, FP32 accumulation), for many vectors."""
    lib = _lib.load()
    n, m = self.shape
    ws_bytes = int(lib.ottb_apply_transport_tc_workspace_size(n, m, self.dim, v2.shape[0], axis))
    if ws_bytes == 0:
      raise NotImplementedError("problem sizes not supported by ottb_apply_transport_tc")
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=v2.device)
    st = lib.ottb_apply_transport_tc(
        self.x.data_ptr(), self.y.data_ptr(), n, m, self.dim, fd.data_ptr(), gd.data_ptr(),
        ctypes.c_float(self.epsilon), ctypes.c_float(self.inv_scale_cost), v2.data_ptr(),
        v2.shape[0], axis, out.data_ptr(), ws.data_ptr(), ws_bytes, _arrays.stream_handle())
    _lib.check(st, "ottb_apply_transport_tc")
    return out

  def _sweep_product(self, f: torch.Tensor, g: torch.Tensor, axis: int, precision: str,
                     num_vec: int = 1) -> Optional["_SweepProduct"]:
    """``_apply_raw`` on the sweep route planned once for fixed potentials
    (``ottb_apply_transport_sweep_plan``): calling the result with
    ``v2 [num_vec, n or m]`` issues stream operations only. None where
    ``precision`` does not take the sweep route."""
    if precision == "auto" and self.dim >= 32:
      precision = "bf16_split3"
    code = {"bf16_split3": _lib.PRECISION_BF16_SPLIT3,
            "sweep_fp32": _lib.PRECISION_FP32}.get(precision)
    if code is None:
      return None
    return _SweepProduct(self, f, g, axis, code, num_vec)

  def _apply_product(self, f: torch.Tensor, g: torch.Tensor, axis: int,
                     num_vec: int = 1) -> "_ApplyProduct":
    """``_apply_raw``'s FP32 product (``ottb_apply_transport``) planned once
    for fixed potentials (``ottb_apply_transport_plan``)."""
    return _ApplyProduct(self, f, g, axis, num_vec)

  def apply_transport_from_potentials(self, f: torch.Tensor, g: torch.Tensor, vec: Any,
                                      axis: int = 0, precision: str = "fp32") -> torch.Tensor:
    """Applies ``P_ij = exp((f_i + g_j - C_ij) / eps)`` to ``vec`` without
    forming P (geometry.py:444-486): ``axis=0`` sums over rows
    (``vec [..., n] -> [..., m]``), ``axis=1`` over columns
    (``vec [..., m] -> [..., n]``). ``vec`` may be 1-D or a batch.
    Differentiable w.r.t. the points, ``f``, ``g`` and ``vec``.

    ``precision`` (not in the reference): "fp32" (FP32 on the CUDA cores),
    or "bf16_split3" / "auto" (d >= 32), which takes batches of at least
    ``TC_PRODUCT_MIN_VECTORS`` vectors on problems of at least
    ``TC_PRODUCT_MIN_ENTRIES`` plan entries to the tensor cores
    (``ottb_apply_transport_tc``) and the rest to FP32."""
    if axis not in (0, 1):
      raise ValueError("axis must be 0 or 1")
    n, m = self.shape
    dev = self.x.device
    v = _arrays.as_f32(vec, dev)
    one = v.ndim == 1
    v2 = v.reshape(1, -1) if one else v.reshape(-1, v.shape[-1])
    if v2.shape[1] != (n if axis == 0 else m):
      raise ValueError(f"vec has length {v2.shape[1]}, expected {n if axis == 0 else m}")
    f = _arrays.as_f32(f, dev)
    g = _arrays.as_f32(g, dev)
    prec = self._product_precision(precision, v2.shape[0])
    if _needs_grad(self.x, self.y, f, g, v2):
      out = _ApplyTransport.apply(self.x, self.y, f, g, v2, self, axis, precision)
    else:
      out = self._apply_raw(f, g, v2, axis, prec)
    return out[0] if one else out.reshape(*v.shape[:-1], out.shape[-1])

  def _product_precision(self, precision: str, num_vec: int) -> str:
    """``_apply_raw``'s route for a batch of ``num_vec`` vectors under the
    public ``precision`` of ``apply_transport_from_potentials``."""
    if precision not in ("fp32", "auto", "bf16_split3"):
      raise ValueError("precision must be 'fp32', 'auto' or 'bf16_split3'")
    if precision == "fp32" or (precision == "auto" and self.dim < 32):
      return "fp32"
    n, m = self.shape
    if num_vec >= TC_PRODUCT_MIN_VECTORS and n * m >= TC_PRODUCT_MIN_ENTRIES:
      return "bf16_split3_tc"
    return "fp32"

  def transport_from_potentials(self, f: torch.Tensor, g: torch.Tensor) -> torch.Tensor:
    """The plan ``[n, m]`` (geometry.py:361-365); differentiable w.r.t. the
    points, ``f`` and ``g``."""
    dev = self.x.device
    f = _arrays.as_f32(f, dev)
    g = _arrays.as_f32(g, dev)
    if _needs_grad(self.x, self.y, f, g):
      return _TransportMatrix.apply(self.x, self.y, f, g, self)
    return self._matrix_raw(f, g)

  def _matrix_raw(self, f: torch.Tensor, g: torch.Tensor) -> torch.Tensor:
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

  def _points_vjp(self, rows: torch.Tensor, gy_rows: torch.Tensor, cols: torch.Tensor,
                  gx_cols: torch.Tensor, gc: Optional[torch.Tensor]
                  ) -> Tuple[torch.Tensor, torch.Tensor]:
    """Gradient w.r.t. the points of a cost cotangent ``G`` (``dL/dC``,
    ``C_ij = inv |x_i - y_j|^2``) given through ``rows = G 1``,
    ``gy_rows = G y``, ``cols = G^T 1``, ``gx_cols = G^T x`` and, for
    ``scale_cost="mean"``, ``gc = <G, |x_i - y_j|^2>`` (the cotangent of
    ``inv = 1 / mean(C_unscaled)``, pointcloud.py:348-351, whose gradient
    is ``-inv^2 (2/n)(x_i - mean(y))``; a float scale is a constant)."""
    x, y = self.x.detach().double(), self.y.detach().double()
    n, m = self.shape
    inv = float(self.inv_scale_cost)
    gx = 2.0 * inv * (rows[:, None] * x - gy_rows)
    gy = 2.0 * inv * (cols[:, None] * y - gx_cols)
    if self._scale_cost == "mean" and gc is not None:
      gx = gx - inv * inv * (2.0 / n) * (x - y.mean(0)) * gc
      gy = gy - inv * inv * (2.0 / m) * (y - x.mean(0)) * gc
    return gx, gy

  def _plan_vjp(self, f: torch.Tensor, g: torch.Tensor, alpha: torch.Tensor,
                beta: torch.Tensor, points: bool = True, precision: str = "fp32"):
    """Backward of the plan for a cotangent of the low-rank form
    ``dL/dP = sum_t alpha_t beta_t^T`` (``alpha [T, n]``, ``beta [T, m]``),
    without forming P. Returns ``(gx, gy, u, w)`` in float64: ``u = P
    beta_t`` ``[T, n]``, ``w = P^T alpha_t`` ``[T, m]`` (so ``dL/df = sum_t
    alpha_t u_t / eps`` and ``dL/dg = sum_t beta_t w_t / eps``) and the
    gradient w.r.t. the points (None unless ``points``) through
    ``dP_ij/dC_ij = -P_ij / eps``. Two applications of the plan: to
    ``[beta_t, beta_t y, beta_t |y|^2]`` and to ``[alpha_t, alpha_t x]``."""
    eps = float(self.epsilon)
    n, m = self.shape
    d = self.dim
    T = alpha.shape[0]
    alpha, beta = alpha.double(), beta.double()
    route = lambda k: self._product_precision(precision, k)  # noqa: E731
    if not points:
      u = self._apply_raw(f, g, beta, 1, route(T)).double()
      w = self._apply_raw(f, g, alpha, 0, route(T)).double()
      return None, None, u, w
    x, y = self.x.detach().double(), self.y.detach().double()
    mean = self._scale_cost == "mean"
    parts = [beta[:, None, :], beta[:, None, :] * y.t()[None]]
    if mean:
      parts.append((beta * (y * y).sum(1)[None])[:, None, :])
    k_r = len(parts) - 1 + d
    r = self._apply_raw(f, g, torch.cat(parts, 1).reshape(T * k_r, m), 1,
                        route(T * k_r)).double()
    r = r.reshape(T, k_r, n)
    u, py = r[:, 0], r[:, 1:1 + d]
    c = self._apply_raw(f, g, torch.cat([alpha[:, None, :], alpha[:, None, :] * x.t()[None]],
                                        1).reshape(T * (1 + d), n), 0,
                        route(T * (1 + d))).double()
    c = c.reshape(T, 1 + d, m)
    w, ptx = c[:, 0], c[:, 1:]
    # G = dL/dC = -(1/eps) sum_t diag(alpha_t) P diag(beta_t)
    rows = -(alpha * u).sum(0) / eps
    gy_rows = -(alpha[:, None, :] * py).sum(0).t() / eps
    cols = -(beta * w).sum(0) / eps
    gx_cols = -(beta[:, None, :] * ptx).sum(0).t() / eps
    gc = None
    if mean:
      pysq = r[:, 1 + d]
      xsq = (x * x).sum(1)
      gc = -(alpha * (xsq[None] * u + pysq - 2.0 * (py * x.t()[None]).sum(1))).sum() / eps
    gx, gy = self._points_vjp(rows, gy_rows, cols, gx_cols, gc)
    return gx, gy, u, w

  def apply_lse_kernel(self, f: torch.Tensor, g: torch.Tensor, eps: float,
                       vec: Any = None, axis: int = 0,
                       precision: str = "fp32") -> Tuple[torch.Tensor, torch.Tensor]:
    """geometry.py:259-299 with ``vec=None``: ``eps log sum exp((f + g - C)
    / eps)`` over rows (``axis=0``, one value per column) or columns,
    minus the finite part of g (axis 0) or f, and the sign 1.
    ``ottb_apply_lse_kernel`` on the solver's sweep ("auto" / "bf16_split3":
    tensor cores for d >= 32)."""
    if vec is not None:
      raise NotImplementedError("the signed-vector form is apply_transport_from_potentials")
    if axis not in (0, 1):
      raise ValueError("axis must be 0 or 1")
    lib = _lib.load()
    n, m = self.shape
    dev = self.x.device
    pot = _arrays.as_f32(f if axis == 0 else g, dev).detach().contiguous()
    rem = _arrays.as_f32(g if axis == 0 else f, dev).detach()
    code = {"auto": _lib.PRECISION_AUTO, "fp32": _lib.PRECISION_FP32,
            "bf16_split3": _lib.PRECISION_BF16_SPLIT3}[precision]
    ws_bytes = lib.ottb_apply_lse_kernel_workspace_size(n, m, self.dim, axis, code)
    if ws_bytes == 0:
      raise NotImplementedError("problem sizes not supported")
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    out = torch.empty(m if axis == 0 else n, dtype=torch.float32, device=dev)
    st = lib.ottb_apply_lse_kernel(self.x.data_ptr(), self.y.data_ptr(), n, m, self.dim,
                                   pot.data_ptr(), ctypes.c_float(eps),
                                   ctypes.c_float(self.inv_scale_cost), axis, code,
                                   out.data_ptr(), ws.data_ptr(), ws_bytes,
                                   _arrays.stream_handle())
    _lib.check(st, "ottb_apply_lse_kernel")
    # a -inf potential on the output side makes every entry -inf there
    out = torch.where(torch.isneginf(rem), torch.full_like(out, -float("inf")), out)
    return out, torch.ones(1, device=dev)

  def update_potential(self, f: torch.Tensor, g: torch.Tensor, log_marginal: Any,
                       iteration: Optional[int] = None, axis: int = 0,
                       precision: str = "fp32") -> torch.Tensor:
    """geometry.py:376-398: one Sinkhorn update, ``eps log_marginal -
    where(isfinite(lse), lse, 0)`` with ``lse = apply_lse_kernel(f, g, eps,
    axis)`` at the scheduled epsilon of ``iteration``: the new g for
    ``axis=0``, the new f for ``axis=1``."""
    eps = float(self.epsilon_scheduler(iteration))
    app, _ = self.apply_lse_kernel(f, g, eps, axis=axis, precision=precision)
    lm = _arrays.as_f32(log_marginal, self.x.device)
    return eps * lm - torch.where(torch.isfinite(app), app, torch.zeros_like(app))

  @property
  def cost_matrix(self) -> torch.Tensor:
    """The scaled cost ``[n, m]`` (geometry.py:95-105; formed, for problems
    whose n x m matrix fits): ``inv (|x|^2 + |y|^2 - 2 <x, y>)``."""
    x, y = self.x, self.y
    c = (x * x).sum(1)[:, None] + (y * y).sum(1)[None, :] - 2.0 * (x @ y.t())
    return self.inv_scale_cost * c

  @property
  def kernel_matrix(self) -> torch.Tensor:
    """geometry.py:137-145: ``exp(-C / eps)``, formed."""
    return torch.exp(-self.cost_matrix / self.epsilon)

  @property
  def diag_cost(self) -> torch.Tensor:
    """pointcloud.py:451-454: the cost function on the pairs (x_i, y_i) of a
    square problem (without ``scale_cost``, as there)."""
    assert self.is_square, "Cost matrix must be square to compute diagonal."
    return ((self.x - self.y) ** 2).sum(1)

  def apply_cost(self, arr: Any, axis: int = 0, fn: Optional[Any] = None,
                 is_linear: bool = False) -> torch.Tensor:
    """geometry.py:568-600 for the squared Euclidean cost without ``fn``:
    ``C^T arr`` (axis 0, arr [n] or [n, p]) or ``C arr`` (axis 1) through the
    rank d + 2 structure ``C = inv (|x|^2 1^T + 1 |y|^2^T - 2 x y^T)``, in
    O((n + m) d p) without forming C."""
    if fn is not None:
      raise NotImplementedError("an elementwise fn of the cost is not on this path")
    v = _arrays.as_f32(arr, self.x.device)
    one = v.ndim == 1
    v2 = v[:, None] if one else v
    x, y = self.x, self.y
    nx, ny = (x * x).sum(1), (y * y).sum(1)
    if axis == 0:   # C^T v: sum over rows
      out = ny[:, None] * v2.sum(0)[None, :] + (nx @ v2)[None, :] - 2.0 * (y @ (x.t() @ v2))
    else:           # C v: sum over columns
      out = nx[:, None] * v2.sum(0)[None, :] + (ny @ v2)[None, :] - 2.0 * (x @ (y.t() @ v2))
    out = self.inv_scale_cost * out
    return out[:, 0] if one else out

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


@functools.lru_cache(maxsize=256)
def _apply_ws_bytes(n: int, m: int, d: int, k: int, axis: int) -> int:
  """Workspace of ``ottb_apply_transport`` (a function of the shapes and the
  device's SM count, fixed per process)."""
  return int(_lib.load().ottb_apply_transport_workspace_size(n, m, d, k, axis))


@functools.lru_cache(maxsize=256)
def _sweep_ws_bytes(n: int, m: int, d: int, k: int, axis: int, code: int) -> int:
  """Workspace of ``ottb_apply_transport_sweep`` (a function of the shapes)."""
  return int(_lib.load().ottb_apply_transport_sweep_workspace_size(n, m, d, k, axis, code))


def _needs_grad(*ts: torch.Tensor) -> bool:
  return torch.is_grad_enabled() and any(t.requires_grad for t in ts)


def _cast(t: Optional[torch.Tensor], like: torch.Tensor, need: bool):
  return t.to(like.dtype) if (need and t is not None) else None


class _ApplyTransport(torch.autograd.Function):
  """``vec -> P^T vec`` (axis 0) or ``P vec`` (axis 1) as a function of
  ``(x, y, f, g, vec)``; its backward is two more applications of the plan
  (``PointCloud._plan_vjp``)."""

  @staticmethod
  def forward(ctx, x, y, f, g, v2, geom, axis, precision):  # pylint: disable=arguments-differ
    out = geom._apply_raw(f, g, v2, axis, geom._product_precision(precision, v2.shape[0]))
    ctx.geom, ctx.axis, ctx.precision = geom, axis, precision
    ctx.save_for_backward(f, g, v2)
    return out

  @staticmethod
  @torch.autograd.function.once_differentiable
  def backward(ctx, gout):  # pylint: disable=arguments-differ
    f, g, v2 = ctx.saved_tensors
    geom, axis = ctx.geom, ctx.axis
    need = ctx.needs_input_grad
    eps = float(geom.epsilon)
    W, V = gout.double(), v2.double()
    # axis 0: out_k = P^T v_k, dL/dP = sum_k v_k W_k^T; axis 1: out_k = P v_k
    alpha, beta = (V, W) if axis == 0 else (W, V)
    gx, gy, u, w = geom._plan_vjp(f, g, alpha, beta, points=need[0] or need[1],
                                  precision=ctx.precision)
    gf = (alpha * u).sum(0) / eps
    gg = (beta * w).sum(0) / eps
    gv = u if axis == 0 else w
    return (_cast(gx, geom.x, need[0]), _cast(gy, geom.y, need[1]), _cast(gf, f, need[2]),
            _cast(gg, g, need[3]), _cast(gv, v2, need[4]), None, None, None)


class _TransportMatrix(torch.autograd.Function):
  """The dense plan as a function of ``(x, y, f, g)``; backward with dense
  products (the plan is formed anyway)."""

  @staticmethod
  def forward(ctx, x, y, f, g, geom):  # pylint: disable=arguments-differ
    p = geom._matrix_raw(f, g)
    ctx.geom = geom
    ctx.save_for_backward(f, g, p)
    return p

  @staticmethod
  @torch.autograd.function.once_differentiable
  def backward(ctx, gp):  # pylint: disable=arguments-differ
    f, g, p = ctx.saved_tensors
    geom = ctx.geom
    need = ctx.needs_input_grad
    eps = float(geom.epsilon)
    e = gp.double() * p.double()
    gf = e.sum(1) / eps
    gg = e.sum(0) / eps
    gx = gy = None
    if need[0] or need[1]:
      x, y = geom.x.detach().double(), geom.y.detach().double()
      G = -e / eps
      rows, cols = G.sum(1), G.sum(0)
      gy_rows, gx_cols = G @ y, G.t() @ x
      gc = ((rows * (x * x).sum(1)).sum() + (cols * (y * y).sum(1)).sum()
            - 2.0 * (x * gy_rows).sum())
      gx, gy = geom._points_vjp(rows, gy_rows, cols, gx_cols, gc)
    return (_cast(gx, geom.x, need[0]), _cast(gy, geom.y, need[1]), _cast(gf, f, need[2]),
            _cast(gg, g, need[3]), None)


def _keep_until_done(*tensors: torch.Tensor) -> None:
  """Marks tensors as in use on the current stream, so the caching allocator
  does not hand their memory to another stream's work before the product
  queued here has run (a product may run on a stream other than the one its
  plan was made on)."""
  st = torch.cuda.current_stream(tensors[0].device)
  for t in tensors:
    t.record_stream(st)


class _SweepProduct:
  """One planned ``ottb_apply_transport_sweep`` product (the plan applied to
  vectors through zero-iteration solves on the solver's sweep engine). It
  owns the handle and the workspace and keeps the points and both
  potentials alive; the handle is freed with the object."""

  def __init__(self, geom: "PointCloud", f: torch.Tensor, g: torch.Tensor, axis: int,
               code: int, num_vec: int):
    lib = _lib.load()
    n, m = geom.shape
    dev = geom.x.device
    self._lib = lib
    self._handle = None
    self._x, self._y = geom.x, geom.y
    self._f = _arrays.as_f32(f, dev).detach().contiguous()
    self._g = _arrays.as_f32(g, dev).detach().contiguous()
    self._axis, self._num_vec = axis, num_vec
    self._rows_in, self._rows_out = (n, m) if axis == 0 else (m, n)
    ws_bytes = _sweep_ws_bytes(n, m, geom.dim, num_vec, axis, code)
    if ws_bytes == 0:
      raise NotImplementedError("problem sizes not supported by the sweep engine")
    self._ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    h = ctypes.c_void_p()
    st = lib.ottb_apply_transport_sweep_plan(
        geom.x.data_ptr(), geom.y.data_ptr(), n, m, geom.dim, self._f.data_ptr(),
        self._g.data_ptr(), ctypes.c_float(geom.epsilon), ctypes.c_float(geom.inv_scale_cost),
        num_vec, axis, code, self._ws.data_ptr(), ws_bytes, _arrays.stream_handle(),
        ctypes.byref(h))
    _lib.check(st, "ottb_apply_transport_sweep_plan")
    self._handle = h.value

  def __call__(self, v2: torch.Tensor) -> torch.Tensor:
    v2 = _arrays.as_f32(v2, self._ws.device).detach().contiguous()
    if v2.shape != (self._num_vec, self._rows_in):
      raise ValueError(f"vectors of shape {tuple(v2.shape)}, planned for "
                       f"{(self._num_vec, self._rows_in)}")
    out = torch.empty((self._num_vec, self._rows_out), dtype=torch.float32,
                      device=self._ws.device)
    pot = self._f if self._axis == 0 else self._g
    _keep_until_done(self._ws, self._f, self._g)
    st = self._lib.ottb_apply_transport_sweep_run(self._handle, pot.data_ptr(), v2.data_ptr(),
                                                  out.data_ptr(), _arrays.stream_handle())
    _lib.check(st, "ottb_apply_transport_sweep_run")
    return out

  def __del__(self):
    if getattr(self, "_handle", None):
      self._lib.ottb_apply_transport_sweep_free(self._handle)
      self._handle = None


class _ApplyProduct:
  """One planned ``ottb_apply_transport`` product (FP32 on the CUDA cores).
  It owns the handle and the workspace and keeps the points and both
  potentials alive and unchanged; the handle is freed with the object."""

  def __init__(self, geom: "PointCloud", f: torch.Tensor, g: torch.Tensor, axis: int,
               num_vec: int):
    lib = _lib.load()
    n, m = geom.shape
    dev = geom.x.device
    self._lib = lib
    self._handle = None
    self._x, self._y = geom.x, geom.y
    self._f = _arrays.as_f32(f, dev).detach().contiguous().clone()
    self._g = _arrays.as_f32(g, dev).detach().contiguous().clone()
    self._num_vec = num_vec
    self._rows_in, self._rows_out = (n, m) if axis == 0 else (m, n)
    ws_bytes = _apply_ws_bytes(n, m, geom.dim, num_vec, axis)
    self._ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    h = ctypes.c_void_p()
    st = lib.ottb_apply_transport_plan(
        geom.x.data_ptr(), geom.y.data_ptr(), n, m, geom.dim, self._f.data_ptr(),
        self._g.data_ptr(), ctypes.c_float(geom.epsilon), ctypes.c_float(geom.inv_scale_cost),
        num_vec, axis, self._ws.data_ptr(), ws_bytes, _arrays.stream_handle(), ctypes.byref(h))
    _lib.check(st, "ottb_apply_transport_plan")
    self._handle = h.value

  def __call__(self, v2: torch.Tensor) -> torch.Tensor:
    v2 = _arrays.as_f32(v2, self._ws.device).detach().contiguous()
    if v2.shape != (self._num_vec, self._rows_in):
      raise ValueError(f"vectors of shape {tuple(v2.shape)}, planned for "
                       f"{(self._num_vec, self._rows_in)}")
    out = torch.empty((self._num_vec, self._rows_out), dtype=torch.float32,
                      device=self._ws.device)
    _keep_until_done(self._ws, self._f, self._g)
    st = self._lib.ottb_apply_transport_run(self._handle, v2.data_ptr(), out.data_ptr(),
                                            _arrays.stream_handle())
    _lib.check(st, "ottb_apply_transport_run")
    return out

  def __del__(self):
    if getattr(self, "_handle", None):
      self._lib.ottb_apply_transport_free(self._handle)
      self._handle = None
