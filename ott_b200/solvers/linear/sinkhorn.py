"""Sinkhorn solver (ott/solvers/linear/sinkhorn.py), log-domain, on B200.

``Sinkhorn.__call__`` mirrors sinkhorn.py:782-801: run the initializer (or
take ``init``), then one C-ABI call (``ottb_sinkhorn_pointcloud``) runs the
whole fixed-point loop of fixed_point_loop.py:23-93 in one persistent
launch and fills ``f``, ``g``, ``errors`` and the scalar results
(``reg_ot_cost``, ``n_iters``, ``converged``).

Supported: balanced problems, ``lse_mode=True``, default ``Momentum()``
(weight 1), sequential updates, ``norm_error >= 1``, epsilon schedules,
``min_iterations`` / ``max_iterations`` / ``inner_iterations``, warm starts
through ``init=(f, g)`` or an initializer. Everything else raises
``NotImplementedError`` rather than silently changing the algorithm.
"""
from __future__ import annotations

import ctypes
import math
import time
from typing import Any, List, NamedTuple, Optional, Sequence, Tuple

import torch

from ott_b200 import _arrays, _lib
from ott_b200.geometry import epsilon_scheduler as eps_scheduler
from ott_b200.initializers.linear import initializers as init_lib
from ott_b200.problems.linear import linear_problem
from ott_b200.solvers.linear import implicit_differentiation as implicit_lib

__all__ = ["set_schedule", "Sinkhorn", "SinkhornGraph", "SinkhornOutput", "run_batch"]

_PRECISIONS = {
    "auto": _lib.PRECISION_AUTO,
    "fp32": _lib.PRECISION_FP32,
    "bf16_split3": _lib.PRECISION_BF16_SPLIT3,
}


class _Results:
  """Device-side ``ottb_result`` records, read back to the host once."""

  def __init__(self, buf: torch.Tensor, num: int):
    self._buf = buf
    self._num = num
    self._host: Optional[List[_lib.OttbResult]] = None

  def get(self, k: int) -> _lib.OttbResult:
    if self._host is None:
      raw = self._buf.cpu().numpy().tobytes()
      sz = _lib.RESULT_BYTES
      self._host = [_lib.OttbResult.from_buffer_copy(raw[i * sz:(i + 1) * sz])
                    for i in range(self._num)]
      for r in self._host:
        if r.status != _lib.OTTB_OK:
          raise _lib.OttbError(r.status, "ottb_sinkhorn_pointcloud (device)")
    return self._host[k]


class SinkhornOutput(NamedTuple):
  """Output of the solver (sinkhorn.py:280-538).

  ``potentials`` are torch CUDA tensors; ``errors`` has length
  ``ceil(max_iterations / inner_iterations)`` with the reference's
  conventions (-1: not reached, inf: not computed).
  """

  potentials: Tuple[torch.Tensor, torch.Tensor]
  errors: Optional[torch.Tensor] = None
  reg_ot_cost_: Optional[Any] = None  # (_Results, index)
  ot_prob: Optional[linear_problem.LinearProblem] = None
  threshold: Optional[float] = None
  inner_iterations: Optional[int] = None
  symmetric: bool = False  # solved with the symmetric update (f = g, x = y)
  use_danskin: bool = True  # gradient of reg_ot_cost with f, g held fixed
  precision: str = "fp32"  # the solve's arithmetic; plan applications follow it

  def _res(self) -> _lib.OttbResult:
    results, k = self.reg_ot_cost_
    return results.get(k)

  @property
  def f(self) -> torch.Tensor:
    return self.potentials[0]

  @property
  def g(self) -> torch.Tensor:
    return self.potentials[1]

  @property
  def reg_ot_cost(self) -> Any:
    """sinkhorn.py:224-277 (balanced), FP64 sums on the device: a float, or
    a differentiable 0-dim float64 tensor when the problem's points or
    weights require gradients (with ``use_danskin`` the gradient holds the
    potentials fixed, sinkhorn.py:329-335; otherwise it also flows through
    the potentials' implicit backward)."""
    val = self._res().reg_ot_cost
    if self.ot_prob is None or not _tracks_grad(self.ot_prob):
      return val
    return _reg_ot_cost_tensor(self)

  @property
  def kl_reg_cost(self) -> float:
    return self.reg_ot_cost

  @property
  def converged(self) -> bool:
    """sinkhorn.py:1020-1023."""
    return bool(self._res().converged)

  @property
  def n_iters(self) -> int:
    """sinkhorn.py:432-434."""
    return int(self._res().n_iters)

  @property
  def geom(self):
    return self.ot_prob.geom

  @property
  def a(self) -> torch.Tensor:
    return self.ot_prob.a

  @property
  def b(self) -> torch.Tensor:
    return self.ot_prob.b

  @property
  def dual_cost(self) -> Any:
    """sinkhorn.py:337-343; a differentiable 0-dim tensor when the problem's
    points or weights require gradients (through the potentials' implicit
    backward), else a float."""
    a, b = self.a.double(), self.b.double()
    f, g = self.f.double(), self.g.double()
    zero = torch.zeros((), dtype=torch.float64, device=a.device)
    # mask before multiplying: a zero weight meets an infinite potential
    val = ((a * torch.where(a > 0, f, zero)).sum() + (b * torch.where(b > 0, g, zero)).sum())
    return val if (self.ot_prob is not None and _tracks_grad(self.ot_prob)) else float(val)

  @property
  def ent_reg_cost(self) -> float:
    """sinkhorn.py:351-370: ``reg_ot_cost - eps * (H(a) + H(b))``."""
    def entr(p):
      p = p.double()
      safe = torch.where(p > 0, p, torch.ones_like(p))
      return torch.where(p > 0, -p * torch.log(safe), torch.zeros_like(p)).sum()
    return self.reg_ot_cost - self.geom.epsilon * float(entr(self.a) + entr(self.b))

  @property
  def transport_mass(self) -> Any:
    """Sum of the transport matrix (sinkhorn.py:451-454, ``marginal(0).sum()``):
    the final sweep's FP64 sum, or a differentiable tensor when the problem's
    points or weights require gradients."""
    if self.ot_prob is not None and _tracks_grad(self.ot_prob):
      return self.marginal(0).double().sum()
    return float(self._res().marginal_sum)

  @property
  def scalings(self) -> Tuple[torch.Tensor, torch.Tensor]:
    """sinkhorn.py:437-441: ``exp(f / eps), exp(g / eps)``
    (geometry.py:535-546)."""
    eps = float(self.geom.epsilon)
    return torch.exp(self.f / eps), torch.exp(self.g / eps)

  @property
  def entropy(self) -> Any:
    """Entropy of the coupling (sinkhorn.py:513-523):
    ``(primal_cost - <f, P 1> - <g, P^T 1>) / eps`` with non-finite
    potentials counted as 0."""
    ma = self.marginal(1).double()
    mb = self.marginal(0).double()
    f, g = self.f.double(), self.g.double()
    zero = torch.zeros((), dtype=torch.float64, device=f.device)
    sf = torch.where(torch.isfinite(f), f, zero)
    sg = torch.where(torch.isfinite(g), g, zero)
    val = (self.primal_cost - torch.dot(sf, ma) - torch.dot(sg, mb)) / float(self.geom.epsilon)
    return val if (self.ot_prob is not None and _tracks_grad(self.ot_prob)) else float(val)

  @property
  def normalized_entropy(self) -> Any:
    """sinkhorn.py:525-530: ``entropy / log(n) - 1`` of an assignment
    problem (equal sizes, uniform weights, balanced)."""
    assert self.ot_prob.is_assignment, "Normalized entropy only valid for assignment problem."
    return self.entropy / math.log(self.geom.shape[0]) - 1.0

  @property
  def diag(self) -> torch.Tensor:
    """Diagonal of the plan of a square problem (sinkhorn.py:532-538):
    ``exp((f_i + g_i - c(x_i, y_i)) / eps)`` with the diagonal cost of
    pointcloud.py:451-454, which is the cost function's value without
    ``scale_cost``."""
    geom = self.geom
    assert geom.is_square, "Problem must be square for transport matrix to have a diag."
    x, y = geom.x, geom.y
    diag = ((x - y) ** 2).sum(1)
    return torch.exp((-diag + self.f + self.g) / float(geom.epsilon))

  def transport_cost_at_geom(self, other_geom) -> Any:
    """``<P, C_other>`` for the plan of this solution and the cost of another
    point cloud of the same sizes (sinkhorn.py:395-417; the squared Euclidean
    cost is a rank d + 2 product there): one application of the plan to
    ``[1, |y'|^2, y']``, times ``other_geom``'s scale."""
    if tuple(other_geom.shape) != tuple(self.geom.shape):
      raise ValueError("the other geometry must have the same shape")
    diff = self.ot_prob is not None and _tracks_grad(self.ot_prob)
    with torch.set_grad_enabled(diff):
      x, y = other_geom.x.double(), other_geom.y.double()
      vecs = torch.cat([torch.ones_like(y[:, :1]), (y * y).sum(1, keepdim=True), y], 1)
      r = self.apply(vecs.t().float(), axis=1).double()  # [d + 2, n]
      tot = (r[0] * (x * x).sum(1) + r[1] - 2.0 * (r[2:].t() * x).sum(1)).sum()
      val = float(other_geom.inv_scale_cost) * tot
    return val if diff else float(val)

  def cost_at_geom(self, other_geom) -> Any:
    """sinkhorn.py:502-507: ``sum(P * C_other) - eps sum(entr(P))`` with
    the plan formed (``matrix``); for problems whose n x m plan fits."""
    p = self.matrix.double()
    x, y = other_geom.x.double(), other_geom.y.double()
    c = float(other_geom.inv_scale_cost) * ((x * x).sum(1)[:, None] + (y * y).sum(1)[None, :]
                                            - 2.0 * x @ y.t())
    zero = torch.zeros((), dtype=torch.float64, device=p.device)
    entr = torch.where(p > 0, -p * torch.log(torch.where(p > 0, p, torch.ones_like(p))), zero)
    val = (p * c).sum() - float(self.geom.epsilon) * entr.sum()
    return val if (self.ot_prob is not None and _tracks_grad(self.ot_prob)) else float(val)

  def to_dual_potentials(self, epsilon: Optional[float] = None):
    """sinkhorn.py:509-511 builds potential functions of the
    ``problems/linear/potentials`` module, which is not on this path."""
    raise NotImplementedError("dual potential functions are not on this path")

  @property
  def matrix(self) -> torch.Tensor:
    """The transport plan ``[n, m]`` (sinkhorn.py:442-448)."""
    return self.geom.transport_from_potentials(self.f, self.g)

  def apply(self, inputs: Any, axis: int = 0) -> torch.Tensor:
    """The plan applied to ``inputs`` (sinkhorn.py:455-469); ``axis=0``
    maps ``[..., n]`` to ``[..., m]``, ``axis=1`` the transpose. After a
    tensor-core solve (precision "bf16_split3", or "auto" at d >= 32) large
    batches of vectors are applied on the tensor cores too."""
    return self.geom.apply_transport_from_potentials(self.f, self.g, inputs, axis=axis,
                                                     precision=self.precision)

  def marginal(self, axis: int) -> torch.Tensor:
    """sinkhorn.py:471-472."""
    return self.geom.marginal_from_potentials(self.f, self.g, axis=axis)

  def reg_ot_cost_grads(self) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor,
                                       torch.Tensor]:
    """Gradient of ``reg_ot_cost`` w.r.t. ``(x, y, a, b)`` with the
    potentials held fixed: the reference's default (``use_danskin=True``,
    sinkhorn.py:329-335, 779-780, which stops gradients through f and g in
    ``compute_kl_reg_cost``, :224-277). With ``P`` the plan,
    ``inv = inv_scale_cost`` and ``r = P 1``, ``c = P^T 1``:

      d/dx_i = 2 inv (r_i x_i - (P y)_i) + d(inv)/dx_i <P, C_unscaled>
      d/dy_j = 2 inv (c_j y_j - (P^T x)_j) + d(inv)/dy_j <P, C_unscaled>
      d/da_i = [a_i > 0] (f_i - eps log a_i - eps) + eps sum(b)
      d/db_j = [b_j > 0] (g_j - eps log b_j - eps) + eps sum(a)

    where ``d(inv)/dx_i = -inv^2 (2/n)(x_i - mean(y))`` for
    ``scale_cost="mean"`` (pointcloud.py:348-351, differentiable there) and
    0 for a fixed scale; epsilon is a constant (geometry.py:157-163 stop
    gradients through a relative epsilon). The plan is applied twice to
    ``d + 1`` vectors (``ottb_apply_transport``), never formed. At a zero
    weight the reference's ``jnp.where`` gives NaN gradients; here that
    term is 0.
    """
    with torch.no_grad():
      return self._reg_ot_cost_grads()

  def _reg_ot_cost_grads(self):
    geom = self.geom
    eps = float(geom.epsilon)
    inv = float(geom.inv_scale_cost)
    x, y = geom.x.detach(), geom.y.detach()
    n, m = geom.shape
    ones_n = torch.ones((1, n), dtype=torch.float32, device=x.device)
    ones_m = torch.ones((1, m), dtype=torch.float32, device=x.device)
    ry = self.apply(torch.cat([ones_m, y.t()], 0), axis=1).double()  # [1 + d, n]
    # symmetric solve: f = g and x = y make P symmetric, so the column
    # application equals the row one
    cx = ry if self.symmetric else self.apply(torch.cat([ones_n, x.t()], 0), axis=0).double()
    xd, yd = x.double(), y.double()
    r, py = ry[0], ry[1:].t()
    c, ptx = cx[0], cx[1:].t()
    gx = 2.0 * inv * (r[:, None] * xd - py)
    gy = 2.0 * inv * (c[:, None] * yd - ptx)
    if geom._scale_cost == "mean":
      tcost = ((r * (xd * xd).sum(1)).sum() + (c * (yd * yd).sum(1)).sum()
               - 2.0 * (xd * py).sum())
      gx = gx - inv * inv * (2.0 / n) * (xd - yd.mean(0)) * tcost
      gy = gy - inv * inv * (2.0 / m) * (yd - xd.mean(0)) * tcost
    a, b = self.a.detach().double(), self.b.detach().double()
    f, g = self.f.detach().double(), self.g.detach().double()
    zero = torch.zeros((), dtype=torch.float64, device=x.device)
    la = torch.log(torch.where(a > 0, a, torch.ones_like(a)))
    lb = torch.log(torch.where(b > 0, b, torch.ones_like(b)))
    ga = torch.where(a > 0, f - eps * la - eps, zero) + eps * b.sum()
    gb = torch.where(b > 0, g - eps * lb - eps, zero) + eps * a.sum()
    return gx, gy, ga, gb

  @property
  def primal_cost(self) -> Any:
    """``<P, C>`` (sinkhorn.py:346-349 through :395-417), from one
    application of the plan to ``[1, |y|^2, y]``. A differentiable 0-dim
    tensor when the problem's points or weights require gradients (the plan
    through the potentials' implicit backward and its own dependence on the
    points, the cost and, for ``scale_cost="mean"``, its scale
    ``1 / mean(C)``), else a float."""
    geom = self.geom
    diff = self.ot_prob is not None and _tracks_grad(self.ot_prob)
    with torch.set_grad_enabled(diff):
      x, y = geom.x.double(), geom.y.double()
      vecs = torch.cat([torch.ones_like(y[:, :1]), (y * y).sum(1, keepdim=True), y], 1)
      r = self.apply(vecs.t().float(), axis=1).double()  # [d + 2, n]
      tot = (r[0] * (x * x).sum(1) + r[1] - 2.0 * (r[2:].t() * x).sum(1)).sum()
      inv = float(geom.inv_scale_cost)
      if diff and geom._scale_cost == "mean":
        # 1 / mean(C_unscaled) as a function of the points (pointcloud.py:
        # 348-351), valued at the device's statistic
        mc = (x * x).sum(1).mean() + (y * y).sum(1).mean() - 2.0 * torch.dot(x.mean(0), y.mean(0))
        inv_t = 1.0 / mc
        inv = inv_t + (inv - inv_t.detach())
      val = inv * tot
    return val if diff else float(val)


def _tracks_grad(p: linear_problem.LinearProblem) -> bool:
  return torch.is_grad_enabled() and any(
      t.requires_grad for t in (p.geom.x, p.geom.y, p.a, p.b))


class _Potentials(torch.autograd.Function):
  """The solved ``(f, g)`` as a function of ``(x, y, a, b)``; backward by
  implicit differentiation of the first-order conditions
  (sinkhorn.py:1102-1136, ``ImplicitDiff.gradient``)."""

  @staticmethod
  def forward(ctx, x, y, a, b, f, g, prob, implicit_diff, precision):  # pylint: disable=arguments-differ
    ctx.prob, ctx.implicit_diff, ctx.precision = prob, implicit_diff, precision
    ctx.save_for_backward(f, g)
    return f.clone(), g.clone()

  @staticmethod
  @torch.autograd.function.once_differentiable
  def backward(ctx, gf, gg):  # pylint: disable=arguments-differ
    if ctx.implicit_diff is None:
      raise NotImplementedError("gradients through the potentials need implicit_diff "
                                "(unrolled differentiation is not on this path)")
    f, g = ctx.saved_tensors
    gf = torch.zeros_like(f) if gf is None else gf
    gg = torch.zeros_like(g) if gg is None else gg
    gx, gy, ga, gb = ctx.implicit_diff.gradient(ctx.prob, f, g, True, (gf, gg),
                                                precision=ctx.precision)
    need = ctx.needs_input_grad
    p = ctx.prob
    cast = lambda t, like, i: t.to(like.dtype) if need[i] else None
    return (cast(gx, p.geom.x, 0), cast(gy, p.geom.y, 1), cast(ga, p.a, 2),
            cast(gb, p.b, 3), None, None, None, None, None)


class _RegOTCost(torch.autograd.Function):
  """``reg_ot_cost`` of a solved problem as a function of ``(x, y, a, b)``,
  its backward the gradient with the potentials held fixed
  (``SinkhornOutput.reg_ot_cost_grads``)."""

  @staticmethod
  def forward(ctx, x, y, a, b, out):  # pylint: disable=arguments-differ
    ctx.out = out
    return torch.tensor(out._res().reg_ot_cost, dtype=torch.float64, device=x.device)

  @staticmethod
  @torch.autograd.function.once_differentiable
  def backward(ctx, gout):  # pylint: disable=arguments-differ
    gx, gy, ga, gb = ctx.out.reg_ot_cost_grads()
    need = ctx.needs_input_grad
    cast = lambda t, i: (gout * t).to(torch.float32) if need[i] else None
    return cast(gx, 0), cast(gy, 1), cast(ga, 2), cast(gb, 3), None


def _reg_ot_cost_tensor(out: SinkhornOutput) -> torch.Tensor:
  """``reg_ot_cost`` as a differentiable tensor: with ``use_danskin`` the
  fixed-potential gradient; otherwise compute_kl_reg_cost (sinkhorn.py:
  224-277) written on the differentiable potentials and plan, valued at
  the device's FP64 result."""
  p = out.ot_prob
  if out.use_danskin:
    return _RegOTCost.apply(p.geom.x, p.geom.y, p.a, p.b, out)
  geom = p.geom
  eps = float(geom.epsilon)
  a, b = p.a.double(), p.b.double()
  f, g = out.f.double(), out.g.double()
  zero = torch.zeros((), dtype=torch.float64, device=a.device)
  fa = torch.where(a > 0, f, zero)
  gb_ = torch.where(b > 0, g, zero)
  la = torch.log(torch.where(a > 0, a, torch.ones_like(a)))
  lb = torch.log(torch.where(b > 0, b, torch.ones_like(b)))
  mb = geom.marginal_from_potentials(out.f, out.g, axis=0).double()
  expr = ((a * (fa - eps * la)).sum() + (b * (gb_ - eps * lb)).sum()
          + eps * (a.sum() * b.sum() - mb.sum()))
  val = out._res().reg_ot_cost
  return expr + (val - expr.detach())


class Sinkhorn:
  """Sinkhorn solver (sinkhorn.py:542-780), same constructor arguments.

  Extra keyword: ``precision`` in ``{"auto", "fp32", "bf16_split3"}``
  selects the arithmetic of the cost inner products: ``"fp32"`` FMAs on the
  CUDA cores; ``"bf16_split3"`` tcgen05 tensor-core products of bf16 hi/lo
  splits (hi*hi + hi*lo + lo*hi, FP32 accumulation); ``"auto"`` (default)
  uses the tensor cores for d >= 32 and FP32 below.

  ``autotune=True``: before the first solve of each shape, time the
  candidate work schedules (``ottb_sinkhorn_autotune``) and use the fastest
  for every later solve of that shape in this process.
  """

  def __init__(
      self,
      lse_mode: bool = True,
      threshold: float = 1e-3,
      norm_error: int = 1,
      inner_iterations: int = 10,
      min_iterations: int = 0,
      max_iterations: int = 2000,
      momentum: Optional[Any] = None,
      anderson: Optional[Any] = None,
      parallel_dual_updates: bool = False,
      recenter_potentials: bool = False,
      use_danskin: Optional[bool] = None,
      implicit_diff: Optional[implicit_lib.ImplicitDiff] = implicit_lib.ImplicitDiff(),
      initializer: Optional[init_lib.SinkhornInitializer] = None,
      progress_fn: Optional[Any] = None,
      precision: str = "auto",
      timeout_ms: int = 0,
      autotune: bool = False,
  ):
    if not lse_mode:
      raise NotImplementedError("kernel mode (lse_mode=False) is not on this path")
    # Momentum: weight 1 (default), or weight 1/2 from iteration 0 together
    # with parallel updates (the symmetric update of the reference's
    # Sinkhorn divergence, run for problems with x = y and a = b).
    w = 1.0 if momentum is None else float(getattr(momentum, "value", 1.0))
    start = 0 if momentum is None else int(getattr(momentum, "start", 0))
    self._symmetric_update = bool(parallel_dual_updates) and w == 0.5 and start == 0
    if w != 1.0 and not self._symmetric_update:
      raise NotImplementedError("momentum other than weight 1 is on this path only as "
                                "Momentum(start=0, value=0.5) with parallel updates")
    if anderson is not None:
      raise NotImplementedError("Anderson acceleration is not on this path")
    if parallel_dual_updates and not self._symmetric_update:
      raise NotImplementedError("parallel dual updates are on this path only with "
                                "Momentum(start=0, value=0.5) on symmetric problems")
    if recenter_potentials:
      raise NotImplementedError("recentred potentials are not on this path")
    if precision not in _PRECISIONS:
      raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
    self.lse_mode = lse_mode
    self.threshold = threshold
    self.norm_error = norm_error
    self.inner_iterations = inner_iterations
    self.min_iterations = min_iterations
    self.max_iterations = max_iterations
    self.parallel_dual_updates = parallel_dual_updates
    self.recenter_potentials = recenter_potentials
    # sinkhorn.py:779-780
    self.use_danskin = (implicit_diff is not None) if use_danskin is None else bool(use_danskin)
    self.implicit_diff = implicit_diff
    self.initializer = (init_lib.DefaultInitializer()
                        if initializer is None else initializer)
    self.progress_fn = progress_fn
    self.precision = precision
    self.timeout_ms = timeout_ms
    self.autotune = autotune
    self._phantom_arrivals = 0

  @property
  def outer_iterations(self) -> int:
    """sinkhorn.py:956-962."""
    return int(math.ceil(self.max_iterations / self.inner_iterations))

  def _cfg(self, mask_init: bool, eps: eps_scheduler.Epsilon) -> _lib.OttbSolverCfg:
    c = _lib.OttbSolverCfg()
    c.threshold = float(self.threshold)
    c.norm_error = int(self.norm_error)
    c.inner_iterations = int(self.inner_iterations)
    c.min_iterations = int(self.min_iterations)
    c.max_iterations = int(self.max_iterations)
    c.eps_init = float(eps.init)
    c.eps_decay = float(eps.decay)
    c.precision = _PRECISIONS[self.precision]
    c.mask_init = 1 if mask_init else 0
    c.timeout_ms = int(self.timeout_ms)
    c.phantom_arrivals = int(self._phantom_arrivals)
    return c

  def __call__(self, ot_prob: linear_problem.LinearProblem,
               init: Optional[Tuple[Any, Any]] = None, **kwargs: Any) -> SinkhornOutput:
    return run_batch([ot_prob], self, [init], **kwargs)[0]


class _Call:
  """Problem records, configuration and device buffers of one C-ABI call
  over a batch of problems (initial potentials from ``inits`` or the
  solver's initializer, computed here, outside any graph)."""

  def __init__(self, probs: Sequence[linear_problem.LinearProblem], solver: Sinkhorn,
               inits: Optional[Sequence[Optional[Tuple[Any, Any]]]],
               f_from_g: Optional[bool], init_kwargs: dict,
               symmetric: Optional[Sequence[bool]] = None, live_errors: bool = False):
    self.lib = _lib.load()
    # live_errors: the kernel writes each block's error into pinned host
    # memory (device-accessible under unified addressing) that the host
    # reads while the solve runs; copied to the device buffers afterwards
    self.host_errors: List[torch.Tensor] = []
    self.probs = list(probs)
    self.solver = solver
    inits = list(inits) if inits is not None else [None] * len(probs)
    d = probs[0].geom.dim
    dev = probs[0].geom.x.device
    scheds = []
    for p in probs:
      if not p.is_balanced:
        raise NotImplementedError("unbalanced problems (tau < 1) are not on this path")
      if p.geom.dim != d:
        raise ValueError("all problems of one batch must have the same dimension")
      scheds.append(p.geom.epsilon_scheduler)
    s0 = scheds[0]
    for sch in scheds:
      if (sch.init, sch.decay) != (s0.init, s0.decay):
        raise ValueError("all problems of one batch must share the epsilon schedule")
    outer = solver.outer_iterations
    arr = (_lib.OttbProblem * len(probs))()
    keep: List[torch.Tensor] = []
    outs = []
    mask_init = False
    explicit = any(i is not None for i in inits)
    if f_from_g is None:
      f_from_g = bool(getattr(solver.initializer, "half_step_from_g", False)) and not explicit
    batch_init = getattr(solver.initializer, "batch_init", None)
    if batch_init is not None and not explicit:
      inits = list(batch_init(probs, **init_kwargs))
      mask_init = True
    for k, p in enumerate(probs):
      n, m = p.geom.shape
      init = inits[k]
      if init is None:
        fi, gi = solver.initializer(p, lse_mode=True, **init_kwargs)
        if fi is not None or gi is not None:
          mask_init = True
      else:
        fi, gi = init
      fi = None if fi is None else _arrays.as_f32(fi, dev)
      gi = None if gi is None else _arrays.as_f32(gi, dev)
      f = torch.empty(n, dtype=torch.float32, device=dev)
      g = torch.empty(m, dtype=torch.float32, device=dev)
      errors = torch.empty(max(outer, 1), dtype=torch.float32, device=dev)
      keep += [t for t in (fi, gi) if t is not None]
      q = arr[k]
      q.x = p.geom.x.data_ptr()
      q.y = p.geom.y.data_ptr()
      q.a = p.a.data_ptr()
      q.b = p.b.data_ptr()
      q.f_init = None if fi is None else fi.data_ptr()
      q.g_init = None if gi is None else gi.data_ptr()
      q.f = f.data_ptr()
      q.g = g.data_ptr()
      if live_errors:
        host = torch.full((max(outer, 1),), -1.0, dtype=torch.float32, pin_memory=True)
        self.host_errors.append(host)
        q.errors = host.data_ptr()
      else:
        q.errors = errors.data_ptr()
      q.n = n
      q.m = m
      q.epsilon = float(p.geom.epsilon)
      q.inv_scale_cost = float(p.geom.inv_scale_cost)
      sym = solver._symmetric_update if symmetric is None else bool(symmetric[k])
      if sym:
        if not _is_symmetric(p):
          raise NotImplementedError(
              "parallel updates with momentum 1/2 need a symmetric problem: the same "
              "points for x and y and the same weights for a and b")
        q.symmetric = 1
        q.b = q.a
      outs.append((f, g, errors[:outer]))
    cfg = solver._cfg(mask_init, s0)
    cfg.init_f_from_g = 1 if f_from_g else 0
    self.arr, self.cfg, self.d, self.nprob = arr, cfg, d, len(probs)
    self.keep, self.bufs = keep, outs
    self.ws_bytes = self.lib.ottb_sinkhorn_workspace_size(arr, self.nprob, d, ctypes.byref(cfg))
    if self.ws_bytes == 0:
      raise NotImplementedError("problem sizes or configuration not supported")
    self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=dev)
    self.res = torch.empty(self.nprob * _lib.RESULT_BYTES, dtype=torch.uint8, device=dev)

  def _check(self, st: int, what: str) -> None:
    if st == _lib.OTTB_ERR_UNSUPPORTED:
      raise NotImplementedError(_lib.status_string(st))
    _lib.check(st, what)

  def autotune(self, stream: int, force: bool = False) -> None:
    st = self.lib.ottb_sinkhorn_autotune(self.arr, self.nprob, self.d, ctypes.byref(self.cfg),
                                         self.res.data_ptr(), self.ws.data_ptr(),
                                         self.ws_bytes, stream, 1 if force else 0)
    self._check(st, "ottb_sinkhorn_autotune")

  def set_schedule(self, split_scale: int = 4, waves: int = 2, dynamic: int = 0,
                   tile_n: int = 256) -> None:
    st = self.lib.ottb_sinkhorn_set_schedule(self.arr, self.nprob, self.d,
                                             ctypes.byref(self.cfg), split_scale, waves,
                                             dynamic, tile_n)
    self._check(st, "ottb_sinkhorn_set_schedule")

  def solve(self, stream: int) -> None:
    st = self.lib.ottb_sinkhorn_pointcloud(self.arr, self.nprob, self.d, ctypes.byref(self.cfg),
                                           self.res.data_ptr(), self.ws.data_ptr(),
                                           self.ws_bytes, stream)
    self._check(st, "ottb_sinkhorn_pointcloud")

  def prepare(self, stream: int) -> None:
    st = self.lib.ottb_sinkhorn_prepare(self.arr, self.nprob, self.d, ctypes.byref(self.cfg),
                                        self.ws.data_ptr(), self.ws_bytes, stream)
    self._check(st, "ottb_sinkhorn_prepare")

  def launch(self, stream: int) -> None:
    st = self.lib.ottb_sinkhorn_launch(self.arr, self.nprob, self.d, ctypes.byref(self.cfg),
                                       self.res.data_ptr(), self.ws.data_ptr(),
                                       self.ws_bytes, stream)
    self._check(st, "ottb_sinkhorn_launch")

  def outputs(self) -> List[SinkhornOutput]:
    results = _Results(self.res, self.nprob)
    out = []
    for k, p in enumerate(self.probs):
      f, g, errors = self.bufs[k]
      if _tracks_grad(p):
        f, g = _Potentials.apply(p.geom.x, p.geom.y, p.a, p.b, f, g, p,
                                 self.solver.implicit_diff, self.solver.precision)
      out.append(SinkhornOutput((f, g), errors=errors, reg_ot_cost_=(results, k),
                                ot_prob=p, threshold=self.solver.threshold,
                                inner_iterations=self.solver.inner_iterations,
                                symmetric=bool(self.arr[k].symmetric),
                                use_danskin=self.solver.use_danskin,
                                precision=self.solver.precision))
    return out

  def keep_alive(self, stream: torch.cuda.Stream) -> None:
    """The workspace and initial potentials must outlive the kernels."""
    self.ws.record_stream(stream)
    for t in self.keep:
      t.record_stream(stream)


def _is_symmetric(p: linear_problem.LinearProblem) -> bool:
  """x and y the same points (one tensor), a and b equal weights."""
  x, y, a, b = p.geom.x, p.geom.y, p.a, p.b
  if x.data_ptr() != y.data_ptr() or x.shape != y.shape:
    return False
  return a.data_ptr() == b.data_ptr() or (a.shape == b.shape and bool(torch.equal(a, b)))


def run_batch(probs: Sequence[linear_problem.LinearProblem], solver: Sinkhorn,
              inits: Optional[Sequence[Optional[Tuple[Any, Any]]]] = None,
              f_from_g: Optional[bool] = None,
              symmetric: Optional[Sequence[bool]] = None,
              **init_kwargs: Any) -> List[SinkhornOutput]:
  """Solves independent problems of the same dimension in ONE persistent
  launch (the batched form of ``jax.vmap`` over ``Sinkhorn``).

  ``symmetric`` (one flag per problem; default: the solver's setting) runs
  a problem with x = y, a = b with the parallel, momentum-1/2 update.

  ``f_from_g``: start with one f-update from the initial g (its
  c-transform), for initializers that predict g. Defaults to the
  initializer's ``half_step_from_g`` when no explicit ``inits`` are given.
  An initializer with a ``batch_init(probs)`` method is called once for the
  whole batch instead of once per problem.
  """
  if not probs:
    return []
  live = solver.progress_fn is not None
  call = _Call(probs, solver, inits, f_from_g, init_kwargs, symmetric, live_errors=live)
  stream = _arrays.stream_handle()
  if solver.autotune:
    call.autotune(stream)
  call.solve(stream)
  if live:
    _live_progress(solver, call)
  out = call.outputs()
  call.keep_alive(torch.cuda.current_stream())
  return out


def set_schedule(probs: Sequence[linear_problem.LinearProblem], solver: Sinkhorn, *,
                 split_scale: int = 4, waves: int = 2, dynamic: int = 0,
                 tile_n: int = 256) -> None:
  """Pins the work schedule of calls with these problems' shapes and the
  solver's configuration (``ottb_sinkhorn_set_schedule``): the choice
  ``Sinkhorn(autotune=True)`` would otherwise time, including the
  tensor-core tile width (256 or 128 columns)."""
  if not probs:
    raise ValueError("no problems")
  _Call(probs, solver, None, None, {}, None).set_schedule(split_scale, waves, dynamic, tile_n)


class SinkhornGraph:
  """A batch of solves captured in a CUDA graph, for repeating them cheaply.

  Construction computes the initial potentials (initializer or ``inits``,
  outside the graph), writes the call header once
  (``ottb_sinkhorn_prepare``), runs the solve once, and captures the device
  half of the call (``ottb_sinkhorn_launch``: header restore, point
  preparation, initial potentials, the persistent loop, finalisation) into
  a ``torch.cuda.CUDAGraph``. ``replay()`` runs the whole solve again on
  the current contents of the problems' tensors (``x``, ``y``, ``a``, ``b``
  and the initial potentials), e.g. after copying new data into them in
  place; sizes, epsilon, the configuration and the tensors themselves are
  fixed at capture. This plays the role of calling a ``jax.jit``-compiled
  ``solve`` again. The potentials of ``replay()``'s outputs live in the
  graph's buffers and are overwritten by the next replay.
  """

  def __init__(self, probs: Sequence[linear_problem.LinearProblem],
               solver: Optional[Sinkhorn] = None,
               inits: Optional[Sequence[Optional[Tuple[Any, Any]]]] = None,
               f_from_g: Optional[bool] = None, **init_kwargs: Any):
    if not probs:
      raise ValueError("no problems")
    solver = Sinkhorn() if solver is None else solver
    self.solver = solver
    self._call = _Call(probs, solver, inits, f_from_g, init_kwargs)
    cur = torch.cuda.current_stream()
    if solver.autotune:
      self._call.autotune(cur.cuda_stream)
    self._call.prepare(cur.cuda_stream)
    self._call.launch(cur.cuda_stream)  # one solve outside the graph
    torch.cuda.synchronize()
    self.graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(cur)
    with torch.cuda.graph(self.graph, stream=side):
      self._call.launch(torch.cuda.current_stream().cuda_stream)
    cur.wait_stream(side)

  def replay(self) -> List[SinkhornOutput]:
    """Runs the captured solve on the current stream; returns its outputs."""
    self.graph.replay()
    out = self._call.outputs()
    if self.solver.progress_fn is not None:
      _replay_progress(self.solver, out)
    return out


class _LiveState(NamedTuple):
  """The solver state a live ``progress_fn`` call sees: the errors buffer so
  far (-1 where a block has not been reached, sinkhorn.py:1008-1013)."""
  errors: torch.Tensor


def _live_progress(solver: Sinkhorn, call: "_Call", poll_s: float = 2e-4) -> None:
  """Calls ``progress_fn`` while the solve runs, as the reference does from
  inside its loop (sinkhorn.py:933-937): the persistent kernel writes each
  block's error into pinned host memory as the block ends; this polls it
  until the solve's stream work completes and makes one call per new block
  of each problem, in block order, then copies the errors into the
  outputs' device buffers."""
  done = torch.cuda.Event()
  done.record()
  inner = solver.inner_iterations
  seen = [0] * len(call.host_errors)
  while True:
    finished = done.query()
    for k, host in enumerate(call.host_errors):
      errs = host.numpy()
      nb = seen[k]
      while nb < errs.shape[0] and errs[nb] != -1.0:
        nb += 1
      for blk in range(seen[k], nb):
        state = _LiveState(errors=host.clone())
        solver.progress_fn(((blk + 1) * inner - 1, inner, solver.max_iterations, state))
      seen[k] = nb
    if finished:
      break
    time.sleep(poll_s)
  for (_, _, dev_err), host in zip(call.bufs, call.host_errors):
    dev_err.copy_(host[:dev_err.shape[0]], non_blocking=True)


def _replay_progress(solver: Sinkhorn, outs: List[SinkhornOutput]) -> None:
  """Calls ``progress_fn`` once per recorded block after a replayed CUDA
  graph (``SinkhornGraph``), with the final potentials in the state; direct
  solves call it live (``_live_progress``)."""
  for o in outs:
    errs = o.errors.cpu()
    for blk in range(int((errs != -1).sum())):
      it = (blk + 1) * solver.inner_iterations - 1
      solver.progress_fn((it, solver.inner_iterations, solver.max_iterations, o))


class StackedSinkhornOutput(NamedTuple):
  """Output of ``run_stacked``: the leaves of ``jax.vmap(solve)`` over
  problems that share one geometry, stacked along axis 0.

  ``f`` [K, n], ``g`` [K, m], ``errors`` [K, outer] are device tensors;
  ``n_iters``, ``converged`` and ``reg_ot_cost`` are host arrays read from
  the device records once.
  """

  f: torch.Tensor
  g: torch.Tensor
  errors: torch.Tensor
  records: torch.Tensor  # [K * sizeof(ottb_result)] device bytes
  geom: Any
  a: torch.Tensor
  b: torch.Tensor

  def _host(self):
    import numpy as np
    raw = self.records.cpu().numpy()
    rec = np.frombuffer(raw.tobytes(), dtype=_lib.numpy_dtype(_lib.OttbResult))
    bad = rec["status"] != _lib.OTTB_OK
    if bad.any():
      raise _lib.OttbError(int(rec["status"][bad][0]), "ottb_sinkhorn_pointcloud (device)")
    return rec

  def scalars(self):
    """(n_iters, converged, reg_ot_cost) as numpy arrays, one device read."""
    rec = self._host()
    return rec["n_iters"].copy(), rec["converged"].astype(bool), rec["reg_ot_cost"].copy()

  @property
  def n_iters(self):
    return self.scalars()[0]

  @property
  def converged(self):
    return self.scalars()[1]

  @property
  def reg_ot_cost(self):
    return self.scalars()[2]


def run_stacked(geom, a: torch.Tensor, b: torch.Tensor, solver: Sinkhorn,
                init: Optional[Tuple[Optional[torch.Tensor], Optional[torch.Tensor]]] = None,
                f_from_g: Optional[bool] = None) -> StackedSinkhornOutput:
  """Solves K problems on ONE geometry with weights ``a`` [K, n] and ``b``
  [K, m] in one persistent launch: ``jax.vmap(lambda a, b:
  solve(geom, a, b))(a, b)`` of the reference, without per-problem host
  objects (the problem records are filled as arrays).

  ``init``: stacked (F, G), either may be None. Without it, an initializer
  with a ``stacked_init(a, b)`` method supplies (F, G) in one call (its
  ``half_step_from_g`` then defaults ``f_from_g``); otherwise the default
  initialisation runs on the device.
  """
  import numpy as np
  lib = _lib.load()
  dev = geom.x.device
  n, m = geom.shape
  a = _arrays.as_f32(a, dev).contiguous()
  b = _arrays.as_f32(b, dev).contiguous()
  K = a.shape[0]
  if a.shape != (K, n) or b.shape != (K, m):
    raise ValueError(f"a must be [K, {n}] and b [K, {m}]")
  mask_init = False
  if init is None:
    fn = getattr(solver.initializer, "stacked_init", None)
    if fn is not None:
      init = fn(a, b)
      mask_init = True
      if f_from_g is None:
        f_from_g = bool(getattr(solver.initializer, "half_step_from_g", False))
    elif not isinstance(solver.initializer, init_lib.DefaultInitializer):
      raise NotImplementedError("run_stacked needs an initializer with stacked_init")
  fi, gi = (None, None) if init is None else init
  fi = None if fi is None else _arrays.as_f32(fi, dev).contiguous()
  gi = None if gi is None else _arrays.as_f32(gi, dev).contiguous()
  outer = solver.outer_iterations
  f = torch.empty((K, n), dtype=torch.float32, device=dev)
  g = torch.empty((K, m), dtype=torch.float32, device=dev)
  errors = torch.empty((K, max(outer, 1)), dtype=torch.float32, device=dev)
  arr = (_lib.OttbProblem * K)()
  rec = np.frombuffer(arr, dtype=_lib.numpy_dtype(_lib.OttbProblem))
  ks = np.arange(K, dtype=np.uint64)
  rec["x"] = geom.x.data_ptr()
  rec["y"] = geom.y.data_ptr()
  rec["a"] = a.data_ptr() + ks * (4 * n)
  rec["b"] = b.data_ptr() + ks * (4 * m)
  rec["f_init"] = 0 if fi is None else fi.data_ptr() + ks * (4 * n)
  rec["g_init"] = 0 if gi is None else gi.data_ptr() + ks * (4 * m)
  rec["f"] = f.data_ptr() + ks * (4 * n)
  rec["g"] = g.data_ptr() + ks * (4 * m)
  rec["errors"] = errors.data_ptr() + ks * (4 * errors.shape[1])
  rec["n"] = n
  rec["m"] = m
  rec["epsilon"] = float(geom.epsilon)
  rec["inv_scale_cost"] = float(geom.inv_scale_cost)
  cfg = solver._cfg(mask_init or init is None, geom.epsilon_scheduler)
  cfg.init_f_from_g = 1 if f_from_g else 0
  ws_bytes = lib.ottb_sinkhorn_workspace_size(arr, K, geom.dim, ctypes.byref(cfg))
  if ws_bytes == 0:
    raise NotImplementedError("problem sizes or configuration not supported")
  ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
  res = torch.empty(K * _lib.RESULT_BYTES, dtype=torch.uint8, device=dev)
  if solver.autotune:
    st = lib.ottb_sinkhorn_autotune(arr, K, geom.dim, ctypes.byref(cfg), res.data_ptr(),
                                    ws.data_ptr(), ws_bytes, _arrays.stream_handle(), 0)
    if st == _lib.OTTB_ERR_UNSUPPORTED:
      raise NotImplementedError(_lib.status_string(st))
    _lib.check(st, "ottb_sinkhorn_autotune")
  st = lib.ottb_sinkhorn_pointcloud(arr, K, geom.dim, ctypes.byref(cfg), res.data_ptr(),
                                    ws.data_ptr(), ws_bytes, _arrays.stream_handle())
  if st == _lib.OTTB_ERR_UNSUPPORTED:
    raise NotImplementedError(_lib.status_string(st))
  _lib.check(st, "ottb_sinkhorn_pointcloud")
  cur = torch.cuda.current_stream()
  for t in (ws, a, b) + tuple(t for t in (fi, gi) if t is not None):
    t.record_stream(cur)
  return StackedSinkhornOutput(f, g, errors[:, :outer], res, geom, a, b)
