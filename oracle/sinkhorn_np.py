"""CPU oracle: NumPy restatement of ott-jax's log-domain Sinkhorn on PointClouds.

TEST INFRASTRUCTURE ONLY. Nothing in the ``ott_b200`` package imports this
module; it is used by ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` as the checker, never as the thing measured or
shipped.

Every function restates, in plain NumPy, the reference function it names
(paths are relative to the ott-jax source tree, ``src/ott/...``).  The op
order of the reference is kept (centre ``f + g - C``, divide by epsilon,
max-shifted logsumexp, multiply by epsilon, subtract the finite potential) so
that the float32 mode reproduces the reference's FP32 rounding behaviour as
closely as a different backend can, and the float64 mode is the accuracy
reference (the reference run with ``jax_enable_x64``).

The arithmetic core of the reference lives in a third-party dependency that is
absent here: ``jax.scipy.special.logsumexp`` (jax, unpinned ``jax>=0.4.0`` in
``pyproject.toml``).  Its published algorithm is restated in
:func:`logsumexp`.  The oracle is pinned against the reference's own Python
executed over a NumPy stand-in for ``jax`` (``oracle/jaxshim``); the golden
fixtures it produced live in ``tests/golden``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

import numpy as np

DEFAULT_EPSILON_SCALE = 0.05  # geometry/epsilon_scheduler.py:22


# ---------------------------------------------------------------------------
# math/utils.py:132-136 -> jax.scipy.special.logsumexp (restated)
# ---------------------------------------------------------------------------
def logsumexp(mat: np.ndarray, axis: Optional[int] = None, b=None,
              return_sign: bool = False):
  """Max-shifted log-sum-exp, as jax.scipy.special.logsumexp computes it.

  Published algorithm: weights ``b == 0`` mask the entry to ``-inf``; the
  shift is the max over the reduced axis, replaced by 0 when it is not finite;
  ``out = log(|sum(b * exp(a - shift))|) + shift``; with ``b`` given and no
  sign requested, a negative sum yields NaN.
  """
  a = np.asarray(mat)
  if b is not None:
    b = np.asarray(b, dtype=a.dtype)
    a, b = np.broadcast_arrays(a, b)
    a = np.where(b != 0, a, -np.inf).astype(a.dtype)
  with np.errstate(invalid="ignore", over="ignore"):
    amax = np.max(a, axis=axis, keepdims=True, initial=-np.inf)
    amax = np.where(np.isfinite(amax), amax, 0).astype(a.dtype)
    exp_a = np.exp(a - amax)
    if b is not None:
      exp_a = exp_a * b
    sumexp = np.sum(exp_a, axis=axis, keepdims=True)
    sign = np.sign(sumexp)
    with np.errstate(divide="ignore"):
      out = np.log(np.abs(sumexp)) + amax
  if axis is not None:
    out = np.squeeze(out, axis=axis)
    sign = np.squeeze(sign, axis=axis)
  else:
    out = out.reshape(())
    sign = sign.reshape(())
  if return_sign:
    return out, sign
  if b is not None:
    out = np.where(sign < 0, np.nan, out)
  return out


# ---------------------------------------------------------------------------
# geometry/costs.py:548-573 (SqEuclidean) and costs.py:82-92 (all_pairs)
# ---------------------------------------------------------------------------
def sq_norm(x: np.ndarray) -> np.ndarray:
  """costs.py:554-556: ``sum(x ** 2, axis=-1)``."""
  return np.sum(x * x, axis=-1)


def sqeuclidean_all_pairs(x: np.ndarray, y: np.ndarray) -> np.ndarray:
  """costs.py:558-561 applied to all pairs: ``|x|^2 + |y|^2 + (-2 <x, y>)``."""
  cross = -2.0 * (x @ y.T)
  return (sq_norm(x)[:, None] + sq_norm(y)[None, :]) + cross.astype(x.dtype)


# ---------------------------------------------------------------------------
# Geometry: epsilon and cost statistics
# ---------------------------------------------------------------------------
def mean_cost_matrix(x, y, inv_scale_cost=1.0) -> float:
  """geometry.py:113-117 through pointcloud.py:170-186 (sqeucl closed form).

  ``tmp = |x|^2 . vec + |y|^2 * sum(vec) - 2 y (x^T vec)`` with
  ``vec = 1/n``, then ``sum(tmp / m)``; uniform weights by construction.
  """
  n, m = x.shape[0], y.shape[0]
  vec = np.full((n,), 1.0 / n, dtype=x.dtype)
  nx, ny = sq_norm(x), sq_norm(y)
  applied = np.dot(nx, vec) + ny * np.sum(vec)
  applied = applied - 2.0 * (y @ (x.T @ vec))
  applied = inv_scale_cost * applied
  return np.sum((1.0 / m) * applied)


def std_cost_matrix(x, y, inv_scale_cost=1.0) -> float:
  """geometry.py:120-135: ``sqrt(relu(mean(C^2) - mean(C)^2))``."""
  n, m = x.shape[0], y.shape[0]
  c = inv_scale_cost * sqeuclidean_all_pairs(x, y)
  vec = np.full((n,), 1.0 / n, dtype=x.dtype)
  tmp = (c * c).T @ vec
  tmp = np.sum((1.0 / m) * tmp) - mean_cost_matrix(x, y, inv_scale_cost) ** 2
  return np.sqrt(max(tmp, 0.0))


def inv_scale_cost(x, y, scale_cost) -> float:
  """pointcloud.py:343-383 for the scalings that do not need the full cost."""
  if isinstance(scale_cost, (int, float)):
    return 1.0 / scale_cost
  if scale_cost == "mean":
    return 1.0 / np.mean(sqeuclidean_all_pairs(x, y))
  if scale_cost == "max_cost":
    return 1.0 / np.max(sqeuclidean_all_pairs(x, y))
  if scale_cost == "median":
    return 1.0 / np.median(sqeuclidean_all_pairs(x, y))
  nx, ny = sq_norm(x), sq_norm(y)
  if scale_cost == "max_norm":
    return 1.0 / max(nx.max(), ny.max())
  if scale_cost == "max_bound":
    xm, ym = nx.max(), ny.max()
    return 1.0 / (xm + ym + 2 * np.sqrt(xm * ym))
  raise ValueError(f"Scaling {scale_cost} not implemented.")


def resolve_epsilon(x, y, epsilon=None, relative_epsilon=None,
                    inv_scale=1.0) -> float:
  """geometry.py:148-176: target epsilon of the scheduler."""
  if relative_epsilon is None:
    if epsilon is not None:
      return epsilon
    return DEFAULT_EPSILON_SCALE * std_cost_matrix(x, y, inv_scale)
  if relative_epsilon == "std":
    scale = std_cost_matrix(x, y, inv_scale)
  elif relative_epsilon == "mean":
    scale = mean_cost_matrix(x, y, inv_scale)
  else:
    raise ValueError(f"Invalid relative epsilon: {relative_epsilon}.")
  mult = DEFAULT_EPSILON_SCALE if epsilon is None else epsilon
  return mult * scale


def epsilon_at(target, it, init=1.0, decay=1.0):
  """epsilon_scheduler.py:47-60: ``max(init * decay**it, 1) * target``."""
  if it is None:
    return target
  return max(init * (decay ** it), 1.0) * target


# ---------------------------------------------------------------------------
# Dense (or row/column-blocked) geometry with the lse kernel
# ---------------------------------------------------------------------------
@dataclass
class Geom:
  """A point-cloud geometry with squared-Euclidean cost.

  ``batch_size`` follows pointcloud.py:438-448: ``None`` materialises the
  cost (geometry.py:260-299); an integer recomputes it in blocks
  (pointcloud.py:85-103), which is what lets the oracle run large inputs.
  ``workers`` > 1 evaluates the blocks on that many threads, BLAS limited to
  one thread per block. Each block is computed as in the serial loop and
  writes its own output slice, so the results are bit-identical to a serial
  run with one BLAS thread (a multi-threaded BLAS blocks its products
  differently, a rounding-level difference).
  """
  x: np.ndarray
  y: np.ndarray
  epsilon: float
  inv_scale: float = 1.0
  eps_init: float = 1.0
  eps_decay: float = 1.0
  batch_size: Optional[int] = None
  workers: int = 1
  _cost: Optional[np.ndarray] = field(default=None, repr=False)

  def _for_blocks(self, total, bs, fn):
    starts = range(0, total, bs)
    if self.workers <= 1 or self.batch_size is None or total <= bs:
      for s in starts:
        fn(s)
      return
    from concurrent.futures import ThreadPoolExecutor

    import threadpoolctl
    with threadpoolctl.threadpool_limits(1), \
        ThreadPoolExecutor(max_workers=self.workers) as ex:
      list(ex.map(fn, starts))

  @property
  def dtype(self):
    return self.x.dtype

  @property
  def shape(self):
    return self.x.shape[0], self.y.shape[0]

  def cost_block(self, rows=slice(None), cols=slice(None)):
    if self.batch_size is None:
      if self._cost is None:
        self._cost = (self.inv_scale * sqeuclidean_all_pairs(self.x, self.y)
                      ).astype(self.dtype)
      return self._cost[rows, cols]
    c = sqeuclidean_all_pairs(self.x[rows], self.y[cols])
    return (self.inv_scale * c).astype(self.dtype)

  def eps_at(self, it):
    return self.dtype.type(
        epsilon_at(self.epsilon, it, self.eps_init, self.eps_decay))

  def apply_lse_kernel(self, f, g, eps, axis, vec=None):
    """geometry.py:260-299 + _softmax :426-442 + _center :423-424.

    Returns ``eps * lse((f + g - C) / eps) - finite(f or g)`` and the sign.
    """
    dt = self.dtype
    eps = dt.type(eps)
    n, m = self.shape
    bs = self.batch_size or (m if axis == 0 else n)
    if axis == 0:
      out = np.empty((m,), dt)
      sgn = np.ones((m,), dt)

      def block(s):
        cols = slice(s, min(s + bs, m))
        center = (f[:, None] + g[None, cols]) - self.cost_block(cols=cols)
        r, sg = logsumexp(center / eps, axis=0,
                          b=None if vec is None else vec[:, None],
                          return_sign=True)
        out[cols] = eps * r
        sgn[cols] = sg
      self._for_blocks(m, bs, block)
      remove = g
    else:
      out = np.empty((n,), dt)
      sgn = np.ones((n,), dt)

      def block(s):
        rows = slice(s, min(s + bs, n))
        center = (f[rows, None] + g[None, :]) - self.cost_block(rows=rows)
        r, sg = logsumexp(center / eps, axis=1,
                          b=None if vec is None else vec[None, :],
                          return_sign=True)
        out[rows] = eps * r
        sgn[rows] = sg
      self._for_blocks(n, bs, block)
      remove = f
    with np.errstate(invalid="ignore"):
      res = out - np.where(np.isfinite(remove), remove, 0).astype(dt)
    return res.astype(dt), sgn

  def update_potential(self, f, g, log_marginal, iteration, axis):
    """geometry.py:376-398."""
    eps = self.eps_at(iteration)
    app = self.apply_lse_kernel(f, g, eps, axis)[0]
    with np.errstate(invalid="ignore"):
      return (eps * log_marginal
              - np.where(np.isfinite(app), app, 0)).astype(self.dtype)

  def marginal_from_potentials(self, f, g, axis=0):
    """geometry.py:326-349 (uses the target epsilon)."""
    eps = self.dtype.type(self.epsilon)
    h = f if axis == 1 else g
    z = self.apply_lse_kernel(f, g, eps, axis)[0]
    with np.errstate(over="ignore", invalid="ignore"):
      return np.exp((z + h) / eps).astype(self.dtype)

  def apply_transport_from_potentials(self, f, g, vec, axis=0):
    """geometry.py:444-486: signed-weight lse applied to ``vec``."""
    eps = self.dtype.type(self.epsilon)
    res, sgn = self.apply_lse_kernel(f, g, eps, axis, vec=vec)
    res = res + (f if axis == 1 else g)
    with np.errstate(over="ignore", invalid="ignore"):
      return (sgn * np.exp(res / eps)).astype(self.dtype)


# ---------------------------------------------------------------------------
# solvers/linear/sinkhorn.py
# ---------------------------------------------------------------------------
def marginal_error(f, g, target, geom: Geom, axis=0, norm_error=1):
  """sinkhorn.py:191-221 (lse mode)."""
  marginal = geom.marginal_from_potentials(f, g, axis=axis)
  with np.errstate(invalid="ignore", over="ignore"):
    return np.sum(np.abs(marginal - target) ** norm_error) ** (1.0 / norm_error)


def compute_kl_reg_cost(f, g, a, b, geom: Geom):
  """sinkhorn.py:224-277, balanced branch (tau_a == tau_b == 1)."""
  dt = geom.dtype
  with np.errstate(divide="ignore", invalid="ignore"):
    fa = geom.dtype.type(geom.epsilon) * np.log(a)
    div_a = np.sum(np.where(a > 0, a * (f - fa), 0.0).astype(dt))
    gb = geom.dtype.type(geom.epsilon) * np.log(b)
    div_b = np.sum(np.where(b > 0, b * (g - gb), 0.0).astype(dt))
  total_sum = np.sum(geom.marginal_from_potentials(f, g))
  return dt.type(div_a + div_b + geom.dtype.type(geom.epsilon)
                 * (np.sum(a) * np.sum(b) - total_sum))


def entr(p):
  """jax.scipy.special.entr: ``-p log p`` (0 at 0, -inf below)."""
  with np.errstate(divide="ignore", invalid="ignore"):
    return np.where(p > 0, -p * np.log(np.where(p > 0, p, 1)),
                    np.where(p == 0, 0.0, -np.inf))


@dataclass
class SinkhornResult:
  f: np.ndarray
  g: np.ndarray
  errors: np.ndarray
  reg_ot_cost: float
  converged: bool
  inner_iterations: int
  threshold: float
  a: np.ndarray
  b: np.ndarray
  epsilon: float

  @property
  def n_iters(self) -> int:
    """sinkhorn.py:432-434."""
    return int(np.sum(self.errors != -1) * self.inner_iterations)

  @property
  def dual_cost(self):
    """sinkhorn.py:337-343."""
    return (np.sum(np.where(self.a > 0, self.a * self.f, 0))
            + np.sum(np.where(self.b > 0, self.b * self.g, 0)))

  @property
  def ent_reg_cost(self):
    """sinkhorn.py:351-370."""
    return self.reg_ot_cost - self.epsilon * (np.sum(entr(self.a))
                                              + np.sum(entr(self.b)))


def default_init(a, b, dtype):
  """initializers.py:70-131: zeros, ``-inf`` where the weight is 0."""
  f = np.where(a > 0, 0.0, -np.inf).astype(dtype)
  g = np.where(b > 0, 0.0, -np.inf).astype(dtype)
  return f, g


def sinkhorn(geom: Geom, a=None, b=None, *, threshold=1e-3, norm_error=1,
             inner_iterations=10, min_iterations=0, max_iterations=2000,
             init: Optional[Tuple[np.ndarray, np.ndarray]] = None,
             progress=None, parallel_dual_updates=False,
             momentum=1.0) -> SinkhornResult:
  """sinkhorn.py:782-801 (__call__), :1052-1099 (run/iterations).

  Loop: math/fixed_point_loop.py:23-93.  One iteration: sinkhorn.py:879-938
  (lse_step :803-857) with a constant ``Momentum(start=0, value=momentum)``
  (acceleration.py:140-142, 164-172; default weight 1) and sequential or
  parallel updates (``parallel_dual_updates``, :836-855). With parallel
  updates the error is that of both marginals (solution_error, :127-188).
  """
  dt = geom.dtype
  n, m = geom.shape
  a = np.full((n,), 1.0 / n, dt) if a is None else np.asarray(a, dt)
  b = np.full((m,), 1.0 / m, dt) if b is None else np.asarray(b, dt)
  if init is None:
    f, g = default_init(a, b, dt)
  else:
    f, g = (np.asarray(init[0], dt).copy(), np.asarray(init[1], dt).copy())
  with np.errstate(divide="ignore"):
    log_a, log_b = np.log(a), np.log(b)
  outer = int(math.ceil(max_iterations / inner_iterations))
  errors = -np.ones((outer,), dt)

  w = dt.type(momentum)

  def momentum_step(old, new):
    # acceleration.py:168-170
    with np.errstate(invalid="ignore"):
      old = np.where(np.isfinite(old), old, 0.0).astype(dt)
      return ((dt.type(1.0) - w) * old + w * new).astype(dt)

  def one_iteration(f, g, it, compute_error):
    old_g = g
    new_g = geom.update_potential(f, g, log_b, it, axis=0)
    g = momentum_step(g, new_g)
    new_f = geom.update_potential(f, old_g if parallel_dual_updates else g, log_a, it,
                                  axis=1)
    f = momentum_step(f, new_f)
    if it == max_iterations - 1 or (compute_error and it >= min_iterations):
      err = marginal_error(f, g, b, geom, 0, norm_error)
      if parallel_dual_updates:
        err = err + marginal_error(f, g, a, geom, 1, norm_error)
    else:
      err = np.inf
    errors[it // inner_iterations] = err
    if progress is not None:
      progress(it, f, g, errors)
    return f, g

  def cond(it):
    # sinkhorn.py:940-953
    err = errors[it // inner_iterations - 1]
    converged = it > 0 and err < threshold
    diverged = not np.isfinite(err)
    return (not diverged) and (not converged)

  it = 0
  force_scan = min_iterations == max_iterations
  if force_scan:
    for _ in range(max_iterations // inner_iterations):
      for k in range(inner_iterations):
        f, g = one_iteration(f, g, it, k == inner_iterations - 1)
        it += 1
  else:
    while it < max_iterations and (it < min_iterations or cond(it)):
      for k in range(inner_iterations):
        f, g = one_iteration(f, g, it, k == inner_iterations - 1)
        it += 1
  # sinkhorn.py:1020-1023
  converged = bool((not np.any(np.isnan(errors))) and errors[-1] < threshold)
  cost = compute_kl_reg_cost(f, g, a, b, geom)
  return SinkhornResult(f=f, g=g, errors=errors, reg_ot_cost=cost,
                        converged=converged, inner_iterations=inner_iterations,
                        threshold=threshold, a=a, b=b, epsilon=geom.epsilon)


def solve(x, y=None, a=None, b=None, *, epsilon=None, relative_epsilon=None,
          scale_cost=1.0, batch_size=None, eps_init=1.0, eps_decay=1.0,
          dtype=np.float64, workers=1, **kw) -> SinkhornResult:
  """_solve.py:29-64 on ``PointCloud(x, y, epsilon, relative_epsilon)``."""
  x = np.asarray(x, dtype)
  y = x if y is None else np.asarray(y, dtype)
  inv = inv_scale_cost(x, y, scale_cost)
  eps = resolve_epsilon(x, y, epsilon, relative_epsilon, inv)
  geom = Geom(x, y, float(eps), inv_scale=float(inv), eps_init=eps_init,
              eps_decay=eps_decay, batch_size=batch_size, workers=workers)
  return sinkhorn(geom, a, b, **kw)


def sinkhorn_divergence(x, y, a=None, b=None, *, epsilon=None, relative_epsilon=None,
                       scale_cost=1.0, symmetric_sinkhorn=True, dtype=np.float64, **kw):
  """tools/sinkhorn_divergence.py:178-352 on PointClouds: three solves with
  the (x, y) epsilon shared (share_epsilon, :231-235), the x/x and y/y
  terms with parallel updates and momentum 1/2 (:318-336) when
  ``symmetric_sinkhorn``. Returns (divergence, (r_xy, r_xx, r_yy))."""
  x = np.asarray(x, dtype)
  y = np.asarray(y, dtype)
  n, m = x.shape[0], y.shape[0]
  a = np.full((n,), 1.0 / n, dtype) if a is None else np.asarray(a, dtype)
  b = np.full((m,), 1.0 / m, dtype) if b is None else np.asarray(b, dtype)
  inv = inv_scale_cost(x, y, scale_cost)
  eps = resolve_epsilon(x, y, epsilon, relative_epsilon, inv)
  sym = dict(parallel_dual_updates=True, momentum=0.5) if symmetric_sinkhorn else {}
  res = []
  for (u, v, wu, wv, extra) in ((x, y, a, b, {}), (x, x, a, a, sym), (y, y, b, b, sym)):
    iv = inv_scale_cost(u, v, scale_cost)
    res.append(sinkhorn(Geom(u, v, float(eps), inv_scale=float(iv)), wu, wv, **kw, **extra))
  div = (res[0].reg_ot_cost - 0.5 * (res[1].reg_ot_cost + res[2].reg_ot_cost)
         + 0.5 * eps * (np.sum(a) - np.sum(b)) ** 2)
  return div, tuple(res)


def segment_point_cloud(x, a=None, num_segments=None, max_measure_size=None,
                        segment_ids=None, num_per_segment=None):
  """geometry/segment.py:23-131: segments padded to ``max_measure_size``
  with zero points of weight 0; default weights 1 / (segment size)."""
  num, dim = x.shape
  if segment_ids is not None:
    counts = np.bincount(segment_ids, minlength=num_segments)
  else:
    counts = np.asarray(num_per_segment)
    if max_measure_size is None:
      max_measure_size = int(counts.max())
    num_segments = len(counts)
    segment_ids = np.repeat(np.arange(num_segments), counts)
  size = min(int(max_measure_size), num)
  if a is None:
    a = (1.0 / counts)[segment_ids]
  xs = np.zeros((num_segments, size, dim), x.dtype)
  ws = np.zeros((num_segments, size), x.dtype)
  for s in range(num_segments):
    idx = np.flatnonzero(segment_ids == s)[:size]
    xs[s, :len(idx)] = x[idx]
    ws[s, :len(idx)] = a[idx]
  return xs, ws


def segment_sinkhorn(x, y, num_segments=None, max_measure_size=None, segment_ids_x=None,
                     segment_ids_y=None, num_per_segment_x=None, num_per_segment_y=None,
                     weights_x=None, weights_y=None, sinkhorn_kwargs=None,
                     dtype=np.float64, **geom_kw):
  """tools/segment_sinkhorn.py:24-138: one padded solve per segment."""
  x, y = np.asarray(x, dtype), np.asarray(y, dtype)
  sx, wx = segment_point_cloud(x, None if weights_x is None else np.asarray(weights_x, dtype),
                               num_segments, max_measure_size, segment_ids_x, num_per_segment_x)
  sy, wy = segment_point_cloud(y, None if weights_y is None else np.asarray(weights_y, dtype),
                               num_segments, max_measure_size, segment_ids_y, num_per_segment_y)
  kw = dict(sinkhorn_kwargs or {})
  return np.array([solve(sx[s], sy[s], wx[s], wy[s], dtype=dtype, **geom_kw, **kw).reg_ot_cost
                   for s in range(sx.shape[0])])


# ---------------------------------------------------------------------------
# Gradient of reg_ot_cost with the potentials held fixed
# (sinkhorn.py:329-335 set_cost with use_danskin=True, :779-780 default)
# ---------------------------------------------------------------------------
def transport_matrix(f, g, geom: Geom):
  """geometry.py:361-365: ``exp((f + g - C) / eps)``, dense."""
  with np.errstate(invalid="ignore", over="ignore"):
    center = (f[:, None] + g[None, :]) - geom.cost_block()
    return np.exp(center / geom.epsilon)


def reg_ot_cost_grads(f, g, a, b, geom: Geom, scale_cost_mean=False):
  """d compute_kl_reg_cost(f, g, a, b) / d(x, y, a, b) at fixed f, g.

  ``compute_kl_reg_cost`` (sinkhorn.py:224-277) depends on the points only
  through ``sum(P)`` with ``P_ij = exp((f_i + g_j - inv C_ij) / eps)``
  (epsilon carries no gradient: geometry.py:157-163), and on the weights
  through the explicit ``a (f - eps log a)``, ``b (g - eps log b)`` and
  ``eps sum(a) sum(b)`` terms. With ``scale_cost="mean"`` the scale
  ``inv = 1 / mean(C_unscaled)`` (pointcloud.py:348-351) also depends on
  the points. Zero weights get 0 from their ``where`` term.
  """
  x, y = geom.x.astype(np.float64), geom.y.astype(np.float64)
  n, m = x.shape[0], y.shape[0]
  inv, eps = geom.inv_scale, geom.epsilon
  P = transport_matrix(f.astype(np.float64), g.astype(np.float64), geom).astype(np.float64)
  r, c = P.sum(1), P.sum(0)
  gx = 2 * inv * (r[:, None] * x - P @ y)
  gy = 2 * inv * (c[:, None] * y - P.T @ x)
  if scale_cost_mean:
    cu = sqeuclidean_all_pairs(x, y)
    t = np.sum(P * cu)
    gx = gx - inv * inv * (2.0 / n) * (x - y.mean(0)) * t
    gy = gy - inv * inv * (2.0 / m) * (y - x.mean(0)) * t
  a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
  with np.errstate(divide="ignore", invalid="ignore"):
    ga = np.where(a > 0, f - eps * np.log(a) - eps, 0.0) + eps * b.sum()
    gb = np.where(b > 0, g - eps * np.log(b) - eps, 0.0) + eps * a.sum()
  return gx, gy, ga, gb


# ---------------------------------------------------------------------------
# Implicit differentiation of the potentials
# (solvers/linear/implicit_differentiation.py, default ImplicitDiff():
# precondition h = eps log, balanced problem, lineax NormalCG)
# ---------------------------------------------------------------------------
def first_order_conditions(f, g, a, b, geom: Geom):
  """implicit_differentiation.py:235-273 (tau = 1: grad_of_marginal_fit is
  the weight itself, unbalanced_functions.py:30-50):
  ``[a > 0](eps log(P 1) - eps log a)`` and ``[b > 0](eps log(P^T 1) -
  eps log b)``."""
  eps = geom.epsilon
  P = transport_matrix(f, g, geom)
  ma, mb = P.sum(1), P.sum(0)
  with np.errstate(divide="ignore", invalid="ignore"):
    ra = np.where(a > 0, eps * np.log(ma) - eps * np.log(a), 0.0)
    rb = np.where(b > 0, eps * np.log(mb) - eps * np.log(b), 0.0)
  return np.concatenate([ra, rb])


def _lstsq_min_norm(mat, rhs):
  """The least-squares solution of least norm: the limit of CG on the
  normal equations started from zero (lineax NormalCG,
  lineax_implicit.py:49-101), which ImplicitDiff uses by default."""
  return np.linalg.lstsq(mat, rhs, rcond=None)[0]


def implicit_solve(gr_f, gr_g, f, g, a, b, geom: Geom):
  """implicit_differentiation.py:80-233 with ``h = eps log``, dense.

  ``-(J^-1)^T gr`` for the Jacobian J of the first-order conditions in
  (f, g): the Schur complement of the larger side's diagonal block is
  solved (size m if n > m, else n). Points of zero weight are left out of
  the system and get 0 (the reference's ``eps / 0`` makes them NaN).
  """
  n, m = geom.shape
  eps = geom.epsilon
  sa, sb = np.asarray(a) > 0, np.asarray(b) > 0
  P = transport_matrix(f, g, geom)[np.ix_(sa, sb)]
  gf, gg = np.asarray(gr_f, np.float64)[sa], np.asarray(gr_g, np.float64)[sb]
  ma, mb = P.sum(1), P.sum(0)
  hp = lambda v: eps / v  # derivative of eps * log
  vjp_fg = lambda z: P @ (z * hp(mb)) / eps
  vjp_gf = lambda z: P.T @ (z * hp(ma)) / eps
  diag_a = ma * hp(ma) / eps
  diag_b = mb * hp(mb) / eps
  if n > m:
    schur = np.diag(diag_b) - P.T @ np.diag(hp(ma) / eps / diag_a) @ P @ np.diag(hp(mb) / eps)
    res = gg - vjp_gf(gf / diag_a)
    sch = _lstsq_min_norm(schur, res)
    lf, lg = (gf - vjp_fg(sch)) / diag_a, sch
  else:
    schur = np.diag(diag_a) - P @ np.diag(hp(mb) / eps / diag_b) @ P.T @ np.diag(hp(ma) / eps)
    res = gf - vjp_fg(gg / diag_b)
    sch = _lstsq_min_norm(schur, res)
    lf, lg = sch, (gg - vjp_gf(sch)) / diag_b
  out_f, out_g = np.zeros(n), np.zeros(m)
  out_f[sa], out_g[sb] = -lf, -lg
  return np.concatenate([out_f, out_g])


def implicit_pullback(lam, f, g, a, b, geom: Geom, scale_cost_mean=False):
  """``lam^T d(first_order_conditions)/d(x, y, a, b)`` at fixed f, g
  (implicit_differentiation.py:275-287, the ``jax.vjp`` there), closed
  form: with ``ma = P 1``, ``mb = P^T 1`` and the plan's
  ``dP_ij / dC_ij = -P_ij / eps``, the cost cotangent is
  ``G_ij = -P_ij (lam_a,i [a_i>0] / ma_i + lam_b,j [b_j>0] / mb_j)``;
  ``C = inv C_unscaled`` carries it to the points (and to ``inv`` for
  ``scale_cost="mean"``, pointcloud.py:348-351); ``d/da_i = -eps lam_a,i /
  a_i`` on ``a > 0``. Epsilon is a constant (geometry.py:157-163)."""
  n, m = geom.shape
  eps, inv = geom.epsilon, geom.inv_scale
  x, y = geom.x.astype(np.float64), geom.y.astype(np.float64)
  a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
  la, lb = np.asarray(lam[:n], np.float64), np.asarray(lam[n:], np.float64)
  P = transport_matrix(f, g, geom).astype(np.float64)
  ma, mb = P.sum(1), P.sum(0)
  with np.errstate(divide="ignore", invalid="ignore"):
    ua = np.where(a > 0, la / ma, 0.0)
    vb = np.where(b > 0, lb / mb, 0.0)
    ga = np.where(a > 0, -eps * la / a, 0.0)
    gb = np.where(b > 0, -eps * lb / b, 0.0)
  G = -P * (ua[:, None] + vb[None, :])
  gx = 2 * inv * (G.sum(1)[:, None] * x - G @ y)
  gy = 2 * inv * (G.sum(0)[:, None] * y - G.T @ x)
  if scale_cost_mean:
    t = np.sum(G * sqeuclidean_all_pairs(x, y))
    gx = gx - inv * inv * (2.0 / n) * (x - y.mean(0)) * t
    gy = gy - inv * inv * (2.0 / m) * (y - x.mean(0)) * t
  return gx, gy, ga, gb


def implicit_grads(gr_f, gr_g, f, g, a, b, geom: Geom, scale_cost_mean=False):
  """Gradient w.r.t. (x, y, a, b) of ``<gr_f, f*> + <gr_g, g*>`` through
  the optimal potentials (sinkhorn.py:1112-1136: the custom VJP of the
  Sinkhorn loop)."""
  lam = implicit_solve(gr_f, gr_g, f, g, a, b, geom)
  return implicit_pullback(lam, f, g, a, b, geom, scale_cost_mean)


# ---------------------------------------------------------------------------
# Learned initializer objective (initializers/neural/meta_initializer.py)
# ---------------------------------------------------------------------------
def meta_dual_loss(f_pred, a, b, geom: Geom):
  """meta_initializer.py:163-175: ``-compute_kl_reg_cost(f, g(f))``.

  ``g(f) = update_potential(f, 0, log b, 0, axis=0)`` with non-finite entries
  replaced by 0.  Returns ``(loss, dloss/df)``; the gradient follows from
  ``g(f)`` being the exact maximiser of the dual in ``g`` (envelope theorem):
  ``d(-J)/df = -(a - rowmarginal(f, g(f)))`` on the support of ``a``.
  """
  dt = geom.dtype
  with np.errstate(divide="ignore"):
    log_b = np.log(b)
  g = geom.update_potential(f_pred, np.zeros_like(b), log_b, 0, axis=0)
  g = np.where(np.isfinite(g), g, 0.0).astype(dt)
  loss = -compute_kl_reg_cost(f_pred, g, a, b, geom)
  row_marg = geom.marginal_from_potentials(f_pred, g, axis=1)
  grad = -(np.where(a > 0, a, 0.0) - row_marg)
  return loss, grad
