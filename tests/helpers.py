"""Runs the CUDA path and the oracle on the same inputs and compares."""
from __future__ import annotations

import numpy as np

from oracle import sinkhorn_np as oracle


def gpu_solve(x, y, a, b, **kw):
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  geom_kw = {k: kw.pop(k) for k in ("epsilon", "relative_epsilon", "scale_cost")
             if k in kw}
  geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(),
                               None if y is None else torch.as_tensor(y).cuda(), **geom_kw)
  out = linear.solve(geom, None if a is None else torch.as_tensor(a).cuda(),
                     None if b is None else torch.as_tensor(b).cuda(), **kw)
  return geom, out


def oracle_solve(x, y, a, b, dtype=np.float64, **kw):
  """The oracle's solve, carrying ``rerun(n)``: the same problem run for
  exactly n iterations (threshold 0, ``max_iterations = n``), which logs the
  error at every block end as the stopping run does."""
  ref = oracle.solve(x, y, a, b, dtype=dtype, **kw)

  def rerun(n_iters):
    return oracle.solve(x, y, a, b, dtype=dtype,
                        **dict(kw, threshold=0.0, max_iterations=n_iters))
  ref.rerun = rerun
  return ref


def oracle_sinkhorn(geom, a, b, **kw):
  """``oracle.sinkhorn`` on a prepared geometry, carrying ``rerun(n)``."""
  ref = oracle.sinkhorn(geom, a, b, **kw)

  def rerun(n_iters):
    return oracle.sinkhorn(geom, a, b, **dict(kw, threshold=0.0, max_iterations=n_iters))
  ref.rerun = rerun
  return ref


def state_at(out_iters, ref):
  """The oracle's state after ``out_iters`` iterations: ``ref`` itself when
  the counts agree, else ``ref.rerun(out_iters)``."""
  if out_iters == ref.n_iters:
    return ref
  rerun = getattr(ref, "rerun", None)
  assert rerun is not None, ("iteration counts differ and the oracle result cannot be "
                             f"re-run at the GPU's count ({out_iters} vs {ref.n_iters})")
  return rerun(out_iters)


def assert_potentials(f, g, at, pot_tol):
  """f, g (float64 arrays) against the oracle state ``at``: same -inf
  pattern, finite entries within pot_tol * epsilon absolute."""
  eps = at.epsilon
  ff, gf = np.isfinite(at.f), np.isfinite(at.g)
  np.testing.assert_array_equal(np.isfinite(f), ff)
  np.testing.assert_array_equal(np.isfinite(g), gf)
  np.testing.assert_allclose(f[ff], at.f[ff], rtol=0, atol=pot_tol * eps)
  np.testing.assert_allclose(g[gf], at.g[gf], rtol=0, atol=pot_tol * eps)


def assert_parity(geom, out, ref, *, pot_tol=1e-4, cost_rtol=1e-5, iter_blocks=1,
                  err_rtol=1e-2, err_atol=1e-6):
  """n_iters within iter_blocks blocks and the same ``converged``;
  reg_ot_cost within cost_rtol relative of the oracle's converged solve; f
  and g within pot_tol * eps of the oracle's state after the GPU's own
  iteration count (re-run for exactly that many iterations when the counts
  differ), and the error log's pattern and values (err_rtol, err_atol)
  against that state."""
  assert abs(out.n_iters - ref.n_iters) <= iter_blocks * out.inner_iterations, \
      (out.n_iters, ref.n_iters)
  assert out.converged == ref.converged
  np.testing.assert_allclose(out.reg_ot_cost, ref.reg_ot_cost, rtol=cost_rtol,
                             atol=cost_rtol * 1e-3)
  at = state_at(out.n_iters, ref)
  f = out.f.cpu().numpy().astype(np.float64)
  g = out.g.cpu().numpy().astype(np.float64)
  assert_potentials(f, g, at, pot_tol)
  errs = out.errors.cpu().numpy()
  if at is ref:
    np.testing.assert_array_equal(errs == -1, ref.errors == -1)
    np.testing.assert_array_equal(np.isinf(errs), np.isinf(ref.errors))
  k = out.n_iters // out.inner_iterations
  mine, theirs = errs[:k], at.errors[:k]
  np.testing.assert_array_equal(np.isinf(mine), np.isinf(theirs))
  fin = np.isfinite(theirs) & (theirs != -1)
  np.testing.assert_allclose(mine[fin], theirs[fin], rtol=err_rtol, atol=err_atol)
