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
  return oracle.solve(x, y, a, b, dtype=dtype, **kw)


def assert_parity(geom, out, ref, *, pot_tol=1e-4, cost_rtol=1e-5, iter_blocks=1):
  """f, g within pot_tol * eps absolute, reg_ot_cost within cost_rtol
  relative, n_iters within iter_blocks blocks."""
  eps = ref.epsilon
  assert abs(out.n_iters - ref.n_iters) <= iter_blocks * out.inner_iterations, \
      (out.n_iters, ref.n_iters)
  assert out.converged == ref.converged
  f = out.f.cpu().numpy().astype(np.float64)
  g = out.g.cpu().numpy().astype(np.float64)
  if out.n_iters == ref.n_iters:
    np.testing.assert_array_equal(np.isfinite(f), np.isfinite(ref.f))
    np.testing.assert_array_equal(np.isfinite(g), np.isfinite(ref.g))
    ff, gf = np.isfinite(ref.f), np.isfinite(ref.g)
    np.testing.assert_allclose(f[ff], ref.f[ff], rtol=0, atol=pot_tol * eps)
    np.testing.assert_allclose(g[gf], ref.g[gf], rtol=0, atol=pot_tol * eps)
    np.testing.assert_allclose(out.reg_ot_cost, ref.reg_ot_cost, rtol=cost_rtol,
                               atol=cost_rtol * 1e-3)
    errs = out.errors.cpu().numpy()
    np.testing.assert_array_equal(errs == -1, ref.errors == -1)
    np.testing.assert_array_equal(np.isinf(errs), np.isinf(ref.errors))
    fin = np.isfinite(errs) & (errs != -1)
    np.testing.assert_allclose(errs[fin], ref.errors[fin], rtol=1e-2, atol=1e-6)
