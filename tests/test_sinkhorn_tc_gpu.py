"""Parity of the tensor-core path (tcgen05, BF16 split-3 inner products,
FP32 accumulation and log-sum-exp) with the float64 oracle.

Tolerances of this path: reg_ot_cost within 1e-4 relative of float64 (the
mixed-precision accuracy bar), f and g within 1e-3 * epsilon, iteration
counts within one block of inner_iterations.
"""
import numpy as np
import pytest

from tests import helpers, problems

pytestmark = pytest.mark.gpu


def _check(x, y, a, b, pot_tol=1e-3, cost_rtol=1e-4, **kw):
  geom, out = helpers.gpu_solve(x, y, a, b, precision="bf16_split3", **kw)
  ref = helpers.oracle_solve(x, y, a, b, **kw)
  assert abs(out.n_iters - ref.n_iters) <= out.inner_iterations, (out.n_iters, ref.n_iters)
  assert out.converged == ref.converged
  np.testing.assert_allclose(out.reg_ot_cost, ref.reg_ot_cost, rtol=cost_rtol)
  if out.n_iters == ref.n_iters:
    f = out.f.cpu().numpy().astype(np.float64)
    g = out.g.cpu().numpy().astype(np.float64)
    ff, gf = np.isfinite(ref.f), np.isfinite(ref.g)
    np.testing.assert_array_equal(np.isfinite(f), ff)
    np.testing.assert_array_equal(np.isfinite(g), gf)
    np.testing.assert_allclose(f[ff], ref.f[ff], rtol=0, atol=pot_tol * ref.epsilon)
    np.testing.assert_allclose(g[gf], ref.g[gf], rtol=0, atol=pot_tol * ref.epsilon)
  return out, ref


@pytest.mark.parametrize("n,m,d", [(128, 128, 64), (300, 257, 32), (1000, 1100, 64),
                                   (129, 513, 100), (640, 700, 128), (17, 29, 33)])
def test_tc_uniform_clouds(n, m, d):
  x, y, a, b = problems.uniform_cloud_problem(n, m, d, seed=n + m + d)
  _check(x, y, a, b, epsilon=0.05, relative_epsilon="mean")


def test_tc_gaussian_shift_small_eps():
  """The n=m=65536, d=64 workload's distribution at n=4096, eps 0.01 mean(C)."""
  x, y, a, b = problems.gaussian_shift_problem(4096, 4096, 64, seed=0)
  _check(x, y, a, b, epsilon=0.01, relative_epsilon="mean")


def test_tc_zero_weights():
  x, y, a, b = problems.ref_test_problem(n=170, m=290, d=64)
  out, ref = _check(x, y, a, b, epsilon=0.1)
  assert np.isneginf(out.f.cpu().numpy()[0]) and np.isneginf(out.g.cpu().numpy()[3])


def test_tc_matches_fp32_path():
  x, y, a, b = problems.uniform_cloud_problem(2000, 1500, 64, seed=4)
  _, o_tc = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean",
                              precision="bf16_split3")
  _, o_32 = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean",
                              precision="fp32")
  assert abs(o_tc.n_iters - o_32.n_iters) <= 10
  np.testing.assert_allclose(o_tc.reg_ot_cost, o_32.reg_ot_cost, rtol=1e-4)


def test_tc_batched_uneven():
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  probs = problems.batched_uneven_problems(10, d=32, lo=64, hi=900, seed=2)
  geoms = [pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                                 epsilon=0.05, relative_epsilon="mean")
           for x, y, _, _ in probs]
  outs = linear.solve_batch(geoms, [torch.as_tensor(p[2]).cuda() for p in probs],
                            [torch.as_tensor(p[3]).cuda() for p in probs],
                            precision="bf16_split3")
  for (x, y, a, b), out in zip(probs, outs):
    ref = helpers.oracle_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean")
    assert abs(out.n_iters - ref.n_iters) <= 10
    np.testing.assert_allclose(out.reg_ot_cost, ref.reg_ot_cost, rtol=1e-4)
