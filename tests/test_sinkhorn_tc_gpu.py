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
  """Potentials within pot_tol * eps of the oracle's state after the GPU's
  iteration count; the error log within 2 * pot_tol (a potential error of
  pot_tol * eps moves each marginal entry by about pot_tol relative)."""
  geom, out = helpers.gpu_solve(x, y, a, b, precision="bf16_split3", **kw)
  ref = helpers.oracle_solve(x, y, a, b, **kw)
  helpers.assert_parity(geom, out, ref, pot_tol=pot_tol, cost_rtol=cost_rtol, iter_blocks=1,
                        err_rtol=1e-2, err_atol=2 * pot_tol)
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
  for (x, y, a, b), out, geom in zip(probs, outs, geoms):
    ref = helpers.oracle_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean")
    helpers.assert_parity(geom, out, ref, pot_tol=1e-3, cost_rtol=1e-4, iter_blocks=1,
                          err_rtol=1e-2, err_atol=2e-3)


def test_tc_batched_uneven_large_sizes():
  """One launch over problems of the batched workload's family at up to
  16384 points a side (4-component Gaussian mixtures, d = 32, Dirichlet(1)
  weights, eps = 0.05 mean(C)), next to small ones; each against the float64
  oracle in blocked mode (batch_size) on every host thread."""
  import os

  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  rng = np.random.default_rng(11)
  shapes = [(16384, 1024), (1536, 16384), (6000, 5000), (128, 200), (300, 129)]
  probs = []
  for n, m in shapes:
    x, y = problems.gmm_cloud(rng, n, 32), problems.gmm_cloud(rng, m, 32)
    a = rng.dirichlet(np.ones(n)).astype(np.float32)
    b = rng.dirichlet(np.ones(m)).astype(np.float32)
    probs.append((x, y, a, b))
  geoms = [pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                                 epsilon=0.05, relative_epsilon="mean")
           for x, y, _, _ in probs]
  outs = linear.solve_batch(geoms, [torch.as_tensor(p[2]).cuda() for p in probs],
                            [torch.as_tensor(p[3]).cuda() for p in probs],
                            precision="bf16_split3")
  workers = os.cpu_count() or 1
  for (x, y, a, b), out, geom in zip(probs, outs, geoms):
    ref = helpers.oracle_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean",
                               batch_size=1024, workers=workers)
    helpers.assert_parity(geom, out, ref, pot_tol=1e-3, cost_rtol=1e-4, iter_blocks=1,
                          err_rtol=1e-2, err_atol=2e-3)
