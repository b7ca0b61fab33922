"""The log-domain kernel application (ottb_apply_lse_kernel) and the
row-sharded solve on one GPU.

Tolerances: apply_lse_kernel within 2e-5 eps (FP32) and 2e-3 eps (BF16
split-3, whose exponents carry 2^-15 |x||y| / eps) of the float64 values;
the sharded solve (one rank) against linear.solve on the same problem: the
same iteration count, potentials within 1e-4 eps (FP32) / 1e-3 eps (BF16
split-3: the two paths round the split products in different sweeps),
reg_ot_cost within 1e-5 relative.
"""
import numpy as np
import pytest

from oracle import sinkhorn_np as o
from tests import problems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,m,d,precision", [(500, 700, 3, "fp32"), (900, 600, 64, "fp32"),
                                             (900, 600, 64, "bf16_split3"),
                                             (333, 1000, 128, "bf16_split3")])
def test_apply_lse_kernel_matches_oracle(n, m, d, precision):
  import torch
  from ott_b200.geometry import pointcloud
  x, y, _, _ = problems.uniform_cloud_problem(n, m, d, seed=n + d)
  eps = 0.05 * o.mean_cost_matrix(x.astype(np.float64), y.astype(np.float64))
  rng = np.random.default_rng(1)
  f = rng.uniform(-1, 1, n) * eps * 5
  g = rng.uniform(-1, 1, m) * eps * 5
  f[3] = -np.inf
  g[[0, 11]] = -np.inf
  geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                               epsilon=float(eps))
  og = o.Geom(x.astype(np.float64), y.astype(np.float64), float(eps))
  for axis in (0, 1):
    got, sgn = geom.apply_lse_kernel(torch.as_tensor(f, dtype=torch.float32).cuda(),
                                     torch.as_tensor(g, dtype=torch.float32).cuda(), float(eps),
                                     axis=axis, precision=precision)
    want = og.apply_lse_kernel(f.astype(np.float32).astype(np.float64),
                               g.astype(np.float32).astype(np.float64), eps, axis)[0]
    got = got.cpu().numpy().astype(np.float64)
    np.testing.assert_array_equal(np.isneginf(got), np.isneginf(want))
    fin = np.isfinite(want)
    tol = (2e-5 if precision == "fp32" else 2e-3) * eps
    np.testing.assert_allclose(got[fin], want[fin], rtol=0, atol=tol)
    assert float(sgn[0]) == 1.0


@pytest.mark.parametrize("n,m,d,precision", [(2000, 1500, 3, "fp32"), (4000, 3000, 64, "fp32"),
                                             (4000, 3000, 64, "auto")])
def test_sharded_solve_one_rank_matches_solve(n, m, d, precision):
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  from ott_b200.solvers.linear import sharded
  x, y, a, b = problems.uniform_cloud_problem(n, m, d, seed=n)
  out = sharded.solve_sharded(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                              torch.as_tensor(a).cuda(), torch.as_tensor(b).cuda(),
                              epsilon=0.05, relative_epsilon="mean", precision=precision)
  geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                               epsilon=0.05, relative_epsilon="mean")
  ref = linear.solve(geom, torch.as_tensor(a).cuda(), torch.as_tensor(b).cuda(),
                     precision=precision)
  assert abs(out.epsilon - geom.epsilon) <= 1e-6 * geom.epsilon
  assert out.n_iters == ref.n_iters and out.converged == ref.converged
  tol = (1e-4 if precision == "fp32" else 1e-3) * geom.epsilon
  np.testing.assert_allclose(out.f.cpu().numpy(), ref.f.cpu().numpy(), rtol=0, atol=tol)
  np.testing.assert_allclose(out.g.cpu().numpy(), ref.g.cpu().numpy(), rtol=0, atol=tol)
  assert abs(out.reg_ot_cost - ref.reg_ot_cost) <= 1e-5 * abs(ref.reg_ot_cost)


def test_geometry_methods_match_oracle():
  """PointCloud.update_potential, cost_matrix, kernel_matrix, diag_cost and
  apply_cost (geometry.py:95-145, 376-398, 568-600; pointcloud.py:451-454)
  against float64."""
  import torch
  from ott_b200.geometry import pointcloud
  n, d = 200, 4
  x, y, a, b = problems.uniform_cloud_problem(n, n, d, seed=51)
  geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                               epsilon=0.1, scale_cost=2.0)
  og = o.Geom(x.astype(np.float64), y.astype(np.float64), 0.1, inv_scale=0.5)
  c = og.cost_block()
  np.testing.assert_allclose(geom.cost_matrix.cpu().numpy(), c, rtol=1e-5, atol=1e-6)
  np.testing.assert_allclose(geom.kernel_matrix.cpu().numpy(), np.exp(-c / 0.1), rtol=1e-4)
  np.testing.assert_allclose(geom.diag_cost.cpu().numpy(),
                             ((x.astype(np.float64) - y) ** 2).sum(1), rtol=1e-5)
  v = np.random.default_rng(0).standard_normal((n, 3))
  for axis in (0, 1):
    got = geom.apply_cost(torch.as_tensor(v, dtype=torch.float32).cuda(), axis=axis)
    want = c.T @ v if axis == 0 else c @ v
    np.testing.assert_allclose(got.cpu().numpy(), want, rtol=0, atol=1e-4 * np.abs(want).max())
  f = np.zeros(n)
  g = np.zeros(n)
  new_g = geom.update_potential(torch.as_tensor(f, dtype=torch.float32).cuda(),
                                torch.as_tensor(g, dtype=torch.float32).cuda(),
                                torch.as_tensor(np.log(b), dtype=torch.float32).cuda(), axis=0)
  want = og.update_potential(f, g, np.log(b.astype(np.float64)), None, axis=0)
  np.testing.assert_allclose(new_g.cpu().numpy(), want, rtol=0, atol=2e-5 * 0.1)
