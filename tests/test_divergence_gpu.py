"""Sinkhorn divergence on the GPU (three solves in one launch; the symmetric
terms with the parallel, momentum-1/2 update) against the reference's own
run (golden vectors) and the float64 oracle.

Tolerances: divergence within 1e-4 relative (1e-5 absolute for values near
0), potentials within 1e-4 * epsilon (FP32 path) or 1e-3 * epsilon (BF16
split-3 path), iteration counts within one block; gradients within 1e-4 of
the largest entry of the oracle's fixed-potential formula.
"""
import numpy as np
import pytest

from oracle import sinkhorn_np as o
from tests import golden_cases, problems

pytestmark = pytest.mark.gpu


def _div(x, y, a, b, geom_kw, dkw, precision="auto", grad=False):
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.tools import sinkhorn_divergence as sd
  xt = torch.as_tensor(x, dtype=torch.float32).cuda().requires_grad_(grad)
  yt = torch.as_tensor(y, dtype=torch.float32).cuda().requires_grad_(grad)
  kw = {} if a is None else dict(a=torch.as_tensor(a, dtype=torch.float32).cuda(),
                                 b=torch.as_tensor(b, dtype=torch.float32).cuda())
  div, out = sd.sinkhorn_divergence(pointcloud.PointCloud, xt, yt, **kw, **geom_kw, **dkw,
                                    solve_kwargs=dict(precision=precision))
  return div, out, xt, yt


@pytest.mark.parametrize("name", golden_cases.divergence_names())
def test_divergence_matches_reference_golden(name):
  data, geom, dkw, weights = golden_cases.load_divergence(name, "f64")
  a, b = (data["a"], data["b"]) if weights else (None, None)
  div, out, _, _ = _div(data["x"], data["y"], a, b, geom, dkw)
  want = float(data["divergence"])
  assert abs(float(div) - want) <= max(1e-4 * abs(want), 1e-5)
  eps = float(data["epsilon"])
  for k, tag in enumerate(("xy", "xx", "yy")):
    assert abs(out.n_iters[k] - int(data["n_iters"][k])) <= 10
    if out.n_iters[k] == int(data["n_iters"][k]):
      f, g = out.potentials[k]
      np.testing.assert_allclose(f.cpu().numpy(), data["f_" + tag], rtol=0, atol=1e-4 * eps)
      np.testing.assert_allclose(g.cpu().numpy(), data["g_" + tag], rtol=0, atol=1e-4 * eps)


@pytest.mark.parametrize("d,precision", [(3, "fp32"), (40, "bf16_split3")])
def test_divergence_and_gradient_match_oracle(d, precision):
  x, y, a, b = problems.uniform_cloud_problem(300, 250, d, seed=d)
  geom_kw = dict(epsilon=0.05, relative_epsilon="mean")
  div, out, xt, yt = _div(x, y, a, b, geom_kw, {}, precision=precision, grad=True)
  ref, res = o.sinkhorn_divergence(x, y, a, b, **geom_kw)
  assert abs(float(div.detach()) - ref) <= 1e-4 * abs(ref)
  tol_pot = (1e-4 if precision == "fp32" else 1e-3) * res[0].epsilon
  for k in range(3):
    assert abs(out.n_iters[k] - res[k].n_iters) <= 10
    if out.n_iters[k] == res[k].n_iters:
      np.testing.assert_allclose(out.potentials[k][0].detach().cpu().numpy(), res[k].f, atol=tol_pot)
  div.backward()
  # d div / dx = d reg(x, y)/dx - (d reg(x, x)/dx in both roles) / 2, each
  # with the GPU's potentials held fixed
  f64 = lambda t: t.detach().cpu().numpy().astype(np.float64)
  pots = [(f64(p[0]), f64(p[1])) for p in out.potentials]
  eps = float(out.geoms[0].epsilon)
  gxy = o.reg_ot_cost_grads(*pots[0], a, b, o.Geom(x.astype(np.float64), y.astype(np.float64), eps))
  gxx = o.reg_ot_cost_grads(*pots[1], a, a, o.Geom(x.astype(np.float64), x.astype(np.float64), eps))
  gyy = o.reg_ot_cost_grads(*pots[2], b, b, o.Geom(y.astype(np.float64), y.astype(np.float64), eps))
  want_x = gxy[0] - 0.5 * (gxx[0] + gxx[1])
  want_y = gxy[1] - 0.5 * (gyy[0] + gyy[1])
  np.testing.assert_allclose(xt.grad.cpu().numpy(), want_x, rtol=0,
                             atol=1e-4 * np.abs(want_x).max())
  np.testing.assert_allclose(yt.grad.cpu().numpy(), want_y, rtol=0,
                             atol=1e-4 * np.abs(want_y).max())


def test_symmetric_solver_option_matches_oracle():
  """Sinkhorn(parallel_dual_updates=True, momentum=Momentum(0, value=0.5))
  on a symmetric problem is the reference's symmetric update."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers.linear import acceleration, sinkhorn
  x, _, a, _ = problems.uniform_cloud_problem(400, 400, 5, seed=4)
  a[7] = 0.0
  a /= a.sum()
  xt = torch.as_tensor(x).cuda()
  at = torch.as_tensor(a).cuda()
  geom = pointcloud.PointCloud(xt, xt, epsilon=0.05)
  solver = sinkhorn.Sinkhorn(parallel_dual_updates=True,
                             momentum=acceleration.Momentum(start=0, value=0.5))
  out = solver(linear_problem.LinearProblem(geom, at, at))
  ref = o.sinkhorn(o.Geom(x.astype(np.float64), x.astype(np.float64), 0.05), a, a,
                   parallel_dual_updates=True, momentum=0.5)
  assert out.n_iters == ref.n_iters
  f = out.f.cpu().numpy()
  assert np.isneginf(f[7]) and np.array_equal(f, out.g.cpu().numpy())
  fin = np.isfinite(ref.f)
  np.testing.assert_allclose(f[fin], ref.f[fin], atol=1e-4 * 0.05)
  np.testing.assert_allclose(out.errors.cpu().numpy(), ref.errors, rtol=1e-2, atol=1e-6)
  np.testing.assert_allclose(out.reg_ot_cost, ref.reg_ot_cost, rtol=1e-5)
  with pytest.raises(NotImplementedError):
    y = torch.as_tensor(x[::-1].copy()).cuda()
    solver(linear_problem.LinearProblem(pointcloud.PointCloud(xt, y, epsilon=0.05), at, at))
