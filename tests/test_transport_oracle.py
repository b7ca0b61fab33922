"""Transport application and the reg_ot_cost gradient in the oracle.

The oracle's ``apply_transport_from_potentials`` reproduces the reference's
own (golden vectors made by running the reference, tests/golden), and its
fixed-potential gradient formula for ``reg_ot_cost`` agrees with finite
differences of whole re-solves at a tight threshold (envelope theorem: at
the optimum the potentials' own sensitivity contributes nothing)."""
import numpy as np
import pytest

from oracle import sinkhorn_np as o
from tests import golden_cases, problems


@pytest.mark.parametrize("name", golden_cases.names())
def test_oracle_apply_matches_reference(name):
  data, geom_kw, _, _ = golden_cases.load(name, "f64")
  x, y = data["x"], data["y"]
  inv = o.inv_scale_cost(x, y, geom_kw.get("scale_cost", 1.0))
  geom = o.Geom(x, y, float(data["epsilon"]), inv_scale=inv)
  for axis, key in ((0, "0"), (1, "1")):
    want = data["apply" + key]
    for k in range(want.shape[0]):
      got_k = geom.apply_transport_from_potentials(data["f"], data["g"],
                                                   data["vec" + key][k], axis=axis)
      scale = np.max(np.abs(want[k])) + 1e-300
      np.testing.assert_allclose(got_k, want[k], rtol=0, atol=1e-11 * scale)


def _reg_cost(x, y, a, b, eps, scale_cost=1.0):
  return o.solve(x, y, a, b, epsilon=eps, scale_cost=scale_cost, threshold=1e-13,
                 max_iterations=20000).reg_ot_cost


@pytest.mark.parametrize("scale_cost", [1.0, "mean"])
def test_gradient_formula_matches_finite_differences(scale_cost):
  x, y, a, b = [v.astype(np.float64) for v in problems.uniform_cloud_problem(13, 17, 3, seed=5)]
  eps = 0.2
  r = o.solve(x, y, a, b, epsilon=eps, scale_cost=scale_cost, threshold=1e-13,
              max_iterations=20000)
  inv = o.inv_scale_cost(x, y, scale_cost)
  geom = o.Geom(x, y, eps, inv_scale=inv)
  gx, gy, ga, gb = o.reg_ot_cost_grads(r.f, r.g, a, b, geom,
                                       scale_cost_mean=scale_cost == "mean")
  h = 1e-5
  for (i, k) in [(0, 0), (5, 2), (12, 1)]:
    xp, xm = x.copy(), x.copy()
    xp[i, k] += h
    xm[i, k] -= h
    fd = (_reg_cost(xp, y, a, b, eps, scale_cost) - _reg_cost(xm, y, a, b, eps, scale_cost)) / (2 * h)
    np.testing.assert_allclose(gx[i, k], fd, rtol=1e-5, atol=1e-8)
  for (j, k) in [(3, 0), (16, 2)]:
    yp, ym = y.copy(), y.copy()
    yp[j, k] += h
    ym[j, k] -= h
    fd = (_reg_cost(x, yp, a, b, eps, scale_cost) - _reg_cost(x, ym, a, b, eps, scale_cost)) / (2 * h)
    np.testing.assert_allclose(gy[j, k], fd, rtol=1e-5, atol=1e-8)
  # weights: a direction that keeps the total mass (balanced problem)
  ap, am = a.copy(), a.copy()
  ap[2] += h
  ap[7] -= h
  am[2] -= h
  am[7] += h
  fd = (_reg_cost(x, y, ap, b, eps, scale_cost) - _reg_cost(x, y, am, b, eps, scale_cost)) / (2 * h)
  np.testing.assert_allclose(ga[2] - ga[7], fd, rtol=1e-5, atol=1e-8)
