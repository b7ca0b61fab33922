"""The oracle's implicit differentiation of the potentials against the
reference's own ImplicitDiff (golden vectors) and against finite
differences of converged float64 Sinkhorn solutions."""
import numpy as np
import pytest

from oracle import sinkhorn_np as o
from tests import golden_cases


def _geom(data, geom_kw):
  x, y = data["x"], data["y"]
  inv = o.inv_scale_cost(x, y, geom_kw.get("scale_cost", 1.0))
  return o.Geom(x, y, float(geom_kw["epsilon"]), inv_scale=inv)


@pytest.mark.parametrize("name", golden_cases.implicit_names())
def test_oracle_matches_reference_implicit_diff(name):
  data, geom_kw = golden_cases.load_implicit(name)
  geom = _geom(data, geom_kw)
  args = (data["f"], data["g"], data["a"], data["b"], geom)
  lam = o.implicit_solve(data["gr_f"], data["gr_g"], *args)
  np.testing.assert_allclose(lam, data["lam"], rtol=0, atol=1e-9 * np.abs(data["lam"]).max())
  foc = o.first_order_conditions(*args)
  assert np.abs(foc).max() < 1e-8
  grads = o.implicit_pullback(data["lam"], *args,
                              scale_cost_mean=geom_kw.get("scale_cost") == "mean")
  for got, key in zip(grads, ("gx", "gy", "ga", "gb")):
    want = data[key]
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-6 * np.abs(want).max(), err_msg=key)


@pytest.mark.parametrize("scale_mean", [False, True])
def test_oracle_gradient_matches_finite_differences_of_solutions(scale_mean):
  """<w, f*(x)> + <v, g*(x)> with sum(w) = sum(v) does not depend on the
  potentials' free constant; its derivative by central differences of
  converged solves equals the implicit gradient."""
  rng = np.random.default_rng(3)
  n, m, d = 9, 7, 2
  x, y = rng.uniform(size=(n, d)), rng.uniform(size=(m, d))
  a = rng.uniform(0.2, 1.2, n)
  a /= a.sum()
  b = rng.uniform(0.2, 1.2, m)
  b /= b.sum()
  w, v = rng.standard_normal(n), rng.standard_normal(m)
  v += (w.sum() - v.sum()) / m

  def geom_of(xx, yy):
    inv = o.inv_scale_cost(xx, yy, "mean" if scale_mean else 1.0)
    return o.Geom(xx, yy, 0.1, inv_scale=inv)

  def loss(xx, yy, aa, bb):
    r = o.sinkhorn(geom_of(xx, yy), aa, bb, threshold=1e-13, max_iterations=200000)
    return w @ r.f + v @ r.g

  r = o.sinkhorn(geom_of(x, y), a, b, threshold=1e-13, max_iterations=200000)
  gx, gy, ga, gb = o.implicit_grads(w, v, r.f, r.g, a, b, geom_of(x, y), scale_cost_mean=scale_mean)
  h = 1e-5
  for i, k in [(0, 0), (4, 1), (8, 0)]:
    xp, xm = x.copy(), x.copy()
    xp[i, k] += h
    xm[i, k] -= h
    fd = (loss(xp, y, a, b) - loss(xm, y, a, b)) / (2 * h)
    assert abs(fd - gx[i, k]) <= 1e-6 * np.abs(gx).max()
  for j in (0, 6):
    yp, ym = y.copy(), y.copy()
    yp[j, 1] += h
    ym[j, 1] -= h
    fd = (loss(x, yp, a, b) - loss(x, ym, a, b)) / (2 * h)
    assert abs(fd - gy[j, 1]) <= 1e-6 * np.abs(gy).max()
  # weights: a direction that keeps the total mass (balanced problems)
  da = np.zeros(n)
  da[2], da[5] = 1.0, -1.0
  fd = (loss(x, y, a + h * da, b) - loss(x, y, a - h * da, b)) / (2 * h)
  assert abs(fd - ga @ da) <= 1e-6 * np.abs(ga).max()


def test_zero_weights_are_left_out():
  """A zero-weight point gets a zero multiplier and zero gradients, and the
  rest equals the problem without it."""
  rng = np.random.default_rng(5)
  n, m, d = 10, 8, 3
  x, y = rng.uniform(size=(n, d)), rng.uniform(size=(m, d))
  a = rng.uniform(0.2, 1.2, n)
  a[3] = 0.0
  a /= a.sum()
  b = np.full(m, 1.0 / m)
  geom = o.Geom(x, y, 0.1)
  r = o.sinkhorn(geom, a, b, threshold=1e-12, max_iterations=100000)
  gf, gg = rng.standard_normal(n), rng.standard_normal(m)
  lam = o.implicit_solve(gf, gg, r.f, r.g, a, b, geom)
  gx, gy, ga, gb = o.implicit_pullback(lam, r.f, r.g, a, b, geom)
  assert lam[3] == 0.0 and ga[3] == 0.0 and np.all(gx[3] == 0.0)
  keep = np.arange(n) != 3
  geom2 = o.Geom(x[keep], y, 0.1)
  r2 = o.sinkhorn(geom2, a[keep], b, threshold=1e-12, max_iterations=100000)
  lam2 = o.implicit_solve(gf[keep], gg, r2.f, r2.g, a[keep], b, geom2)
  gx2, gy2, _, _ = o.implicit_pullback(lam2, r2.f, r2.g, a[keep], b, geom2)
  np.testing.assert_allclose(gx[keep], gx2, rtol=1e-6, atol=1e-9)
  np.testing.assert_allclose(gy, gy2, rtol=1e-6, atol=1e-9)
