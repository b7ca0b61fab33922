"""The Krylov solvers behind ImplicitDiff, on the CPU (plain torch
tensors): solve_jax_cg (jax.scipy's stopping rule), solve_normal_cg
(lineax CG / NormalCG defaults), the host MINRES loop, and the default
solve's two forms of its symmetric operator on a dense FP32 plan."""
import numpy as np
import torch

from ott_b200.solvers.linear import implicit_differentiation as imp


def _spd(k, seed):
  rng = np.random.default_rng(seed)
  q = rng.standard_normal((k, k))
  return torch.as_tensor(q @ q.T + k * np.eye(k))


def test_symmetric_cg_solves_spd_system():
  a = _spd(30, 0)
  b = torch.as_tensor(np.random.default_rng(1).standard_normal(30))
  x = imp.solve_normal_cg(lambda z: a @ z, b, None, True, rtol=1e-12, atol=0.0)
  np.testing.assert_allclose((a @ x).numpy(), b.numpy(), atol=1e-9)
  x2 = imp.solve_jax_cg(lambda z: a @ z, b, None, True, tol=1e-12)
  np.testing.assert_allclose(x2.numpy(), x.numpy(), atol=1e-9)


def test_normal_cg_least_squares_min_norm():
  """Non-symmetric, singular: NormalCG's limit is the least-squares
  solution of least norm."""
  rng = np.random.default_rng(2)
  k = 20
  m = rng.standard_normal((k, k))
  m[:, -1] = m[:, 0]  # rank k - 1
  mt = torch.as_tensor(m)
  b = torch.as_tensor(rng.standard_normal(k))
  x = imp.solve_normal_cg(lambda z: mt @ z, b, lambda z: mt.T @ z, False,
                          rtol=1e-13, atol=0.0, max_steps=2000)
  want = np.linalg.lstsq(m, b.numpy(), rcond=None)[0]
  np.testing.assert_allclose(x.numpy(), want, atol=1e-7 * np.abs(want).max())


def test_jax_cg_normal_operator_and_ridge():
  """solve_jax_cg on a non-symmetric operator runs CG on lin_t(lin(.))
  against b as given (implicit_differentiation.py:314-322), ridge terms
  added to that operator."""
  rng = np.random.default_rng(3)
  k = 15
  m = torch.as_tensor(rng.standard_normal((k, k)) + 4 * np.eye(k))
  b = torch.as_tensor(rng.standard_normal(k))
  x = imp.solve_jax_cg(lambda z: m @ z, b, lambda z: m.T @ z, False, ridge_identity=0.5,
                       ridge_kernel=0.25, tol=1e-13)
  op = m.T @ m + 0.5 * torch.eye(k, dtype=torch.float64) + 0.25 * torch.ones(k, k,
                                                                             dtype=torch.float64)
  np.testing.assert_allclose((op @ x).numpy(), b.numpy(), atol=1e-9)


def test_minres_solves_spd_and_singular_systems():
  """MINRES: an SPD system to the tolerance; a consistent singular one
  (null vector removed from the right-hand side) to the solution
  orthogonal to the null space; the residual estimate never increases."""
  rng = np.random.default_rng(6)
  a = _spd(40, 7)
  b = torch.as_tensor(rng.standard_normal(40))
  x = imp._minres(lambda z: a @ z, b, 1e-12, 500)
  np.testing.assert_allclose((a @ x).numpy(), b.numpy(), atol=1e-9)
  assert imp.last_solve_info["true_rel_residual"] < 1e-10
  q, _ = np.linalg.qr(rng.standard_normal((30, 30)))
  lam = np.concatenate([[0.0], rng.uniform(0.01, 1.0, 29)])
  s = torch.as_tensor(q @ np.diag(lam) @ q.T)
  rhs = torch.as_tensor(q[:, 1:] @ rng.standard_normal(29))
  hist = []

  def op(z):
    hist.append(1)
    return s @ z

  x = imp._minres(op, rhs, 1e-12, 500)
  want = np.linalg.lstsq(s.numpy(), rhs.numpy(), rcond=1e-10)[0]
  np.testing.assert_allclose(x.numpy(), want, atol=1e-8 * np.abs(want).max())


def test_minres_step_limit_reports_residual():
  a = _spd(40, 8)
  b = torch.as_tensor(np.random.default_rng(9).standard_normal(40))
  x = imp._minres(lambda z: a @ z, b, 1e-14, 3)
  info = imp.last_solve_info
  assert info["steps"] == 3 and info["rel_residual"] > 1e-6
  true = float(torch.linalg.vector_norm(b - a @ x) / torch.linalg.vector_norm(b))
  assert abs(info["true_rel_residual"] - true) < 1e-12


def test_implicit_diff_fields_and_replace():
  d = imp.ImplicitDiff()
  assert d.solver is None and d.precondition_fun is None and d.symmetric is False
  d2 = d.replace(symmetric=True, solver_kwargs={"rtol": 1e-8})
  assert d2.symmetric and d2.solver_kwargs == {"rtol": 1e-8} and not d.symmetric


def _dense_app(p, with_f32):
  """The backward's plan product on a dense CPU plan, FP32 like the GPU's
  (optionally with the FP32-in, FP32-out form ``app.f32``)."""
  p32 = p.to(torch.float32)

  def app32(v, axis):
    v32 = v.to(torch.float32)
    return v32 @ p32 if axis == 0 else p32 @ v32

  def app(v, axis):
    return app32(v, axis).double()
  if with_f32:
    app.f32 = app32
  return app


def test_default_solve_operator_forms_agree():
  """``_solve_default`` with the fused symmetric operator (FP32 inputs
  written in place, output by two multiply-adds) and with the plain
  expression: the same solution to rounding, on both side orders, and a
  recomputed residual at the FP32 products' floor."""
  rng = np.random.default_rng(7)
  for n, m in ((40, 25), (25, 40)):
    p = torch.as_tensor(rng.uniform(0.1, 1.0, (n, m)))
    p = p / p.sum()
    ma, mb = p.sum(1), p.sum(0)
    ones_a, ones_b = torch.ones(n, dtype=torch.bool), torch.ones(m, dtype=torch.bool)
    gr_f = torch.as_tensor(rng.standard_normal(n))
    gr_g = torch.as_tensor(rng.standard_normal(m))
    sols = []
    for with_f32 in (False, True):
      lf, lg = imp.ImplicitDiff()._solve_default(gr_f, gr_g, ma, mb, ones_a, ones_b,
                                                 _dense_app(p, with_f32), n > m)
      assert imp.last_solve_info["true_rel_residual"] < 1e-5, imp.last_solve_info
      sols.append(torch.cat([lf, lg]))
    scale = float(sols[0].abs().max())
    assert float((sols[0] - sols[1]).abs().max()) <= 1e-8 * scale


def test_app_plans_each_axis_once_and_falls_back():
  """``ImplicitDiff._app``: each axis asks the geometry for a planned
  product once and reuses it; without one it calls ``_apply_raw``; ``app``
  is ``app.f32`` in float64. Below 2^25 plan entries the chosen precision
  becomes FP32."""
  p = torch.as_tensor(np.random.default_rng(3).uniform(size=(6, 4)))

  class Geom:
    shape = (6, 4)

    def __init__(self, planned):
      self.planned, self.asked, self.raw = planned, [], []

    def _sweep_product(self, f, g, axis, precision):
      self.asked.append((axis, precision))
      if not self.planned:
        return None
      return lambda v2: (v2.float() @ p.float()) if axis == 0 else (v2.float() @ p.float().T)

    def _apply_raw(self, f, g, v2, axis, precision):
      self.raw.append((axis, precision))
      return (v2.float() @ p.float()) if axis == 0 else (v2.float() @ p.float().T)

  for planned in (True, False):
    geom = Geom(planned)
    app = imp.ImplicitDiff._app(geom, None, None, "auto")
    v0, v1 = torch.ones(6, dtype=torch.float64), torch.ones(4, dtype=torch.float64)
    for _ in range(3):
      a0, a1 = app(v0, 0), app(v1, 1)
      assert a0.dtype == torch.float64 and a0.shape == (4,) and a1.shape == (6,)
      assert torch.equal(app.f32(v0, 0).double(), a0)
    np.testing.assert_allclose(a0.numpy(), p.sum(0).numpy(), rtol=1e-6)
    np.testing.assert_allclose(a1.numpy(), p.sum(1).numpy(), rtol=1e-6)
    assert geom.asked == [(0, "fp32"), (1, "fp32")]
    assert (len(geom.raw) == 0) if planned else (len(geom.raw) == 9)
