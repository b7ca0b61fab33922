"""Pins the oracle: its float64 restatement reproduces the reference's own
code (golden vectors from tests/golden/gen_golden.py) to 1e-12, and its
float32 mode and C port reproduce the reference's float32 run within FP32
rounding (potentials 1e-4 * epsilon, reg_ot_cost 1e-5 relative)."""
import numpy as np
import pytest

from oracle import sinkhorn_c, sinkhorn_np as o
from tests import golden_cases


def _oracle(data, geom, solver, init, dtype):
  kw = dict(geom)
  kw.update(solver)
  if init == "restart":
    kw["init"] = (data["f_init"], data["g_init"])
  return o.solve(data["x"], data["y"], data["a"], data["b"], dtype=dtype, **kw)


@pytest.mark.parametrize("name", golden_cases.names())
def test_float64_oracle_matches_reference_exactly(name):
  data, geom, solver, init = golden_cases.load(name, "f64")
  r = _oracle(data, geom, solver, init, np.float64)
  assert r.n_iters == int(data["n_iters"]) and r.converged == bool(data["converged"])
  np.testing.assert_allclose(r.epsilon, float(data["epsilon"]), rtol=1e-14)
  np.testing.assert_array_equal(np.isfinite(r.f), np.isfinite(data["f"]))
  fin = np.isfinite(data["f"])
  np.testing.assert_allclose(r.f[fin], data["f"][fin], rtol=0, atol=1e-12)
  fin = np.isfinite(data["g"])
  np.testing.assert_allclose(r.g[fin], data["g"][fin], rtol=0, atol=1e-12)
  np.testing.assert_allclose(r.errors, data["errors"], rtol=1e-10, atol=1e-15)
  np.testing.assert_allclose(r.reg_ot_cost, float(data["reg_ot_cost"]), rtol=1e-13)


@pytest.mark.parametrize("name", golden_cases.names())
def test_float32_oracle_matches_reference_float32(name):
  data, geom, solver, init = golden_cases.load(name, "f32")
  r = _oracle(data, geom, solver, init, np.float32)
  eps = float(data["epsilon"])
  assert abs(r.n_iters - int(data["n_iters"])) <= r.inner_iterations
  if r.n_iters == int(data["n_iters"]):
    fin = np.isfinite(data["f"])
    np.testing.assert_allclose(r.f[fin], data["f"][fin], rtol=0, atol=1e-4 * eps)
  np.testing.assert_allclose(r.reg_ot_cost, float(data["reg_ot_cost"]), rtol=1e-5)


@pytest.mark.parametrize("name", [n for n in golden_cases.names() if "scalemean" not in n])
def test_c_port_matches_reference_float32(name):
  data, geom, solver, init = golden_cases.load(name, "f32")
  eps = float(data["epsilon"])
  kw = dict(solver)
  if "eps_init" in geom:
    kw.update(eps_init=geom["eps_init"], eps_decay=geom["eps_decay"])
  if init == "restart":
    kw["init"] = (data["f_init"], data["g_init"])
  r = sinkhorn_c.solve(data["x"], data["y"], data["a"], data["b"], epsilon=eps, **kw)
  assert abs(r.n_iters - int(data["n_iters"])) <= r.inner_iterations
  if r.n_iters == int(data["n_iters"]):
    fin = np.isfinite(data["f"])
    np.testing.assert_array_equal(np.isfinite(r.f), fin)
    np.testing.assert_allclose(r.f[fin], data["f"][fin], rtol=0, atol=2e-4 * eps)
  np.testing.assert_allclose(r.reg_ot_cost, float(data["reg_ot_cost"]), rtol=2e-5)
