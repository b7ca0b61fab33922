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


@pytest.mark.parametrize("variant", ["scalar", "tiled"])
@pytest.mark.parametrize("name", [n for n in golden_cases.names() if "scalemean" not in n])
def test_c_port_matches_reference_float32(name, variant):
  """Both forms of the C port: the scalar restatement and the tiled,
  vectorised one timed as the CPU baseline."""
  data, geom, solver, init = golden_cases.load(name, "f32")
  eps = float(data["epsilon"])
  kw = dict(solver)
  if "eps_init" in geom:
    kw.update(eps_init=geom["eps_init"], eps_decay=geom["eps_decay"])
  if init == "restart":
    kw["init"] = (data["f_init"], data["g_init"])
  r = sinkhorn_c.solve(data["x"], data["y"], data["a"], data["b"], epsilon=eps,
                       variant=variant, **kw)
  assert abs(r.n_iters - int(data["n_iters"])) <= r.inner_iterations
  if r.n_iters == int(data["n_iters"]):
    fin = np.isfinite(data["f"])
    np.testing.assert_array_equal(np.isfinite(r.f), fin)
    np.testing.assert_allclose(r.f[fin], data["f"][fin], rtol=0, atol=2e-4 * eps)
  np.testing.assert_allclose(r.reg_ot_cost, float(data["reg_ot_cost"]), rtol=2e-5)


@pytest.mark.parametrize("name", [n for n in golden_cases.names() if "scan" not in n])
def test_rerun_at_the_same_count_reproduces_the_reference_state(name):
  """The re-run the GPU parity tests fall back to when a solve stops a block
  from the reference (threshold 0, max_iterations = the count) holds the
  reference's own state when given the reference's count."""
  data, geom, solver, init = golden_cases.load(name, "f64")
  n = int(data["n_iters"])
  r = golden_cases.oracle_run(data, geom, solver, init, n)
  assert r.n_iters == n
  for got, want in ((r.f, data["f"]), (r.g, data["g"])):
    fin = np.isfinite(want)
    np.testing.assert_array_equal(np.isfinite(got), fin)
    np.testing.assert_allclose(got[fin], want[fin], rtol=0, atol=1e-12)
  k = n // r.inner_iterations
  np.testing.assert_allclose(r.errors[:k], data["errors"][:k], rtol=1e-10, atol=1e-15)


def test_helper_rerun_matches_a_shorter_solve():
  """helpers.oracle_solve's rerun(n) is the state after n iterations: a
  solve with a looser threshold that stops at n gives the same potentials."""
  from tests import helpers, problems
  x, y, a, b = problems.uniform_cloud_problem(40, 50, 3, seed=3)
  tight = helpers.oracle_solve(x, y, a, b, epsilon=0.05, threshold=1e-6)
  loose = helpers.oracle_solve(x, y, a, b, epsilon=0.05, threshold=1e-2)
  assert loose.n_iters < tight.n_iters
  at = tight.rerun(loose.n_iters)
  np.testing.assert_array_equal(at.f, loose.f)
  np.testing.assert_array_equal(at.g, loose.g)
  k = loose.n_iters // loose.inner_iterations
  np.testing.assert_array_equal(at.errors[:k], loose.errors[:k])
