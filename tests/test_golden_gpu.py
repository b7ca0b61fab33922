"""The CUDA path (through the C ABI) against the golden vectors computed by
the reference's own code in float64: f and g within 1e-4 * epsilon,
reg_ot_cost within 1e-5 relative, identical n_iters, convergence flag and
error pattern (FP32 engine); the tensor-core engine within its own bar
(reg_ot_cost 1e-4 relative, potentials 1e-3 * epsilon)."""
import numpy as np
import pytest

from tests import golden_cases

pytestmark = pytest.mark.gpu


def _gpu(data, geom, solver, init, precision):
  import torch
  from ott_b200.geometry import epsilon_scheduler, pointcloud
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers.linear import sinkhorn
  g = dict(geom)
  if "eps_init" in g:
    g["epsilon"] = epsilon_scheduler.Epsilon(target=g.pop("epsilon"), init=g.pop("eps_init"),
                                             decay=g.pop("eps_decay"))
  t = lambda v: torch.as_tensor(np.asarray(v, np.float32)).cuda()
  pc = pointcloud.PointCloud(t(data["x"]), t(data["y"]), **g)
  prob = linear_problem.LinearProblem(pc, t(data["a"]), t(data["b"]))
  solver = sinkhorn.Sinkhorn(precision=precision, **solver)
  init_fg = (t(data["f_init"]), t(data["g_init"])) if init == "restart" else None
  return solver(prob, init=init_fg)


@pytest.mark.parametrize("name", golden_cases.names())
@pytest.mark.parametrize("precision", ["fp32", "bf16_split3"])
def test_gpu_matches_reference_golden(name, precision):
  data, geom, solver, init = golden_cases.load(name, "f64")
  out = _gpu(data, geom, solver, init, precision)
  eps = float(data["epsilon"])
  strict = precision == "fp32"
  pot_tol, cost_rtol = (1e-4, 1e-5) if strict else (1e-3, 1e-4)
  blocks = 0 if strict else 1
  assert abs(out.n_iters - int(data["n_iters"])) <= blocks * out.inner_iterations
  assert out.converged == bool(data["converged"])
  np.testing.assert_allclose(out.reg_ot_cost, float(data["reg_ot_cost"]), rtol=cost_rtol)
  f = out.f.cpu().numpy().astype(np.float64)
  g = out.g.cpu().numpy().astype(np.float64)
  errs = out.errors.cpu().numpy()
  if out.n_iters == int(data["n_iters"]):
    # the reference's own state after the same iterations
    at_f, at_g, at_err = data["f"], data["g"], data["errors"]
    np.testing.assert_array_equal(errs == -1, data["errors"] == -1)
  else:
    # stopped a block apart: the float64 oracle (equal to the reference's
    # float64 run to 1e-12 on every case) run for the GPU's iteration count
    at = golden_cases.oracle_run(data, geom, solver, init, out.n_iters)
    at_f, at_g, at_err = at.f, at.g, at.errors
  ff, gf = np.isfinite(at_f), np.isfinite(at_g)
  np.testing.assert_array_equal(np.isfinite(f), ff)
  np.testing.assert_array_equal(np.isfinite(g), gf)
  np.testing.assert_allclose(f[ff], at_f[ff], rtol=0, atol=pot_tol * eps)
  np.testing.assert_allclose(g[gf], at_g[gf], rtol=0, atol=pot_tol * eps)
  k = out.n_iters // out.inner_iterations
  np.testing.assert_array_equal(np.isinf(errs[:k]), np.isinf(at_err[:k]))
