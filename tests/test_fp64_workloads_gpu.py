"""Both engines at the measured workloads' full sizes against float64 solves
of the same inputs (tests/golden/*.fp64.npz, made by
tests/golden/gen_fp64_workloads.py with the float64 oracle).

Bars: the FP32 engine's f and g within 1e-4 * epsilon, reg_ot_cost within
1e-5 relative, the same n_iters; the BF16 split-3 tensor-core engine's
reg_ot_cost within 1e-4 relative, f and g within 1e-3 * epsilon, the same
n_iters (the float64 state is known only at its own count).
"""
import os

import numpy as np
import pytest

from tests import problems

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

CASES = {
    # name: (inputs, epsilon multiplier of mean(C), engines)
    "gauss65536_d64": (lambda: problems.gaussian_shift_problem(65536, 65536, 64, seed=0), 0.01,
                       ("fp32", "bf16_split3")),
    "uniform2048_d2": (lambda: problems.uniform_cloud_problem(2048, 2048, 2, seed=0), 0.05,
                       ("fp32",)),
}
BARS = {"fp32": (1e-4, 1e-5), "bf16_split3": (1e-3, 1e-4)}


def _checksums(x, y, a, b):
  out = []
  for v in (x, y, a, b):
    v = np.asarray(v, np.float64)
    out += [v.sum(), (v * v).sum()]
  return np.array(out)


@pytest.mark.parametrize("name,precision",
                         [(k, p) for k, v in CASES.items() for p in v[2]])
def test_engine_matches_float64_at_full_size(name, precision):
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  rec = np.load(os.path.join(HERE, f"{name}.fp64.npz"))
  make, mult, _ = CASES[name]
  x, y, a, b = make()
  np.testing.assert_allclose(_checksums(x, y, a, b), rec["checksums"], rtol=1e-12)
  geom = pointcloud.PointCloud(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(),
                               epsilon=mult, relative_epsilon="mean")
  out = linear.solve(geom, torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(),
                     threshold=float(rec["threshold"]), precision=precision)
  eps = float(rec["epsilon"])
  np.testing.assert_allclose(geom.epsilon, eps, rtol=1e-6)
  pot_tol, cost_rtol = BARS[precision]
  assert out.n_iters == int(rec["n_iters"]), (out.n_iters, int(rec["n_iters"]))
  assert out.converged == bool(rec["converged"])
  np.testing.assert_allclose(out.reg_ot_cost, float(rec["reg_ot_cost"]), rtol=cost_rtol)
  f = out.f.cpu().numpy().astype(np.float64)
  g = out.g.cpu().numpy().astype(np.float64)
  np.testing.assert_allclose(f, rec["f"], rtol=0, atol=pot_tol * eps)
  np.testing.assert_allclose(g, rec["g"], rtol=0, atol=pot_tol * eps)
  k = out.n_iters // out.inner_iterations
  errs = out.errors.cpu().numpy()[:k]
  np.testing.assert_allclose(errs, rec["errors"][:k], rtol=0.05, atol=2 * pot_tol)
