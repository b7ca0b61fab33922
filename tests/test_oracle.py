"""The oracle itself: its loop semantics against the reference's own test
relations (tests/solvers/linear/sinkhorn_test.py), the float32 restatement
against float64, and the C port against the NumPy restatement."""
import numpy as np
import pytest

from oracle import sinkhorn_c, sinkhorn_np as o
from tests import problems


def test_zero_weights_give_minus_inf_potentials():
  x, y, a, b = problems.ref_test_problem()
  r = o.solve(x, y, a, b, epsilon=0.1)
  assert r.converged
  assert np.isneginf(r.f[0]) and np.isneginf(r.g[3])
  assert np.isfinite(r.f[1:]).all() and np.isfinite(np.delete(r.g, 3)).all()


def test_min_iterations_error_pattern():
  """sinkhorn_test.py:248-265."""
  x, y, a, b = problems.ref_test_problem()
  r = o.solve(x, y, a, b, epsilon=0.1, threshold=1e-3, min_iterations=34)
  e = r.errors
  assert np.isinf(e[:3]).all() and e[3] > 0
  last = e[(e > -1) & np.isfinite(e)][-1]
  assert last < 1e-3


def test_scan_loop_converged():
  """sinkhorn_test.py:267-284: min == max runs a scan of max // inner blocks."""
  x, y, a, b = problems.ref_test_problem()
  r = o.solve(x, y, a, b, epsilon=0.1, threshold=1e-3, min_iterations=50,
              max_iterations=50)
  assert r.converged and 0 < r.errors[-1] < 1e-3
  assert r.n_iters == 50


def test_full_blocks_past_max_iterations():
  """fixed_point_loop.py: a block always runs to its end, so max=25 runs 30."""
  x, y, a, b = problems.ref_test_problem()
  r = o.solve(x, y, a, b, epsilon=0.1, threshold=1e-9, max_iterations=25)
  assert r.n_iters == 30 and np.isfinite(r.errors).all()


def test_n_iters_is_multiple_of_inner():
  x, y, a, b = problems.ref_test_problem()
  for inner in (1, 3, 10):
    r = o.solve(x, y, a, b, epsilon=0.1, inner_iterations=inner)
    assert r.n_iters % inner == 0


def test_float32_close_to_float64():
  x, y, a, b = problems.uniform_cloud_problem(300, 257, 2, seed=5)
  r64 = o.solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean")
  r32 = o.solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean", dtype=np.float32)
  assert r32.n_iters == r64.n_iters
  np.testing.assert_allclose(r32.f, r64.f, atol=1e-4 * r64.epsilon)
  np.testing.assert_allclose(r32.reg_ot_cost, r64.reg_ot_cost, rtol=1e-5)


def test_online_blocks_equal_dense():
  """pointcloud.py online mode equals the materialised cost (the reference's
  sinkhorn_test.py:310-375 relation)."""
  x, y, a, b = problems.uniform_cloud_problem(100, 130, 3, seed=2)
  r1 = o.solve(x, y, a, b, epsilon=0.05)
  r2 = o.solve(x, y, a, b, epsilon=0.05, batch_size=17)
  np.testing.assert_allclose(r1.f, r2.f, rtol=1e-12, atol=1e-12)
  assert r1.n_iters == r2.n_iters


def test_restart_converges_in_one_block():
  """sinkhorn_test.py:491-546."""
  x, y, a, b = problems.ref_test_problem()
  r = o.solve(x, y, a, b, epsilon=0.1)
  r2 = o.solve(x, y, a, b, epsilon=0.1, init=(r.f, r.g))
  assert r2.n_iters == 10 and r2.errors[0] < r.errors[r.errors > -1][-1]


def test_mean_cost_closed_form_matches_dense():
  x, y, _, _ = problems.uniform_cloud_problem(50, 60, 4, seed=3)
  c = o.sqeuclidean_all_pairs(x.astype(np.float64), y.astype(np.float64))
  np.testing.assert_allclose(o.mean_cost_matrix(x.astype(np.float64), y.astype(np.float64)),
                             c.mean(), rtol=1e-12)


@pytest.mark.parametrize("kw", [dict(), dict(min_iterations=34), dict(max_iterations=25),
                                dict(norm_error=2), dict(inner_iterations=3)])
def test_c_port_matches_numpy(kw):
  x, y, a, b = problems.ref_test_problem()
  r_np = o.solve(x, y, a, b, epsilon=0.1, dtype=np.float32, **kw)
  r_c = sinkhorn_c.solve(x, y, a, b, epsilon=0.1, **kw)
  assert r_c.n_iters == r_np.n_iters and r_c.converged == r_np.converged
  fin = np.isfinite(r_np.f)
  np.testing.assert_array_equal(np.isfinite(r_c.f), fin)
  np.testing.assert_allclose(r_c.f[fin], r_np.f[fin], atol=2e-5 * 0.1)
  np.testing.assert_allclose(r_c.reg_ot_cost, r_np.reg_ot_cost, rtol=2e-6)
