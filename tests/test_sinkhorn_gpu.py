"""Parity of the CUDA path (through the C ABI) with the float64 oracle.

Tolerances: f and g within 1e-4 * epsilon absolute, reg_ot_cost within
1e-5 relative, n_iters equal (within one block where a stopping test sits
on the threshold). Relations mirror the reference's own tests
(tests/solvers/linear/sinkhorn_test.py).
"""
import numpy as np
import pytest

from oracle import sinkhorn_np as o
from tests import helpers, problems

pytestmark = pytest.mark.gpu


def test_reference_problem_zero_weights():
  """sinkhorn_test.py:38-54 problem (a[0] = b[3] = 0), epsilon 0.1."""
  x, y, a, b = problems.ref_test_problem()
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.1)
  ref = helpers.oracle_solve(x, y, a, b, epsilon=0.1)
  assert np.isneginf(out.f.cpu().numpy()[0]) and np.isneginf(out.g.cpu().numpy()[3])
  helpers.assert_parity(geom, out, ref)


@pytest.mark.parametrize("n,m,d", [(1, 1, 1), (2, 3, 2), (17, 29, 3), (127, 129, 31),
                                   (129, 127, 33), (300, 257, 2), (1000, 1100, 16),
                                   (513, 200, 64), (130, 140, 128)])
def test_ragged_shapes(n, m, d):
  x, y, a, b = problems.uniform_cloud_problem(n, m, d, seed=n + m + d)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean",
                                precision="fp32")
  ref = helpers.oracle_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean")
  helpers.assert_parity(geom, out, ref)


def test_gaussian_shift_d64_fp32():
  """The n=m=65536, d=64 workload's distribution at n=4096 (eps 0.01 mean(C),
  potentials ~100 eps): the FP32 path holds 1e-4 eps."""
  x, y, a, b = problems.gaussian_shift_problem(4096, 4096, 64, seed=0)
  kw = dict(epsilon=0.01, relative_epsilon="mean")
  geom, out = helpers.gpu_solve(x, y, a, b, precision="fp32", **kw)
  ref = helpers.oracle_solve(x, y, a, b, batch_size=1024, **kw)
  helpers.assert_parity(geom, out, ref)


def test_uniform_2048_d2():
  """n = m = 2048, d = 2, epsilon = 0.05 mean(C), threshold 1e-3."""
  x, y, a, b = problems.uniform_cloud_problem(2048, 2048, 2, seed=0)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean")
  ref = helpers.oracle_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean")
  assert out.converged
  helpers.assert_parity(geom, out, ref)


def test_min_iterations_pattern():
  """sinkhorn_test.py:248-265: errors inf, inf, inf, then > 0."""
  x, y, a, b = problems.ref_test_problem()
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.1, threshold=1e-3,
                                min_iterations=34)
  errs = out.errors.cpu().numpy()
  assert np.isinf(errs[:3]).all() and errs[3] > 0
  ref = helpers.oracle_solve(x, y, a, b, epsilon=0.1, threshold=1e-3, min_iterations=34)
  helpers.assert_parity(geom, out, ref)


def test_scan_loop():
  """sinkhorn_test.py:267-284: min == max runs a scan, last error computed."""
  x, y, a, b = problems.ref_test_problem()
  kw = dict(threshold=1e-3, min_iterations=50, max_iterations=50)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.1, **kw)
  errs = out.errors.cpu().numpy()
  assert out.converged and 0 < errs[-1] < 1e-3
  ref = helpers.oracle_solve(x, y, a, b, epsilon=0.1, **kw)
  helpers.assert_parity(geom, out, ref)


@pytest.mark.parametrize("kw", [dict(max_iterations=25), dict(max_iterations=7),
                                dict(min_iterations=10), dict(max_iterations=5),
                                dict(inner_iterations=3, max_iterations=40),
                                dict(norm_error=2), dict(threshold=1e-6, max_iterations=60)])
def test_loop_edge_cases(kw):
  x, y, a, b = problems.ref_test_problem()
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.1, **dict(kw))
  ref = helpers.oracle_solve(x, y, a, b, epsilon=0.1, **dict(kw))
  assert out.n_iters == ref.n_iters
  helpers.assert_parity(geom, out, ref, iter_blocks=0)


def test_epsilon_decay_schedule():
  import torch
  from ott_b200.geometry import epsilon_scheduler, pointcloud
  from ott_b200.solvers import linear
  from oracle import sinkhorn_np as oracle
  x, y, a, b = problems.uniform_cloud_problem(200, 300, 3, seed=3)
  eps = epsilon_scheduler.Epsilon(target=0.01, init=20.0, decay=0.8)
  geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                               epsilon=eps)
  out = linear.solve(geom, torch.as_tensor(a).cuda(), torch.as_tensor(b).cuda())
  ref = oracle.solve(x, y, a, b, epsilon=0.01, eps_init=20.0, eps_decay=0.8)
  helpers.assert_parity(geom, out, ref)


def test_warm_restart_converges_in_one_block():
  """sinkhorn_test.py:491-546: restarting from (f, g) stops after one block
  with a smaller error."""
  x, y, a, b = problems.ref_test_problem()
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.1, threshold=1e-3)
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers.linear import sinkhorn
  prob = linear_problem.LinearProblem(geom, out.a, out.b)
  out2 = sinkhorn.Sinkhorn(threshold=1e-3)(prob, init=(out.f, out.g))
  assert out2.n_iters == 10
  e1 = out.errors.cpu().numpy()
  e2 = out2.errors.cpu().numpy()
  assert e2[0] < e1[e1 > -1][-1]


def test_default_epsilon_std_and_scale_mean():
  x, y, a, b = problems.uniform_cloud_problem(300, 200, 5, seed=5)
  geom, out = helpers.gpu_solve(x, y, a, b)  # epsilon = 0.05 * std(C)
  ref = helpers.oracle_solve(x, y, a, b)
  np.testing.assert_allclose(geom.epsilon, ref.epsilon, rtol=1e-6)
  helpers.assert_parity(geom, out, ref)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.1, relative_epsilon="mean",
                                scale_cost="mean")
  ref = helpers.oracle_solve(x, y, a, b, epsilon=0.1, relative_epsilon="mean",
                             scale_cost="mean")
  helpers.assert_parity(geom, out, ref)


def test_uniform_default_marginals_and_self_cloud():
  x, _, _, _ = problems.uniform_cloud_problem(400, 400, 2, seed=7)
  geom, out = helpers.gpu_solve(x, None, None, None, epsilon=0.01)
  ref = helpers.oracle_solve(x, None, None, None, epsilon=0.01)
  helpers.assert_parity(geom, out, ref)


def test_batched_matches_single():
  """One persistent launch over uneven problems equals one solve each."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  probs = problems.batched_uneven_problems(12, d=8, lo=16, hi=700, seed=1)
  geoms = [pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                                 epsilon=0.05, relative_epsilon="mean")
           for x, y, _, _ in probs]
  outs = linear.solve_batch(geoms, [torch.as_tensor(p[2]).cuda() for p in probs],
                            [torch.as_tensor(p[3]).cuda() for p in probs])
  for (x, y, a, b), geom, out in zip(probs, geoms, outs):
    ref = helpers.oracle_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean")
    helpers.assert_parity(geom, out, ref)


def test_device_wait_timeout_reports_status():
  """A grid barrier waiting for arrivals that never come gives up after its
  time limit and reports OTTB_ERR_TIMEOUT; the context stays usable."""
  import torch
  from ott_b200 import _lib
  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers.linear import sinkhorn
  x, y, a, b = problems.ref_test_problem()
  geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                               epsilon=0.1)
  solver = sinkhorn.Sinkhorn(timeout_ms=200)
  solver._phantom_arrivals = 1
  out = solver(linear_problem.LinearProblem(geom, torch.as_tensor(a).cuda(),
                                            torch.as_tensor(b).cuda()))
  with pytest.raises(_lib.OttbError) as e:
    _ = out.n_iters
  assert e.value.status == _lib.OTTB_ERR_TIMEOUT
  geom2, out2 = helpers.gpu_solve(x, y, a, b, epsilon=0.1)
  assert out2.converged


def test_diag_sum_of_self_transport():
  """The reference's test_diag_sum (tests/solvers/linear/sinkhorn_test.py:
  56-66): a cloud against itself at epsilon = 0.01 keeps more than 99 % of
  the mass on the diagonal of the plan, and less than all of it (on a draw
  whose points are at least 0.3 apart: a closer pair, cost ~ epsilon,
  shares its mass, in the oracle as here), equal to the oracle's sum."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  x = np.random.default_rng(0).uniform(size=(17, 4)).astype(np.float32)
  out = linear.solve(pointcloud.PointCloud(torch.as_tensor(x).cuda(), epsilon=0.01))
  s = float(out.diag.sum())
  assert 0.99 < s < 1.0
  x64 = x.astype(np.float64)
  ref = o.solve(x64, None, epsilon=0.01)
  want = np.trace(o.transport_matrix(ref.f, ref.g, o.Geom(x64, x64, 0.01)))
  assert abs(s - want) <= 1e-5


def test_low_epsilon_plan_matches_assignment():
  """The reference's test_SqEucl_matches_hungarian (sinkhorn_test.py:68-90,
  n = 17, d = 4): at epsilon = 0.01 the plan is within cosine distance 0.2
  of the optimal assignment's (scipy's linear_sum_assignment on the cost),
  and that distance equals the oracle plan's."""
  import torch
  from scipy.optimize import linear_sum_assignment
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  rng = np.random.default_rng(17)
  n = 17
  x = rng.uniform(size=(n, 4)).astype(np.float32)
  y = rng.uniform(size=(n, 4)).astype(np.float32)
  geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                               epsilon=0.01)
  p = linear.solve(geom).matrix.cpu().numpy().astype(np.float64).ravel()
  rows, cols = linear_sum_assignment(geom.cost_matrix.cpu().numpy())
  h = np.zeros((n, n))
  h[rows, cols] = 1.0 / n
  h = h.ravel()
  cosd = lambda u, v: 1.0 - u @ v / (np.linalg.norm(u) * np.linalg.norm(v))
  assert cosd(p, h) < 0.2
  x64, y64 = x.astype(np.float64), y.astype(np.float64)
  ref = o.solve(x64, y64, epsilon=0.01)
  p_ref = o.transport_matrix(ref.f, ref.g, o.Geom(x64, y64, 0.01)).ravel()
  assert abs(cosd(p, h) - cosd(p_ref, h)) <= 1e-4


def test_progress_callbacks():
  """The reference's test_custom_progress_fn and test_progress_fn
  (sinkhorn_test.py:658-749): called on iterations 9, 19, 29 with
  decreasing errors and the iteration budget; default_progress_fn prints
  "foo 7/14" first."""
  import io
  import torch
  from ott_b200 import utils
  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers import linear
  from ott_b200.solvers.linear import sinkhorn
  x, y, a, b = problems.ref_test_problem()
  traced = {"iters": [], "error": [], "total": []}

  def progress_fn(status):
    iteration, inner, total, state = status
    errors = state.errors.cpu().numpy().ravel()
    if (int(iteration) + 1) % int(inner) == 0:
      traced["iters"].append(int(iteration))
      traced["error"].append(errors[max((int(iteration) + 1) // int(inner) - 1, 0)])
      traced["total"].append(int(total))

  geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                               epsilon=1e-3)
  prob = linear_problem.LinearProblem(geom, torch.as_tensor(a).cuda(), torch.as_tensor(b).cuda())
  sinkhorn.Sinkhorn(progress_fn=progress_fn, max_iterations=30, inner_iterations=10)(prob)
  assert traced["iters"] == [9, 19, 29]
  assert np.all(np.diff(traced["error"]) < 0)
  assert traced["total"] == [30, 30, 30]
  stream = io.StringIO()
  geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                               epsilon=1e-1)
  linear.solve(geom, progress_fn=utils.default_progress_fn(fmt="foo {iter}/{max_iter}",
                                                          stream=stream),
               min_iterations=0, inner_iterations=7, max_iterations=14)
  assert stream.getvalue().startswith("foo 7/14"), stream.getvalue()


def test_progress_callbacks_run_while_the_solve_runs():
  """progress_fn is called live, from the errors the persistent kernel
  writes into pinned host memory at each block's end (the reference calls
  it from inside its loop, sinkhorn.py:933-937): the first calls come
  while the solve's stream is still busy, every block is reported once and
  in order, each call's state holds that block's error, and the output's
  errors (device) equal what the calls saw."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  n, d = 16384, 64
  x, y, _, _ = problems.gaussian_shift_problem(n, n, d, seed=4)
  geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                               epsilon=0.002, relative_epsilon="mean")
  calls = []

  def progress_fn(status):
    iteration, inner, total, state = status
    blk = (int(iteration) + 1) // int(inner) - 1
    calls.append((int(iteration), float(state.errors[blk]),
                  bool(torch.cuda.current_stream().query())))

  out = linear.solve(geom, progress_fn=progress_fn, threshold=1e-12, inner_iterations=10,
                     max_iterations=600)
  assert [c[0] for c in calls] == [10 * k + 9 for k in range(60)]
  assert not calls[0][2], "the first call came after the solve had finished"
  errs = out.errors.cpu().numpy()
  np.testing.assert_array_equal(errs, np.array([c[1] for c in calls], dtype=np.float32))
  assert out.n_iters == 600
