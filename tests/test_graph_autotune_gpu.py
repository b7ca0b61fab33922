"""Replays of a solve captured in a CUDA graph (ottb_sinkhorn_prepare once,
ottb_sinkhorn_launch captured) and autotuned work schedules
(ottb_sinkhorn_autotune).

A replay runs the same kernels with the same schedule as a direct call, so
its results are bit-identical to the direct solve, also after new inputs are
copied into the captured tensors. Autotuned schedules change only how the
work is split, so the results keep the path's parity tolerances against the
float64 oracle.
"""
import numpy as np
import pytest

from tests import helpers, problems

pytestmark = pytest.mark.gpu


def _problems(specs, d, eps, seed):
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  out, raw = [], []
  for k, (n, m) in enumerate(specs):
    x, y, a, b = problems.uniform_cloud_problem(n, m, d, seed=seed + k)
    geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                                 epsilon=eps)
    out.append(linear_problem.LinearProblem(geom, torch.as_tensor(a).cuda(),
                                            torch.as_tensor(b).cuda()))
    raw.append((x, y, a, b))
  return out, raw


def _same(o1, o2):
  for u, v in zip(o1, o2):
    np.testing.assert_array_equal(u.f.cpu().numpy(), v.f.cpu().numpy())
    np.testing.assert_array_equal(u.g.cpu().numpy(), v.g.cpu().numpy())
    np.testing.assert_array_equal(u.errors.cpu().numpy(), v.errors.cpu().numpy())
    assert u.n_iters == v.n_iters
    assert u.reg_ot_cost == v.reg_ot_cost


@pytest.mark.parametrize("d,precision,specs", [
    (3, "fp32", [(300, 257)]),
    (64, "bf16_split3", [(500, 700), (130, 90), (260, 400)]),
])
def test_graph_replay_matches_direct_solve(d, precision, specs):
  from ott_b200.solvers.linear import sinkhorn
  solver = sinkhorn.Sinkhorn(precision=precision)
  probs, _ = _problems(specs, d, 0.05, seed=11)
  direct = sinkhorn.run_batch(probs, solver)
  graph = sinkhorn.SinkhornGraph(probs, solver)
  _same(graph.replay(), direct)
  _same(graph.replay(), direct)  # replays restore the header every time

  # new inputs copied into the captured tensors, same shapes and epsilon
  import torch
  fresh, raw = _problems(specs, d, 0.05, seed=99)
  for p, (x, y, a, b) in zip(probs, raw):
    p.geom.x.copy_(torch.as_tensor(x))
    p.geom.y.copy_(torch.as_tensor(y))
    p.a.copy_(torch.as_tensor(a))
    p.b.copy_(torch.as_tensor(b))
  replayed = graph.replay()
  _same(replayed, sinkhorn.run_batch(fresh, solver))
  for out, (x, y, a, b) in zip(replayed, raw):
    ref = helpers.oracle_solve(x, y, a, b, epsilon=0.05)
    assert abs(out.n_iters - ref.n_iters) <= out.inner_iterations
    np.testing.assert_allclose(out.reg_ot_cost, ref.reg_ot_cost, rtol=1e-4)


def test_autotuned_single_problem_keeps_parity():
  """One problem (shape used by no other test): the tuned schedule (column
  split x1/2, x1 or x2; round-robin or queued units) leaves the results at
  the FP32 path's tolerances."""
  from ott_b200.solvers.linear import sinkhorn
  x, y, a, b = problems.uniform_cloud_problem(1531, 1707, 5, seed=3)
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                               epsilon=0.05)
  prob = linear_problem.LinearProblem(geom, torch.as_tensor(a).cuda(), torch.as_tensor(b).cuda())
  solver = sinkhorn.Sinkhorn(precision="fp32", autotune=True)
  out = solver(prob)
  ref = helpers.oracle_solve(x, y, a, b, epsilon=0.05)
  helpers.assert_parity(geom, out, ref)
  again = solver(prob)  # the cached schedule, no trials
  np.testing.assert_allclose(again.reg_ot_cost, out.reg_ot_cost, rtol=0, atol=0)


def test_autotuned_batch_keeps_parity():
  """Several uneven problems on the tensor cores: the tuned growth of the
  column splits as problems converge leaves every problem within the
  mixed-precision tolerances."""
  from ott_b200.solvers.linear import sinkhorn
  specs = [(1200, 900), (70, 1500), (333, 333), (2049, 100), (640, 641)]
  probs, raw = _problems(specs, 40, 0.05, seed=21)
  outs = sinkhorn.run_batch(probs, sinkhorn.Sinkhorn(precision="bf16_split3", autotune=True))
  for out, (x, y, a, b) in zip(outs, raw):
    ref = helpers.oracle_solve(x, y, a, b, epsilon=0.05)
    assert abs(out.n_iters - ref.n_iters) <= out.inner_iterations
    np.testing.assert_allclose(out.reg_ot_cost, ref.reg_ot_cost, rtol=1e-4)


@pytest.mark.parametrize("specs", [[(1000, 1100)], [(300, 200), (129, 700), (900, 400)]])
def test_tile_128_keeps_parity(specs):
  """The 128-column tensor-core tile (four accumulators), pinned with
  ottb_sinkhorn_set_schedule, keeps the tensor-core path's parity bars
  against the float64 oracle, single and batched; its results equal the
  256-column tile's within those bars."""
  from ott_b200.solvers.linear import sinkhorn
  probs, raw = _problems(specs, 64, 0.05, seed=40)
  solver = sinkhorn.Sinkhorn(precision="bf16_split3")
  wide = sinkhorn.run_batch(probs, solver)
  sinkhorn.set_schedule(probs, solver, waves=2, dynamic=1 if len(specs) > 1 else 0,
                        tile_n=128)
  narrow = sinkhorn.run_batch(probs, solver)
  for (x, y, a, b), o, w, p in zip(raw, narrow, wide, probs):
    ref = helpers.oracle_solve(x, y, a, b, epsilon=0.05)
    helpers.assert_parity(p.geom, o, ref, pot_tol=1e-3, cost_rtol=1e-4, iter_blocks=1,
                          err_rtol=1e-2, err_atol=2e-3)
    np.testing.assert_allclose(o.reg_ot_cost, w.reg_ot_cost, rtol=1e-4)
  # restore the default schedule for these shapes
  sinkhorn.set_schedule(probs, solver, waves=2, dynamic=1 if len(specs) > 1 else 0,
                        tile_n=256)


def test_set_schedule_rejects_bad_values():
  from ott_b200 import _lib
  from ott_b200.solvers.linear import sinkhorn
  probs, _ = _problems([(200, 300)], 64, 0.05, seed=50)
  solver = sinkhorn.Sinkhorn(precision="bf16_split3")
  for kw in (dict(tile_n=64), dict(split_scale=0), dict(waves=-1), dict(dynamic=2)):
    with pytest.raises(_lib.OttbError):
      sinkhorn.set_schedule(probs, solver, **kw)
