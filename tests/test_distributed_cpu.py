"""The multi-process host logic on the CPU: two gloo ranks (one process per
GPU in production, NCCL there) partition independent problems, reduce
timings and gather per-problem scalars."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ott_b200 import distributed as odist


def test_shard_bounds_cover_balance_and_order():
  work = [float(n * m) for n, m in [(128, 300), (16384, 16384), (500, 700), (9000, 128),
                                    (2000, 2000), (128, 128), (16000, 4000)]]
  for world in (1, 2, 3, 4, 8, 12):
    b = odist.shard_bounds(work, world)
    assert len(b) == world and b[0][0] == 0 and b[-1][1] == len(work)
    assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
    assert all(lo <= hi for lo, hi in b)
  # equal work splits evenly
  assert odist.shard_bounds([1.0] * 10, 2) == [(0, 5), (5, 10)]
  assert odist.shard_bounds([1.0] * 3, 4)[-1][1] == 3
  assert odist.shard_bounds([], 3) == [(0, 0)] * 3
  # the heavy problem sits alone when it carries most of the work
  b = odist.shard_bounds([1.0, 1.0, 100.0, 1.0, 1.0], 3)
  assert [hi - lo for lo, hi in b].count(1) >= 1


def _free_port():
  with socket.socket() as s:
    s.bind(("127.0.0.1", 0))
    return s.getsockname()[1]


def _worker(rank, world, port, q):
  os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
  dist.init_process_group("gloo", rank=rank, world_size=world)
  try:
    r, w = odist.rank_and_world()
    mx = odist.max_over_ranks(1.5 + rank)
    sm = odist.sum_over_ranks(2.0 * (rank + 1))
    bounds = odist.shard_bounds([float(k + 1) for k in range(9)], w)
    lo, hi = bounds[r]
    mine = [float(k * k) for k in range(lo, hi)]
    gathered = odist.all_gather_values(mine)
    # the partition and gather of solve_batch_sharded, its per-rank solve
    # replaced by a fake that records which problems it was given
    from ott_b200.solvers.linear import _solve
    seen = []

    class _Out:
      def __init__(self, k):
        self.reg_ot_cost, self.n_iters, self.converged = 0.5 * k, 10 * k, k % 2 == 0

    def fake_solve_batch(geoms, a, b, **kw):
      seen.extend(g for g in geoms)
      return [_Out(g) for g in geoms]

    _solve.solve_batch = fake_solve_batch
    shapes = [(100 * (k + 1), 50) for k in range(7)]
    makers = [(lambda k=k: k) for k in range(7)]
    res = odist.solve_batch_sharded(makers, shapes=shapes)
    q.put((rank, r, w, mx, sm, gathered, seen, res.bounds, res.reg_ot_cost, res.n_iters,
           res.converged))
  finally:
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_gather():
  ctx = mp.get_context("spawn")
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
  for p in procs:
    p.start()
  res = sorted(q.get(timeout=120) for _ in procs)
  for p in procs:
    p.join(timeout=60)
    assert p.exitcode == 0
  for rank, r, w, mx, sm, gathered, seen, bounds, costs, iters, conv in res:
    assert (r, w) == (rank, 2)
    assert mx == 2.5 and sm == 6.0
    assert gathered == [float(k * k) for k in range(9)]
    assert seen == list(range(*bounds))
    assert costs == [0.5 * k for k in range(7)]
    assert iters == [10 * k for k in range(7)]
    assert conv == [k % 2 == 0 for k in range(7)]
  assert res[0][7][1] == res[1][7][0] and res[1][7][1] == 7 and res[0][7][0] == 0
  assert res[0][7][1] - res[0][7][0] > 0 and res[1][7][1] - res[1][7][0] > 0


def test_single_process_defaults():
  assert odist.rank_and_world() == (0, 1)
  assert odist.max_over_ranks(3.0) == 3.0
  assert odist.all_gather_values([1, 2]) == [1.0, 2.0]


def _sharded_case(seed=0, n=37, m=23, d=3, zero_w=False):
  import numpy as np
  rng = np.random.default_rng(seed)
  x = rng.uniform(size=(n, d))
  y = rng.uniform(size=(m, d))
  a = rng.uniform(0.2, 1.2, n)
  b = rng.uniform(0.2, 1.2, m)
  if zero_w:
    a[[2, 30]] = 0.0
    b[5] = 0.0
  return x, y, a / a.sum(), b / b.sum()


def _oracle_lse(x_shard, y, eps):
  """float64 stand-in for the per-rank kernel (ottb_apply_lse_kernel)."""
  import numpy as np
  from oracle import sinkhorn_np as o
  c = o.sqeuclidean_all_pairs(np.asarray(x_shard), np.asarray(y))

  def lse(pot, axis):
    p = pot.double().numpy()
    if axis == 0:
      return torch.as_tensor(eps * o.logsumexp((p[:, None] - c) / eps, axis=0))
    return torch.as_tensor(eps * o.logsumexp((p[None, :] - c) / eps, axis=1))
  return lse


def _sharded_solve(rank, world, x, y, a, b, kw, group=None):
  from ott_b200 import distributed as odist
  from ott_b200.solvers.linear import sharded
  from oracle import sinkhorn_np as o
  lo, hi = odist.shard_bounds([1.0] * x.shape[0], world)[rank]
  eps = kw["epsilon"]
  if kw.get("relative_epsilon") == "mean":
    eps = eps * o.mean_cost_matrix(x, y)
  return sharded.solve_sharded(x[lo:hi], y, a[lo:hi], b, lse=_oracle_lse(x[lo:hi], y, eps),
                               group=group, **kw), (lo, hi)


def _sharded_worker(rank, world, port, q, case, kw):
  os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
  dist.init_process_group("gloo", rank=rank, world_size=world)
  try:
    x, y, a, b = _sharded_case(**case)
    out, (lo, hi) = _sharded_solve(rank, world, x, y, a, b, kw)
    q.put((rank, lo, hi, out.f.numpy(), out.g.numpy(), out.errors.numpy(), out.n_iters,
           out.reg_ot_cost, out.converged, out.row_offset))
  finally:
    dist.destroy_process_group()


_SHARDED_CASES = [
    (dict(seed=0), dict(epsilon=0.1)),
    (dict(seed=1, zero_w=True), dict(epsilon=0.05, relative_epsilon="mean", threshold=1e-6,
                                      inner_iterations=3)),
    (dict(seed=2), dict(epsilon=0.1, min_iterations=20, max_iterations=20)),
]


def _check_against_oracle(case, kw, f, g, errors, n_iters, cost, converged):
  import numpy as np
  from oracle import sinkhorn_np as o
  x, y, a, b = _sharded_case(**case)
  okw = {k: v for k, v in kw.items() if k not in ("epsilon", "relative_epsilon")}
  ref = o.solve(x, y, a, b, epsilon=kw["epsilon"], relative_epsilon=kw.get("relative_epsilon"),
                **okw)
  assert n_iters == ref.n_iters and converged == ref.converged
  np.testing.assert_array_equal(np.isneginf(f), np.isneginf(ref.f))
  fin = np.isfinite(ref.f)
  np.testing.assert_allclose(f[fin], ref.f[fin], rtol=0, atol=1e-10)
  fin = np.isfinite(ref.g)
  np.testing.assert_allclose(g[fin], ref.g[fin], rtol=0, atol=1e-10)
  np.testing.assert_allclose(errors, ref.errors, rtol=1e-8, atol=1e-14)
  np.testing.assert_allclose(cost, ref.reg_ot_cost, rtol=1e-10)


@pytest.mark.parametrize("case,kw", _SHARDED_CASES)
def test_sharded_solve_single_process_matches_oracle(case, kw):
  x, y, a, b = _sharded_case(**case)
  out, _ = _sharded_solve(0, 1, x, y, a, b, kw)
  _check_against_oracle(case, kw, out.f.numpy(), out.g.numpy(), out.errors.numpy(),
                        out.n_iters, out.reg_ot_cost, out.converged)


@pytest.mark.parametrize("case,kw", _SHARDED_CASES)
def test_sharded_solve_two_gloo_ranks_match_oracle(case, kw):
  """The row-sharded loop over two ranks: column log-sum-exps all-gathered
  and combined, rows updated locally, scalars all-reduced; the result is the
  single-process solve of the whole problem."""
  import numpy as np
  ctx = mp.get_context("spawn")
  q = ctx.Queue()
  port = _free_port()
  procs = [ctx.Process(target=_sharded_worker, args=(r, 2, port, q, case, kw))
           for r in range(2)]
  for p in procs:
    p.start()
  res = sorted((q.get(timeout=180) for _ in procs), key=lambda t: t[0])
  for p in procs:
    p.join(timeout=60)
    assert p.exitcode == 0
  f = np.concatenate([r[3] for r in res])
  assert res[0][1] == 0 and res[0][2] == res[1][1] and res[1][9] == res[0][2]
  for r in res[1:]:  # g, errors and scalars identical on every rank
    np.testing.assert_array_equal(r[4], res[0][4])
    assert r[6] == res[0][6] and r[7] == res[0][7]
  _check_against_oracle(case, kw, f, res[0][4], res[0][5], res[0][6], res[0][7], res[0][8])
