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
