"""Epsilon annealing over stages: the schedule (CPU) and the staged solves
against the oracle chained the same way (GPU)."""
import numpy as np
import pytest

from oracle import sinkhorn_np as oracle
from tests import problems


def test_stage_multipliers():
  from ott_b200.solvers.linear import annealing
  m = annealing.stage_multipliers(10, 1.0, 1e-3)
  assert len(m) == 10 and m[0] == 1.0
  np.testing.assert_allclose(m[-1], 1e-3, rtol=1e-12)
  np.testing.assert_allclose(m[1:] / m[:-1], 10 ** (-1 / 3), rtol=1e-12)
  np.testing.assert_array_equal(annealing.stage_multipliers(1, 1.0, 0.01), [0.01])
  with pytest.raises(ValueError):
    annealing.stage_multipliers(0)


@pytest.mark.gpu
@pytest.mark.parametrize("d,precision", [(16, "fp32"), (32, "auto")])
def test_annealed_stages_match_oracle(d, precision):
  """Two pairs, 4 stages from 1 to 1e-2 mean(C): per-stage iteration counts
  and final potentials as the oracle solving the same chain in float64."""
  import torch
  from ott_b200.solvers.linear import annealing
  pairs = [problems.gmm8_pair(300, 257, d, seed=s) for s in (1, 2)]
  xs = [torch.tensor(p[0]).cuda() for p in pairs]
  ys = [torch.tensor(p[1]).cuda() for p in pairs]
  out = annealing.solve_annealed(xs, ys, stages=4, start=1.0, final=1e-2,
                                 precision=precision, fallback_precision=None)
  assert not out.fallbacks
  for k, (x, y, a, b) in enumerate(pairs):
    xd, yd = x.astype(np.float64), y.astype(np.float64)
    mean_c = oracle.mean_cost_matrix(xd, yd)
    init = None
    for s, mult in enumerate(annealing.stage_multipliers(4, 1.0, 1e-2)):
      geom = oracle.Geom(xd, yd, float(mult * mean_c))
      ref = oracle.sinkhorn(geom, a, b, init=init)
      init = (ref.f, ref.g)
      assert abs(int(out.stage_iters[s, k]) - ref.n_iters) <= 10, (s, k)
      np.testing.assert_allclose(out.stage_epsilons[s, k], geom.epsilon, rtol=1e-6)
    o = out.outputs[k]
    assert o.converged
    eps = out.stage_epsilons[-1, k]
    f = o.f.cpu().numpy().astype(np.float64)
    g = o.g.cpu().numpy().astype(np.float64)
    # Over a chain of ~120 iterations, FP32 rounding moves (f, g) along the
    # direction (f + c, g - c) that leaves the transport plan unchanged: the
    # float32 oracle itself drifts by up to 4.6e-4 eps from float64 on these
    # chains. The drift c is bounded; the potentials match after removing it.
    # float32 storage of O(mean C) potentials adds ~1e-7 of their size.
    tol = 1e-4 * eps + 1e-6 * np.abs(ref.f).max()
    if d >= 32:
      # bf16 split-3 products: x = hi + lo + r with |r_k| <= 2^-18 |x_k|, and
      # lo*lo is dropped, so each <x, y> is off by at most 3 * 2^-18 sum_k
      # |x_k y_k| <= 3 * 2^-18 |x| |y| (centred clouds); a cost entry by twice
      # that. Entries err with both signs and the LSE averages them: the
      # typical (RMS) potential error stays within 1e-4 eps, the largest
      # within the per-entry bound.
      ctr = 0.5 * (xd.mean(0) + yd.mean(0))
      nx = np.linalg.norm(xd - ctr, axis=1).max()
      ny = np.linalg.norm(yd - ctr, axis=1).max()
      tol_max = tol + 6 * 2.0 ** -18 * nx * ny
    else:
      tol_max = tol
    if int(out.stage_iters[-1, k]) == ref.n_iters:
      c = float(np.sum(a.astype(np.float64) * (f - ref.f)))
      assert abs(c) <= 1e-3 * eps, c / eps
      np.testing.assert_allclose(f - c, ref.f, rtol=0, atol=tol_max)
      np.testing.assert_allclose(g + c, ref.g, rtol=0, atol=tol_max)
      assert np.sqrt(np.mean((f - c - ref.f) ** 2)) <= tol
      assert np.sqrt(np.mean((g + c - ref.g) ** 2)) <= tol
      np.testing.assert_allclose(o.reg_ot_cost, ref.reg_ot_cost, rtol=1e-5)


def test_stage_features_cpu():
  """The predictor's features: centred changes in units of the next epsilon
  and their linear extrapolation in epsilon."""
  import torch
  from ott_b200.solvers.linear import annealing
  f0 = torch.tensor([0.0, 1.0, 2.0, 3.0])
  f1 = f0 + torch.tensor([0.5, -0.5, 0.25, 0.0])
  f2 = f1 + torch.tensor([0.2, 0.1, -0.3, 0.0])
  eps = [1.0, 0.5]
  x = annealing.stage_features([f0, f1], eps, 0.25)
  assert x.shape == (4, annealing.FEATURES)
  d1 = (f1 - f0) - (f1 - f0).mean()
  np.testing.assert_allclose(x[:, 1], d1 / 0.25, rtol=1e-6)
  np.testing.assert_allclose(x[:, 0], d1 / 0.25 * (0.25 - 0.5) / (0.5 - 1.0), rtol=1e-6)
  np.testing.assert_allclose(x[:, 2], 0.0)
  x3 = annealing.stage_features([f0, f1, f2], [1.0, 0.5, 0.25], 0.125)
  d2 = (f1 - f0) - (f1 - f0).mean()
  np.testing.assert_allclose(x3[:, 2], d2 / 0.125, rtol=1e-6)
  np.testing.assert_allclose(x3[:, 3], 0.5, rtol=1e-6)
  assert float(x3[:, 6:].abs().max()) == 0.0
  with pytest.raises(ValueError):
    annealing.stage_features([f0], [1.0], 0.5)


@pytest.mark.gpu
def test_learned_stage_warm_start_cuts_iterations():
  """The per-stage learned warm start, trained on annealed chains the plain
  FP32 kernel solved for four pairs of the family, on two held-out pairs:
  fewer stage iterations than starting each stage from the previous stage's
  potentials, the same final reg_ot_cost (1e-4 relative), every pair
  converged."""
  import torch
  from ott_b200.solvers.linear import annealing
  n, d = 2048, 128

  def pairs(seeds):
    ps = [problems.gmm8_pair(n, n, d, seed=s) for s in seeds]
    return [torch.tensor(p[0]).cuda() for p in ps], [torch.tensor(p[1]).cuda() for p in ps]

  xs, ys = pairs([10, 11, 12, 13])
  train = annealing.solve_annealed(xs, ys, precision="fp32", fallback_precision=None,
                                   record_f=True)
  chains = [(train.f_history[k], train.stage_epsilons[:, k]) for k in range(len(xs))]
  pred = annealing.StagePredictor(seed=0)
  losses = pred.fit(chains, steps=1500).cpu().numpy()
  assert losses[-100:].mean() < 0.5 * losses[:20].mean()
  xs, ys = pairs([0, 1])
  prev = annealing.solve_annealed(xs, ys)
  warm = annealing.solve_annealed(xs, ys, warm_start=pred)
  assert all(o.converged for o in prev.outputs) and all(o.converged for o in warm.outputs)
  assert warm.stage_iters.sum() < prev.stage_iters.sum(), (warm.stage_iters, prev.stage_iters)
  for o1, o2 in zip(prev.outputs, warm.outputs):
    np.testing.assert_allclose(o2.reg_ot_cost, o1.reg_ot_cost, rtol=1e-4)
