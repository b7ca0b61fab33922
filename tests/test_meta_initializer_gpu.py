"""The learned warm start on the GPU: the tcgen05 MLP kernels against the
float64 network oracle (forward, gradients, Adam), the f half-update from an
initial g against the Sinkhorn oracle, and a trained network cutting the
iterations of the plain solver at equal accuracy (the reference's
tests/initializers/neural/meta_initializer_test.py:62-93 asks the same of its
MetaInitializer)."""
import numpy as np
import pytest

from oracle import mlp_np
from oracle import sinkhorn_np as oracle
from tests import problems

pytestmark = pytest.mark.gpu


def _mlp(dims, seed):
  from ott_b200.initializers.neural import meta_initializer
  return meta_initializer.MLP(dims, seed=seed)


def _rel(a, b):
  return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_mlp_forward_matches_oracle():
  import torch
  net = _mlp([256, 384, 256, 128], seed=1)
  x = np.random.default_rng(0).standard_normal((256, 256)).astype(np.float32)
  y = net.forward(torch.tensor(x, device="cuda")).cpu().numpy()
  net.check_status()
  params = net.params_numpy()
  y_emul, _ = mlp_np.forward_bf16(params, x)
  y_exact, _ = mlp_np.forward(params, x.astype(np.float64))
  # same roundings as the device: only summation order and tanh differ
  assert _rel(y, y_emul) < 2e-3
  # against float64 weights and activations: bf16 operand error
  assert _rel(y, y_exact) < 2e-2


@pytest.mark.parametrize("weighted", [False, True])
def test_mlp_gradients_match_oracle(weighted):
  import torch
  dims = [256, 256, 128, 128]
  net = _mlp(dims, seed=2)
  rng = np.random.default_rng(1)
  batch = 384
  x = rng.standard_normal((batch, 256)).astype(np.float32)
  t = rng.standard_normal((batch, 128)).astype(np.float32)
  w = rng.uniform(0.05, 2.0, size=(batch, 128)).astype(np.float32) if weighted else None
  loss = net.gradients(torch.tensor(x, device="cuda"), torch.tensor(t, device="cuda"),
                       None if w is None else torch.tensor(w, device="cuda"))
  loss = loss.cpu().numpy()
  net.check_status()
  params = net.params_numpy()
  bparams = [(mlp_np.bf16(wt).astype(np.float64), b) for wt, b in params]
  loss_ref, grads = mlp_np.loss_and_grads(bparams, mlp_np.bf16(x).astype(np.float64),
                                          t.astype(np.float64), w)
  np.testing.assert_allclose(loss, loss_ref, rtol=2e-2)
  for l, tens in enumerate(net.tensors):
    gw = tens["w_grad"].cpu().numpy()
    gb = tens["b_grad"].cpu().numpy()
    # bf16 activations and bf16 output gradient, FP32 accumulation
    assert _rel(gw, grads[l][0]) < 3e-2, (l, _rel(gw, grads[l][0]))
    assert _rel(gb, grads[l][1]) < 3e-2, (l, _rel(gb, grads[l][1]))


@pytest.mark.parametrize("batch,width,tile", [(512, 1024, 32), (768, 1024, 64),
                                              (1536, 1024, 128)])
def test_mlp_gradients_every_tile_width(batch, width, tile):
  """The GEMMs' tile width (128, 64 or 32 columns, the widest giving 96 or
  more CTAs) follows M N: the layer GEMMs of these shapes take the given
  width for the forward and data-gradient products (M = batch, N =
  width). Forward output and every gradient against the float64 oracle on
  the same bf16 operands."""
  import torch
  tiles128 = (batch // 128) * (width // 128)
  assert (128 if tiles128 >= 96 else 64 if 2 * tiles128 >= 96 else 32) == tile
  dims = [256, width, 128]
  net = _mlp(dims, seed=4)
  rng = np.random.default_rng(5)
  x = rng.standard_normal((batch, 256)).astype(np.float32)
  t = rng.standard_normal((batch, 128)).astype(np.float32)
  loss = net.gradients(torch.tensor(x, device="cuda"), torch.tensor(t, device="cuda"), None)
  loss = loss.cpu().numpy()
  net.check_status()
  params = net.params_numpy()
  bparams = [(mlp_np.bf16(wt).astype(np.float64), b) for wt, b in params]
  loss_ref, grads = mlp_np.loss_and_grads(bparams, mlp_np.bf16(x).astype(np.float64),
                                          t.astype(np.float64), None)
  np.testing.assert_allclose(loss, loss_ref, rtol=2e-2)
  for l, tens in enumerate(net.tensors):
    assert _rel(tens["w_grad"].cpu().numpy(), grads[l][0]) < 3e-2, l
    assert _rel(tens["b_grad"].cpu().numpy(), grads[l][1]) < 3e-2, l
  y = net.forward(torch.tensor(x, device="cuda")).cpu().numpy()
  y_emul, _ = mlp_np.forward_bf16(params, x)
  assert _rel(y, y_emul) < 2e-3


def test_fit_graph_replay_matches_direct_steps():
  """meta_initializer.fit with the training step captured in a CUDA graph
  (device step counter, device Adam schedule) against the direct loop on
  the same data and minibatches: the same kernels on the same values, so
  the same losses and weights."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.initializers.neural import meta_initializer
  grid = problems.grid_support(16)
  geom = pointcloud.PointCloud(torch.tensor(grid).cuda(), epsilon=1e-2)
  W = problems.grid_mixture_weights(2 * 640, grid, seed=3, device="cuda")
  A, B = W[0::2].contiguous(), W[1::2].contiguous()
  G = torch.randn(A.shape, device="cuda") * 1e-2
  res = []
  for graph in (False, True):
    meta = meta_initializer.MetaInitializer(geom, dims=(256,), seed=7)
    losses = meta_initializer.fit(meta, A, B, G, steps=25, batch_size=128, graph=graph)
    res.append((losses.cpu().numpy(), [t["w"].cpu().numpy() for t in meta.mlp.tensors],
                meta.mlp.step))
  (l0, w0, s0), (l1, w1, s1) = res
  assert s0 == s1 == 25
  np.testing.assert_array_equal(l1, l0)
  for u, v in zip(w1, w0):
    np.testing.assert_array_equal(u, v)


def test_mlp_adam_step_matches_oracle():
  import torch
  net = _mlp([128, 256, 128], seed=3)
  rng = np.random.default_rng(2)
  x = torch.tensor(rng.standard_normal((128, 128)).astype(np.float32), device="cuda")
  t = torch.tensor(rng.standard_normal((128, 128)).astype(np.float32), device="cuda")
  params = net.params_numpy()
  state = [[np.zeros_like(w), np.zeros_like(w), np.zeros_like(b), np.zeros_like(b)]
           for w, b in params]
  for step in (1, 2, 3):
    net.gradients(x, t)
    grads = [(tn["w_grad"].double().cpu().numpy(), tn["b_grad"].double().cpu().numpy())
             for tn in net.tensors]
    net.adam(lr=1e-3)
    params = mlp_np.adam_step(params, grads, state, step, lr=1e-3)
    got = net.params_numpy()
    for (w, b), (w_ref, b_ref) in zip(got, params):
      np.testing.assert_allclose(w, w_ref, rtol=0, atol=1e-6)
      np.testing.assert_allclose(b, b_ref, rtol=0, atol=1e-6)
  net.check_status()
  for tn in net.tensors:  # bf16 copies refreshed from the FP32 weights
    wb = tn["w_bf16"].float().cpu().numpy()
    np.testing.assert_array_equal(wb, mlp_np.bf16(tn["w"].cpu().numpy()))
    np.testing.assert_array_equal(tn["wt_bf16"].float().cpu().numpy(), wb.T)


@pytest.mark.parametrize("n,m,d,precision", [(200, 300, 2, "fp32"), (300, 257, 64, "auto")])
def test_f_from_g_matches_oracle(n, m, d, precision):
  """init (f, g) = (c-transform of g0, g0): one f-update before the loop."""
  import torch
  from ott_b200.solvers import linear
  from ott_b200.geometry import pointcloud
  x, y, a, b = problems.uniform_cloud_problem(n, m, d, seed=n + d)
  rng = np.random.default_rng(7)
  g0 = (0.3 * rng.standard_normal(m)).astype(np.float32)
  geom = pointcloud.PointCloud(torch.tensor(x).cuda(), torch.tensor(y).cuda(), epsilon=0.05,
                               relative_epsilon="mean")
  out = linear.solve_batch([geom], [torch.tensor(a).cuda()], [torch.tensor(b).cuda()],
                           init=[(None, torch.tensor(g0).cuda())], f_from_g=True,
                           precision=precision)[0]
  xd, yd = x.astype(np.float64), y.astype(np.float64)
  eps = oracle.resolve_epsilon(xd, yd, 0.05, "mean", 1.0)
  og = oracle.Geom(xd, yd, float(eps))
  f0 = og.update_potential(np.zeros(n), g0.astype(np.float64), np.log(a.astype(np.float64)),
                           0, axis=1)
  ref = oracle.sinkhorn(og, a, b, init=(f0, g0.astype(np.float64)))
  from tests import helpers
  helpers.assert_parity(geom, out, ref)


def test_run_stacked_matches_run_batch():
  """The array-filled problem records give the per-problem path's results."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers.linear import sinkhorn
  grid = problems.grid_support(16)
  W = torch.tensor(problems.grid_mixture_weights(12, grid, seed=5)).cuda()
  geom = pointcloud.PointCloud(torch.tensor(grid).cuda(), epsilon=1e-2)
  A, B = W[0::2], W[1::2]
  st = sinkhorn.run_stacked(geom, A, B, sinkhorn.Sinkhorn())
  outs = sinkhorn.run_batch([linear_problem.LinearProblem(geom, A[k], B[k]) for k in range(6)],
                            sinkhorn.Sinkhorn())
  n_it, conv, cost = st.scalars()
  for k, o in enumerate(outs):
    assert n_it[k] == o.n_iters and conv[k] == o.converged
    assert cost[k] == o.reg_ot_cost
    torch.testing.assert_close(st.f[k], o.f, rtol=0, atol=0)
    torch.testing.assert_close(st.g[k], o.g, rtol=0, atol=0)


def test_trained_warm_start_cuts_iterations():
  """A 16 x 16 grid (n = m = 256, eps 1e-2), measures as in the 32 x 32
  learned-warm-start workload; the network is trained for 1500 Adam steps on
  16384 problems solved by the plain kernel, then warm-starts 256 held-out
  problems. Both runs converge to the same threshold; the costs agree to the
  accuracy the threshold allows."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.initializers.neural import meta_initializer
  from ott_b200.solvers.linear import sinkhorn
  grid = problems.grid_support(16)
  ntr = 16384
  W = problems.grid_mixture_weights(2 * (ntr + 256), grid, seed=11, device="cuda")
  A, B = W[0::2].contiguous(), W[1::2].contiguous()
  geom = pointcloud.PointCloud(torch.tensor(grid).cuda(), epsilon=1e-2)
  solved = sinkhorn.run_stacked(geom, A[:ntr], B[:ntr], sinkhorn.Sinkhorn())
  assert solved.converged.all()

  meta = meta_initializer.MetaInitializer(geom, dims=(512, 512), lr=1e-3, seed=0)
  losses = meta_initializer.fit(meta, A[:ntr], B[:ntr], solved.g, steps=1500, batch_size=512)
  meta.mlp.check_status()
  losses = losses.cpu().numpy()
  assert losses[-50:].mean() < 0.1 * losses[:10].mean(), (losses[:10].mean(), losses[-50:])

  cold = sinkhorn.run_stacked(geom, A[ntr:], B[ntr:], sinkhorn.Sinkhorn())
  warm, redo = meta_initializer.solve_warm_started(geom, A[ntr:], B[ntr:], meta)
  it_cold, conv_cold, c_cold = cold.scalars()
  it_warm, conv_warm, c_warm = warm.scalars()
  assert conv_cold.all() and conv_warm.all()
  print(f"iterations: cold {it_cold.mean():.1f}, warm {it_warm.mean():.1f}, "
        f"fallbacks {len(redo)}, loss {losses[:10].mean():.3e} -> {losses[-50:].mean():.3e}")
  assert it_warm.mean() < 0.8 * it_cold.mean()
  np.testing.assert_allclose(c_warm, c_cold, rtol=1e-3)


def test_warm_start_fallback_restores_default_init():
  """A budget too small for the warm start: every problem falls back to the
  default initialisation and ends with the plain solver's result."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.initializers.neural import meta_initializer
  from ott_b200.solvers.linear import sinkhorn
  grid = problems.grid_support(16)
  W = torch.tensor(problems.grid_mixture_weights(16, grid, seed=9)).cuda()
  A, B = W[0::2], W[1::2]
  geom = pointcloud.PointCloud(torch.tensor(grid).cuda(), epsilon=1e-2)
  meta = meta_initializer.MetaInitializer(geom, dims=(256,), seed=1)  # untrained
  out, redo = meta_initializer.solve_warm_started(geom, A, B, meta, budget=10)
  plain = sinkhorn.run_stacked(geom, A, B, sinkhorn.Sinkhorn())
  n_it, conv, cost = out.scalars()
  n0, c0, cost0 = plain.scalars()
  assert len(redo) == 8 and conv.all()
  np.testing.assert_array_equal(n_it, n0 + 10)
  np.testing.assert_array_equal(cost, cost0)
  torch.testing.assert_close(out.g, plain.g, rtol=0, atol=0)
