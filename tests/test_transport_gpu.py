"""The plan from the potentials on the GPU (ottb_apply_transport,
ottb_transport_matrix) and the gradient of reg_ot_cost built on it.

Tolerances: applications of the plan within 8 FP32 roundings of the
largest exponent magnitude |f_i + g_j - C_ij| / eps (at least 1e-5) of the
largest output (FP32 inputs, exponentials and sums against the reference's
float64 run: with potentials ~100 eps the inputs' own rounding is ~1e-5
relative); gradients within 1e-4 relative of the float64 oracle's formula
evaluated at the same potentials.
"""
import numpy as np
import pytest

from oracle import sinkhorn_np as o
from tests import golden_cases, helpers, problems

pytestmark = pytest.mark.gpu


def _geom(x, y, eps, **kw):
  import torch
  from ott_b200.geometry import pointcloud
  return pointcloud.PointCloud(torch.as_tensor(x, dtype=torch.float32).cuda(),
                               torch.as_tensor(y, dtype=torch.float32).cuda(), epsilon=eps, **kw)


@pytest.mark.parametrize("name", golden_cases.names())
def test_apply_matches_reference_golden(name):
  """The reference's own SinkhornOutput.apply on its own potentials."""
  import torch
  data, geom_kw, _, _ = golden_cases.load(name, "f64")
  geom = _geom(data["x"], data["y"], float(data["epsilon"]),
               scale_cost=geom_kw.get("scale_cost", 1.0))
  f = torch.as_tensor(data["f"], dtype=torch.float32).cuda()
  g = torch.as_tensor(data["g"], dtype=torch.float32).cuda()
  fin_f, fin_g = data["f"][np.isfinite(data["f"])], data["g"][np.isfinite(data["g"])]
  cmax = o.sqeuclidean_all_pairs(data["x"], data["y"]).max() * o.inv_scale_cost(
      data["x"], data["y"], geom_kw.get("scale_cost", 1.0))
  zmax = (np.abs(fin_f).max() + np.abs(fin_g).max() + cmax) / float(data["epsilon"])
  rel = max(1e-5, 8 * 2.0 ** -24 * zmax)
  for axis, key in ((0, "0"), (1, "1")):
    got = geom.apply_transport_from_potentials(
        f, g, torch.as_tensor(data["vec" + key], dtype=torch.float32).cuda(), axis=axis)
    want = data["apply" + key]
    got = got.cpu().numpy().astype(np.float64)
    for k in range(want.shape[0]):
      scale = np.max(np.abs(want[k]))
      np.testing.assert_allclose(got[k], want[k], rtol=0, atol=rel * scale)


@pytest.mark.parametrize("n,m,d", [(200, 300, 3), (1000, 700, 64), (129, 257, 100)])
def test_matrix_marginals_and_primal_cost(n, m, d):
  from ott_b200.solvers import linear
  import torch
  x, y, a, b = problems.uniform_cloud_problem(n, m, d, seed=n + d)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean")
  f = out.f.cpu().numpy().astype(np.float64)
  g = out.g.cpu().numpy().astype(np.float64)
  og = o.Geom(x.astype(np.float64), y.astype(np.float64), float(geom.epsilon))
  p_ref = o.transport_matrix(f, g, og)
  p = out.matrix.cpu().numpy().astype(np.float64)
  np.testing.assert_allclose(p, p_ref, rtol=2e-4, atol=1e-6 * p_ref.max())
  np.testing.assert_allclose(out.marginal(0).cpu().numpy(), p_ref.sum(0), rtol=1e-4)
  np.testing.assert_allclose(out.marginal(1).cpu().numpy(), p_ref.sum(1), rtol=1e-4)
  cost = np.sum(p_ref * o.sqeuclidean_all_pairs(og.x, og.y))
  np.testing.assert_allclose(out.primal_cost, cost, rtol=1e-4)
  # batched application: [k, n] -> [k, m]
  v = torch.randn(5, n, device="cuda")
  got = out.apply(v, axis=0).cpu().numpy()
  np.testing.assert_allclose(got, v.cpu().numpy().astype(np.float64) @ p_ref, rtol=0,
                             atol=2e-5 * np.abs(v.cpu().numpy() @ p_ref).max())


@pytest.mark.parametrize("scale_cost,rel", [(1.0, None), ("mean", "mean"), (2.5, "std")])
def test_reg_ot_cost_gradients_match_oracle(scale_cost, rel):
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  x, y, a, b = problems.uniform_cloud_problem(300, 400, 8, seed=2)
  a[5] = 0.0
  a /= a.sum()
  xt = torch.as_tensor(x).cuda().requires_grad_()
  yt = torch.as_tensor(y).cuda().requires_grad_()
  at = torch.as_tensor(a).cuda().requires_grad_()
  bt = torch.as_tensor(b).cuda().requires_grad_()
  geom = pointcloud.PointCloud(xt, yt, epsilon=0.05, relative_epsilon=rel, scale_cost=scale_cost)
  cost = linear.reg_ot_cost(geom, at, bt, threshold=1e-6)
  cost.backward()
  out = linear.solve(geom, at, bt, threshold=1e-6)
  f = out.f.detach().cpu().numpy().astype(np.float64)
  g = out.g.detach().cpu().numpy().astype(np.float64)
  og = o.Geom(x.astype(np.float64), y.astype(np.float64), float(geom.epsilon),
              inv_scale=float(geom.inv_scale_cost))
  gx, gy, ga, gb = o.reg_ot_cost_grads(f, g, a.astype(np.float64), b.astype(np.float64), og,
                                       scale_cost_mean=scale_cost == "mean")
  np.testing.assert_allclose(xt.grad.cpu().numpy(), gx, rtol=0, atol=1e-4 * np.abs(gx).max())
  np.testing.assert_allclose(yt.grad.cpu().numpy(), gy, rtol=0, atol=1e-4 * np.abs(gy).max())
  np.testing.assert_allclose(at.grad.cpu().numpy(), ga, rtol=0, atol=1e-4 * np.abs(ga).max())
  np.testing.assert_allclose(bt.grad.cpu().numpy(), gb, rtol=0, atol=1e-4 * np.abs(gb).max())
  assert abs(float(cost.detach()) - out.reg_ot_cost) <= 1e-6 * abs(out.reg_ot_cost)


def test_gradient_of_self_transport_sums_both_roles():
  """PointCloud(x) uses x for rows and columns: autograd adds both."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  x, _, a, _ = problems.uniform_cloud_problem(150, 150, 4, seed=9)
  xt = torch.as_tensor(x).cuda().requires_grad_()
  geom = pointcloud.PointCloud(xt, epsilon=0.1)
  linear.reg_ot_cost(geom, torch.as_tensor(a).cuda(), torch.as_tensor(a).cuda(),
                     threshold=1e-6).backward()
  out = linear.solve(geom, torch.as_tensor(a).cuda(), torch.as_tensor(a).cuda(), threshold=1e-6)
  gx, gy, _, _ = out.reg_ot_cost_grads()
  np.testing.assert_allclose(xt.grad.cpu().numpy(), (gx + gy).cpu().numpy(), rtol=1e-5,
                             atol=1e-7)


@pytest.mark.parametrize("k", [1, 2, 7])
def test_column_splits_match_single_pass(k):
  """The same application with the workspace (column splits, and the
  prepared operands of the pipelined kernels) and without (one pass,
  operands transposed inside the kernel): equal up to FP32 summation
  order."""
  import ctypes
  import torch
  from ott_b200 import _lib
  lib = _lib.load()
  x, y, a, b = problems.uniform_cloud_problem(900, 3000, 16, seed=12)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean")
  n, m, d = 900, 3000, 16
  vec = torch.randn(k, m, device="cuda")
  res = []
  for use_ws in (False, True):
    ws_bytes = lib.ottb_apply_transport_workspace_size(n, m, d, k, 1) if use_ws else 0
    assert (ws_bytes > 0) == use_ws
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device="cuda")
    o = torch.empty(k, n, device="cuda")
    st = lib.ottb_apply_transport(geom.x.data_ptr(), geom.y.data_ptr(), n, m, d,
                                  out.f.data_ptr(), out.g.data_ptr(),
                                  ctypes.c_float(geom.epsilon), ctypes.c_float(1.0),
                                  vec.data_ptr(), k, 1, o.data_ptr(), ws.data_ptr(), ws_bytes,
                                  torch.cuda.current_stream().cuda_stream)
    assert st == 0
    res.append(o.cpu().numpy())
  scale = np.abs(res[0]).max()
  np.testing.assert_allclose(res[1], res[0], rtol=0, atol=1e-5 * scale)


@pytest.mark.parametrize("n,m,d,k", [(130, 5000, 3, 1), (1000, 700, 64, 2), (257, 129, 128, 1),
                                     (5000, 300, 16, 2), (64, 64, 8, 1)])
def test_one_and_two_vector_applications_match_oracle(n, m, d, k):
  """The register path for one or two vectors (column splits when the rows
  alone underfill the GPU) against the float64 plan at the same potentials."""
  import torch
  x, y, a, b = problems.uniform_cloud_problem(n, m, d, seed=n + m + d)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean",
                                precision="fp32")
  f = out.f.cpu().numpy().astype(np.float64)
  g = out.g.cpu().numpy().astype(np.float64)
  og = o.Geom(x.astype(np.float64), y.astype(np.float64), float(geom.epsilon))
  p_ref = o.transport_matrix(f, g, og)
  zmax = (np.abs(f).max() + np.abs(g).max() + og.cost_block().max()) / og.epsilon
  rel = max(1e-5, 8 * 2.0 ** -24 * zmax)
  rng = np.random.default_rng(k)
  for axis in (0, 1):
    vec = rng.standard_normal((k, n if axis == 0 else m))
    got = out.apply(torch.as_tensor(vec, dtype=torch.float32).cuda(), axis=axis)
    want = vec @ p_ref if axis == 0 else vec @ p_ref.T
    for r in range(k):
      np.testing.assert_allclose(got[r].cpu().numpy(), want[r], rtol=0,
                                 atol=rel * np.abs(want[r]).max())


@pytest.mark.parametrize("n,m,d,precision", [(700, 900, 8, "fp32"), (1000, 600, 64, "fp32"),
                                             (1000, 600, 64, "bf16_split3"),
                                             (513, 1500, 40, "bf16_split3"),
                                             (300, 257, 128, "bf16_split3")])
def test_sweep_engine_application_matches_oracle(n, m, d, precision):
  """ottb_apply_transport_sweep (two zero-iteration solves per vector on
  the solver's sweep) against the float64 plan. FP32: the golden
  tolerance. BF16 split-3: its products drop the lo*lo term and the
  inputs' bits below 2^-16, an exponent error up to
  2^-15 * 2 inv |x_i| |y_j| / eps after centring, relative to the sum of
  |P| |v|."""
  import torch
  x, y, a, b = problems.uniform_cloud_problem(n, m, d, seed=n + d)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean",
                                precision="fp32")
  f = out.f.cpu().numpy().astype(np.float64)
  g = out.g.cpu().numpy().astype(np.float64)
  og = o.Geom(x.astype(np.float64), y.astype(np.float64), float(geom.epsilon))
  p_ref = o.transport_matrix(f, g, og)
  if precision == "fp32":
    zmax = (np.abs(f).max() + np.abs(g).max() + og.cost_block().max()) / og.epsilon
    rel = max(1e-5, 8 * 2.0 ** -24 * zmax)
  else:
    c = 0.5 * (x.mean(0) + y.mean(0))
    r = np.linalg.norm(x - c, axis=1).max() * np.linalg.norm(y - c, axis=1).max()
    rel = 2.0 ** -15 * 2 * r / og.epsilon + 1e-5
  rng = np.random.default_rng(d)
  for axis in (0, 1):
    vec = rng.standard_normal((2, n if axis == 0 else m))
    got = geom._apply_raw(out.f, out.g, torch.as_tensor(vec, dtype=torch.float32).cuda(),
                          axis, precision if precision != "fp32" else "sweep_fp32")
    want = vec @ p_ref if axis == 0 else vec @ p_ref.T
    scale = np.abs(vec) @ p_ref if axis == 0 else np.abs(vec) @ p_ref.T
    err = np.abs(got.cpu().numpy() - want)
    assert np.all(err <= rel * scale.max(axis=1, keepdims=True)), (err.max(), rel)


@pytest.mark.parametrize("precision", ["sweep_fp32", "bf16_split3"])
def test_sweep_engine_application_edge_cases(precision):
  """Zero-weight points on both sides (-inf potentials), a vector with zero
  entries and an all-zero vector, three vectors in one launch (six
  zero-iteration problems)."""
  import torch
  n, m, d = 300, 260, 40
  x, y, a, b = problems.uniform_cloud_problem(n, m, d, seed=31)
  a[[0, 7, 150]] = 0.0
  a /= a.sum()
  b[[3, 259]] = 0.0
  b /= b.sum()
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean",
                                precision="fp32")
  f = out.f.cpu().numpy().astype(np.float64)
  g = out.g.cpu().numpy().astype(np.float64)
  assert np.isneginf(f[[0, 7, 150]]).all() and np.isneginf(g[[3, 259]]).all()
  og = o.Geom(x.astype(np.float64), y.astype(np.float64), float(geom.epsilon))
  p_ref = np.nan_to_num(o.transport_matrix(f, g, og))
  c = 0.5 * (x.mean(0) + y.mean(0))
  r = np.linalg.norm(x - c, axis=1).max() * np.linalg.norm(y - c, axis=1).max()
  rel = 2.0 ** -15 * 2 * r / og.epsilon + 1e-5 if precision == "bf16_split3" else 2e-5
  rng = np.random.default_rng(2)
  for axis in (0, 1):
    k = n if axis == 0 else m
    vec = rng.standard_normal((3, k))
    vec[0, ::3] = 0.0
    vec[2] = 0.0
    got = geom._apply_raw(out.f, out.g, torch.as_tensor(vec, dtype=torch.float32).cuda(),
                          axis, precision).cpu().numpy()
    want = vec @ p_ref if axis == 0 else vec @ p_ref.T
    scale = np.abs(vec) @ p_ref if axis == 0 else np.abs(vec) @ p_ref.T
    assert np.isfinite(got).all()
    assert np.all(got[2] == 0.0)
    for i in range(2):
      assert np.all(np.abs(got[i] - want[i]) <= rel * scale[i].max() + 1e-30)


def test_output_members_match_oracle():
  """entropy, normalized_entropy, diag, scalings, transport_mass,
  transport_cost_at_geom and cost_at_geom (sinkhorn.py:395-538) against the
  float64 plan at the GPU's potentials."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  n, d = 300, 5
  x, y, _, _ = problems.uniform_cloud_problem(n, n, d, seed=41)
  geom = pointcloud.PointCloud(torch.as_tensor(x).cuda(), torch.as_tensor(y).cuda(),
                               epsilon=0.05, scale_cost=2.0)
  out = linear.solve(geom, threshold=1e-6, precision="fp32")  # uniform weights: an assignment
  f = out.f.cpu().numpy().astype(np.float64)
  g = out.g.cpu().numpy().astype(np.float64)
  og = o.Geom(x.astype(np.float64), y.astype(np.float64), 0.05, inv_scale=0.5)
  p = o.transport_matrix(f, g, og)
  c = og.cost_block()
  eps = 0.05
  ent = (np.sum(p * c) - f @ p.sum(1) - g @ p.sum(0)) / eps
  assert abs(out.entropy - ent) <= 1e-4 * abs(ent)
  assert abs(out.normalized_entropy - (ent / np.log(n) - 1.0)) <= 1e-4 * abs(ent / np.log(n))
  raw_diag = ((x.astype(np.float64) - y) ** 2).sum(1)
  np.testing.assert_allclose(out.diag.cpu().numpy(), np.exp((-raw_diag + f + g) / eps),
                             rtol=2e-4)
  u, v = out.scalings
  np.testing.assert_allclose(u.cpu().numpy(), np.exp(f / eps), rtol=1e-5)
  np.testing.assert_allclose(v.cpu().numpy(), np.exp(g / eps), rtol=1e-5)
  assert abs(out.transport_mass - p.sum()) <= 1e-4 * p.sum()
  x2, y2, _, _ = problems.uniform_cloud_problem(n, n, d, seed=42)
  other = pointcloud.PointCloud(torch.as_tensor(x2).cuda(), torch.as_tensor(y2).cuda(),
                                epsilon=0.05, scale_cost=3.0)
  c2 = o.sqeuclidean_all_pairs(x2.astype(np.float64), y2.astype(np.float64)) / 3.0
  want = np.sum(p * c2)
  assert abs(out.transport_cost_at_geom(other) - want) <= 1e-4 * abs(want)
  with np.errstate(divide="ignore", invalid="ignore"):
    entr = np.where(p > 0, -p * np.log(p), 0.0).sum()
  want = np.sum(p * c2) - eps * entr
  assert abs(out.cost_at_geom(other) - want) <= 1e-4 * abs(want)
  with pytest.raises(NotImplementedError):
    out.to_dual_potentials()


@pytest.mark.parametrize("precision", ["sweep_fp32", "bf16_split3"])
@pytest.mark.parametrize("num_vec", [1, 3])
def test_planned_sweep_product_equals_one_shot(precision, num_vec):
  """``ottb_apply_transport_sweep_plan`` / ``_run`` against the one-shot
  ``ottb_apply_transport_sweep`` on the same inputs: the same kernels, so
  the same values to 1e-6 of the largest entry, for several vectors run in
  a row on one plan (nothing carries over from one run to the next), on
  both axes."""
  import torch
  x, y, a, b = problems.uniform_cloud_problem(700, 1100, 48, seed=5)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean",
                                precision="fp32")
  gen = torch.Generator().manual_seed(num_vec)
  for axis in (0, 1):
    prod = geom._sweep_product(out.f, out.g, axis, precision, num_vec=num_vec)
    rows = 700 if axis == 0 else 1100
    for _ in range(3):
      vec = torch.randn(num_vec, rows, generator=gen).cuda()
      got = prod(vec)
      want = geom._apply_raw(out.f, out.g, vec, axis, precision)
      assert float((got - want).abs().max()) <= 1e-6 * float(want.abs().max())
    with pytest.raises(ValueError):
      prod(torch.zeros(num_vec + 1, rows, device="cuda"))
    del prod
  assert geom._sweep_product(out.f, out.g, 0, "fp32") is None


@pytest.mark.parametrize("d", [48, 100])
@pytest.mark.parametrize("num_vec", [1, 2, 3])
def test_planned_fp32_product_equals_one_shot(d, num_vec):
  """``ottb_apply_transport_plan`` / ``_run`` against the one-shot
  ``ottb_apply_transport`` (FP32): the centre, B and its column terms
  prepared once at d <= 64 (nothing to prepare at d = 100), several
  vectors run in a row on one plan, both axes, within 1e-6 of the largest
  entry."""
  import torch
  x, y, a, b = problems.uniform_cloud_problem(900, 1300, d, seed=d)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean",
                                precision="fp32")
  gen = torch.Generator().manual_seed(num_vec)
  for axis in (0, 1):
    prod = geom._apply_product(out.f, out.g, axis, num_vec=num_vec)
    rows = 900 if axis == 0 else 1300
    for _ in range(3):
      vec = torch.randn(num_vec, rows, generator=gen).cuda()
      got = prod(vec)
      want = geom._apply_raw(out.f, out.g, vec, axis, "fp32")
      assert float((got - want).abs().max()) <= 1e-6 * float(want.abs().max())
    with pytest.raises(ValueError):
      prod(torch.zeros(num_vec, rows + 1, device="cuda"))
    del prod
