"""The plan applied to many vectors on the tensor cores
(ottb_apply_transport_tc: S = <x, y> and O = P V^T both as tcgen05 BF16
split-3 MMAs, P passed through tensor memory), against the float64 plan,
the reference's own golden applications and the FP32 kernel.

Tolerance, relative to the sum of |P| |v| of each output entry: the cost
products drop the lo*lo term and the inputs' bits below 2^-16 (an exponent
error up to 2^-15 * 2 inv |x_i| |y_j| / eps after centring, as for the
sweep engine's products), plus 2^-14 for the P V products (the weights'
and vectors' bf16 hi/lo splits), plus 1e-5 for the FP32 inputs and sums.
"""
import ctypes

import numpy as np
import pytest

from oracle import sinkhorn_np as o
from tests import golden_cases, helpers, problems

pytestmark = pytest.mark.gpu


def _rel(x, y, eps):
  c = 0.5 * (x.mean(0) + y.mean(0))
  r = np.linalg.norm(x - c, axis=1).max() * np.linalg.norm(y - c, axis=1).max()
  return 2.0 ** -15 * 2 * r / eps + 2.0 ** -14 + 1e-5


def _check(got, vec, p_ref, axis, rel):
  want = vec @ p_ref if axis == 0 else vec @ p_ref.T
  scale = np.abs(vec) @ p_ref if axis == 0 else np.abs(vec) @ p_ref.T
  err = np.abs(got - want)
  bound = rel * np.maximum(scale, scale.max(axis=1, keepdims=True) * 1e-3)
  assert np.all(err <= bound), (float((err / bound).max()), rel)


def _raw_tc(geom, f, g, vec, axis):
  """One ottb_apply_transport_tc call through the C ABI; returns the output
  and the workspace's status word."""
  import torch
  from ott_b200 import _arrays, _lib
  lib = _lib.load()
  n, m = geom.shape
  v = torch.as_tensor(vec, dtype=torch.float32).cuda().contiguous()
  out = torch.full((v.shape[0], m if axis == 0 else n), float("nan"), device="cuda")
  ws_bytes = int(lib.ottb_apply_transport_tc_workspace_size(n, m, geom.dim, v.shape[0], axis))
  assert ws_bytes > 0
  ws = torch.full((ws_bytes,), 0xAB, dtype=torch.uint8, device="cuda")
  st = lib.ottb_apply_transport_tc(geom.x.data_ptr(), geom.y.data_ptr(), n, m, geom.dim,
                                   f.data_ptr(), g.data_ptr(), ctypes.c_float(geom.epsilon),
                                   ctypes.c_float(geom.inv_scale_cost), v.data_ptr(),
                                   v.shape[0], axis, out.data_ptr(), ws.data_ptr(), ws_bytes,
                                   _arrays.stream_handle())
  _lib.check(st, "ottb_apply_transport_tc")
  status = int(ws[:4].view(torch.int32).item())
  return out.cpu().numpy().astype(np.float64), status


@pytest.mark.parametrize("n,m,d", [(300, 500, 3), (1000, 700, 64), (129, 257, 100),
                                   (777, 1234, 32)])
@pytest.mark.parametrize("num_vec", [1, 8, 65, 130])
def test_tc_application_matches_oracle(n, m, d, num_vec):
  """Both axes, one to three vector chunks (96 vectors per chunk at d <= 64,
  64 above), ragged row blocks and column tiles."""
  x, y, a, b = problems.uniform_cloud_problem(n, m, d, seed=n + d)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean",
                                precision="fp32")
  f = out.f.cpu().numpy().astype(np.float64)
  g = out.g.cpu().numpy().astype(np.float64)
  og = o.Geom(x.astype(np.float64), y.astype(np.float64), float(geom.epsilon))
  p_ref = o.transport_matrix(f, g, og)
  rel = _rel(x, y, og.epsilon)
  rng = np.random.default_rng(num_vec + d)
  for axis in (0, 1):
    vec = rng.standard_normal((num_vec, n if axis == 0 else m))
    got, status = _raw_tc(geom, out.f, out.g, vec, axis)
    assert status == 0
    _check(got, vec, p_ref, axis, rel)


def test_tc_application_edge_cases():
  """Zero-weight points on both sides (-inf potentials: zero rows and
  columns of the plan), a vector with zero entries, an all-zero vector,
  potentials far from any solve (every weight of a row far above 1 before
  the row's shift)."""
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
  rel = _rel(x, y, og.epsilon)
  rng = np.random.default_rng(2)
  for shift in (0.0, 40.0):
    # f + shift * eps: every plan entry times e^40 (FP32 overflows without
    # the rows' shift)
    fs = f + shift * og.epsilon
    p_ref = np.nan_to_num(o.transport_matrix(fs, g, og))
    ft = torch.as_tensor(fs, dtype=torch.float32).cuda()
    for axis in (0, 1):
      k = n if axis == 0 else m
      vec = rng.standard_normal((9, k))
      vec[0, ::3] = 0.0
      vec[2] = 0.0
      got, status = _raw_tc(geom, ft, out.g, vec, axis)
      assert status == 0
      assert np.isfinite(got).all()
      _check(got, vec, p_ref, axis, rel)
  # the zero-weight rows of the output are exactly zero
  got, _ = _raw_tc(geom, out.f, out.g, rng.standard_normal((9, m)), 1)
  assert np.all(got[:, [0, 7, 150]] == 0.0)


@pytest.mark.parametrize("name", golden_cases.names())
def test_tc_application_matches_reference_golden(name):
  """The reference's own SinkhornOutput.apply on its own potentials."""
  import torch
  data, geom_kw, _, _ = golden_cases.load(name, "f64")
  from ott_b200.geometry import pointcloud
  x = np.asarray(data["x"], dtype=np.float64)
  y = np.asarray(data["y"], dtype=np.float64)
  geom = pointcloud.PointCloud(torch.as_tensor(x, dtype=torch.float32).cuda(),
                               torch.as_tensor(y, dtype=torch.float32).cuda(),
                               epsilon=float(data["epsilon"]),
                               scale_cost=geom_kw.get("scale_cost", 1.0))
  f = torch.as_tensor(data["f"], dtype=torch.float32).cuda()
  g = torch.as_tensor(data["g"], dtype=torch.float32).cuda()
  inv = o.inv_scale_cost(x, y, geom_kw.get("scale_cost", 1.0))
  fin_f, fin_g = data["f"][np.isfinite(data["f"])], data["g"][np.isfinite(data["g"])]
  cmax = o.sqeuclidean_all_pairs(x, y).max() * inv
  zmax = (np.abs(fin_f).max() + np.abs(fin_g).max() + cmax) / float(data["epsilon"])
  rel = max(1e-5, 8 * 2.0 ** -24 * zmax) + _rel(x * np.sqrt(inv), y * np.sqrt(inv),
                                                 float(data["epsilon"]))
  for axis, key in ((0, "0"), (1, "1")):
    vec = np.asarray(data["vec" + key], dtype=np.float64)
    got, status = _raw_tc(geom, f, g, vec, axis)
    assert status == 0
    want = data["apply" + key]
    for k in range(want.shape[0]):
      scale = np.max(np.abs(want[k]))
      np.testing.assert_allclose(got[k], want[k], rtol=0, atol=rel * scale)


def test_tc_application_matches_fp32_kernel_large():
  """n = m = 8192, d = 64, 65 vectors (the Danskin gradient's [1, y^T]):
  against ottb_apply_transport (FP32) on the same potentials, both axes,
  column splits and a partial last vector chunk included."""
  import torch
  n = m = 8192
  x, y, a, b = problems.gaussian_shift_problem(n, m, 64, seed=3)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.01, relative_epsilon="mean",
                                precision="bf16_split3")
  rel = _rel(x, y, float(geom.epsilon))
  gen = torch.Generator(device="cuda").manual_seed(0)
  for axis in (0, 1):
    vec = torch.randn((65, n if axis == 0 else m), device="cuda", generator=gen)
    want = geom._apply_raw(out.f, out.g, vec, axis, "fp32").double()
    scale = geom._apply_raw(out.f, out.g, vec.abs(), axis, "fp32").double()
    got, status = _raw_tc(geom, out.f, out.g, vec.cpu().numpy(), axis)
    assert status == 0
    err = (torch.as_tensor(got, device="cuda") - want).abs()
    bound = rel * torch.maximum(scale, scale.amax(1, keepdim=True) * 1e-3)
    assert bool((err <= bound).all()), float((err / bound).max())


def test_public_apply_and_danskin_gradients_take_the_tc_route():
  """After a chosen-form solve, SinkhornOutput.apply on 16 vectors and the
  reg_ot_cost gradient (1 + d vectors per axis) go to the tensor cores and
  agree with the FP32 products at the same potentials."""
  import torch
  from ott_b200.geometry import pointcloud
  n, m, d = 2304, 2048, 48
  assert n * m >= pointcloud.TC_PRODUCT_MIN_ENTRIES
  x, y, a, b = problems.gaussian_shift_problem(n, m, d, seed=9)
  geom, out = helpers.gpu_solve(x, y, a, b, epsilon=0.05, relative_epsilon="mean",
                                precision="bf16_split3")
  assert out.precision == "bf16_split3"
  assert geom._product_precision(out.precision, 16) == "bf16_split3_tc"
  assert geom._product_precision(out.precision, 2) == "fp32"
  rel = _rel(x, y, float(geom.epsilon))
  v = torch.randn(16, n, device="cuda")
  got = out.apply(v, axis=0).double()
  want = geom._apply_raw(out.f, out.g, v, 0, "fp32").double()
  scale = geom._apply_raw(out.f, out.g, v.abs(), 0, "fp32").double()
  assert bool(((got - want).abs() <= rel * scale.amax(1, keepdim=True)).all())
  gx, gy, ga, gb = out.reg_ot_cost_grads()
  fp = out._replace(precision="fp32")
  hx, hy, ha, hb = fp.reg_ot_cost_grads()
  for u, w in ((gx, hx), (gy, hy)):
    np.testing.assert_allclose(u.cpu().numpy(), w.cpu().numpy(), rtol=0,
                               atol=20 * rel * float(w.abs().max()))
  np.testing.assert_array_equal(ga.cpu().numpy(), ha.cpu().numpy())
  np.testing.assert_array_equal(gb.cpu().numpy(), hb.cpu().numpy())
