"""Implicit differentiation of the potentials on the GPU: ImplicitDiff, the
potentials' autograd backward, and differentiable plan applications.

Tolerances (relative to the largest magnitude of the compared quantity):
- 5e-5 against the reference's own ImplicitDiff results (golden vectors).
  Float32 inputs and plan applications inside the CG solve give ~1e-6 there.
- 1e-4 against the float64 oracle at the GPU's potentials, for larger and
  less well-conditioned systems.
- 5e-5 for gradients of plan applications against float64 torch autograd
  on the dense plan.
"""
import numpy as np
import pytest

from oracle import sinkhorn_np as o
from tests import golden_cases, problems

pytestmark = pytest.mark.gpu


def _t(v, grad=False):
  import torch
  t = torch.as_tensor(np.asarray(v), dtype=torch.float32).cuda()
  return t.requires_grad_() if grad else t


def _rel(got, want):
  got = got.detach().cpu().numpy() if hasattr(got, "detach") else np.asarray(got)
  return float(np.abs(got - want).max() / max(np.abs(want).max(), 1e-300))


@pytest.mark.parametrize("name", golden_cases.implicit_names())
def test_implicit_matches_reference_golden(name):
  """lam from the reference's ImplicitDiff.solve, gradients from finite
  differences of its first_order_conditions, at its own potentials."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers.linear import implicit_differentiation as imp
  data, gkw = golden_cases.load_implicit(name)
  geom = pointcloud.PointCloud(_t(data["x"]), _t(data["y"]), epsilon=float(gkw["epsilon"]),
                               scale_cost=gkw.get("scale_cost", 1.0))
  prob = linear_problem.LinearProblem(geom, _t(data["a"]), _t(data["b"]))
  f, g = _t(data["f"]), _t(data["g"])
  gr = (torch.as_tensor(data["gr_f"]).cuda(), torch.as_tensor(data["gr_g"]).cuda())
  idiff = imp.ImplicitDiff()
  assert _rel(idiff.solve(gr, prob, f, g), data["lam"]) < 5e-5
  assert float(idiff.first_order_conditions(prob, f, g).abs().max()) < 1e-5
  for got, key in zip(idiff.gradient(prob, f, g, True, gr), ("gx", "gy", "ga", "gb")):
    assert _rel(got, data[key]) < 5e-5, key


@pytest.mark.parametrize("n,m,d,eps,scale", [(300, 200, 3, 0.05, 1.0), (257, 400, 16, 0.1, "mean"),
                                             (640, 640, 64, 0.05, 1.0)])
def test_autograd_through_potentials_matches_oracle(n, m, d, eps, scale):
  """torch.autograd of <w, f> + <v, g> (sum w = sum v: independent of the
  potentials' free constant) through linear.solve."""
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  x, y, a, b = problems.uniform_cloud_problem(n, m, d, seed=n + m)
  rng = np.random.default_rng(1)
  w, v = rng.standard_normal(n), rng.standard_normal(m)
  v += (w.sum() - v.sum()) / m
  xt, yt, at, bt = _t(x, True), _t(y, True), _t(a, True), _t(b, True)
  geom = pointcloud.PointCloud(xt, yt, epsilon=eps, relative_epsilon="mean", scale_cost=scale)
  out = linear.solve(geom, at, bt, threshold=1e-5, max_iterations=5000, precision="fp32")
  loss = (out.f.double() * _t(w).double()).sum() + (out.g.double() * _t(v).double()).sum()
  loss.backward()
  og = o.Geom(x.astype(np.float64), y.astype(np.float64), float(geom.epsilon),
              inv_scale=float(geom.inv_scale_cost))
  f = out.f.detach().double().cpu().numpy()
  g = out.g.detach().double().cpu().numpy()
  want = o.implicit_grads(w, v, f, g, a.astype(np.float64), b.astype(np.float64), og,
                          scale_cost_mean=scale == "mean")
  for t, ref, key in zip((xt, yt, at, bt), want, "xyab"):
    assert _rel(t.grad, ref) < 1e-4, key


def test_zero_weight_points_get_zero_gradients():
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  x, y, a, b = problems.uniform_cloud_problem(120, 90, 4, seed=4)
  a[[3, 50]] = 0.0
  a /= a.sum()
  xt, at = _t(x, True), _t(a, True)
  geom = pointcloud.PointCloud(xt, _t(y), epsilon=0.1)
  out = linear.solve(geom, at, _t(b), threshold=1e-6)
  w = np.random.default_rng(0).standard_normal(120)
  w[[3, 50]] = 0.0
  (out.f.double() * _t(w).double()).sum().backward()
  gx = xt.grad.cpu().numpy()
  assert np.isfinite(gx).all() and np.all(gx[[3, 50]] == 0.0)
  assert np.all(at.grad.cpu().numpy()[[3, 50]] == 0.0)
  og = o.Geom(x.astype(np.float64), y.astype(np.float64), 0.1)
  f = out.f.detach().double().cpu().numpy()
  g = out.g.detach().double().cpu().numpy()
  want = o.implicit_grads(w, np.zeros(90), f, g, a.astype(np.float64), b.astype(np.float64), og)
  assert _rel(xt.grad, want[0]) < 1e-4


def test_reg_ot_cost_without_danskin_equals_danskin_at_optimum():
  """At the optimum the cost is stationary in (f, g): differentiating the
  potentials too (use_danskin=False) changes the gradient only by the
  first-order conditions' residual."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  x, y, a, b = problems.uniform_cloud_problem(200, 150, 5, seed=6)
  grads = []
  for danskin in (True, False):
    xt, yt, at, bt = _t(x, True), _t(y, True), _t(a, True), _t(b, True)
    geom = pointcloud.PointCloud(xt, yt, epsilon=0.05, relative_epsilon="mean")
    cost = linear.reg_ot_cost(geom, at, bt, threshold=1e-6, use_danskin=danskin,
                              max_iterations=10000)
    assert isinstance(cost, torch.Tensor)
    cost.backward()
    grads.append([t.grad.cpu().numpy().astype(np.float64) for t in (xt, yt, at, bt)])
  for g0, g1, key in zip(grads[0], grads[1], "xyab"):
    if key in "ab":  # balanced: the weights' gradients are defined up to a constant
      g0, g1 = g0 - g0.mean(), g1 - g1.mean()
    assert _rel(g1, g0) < 1e-3, key


def test_output_reg_ot_cost_is_differentiable():
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  x, y, a, b = problems.uniform_cloud_problem(100, 80, 3, seed=8)
  xt = _t(x, True)
  out = linear.solve(pointcloud.PointCloud(xt, _t(y), epsilon=0.1), _t(a), _t(b))
  cost = out.reg_ot_cost
  assert isinstance(cost, torch.Tensor) and cost.requires_grad
  cost.backward()
  gx, _, _, _ = out.reg_ot_cost_grads()
  assert _rel(xt.grad, gx.cpu().numpy()) < 1e-6
  with torch.no_grad():
    out2 = linear.solve(pointcloud.PointCloud(_t(x), _t(y), epsilon=0.1), _t(a), _t(b))
  assert isinstance(out2.reg_ot_cost, float)


def test_generic_solver_path_agrees_on_point_gradients():
  """A user solver (the reference's NormalCG-equivalent) through the
  reference's generic construction: same point gradients; the weights'
  gradients agree up to the balanced problem's free constant."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers import linear
  from ott_b200.solvers.linear import implicit_differentiation as imp
  x, y, a, b = problems.uniform_cloud_problem(150, 110, 4, seed=10)
  geom = pointcloud.PointCloud(_t(x), _t(y), epsilon=0.1)
  out = linear.solve(geom, _t(a), _t(b), threshold=1e-7, max_iterations=10000)
  prob = linear_problem.LinearProblem(geom, _t(a), _t(b))
  rng = np.random.default_rng(2)
  gr = (torch.as_tensor(rng.standard_normal(150)).cuda(),
        torch.as_tensor(rng.standard_normal(110)).cuda())
  d0 = imp.ImplicitDiff().gradient(prob, out.f, out.g, True, gr)
  d1 = imp.ImplicitDiff(solver=imp.solve_normal_cg).gradient(prob, out.f, out.g, True, gr)
  assert _rel(d1[0], d0[0].cpu().numpy()) < 1e-3
  assert _rel(d1[1], d0[1].cpu().numpy()) < 1e-3
  for k in (2, 3):
    u, v = d1[k] - d1[k].mean(), d0[k] - d0[k].mean()
    assert _rel(u, v.cpu().numpy()) < 1e-3


def test_unrolled_differentiation_is_refused():
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  x, y, a, b = problems.uniform_cloud_problem(60, 50, 2, seed=12)
  xt = _t(x, True)
  out = linear.solve(pointcloud.PointCloud(xt, _t(y), epsilon=0.1), _t(a), _t(b),
                     implicit_diff=None)
  with pytest.raises(NotImplementedError):
    out.f.sum().backward()


@pytest.mark.parametrize("axis", [0, 1])
@pytest.mark.parametrize("scale", [1.0, "mean"])
def test_apply_and_matrix_gradients_match_dense_autograd(axis, scale):
  """Gradients of plan applications and of the dense plan w.r.t. the
  points, the potentials and the vectors against float64 torch autograd on
  the dense plan."""
  import torch
  from ott_b200.geometry import pointcloud
  n, m, d = 190, 260, 8
  x, y, _, _ = problems.uniform_cloud_problem(n, m, d, seed=14)
  rng = np.random.default_rng(3)
  f0 = 0.05 * rng.standard_normal(n)
  g0 = 0.05 * rng.standard_normal(m)
  vec = rng.standard_normal((4, n if axis == 0 else m))
  xt, yt, ft, gt, vt = (_t(x, True), _t(y, True), _t(f0, True), _t(g0, True), _t(vec, True))
  geom = pointcloud.PointCloud(xt, yt, epsilon=0.2, scale_cost=scale)
  outp = geom.apply_transport_from_potentials(ft, gt, vt, axis=axis)
  wc = torch.randn_like(outp)
  got = torch.autograd.grad((outp * wc).sum(), (xt, yt, ft, gt, vt))
  mat = geom.transport_from_potentials(ft, gt)
  dc = torch.randn_like(mat)
  got_m = torch.autograd.grad((mat * dc).sum(), (xt, yt, ft, gt))

  def dense(xd, yd, fd, gd):
    c = ((xd[:, None, :] - yd[None]) ** 2).sum(-1)
    c = c / c.mean() if scale == "mean" else c
    return torch.exp((fd[:, None] + gd[None] - c) / 0.2)

  leaves = [torch.as_tensor(np.asarray(v, np.float64)).requires_grad_()
            for v in (xt.detach().cpu(), yt.detach().cpu(), ft.detach().cpu(),
                      gt.detach().cpu(), vt.detach().cpu())]
  p = dense(*leaves[:4])
  ref_out = leaves[4] @ p if axis == 0 else leaves[4] @ p.t()
  want = torch.autograd.grad((ref_out * wc.double().cpu()).sum(), leaves)
  for u, v, key in zip(got, want, ("x", "y", "f", "g", "vec")):
    assert _rel(u, v.numpy()) < 5e-5, key
  p = dense(*leaves[:4])
  want_m = torch.autograd.grad((p * dc.double().cpu()).sum(), leaves[:4])
  for u, v, key in zip(got_m, want_m, "xyfg"):
    assert _rel(u, v.numpy()) < 5e-5, key


@pytest.mark.parametrize("n,d", [(8192, 64), (16384, 8)])
def test_solver_converges_at_scale(n, d):
  """Shapes where conjugate gradients' residual rose for tens of steps
  (stopping tests on it misfire): MINRES reaches the tolerance with no
  warning and finite gradients. The residual recomputed with the FP32 plan
  products stays within 5e-3: their rounding (exponents up to ~500 at
  d = 8 here) times the system's conditioning sets that floor (6e-4 to
  1.3e-3 measured, depending on the rounding of the points' centre)."""
  import warnings
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  from ott_b200.solvers.linear import implicit_differentiation as imp
  x, y, _, _ = problems.gaussian_shift_problem(n, n, d, seed=0)
  xt = torch.from_numpy(x).cuda().requires_grad_()
  geom = pointcloud.PointCloud(xt, torch.from_numpy(y).cuda(), epsilon=0.01,
                               relative_epsilon="mean")
  out = linear.solve(geom, threshold=1e-3)
  rng = np.random.default_rng(0)
  w = torch.from_numpy(rng.standard_normal(n)).cuda()
  v = torch.from_numpy(rng.standard_normal(n)).cuda()
  v += (w.sum() - v.sum()) / n
  with warnings.catch_warnings():
    warnings.simplefilter("error", RuntimeWarning)
    ((out.f.double() * w).sum() + (out.g.double() * v).sum()).backward()
  info = imp.last_solve_info
  assert info["rel_residual"] <= 1e-6 and info["true_rel_residual"] <= 5e-3, info
  assert torch.isfinite(xt.grad).all()


def test_solver_budget_exhaustion_warns():
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers import linear
  from ott_b200.solvers.linear import implicit_differentiation as imp
  x, y, a, b = problems.uniform_cloud_problem(300, 200, 4, seed=20)
  geom = pointcloud.PointCloud(_t(x), _t(y), epsilon=0.02)
  out = linear.solve(geom, _t(a), _t(b), threshold=1e-5)
  prob = linear_problem.LinearProblem(geom, _t(a), _t(b))
  gr = (torch.randn(300, dtype=torch.float64, device="cuda"),
        torch.randn(200, dtype=torch.float64, device="cuda"))
  with pytest.warns(RuntimeWarning, match="MINRES stopped"):
    imp.ImplicitDiff(solver_kwargs={"max_steps": 2}).solve(gr, prob, out.f, out.g)


def test_preconditioner_does_not_change_the_gradient():
  """The implicit derivative of the potentials does not depend on the
  preconditioner h of the first-order conditions: h = identity with the
  symmetric CG route of the reference's generic construction
  (implicit_differentiation.py:162-170, 193-232) gives the default
  (h = eps log) point gradients."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers import linear
  from ott_b200.solvers.linear import implicit_differentiation as imp
  x, y, a, b = problems.uniform_cloud_problem(160, 120, 3, seed=22)
  geom = pointcloud.PointCloud(_t(x), _t(y), epsilon=0.1)
  out = linear.solve(geom, _t(a), _t(b), threshold=1e-7, max_iterations=10000)
  prob = linear_problem.LinearProblem(geom, _t(a), _t(b))
  rng = np.random.default_rng(4)
  gf, gg = rng.standard_normal(160), rng.standard_normal(120)
  gg += (gf.sum() - gg.sum()) / 120
  gr = (torch.as_tensor(gf).cuda(), torch.as_tensor(gg).cuda())
  d0 = imp.ImplicitDiff().gradient(prob, out.f, out.g, True, gr)
  ident = imp.ImplicitDiff(precondition_fun=lambda v: v, symmetric=True,
                           solver=imp.solve_jax_cg, solver_kwargs={"tol": 1e-10})
  d1 = ident.gradient(prob, out.f, out.g, True, gr)
  assert _rel(d1[0], d0[0].cpu().numpy()) < 1e-3
  assert _rel(d1[1], d0[1].cpu().numpy()) < 1e-3


@pytest.mark.parametrize("arg", ["a", "x"])
@pytest.mark.parametrize("axis", [0, 1])
def test_apply_transport_jacobian_matches_finite_differences(arg, axis):
  """The reference's test of the same name (tests/solvers/linear/
  sinkhorn_diff_test.py:352-455, balanced, lse mode): the derivative of
  ``out.apply(vec, axis)`` through the solve, in a direction of the weights
  (mass-preserving) or of the points, against central differences of
  float64 oracle solves. The reference allows 1e-2 absolute and 1e-1
  relative; here 1e-3 of the derivative's magnitude."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  n, m, d, eps = 27, 13, 4, 0.01
  rng = np.random.default_rng(7 + axis + 2 * (arg == "x"))
  x = rng.uniform(size=(n, d)) / d
  y = rng.uniform(size=(m, d)) / d
  a = rng.uniform(size=n) + 0.2
  a /= a.sum()
  b = rng.uniform(size=m) + 0.2
  b /= b.sum()
  vec = rng.uniform(size=m if axis else n) - 0.5
  cot = rng.standard_normal(n if axis else m)
  delta = rng.uniform(size=n) if arg == "a" else rng.uniform(size=(n, d))
  if arg == "a":
    delta -= delta.mean()
  xt, at = _t(x, arg == "x"), _t(a, arg == "a")
  geom = pointcloud.PointCloud(xt, _t(y), epsilon=eps)
  out = linear.solve(geom, at, _t(b), threshold=1e-6, max_iterations=20000)
  app = out.apply(_t(vec), axis=axis)
  (app.double() * torch.as_tensor(cot).cuda()).sum().backward()
  grad = (at if arg == "a" else xt).grad.double().cpu().numpy()
  got = float((grad * delta).sum())

  def applied(a_, x_):
    og = o.Geom(x_, y, eps)
    r = o.sinkhorn(og, a_, b, threshold=1e-12, max_iterations=200000)
    p = o.transport_matrix(r.f, r.g, og)
    return float(cot @ (vec @ p if axis == 0 else p @ vec))

  h = 1e-5
  if arg == "a":
    fd = (applied(a + h * delta, x) - applied(a - h * delta, x)) / (2 * h)
  else:
    fd = (applied(a, x + h * delta) - applied(a, x - h * delta)) / (2 * h)
  assert abs(got - fd) <= 1e-3 * float(np.abs(grad * delta).sum()), (got, fd)


@pytest.mark.parametrize("scale", [1.0, "mean"])
def test_primal_and_dual_cost_gradients_match_finite_differences(scale):
  """``out.primal_cost`` and ``out.dual_cost`` are differentiable through
  the solve (implicit backward of the potentials, the plan's own dependence
  on the points and, for scale_cost="mean", the scale): their derivatives in
  a direction of the points against central differences of float64 solves."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  n, m, d, eps = 40, 30, 3, 0.05
  rng = np.random.default_rng(11)
  x, y = rng.uniform(size=(n, d)), rng.uniform(size=(m, d))
  a = rng.uniform(0.2, 1.2, n)
  a /= a.sum()
  b = rng.uniform(0.2, 1.2, m)
  b /= b.sum()
  delta = rng.standard_normal((n, d))
  xt = _t(x, True)
  out = linear.solve(pointcloud.PointCloud(xt, _t(y), epsilon=eps, scale_cost=scale),
                     _t(a), _t(b), threshold=1e-7, max_iterations=20000, precision="fp32")
  got = {}
  for name in ("primal_cost", "dual_cost"):
    val = getattr(out, name)
    assert isinstance(val, torch.Tensor) and val.requires_grad
    (g,) = torch.autograd.grad(val, xt, retain_graph=True)
    got[name] = (float((g.double().cpu().numpy() * delta).sum()),
                 float(np.abs(g.double().cpu().numpy() * delta).sum()))

  def costs(xx):
    inv = o.inv_scale_cost(xx, y, scale)
    og = o.Geom(xx, y, eps, inv_scale=inv)
    r = o.sinkhorn(og, a, b, threshold=1e-13, max_iterations=200000)
    p = o.transport_matrix(r.f, r.g, og)
    primal = float(np.sum(p * og.cost_block()))
    dual = float(a @ r.f + b @ r.g)
    return primal, dual

  h = 1e-5
  up, dn = costs(x + h * delta), costs(x - h * delta)
  for k, name in enumerate(("primal_cost", "dual_cost")):
    fd = (up[k] - dn[k]) / (2 * h)
    assert abs(got[name][0] - fd) <= 1e-3 * got[name][1], (name, got[name][0], fd)


@pytest.mark.parametrize("case", ["spd", "singular", "closes", "indefinite", "step_cap",
                                  "window", "identity"])
def test_device_minres_matches_host_minres(case):
  """``ottb_minres_step`` (scalars on the device, stop flag read every few
  steps) against the host loop on the same float64 operator: the same step
  count and iterate to rounding. The indefinite system stops on a boundary
  of its tolerance, so its step count may differ by one. The inconsistent
  system's plateau stops it on the 1 % window rule, with a ratio 3e-3 away
  from 0.99 on either side of the stop step."""
  import torch
  from ott_b200.solvers.linear import implicit_differentiation as imp
  gen = torch.Generator().manual_seed(3)
  n = 300
  q, _ = torch.linalg.qr(torch.randn(n, n, dtype=torch.float64, generator=gen))
  ev = torch.linspace(0.01, 2.0, n, dtype=torch.float64)
  rtol, max_steps, window = 1e-12, 2000, 50
  if case == "singular":
    ev[:7] = 0.0
  elif case == "closes":  # four distinct eigenvalues: the Krylov space closes
    ev = torch.cat([torch.ones(n - 3), torch.tensor([2.0, 3.0, 0.5])]).double()
  elif case == "indefinite":
    ev = torch.linspace(-1.0, 2.0, n, dtype=torch.float64)
  elif case == "step_cap":
    rtol, max_steps = 1e-14, 13
  elif case == "window":  # inconsistent singular system: the estimate levels off
    ev[:7] = 0.0
    window = 5
  a = (q * ev) @ q.T
  b = torch.randn(n, dtype=torch.float64, generator=gen)
  if case == "singular":
    b = a @ b
  a, b = a.cuda(), b.cuda()
  op = (lambda z: z) if case == "identity" else (lambda z: a @ z)
  xh = imp._minres_host(op, b, rtol, max_steps, window)
  ih = dict(imp.last_solve_info)
  xd = imp._minres_device(op, b, rtol, max_steps, window)
  idv = dict(imp.last_solve_info)
  tol_steps = 1 if case == "indefinite" else 0
  assert abs(idv["steps"] - ih["steps"]) <= tol_steps, (ih, idv)
  assert _rel(xd, xh.cpu().numpy()) < 1e-9
  assert abs(idv["rel_residual"] - ih["rel_residual"]) <= 1e-9 * max(ih["rel_residual"], 1e-3)
  assert abs(idv["true_rel_residual"] - ih["true_rel_residual"]) < 1e-9
  if case == "identity":
    assert idv["steps"] == 1 and _rel(xd, b.cpu().numpy()) < 1e-15
  # the public dispatch takes the device loop for CUDA tensors
  xp = imp._minres(op, b, rtol, max_steps, window)
  assert _rel(xp, xd.cpu().numpy()) < 1e-12
  # blocks of 4 and 8 steps replayed from a CUDA graph
  # (ottb_minres_step_next, the step count on the device) give the step
  # count and iterate of the steps issued one by one from the host
  # (ottb_minres_step): the same launches in the same order (frozen steps
  # past the stop change nothing; the operator's own library products may
  # round differently when captured, hence the host-loop tolerances)
  for block in (4, 8):
    xb = imp._minres_device(op, b, rtol, max_steps, window, graph_block=block)
    ib = dict(imp.last_solve_info)
    assert abs(ib["steps"] - idv["steps"]) <= tol_steps, (block, ib, idv)
    assert _rel(xb, xd.cpu().numpy()) < 1e-9, block
    assert abs(ib["rel_residual"] - idv["rel_residual"]) <= 1e-9 * max(idv["rel_residual"],
                                                                       1e-3)


def test_tensor_core_products_give_the_fp32_gradient():
  """Above 2^25 plan entries at d >= 32 the chosen precision runs the
  backward's one-vector products as planned zero-iteration solves on the
  tensor-core sweep (``ottb_apply_transport_sweep_plan`` / ``_run``) and
  the pullback's many-vector products on ``ottb_apply_transport_tc``. At
  the same potentials and cotangent its input cotangents agree with those
  of the FP32 products within 1e-2 of each one's largest entry (products
  within ~1.5e-4 relative, amplified by the system's conditioning; the
  points' cotangents also carry the pullback products' BF16 split-3
  exponent error, ~1e-3 in log2 units at this epsilon: measured 7.0e-3)."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers import linear
  from ott_b200.solvers.linear import implicit_differentiation as imp
  n, d = 6144, 64
  assert n * n >= imp.ImplicitDiff._TC_MIN_ENTRIES
  x, y, _, _ = problems.gaussian_shift_problem(n, n, d, seed=1)
  geom = pointcloud.PointCloud(_t(x), _t(y), epsilon=0.01, relative_epsilon="mean")
  out = linear.solve(geom, threshold=1e-5, max_iterations=5000, precision="fp32")
  assert geom._sweep_product(out.f, out.g, 0, "auto") is not None
  prob = linear_problem.LinearProblem(geom)
  gen = torch.Generator().manual_seed(2)
  gr = (torch.randn(n, dtype=torch.float64, generator=gen).cuda(),
        torch.randn(n, dtype=torch.float64, generator=gen).cuda())
  tc = imp.ImplicitDiff().gradient(prob, out.f, out.g, True, gr, precision="auto")
  tc_steps = imp.last_solve_info["steps"]
  ref = imp.ImplicitDiff().gradient(prob, out.f, out.g, True, gr, precision="fp32")
  assert tc_steps > 0
  for got, want in zip(tc, ref):
    want = want.detach().cpu().numpy()
    assert _rel(got, want) < 1e-2, _rel(got, want)
