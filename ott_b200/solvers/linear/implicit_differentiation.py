"""Implicit differentiation of the Sinkhorn potentials
(ott/solvers/linear/implicit_differentiation.py).

At the solution the first-order conditions
``F(f, g; C, a, b) = [h(P 1) - h(a), h(P^T 1) - h(b)] = 0`` hold (with the
preconditioner ``h = eps log`` by default, :235-273). The backward of the
potentials applies ``-(dF/d(f, g))^-T`` to their cotangent (:80-233) and
pulls the result back through ``F``'s dependence on the inputs (:275-287).
Every product with the plan is one ``ottb_apply_transport`` launch; the plan
is never formed.

Default solver (``solver=None``, ``precondition_fun=None``): the Schur
complement of the reference's block system on the smaller side,
``S = I - R D_l^-1 R^T D_s^-1`` (``R`` the plan or its transpose, ``D`` the
marginals of the two sides), is solved by MINRES on its symmetric form
``D_s^-1/2 S D_s^1/2 = I - K K^T`` (the MINRES residual never increases;
CG's rises for tens of steps on these systems before it falls, which
defeats any stopping test on it). The reference runs lineax
``NormalCG`` on ``S`` itself (lineax_implicit.py:49-101), whose limit from
zero is the least-squares solution of least norm; ``S`` is singular
(``S ma = 0`` and ``1^T S = 0`` for the small side's marginal ``ma``), so
here the right-hand side is projected onto ``range(S) = 1^perp`` and the
solution onto ``ma^perp``, which is that same solution, with the condition
number of ``S`` instead of its square. A user ``solver`` or
``precondition_fun`` runs the reference's generic form instead.

Zero-weight points are left out of the system (their gradients are 0; the
reference's ``eps / 0`` makes them NaN).
"""
from __future__ import annotations

import dataclasses
import warnings
from typing import Any, Callable, Dict, Optional, Tuple

import torch

__all__ = ["ImplicitDiff", "solve_jax_cg", "solve_normal_cg"]

LinOp = Callable[[torch.Tensor], torch.Tensor]


# Steps and final relative residual of the last iterative solve in this
# process (introspection only; nothing in the package reads it back).
last_solve_info: Dict[str, float] = {}


def _cg(op: LinOp, rhs: torch.Tensor, stop: Callable[[torch.Tensor], bool],
        max_steps: int) -> torch.Tensor:
  """Conjugate gradients from zero for a symmetric positive semi-definite
  ``op``; ``stop(residual)`` ends it."""
  bnorm = max(float(torch.linalg.vector_norm(rhs)), 1e-300)
  x = torch.zeros_like(rhs)
  r = rhs.clone()
  last_solve_info.clear()
  last_solve_info.update(steps=0, rel_residual=1.0)
  if stop(r):
    return x
  p = r.clone()
  rr = torch.dot(r, r)
  for step in range(1, max_steps + 1):
    ap = op(p)
    pap = torch.dot(p, ap)
    if float(pap) <= 0.0:
      break
    alpha = rr / pap
    x = x + alpha * p
    r = r - alpha * ap
    last_solve_info.update(steps=step,
                           rel_residual=float(torch.linalg.vector_norm(r)) / bnorm)
    if stop(r):
      return x
    rr_new = torch.dot(r, r)
    p = r + (rr_new / rr) * p
    rr = rr_new
  return x


def _minres(op: LinOp, rhs: torch.Tensor, rtol: float, max_steps: int,
            window: int = 50) -> torch.Tensor:
  """MINRES (Paige and Saunders, SIAM J. Numer. Anal. 12, 1975) from zero for
  a symmetric ``op``: Lanczos vectors with the tridiagonal system reduced by
  Givens rotations, so the residual norm estimate never increases. Stops
  when it falls to ``rtol |rhs|``, after ``max_steps``, or when ``window``
  steps lower it by less than 1 %. Records steps, the estimate and the
  true relative residual ``|rhs - op(x)| / |rhs|`` (one more product).
  On a CUDA device each step after the product is one ``ottb_minres_step``
  launch (``_minres_device``); elsewhere the steps run here."""
  if rhs.is_cuda:
    return _minres_device(op, rhs, rtol, max_steps, window)
  return _minres_host(op, rhs, rtol, max_steps, window)


# ottb_minres_step's state slots read back by the host
_ST_PHIBAR, _ST_ACTIVE, _ST_STEPS = 4, 9, 10

# Steps that one CUDA graph replay runs (a multiple of 4, the period of the
# graph path's buffer rotation); 0 issues every step from the host. Off by
# default: on B200 at d = 64 the replayed blocks gave the same gradients bit
# for bit but no steady gain (n = m = 4096: 21.8 ms either way; 8192: 47-59
# ms against 52-53 ms; 65536: 0.877 s against 0.850 s, where up to a block
# of 2.9 ms products runs past the stop), since the plan products' own
# device time, not the host's issue time, bounds a step.
MINRES_GRAPH_BLOCK = 0


def _minres_device(op: LinOp, rhs: torch.Tensor, rtol: float, max_steps: int,
                   window: int = 50, graph_block: Optional[int] = None) -> torch.Tensor:
  """``_minres_host``'s iteration with its scalars on the device: per step
  the product ``op(v)`` and one ``ottb_minres_step`` launch, which freezes
  the iterate once the stop test fires, then an asynchronous copy of the
  stop flag to pinned memory. After issuing step k the host waits for step
  k - 1's flag only, so step k keeps the GPU busy meanwhile; the one step
  issued past the stop is discarded work, not a change of the result.

  With ``graph_block`` (default ``MINRES_GRAPH_BLOCK``) > 0 the steps run
  in blocks replayed from one CUDA graph instead (``_minres_graph``)."""
  block = MINRES_GRAPH_BLOCK if graph_block is None else int(graph_block)
  if block > 0:
    return _minres_graph(op, rhs, rtol, max_steps, window, block)
  from ott_b200 import _arrays, _lib
  lib = _lib.load()
  rhs = rhs.to(torch.float64).contiguous()
  s = rhs.numel()
  beta1 = float(torch.linalg.vector_norm(rhs))
  x = torch.zeros_like(rhs)
  last_solve_info.clear()
  last_solve_info.update(steps=0, rel_residual=1.0, true_rel_residual=1.0)
  if beta1 == 0.0 or max_steps < 1:
    if beta1 == 0.0:
      last_solve_info.update(rel_residual=0.0, true_rel_residual=0.0)
    return x
  dev = rhs.device
  state = torch.tensor([beta1, 0.0, 0.0, 0.0, beta1, -1.0, 0.0, beta1, float(rtol), 1.0, 0.0]
                       + [0.0] * 5, dtype=torch.float64).to(dev)
  hist = torch.zeros(max_steps + 1, dtype=torch.float64, device=dev)
  hist[0] = beta1
  v = rhs / beta1
  v_next = torch.empty_like(rhs)
  r1, r2 = rhs, rhs.clone()
  w, w_prev = torch.zeros_like(rhs), torch.zeros_like(rhs)
  stream = _arrays.stream_handle()
  flags = torch.ones(2, dtype=torch.float64).pin_memory()
  done = [torch.cuda.Event(), torch.cuda.Event()]
  for step in range(1, max_steps + 1):
    y = op(v)
    if y.dtype != torch.float64 or not y.is_contiguous() or y.numel() != s:
      y = y.to(torch.float64).contiguous().reshape(s)
    if y.data_ptr() in (v.data_ptr(), v_next.data_ptr(), r1.data_ptr(), r2.data_ptr(),
                        w.data_ptr(), w_prev.data_ptr(), x.data_ptr()):
      y = y.clone()  # the step rewrites y in place
    st = lib.ottb_minres_step(state.data_ptr(), step, int(window), v.data_ptr(), y.data_ptr(),
                              r1.data_ptr(), r2.data_ptr(), w.data_ptr(), w_prev.data_ptr(),
                              x.data_ptr(), v_next.data_ptr(), hist.data_ptr(), hist.numel(),
                              s, stream)
    _lib.check(st, "ottb_minres_step")
    r1, r2 = r2, y
    w, w_prev = w_prev, w
    v, v_next = v_next, v
    flags[step % 2].copy_(state[_ST_ACTIVE], non_blocking=True)
    done[step % 2].record()
    if step >= 2:
      done[(step - 1) % 2].synchronize()
      if float(flags[(step - 1) % 2]) == 0.0:
        break
  steps, phibar = state[[_ST_STEPS, _ST_PHIBAR]].tolist()
  true_res = float(torch.linalg.vector_norm(rhs - op(x))) / beta1
  last_solve_info.update(steps=int(steps), rel_residual=phibar / beta1,
                         true_rel_residual=true_res)
  return x


def _minres_graph(op: LinOp, rhs: torch.Tensor, rtol: float, max_steps: int, window: int,
                  block: int) -> torch.Tensor:
  """``_minres_device`` with its steps in blocks of ``block`` replayed from
  one CUDA graph, so that the host's issue time of a step (the products'
  launches, the MINRES launch, the small vector kernels around them) is
  paid once, at capture, instead of at every step.

  ``ottb_minres_step_next`` counts the steps on the device, and every step
  reads and writes fixed buffers (the Lanczos vectors in a ring of four, v
  and the search directions in pairs), so a block that starts at step
  4j + 1 is one fixed sequence of launches. The first block runs
  uncaptured: it plans the products and initialises whatever the operator
  calls. After it the host replays the graph, copies the stop flag to
  pinned memory behind each replay and waits for the previous replay's
  flag only; at most one block past the stop runs, as frozen steps that
  leave the iterate unchanged. Steps left over at the step cap run
  uncaptured, and so does every step after an operator that cannot be
  captured. The arithmetic is ``_minres_device``'s, launch for launch."""
  from ott_b200 import _arrays, _lib
  lib = _lib.load()
  if block < 4 or block % 4:
    raise ValueError("graph_block must be a positive multiple of 4")
  rhs = rhs.to(torch.float64).contiguous()
  s = rhs.numel()
  beta1 = float(torch.linalg.vector_norm(rhs))
  x = torch.zeros_like(rhs)
  last_solve_info.clear()
  last_solve_info.update(steps=0, rel_residual=1.0, true_rel_residual=1.0)
  if beta1 == 0.0 or max_steps < 1:
    if beta1 == 0.0:
      last_solve_info.update(rel_residual=0.0, true_rel_residual=0.0)
    return x
  dev = rhs.device
  state = torch.tensor([beta1, 0.0, 0.0, 0.0, beta1, -1.0, 0.0, beta1, float(rtol), 1.0, 0.0]
                       + [0.0] * 5, dtype=torch.float64).to(dev)
  hist = torch.zeros(max_steps + 1, dtype=torch.float64, device=dev)
  hist[0] = beta1
  vs = [rhs / beta1, torch.empty_like(rhs)]
  dirs = [torch.zeros_like(rhs), torch.zeros_like(rhs)]
  rs = [rhs.clone()] + [torch.empty_like(rhs) for _ in range(3)]

  def step(k: int) -> None:
    # step k: v = vs[(k-1)%2] -> v_next = vs[k%2]; direction w = dirs[(k-1)%2],
    # the new one into dirs[k%2]; y = op(v) in rs[k%4], r2 = rs[(k-1)%4],
    # r1 = rs[(k-2)%4] (unused at step 1); the stream is read at every call,
    # the capture's own while capturing
    v, y = vs[(k - 1) % 2], rs[k % 4]
    y.copy_(op(v).reshape(s))
    st = lib.ottb_minres_step_next(
        state.data_ptr(), int(window), v.data_ptr(), y.data_ptr(), rs[(k - 2) % 4].data_ptr(),
        rs[(k - 1) % 4].data_ptr(), dirs[(k - 1) % 2].data_ptr(), dirs[k % 2].data_ptr(),
        x.data_ptr(), vs[k % 2].data_ptr(), hist.data_ptr(), hist.numel(), s,
        _arrays.stream_handle())
    _lib.check(st, "ottb_minres_step_next")

  def capture(k0: int) -> Optional[torch.cuda.CUDAGraph]:
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream(device=dev)
    try:
      with torch.cuda.stream(side):
        graph.capture_begin()
        try:
          for j in range(block):
            step(k0 + 1 + j)
        except BaseException:
          try:
            graph.capture_end()
          except RuntimeError:
            pass
          raise
        graph.capture_end()
    except RuntimeError:
      return None
    return graph

  flags = torch.ones(2, dtype=torch.float64).pin_memory()
  done = [torch.cuda.Event(), torch.cuda.Event()]

  def mark(i: int) -> None:
    flags[i % 2].copy_(state[_ST_ACTIVE], non_blocking=True)
    done[i % 2].record()

  k = 0
  for _ in range(min(block, max_steps)):
    k += 1
    step(k)
  mark(0)
  graph = capture(k) if max_steps - k >= block else None
  i = 0
  while k < max_steps:
    i += 1
    if graph is not None and max_steps - k >= block:
      graph.replay()
      k += block
    else:
      for _ in range(min(block, max_steps - k)):
        k += 1
        step(k)
    mark(i)
    done[(i - 1) % 2].synchronize()
    if float(flags[(i - 1) % 2]) == 0.0:
      break
  steps, phibar = state[[_ST_STEPS, _ST_PHIBAR]].tolist()  # waits for every step issued
  del graph
  true_res = float(torch.linalg.vector_norm(rhs - op(x))) / beta1
  last_solve_info.update(steps=int(steps), rel_residual=phibar / beta1,
                         true_rel_residual=true_res)
  return x


def _minres_host(op: LinOp, rhs: torch.Tensor, rtol: float, max_steps: int,
                 window: int = 50) -> torch.Tensor:
  """``_minres`` with every step on the host (one read of the two Lanczos
  scalars per step)."""
  beta1 = float(torch.linalg.vector_norm(rhs))
  x = torch.zeros_like(rhs)
  last_solve_info.clear()
  last_solve_info.update(steps=0, rel_residual=1.0, true_rel_residual=1.0)
  if beta1 == 0.0:
    last_solve_info.update(rel_residual=0.0, true_rel_residual=0.0)
    return x
  r1 = rhs.clone()
  r2 = rhs.clone()
  y = rhs.clone()
  w = torch.zeros_like(rhs)
  w2 = torch.zeros_like(rhs)
  beta, oldb = beta1, 0.0
  dbar, epsln, phibar = 0.0, 0.0, beta1
  cs, sn = -1.0, 0.0
  history = [phibar]
  step = 0
  for step in range(1, max_steps + 1):
    v = y / beta
    y = op(v)
    if step >= 2:
      y = y - (beta / oldb) * r1
    alfa_t = torch.dot(v, y)
    y = y - (alfa_t / beta) * r2
    r1, r2 = r2, y
    oldb = beta
    # one host read per step for both Lanczos scalars
    alfa, beta = torch.stack([alfa_t, torch.linalg.vector_norm(r2)]).tolist()
    # previous rotation applied to the new column of the tridiagonal matrix
    oldeps = epsln
    delta = cs * dbar + sn * alfa
    gbar = sn * dbar - cs * alfa
    epsln = sn * beta
    dbar = -cs * beta
    # the next rotation
    gamma = max((gbar * gbar + beta * beta) ** 0.5, 2.220446049250313e-16)
    cs, sn = gbar / gamma, beta / gamma
    phi = cs * phibar
    phibar = sn * phibar
    w1, w2 = w2, w
    w = (v - oldeps * w1 - delta * w2) / gamma
    x = x + phi * w
    history.append(phibar)
    if phibar <= rtol * beta1 or beta <= 1e-14 * beta1:  # converged, or Krylov space closed
      break
    if step >= window and phibar > 0.99 * history[step - window]:
      break
  true_res = float(torch.linalg.vector_norm(rhs - op(x))) / beta1
  last_solve_info.update(steps=step, rel_residual=phibar / beta1, true_rel_residual=true_res)
  return x


def _ridge(op: LinOp, ridge_kernel: float, ridge_identity: float) -> LinOp:
  if ridge_kernel > 0.0 or ridge_identity > 0.0:
    return lambda z: op(z) + ridge_kernel * torch.sum(z) + ridge_identity * z
  return op


def solve_jax_cg(lin: LinOp, b: torch.Tensor, lin_t: Optional[LinOp] = None,
                 symmetric: bool = False, ridge_identity: float = 0.0,
                 ridge_kernel: float = 0.0, tol: float = 1e-5, atol: float = 0.0,
                 maxiter: Optional[int] = None, **kwargs: Any) -> torch.Tensor:
  """implicit_differentiation.py:290-322 with the stopping rule of
  ``jax.scipy.sparse.linalg.cg`` (``|r| <= max(tol |b|, atol)``, at most
  ``maxiter = 10 size`` steps): CG on ``lin`` if ``symmetric``, else on
  ``lin_t(lin(.))``, with the optional ridge terms, against ``b`` as
  given there."""
  op = lin if symmetric else (lambda z: lin_t(lin(z)))
  op = _ridge(op, ridge_kernel, ridge_identity)
  bound = max(tol * float(torch.linalg.vector_norm(b)), atol)
  steps = 10 * b.numel() if maxiter is None else int(maxiter)
  return _cg(op, b, lambda r: float(torch.linalg.vector_norm(r)) <= bound, steps)


def solve_normal_cg(lin: LinOp, b: torch.Tensor, lin_t: Optional[LinOp] = None,
                    symmetric: bool = False, ridge_identity: float = 0.0,
                    ridge_kernel: float = 0.0, rtol: float = 1e-6, atol: float = 1e-6,
                    max_steps: Optional[int] = None, **kwargs: Any) -> torch.Tensor:
  """The reference's default solver (lineax_implicit.py:49-101: lineax
  ``CG`` if ``symmetric`` else ``NormalCG``, ``rtol = atol = 1e-6``, max
  norm): CG on ``lin`` against ``b``, or on ``lin_t(lin(.))`` against
  ``lin_t(b)``. At most ``max_steps`` steps (default ``10 size``; lineax has
  no bound)."""
  lin = _ridge(lin, ridge_kernel, ridge_identity)
  if symmetric:
    op, rhs = lin, b
  else:
    lin_t = _ridge(lin_t, ridge_kernel, ridge_identity)
    op, rhs = (lambda z: lin_t(lin(z))), lin_t(b)
  bound = atol + rtol * float(rhs.abs().max())
  steps = 10 * b.numel() if max_steps is None else int(max_steps)
  return _cg(op, rhs, lambda r: float(r.abs().max()) <= bound, steps)


def _elementwise_derivative(fun: Callable[[torch.Tensor], torch.Tensor],
                            v: torch.Tensor) -> torch.Tensor:
  """``vmap(grad(fun))(v)`` for an elementwise scalar function."""
  with torch.enable_grad():
    t = v.detach().clone().requires_grad_()
    (gt,) = torch.autograd.grad(fun(t).sum(), t)
  return gt.detach()


@dataclasses.dataclass
class ImplicitDiff:
  """implicit_differentiation.py:34-80, same fields.

  ``solver(lin, b, lin_t, symmetric, **solver_kwargs)`` solves the Schur
  system; ``None`` picks MINRES on the symmetric form described in the
  module docstring (keywords ``rtol`` (1e-6), ``max_steps`` (1000)).
  ``precondition_fun`` replaces ``h = eps log``.
  """

  solver: Optional[Callable[..., torch.Tensor]] = None
  solver_kwargs: Optional[Dict[str, Any]] = None
  symmetric: bool = False
  precondition_fun: Optional[Callable[[torch.Tensor], torch.Tensor]] = None

  def replace(self, **kwargs: Any) -> "ImplicitDiff":
    return dataclasses.replace(self, **kwargs)

  # -- plan products ---------------------------------------------------------
  # Below this many plan entries "auto" keeps the FP32 one-vector kernel:
  # the tensor-core route's fixed cost per product (two zero-iteration
  # solves) outweighs its faster sweep (measured per product: 0.19 vs 0.25 ms
  # at 8192^2, 0.39 vs 0.82 ms at 16384^2).
  _TC_MIN_ENTRIES = 1 << 25

  @classmethod
  def _app(cls, geom, f, g, precision: str = "fp32"):
    """The one-vector plan product of the backward, planned once per axis:
    on the sweep route (``ottb_apply_transport_sweep_plan``) or the FP32
    one (``ottb_apply_transport_plan``); every product after that is
    stream operations only."""
    n, m = geom.shape
    if precision == "auto" and n * m < cls._TC_MIN_ENTRIES:
      precision = "fp32"
    planned: Dict[int, Any] = {}

    def app32(v: torch.Tensor, axis: int) -> torch.Tensor:
      # FP32 in and out: the products' own precision
      if axis not in planned:
        prod = geom._sweep_product(f, g, axis, precision)
        if prod is None and hasattr(geom, "_apply_product"):
          prod = geom._apply_product(f, g, axis)
        planned[axis] = prod
      prod = planned[axis]
      if prod is None:
        return geom._apply_raw(f, g, v.reshape(1, -1), axis, precision)[0]
      return prod(v.reshape(1, -1))[0]

    def app(v: torch.Tensor, axis: int) -> torch.Tensor:
      return app32(v, axis).double()
    app.f32 = app32
    return app

  def _precond(self, geom) -> Callable[[torch.Tensor], torch.Tensor]:
    if self.precondition_fun is not None:
      return self.precondition_fun
    eps = float(geom.epsilon)
    return lambda v: eps * torch.log(v)

  def _derivative(self, geom, v: torch.Tensor) -> torch.Tensor:
    if self.precondition_fun is None:
      return float(geom.epsilon) / v
    return _elementwise_derivative(self.precondition_fun, v)

  @staticmethod
  def _check(ot_prob, lse_mode: bool) -> None:
    if not lse_mode:
      raise NotImplementedError("kernel mode (lse_mode=False) is not on this path")
    if not ot_prob.is_balanced:
      raise NotImplementedError("unbalanced problems (tau < 1) are not on this path")

  def first_order_conditions(self, prob, f: torch.Tensor, g: torch.Tensor,
                             lse_mode: bool = True) -> torch.Tensor:
    """implicit_differentiation.py:235-273: ``[a > 0](h(P 1) - h(a))``,
    ``[b > 0](h(P^T 1) - h(b))`` (float64, length n + m)."""
    self._check(prob, lse_mode)
    geom = prob.geom
    n, m = geom.shape
    app = self._app(geom, f, g)
    dev = f.device
    ma = app(torch.ones(m, dtype=torch.float64, device=dev), 1)
    mb = app(torch.ones(n, dtype=torch.float64, device=dev), 0)
    h = self._precond(geom)
    a, b = prob.a.detach().double(), prob.b.detach().double()
    one = lambda v, w: torch.where(w > 0, v, torch.ones_like(v))
    ra = torch.where(a > 0, h(one(ma, a)) - h(one(a, a)), torch.zeros_like(a))
    rb = torch.where(b > 0, h(one(mb, b)) - h(one(b, b)), torch.zeros_like(b))
    return torch.cat([ra, rb])

  # -- the linear solve --------------------------------------------------------
  def solve(self, gr: Tuple[torch.Tensor, torch.Tensor], ot_prob, f: torch.Tensor,
            g: torch.Tensor, lse_mode: bool = True, precision: str = "fp32") -> torch.Tensor:
    """implicit_differentiation.py:80-233: ``-(dF/d(f, g))^-T gr`` for the
    first-order conditions ``F`` (float64, length n + m). ``precision`` of
    the one-vector plan products: "fp32", or "auto" / "bf16_split3" for the
    solver's tensor-core sweep at d >= 32 (what the potentials' backward
    uses after a tensor-core solve)."""
    return self._solve(gr, ot_prob, f, g, lse_mode, precision)[0]

  def _solve(self, gr, ot_prob, f, g, lse_mode, precision="fp32"):
    """``solve`` and the plan's marginals ``(P 1, P^T 1)`` it used."""
    self._check(ot_prob, lse_mode)
    geom = ot_prob.geom
    n, m = geom.shape
    dev = f.device
    app = self._app(geom, f, g, precision)
    gr_f = gr[0].detach().double().reshape(n)
    gr_g = gr[1].detach().double().reshape(m)
    sa = ot_prob.a.detach() > 0
    sb = ot_prob.b.detach() > 0
    ma = app(torch.ones(m, dtype=torch.float64, device=dev), 1)
    mb = app(torch.ones(n, dtype=torch.float64, device=dev), 0)
    sa, sb = sa & (ma > 0), sb & (mb > 0)
    if self.solver is None and self.precondition_fun is None:
      lf, lg = self._solve_default(gr_f, gr_g, ma, mb, sa, sb, app, n > m)
    else:
      lf, lg = self._solve_generic(geom, gr_f, gr_g, ma, mb, sa, sb, app, n > m)
    zero = torch.zeros((), dtype=torch.float64, device=dev)
    return torch.cat([torch.where(sa, -lf, zero), torch.where(sb, -lg, zero)]), ma, mb

  def _solve_default(self, gr_f, gr_g, ma, mb, sa, sb, app, n_gt_m):
    kw = dict(self.solver_kwargs or {})
    rtol = float(kw.get("rtol", 1e-6))
    max_steps = int(kw.get("max_steps", 1000))
    zero = torch.zeros((), dtype=torch.float64, device=ma.device)
    safe_inv = lambda v, s: torch.where(s, 1.0 / torch.where(s, v, torch.ones_like(v)), zero)
    inv_ma, inv_mb = safe_inv(ma, sa), safe_inv(mb, sb)
    # small side s (the Schur system's), large side l; R maps l -> s
    if n_gt_m:
      gr_s, gr_l, m_s, s_s = gr_g, gr_f, mb, sb
      inv_s, inv_l = inv_mb, inv_ma
      r_op, rt_op = (lambda v: app(v, 0)), (lambda v: app(v, 1))
    else:
      gr_s, gr_l, m_s, s_s = gr_f, gr_g, ma, sa
      inv_s, inv_l = inv_ma, inv_mb
      r_op, rt_op = (lambda v: app(v, 1)), (lambda v: app(v, 0))
    res = torch.where(s_s, gr_s - r_op(gr_l * inv_l), zero)
    cnt = s_s.sum().clamp(min=1).double()
    res = torch.where(s_s, res - res.sum() / cnt, zero)  # onto range(S)
    c = torch.sqrt(inv_s)
    # null vector of the symmetric form: sqrt(m_s)
    q = torch.where(s_s, torch.sqrt(torch.where(s_s, m_s, torch.ones_like(m_s))), zero)
    q = q / torch.linalg.vector_norm(q).clamp(min=1e-300)

    a32 = getattr(app, "f32", None)
    if a32 is None:
      def sym_op(yv):
        # (I - K K^T) y with K = D_s^-1/2 R D_l^-1/2, plus q q^T y: the null
        # eigenvalue moved to 1 (the solution is orthogonal to q)
        return yv - c * r_op(inv_l * rt_op(c * yv)) + q * torch.dot(q, yv)
    else:
      # the same with the products' FP32 inputs written in place (the
      # scaling computed in float64, rounded once) and the output formed
      # by two fused multiply-adds: 6 small kernels a step instead of 12
      r32, rt32 = ((lambda v: a32(v, 0)), (lambda v: a32(v, 1))) if n_gt_m else \
                  ((lambda v: a32(v, 1)), (lambda v: a32(v, 0)))
      in_s = torch.empty(c.shape, dtype=torch.float32, device=c.device)
      in_l = torch.empty(inv_l.shape, dtype=torch.float32, device=c.device)

      def sym_op(yv):
        t = rt32(torch.mul(c, yv, out=in_s))
        u = r32(torch.mul(inv_l, t, out=in_l))
        return torch.addcmul(yv, q, torch.dot(q, yv)).addcmul_(c, u, value=-1.0)

    rhs = c * res
    rhs = rhs - q * torch.dot(q, rhs)
    yv = _minres(sym_op, rhs, rtol, max_steps)
    est, true = last_solve_info["rel_residual"], last_solve_info["true_rel_residual"]
    # the solver's own residual (not converged), or the residual recomputed
    # with the FP32 plan products (whose rounding sets a floor under it)
    if est > max(1e3 * rtol, 1e-3) or true > 1e-2:
      warnings.warn("implicit differentiation: MINRES stopped at relative residual "
                    f"{est:.3g} (recomputed: {true:.3g}) after "
                    f"{last_solve_info['steps']} steps", RuntimeWarning, stacklevel=4)
    z = torch.where(s_s, yv / torch.where(s_s, c, torch.ones_like(c)), zero)
    z = z - (torch.dot(z, m_s) / torch.dot(m_s, m_s)) * m_s  # onto ma^perp
    other = gr_l - rt_op(z * inv_s)
    return (other, z) if n_gt_m else (z, other)

  def _solve_generic(self, geom, gr_f, gr_g, ma, mb, sa, sb, app, n_gt_m):
    """The reference's construction (:156-233) with any solver and
    preconditioner."""
    eps = float(geom.epsilon)
    zero = torch.zeros((), dtype=torch.float64, device=ma.device)
    one = lambda v, s: torch.where(s, v, torch.ones_like(v))
    da = torch.where(sa, self._derivative(geom, one(ma, sa)), zero)
    db = torch.where(sb, self._derivative(geom, one(mb, sb)), zero)
    symmetric = self.symmetric if self.precondition_fun is not None else False
    solver = self.solver if self.solver is not None else solve_normal_cg
    kw = dict(self.solver_kwargs or {})
    vjp_fg = lambda z: app(z * db, 1) / eps
    vjp_gf = lambda z: app(z * da, 0) / eps
    vjp_fgt = lambda z: app(z, 0) * db / eps
    vjp_gft = lambda z: app(z, 1) * da / eps
    diag_a = torch.where(sa, ma * da / eps, torch.ones_like(ma))
    diag_b = torch.where(sb, mb * db / eps, torch.ones_like(mb))
    if n_gt_m:
      inv_ff = lambda z: z / diag_a
      schur = lambda z: z * diag_b - vjp_gf(inv_ff(vjp_fg(z)))
      schur_t = None if symmetric else (lambda z: z * diag_b - vjp_fgt(inv_ff(vjp_gft(z))))
      res = gr_g - vjp_gf(inv_ff(gr_f))
      sch = solver(schur, res, schur_t, symmetric, **kw)
      return inv_ff(gr_f - vjp_fg(sch)), sch
    inv_gg = lambda z: z / diag_b
    schur = lambda z: z * diag_a - vjp_fg(inv_gg(vjp_gf(z)))
    schur_t = None if symmetric else (lambda z: z * diag_a - vjp_gft(inv_gg(vjp_fgt(z))))
    res = gr_f - vjp_fg(inv_gg(gr_g))
    sch = solver(schur, res, schur_t, symmetric, **kw)
    return sch, inv_gg(gr_g - vjp_gf(sch))

  # -- the pullback ------------------------------------------------------------
  def gradient(self, prob, f: torch.Tensor, g: torch.Tensor, lse_mode: bool,
               gr: Tuple[torch.Tensor, torch.Tensor], precision: str = "fp32"
               ) -> Tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
    """implicit_differentiation.py:275-287: the cotangent of the inputs
    ``(x, y, a, b)`` (float64) for the cotangent ``gr`` of ``(f, g)``:
    ``lam = solve(gr)`` pulled back through the first-order conditions at
    fixed ``f, g`` (``d h(P 1)_i / dP_ij = h'(P 1)_i``, ``dP_ij/dC_ij =
    -P_ij / eps``; ``d/da_i = -lam_i h'(a_i)`` on ``a > 0``)."""
    lam, ma, mb = self._solve(gr, prob, f, g, lse_mode, precision)
    geom = prob.geom
    n, m = geom.shape
    dev = f.device
    la, lb = lam[:n], lam[n:]
    a, b = prob.a.detach().double(), prob.b.detach().double()
    zero = torch.zeros((), dtype=torch.float64, device=dev)
    sa, sb = (a > 0) & (ma > 0), (b > 0) & (mb > 0)
    one = lambda v, s: torch.where(s, v, torch.ones_like(v))
    alpha1 = torch.where(sa, la * self._derivative(geom, one(ma, sa)), zero)
    beta2 = torch.where(sb, lb * self._derivative(geom, one(mb, sb)), zero)
    alpha = torch.stack([alpha1, torch.ones(n, dtype=torch.float64, device=dev)])
    beta = torch.stack([torch.ones(m, dtype=torch.float64, device=dev), beta2])
    gx, gy, _, _ = geom._plan_vjp(f, g, alpha, beta, points=True, precision=precision)
    ga = torch.where(a > 0, -la * self._derivative(geom, one(a, a > 0)), zero)
    gb = torch.where(b > 0, -lb * self._derivative(geom, one(b, b > 0)), zero)
    return gx, gy, ga, gb
