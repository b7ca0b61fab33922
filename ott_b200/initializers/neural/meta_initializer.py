"""Learned Sinkhorn initializer on a fixed support
(ott/initializers/neural/meta_initializer.py:36-213).

The network maps the measure weights concat(a, b) to a dual potential. The
reference's meta model predicts f (``init_fu``, :137-158) and trains it on
the dual objective (:160-190). Here the network predicts g, regressed on the
centred g of problems solved by the plain kernel. The solver then starts
with one f-update from that g (its c-transform,
``ottb_solver_cfg.init_f_from_g``), because a g alone would be discarded by
the first g-update of the loop. Forward, backward and Adam run in this
library's tcgen05 bf16 kernels (``ottb_mlp_*``).
"""
from __future__ import annotations

import ctypes
import math
from typing import Optional, Sequence

import numpy as np
import torch

from ott_b200 import _arrays, _lib
from ott_b200.initializers.linear import initializers


class MLP:
  """Dense layers with tanh-GELU between them, parameters on the device.

  Initialisation follows flax ``nn.Dense`` defaults: weights from a
  truncated normal with variance 1 / fan_in (lecun normal), zero biases.
  """

  def __init__(self, dims: Sequence[int], seed: int = 0, device=None):
    self.dims = list(dims)
    dev = device or _arrays.device()
    rng = np.random.default_rng(seed)
    self.tensors = []
    self.net = _lib.OttbMlp()
    self.net.num_layers = len(dims) - 1
    for l in range(len(dims) - 1):
      fan_in, fan_out = dims[l], dims[l + 1]
      std = np.sqrt(1.0 / fan_in) / 0.87962566103423978  # truncated-normal variance fix
      w0 = np.clip(rng.standard_normal((fan_out, fan_in)), -2, 2) * std
      t = dict(
          w=torch.tensor(w0, dtype=torch.float32, device=dev),
          w_bf16=torch.empty((fan_out, fan_in), dtype=torch.bfloat16, device=dev),
          wt_bf16=torch.empty((fan_in, fan_out), dtype=torch.bfloat16, device=dev),
          b=torch.zeros(fan_out, dtype=torch.float32, device=dev),
          w_m=torch.zeros((fan_out, fan_in), dtype=torch.float32, device=dev),
          w_v=torch.zeros((fan_out, fan_in), dtype=torch.float32, device=dev),
          b_m=torch.zeros(fan_out, dtype=torch.float32, device=dev),
          b_v=torch.zeros(fan_out, dtype=torch.float32, device=dev),
          w_grad=torch.zeros((fan_out, fan_in), dtype=torch.float32, device=dev),
          b_grad=torch.zeros(fan_out, dtype=torch.float32, device=dev))
      self.tensors.append(t)
      ly = self.net.layers[l]
      ly.in_, ly.out = fan_in, fan_out
      for k, v in t.items():
        setattr(ly, k, v.data_ptr())
    self.lib = _lib.load()
    self.status = torch.zeros(1, dtype=torch.int32, device=dev)
    self.step = 0
    self._ws = {}
    _lib.check(self.lib.ottb_mlp_sync_bf16(ctypes.byref(self.net), _arrays.stream_handle()),
               "ottb_mlp_sync_bf16")

  def _workspace(self, batch: int) -> torch.Tensor:
    if batch not in self._ws:
      nbytes = self.lib.ottb_mlp_workspace_size(ctypes.byref(self.net), batch)
      if nbytes == 0:
        raise ValueError(f"batch {batch} and widths {self.dims} must be multiples of 128")
      self._ws[batch] = torch.empty(nbytes, dtype=torch.uint8, device=self.status.device)
    return self._ws[batch]

  def params_numpy(self):
    return [(t["w"].double().cpu().numpy(), t["b"].double().cpu().numpy()) for t in self.tensors]

  def forward(self, x: torch.Tensor) -> torch.Tensor:
    x = x.contiguous().float()
    batch = x.shape[0]
    y = torch.empty((batch, self.dims[-1]), dtype=torch.float32, device=x.device)
    ws = self._workspace(batch)
    st = self.lib.ottb_mlp_forward(ctypes.byref(self.net), x.data_ptr(), batch, y.data_ptr(),
                                   self.status.data_ptr(), ws.data_ptr(), ws.numel(),
                                   _arrays.stream_handle())
    _lib.check(st, "ottb_mlp_forward")
    return y

  def gradients(self, x: torch.Tensor, target: torch.Tensor,
                weight: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Gradients of the centred squared error into the layers' w_grad /
    b_grad (``weight``: per-entry weights, or None for 1). Returns the
    per-sample losses."""
    x = x.contiguous().float()
    target = target.contiguous().float()
    if weight is not None:
      weight = weight.contiguous().float()
    batch = x.shape[0]
    loss = torch.empty(batch, dtype=torch.float32, device=x.device)
    ws = self._workspace(batch)
    st = self.lib.ottb_mlp_gradients(ctypes.byref(self.net), x.data_ptr(), target.data_ptr(),
                                     None if weight is None else weight.data_ptr(),
                                     batch, loss.data_ptr(), self.status.data_ptr(),
                                     ws.data_ptr(), ws.numel(), _arrays.stream_handle())
    _lib.check(st, "ottb_mlp_gradients")
    return loss

  def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    self.step += 1
    _lib.check(self.lib.ottb_mlp_adam(ctypes.byref(self.net), lr, b1, b2, eps, self.step,
                                      _arrays.stream_handle()), "ottb_mlp_adam")

  def adam_device(self, hyper: torch.Tensor, b1=0.9, b2=0.999, eps=1e-8):
    """An Adam step whose learning rate and bias corrections are read from
    the device (``hyper`` = float32 ``[lr, 1 - b1^t, 1 - b2^t]``), for a
    step captured in a CUDA graph; the caller keeps the step count."""
    _lib.check(self.lib.ottb_mlp_adam_device(ctypes.byref(self.net), hyper.data_ptr(), b1, b2,
                                             eps, _arrays.stream_handle()),
               "ottb_mlp_adam_device")

  def check_status(self):
    st = int(self.status.item())
    if st != _lib.OTTB_OK:
      raise _lib.OttbError(st, "ottb_mlp (device)")


class MetaInitializer(initializers.SinkhornInitializer):
  """Meta-OT initializer for problems on one fixed support.

  The network output h is read as g = eps log b + h: g_j - eps log b_j is
  the soft c-transform of f, a smooth function of the support point, while
  eps log b_j carries the sharp dependence on the weights (b has a 1e-6
  floor in the grid workload: eps log b spans ~0.14 there). The regression
  is on centred h (potentials are defined up to a constant), each entry
  weighted by m b_j + ``mass_floor``: errors of g where b_j is tiny barely
  move the c-transform f = -eps lse_j((g_j - C_ij) / eps) + eps log a_i
  that the solver starts from.

  Args:
    geom: the fixed geometry (n and m multiples of 128).
    dims: hidden widths; the network is (n + m) -> dims... -> m.
    lr: Adam learning rate (the reference's default, 1e-3).
    seed: initialisation seed.
    mass_floor: additive floor of the loss weights (None: unweighted).
  """

  half_step_from_g = True

  def __init__(self, geom, dims: Sequence[int] = (1024, 1024, 1024), lr: float = 1e-3,
               seed: int = 0, mass_floor: Optional[float] = 0.1):
    self.geom = geom
    n, m = geom.shape
    self.lr = lr
    self.mass_floor = mass_floor
    self.mlp = MLP([n + m, *dims, m], seed=seed, device=geom.x.device)

  def _inputs(self, a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    # concat(a, b) as in _compute_f (:192-207), scaled by the support sizes
    # so that a uniform measure reads 1: raw weights of a 1024-point support
    # are ~1e-3, far below the scale the initialisation expects.
    n, m = self.geom.shape
    a2 = a if a.ndim == 2 else a[None]
    b2 = b if b.ndim == 2 else b[None]
    return torch.cat([a2 * n, b2 * m], dim=1).float()

  def _eps_log(self, b: torch.Tensor) -> torch.Tensor:
    b2 = (b if b.ndim == 2 else b[None]).float()
    return float(self.geom.epsilon) * torch.log(b2)

  def _loss_gradients(self, a: torch.Tensor, b: torch.Tensor,
                      g_target: torch.Tensor) -> torch.Tensor:
    """Network inputs, regression targets and weights of a batch, then the
    gradients into the layers; returns the per-sample losses."""
    x = self._inputs(a, b)
    b = b.float()
    pos = b > 0
    t = torch.where(pos, g_target.float() - self._eps_log(b), torch.zeros_like(b))
    m = b.shape[1]
    w = pos.float() if self.mass_floor is None else pos * (m * b + self.mass_floor)
    return self.mlp.gradients(x, t, w)

  def update(self, a: torch.Tensor, b: torch.Tensor, g_target: torch.Tensor) -> torch.Tensor:
    """One Adam step on a batch (batch a multiple of 128) regressing the g
    of solved problems. Returns the batch-mean loss (device scalar)."""
    loss = self._loss_gradients(a, b, g_target)
    self.mlp.adam(lr=self.lr)
    return loss.mean()

  def predict_g(self, a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    x = self._inputs(a, b)
    batch = x.shape[0]
    padded = (batch + 127) // 128 * 128
    if padded != batch:
      x = torch.cat([x, torch.zeros((padded - batch, x.shape[1]), device=x.device)], dim=0)
    return self.mlp.forward(x)[:batch] + self._eps_log(b)

  def stacked_init(self, a: torch.Tensor, b: torch.Tensor):
    """(None, G) for stacked weights a [K, n], b [K, m]: one network call."""
    return None, self.predict_g(a, b)

  def batch_init(self, probs, **unused):
    """One network call for a batch of problems: [(None, g_k)]."""
    a = torch.stack([p.a for p in probs])
    b = torch.stack([p.b for p in probs])
    g = self.predict_g(a, b)
    return [(None, g[k]) for k in range(len(probs))]

  def init_fu(self, ot_prob, lse_mode: bool, rng=None):
    return None  # derived in the solver from g (init_f_from_g)

  def init_gv(self, ot_prob, lse_mode: bool, rng=None):
    return self.predict_g(ot_prob.a, ot_prob.b)[0]


def fit(meta: MetaInitializer, a: torch.Tensor, b: torch.Tensor, g: torch.Tensor, steps: int,
        batch_size: int = 512, seed: int = 0, cosine: bool = True, log_every: int = 0,
        graph: bool = True):
  """Adam steps on random minibatches of solved problems (rows of a, b and
  their solved g), the learning rate decayed from ``meta.lr`` to 0 along a
  cosine when ``cosine``. Returns the per-step batch losses (device).

  With ``graph`` (and no ``log_every``) the first step runs directly and one
  training step (minibatch gather by a device step counter, inputs and
  targets, the MLP's forward and backward, Adam with the step's learning
  rate and bias corrections read from a device schedule) is captured in a
  CUDA graph and replayed for the others: the same kernels on the same
  values in the same order as the direct loop, without its ~40 host-side
  launches per step."""
  gen = torch.Generator(device="cpu").manual_seed(seed)
  num = a.shape[0]
  lr0 = meta.lr
  # every step's minibatch indices drawn at once and copied to the device
  # once (no host-to-device copy per step)
  idx_all = torch.randint(0, num, (steps, batch_size), generator=gen).to(a.device)
  lrs = [lr0 * 0.5 * (1.0 + math.cos(math.pi * s / steps)) if cosine else lr0
         for s in range(steps)]
  if not graph or log_every or steps < 2:
    losses = []
    for step in range(steps):
      meta.lr = lrs[step]
      idx = idx_all[step]
      losses.append(meta.update(a[idx], b[idx], g[idx]))
      if log_every and (step + 1) % log_every == 0:
        print(f"step {step + 1}: loss {float(losses[-1]):.3e}", flush=True)
    meta.lr = lr0
    return torch.stack(losses)
  mlp = meta.mlp
  b1, b2 = 0.9, 0.999
  t0 = mlp.step
  # Adam's schedule per step: lr, 1 - b1^t, 1 - b2^t, as ottb_mlp_adam
  # forms them (the float32 betas, powers in double, rounded once)
  fb1, fb2 = float(np.float32(b1)), float(np.float32(b2))
  hyper = torch.tensor(np.array(
      [[lrs[s], 1.0 - fb1 ** float(t0 + s + 1), 1.0 - fb2 ** float(t0 + s + 1)]
       for s in range(steps)], dtype=np.float64).astype(np.float32), device=a.device)
  losses = torch.empty(steps, dtype=torch.float32, device=a.device)
  step_t = torch.zeros(1, dtype=torch.int64, device=a.device)
  hyper_cur = torch.empty(3, dtype=torch.float32, device=a.device)

  def body():
    idx = idx_all.index_select(0, step_t).reshape(-1)
    loss = meta._loss_gradients(a.index_select(0, idx), b.index_select(0, idx),
                                g.index_select(0, idx))
    hyper_cur.copy_(hyper.index_select(0, step_t).reshape(-1))
    mlp.adam_device(hyper_cur, b1, b2)
    losses.index_copy_(0, step_t, loss.mean().reshape(1))
    step_t.add_(1)

  body()  # the first step, directly: also warms up every kernel
  side = torch.cuda.Stream()
  side.wait_stream(torch.cuda.current_stream())
  gr = torch.cuda.CUDAGraph()
  with torch.cuda.graph(gr, stream=side):
    body()
  torch.cuda.current_stream().wait_stream(side)
  for _ in range(steps - 1):
    gr.replay()
  mlp.step = t0 + steps
  return losses


def solve_warm_started(geom, a: torch.Tensor, b: torch.Tensor, meta: MetaInitializer,
                       budget: Optional[int] = None, **solver_kwargs):
  """Solves the stacked problems (a [K, n], b [K, m] on ``geom``) with the
  learned warm start; problems that have not converged within ``budget``
  iterations are solved again from the default initialisation with the
  full ``max_iterations`` (the plain solver stays the fallback and decides
  convergence).

  Returns (output, fallback_indices); the output's rows of the fallback
  problems hold the fallback solve.
  """
  from ott_b200.solvers.linear import sinkhorn
  max_it = solver_kwargs.get("max_iterations", 2000)
  warm_kw = dict(solver_kwargs, max_iterations=budget or max_it)
  out = sinkhorn.run_stacked(geom, a, b, sinkhorn.Sinkhorn(initializer=meta, **warm_kw))
  n_it, conv, cost = out.scalars()
  redo = np.nonzero(~conv)[0]
  if redo.size == 0:
    return out, redo
  idx = torch.as_tensor(redo, device=a.device)
  again = sinkhorn.run_stacked(geom, a[idx], b[idx], sinkhorn.Sinkhorn(**solver_kwargs))
  # merged output: warm rows, fallback rows replaced (iteration counts add up)
  f, g = out.f.clone(), out.g.clone()
  f[idx], g[idx] = again.f, again.g
  return _Merged(out, again, redo, f, g), redo


class _Merged:
  """A warm-started stacked output with its fallback rows replaced."""

  def __init__(self, warm, again, redo, f, g):
    self.f, self.g = f, g
    self._warm, self._again, self._redo = warm, again, redo

  def scalars(self):
    n_it, conv, cost = self._warm.scalars()
    n2, c2, cost2 = self._again.scalars()
    n_it = n_it.copy()
    n_it[self._redo] += n2  # the wasted warm iterations count too
    conv = conv.copy()
    conv[self._redo] = c2
    cost = cost.copy()
    cost[self._redo] = cost2
    return n_it, conv, cost
