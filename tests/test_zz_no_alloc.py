"""ottb_sinkhorn_pointcloud_noalloc: the solve for callers that cannot
allocate device memory where they call the solver (a handler inside a host
framework that only passes it input and output buffers, or a service whose
GPU memory budget is fixed at start-up).

It runs the same solve as ottb_sinkhorn_pointcloud with its scratch in a
16 MiB array compiled into the library. These tests call both entry points
through the C ABI on the same inputs and check that two no-allocation calls
in a row each match the standard call within the parity tolerances used
throughout the tests (potentials within 1e-4 * epsilon, reg_ot_cost within
1e-5 relative, identical iteration counts and error pattern), and that a
problem too large for the fixed scratch is refused before any work is
enqueued. This file is named to be collected last.
"""
import ctypes
import math

import numpy as np
import pytest

from tests import problems

pytestmark = pytest.mark.gpu


def _lib():
  from ott_b200 import _lib as L
  lib = L.load()
  fn = lib.ottb_sinkhorn_pointcloud_noalloc
  fn.argtypes = [ctypes.POINTER(L.OttbProblem), ctypes.c_int32, ctypes.c_int32,
                 ctypes.POINTER(L.OttbSolverCfg), ctypes.c_void_p, ctypes.c_void_p]
  fn.restype = ctypes.c_int32
  return L, lib


def _cfg(L):
  return L.OttbSolverCfg(threshold=1e-3, norm_error=1, inner_iterations=10,
                         min_iterations=0, max_iterations=2000, eps_init=1.0,
                         eps_decay=1.0, precision=-1, mask_init=0, timeout_ms=0,
                         phantom_arrivals=0)


def _inputs(torch, specs):
  """Device tensors of each (x, y, a, b, epsilon) problem."""
  out = []
  for x, y, a, b, eps in specs:
    out.append(dict(x=torch.as_tensor(x).cuda(), y=torch.as_tensor(y).cuda(),
                    a=torch.as_tensor(a).cuda(), b=torch.as_tensor(b).cuda(), eps=eps))
  return out


def _run(torch, L, lib, inputs, noalloc):
  """One call over all problems; returns host copies of every output."""
  outer = math.ceil(2000 / 10)
  arr = (L.OttbProblem * len(inputs))()
  outs = []
  for k, p in enumerate(inputs):
    n, m = p["x"].shape[0], p["y"].shape[0]
    f = torch.full((n,), float("nan"), device="cuda")
    g = torch.full((m,), float("nan"), device="cuda")
    e = torch.full((outer,), float("nan"), device="cuda")
    q = arr[k]
    q.x, q.y = p["x"].data_ptr(), p["y"].data_ptr()
    q.a, q.b = p["a"].data_ptr(), p["b"].data_ptr()
    q.f_init = q.g_init = None
    q.f, q.g, q.errors = f.data_ptr(), g.data_ptr(), e.data_ptr()
    q.n, q.m = n, m
    q.epsilon, q.inv_scale_cost = p["eps"], 1.0
    outs.append((f, g, e))
  d = inputs[0]["x"].shape[1]
  cfg = _cfg(L)
  res = torch.zeros(len(inputs) * L.RESULT_BYTES, dtype=torch.uint8, device="cuda")
  stream = torch.cuda.current_stream().cuda_stream
  if noalloc:
    st = lib.ottb_sinkhorn_pointcloud_noalloc(arr, len(inputs), d, ctypes.byref(cfg),
                                              res.data_ptr(), stream)
  else:
    ws_bytes = lib.ottb_sinkhorn_workspace_size(arr, len(inputs), d, ctypes.byref(cfg))
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device="cuda")
    st = lib.ottb_sinkhorn_pointcloud(arr, len(inputs), d, ctypes.byref(cfg),
                                      res.data_ptr(), ws.data_ptr(), ws_bytes, stream)
  assert st == L.OTTB_OK, L.status_string(st)
  torch.cuda.synchronize()
  raw = res.cpu().numpy().tobytes()
  results = [L.OttbResult.from_buffer_copy(raw[i * L.RESULT_BYTES:(i + 1) * L.RESULT_BYTES])
             for i in range(len(inputs))]
  return [(f.cpu().numpy(), g.cpu().numpy(), e.cpu().numpy(), r)
          for (f, g, e), r in zip(outs, results)]


def _assert_close(a, b, eps):
  fa, ga, ea, ra = a
  fb, gb, eb, rb = b
  assert ra.status == 0 and rb.status == 0
  assert ra.n_iters == rb.n_iters and ra.converged == rb.converged
  np.testing.assert_array_equal(np.isfinite(fa), np.isfinite(fb))
  np.testing.assert_array_equal(np.isfinite(ga), np.isfinite(gb))
  ff, gf = np.isfinite(fb), np.isfinite(gb)
  np.testing.assert_allclose(fa[ff], fb[ff], rtol=0, atol=1e-4 * eps)
  np.testing.assert_allclose(ga[gf], gb[gf], rtol=0, atol=1e-4 * eps)
  np.testing.assert_allclose(ra.reg_ot_cost, rb.reg_ot_cost, rtol=1e-5)
  np.testing.assert_array_equal(ea == -1, eb == -1)
  np.testing.assert_array_equal(np.isinf(ea), np.isinf(eb))


def test_noalloc_matches_standard_entry_point_twice():
  import torch
  L, lib = _lib()
  x1, y1, a1, b1 = problems.ref_test_problem()                     # zero weights
  x2, y2, a2, b2 = problems.uniform_cloud_problem(3000, 2500, 3, seed=11)
  specs = [(x1, y1, a1, b1, 0.1), (x2, y2, a2, b2, 0.02)]
  inputs = _inputs(torch, specs)
  ref = _run(torch, L, lib, inputs, noalloc=False)
  first = _run(torch, L, lib, inputs, noalloc=True)
  second = _run(torch, L, lib, inputs, noalloc=True)
  for k, (_, _, _, _, eps) in enumerate(specs):
    _assert_close(first[k], ref[k], eps)
    _assert_close(second[k], ref[k], eps)
  # single problem: a different plan (column splits) in the same scratch
  inputs = _inputs(torch, [specs[1]])
  ref = _run(torch, L, lib, inputs, noalloc=False)
  for _ in range(2):
    _assert_close(_run(torch, L, lib, inputs, noalloc=True)[0], ref[0], 0.02)


def test_noalloc_refuses_problems_beyond_its_scratch():
  import torch
  L, lib = _lib()
  n = m = 200_000
  d = 64
  x = torch.zeros((n, d), device="cuda")
  y = torch.zeros((m, d), device="cuda")
  a = torch.full((n,), 1.0 / n, device="cuda")
  b = torch.full((m,), 1.0 / m, device="cuda")
  f = torch.empty(n, device="cuda")
  g = torch.empty(m, device="cuda")
  e = torch.empty(200, device="cuda")
  arr = (L.OttbProblem * 1)()
  q = arr[0]
  q.x, q.y, q.a, q.b = x.data_ptr(), y.data_ptr(), a.data_ptr(), b.data_ptr()
  q.f, q.g, q.errors = f.data_ptr(), g.data_ptr(), e.data_ptr()
  q.n, q.m, q.epsilon, q.inv_scale_cost = n, m, 1.0, 1.0
  cfg = _cfg(L)
  need = lib.ottb_sinkhorn_workspace_size(arr, 1, d, ctypes.byref(cfg))
  assert need > 16 * 1024 * 1024
  res = torch.zeros(L.RESULT_BYTES, dtype=torch.uint8, device="cuda")
  st = lib.ottb_sinkhorn_pointcloud_noalloc(arr, 1, d, ctypes.byref(cfg), res.data_ptr(),
                                            torch.cuda.current_stream().cuda_stream)
  assert st == L.OTTB_ERR_WORKSPACE
  torch.cuda.synchronize()


def test_noalloc_calls_leave_free_device_memory_unchanged():
  """The entry point's own claim: after one call (the address look-up and
  module load), further calls change neither the device's free memory
  (cudaMemGetInfo) nor torch's allocated bytes. Every buffer the calls use
  is made before the first reading."""
  import torch
  L, lib = _lib()
  x, y, a, b = problems.uniform_cloud_problem(3000, 2500, 3, seed=11)
  p = _inputs(torch, [(x, y, a, b, 0.02)])[0]
  n, m = x.shape[0], y.shape[0]
  f = torch.empty(n, device="cuda")
  g = torch.empty(m, device="cuda")
  e = torch.empty(200, device="cuda")
  arr = (L.OttbProblem * 1)()
  q = arr[0]
  q.x, q.y, q.a, q.b = p["x"].data_ptr(), p["y"].data_ptr(), p["a"].data_ptr(), p["b"].data_ptr()
  q.f_init = q.g_init = None
  q.f, q.g, q.errors = f.data_ptr(), g.data_ptr(), e.data_ptr()
  q.n, q.m, q.epsilon, q.inv_scale_cost = n, m, 0.02, 1.0
  cfg = _cfg(L)
  res = torch.zeros(L.RESULT_BYTES, dtype=torch.uint8, device="cuda")
  stream = torch.cuda.current_stream().cuda_stream

  def call():
    st = lib.ottb_sinkhorn_pointcloud_noalloc(arr, 1, 3, ctypes.byref(cfg), res.data_ptr(),
                                              stream)
    assert st == L.OTTB_OK, L.status_string(st)

  call()
  torch.cuda.synchronize()
  free0, _ = torch.cuda.mem_get_info()
  alloc0 = torch.cuda.memory_allocated()
  call()
  call()
  torch.cuda.synchronize()
  free1, _ = torch.cuda.mem_get_info()
  assert free1 == free0, (free0, free1)
  assert torch.cuda.memory_allocated() == alloc0
  r = L.OttbResult.from_buffer_copy(res.cpu().numpy().tobytes()[:L.RESULT_BYTES])
  assert r.status == 0 and r.n_iters > 0
