"""Host-side checks of the C ABI that need no GPU: the library loads and
exports every function include/ott_b200.h declares."""
import ctypes
import os
import re

from ott_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
  text = open(os.path.join(ROOT, "include", "ott_b200.h")).read()
  text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
  names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(ottb_[a-z_0-9]+)\s*\(",
                     text, flags=re.M)
  return sorted(set(names))


def test_header_declares_expected_functions():
  names = declared_functions()
  assert set(_lib.EXPORTED_SYMBOLS) <= set(names), names


def test_library_exports_every_declared_symbol():
  lib = _lib.load()
  for name in declared_functions():
    assert hasattr(lib, name), name


def test_status_strings_and_version():
  lib = _lib.load()
  assert lib.ottb_version().decode().count(".") == 2
  for st in range(8):
    assert lib.ottb_status_string(st) != b"unknown status"
  assert lib.ottb_status_string(8) == b"unknown status"
  assert _lib.status_string(_lib.OTTB_ERR_TIMEOUT) == "device wait timed out"
  assert _lib.status_string(_lib.OTTB_ERR_HOST_MEMORY) == "host memory allocation failed"


def test_struct_layouts_match_header():
  # sizes follow from the C declarations on LP64
  assert ctypes.sizeof(_lib.OttbProblem) == 9 * 8 + 2 * 8 + 2 * 4 + 2 * 4
  assert ctypes.sizeof(_lib.OttbSolverCfg) == 12 * 4
  assert ctypes.sizeof(_lib.OttbResult) == 2 * 8 + 4 * 4
  assert ctypes.sizeof(_lib.OttbMlpLayer) == 2 * 4 + 10 * 8
  assert ctypes.sizeof(_lib.OttbMlp) == 8 + _lib.MLP_MAX_LAYERS * (2 * 4 + 10 * 8)


def test_numpy_record_views_match_ctypes():
  import numpy as np
  arr = (_lib.OttbProblem * 3)()
  rec = np.frombuffer(arr, dtype=_lib.numpy_dtype(_lib.OttbProblem))
  rec["n"] = [1, 2, 3]
  rec["b"] = np.arange(3, dtype=np.uint64) * 8 + 64
  rec["inv_scale_cost"] = 0.25
  assert [p.n for p in arr] == [1, 2, 3]
  assert arr[2].b == 80 and arr[1].inv_scale_cost == 0.25
  res = (_lib.OttbResult * 2)()
  res[1].n_iters, res[1].reg_ot_cost = 7, 1.5
  view = np.frombuffer(bytes(res), dtype=_lib.numpy_dtype(_lib.OttbResult))
  assert view["n_iters"][1] == 7 and view["reg_ot_cost"][1] == 1.5


def test_invalid_arguments_rejected_without_device():
  lib = _lib.load()
  cfg = _lib.OttbSolverCfg(threshold=1e-3, norm_error=1, inner_iterations=10,
                           min_iterations=0, max_iterations=100, eps_init=1.0,
                           eps_decay=1.0, precision=-1)
  # null problem array / zero problems -> 0 workspace
  assert lib.ottb_sinkhorn_workspace_size(None, 0, 2, ctypes.byref(cfg)) == 0
  st = lib.ottb_sinkhorn_pointcloud(None, 1, 2, ctypes.byref(cfg), None, None, 0, None)
  assert st == _lib.OTTB_ERR_INVALID
  assert lib.ottb_cost_stats(None, None, 0, 0, 2, ctypes.c_float(1.0), 1, None, None, 0,
                             None) == _lib.OTTB_ERR_INVALID
  one = ctypes.c_float(1.0)
  assert lib.ottb_apply_transport(None, None, 10, 10, 2, None, None, one, one, None, 1, 0, None,
                                  None, 0, None) == _lib.OTTB_ERR_INVALID
  assert lib.ottb_apply_transport_sweep(None, None, 10, 10, 2, None, None, one, one, None, 1,
                                        0, 1, None, None, 0, None) == _lib.OTTB_ERR_INVALID
  # workspace sizes: zero for invalid shapes or axes, d > 128 unsupported
  assert lib.ottb_apply_transport_sweep_workspace_size(0, 20, 64, 1, 0, 1) == 0
  assert lib.ottb_apply_transport_sweep_workspace_size(10, 20, 64, 1, 2, 1) == 0
  assert lib.ottb_apply_transport_sweep_workspace_size(10, 20, 200, 1, 0, 0) == 0
  ws_tc = lib.ottb_apply_transport_sweep_workspace_size(1000, 2000, 64, 1, 0, 1)
  assert ws_tc > 0 and ws_tc % 256 == 0
  # two zero-iteration problems per vector: more vectors, more workspace
  assert lib.ottb_apply_transport_sweep_workspace_size(1000, 2000, 64, 3, 0, 1) > ws_tc
  assert lib.ottb_apply_transport_workspace_size(1000, 2000, 64, 1, 3) == 0
  # planned FP32 products: no handle slot, a missing potential, d > 128 or
  # no vectors are refused before any launch and leave no handle
  hp = ctypes.c_void_p(99)
  assert lib.ottb_apply_transport_plan(4096, 4096, 10, 10, 8, 4096, 4096, one, one, 1, 0, 4096,
                                       1 << 20, None, None) == _lib.OTTB_ERR_INVALID
  assert lib.ottb_apply_transport_plan(4096, 4096, 10, 10, 8, 4096, None, one, one, 1, 0, 4096,
                                       1 << 20, None, ctypes.byref(hp)) == _lib.OTTB_ERR_INVALID
  assert hp.value is None
  assert lib.ottb_apply_transport_plan(4096, 4096, 10, 10, 200, 4096, 4096, one, one, 1, 0,
                                       4096, 1 << 20, None,
                                       ctypes.byref(hp)) == _lib.OTTB_ERR_UNSUPPORTED
  assert lib.ottb_apply_transport_plan(4096, 4096, 10, 10, 8, 4096, 4096, one, one, 0, 0, 4096,
                                       1 << 20, None, ctypes.byref(hp)) == _lib.OTTB_ERR_INVALID
  assert hp.value is None
  assert lib.ottb_apply_transport_run(None, 4096, 4096, None) == _lib.OTTB_ERR_INVALID
  lib.ottb_apply_transport_free(None)
  # planned sweep products: no handle slot, no bound potential of the output
  # side, a bad axis or an unaligned workspace are refused and leave no
  # handle; a run without a handle is refused; freeing NULL is a no-op
  h = ctypes.c_void_p(1234)
  fake = 4096
  assert lib.ottb_apply_transport_sweep_plan(fake, fake, 10, 10, 64, fake, fake, one, one, 1, 0,
                                             1, fake, 1 << 20, None, None) == _lib.OTTB_ERR_INVALID
  assert lib.ottb_apply_transport_sweep_plan(fake, fake, 10, 10, 64, fake, None, one, one, 1, 0,
                                             1, fake, 1 << 20, None,
                                             ctypes.byref(h)) == _lib.OTTB_ERR_INVALID
  assert h.value is None
  assert lib.ottb_apply_transport_sweep_plan(fake, fake, 10, 10, 64, None, fake, one, one, 1, 2,
                                             1, fake, 1 << 20, None,
                                             ctypes.byref(h)) == _lib.OTTB_ERR_INVALID
  assert lib.ottb_apply_transport_sweep_plan(fake, fake, 10, 10, 64, None, fake, one, one, 1, 0,
                                             1, fake + 8, 1 << 20, None,
                                             ctypes.byref(h)) == _lib.OTTB_ERR_WORKSPACE
  assert h.value is None
  assert lib.ottb_apply_transport_sweep_run(None, fake, fake, fake, None) == _lib.OTTB_ERR_INVALID
  lib.ottb_apply_transport_sweep_free(None)
  # MINRES step: null vectors, step outside [1, history_len), window < 1 or
  # an empty system are refused before any launch (the pointers below are
  # never dereferenced)
  p = [256 * (k + 1) for k in range(10)]
  def step(*, ptrs=p, step=1, window=50, hist_len=11, s=8):
    return lib.ottb_minres_step(ptrs[0], step, window, *ptrs[1:], hist_len, s, None)
  assert step(ptrs=[None] + p[1:]) == _lib.OTTB_ERR_INVALID
  assert step(ptrs=p[:5] + [None] + p[6:]) == _lib.OTTB_ERR_INVALID
  assert step(step=0) == _lib.OTTB_ERR_INVALID
  assert step(step=11) == _lib.OTTB_ERR_INVALID
  assert step(window=0) == _lib.OTTB_ERR_INVALID
  assert step(s=0) == _lib.OTTB_ERR_INVALID
  # the device-counted step: the same refusals, and a history of fewer than
  # two entries (no step fits)
  def step_next(*, ptrs=p, window=50, hist_len=11, s=8):
    return lib.ottb_minres_step_next(ptrs[0], window, *ptrs[1:], hist_len, s, None)
  assert step_next(ptrs=[None] + p[1:]) == _lib.OTTB_ERR_INVALID
  assert step_next(ptrs=p[:9] + [None]) == _lib.OTTB_ERR_INVALID
  assert step_next(hist_len=1) == _lib.OTTB_ERR_INVALID
  assert step_next(window=0) == _lib.OTTB_ERR_INVALID
  assert step_next(s=0) == _lib.OTTB_ERR_INVALID


def test_mlp_shape_checks_without_device():
  lib = _lib.load()
  net = _lib.OttbMlp()
  net.num_layers = 2
  net.layers[0].in_, net.layers[0].out = 256, 128
  net.layers[1].in_, net.layers[1].out = 128, 128
  ws = lib.ottb_mlp_workspace_size(ctypes.byref(net), 128)
  # bf16 input (+ transpose), one hidden layer's five bf16 buffers, fp32 output and
  # its bf16 gradient (+ transpose)
  assert ws == 2 * (2 * 128 * 256) + 5 * (2 * 128 * 128) + 4 * 128 * 128 + 2 * (2 * 128 * 128)
  assert lib.ottb_mlp_workspace_size(ctypes.byref(net), 100) == 0  # batch not a multiple of 128
  net.layers[1].in_ = 256  # widths must chain
  assert lib.ottb_mlp_workspace_size(ctypes.byref(net), 128) == 0
  assert lib.ottb_mlp_forward(None, None, 128, None, None, None, 0, None) == _lib.OTTB_ERR_INVALID
  assert lib.ottb_mlp_adam(ctypes.byref(net), 1e-3, 0.9, 0.999, 1e-8, 0, None) == \
      _lib.OTTB_ERR_INVALID
