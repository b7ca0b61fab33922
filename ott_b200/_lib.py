"""ctypes binding of the ott_b200 C ABI (``include/ott_b200.h``).

The shared library is built in-tree (``ott_b200/_lib/libottb200.so``) by
``ott_b200.build``. There is no fallback: if the library or a CUDA device is
missing, calls raise.
"""
from __future__ import annotations

import ctypes
import os
import threading
from typing import Optional

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libottb200.so")

OTTB_OK = 0
OTTB_ERR_INVALID = 1
OTTB_ERR_UNSUPPORTED = 2
OTTB_ERR_CUDA = 3
OTTB_ERR_TIMEOUT = 4
OTTB_ERR_WORKSPACE = 5
OTTB_ERR_NO_DEVICE = 6
OTTB_ERR_HOST_MEMORY = 7

PRECISION_AUTO = -1
PRECISION_FP32 = 0
PRECISION_BF16_SPLIT3 = 1

EXPORTED_SYMBOLS = (
    "ottb_sinkhorn_workspace_size",
    "ottb_sinkhorn_pointcloud",
    "ottb_sinkhorn_prepare",
    "ottb_sinkhorn_launch",
    "ottb_sinkhorn_autotune",
    "ottb_sinkhorn_set_schedule",
    "ottb_apply_transport_workspace_size",
    "ottb_apply_transport",
    "ottb_apply_transport_tc_workspace_size",
    "ottb_apply_transport_tc",
    "ottb_apply_transport_sweep_workspace_size",
    "ottb_apply_transport_sweep",
    "ottb_apply_lse_kernel_workspace_size",
    "ottb_apply_transport_plan",
    "ottb_apply_transport_run",
    "ottb_apply_transport_free",
    "ottb_apply_transport_sweep_plan",
    "ottb_apply_transport_sweep_run",
    "ottb_apply_transport_sweep_free",
    "ottb_apply_lse_kernel",
    "ottb_minres_step",
    "ottb_minres_step_next",
    "ottb_transport_matrix",
    "ottb_cost_stats_workspace_size",
    "ottb_cost_stats",
    "ottb_sinkhorn_pointcloud_noalloc",
    "ottb_mlp_workspace_size",
    "ottb_mlp_forward",
    "ottb_mlp_gradients",
    "ottb_mlp_adam",
    "ottb_mlp_adam_device",
    "ottb_mlp_sync_bf16",
    "ottb_status_string",
    "ottb_version",
)


class OttbProblem(ctypes.Structure):
  _fields_ = [
      ("x", ctypes.c_void_p),
      ("y", ctypes.c_void_p),
      ("a", ctypes.c_void_p),
      ("b", ctypes.c_void_p),
      ("f_init", ctypes.c_void_p),
      ("g_init", ctypes.c_void_p),
      ("f", ctypes.c_void_p),
      ("g", ctypes.c_void_p),
      ("errors", ctypes.c_void_p),
      ("n", ctypes.c_int64),
      ("m", ctypes.c_int64),
      ("epsilon", ctypes.c_float),
      ("inv_scale_cost", ctypes.c_float),
      ("symmetric", ctypes.c_int32),
      ("reserved", ctypes.c_int32),
  ]


class OttbSolverCfg(ctypes.Structure):
  _fields_ = [
      ("threshold", ctypes.c_float),
      ("norm_error", ctypes.c_int32),
      ("inner_iterations", ctypes.c_int32),
      ("min_iterations", ctypes.c_int32),
      ("max_iterations", ctypes.c_int32),
      ("eps_init", ctypes.c_float),
      ("eps_decay", ctypes.c_float),
      ("precision", ctypes.c_int32),
      ("mask_init", ctypes.c_int32),
      ("timeout_ms", ctypes.c_int32),
      ("phantom_arrivals", ctypes.c_int32),
      ("init_f_from_g", ctypes.c_int32),
  ]


class OttbResult(ctypes.Structure):
  _fields_ = [
      ("reg_ot_cost", ctypes.c_double),
      ("marginal_sum", ctypes.c_double),
      ("n_iters", ctypes.c_int32),
      ("converged", ctypes.c_int32),
      ("status", ctypes.c_int32),
      ("reserved", ctypes.c_int32),
  ]


MLP_MAX_LAYERS = 8


class OttbMlpLayer(ctypes.Structure):
  _fields_ = [("in_", ctypes.c_int32), ("out", ctypes.c_int32)] + [
      (name, ctypes.c_void_p) for name in
      ("w", "w_bf16", "wt_bf16", "b", "w_m", "w_v", "b_m", "b_v", "w_grad", "b_grad")]


class OttbMlp(ctypes.Structure):
  _fields_ = [("num_layers", ctypes.c_int32), ("layers", OttbMlpLayer * MLP_MAX_LAYERS)]


RESULT_BYTES = ctypes.sizeof(OttbResult)

_NP_CODES = {ctypes.c_void_p: "<u8", ctypes.c_int64: "<i8", ctypes.c_int32: "<i4",
             ctypes.c_float: "<f4", ctypes.c_double: "<f8"}


def numpy_dtype(struct) -> "np.dtype":
  """NumPy structured dtype with the layout of a flat ctypes Structure."""
  import numpy as np
  names, formats, offsets = [], [], []
  for name, ctype in struct._fields_:
    names.append(name)
    formats.append(_NP_CODES[ctype])
    offsets.append(getattr(struct, name).offset)
  return np.dtype({"names": names, "formats": formats, "offsets": offsets,
                   "itemsize": ctypes.sizeof(struct)})

_lock = threading.Lock()
_lib: Optional[ctypes.CDLL] = None


class OttbError(RuntimeError):
  """A C-ABI call returned a non-OK status."""

  def __init__(self, status: int, what: str):
    self.status = status
    super().__init__(f"{what}: {status_string(status)} (status {status})")


def load() -> ctypes.CDLL:
  """Loads the library (once). Raises if it has not been built."""
  global _lib
  with _lock:
    if _lib is not None:
      return _lib
    if not os.path.exists(LIB_PATH):
      raise RuntimeError(
          f"libottb200.so not found at {LIB_PATH}; build it with "
          "`python -m ott_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    vp, sz, i32, i64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32, ctypes.c_int64
    lib.ottb_sinkhorn_workspace_size.argtypes = [
        ctypes.POINTER(OttbProblem), i32, i32, ctypes.POINTER(OttbSolverCfg)]
    lib.ottb_sinkhorn_workspace_size.restype = sz
    lib.ottb_sinkhorn_pointcloud.argtypes = [
        ctypes.POINTER(OttbProblem), i32, i32, ctypes.POINTER(OttbSolverCfg),
        vp, vp, sz, vp]
    lib.ottb_sinkhorn_pointcloud.restype = i32
    lib.ottb_sinkhorn_prepare.argtypes = [
        ctypes.POINTER(OttbProblem), i32, i32, ctypes.POINTER(OttbSolverCfg), vp, sz, vp]
    lib.ottb_sinkhorn_prepare.restype = i32
    lib.ottb_sinkhorn_launch.argtypes = [
        ctypes.POINTER(OttbProblem), i32, i32, ctypes.POINTER(OttbSolverCfg),
        vp, vp, sz, vp]
    lib.ottb_sinkhorn_launch.restype = i32
    lib.ottb_sinkhorn_autotune.argtypes = [
        ctypes.POINTER(OttbProblem), i32, i32, ctypes.POINTER(OttbSolverCfg),
        vp, vp, sz, vp, i32]
    lib.ottb_sinkhorn_autotune.restype = i32
    lib.ottb_sinkhorn_set_schedule.argtypes = [
        ctypes.POINTER(OttbProblem), i32, i32, ctypes.POINTER(OttbSolverCfg), i32, i32, i32, i32]
    lib.ottb_sinkhorn_set_schedule.restype = i32
    f32_ = ctypes.c_float
    lib.ottb_apply_transport_workspace_size.argtypes = [i64, i64, i32, i32, i32]
    lib.ottb_apply_transport_workspace_size.restype = sz
    lib.ottb_apply_transport.argtypes = [vp, vp, i64, i64, i32, vp, vp, f32_, f32_, vp, i32,
                                         i32, vp, vp, sz, vp]
    lib.ottb_apply_transport.restype = i32
    lib.ottb_apply_transport_tc_workspace_size.argtypes = [i64, i64, i32, i32, i32]
    lib.ottb_apply_transport_tc_workspace_size.restype = sz
    lib.ottb_apply_transport_tc.argtypes = [vp, vp, i64, i64, i32, vp, vp, f32_, f32_, vp, i32,
                                            i32, vp, vp, sz, vp]
    lib.ottb_apply_transport_tc.restype = i32
    lib.ottb_apply_transport_sweep_workspace_size.argtypes = [i64, i64, i32, i32, i32, i32]
    lib.ottb_apply_transport_sweep_workspace_size.restype = sz
    lib.ottb_apply_transport_sweep.argtypes = [vp, vp, i64, i64, i32, vp, vp, f32_, f32_, vp,
                                               i32, i32, i32, vp, vp, sz, vp]
    lib.ottb_apply_transport_sweep.restype = i32
    lib.ottb_apply_lse_kernel_workspace_size.argtypes = [i64, i64, i32, i32, i32]
    lib.ottb_apply_lse_kernel_workspace_size.restype = sz
    lib.ottb_apply_lse_kernel.argtypes = [vp, vp, i64, i64, i32, vp, f32_, f32_, i32, i32, vp,
                                          vp, sz, vp]
    lib.ottb_apply_lse_kernel.restype = i32
    lib.ottb_apply_transport_plan.argtypes = [vp, vp, i64, i64, i32, vp, vp, f32_, f32_, i32,
                                              i32, vp, sz, vp, ctypes.POINTER(ctypes.c_void_p)]
    lib.ottb_apply_transport_plan.restype = i32
    lib.ottb_apply_transport_run.argtypes = [vp, vp, vp, vp]
    lib.ottb_apply_transport_run.restype = i32
    lib.ottb_apply_transport_free.argtypes = [vp]
    lib.ottb_apply_transport_free.restype = None
    lib.ottb_apply_transport_sweep_plan.argtypes = [vp, vp, i64, i64, i32, vp, vp, f32_, f32_,
                                                    i32, i32, i32, vp, sz, vp,
                                                    ctypes.POINTER(ctypes.c_void_p)]
    lib.ottb_apply_transport_sweep_plan.restype = i32
    lib.ottb_apply_transport_sweep_run.argtypes = [vp, vp, vp, vp, vp]
    lib.ottb_apply_transport_sweep_run.restype = i32
    lib.ottb_apply_transport_sweep_free.argtypes = [vp]
    lib.ottb_apply_transport_sweep_free.restype = None
    lib.ottb_minres_step.argtypes = [vp, i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64,
                                     i64, vp]
    lib.ottb_minres_step.restype = i32
    lib.ottb_minres_step_next.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, i64, i64,
                                          vp]
    lib.ottb_minres_step_next.restype = i32
    lib.ottb_transport_matrix.argtypes = [vp, vp, i64, i64, i32, vp, vp, f32_, f32_, vp, vp]
    lib.ottb_transport_matrix.restype = i32
    lib.ottb_cost_stats_workspace_size.argtypes = [i64, i64, i32]
    lib.ottb_cost_stats_workspace_size.restype = sz
    lib.ottb_cost_stats.argtypes = [vp, vp, i64, i64, i32, ctypes.c_float, i32, vp, vp, sz, vp]
    lib.ottb_cost_stats.restype = i32
    mlp = ctypes.POINTER(OttbMlp)
    f32 = ctypes.c_float
    lib.ottb_mlp_workspace_size.argtypes = [mlp, i32]
    lib.ottb_mlp_workspace_size.restype = sz
    lib.ottb_mlp_forward.argtypes = [mlp, vp, i32, vp, vp, vp, sz, vp]
    lib.ottb_mlp_forward.restype = i32
    lib.ottb_mlp_gradients.argtypes = [mlp, vp, vp, vp, i32, vp, vp, vp, sz, vp]
    lib.ottb_mlp_gradients.restype = i32
    lib.ottb_mlp_adam.argtypes = [mlp, f32, f32, f32, f32, i32, vp]
    lib.ottb_mlp_adam.restype = i32
    lib.ottb_mlp_adam_device.argtypes = [mlp, vp, f32, f32, f32, vp]
    lib.ottb_mlp_adam_device.restype = i32
    lib.ottb_mlp_sync_bf16.argtypes = [mlp, vp]
    lib.ottb_mlp_sync_bf16.restype = i32
    lib.ottb_status_string.argtypes = [i32]
    lib.ottb_status_string.restype = ctypes.c_char_p
    lib.ottb_version.argtypes = []
    lib.ottb_version.restype = ctypes.c_char_p
    _lib = lib
    return lib


def status_string(status: int) -> str:
  try:
    return load().ottb_status_string(int(status)).decode()
  except Exception:  # library not loadable: still give a message
    return f"status {status}"


def check(status: int, what: str) -> None:
  if status != OTTB_OK:
    raise OttbError(status, what)
