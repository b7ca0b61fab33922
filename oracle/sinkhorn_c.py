"""ctypes wrapper of the C port of the oracle (test infrastructure only).

Built by ``make -C oracle`` into ``oracle/_build/``: the scalar restatement
``libsinkhorn_oracle.so`` and its tiled, vectorised form (the timed CPU
baseline), ``libsinkhorn_tiled_v4.so`` for AVX-512 hosts and
``libsinkhorn_tiled_v3.so`` for AVX2 hosts.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

from oracle import sinkhorn_np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_build", "libsinkhorn_oracle.so")
_libs = {}


def host_has_avx512() -> bool:
  try:
    with open("/proc/cpuinfo") as fh:
      for line in fh:
        if line.startswith("flags"):
          return "avx512f" in line.split()
  except OSError:
    pass
  return False


def library_path(variant="scalar") -> str:
  if variant == "scalar":
    return LIB
  if variant == "tiled":
    tag = "v4" if host_has_avx512() else "v3"
    return os.path.join(_HERE, "_build", f"libsinkhorn_tiled_{tag}.so")
  raise ValueError(f"unknown variant {variant!r}")


def load(variant="scalar"):
  if variant not in _libs:
    path = library_path(variant)
    if not os.path.exists(path):
      subprocess.run(["make", "-s", "-C", _HERE], check=True)
    lib = ctypes.CDLL(path)
    P = ctypes.c_void_p
    i64, i32, f32 = ctypes.c_int64, ctypes.c_int, ctypes.c_float
    lib.oracle_sinkhorn.argtypes = [P, P, P, P, i64, i64, i32, f32, f32, f32, f32, f32,
                                    i32, i32, i32, i32, P, P, P, P, P, P, P, P, i32]
    lib.oracle_sinkhorn.restype = i32
    lib.oracle_threads.restype = i32
    _libs[variant] = lib
  return _libs[variant]


def threads(variant="scalar") -> int:
  return int(load(variant).oracle_threads())


def solve(x, y, a, b, *, epsilon, inv_scale=1.0, eps_init=1.0, eps_decay=1.0,
          threshold=1e-3, norm_error=1, inner_iterations=10, min_iterations=0,
          max_iterations=2000, init=None, nthreads=0,
          variant="scalar") -> sinkhorn_np.SinkhornResult:
  """FP32 solve with ``epsilon`` already resolved (the C ABI's contract);
  ``variant`` "scalar" (the restatement) or "tiled" (the timed baseline)."""
  lib = load(variant)
  c = lambda v: np.ascontiguousarray(v, dtype=np.float32)
  x, y, a, b = c(x), c(y), c(a), c(b)
  n, d = x.shape
  m = y.shape[0]
  f = np.empty(n, np.float32)
  g = np.empty(m, np.float32)
  outer = max(1, int(math.ceil(max_iterations / inner_iterations)))
  errors = np.empty(outer, np.float32)
  cost = ctypes.c_double()
  nit = ctypes.c_int()
  conv = ctypes.c_int()
  fi = gi = None
  if init is not None:
    fi, gi = c(init[0]), c(init[1])
  ptr = lambda v: None if v is None else v.ctypes.data
  lib.oracle_sinkhorn(ptr(x), ptr(y), ptr(a), ptr(b), n, m, d, epsilon, inv_scale,
                      eps_init, eps_decay, threshold, norm_error, inner_iterations,
                      min_iterations, max_iterations, ptr(fi), ptr(gi), ptr(f), ptr(g),
                      ptr(errors), ctypes.byref(cost), ctypes.byref(nit),
                      ctypes.byref(conv), nthreads)
  errors = errors[:int(math.ceil(max_iterations / inner_iterations))]
  return sinkhorn_np.SinkhornResult(f=f, g=g, errors=errors, reg_ot_cost=cost.value,
                                    converged=bool(conv.value),
                                    inner_iterations=inner_iterations,
                                    threshold=threshold, a=a, b=b, epsilon=epsilon)
