"""Builds libottb200.so in-tree for sm_100a.

``python -m ott_b200.build`` compiles ``ott_b200/csrc/capi.cu`` (which
includes every kernel) with nvcc into ``ott_b200/_lib/libottb200.so``.
Runs without a GPU (nvcc cross-compiles).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OUT = os.path.join(OUT_DIR, "libottb200.so")
PEAKS_OUT = os.path.join(OUT_DIR, "libottb200_peaks.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
  for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
    if cand and os.path.exists(cand):
      return cand
  raise RuntimeError("nvcc not found")


def sources(root=CSRC):
  return sorted(os.path.join(root, f) for f in os.listdir(root)
                if f.endswith((".cu", ".cuh", ".h")))


def up_to_date(out, deps) -> bool:
  if not os.path.exists(out):
    return False
  t = os.path.getmtime(out)
  deps = list(deps) + [__file__]
  return all(os.path.getmtime(s) <= t for s in deps if os.path.exists(s))


def _nvcc_shared(srcs, out, verbose):
  os.makedirs(OUT_DIR, exist_ok=True)
  srcs = [srcs] if isinstance(srcs, str) else list(srcs)
  cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
         "-shared", "-o", out + ".tmp", *srcs]
  if verbose:
    cmd.insert(1, "-Xptxas=-v")
  r = subprocess.run(cmd, capture_output=True, text=True)
  if r.returncode != 0:
    sys.stderr.write(r.stdout + r.stderr)
    raise RuntimeError(f"nvcc failed building {os.path.basename(out)}")
  if verbose:
    sys.stderr.write(r.stderr)
  os.replace(out + ".tmp", out)


def build(force: bool = False, verbose: bool = False) -> str:
  deps = sources() + [os.path.join(HERE, "..", "include", "ott_b200.h")]
  if force or not up_to_date(OUT, deps):
    _nvcc_shared([os.path.join(CSRC, "capi.cu"), os.path.join(CSRC, "noalloc.cu"),
                  os.path.join(CSRC, "mlp.cu"), os.path.join(CSRC, "transport.cu"),
                  os.path.join(CSRC, "transport_tc.cu"),
                  os.path.join(CSRC, "krylov.cu")], OUT,
                 verbose)
  peaks = os.path.join(CSRC, "peaks", "peaks.cu")
  if force or not up_to_date(PEAKS_OUT, [peaks]):
    _nvcc_shared(peaks, PEAKS_OUT, verbose)
  return OUT


if __name__ == "__main__":
  print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
