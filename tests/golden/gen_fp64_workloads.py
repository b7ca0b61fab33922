"""Float64 solutions of the measured workloads, for accuracy checks at full size.

The float64 oracle (``oracle/sinkhorn_np.py``, the reference's algorithm in
``jax_enable_x64`` semantics; pinned against the reference's own code at small
sizes by ``tests/test_golden_oracle.py``) solves each workload on the same
seeded float32 inputs the bench and the GPU tests generate, cast to float64,
with the cost recomputed in column or row blocks (``batch_size``; the dense
cost would not fit) on all host threads. The committed ``*.fp64.npz`` hold
the potentials, the error log, ``n_iters``, ``converged``, ``reg_ot_cost`` and
epsilon, plus checksums of the inputs so a test can tell that it regenerated
the same points.

    python tests/golden/gen_fp64_workloads.py [name ...]

The headline workload (n = m = 65536, d = 64) takes about 20 minutes on 8
cores; the GPU machine only reads the committed files. ``ANNEALED`` adds an
epsilon-annealed chain at a reduced size (the float64 reference of the
annealing workload's accuracy).
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import sinkhorn_np as oracle  # noqa: E402
from tests import problems  # noqa: E402

# name -> (inputs, relative epsilon multiplier of mean(C), threshold)
WORKLOADS = {
    # n = m = 65536, d = 64, x ~ N(0, I), y ~ N(0.5, diag(U[0.5, 2])), uniform
    # weights, epsilon = 0.01 * mean(C): the single large solve
    "gauss65536_d64": (lambda: problems.gaussian_shift_problem(65536, 65536, 64, seed=0),
                       0.01, 1e-3),
    # n = m = 2048, d = 2, x, y ~ U[0, 1]^2, a, b = U(0, 1) + 0.2 normalised,
    # epsilon = 0.05 * mean(C): the reference's CPU-runnable configuration
    "uniform2048_d2": (lambda: problems.uniform_cloud_problem(2048, 2048, 2, seed=0),
                       0.05, 1e-3),
}


# name -> (inputs, stages, start, final): epsilon-annealed chains, every
# stage from the previous stage's potentials, threshold 1e-3 per stage
ANNEALED = {
    # two 8-component Gaussian mixtures in R^128, uniform weights (the
    # annealing workload's family, pair seed 0) at n = m = 2048
    "anneal_gmm8_n2048_d128": (lambda: problems.gmm8_pair(2048, 2048, 128, seed=0), 10, 1.0,
                               1e-3),
}


def input_checksums(x, y, a, b):
  """Float64 sums of the float32 inputs and of their squares."""
  out = []
  for v in (x, y, a, b):
    v = np.asarray(v, np.float64)
    out += [v.sum(), (v * v).sum()]
  return np.array(out)


def generate(name, workers=None):
  make, mult, thr = WORKLOADS[name]
  x, y, a, b = make()
  workers = workers or os.cpu_count()
  n = x.shape[0]
  bs = 256 if n > 8192 else None
  t0 = time.time()
  r = oracle.solve(x, y, a, b, epsilon=mult, relative_epsilon="mean", threshold=thr,
                   dtype=np.float64, batch_size=bs, workers=workers)
  dt = time.time() - t0
  path = os.path.join(HERE, f"{name}.fp64.npz")
  np.savez_compressed(path, f=r.f, g=r.g, errors=r.errors, n_iters=r.n_iters,
                      converged=r.converged, reg_ot_cost=r.reg_ot_cost,
                      epsilon=r.epsilon, threshold=thr, checksums=input_checksums(x, y, a, b))
  print(f"{name}: n_iters={r.n_iters} converged={r.converged} "
        f"reg_ot_cost={r.reg_ot_cost:.12g} eps={r.epsilon:.9g} ({dt:.0f} s, {workers} threads)"
        f" -> {os.path.basename(path)}")


def generate_annealed(name, workers=None):
  make, stages, start, final = ANNEALED[name]
  x, y, a, b = make()
  x64, y64 = x.astype(np.float64), y.astype(np.float64)
  mean_c = float(oracle.mean_cost_matrix(x64, y64))
  mults = start * (final / start) ** (np.arange(stages) / max(1, stages - 1))
  init, iters, t0 = None, [], time.time()
  for m in mults:
    geom = oracle.Geom(x64, y64, float(m * mean_c), workers=workers or os.cpu_count())
    r = oracle.sinkhorn(geom, a, b, init=init, threshold=1e-3)
    init = (r.f, r.g)
    iters.append(r.n_iters)
  path = os.path.join(HERE, f"{name}.fp64.npz")
  np.savez_compressed(path, f=r.f, g=r.g, stage_iters=np.array(iters),
                      reg_ot_cost=r.reg_ot_cost, epsilon=r.epsilon, mean_cost=mean_c,
                      checksums=input_checksums(x, y, a, b))
  print(f"{name}: stage iterations {iters}, final reg_ot_cost={r.reg_ot_cost:.12g} "
        f"({time.time() - t0:.0f} s) -> {os.path.basename(path)}")


if __name__ == "__main__":
  for nm in (sys.argv[1:] or list(WORKLOADS) + list(ANNEALED)):
    if nm in ANNEALED:
      generate_annealed(nm)
    else:
      generate(nm)
