"""Loads the golden vectors of tests/golden (made by gen_golden.py from the
reference's own code) and maps each case to solver arguments."""
import json
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names():
  with open(os.path.join(HERE, "manifest.json")) as fh:
    return sorted(json.load(fh))


def load(name, tag="f64"):
  with open(os.path.join(HERE, "manifest.json")) as fh:
    meta = json.load(fh)[name]
  data = dict(np.load(os.path.join(HERE, f"{name}.{tag}.npz")))
  geom = {}
  for k, v in meta["geometry"].items():
    if k == "epsilon" and v == "decay":
      geom.update(epsilon=0.01, eps_init=20.0, eps_decay=0.8)
    elif k in ("epsilon",):
      geom[k] = float(v)
    else:
      geom[k] = v
  return data, geom, dict(meta["solver"]), meta["init"]


def oracle_run(data, geom, solver, init, n_iters):
  """The float64 oracle on a case's inputs and arguments, run for exactly
  n_iters iterations (threshold 0): the state a solve that stopped after
  n_iters iterations should hold."""
  from oracle import sinkhorn_np as oracle
  kw = dict(geom)
  kw.update(solver)
  kw.update(threshold=0.0, max_iterations=n_iters)
  if init == "restart":
    kw["init"] = (data["f_init"], data["g_init"])
  return oracle.solve(data["x"], data["y"], data["a"], data["b"], dtype=np.float64, **kw)


def divergence_names():
  with open(os.path.join(HERE, "divergence_manifest.json")) as fh:
    return sorted(json.load(fh))


def load_divergence(name, tag="f64"):
  """Inputs and reference outputs of one Sinkhorn-divergence case, with the
  PointCloud and sinkhorn_divergence keyword arguments."""
  with open(os.path.join(HERE, "divergence_manifest.json")) as fh:
    meta = json.load(fh)[name]
  data = dict(np.load(os.path.join(HERE, f"{name}.{tag}.npz")))
  geom = {k: (float(v) if k == "epsilon" else v) for k, v in meta["geometry"].items()}
  return data, geom, dict(meta["divergence"]), bool(meta["weights"])


def segment_names():
  with open(os.path.join(HERE, "segment_manifest.json")) as fh:
    return sorted(json.load(fh))


def load_segment(name, tag="f64"):
  """Inputs, segment_sinkhorn keyword arguments and the reference's costs
  of one segmented case."""
  with open(os.path.join(HERE, "segment_manifest.json")) as fh:
    meta = json.load(fh)[name]
  data = dict(np.load(os.path.join(HERE, f"{name}.{tag}.npz")))
  kw = dict(meta["kwargs"])
  for k in ("segment_ids_x", "segment_ids_y", "weights_x", "weights_y"):
    if k in data:
      kw[k] = data[k]
  return data, kw


def implicit_names():
  with open(os.path.join(HERE, "implicit_manifest.json")) as fh:
    return sorted(json.load(fh))


def load_implicit(name):
  """Inputs, potentials, cotangents and the reference's implicit-diff
  results (lam, finite-difference gradients) of one case, with the
  PointCloud keyword arguments."""
  with open(os.path.join(HERE, "implicit_manifest.json")) as fh:
    meta = json.load(fh)[name]
  data = dict(np.load(os.path.join(HERE, f"{name}.f64.npz")))
  return data, dict(meta["geometry"])
