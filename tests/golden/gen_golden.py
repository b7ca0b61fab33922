"""Generates the golden vectors in this directory from the reference itself.

Runs ott-jax's own source for the Sinkhorn path (``ott.solvers.linear.solve``
on ``ott.geometry.pointcloud.PointCloud``, then ``SinkhornOutput.apply`` on
seeded vectors) over the NumPy stand-in for jax
(``oracle/jaxshim.py``, loaded by ``oracle/reference_loader.py``), in float64
(``jax_enable_x64`` semantics) and in float32, on seeded inputs from
``tests/problems.py``. Needs the reference source tree (the argument, else
$OTT_REFERENCE_SRC, else ``reference/src`` beside this repository); the GPU
machine only reads the committed ``*.npz``.

    python tests/golden/gen_golden.py [reference_src_root]
"""
import json
import os
import sys
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests import problems  # noqa: E402

# name -> (inputs, geometry kwargs, solver kwargs, init: None or "restart")
CASES = {
    "refprob_eps0.1": ("ref", dict(epsilon=0.1), dict(), None),
    "refprob_min34": ("ref", dict(epsilon=0.1), dict(min_iterations=34), None),
    "refprob_scan50": ("ref", dict(epsilon=0.1), dict(min_iterations=50, max_iterations=50), None),
    "refprob_max25": ("ref", dict(epsilon=0.1), dict(threshold=1e-9, max_iterations=25), None),
    "refprob_norm2": ("ref", dict(epsilon=0.1), dict(norm_error=2), None),
    "refprob_inner3": ("ref", dict(epsilon=0.1), dict(inner_iterations=3), None),
    "refprob_restart": ("ref", dict(epsilon=0.1), dict(), "restart"),
    "uniform_64x80_d2_relmean": ("unif:64:80:2", dict(epsilon=0.05, relative_epsilon="mean"), dict(), None),
    "uniform_50x40_d3_defaulteps": ("unif:50:40:3", dict(), dict(), None),
    "uniform_60x70_d5_scalemean": ("unif:60:70:5", dict(epsilon=0.1, relative_epsilon="mean",
                                                        scale_cost="mean"), dict(), None),
    "uniform_40x45_d3_decay": ("unif:40:45:3", dict(epsilon="decay"), dict(), None),
    "uniform_31x47_d33_relmean": ("unif:31:47:33", dict(epsilon=0.05, relative_epsilon="mean"), dict(), None),
    "gauss_96x96_d64_relmean0.01": ("gauss:96:96:64", dict(epsilon=0.01, relative_epsilon="mean"), dict(), None),
}


def make_inputs(spec):
  if spec == "ref":
    return problems.ref_test_problem()
  kind, n, m, d = spec.split(":")
  n, m, d = int(n), int(m), int(d)
  if kind == "unif":
    return problems.uniform_cloud_problem(n, m, d, seed=n + m + d)
  return problems.gaussian_shift_problem(n, m, d, seed=0)


def run(ref, case, dtype):
  spec, gkw, skw, init = CASES[case]
  x, y, a, b = [np.asarray(v, dtype) for v in make_inputs(spec)]
  gkw = dict(gkw)
  if gkw.get("epsilon") == "decay":
    gkw["epsilon"] = ref.epsilon_scheduler.Epsilon(target=0.01, init=20.0, decay=0.8)
  geom = ref.pointcloud.PointCloud(x, y, **gkw)
  kw = dict(skw)
  if init == "restart":
    out0 = ref.solve(geom, a, b, **kw)
    prob = ref.linear_problem.LinearProblem(geom, a, b)
    out = ref.sinkhorn.Sinkhorn(**kw)(prob, init=(out0.f, out0.g))
  else:
    out = ref.solve(geom, a, b, **kw)
  res = dict(f=np.asarray(out.f), g=np.asarray(out.g), errors=np.asarray(out.errors),
             reg_ot_cost=np.asarray(out.reg_ot_cost), n_iters=np.asarray(out.n_iters),
             converged=np.asarray(out.converged), epsilon=np.asarray(geom.epsilon))
  if init == "restart":
    res["f_init"] = np.asarray(out0.f)
    res["g_init"] = np.asarray(out0.g)
  # the plan applied to seeded signed vectors, both axes
  # (geometry.py:444-486 through SinkhornOutput.apply, sinkhorn.py:455-469)
  rng = np.random.default_rng(7)
  vec0 = rng.standard_normal((3, x.shape[0])).astype(dtype)
  vec1 = rng.standard_normal((3, y.shape[0])).astype(dtype)
  res["vec0"], res["vec1"] = vec0, vec1
  res["apply0"] = np.asarray(out.apply(vec0, axis=0))
  res["apply1"] = np.asarray(out.apply(vec1, axis=1))
  return (x, y, a, b), res


# Sinkhorn divergences (tools/sinkhorn_divergence.py:178-352):
# name -> (inputs, PointCloud kwargs, sinkhorn_divergence kwargs, weights)
DIV_CASES = {
    "div_unif_30x40_d3": ("unif:30:40:3", dict(epsilon=0.1), dict(), True),
    "div_unif_50x45_d5_relmean": ("unif:50:45:5", dict(epsilon=0.05, relative_epsilon="mean"),
                                  dict(), True),
    "div_unif_40x40_d2_nonsym": ("unif:40:40:2", dict(epsilon=0.05), dict(
        symmetric_sinkhorn=False), True),
    "div_gauss_64x80_d8_uniform": ("gauss:64:80:8", dict(epsilon=0.05, relative_epsilon="mean"),
                                   dict(), False),
}


def run_divergence(ref, div_mod, case, dtype):
  spec, gkw, dkw, weights = DIV_CASES[case]
  x, y, a, b = [np.asarray(v, dtype) for v in make_inputs(spec)]
  kw = dict(a=a, b=b) if weights else {}
  div, out = div_mod.sinkhorn_divergence(ref.pointcloud.PointCloud, x, y, **kw, **dkw, **gkw)
  res = dict(divergence=np.asarray(div), epsilon=np.asarray(out.geoms[0].epsilon),
             n_iters=np.asarray(out.n_iters))
  for k, tag in enumerate(("xy", "xx", "yy")):
    res[f"f_{tag}"] = np.asarray(out.potentials[k][0])
    res[f"g_{tag}"] = np.asarray(out.potentials[k][1])
  return (x, y, a, b), res


# Segmented solves (tools/segment_sinkhorn.py:24-138):
# name -> (x size, y size, d, keyword arguments)
SEG_CASES = {
    "seg_contig_relmean": (208, 183, 3, dict(num_per_segment_x=(40, 7, 100, 61),
                                             num_per_segment_y=(30, 80, 12, 61),
                                             epsilon=0.1, relative_epsilon="mean")),
    "seg_ids_weights_max60": (150, 170, 4, dict(num_segments=5, max_measure_size=60,
                                                epsilon=0.05)),
}


def run_segment(tools, case, dtype):
  nx, ny, d, kw = SEG_CASES[case]
  rng = np.random.default_rng(nx + ny + d)
  x = rng.uniform(size=(nx, d)).astype(dtype)
  y = rng.uniform(size=(ny, d)).astype(dtype)
  kw = dict(kw)
  extra = {}
  if "num_segments" in kw:
    ns = kw["num_segments"]
    ids_x = rng.integers(0, ns, size=nx)
    ids_y = rng.integers(0, ns, size=ny)
    wx = rng.uniform(0.5, 1.5, size=nx)
    wy = rng.uniform(0.5, 1.5, size=ny)
    for s in range(ns):
      wx[ids_x == s] /= wx[ids_x == s].sum()
      wy[ids_y == s] /= wy[ids_y == s].sum()
    extra = dict(segment_ids_x=ids_x, segment_ids_y=ids_y, weights_x=wx.astype(dtype),
                 weights_y=wy.astype(dtype))
  out = tools.segment_sinkhorn.segment_sinkhorn(x, y, **kw, **extra)
  return x, y, extra, np.asarray(out)


# Implicit differentiation of the potentials
# (solvers/linear/implicit_differentiation.py, default ImplicitDiff()):
# name -> (n, m, d, PointCloud kwargs with an absolute epsilon, inputs)
IMP_CASES = {
    "imp_unif_13x9_d3": (13, 9, 3, dict(epsilon=0.1), "unif"),
    "imp_unif_8x15_d2_scalemean": (8, 15, 2, dict(epsilon=0.05, scale_cost="mean"), "unif"),
    "imp_gauss_24x30_d8": (24, 30, 8, dict(epsilon=0.5), "gauss"),
    "imp_unif_18x18_d4_scale2": (18, 18, 4, dict(epsilon=0.02, scale_cost=2.0), "unif"),
}


def lstsq_solver(lin, b, lin_t=None, symmetric=False, **kwargs):
  """Stands in for lineax's NormalCG (not installed): the least-squares
  solution of least norm, its limit from zero, on the materialised
  operator."""
  b = np.asarray(b, np.float64)
  k = b.shape[0]
  mat = np.stack([np.asarray(lin(np.eye(k)[:, i])) for i in range(k)], 1)
  return np.linalg.lstsq(mat, b, rcond=None)[0]


def run_implicit(ref, imp_mod, case):
  """The reference's ImplicitDiff.solve on its own converged potentials,
  then the gradient of ``<lam, first_order_conditions>`` w.r.t. every
  coordinate of x, y, a and b by central differences of the reference's
  own first_order_conditions (its ``jax.vjp``, :275-287, needs autodiff).
  Epsilon is absolute: the reference stops gradients through a relative
  one (geometry.py:157-163), which finite differences would not."""
  n, m, d, gkw, kind = IMP_CASES[case]
  rng = np.random.default_rng(n * m + d)
  if kind == "unif":
    x = rng.uniform(size=(n, d))
    y = rng.uniform(size=(m, d))
  else:
    x = rng.standard_normal((n, d))
    y = 0.5 + rng.standard_normal((m, d)) * rng.uniform(0.5, 1.5, size=d)
  a = rng.uniform(0.2, 1.2, n)
  a /= a.sum()
  b = rng.uniform(0.2, 1.2, m)
  b /= b.sum()
  geom = ref.pointcloud.PointCloud(x, y, **gkw)
  out = ref.solve(geom, a, b, threshold=1e-11, max_iterations=200000)
  f, g = np.asarray(out.f), np.asarray(out.g)
  prob = ref.linear_problem.LinearProblem(geom, a, b)
  gr_f, gr_g = rng.standard_normal(n), rng.standard_normal(m)
  idiff = imp_mod.ImplicitDiff()
  lam = np.asarray(idiff.solve((gr_f, gr_g), prob, f, g, True))

  def objective(xx, yy, aa, bb):
    pr = ref.linear_problem.LinearProblem(ref.pointcloud.PointCloud(xx, yy, **gkw), aa, bb)
    return float(np.dot(lam, np.asarray(idiff.first_order_conditions(pr, f, g, True))))

  def fd(arr, which):
    grad = np.zeros_like(arr)
    flat = grad.reshape(-1)
    for i in range(arr.size):
      h = 1e-6 * max(1.0, abs(arr.reshape(-1)[i]))
      args = {"x": x, "y": y, "a": a, "b": b}
      up, dn = arr.copy(), arr.copy()
      up.reshape(-1)[i] += h
      dn.reshape(-1)[i] -= h
      args[which] = up
      fu = objective(args["x"], args["y"], args["a"], args["b"])
      args[which] = dn
      fl = objective(args["x"], args["y"], args["a"], args["b"])
      flat[i] = (fu - fl) / (2 * h)
    return grad

  res = dict(f=f, g=g, gr_f=gr_f, gr_g=gr_g, lam=lam, n_iters=np.asarray(out.n_iters),
             gx=fd(x, "x"), gy=fd(y, "y"), ga=fd(a, "a"), gb=fd(b, "b"))
  return (x, y, a, b), res


def main():
  from oracle import reference_loader
  root = sys.argv[1] if len(sys.argv) > 1 else reference_loader.DEFAULT_ROOT
  warnings.filterwarnings("ignore")
  manifest = {}
  for x64, tag in ((True, "f64"), (False, "f32")):
    ref = reference_loader.load(root, x64=x64)
    import ott.geometry.epsilon_scheduler as es  # noqa: E402  (loaded module)
    ref.epsilon_scheduler = es
    for case in CASES:
      (x, y, a, b), res = run(ref, case, np.float64 if x64 else np.float32)
      np.savez_compressed(os.path.join(HERE, f"{case}.{tag}.npz"), x=x, y=y, a=a, b=b, **res)
      spec, gkw, skw, init = CASES[case]
      manifest[case] = dict(inputs=spec, geometry={k: str(v) for k, v in gkw.items()},
                            solver=skw, init=init)
      print(tag, case, "n_iters", int(res["n_iters"]), "reg_ot_cost", float(res["reg_ot_cost"]))
    tools = reference_loader.load_tools(root)
    div_mod = tools.sinkhorn_divergence
    for case in DIV_CASES:
      (x, y, a, b), res = run_divergence(ref, div_mod, case, np.float64 if x64 else np.float32)
      np.savez_compressed(os.path.join(HERE, f"{case}.{tag}.npz"), x=x, y=y, a=a, b=b, **res)
      print(tag, case, "n_iters", res["n_iters"].tolist(), "divergence", float(res["divergence"]))
    for case in SEG_CASES:
      x, y, extra, costs = run_segment(tools, case, np.float64 if x64 else np.float32)
      np.savez_compressed(os.path.join(HERE, f"{case}.{tag}.npz"), x=x, y=y, costs=costs,
                          **extra)
      print(tag, case, "costs", costs.tolist())
  ref = reference_loader.load(root, x64=True)
  imp_mod = reference_loader.load_implicit(lstsq_solver, root)
  for case in IMP_CASES:
    (x, y, a, b), res = run_implicit(ref, imp_mod, case)
    np.savez_compressed(os.path.join(HERE, f"{case}.f64.npz"), x=x, y=y, a=a, b=b, **res)
    print("f64", case, "n_iters", int(res["n_iters"]), "|lam|", float(np.abs(res["lam"]).max()))
  imp_meta = {c: dict(sizes=[n, m, d], geometry={k: v for k, v in g.items()}, inputs=kind)
              for c, (n, m, d, g, kind) in IMP_CASES.items()}
  with open(os.path.join(HERE, "implicit_manifest.json"), "w") as fh:
    json.dump(imp_meta, fh, indent=1, sort_keys=True)
  with open(os.path.join(HERE, "manifest.json"), "w") as fh:
    json.dump(manifest, fh, indent=1, sort_keys=True)
  div_meta = {c: dict(inputs=s, geometry={k: str(v) for k, v in g.items()}, divergence=d,
                      weights=w) for c, (s, g, d, w) in DIV_CASES.items()}
  with open(os.path.join(HERE, "divergence_manifest.json"), "w") as fh:
    json.dump(div_meta, fh, indent=1, sort_keys=True)
  seg_meta = {c: dict(sizes=[nx, ny, d], kwargs={k: (list(v) if isinstance(v, tuple) else v)
                                                 for k, v in kw.items()})
              for c, (nx, ny, d, kw) in SEG_CASES.items()}
  with open(os.path.join(HERE, "segment_manifest.json"), "w") as fh:
    json.dump(seg_meta, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
  main()
