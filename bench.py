#!/usr/bin/env python
"""Benchmark: seconds to 1e-3 marginal error and Sinkhorn iterations/s.

Workload: one log-domain Sinkhorn solve (ott ``linear.solve`` semantics) on
a squared-Euclidean point cloud, n = m = 65536, d = 64, x ~ N(0, I),
y ~ N(0.5 * 1, diag(U[0.5, 2])), uniform weights, epsilon = 0.01 * mean(C),
threshold 1e-3 (L1 marginal error), max_iterations 2000. Synthetic seeded
data (numpy default_rng(0)). A step is one full solve to the threshold.

``python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]``
prints one JSON line (rank 0). Under torchrun each rank solves its own
replica of the workload (the path does not shard: replicas only); times are
device times, max over ranks.

``--impl reference`` times the CPU restatement of the reference algorithm
(C port of the oracle, OpenMP, all host threads) on a bounded row sample of
the same workload and converts it to the same metric.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
  sys.path.insert(0, ROOT)

METRIC = "s to 1e-3 marginal err & Sinkhorn iters/s: chosen form vs plain FP32, 1 B200"
L2_BYTES = 126 * 1024 * 1024
GOLDEN = os.path.join(ROOT, "tests", "golden")


def parse_args():
  p = argparse.ArgumentParser()
  p.add_argument("--gpus", type=int, default=1)
  p.add_argument("--steps", type=int, default=3)
  p.add_argument("--warmup", type=int, default=3)
  p.add_argument("--impl", choices=["ours", "reference"], default="ours")
  p.add_argument("--precision", default="auto", choices=["auto", "fp32", "bf16_split3"])
  p.add_argument("--n", type=int, default=None, help="points per side (default: the workload's)")
  p.add_argument("--d", type=int, default=None, help="dimension (default: the workload's)")
  p.add_argument("--no-plain", action="store_true", help="skip the plain FP32 comparison")
  p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
  p.add_argument("--workload", default="gaussian64",
                 choices=["gaussian64", "uniform2048", "warmstart", "batched", "anneal",
                          "divergence", "implicit", "sharded"],
                 help="gaussian64: the headline single large solve (default); "
                      "uniform2048: n=m=2048, d=2 uniform clouds (the reference's "
                      "CPU-runnable configuration, solved to convergence on the CPU too); "
                      "warmstart: learned warm start on a 32x32 grid; batched: 512 "
                      "uneven problems in one launch; anneal: epsilon-annealed solves; "
                      "divergence: Sinkhorn divergence and its gradient")
  p.add_argument("--train-pairs", type=int, default=100000)
  p.add_argument("--test-pairs", type=int, default=10000)
  p.add_argument("--train-steps", type=int, default=12000)
  p.add_argument("--problems", type=int, default=512)
  p.add_argument("--pairs", type=int, default=8)
  p.add_argument("--stages", type=int, default=10)
  p.add_argument("--train-chains", type=int, default=8,
                 help="anneal: pairs of the family solved to train the stage predictor")
  p.add_argument("--train-n", type=int, default=None,
                 help="anneal: points per side of the training pairs (default: --n)")
  args = p.parse_args()
  default_n, default_d = {"uniform2048": (2048, 2), "anneal": (16384, 128),
                          "divergence": (32768, 64)}.get(args.workload, (65536, 64))
  args.n = default_n if args.n is None else args.n
  args.d = default_d if args.d is None else args.d
  return args


# The single-solve workloads: seeded inputs, epsilon = mult * mean(C), and the
# committed float64 solution of the same inputs where one exists.
SOLVE_WORKLOADS = {
    "gaussian64": dict(mult=0.01, fp64={(65536, 64): "gauss65536_d64"},
                       data="x~N(0,I), y~N(0.5,diag(U[0.5,2])), uniform weights, seed 0"),
    "uniform2048": dict(mult=0.05, fp64={(2048, 2): "uniform2048_d2"},
                        data="x,y~U[0,1]^d, a,b=U(0,1)+0.2 normalised, seed 0"),
}


def workload(args):
  from tests import problems
  n = args.n
  if args.workload == "uniform2048":
    return problems.uniform_cloud_problem(n, n, args.d, seed=0)
  return problems.gaussian_shift_problem(n, n, args.d, seed=0)


def fp64_record(args):
  """The committed float64 solve of this workload's inputs
  (tests/golden/gen_fp64_workloads.py), or None."""
  name = SOLVE_WORKLOADS[args.workload]["fp64"].get((args.n, args.d))
  path = os.path.join(GOLDEN, f"{name}.fp64.npz") if name else None
  if not path or not os.path.exists(path):
    return None
  rec = dict(np.load(path))
  rec["name"] = name
  return rec


def accuracy_vs_fp64(out, rec):
  """Errors of a solve against the float64 solution of the same inputs."""
  if rec is None:
    return None
  eps = float(rec["epsilon"])
  f = out.f.detach().cpu().numpy().astype(np.float64)
  g = out.g.detach().cpu().numpy().astype(np.float64)
  ff, gf = np.isfinite(rec["f"]), np.isfinite(rec["g"])
  return {"reference": f"tests/golden/{rec['name']}.fp64.npz (float64 oracle, same inputs)",
          "reg_ot_cost_rel": abs(out.reg_ot_cost - float(rec["reg_ot_cost"]))
                             / abs(float(rec["reg_ot_cost"])),
          "f_max_abs_over_eps": float(np.max(np.abs(f[ff] - rec["f"][ff]))) / eps,
          "g_max_abs_over_eps": float(np.max(np.abs(g[gf] - rec["g"][gf]))) / eps,
          "n_iters": int(out.n_iters), "n_iters_fp64": int(rec["n_iters"])}


def config_dict(args, n_iters=None):
  w = SOLVE_WORKLOADS[args.workload]
  big = 2 * args.n * args.d * 4 > L2_BYTES
  return {"workload": f"sinkhorn sqeuclidean n=m={args.n} d={args.d} "
                      f"eps={w['mult']}*mean(C) thr=1e-3 (L1)",
          "n": args.n, "m": args.n, "d": args.d, "epsilon": f"{w['mult']}*mean(C)",
          "threshold": 1e-3, "max_iterations": 2000, "n_iters": n_iters,
          "data": w["data"],
          "l2": "flushed between timed steps (256 MiB write); inputs "
                f"{2 * args.n * args.d * 4 / 2**20:.2f} MiB {'>' if big else '<'} L2",
          "parallelism": f"replicas x{args.gpus}"}


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
  QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
           "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
           "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

  def __init__(self, index: int):
    self.index = index
    self.proc = None
    self.path = None

  def start(self):
    fd, self.path = tempfile.mkstemp(suffix=".csv")
    os.close(fd)
    try:
      self.proc = subprocess.Popen(
          ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
           "--format=csv,noheader,nounits", "-lms", "200"],
          stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
    except OSError:
      self.proc = None

  def stop(self):
    if self.proc is None:
      return None
    self.proc.terminate()
    try:
      self.proc.wait(timeout=5)
    except subprocess.TimeoutExpired:
      self.proc.kill()
    rows = []
    for line in open(self.path):
      parts = [p.strip() for p in line.split(",")]
      if len(parts) >= 9:
        rows.append(parts)
    os.unlink(self.path)
    if not rows:
      return None
    sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
    mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
    pw = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
    return {"sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
            "power_w_median": statistics.median(pw) if pw else None,
            "samples": len(rows)}


# ---------------------------------------------------------------------------
# measured pipe peaks (no driver figure exists for these pipes)
# ---------------------------------------------------------------------------
def measure_pipe_peaks(torch):
  """FFMA and MUFU ex2 throughput of this GPU (best of 3 runs each). Called
  before any solve, while the GPU is cool: under a sustained load the power
  cap lowers the clock and a probe run then would understate the peak."""
  lib = ctypes.CDLL(os.path.join(ROOT, "ott_b200", "_lib", "libottb200_peaks.so"))
  lib.ottb_peaks_launch.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 2
  out = torch.zeros(4096, device="cuda")
  sms = torch.cuda.get_device_properties(0).multi_processor_count
  blocks, res = sms * 8, {}
  stream = torch.cuda.current_stream().cuda_stream
  for kind, name, iters in ((0, "ffma_per_s", 20000), (1, "ex2_per_s", 4000)):
    lib.ottb_peaks_launch(kind, blocks, iters, out.data_ptr(), stream)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(3):
      e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
      e0.record()
      lib.ottb_peaks_launch(kind, blocks, iters, out.data_ptr(), stream)
      e1.record()
      torch.cuda.synchronize()
      best = max(best, blocks * 256 * iters * 8 / (e0.elapsed_time(e1) * 1e-3))
    res[name] = best
  return res


def load_peaks_json():
  path = os.path.join(ROOT, "MEASURED_PEAKS.json")
  try:
    return json.load(open(path))
  except Exception:
    return None


def bf16_peak_tflops():
  """The measured cuBLAS bf16 burst peak (MEASURED_PEAKS.json) and its source,
  else the 1.59 PFLOP/s fallback, an earlier B200 measurement."""
  mp = load_peaks_json()
  if mp and mp.get("bf16_tflops"):
    return float(mp["bf16_tflops"]), "MEASURED_PEAKS.json bf16_tflops (burst)"
  return 1590.0, "fallback: 1.59 PFLOP/s, an earlier B200 measurement (file absent)"


def tc_apply_flops_per_entry(d, k):
  """BF16 tensor flops that ottb_apply_transport_tc executes per plan entry
  for k vectors: its first pass (the hi*hi product and the shift block, DK
  / 16 + 1 MMAs of K = 16, 2 flops per multiply-add), the cost tile of each
  vector chunk (3 DK / 16 + 1 MMAs) and its P V products (P_hi [V_hi |
  V_lo] and P_lo V_hi: 3 products of the chunk's padded width)."""
  dk = 64 if d <= 64 else 128
  kvmax = 96 if dk == 64 else 64
  nch = -(-k // kvmax)
  kvp = -(-(-(-k // nch)) // 16) * 16
  first = 2 * 16 * (dk // 16 + 1)
  cost = 2 * 16 * (3 * dk // 16 + 1)
  return first + nch * (cost + 2 * 3 * kvp)


def ncu_traffic(name):
  """Per-launch DRAM bytes of a kernel from the committed ncu summary."""
  path = os.path.join(ROOT, "profiles", "traffic.json")
  try:
    return json.load(open(path)).get(name)
  except Exception:
    return None


# ---------------------------------------------------------------------------
# CPU baselines: the C port of the oracle (tiled, vectorised, OpenMP on every
# host thread) and the float32 NumPy restatement (BLAS products per block)
# ---------------------------------------------------------------------------
def reference_sweeps(n_iters, inner=10):
  """Full n x m sweeps of the reference loop to n_iters iterations: two
  potential updates per iteration, one error sweep per block of inner
  iterations, one for reg_ot_cost."""
  return 2 * n_iters + n_iters // inner + 1


def cpu_solves_to_convergence(args):
  """Whether a CPU step is a whole solve to the threshold (the small
  configuration) or one full-size iteration (the large ones)."""
  return args.n <= 8192


def cpu_step(args, x, y, a, b, eps, variant="tiled"):
  """One CPU step. Small workloads: the whole solve to the threshold.
  Large: one full-size iteration as a 1-iteration solve (inner_iterations
  1, max_iterations 1: the g- and f-update sweeps, the error sweep and the
  reg_ot_cost sweep, 4 sweeps over all n x m entries). Returns seconds and
  the result."""
  from oracle import sinkhorn_c
  kw = {} if cpu_solves_to_convergence(args) else dict(inner_iterations=1, max_iterations=1)
  t0 = time.perf_counter()
  r = sinkhorn_c.solve(x, y, a, b, epsilon=eps, threshold=1e-3, variant=variant, **kw)
  return time.perf_counter() - t0, r


def cpu_seconds_to_threshold(args, step_s, n_iters):
  """Seconds to the threshold from one step's time: the step itself when it
  is a whole solve, else 4 full sweeps scaled to the loop's sweep count."""
  if cpu_solves_to_convergence(args):
    return step_s
  return step_s / 4.0 * reference_sweeps(n_iters)


def cpu_iteration_count(args, rec, fallback=None):
  """Iterations the CPU loop runs to the threshold, for the extrapolation:
  the float64 solve of the same inputs (its count equals the FP32 GPU
  engine's on every parity case), else the fallback given."""
  if rec is not None:
    return int(rec["n_iters"]), f"float64 solve of the same inputs ({rec['name']})"
  return (fallback or 30), "GPU FP32 engine's count" if fallback else "assumed (no record)"


def cpu_sample_text(args, n_iters, src):
  if cpu_solves_to_convergence(args):
    return (f"whole solve to 1e-3 (n=m={args.n}, d={args.d}) per step, tiled C port "
            "on all host threads")
  return (f"one full-size iteration per step (g- and f-update sweeps, error sweep, "
          f"reg_ot_cost sweep: 4 sweeps over all {args.n}x{args.n} entries, d={args.d}), "
          f"scaled to {reference_sweeps(n_iters)} sweeps = {n_iters} iterations "
          f"({src}) + error and reg_ot_cost sweeps")


def numpy_f32_baseline(args, x, y, a, b, eps):
  """The oracle in float32: the cost of each 1024-column (or row) block from
  a BLAS product, the reference's centring and max-shifted log-sum-exp, blocks
  on all host threads. Small workloads: the whole solve to the threshold;
  large: a 1-iteration solve of the first 4096 rows against every column,
  its per-entry time scaled to the full loop."""
  from oracle import sinkhorn_np
  workers = os.cpu_count() or 1
  small = cpu_solves_to_convergence(args)
  rows = args.n if small else min(args.n, 4096)
  xs, as_ = x[:rows], a[:rows] / a[:rows].sum()
  kw = {} if small else dict(inner_iterations=1, max_iterations=1)
  t0 = time.perf_counter()
  r = sinkhorn_np.solve(xs, y, as_, b, epsilon=eps, dtype=np.float32, batch_size=1024,
                        workers=workers, threshold=1e-3, **kw)
  dt = time.perf_counter() - t0
  return dt, r, rows, workers


def run_reference(args):
  """The reference arm: the CPU restatement of the reference's loop (the
  reference itself needs JAX, absent here and on the GPU machine), timed on
  every host thread. Each step is what ``cpu_step`` describes; ``steps`` and
  ``ms_per_step`` are the measured steps, ``value`` the seconds to the
  threshold they give (extrapolated over iterations on the large
  workloads, and marked so)."""
  rank = int(os.environ.get("RANK", "0"))
  if rank != 0:
    return 0
  from oracle import sinkhorn_c, sinkhorn_np
  if args.workload not in SOLVE_WORKLOADS:
    print(json.dumps({"impl": "reference", "unavailable":
                      f"no CPU arm for the {args.workload} workload; the reference arm "
                      "times the single-solve workloads"}))
    return 0
  x, y, a, b = workload(args)
  mult = SOLVE_WORKLOADS[args.workload]["mult"]
  eps = mult * float(sinkhorn_np.mean_cost_matrix(x.astype(np.float64), y.astype(np.float64)))
  rec = fp64_record(args)
  for _ in range(args.warmup):
    cpu_step(args, x, y, a, b, eps)
  times, r = [], None
  for _ in range(args.steps):
    dt, r = cpu_step(args, x, y, a, b, eps)
    times.append(dt)
  step_s = statistics.median(times)
  small = cpu_solves_to_convergence(args)
  if small:
    n_iters, src = r.n_iters, "the CPU solve's own count"
  else:
    n_iters, src = cpu_iteration_count(args, rec)
  val = cpu_seconds_to_threshold(args, step_s, n_iters)
  sweep_s = step_s / (reference_sweeps(n_iters) if small else 4.0)
  cores = sinkhorn_c.threads("tiled")
  sample = cpu_sample_text(args, n_iters, src)
  line = {
      "metric": METRIC, "value": val, "unit": "s", "impl": "reference",
      "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
      "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": False,
      "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
      "config": config_dict(args, n_iters),
      "extrapolated": not small, "measured_s_per_step": step_s,
      "n_iters": n_iters, "n_iters_source": src,
      "iters_per_s": 1.0 / (2 * sweep_s), "entries_per_s": args.n * args.n / sweep_s,
      "cpu_baseline": {"value": val, "unit": "s", "cores": cores, "kind": "port",
                       "sample": sample},
      "e2e": {"value": val, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
  }
  if small:
    line["converged"] = bool(r.converged)
    line["reg_ot_cost"] = float(r.reg_ot_cost)
    if rec is not None:
      line["n_iters_fp64"] = int(rec["n_iters"])
      line["reg_ot_cost_rel_vs_fp64"] = abs(r.reg_ot_cost - float(rec["reg_ot_cost"])) / abs(
          float(rec["reg_ot_cost"]))
  print(json.dumps(line))
  return 0


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
  import torch
  import torch.distributed as dist
  from datetime import timedelta

  world = int(os.environ.get("WORLD_SIZE", "1"))
  rank = int(os.environ.get("RANK", "0"))
  local = int(os.environ.get("LOCAL_RANK", "0"))
  torch.cuda.set_device(local)
  if world > 1:
    dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                            device_id=torch.device("cuda", local))

  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers import linear
  from ott_b200.solvers.linear import sinkhorn

  from ott_b200 import distributed as odist

  def barrier():
    if world > 1:
      dist.barrier()
    torch.cuda.synchronize()

  max_over_ranks = odist.max_over_ranks

  peaks = measure_pipe_peaks(torch)
  x, y, a, b = workload(args)
  xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
  ad, bd = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()
  mult = SOLVE_WORKLOADS[args.workload]["mult"]
  geom = pointcloud.PointCloud(xd, yd, epsilon=mult, relative_epsilon="mean")
  eps = geom.epsilon
  prob = linear_problem.LinearProblem(geom, ad, bd)
  flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device="cuda")

  def timed_solves(solver, steps, warm):
    for _ in range(warm):
      out = solver(prob)
      _ = out.n_iters
    barrier()
    ms, out = 0.0, None
    for _ in range(steps):
      flush.zero_()
      e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
      e0.record()
      out = solver(prob)
      e1.record()
      e1.synchronize()
      ms += e0.elapsed_time(e1)
    barrier()
    return max_over_ranks(ms / steps), out

  solver = sinkhorn.Sinkhorn(threshold=1e-3, max_iterations=2000, precision=args.precision)
  clocks = ClockSampler(local)
  clocks.start()
  ms, out = timed_solves(solver, args.steps, args.warmup)
  clk = clocks.stop()
  n_iters, converged = out.n_iters, out.converged
  form = "bf16_split3" if (args.precision == "bf16_split3" or
                           (args.precision == "auto" and args.d >= 32)) else "fp32"

  # plain FP32 comparison (the "vs plain FP32" half of the metric)
  plain = None
  if not args.no_plain and form != "fp32":
    pms, plain_out = timed_solves(sinkhorn.Sinkhorn(threshold=1e-3, precision="fp32"), 1, 1)
    plain = {"s_to_threshold": pms * 1e-3, "n_iters": plain_out.n_iters,
             "iters_per_s": plain_out.n_iters / (pms * 1e-3)}

  # end to end through the public API, host buffers in, results out
  xh = torch.from_numpy(x).pin_memory()
  yh = torch.from_numpy(y).pin_memory()
  ah = torch.from_numpy(a).pin_memory()
  bh = torch.from_numpy(b).pin_memory()

  def e2e_step():
    g = pointcloud.PointCloud(xh, yh, epsilon=mult, relative_epsilon="mean")
    o = linear.solve(g, ah, bh, threshold=1e-3, precision=args.precision)
    f_host, g_host = o.f.cpu(), o.g.cpu()
    err_host = o.errors.cpu()
    return o.reg_ot_cost, f_host, g_host, err_host

  for _ in range(max(1, args.warmup)):
    e2e_step()
  barrier()
  e2e_ms = 0.0
  for _ in range(args.steps):
    flush.zero_()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    e2e_step()
    e1.record()
    e1.synchronize()
    e2e_ms += e0.elapsed_time(e1)
  barrier()
  e2e_ms = max_over_ranks(e2e_ms / args.steps)
  h2d = (x.nbytes + y.nbytes + a.nbytes + b.nbytes)
  d2h = 4 * (2 * args.n) + 4 * out.errors.numel() + 16 + 32

  # roofline of the dominant kernel (the persistent solve kernel)
  entries = 2.0 * args.n * args.n * n_iters      # algorithmic: 2 sweeps/iteration
  t = ms * 1e-3
  mp = load_peaks_json()
  if form == "fp32" and args.d > 8:
    achieved = 2.0 * args.d * entries / t / 1e12
    peak = 2.0 * peaks["ffma_per_s"] / 1e12
    roof = {"bound": "fp32_fma", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak,
            "peak_source": "measured in bench.py (FFMA probe kernel, 8 chains/thread)"}
  else:
    achieved = entries / t / 1e9
    peak = peaks["ex2_per_s"] / 1e9
    roof = {"bound": "mufu_ex2", "achieved": achieved, "peak": peak, "unit": "Gex2/s",
            "frac": achieved / peak,
            "peak_source": "measured in bench.py (MUFU ex2 probe kernel)"}
    if clk and clk.get("sm_mhz"):
      # the solves run power-capped below the probe's clock: also against
      # 16 ex2 / clk / SM at the median SM clock sampled during the solves
      sms = torch.cuda.get_device_properties(0).multi_processor_count
      at_clk = 16 * sms * clk["sm_mhz"] * 1e6 / 1e9
      roof["peak_at_sampled_clock"] = at_clk
      roof["frac_at_sampled_clock"] = achieved / at_clk
    if form != "fp32":
      # against the measured cuBLAS bf16 burst peak when the peaks file is
      # there, else an earlier B200 measurement of it (1.59 PFLOP/s)
      bf16 = mp.get("bf16_tflops") if mp else None
      src = "MEASURED_PEAKS.json bf16_tflops (burst)"
      if not bf16:
        bf16, src = 1590.0, "fallback: 1.59 PFLOP/s, an earlier B200 measurement (file absent)"
      dk = 64 if args.d <= 64 else 128
      tf = 3 * 2 * dk * entries / t / 1e12   # split-3 MMA flops
      roof["tensor_secondary"] = {"achieved": tf, "peak": bf16, "unit": "TFLOP/s",
                                  "frac": tf / bf16, "peak_source": src}
  traffic = ncu_traffic(f"sinkhorn_{form}_n{args.n}_d{args.d}")
  roof["traffic"] = traffic
  roof["work_per_launch"] = f"{entries:.4g} cost entries (2*n*m per iteration x {n_iters})"
  if mp:
    roof["measured_peaks_file"] = {"hbm_gbs": mp.get("hbm_gbs"),
                                   "bf16_tflops": mp.get("bf16_tflops")}

  # accuracy of both forms against the float64 solve of the same inputs
  rec = fp64_record(args)
  accuracy = {form: accuracy_vs_fp64(out, rec)}
  if plain is not None:
    accuracy["fp32"] = accuracy_vs_fp64(plain_out, rec)

  cpu = cpu_np = None
  if not args.no_cpu and rank == 0 and world == 1:
    from oracle import sinkhorn_c
    cpu_step(args, x, y, a, b, eps)  # warm-up (library load, page-in)
    step_s, r = cpu_step(args, x, y, a, b, eps)
    small = cpu_solves_to_convergence(args)
    c_iters, src = ((r.n_iters, "the CPU solve's own count") if small
                    else cpu_iteration_count(args, rec, fallback=n_iters))
    val = cpu_seconds_to_threshold(args, step_s, c_iters)
    cpu = {"value": val, "unit": "s", "cores": sinkhorn_c.threads("tiled"), "kind": "port",
           "extrapolated": not small, "measured_s": step_s,
           "sample": cpu_sample_text(args, c_iters, src)}
    if small:
      cpu.update(n_iters=r.n_iters, converged=bool(r.converged),
                 reg_ot_cost_rel_vs_gpu=abs(r.reg_ot_cost - out.reg_ot_cost)
                 / abs(out.reg_ot_cost))
    np_s, r_np, rows, workers = numpy_f32_baseline(args, x, y, a, b, eps)
    if small:
      np_val = np_s
      np_sample = f"whole solve to 1e-3 in float32 NumPy ({r_np.n_iters} iterations)"
    else:
      np_val = np_s / (4.0 * rows * args.n) * reference_sweeps(c_iters) * args.n * args.n
      np_sample = (f"1-iteration solve (4 sweeps) of the first {rows} of {args.n} rows x all "
                   f"{args.n} columns, per-entry time scaled to {reference_sweeps(c_iters)} "
                   "full sweeps")
    cpu_np = {"value": np_val, "unit": "s", "cores": workers, "kind": "port",
              "extrapolated": not small, "measured_s": np_s, "sample": np_sample}

  # error log fill, common centre, point preparation, potential init, the
  # persistent solve, finalize
  launches_per_solve = 6
  line = {
      "metric": METRIC, "value": ms * 1e-3, "unit": "s", "n_gpus": world,
      "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
      "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
      "dtype": "f32" if form == "fp32" else "bf16x3/f32", "data": "synthetic",
      "config": config_dict(args, n_iters), "form": form, "converged": converged,
      "iters_per_s": n_iters / t, "entries_per_s": entries / t,
      "plain_fp32": plain,
      "roofline": roof, "cpu_baseline": cpu, "cpu_baseline_numpy_f32": cpu_np,
      "accuracy_vs_fp64": accuracy,
      "e2e": {"value": e2e_ms * 1e-3, "unit": "s", "h2d_bytes_per_step": h2d,
              "d2h_bytes_per_step": d2h},
      "clocks": clk, "gpu_launches": launches_per_solve * args.steps,
      "pipe_peaks": peaks,
  }
  if rank == 0:
    print(json.dumps(line))
  if world > 1:
    dist.destroy_process_group()
  return 0


# ---------------------------------------------------------------------------
# learned warm start on a fixed 32 x 32 grid
# ---------------------------------------------------------------------------
def run_warmstart(args):
  """Trains the learned initializer on problems solved by the plain kernel
  and times held-out solves from zero init and from the warm start.

  Problems: 32 x 32 grid on [0, 1]^2 (n = m = 1024), sqeuclidean cost,
  epsilon 1e-2, weights from mixtures of 1-5 Gaussians plus a 1e-6 floor.
  Network 2048 -> 1024 x 3 -> 1024 (GELU), bf16 operands, FP32 master
  weights, Adam lr 1e-3 with cosine decay, batch 512, mass-weighted loss on
  g - eps log b. Held-out timing covers the network call,
  the warm solve and any fallback solves; the L2 is flushed before each
  timed chunk.
  """
  import torch
  from tests import problems
  from ott_b200.geometry import pointcloud
  from ott_b200.initializers.neural import meta_initializer
  from ott_b200.solvers.linear import sinkhorn
  torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
  grid = problems.grid_support(32)
  ntr, nte = args.train_pairs, args.test_pairs
  ev = lambda: torch.cuda.Event(enable_timing=True)
  W = problems.grid_mixture_weights(2 * (ntr + nte), grid, seed=0, device="cuda")
  A, B = W[0::2].contiguous(), W[1::2].contiguous()
  del W
  geom = pointcloud.PointCloud(torch.tensor(grid).cuda(), epsilon=1e-2)
  chunk = 2048
  flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device="cuda")

  # 1. training targets: the plain solver's g
  e0, e1 = ev(), ev()
  e0.record()
  G = torch.empty((ntr, 1024), dtype=torch.float32, device="cuda")
  it_train = []
  for s in range(0, ntr, chunk):
    e = min(s + chunk, ntr)
    out = sinkhorn.run_stacked(geom, A[s:e], B[s:e], sinkhorn.Sinkhorn())
    G[s:e] = out.g
    it_train.append(out.n_iters)
  e1.record()
  e1.synchronize()
  gen_s = e0.elapsed_time(e1) * 1e-3
  it_train = np.concatenate(it_train)

  # 2. training
  meta = meta_initializer.MetaInitializer(geom, dims=(1024, 1024, 1024), lr=1e-3, seed=0)
  e0.record()
  losses = meta_initializer.fit(meta, A[:ntr], B[:ntr], G, steps=args.train_steps,
                                batch_size=512).cpu().numpy()
  e1.record()
  e1.synchronize()
  train_s = e0.elapsed_time(e1) * 1e-3
  meta.mlp.check_status()
  dims = meta.mlp.dims
  mlp_flops = 3.0 * 2.0 * 512 * sum(dims[i] * dims[i + 1] for i in range(len(dims) - 1)) \
      * args.train_steps
  mp = load_peaks_json()
  bf16_sust = mp.get("bf16_tflops_sustained") if mp else None
  bf16_src = ("MEASURED_PEAKS.json bf16_tflops_sustained" if bf16_sust else
              "fallback: 1.4 PFLOP/s sustained, an earlier B200 measurement (file absent)")
  bf16_sust = bf16_sust or 1400.0
  del G

  # 3. held-out: zero init vs warm start (with fallback), same chunks
  At, Bt = A[ntr:], B[ntr:]

  def cold(a, b):
    o = sinkhorn.run_stacked(geom, a, b, sinkhorn.Sinkhorn())
    return o, np.zeros(0, np.int64)

  def warm(a, b):
    return meta_initializer.solve_warm_started(geom, a, b, meta)

  def timed(fn):
    fn(At[:chunk], Bt[:chunk])  # warm-up
    fn(At[:chunk], Bt[:chunk])
    fn(At[:chunk], Bt[:chunk])
    ms, its, costs, conv, redo = 0.0, [], [], [], 0
    for s in range(0, nte, chunk):
      flush.zero_()
      e0.record()
      o, r = fn(At[s:s + chunk], Bt[s:s + chunk])
      e1.record()
      e1.synchronize()
      ms += e0.elapsed_time(e1)
      n_it, cv, c = o.scalars()
      its.append(n_it)
      costs.append(c)
      conv.append(cv)
      redo += len(r)
    return (ms * 1e-3, np.concatenate(its), np.concatenate(costs), np.concatenate(conv),
            redo)

  clocks = ClockSampler(0)
  clocks.start()
  cold_s, it_c, cost_c, conv_c, _ = timed(cold)
  warm_s, it_w, cost_w, conv_w, redo = timed(warm)
  clk = clocks.stop()
  rel = np.abs(cost_w - cost_c) / np.abs(cost_c)

  # plain FP32 kernel, one problem per launch from zero init (the plain
  # form), on the first `sample` held-out problems, scaled to all of them
  sample = min(nte, 400)
  solver1 = sinkhorn.Sinkhorn()
  from ott_b200.problems.linear import linear_problem
  probs1 = [linear_problem.LinearProblem(geom, At[k], Bt[k]) for k in range(sample)]
  for p1 in probs1[:3]:
    solver1(p1).n_iters
  torch.cuda.synchronize()
  flush.zero_()
  e0.record()
  outs1 = [solver1(p1) for p1 in probs1]
  e1.record()
  e1.synchronize()
  plain_s = e0.elapsed_time(e1) * 1e-3 * nte / sample
  plain_it = float(np.mean([o1.n_iters for o1 in outs1]))
  line = {
      "metric": "s to 1e-3 marginal err: learned warm start vs zero init, 32x32 grid",
      "value": warm_s, "unit": "s", "higher_is_better": False, "n_gpus": 1,
      "workload": "warmstart", "dtype": "f32 solve / bf16 MLP", "data": "synthetic",
      "config": {"workload": f"{nte} held-out grid problems n=m=1024 d=2 eps=1e-2 thr=1e-3",
                 "train_pairs": ntr, "train_steps": args.train_steps, "batch": 512,
                 "net": "2048-1024-1024-1024-1024 GELU, Adam lr 1e-3 cosine",
                 "l2": "flushed before each timed chunk of 2048 problems"},
      "zero_init": {"s": cold_s, "mean_iters": float(it_c.mean()),
                    "converged": int(conv_c.sum())},
      "warm_start": {"s": warm_s, "mean_iters": float(it_w.mean()),
                     "converged": int(conv_w.sum()), "fallbacks": int(redo)},
      "speedup": cold_s / warm_s, "iteration_ratio": float(it_w.mean() / it_c.mean()),
      "plain_fp32_one_launch_per_problem": {
          "s": plain_s, "mean_iters": plain_it,
          "sample": f"first {sample} of {nte} held-out problems, time scaled by {nte}/{sample}"},
      "speedup_vs_plain_fp32": plain_s / warm_s,
      "cost_rel_diff": {"max": float(rel.max()), "median": float(np.median(rel))},
      "training": {"target_solve_s": gen_s, "target_mean_iters": float(it_train.mean()),
                   "train_s": train_s, "loss_first": float(losses[:20].mean()),
                   "loss_last": float(losses[-100:].mean()),
                   "mlp_train_tflops": mlp_flops / train_s / 1e12,
                   "mlp_train_frac_of_bf16_sustained": (
                       mlp_flops / train_s / 1e12 / bf16_sust if bf16_sust else None),
                   "bf16_sustained_source": bf16_src,
                   "mlp_flops": "3 x forward GEMM flops (forward, data and weight "
                                "gradients) x batch 512 x steps"},
      "clocks": clk,
  }
  print(json.dumps(line))
  return 0


# ---------------------------------------------------------------------------
# batched uneven problems in one persistent launch
# ---------------------------------------------------------------------------
def run_batched(args):
  """512 independent problems, n_k and m_k log-uniform in [128, 16384],
  d = 32, 4-component Gaussian-mixture clouds, Dirichlet(1) weights,
  epsilon_k = 0.05 * mean(C_k), threshold 1e-3: one launch for all of them
  (chosen precision and FP32), and one launch per problem for comparison.
  Inputs (~440 MB) exceed the L2."""
  import torch
  import torch.distributed as dist
  from datetime import timedelta
  from tests import problems
  from ott_b200 import distributed as odist
  from ott_b200.geometry import pointcloud
  from ott_b200.problems.linear import linear_problem
  from ott_b200.solvers.linear import sinkhorn
  world = int(os.environ.get("WORLD_SIZE", "1"))
  rank = int(os.environ.get("RANK", "0"))
  local = int(os.environ.get("LOCAL_RANK", "0"))
  torch.cuda.set_device(local)
  if world > 1:
    # one process per GPU; each rank solves its own batch (the job is
    # world x problems independent problems), no data-path collective
    dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                            device_id=torch.device("cuda", local))
  peaks = measure_pipe_peaks(torch)
  data = problems.batched_uneven_problems(args.problems, d=32, seed=rank)
  probs = []
  for x, y, a, b in data:
    geom = pointcloud.PointCloud(torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(),
                                 epsilon=0.05, relative_epsilon="mean")
    probs.append(linear_problem.LinearProblem(geom, torch.from_numpy(a).cuda(),
                                              torch.from_numpy(b).cuda()))
  for p in probs:
    _ = p.geom.epsilon  # resolve the relative epsilons before timing
  entries_per_it = 2.0 * sum(p.geom.shape[0] * p.geom.shape[1] for p in probs)
  ev = lambda: torch.cuda.Event(enable_timing=True)

  def barrier():
    if world > 1:
      dist.barrier()
    torch.cuda.synchronize()

  def timed(fn, steps, warm):
    for _ in range(warm):
      fn()
    barrier()
    ms, outs = 0.0, None
    for _ in range(steps):
      e0, e1 = ev(), ev()
      e0.record()
      outs = fn()
      e1.record()
      e1.synchronize()
      ms += e0.elapsed_time(e1)
    barrier()
    return odist.max_over_ranks(ms / steps * 1e-3), outs

  def batch(precision, autotune=False):
    solver = sinkhorn.Sinkhorn(precision=precision, autotune=autotune)
    return lambda: sinkhorn.run_batch(probs, solver)

  def one_by_one(precision):
    solver = sinkhorn.Sinkhorn(precision=precision)
    return lambda: [solver(p) for p in probs]

  # the chosen form: schedule picked by the autotuner (its trials run here,
  # before timing), the whole solve captured once in a CUDA graph and replayed
  graph = sinkhorn.SinkhornGraph(probs, sinkhorn.Sinkhorn(precision="auto", autotune=True))
  clocks = ClockSampler(0)
  clocks.start()
  t_b, o_b = timed(graph.replay, args.steps, args.warmup)
  clk = clocks.stop()
  t_d, _ = timed(batch("auto", autotune=True), 1, 1)
  # each tensor-core tile width pinned (the autotuner's other dimension)
  tiles = {}
  for tile in (256, 128):
    sinkhorn.set_schedule(probs, sinkhorn.Sinkhorn(precision="auto"), waves=2, dynamic=1,
                          tile_n=tile)
    tiles[str(tile)] = timed(batch("auto"), 1, 1)[0]
  t_f, o_f = timed(batch("fp32"), 1, 1)
  t_s, o_s = timed(one_by_one("auto"), 1, 1)
  it_b = np.array([o.n_iters for o in o_b])
  it_f = np.array([o.n_iters for o in o_f])
  conv = np.array([o.converged for o in o_b])
  c_b = np.array([o.reg_ot_cost for o in o_b])
  c_f = np.array([o.reg_ot_cost for o in o_f])
  entries = sum(2.0 * p.geom.shape[0] * p.geom.shape[1] * o.n_iters
                for p, o in zip(probs, o_b))
  ach = entries / t_b / 1e9
  roof = {"bound": "mufu_ex2", "achieved": ach, "peak": peaks["ex2_per_s"] / 1e9,
          "unit": "Gex2/s", "frac": ach / (peaks["ex2_per_s"] / 1e9),
          "peak_source": "measured in bench.py (MUFU ex2 probe kernel)"}
  if clk and clk.get("sm_mhz"):
    at = 16 * torch.cuda.get_device_properties(0).multi_processor_count * clk["sm_mhz"] * 1e-3
    roof["peak_at_sampled_clock"] = at
    roof["frac_at_sampled_clock"] = ach / at
  sizes = np.array([p.geom.shape for p in probs])
  n_conv = int(odist.sum_over_ranks(float(conv.sum())))
  line = {
      "metric": "s to 1e-3 marginal err, 512 uneven problems in one launch",
      "value": t_b, "unit": "s", "higher_is_better": False, "n_gpus": world,
      "scaling": "weak", "parallelism": f"{world} rank(s) x {args.problems} problems, "
                                         "no data-path collective",
      "workload": "batched", "dtype": "bf16x3/f32", "data": "synthetic",
      "steps": args.steps, "warmup": args.warmup,
      "config": {"workload": f"{args.problems} problems n,m log-uniform [128,16384] d=32 "
                             "GMM clouds, Dirichlet(1) weights, eps=0.05*mean(C_k), thr=1e-3",
                 "form": "one persistent launch, schedule from the autotuner, solve "
                         "captured in a CUDA graph and replayed",
                 "total_entries_per_iteration": entries_per_it,
                 "n_range": [int(sizes[:, 0].min()), int(sizes[:, 0].max())],
                 "l2": "inputs ~440 MB > L2"},
      "converged": n_conv, "mean_iters": float(it_b.mean()),
      "max_iters": int(it_b.max()),
      "entries_per_s": odist.sum_over_ranks(entries) / t_b,  # whole job, all ranks
      "direct_call_no_graph": {"s": t_d},
      "tile_width_s": tiles,
      "plain_fp32_batched": {"s": t_f, "mean_iters": float(it_f.mean())},
      "one_launch_per_problem": {"s": t_s},
      "speedup_vs_plain_fp32": t_f / t_b, "speedup_vs_per_problem": t_s / t_b,
      "cost_rel_diff_vs_fp32": float(np.max(np.abs(c_b - c_f) / np.abs(c_f))),
      "iters_equal_fp32": int((it_b == it_f).sum()),
      "roofline": roof, "clocks": clk,
  }
  if rank == 0:
    print(json.dumps(line))
  if world > 1:
    dist.destroy_process_group()
  return 0


# ---------------------------------------------------------------------------
# epsilon-annealed solves
# ---------------------------------------------------------------------------
def run_anneal(args):
  """``--pairs`` pairs of 8-component Gaussian mixtures in R^128 (means
  N(0, I), std U[0.2, 1]), n = m = ``--n``, uniform weights; epsilon annealed
  geometrically from 1 to 1e-3 * mean(C) over ``--stages`` stages, threshold
  1e-3 per stage, every pair in one launch per stage; FP32 redoes any stage
  the chosen form does not converge. The timed form starts stages from the
  third on from the learned stage predictor (a per-point MLP trained here on
  ``--train-chains`` other pairs of the family, solved by the plain FP32
  kernel); beside it the same chain started from the previous stage's
  potentials and from their linear extrapolation in epsilon. The plain FP32
  chain on pair 0 is the accuracy reference at full size, a committed
  float64 chain at n = m = 2048 below it."""
  import torch
  from tests import problems
  from ott_b200.solvers.linear import annealing
  torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
  d = 128
  pairs = [problems.gmm8_pair(args.n, args.n, d, seed=s) for s in range(args.pairs)]
  xs = [torch.from_numpy(p[0]).cuda() for p in pairs]
  ys = [torch.from_numpy(p[1]).cuda() for p in pairs]
  del pairs
  ev = lambda: torch.cuda.Event(enable_timing=True)

  def timed(fn):
    e0, e1 = ev(), ev()
    e0.record()
    out = fn()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3, out

  run = lambda xs_, ys_, prec, fb, warm=None: annealing.solve_annealed(
      xs_, ys_, stages=args.stages, start=1.0, final=1e-3, precision=prec,
      fallback_precision=fb, warm_start=warm)
  # warm-up on a reduced copy (compiles nothing; loads modules, sizes caches)
  run([x[:4096] for x in xs[:1]], [y[:4096] for y in ys[:1]], "auto", "fp32")

  # the learned warm start: chains of other pairs of the family solved by the
  # plain FP32 kernel, the per-point stage predictor fitted to them
  tn = args.train_n or args.n
  tr = [problems.gmm8_pair(tn, tn, d, seed=1000 + s) for s in range(args.train_chains)]
  txs = [torch.from_numpy(p[0]).cuda() for p in tr]
  tys = [torch.from_numpy(p[1]).cuda() for p in tr]
  del tr
  t_chain, train = timed(lambda: annealing.solve_annealed(
      txs, tys, stages=args.stages, start=1.0, final=1e-3, precision="fp32",
      fallback_precision=None, record_f=True))
  del txs, tys
  chains = [(train.f_history[k], train.stage_epsilons[:, k]) for k in range(args.train_chains)]
  pred = annealing.StagePredictor(seed=0)
  t_fit, losses = timed(lambda: pred.fit(chains, steps=2000).cpu().numpy())
  del chains, train

  class Extrapolated:
    """Non-learned comparison: f_s = f_{s-1} + linear extrapolation in eps."""

    def predict_f(self, f_hist, eps_hist, eps):
      return f_hist[-1].float() + float(eps) * annealing.stage_features(
          f_hist, eps_hist, eps)[:, 0]

  run(xs[:1], ys[:1], "auto", "fp32", pred)  # warm-up of the predictor's workspaces
  clocks = ClockSampler(0)
  clocks.start()
  t_c, out = timed(lambda: run(xs, ys, "auto", "fp32"))
  t_w, wout = timed(lambda: run(xs, ys, "auto", "fp32", pred))
  clk = clocks.stop()
  t_x, xout = timed(lambda: run(xs, ys, "auto", "fp32", Extrapolated()))
  it = out.stage_iters
  entries = float((2.0 * args.n * args.n * it).sum())
  wit = wout.stage_iters
  w_entries = float((2.0 * args.n * args.n * wit).sum())
  cost_rel = max(abs(o2.reg_ot_cost - o1.reg_ot_cost) / abs(o1.reg_ot_cost)
                 for o1, o2 in zip(out.outputs, wout.outputs))
  line = {
      "metric": "s to 1e-3 marginal err per stage, epsilon annealed 1 -> 1e-3 mean(C)",
      "value": t_w, "unit": "s", "higher_is_better": False, "n_gpus": 1,
      "workload": "anneal", "dtype": "bf16x3/f32", "data": "synthetic",
      "config": {"workload": f"{args.pairs} pairs GMM8 n=m={args.n} d={d}, "
                             f"{args.stages} geometric stages 1 -> 1e-3 mean(C), thr 1e-3",
                 "l2": f"inputs {2 * args.pairs * args.n * d * 4 / 2**20:.0f} MiB"},
      "stage_iters_mean": wit.mean(axis=1).tolist(), "total_iters": int(wit.sum()),
      "entries_per_s": w_entries / t_w, "fallbacks": wout.fallbacks,
      "converged": int(sum(o.converged for o in wout.outputs)),
      "form": "learned stage warm start (per-point MLP, tcgen05 bf16) + BF16 split-3 "
              "solves, FP32 fallback",
      "previous_stage_start": {"s": t_c, "stage_iters_mean": it.mean(axis=1).tolist(),
                               "total_iters": int(it.sum()), "entries_per_s": entries / t_c,
                               "fallbacks": out.fallbacks},
      "extrapolated_start": {"s": t_x, "stage_iters_mean":
                             xout.stage_iters.mean(axis=1).tolist(),
                             "total_iters": int(xout.stage_iters.sum()),
                             "fallbacks": xout.fallbacks},
      "learned_vs_previous": {"speedup": t_c / t_w,
                              "iteration_ratio": float(wit.sum() / it.sum()),
                              "reg_ot_cost_max_rel_diff": cost_rel},
      "training": {"pairs": args.train_chains, "n": tn, "chains_fp32_s": t_chain, "fit_s": t_fit,
                   "steps": 2000, "loss_first": float(losses[:20].mean()),
                   "loss_last": float(losses[-100:].mean())},
      "clocks": clk,
  }
  # accuracy against a float64 annealed chain at a reduced size (pair seed 0,
  # n = m = 2048): the float64 oracle's chain is committed in tests/golden
  rec_path = os.path.join(GOLDEN, "anneal_gmm8_n2048_d128.fp64.npz")
  if os.path.exists(rec_path) and args.stages == 10:
    rec = np.load(rec_path)
    p0 = problems.gmm8_pair(2048, 2048, d, seed=0)
    sx, sy = [torch.from_numpy(p0[0]).cuda()], [torch.from_numpy(p0[1]).cuda()]
    acc = {"n": 2048, "reference": "tests/golden/anneal_gmm8_n2048_d128.fp64.npz "
                                   "(float64 oracle, same chain)",
           "stage_iters_fp64": rec["stage_iters"].tolist()}
    for name, w in (("previous_stage_start", None), ("learned", pred)):
      o = run(sx, sy, "auto", "fp32", w)
      acc[name] = {"reg_ot_cost_rel": abs(o.outputs[0].reg_ot_cost - float(rec["reg_ot_cost"]))
                                      / abs(float(rec["reg_ot_cost"])),
                   "stage_iters": o.stage_iters[:, 0].tolist()}
    line["accuracy_vs_fp64"] = acc
  if not args.no_plain:
    t_p, plain = timed(lambda: run(xs[:1], ys[:1], "fp32", None))
    c0, c1 = wout.outputs[0].reg_ot_cost, plain.outputs[0].reg_ot_cost
    line["plain_fp32_pair0"] = {
        "s": t_p, "stage_iters": plain.stage_iters[:, 0].tolist(),
        "chosen_stage_iters": wit[:, 0].tolist(),
        "reg_ot_cost_rel_diff": abs(c0 - c1) / abs(c1),
        "speedup_per_pair": t_p / (t_w / args.pairs)}
  print(json.dumps(line))
  return 0


# ---------------------------------------------------------------------------
# Sinkhorn divergence and its gradient
# ---------------------------------------------------------------------------
def run_divergence(args):
  """Sinkhorn divergence of the Gaussian-shift clouds (n = m = ``--n``,
  d = ``--d``, uniform weights, epsilon = 0.05 * mean(C) of (x, y)): the
  (x, y), (x, x), (y, y) solves in one launch (symmetric terms with the
  parallel, momentum-1/2 update), then the gradient w.r.t. x and y (two
  applications of each plan to d + 1 vectors). Chosen precision and FP32."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.tools import sinkhorn_divergence as sd
  torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
  peaks = measure_pipe_peaks(torch)
  x, y, _, _ = workload(args)
  xt = torch.from_numpy(x).cuda().requires_grad_()
  yt = torch.from_numpy(y).cuda().requires_grad_()
  ev = lambda: torch.cuda.Event(enable_timing=True)
  flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device="cuda")

  def step(precision):
    xt.grad = None
    yt.grad = None
    e0, e1, e2 = ev(), ev(), ev()
    flush.zero_()
    e0.record()
    div, out = sd.sinkhorn_divergence(pointcloud.PointCloud, xt, yt, epsilon=0.05,
                                      relative_epsilon="mean",
                                      solve_kwargs=dict(precision=precision))
    e1.record()
    div.backward()
    e2.record()
    e2.synchronize()
    return e0.elapsed_time(e1), e1.elapsed_time(e2), float(div), out

  for _ in range(args.warmup):
    step("auto")
  clocks = ClockSampler(0)
  clocks.start()
  fw, bw = [], []
  for _ in range(args.steps):
    a, b_, div, out = step("auto")
    fw.append(a)
    bw.append(b_)
  clk = clocks.stop()
  gx, gy = xt.grad.clone(), yt.grad.clone()
  step("fp32")  # warm-up of the FP32 arm
  pf, pb, pdiv, pout = step("fp32")
  grad_diff = max(float((gx - xt.grad).abs().max() / xt.grad.abs().max()),
                  float((gy - yt.grad).abs().max() / yt.grad.abs().max()))
  n, d = args.n, args.d
  iters = list(out.n_iters)
  fwd_s = statistics.median(fw) * 1e-3
  bwd_s = statistics.median(bw) * 1e-3
  # backward: 4 applications of an n x n plan to d + 1 vectors (2 for the
  # (x, y) term, 1 for each symmetric term, whose plan is symmetric). The
  # chosen form runs each on ottb_apply_transport_tc: the kernel's max-only
  # first pass and its product, both tcgen05 BF16 (tensor flops per plan
  # entry from tc_apply_flops_per_entry); FP32 (the plain arm): 2 d +
  # 2 (d + 1) flops per entry on the FMA pipe
  tc_flops = 4.0 * n * n * tc_apply_flops_per_entry(d, d + 1)
  bf16_peak, bf16_src = bf16_peak_tflops()
  roof = {"bound": "tensor", "kernel": "apply_tc_kernel (its first pass and the product)",
          "achieved": tc_flops / bwd_s / 1e12, "peak": bf16_peak, "unit": "TFLOP/s",
          "frac": tc_flops / bwd_s / 1e12 / bf16_peak, "peak_source": bf16_src,
          "work_per_backward": f"{tc_flops:.3e} BF16 tensor flops (4 applications to "
                               f"{d + 1} vectors, split-3 products)"}
  fp32_flops = 4.0 * n * n * (2 * d + 2 * (d + 1))
  roof_fp32 = {"bound": "fp32_fma", "kernel": "apply_pipelined_kernel",
               "achieved": fp32_flops / (pb * 1e-3) / 1e12,
               "peak": 2 * peaks["ffma_per_s"] / 1e12, "unit": "TFLOP/s",
               "frac": fp32_flops / (pb * 1e-3) / (2 * peaks["ffma_per_s"]),
               "peak_source": "measured in bench.py (FFMA probe kernel)"}
  line = {
      "metric": "s per Sinkhorn divergence (3 solves to 1e-3 in one launch) and its gradient",
      "value": fwd_s + bwd_s, "unit": "s", "higher_is_better": False, "n_gpus": 1,
      "workload": "divergence", "dtype": "bf16x3/f32", "data": "synthetic",
      "steps": args.steps, "warmup": args.warmup,
      "config": {"workload": f"sinkhorn_divergence n=m={n} d={d} x~N(0,I), "
                             "y~N(0.5,diag(U[0.5,2])), uniform weights, eps=0.05*mean(C_xy)",
                 "l2": "flushed before each step (256 MiB write)"},
      "forward_s": fwd_s, "backward_s": bwd_s, "divergence": div, "n_iters": iters,
      "plain_fp32": {"forward_s": pf * 1e-3, "backward_s": pb * 1e-3, "divergence": pdiv,
                     "n_iters": list(pout.n_iters), "roofline_backward": roof_fp32},
      "divergence_rel_diff_vs_fp32": abs(div - pdiv) / abs(pdiv),
      "grad_rel_diff_vs_fp32": grad_diff,
      "speedup_forward_vs_plain_fp32": pf * 1e-3 / fwd_s,
      "speedup_backward_vs_plain_fp32": pb * 1e-3 / bwd_s,
      "roofline_backward": roof, "clocks": clk,
  }
  print(json.dumps(line))
  return 0


def run_implicit(args):
  """Gradient through the potentials of the headline problem (Gaussian-shift
  clouds, n = m = ``--n``, d = ``--d``, uniform weights, epsilon = 0.01 *
  mean(C), threshold 1e-3): the solve (chosen precision), then the backward
  of ``<w, f> + <v, g>`` (sum w = sum v) by implicit differentiation. Its
  MINRES steps apply the plan to one vector twice each; with the chosen
  precision at d >= 32 each such product is two zero-iteration solves on
  the tensor-core sweep (``ottb_apply_transport_sweep``). Also reported:
  the same gradient with the solve and the backward in FP32."""
  import torch
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  from ott_b200.solvers.linear import implicit_differentiation as imp
  torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
  peaks = measure_pipe_peaks(torch)
  x, y, _, _ = workload(args)
  n, d = args.n, args.d
  xt = torch.from_numpy(x).cuda().requires_grad_()
  yt = torch.from_numpy(y).cuda().requires_grad_()
  rng = np.random.default_rng(0)
  w = torch.from_numpy(rng.standard_normal(n)).cuda()
  v = torch.from_numpy(rng.standard_normal(n)).cuda()
  v += (w.sum() - v.sum()) / n
  ev = lambda: torch.cuda.Event(enable_timing=True)
  flush = torch.empty(2 * L2_BYTES, dtype=torch.uint8, device="cuda")

  def step(precision):
    xt.grad = None
    yt.grad = None
    e0, e1, e2 = ev(), ev(), ev()
    flush.zero_()
    e0.record()
    geom = pointcloud.PointCloud(xt, yt, epsilon=0.01, relative_epsilon="mean")
    out = linear.solve(geom, threshold=1e-3, precision=precision)
    loss = (out.f.double() * w).sum() + (out.g.double() * v).sum()
    e1.record()
    loss.backward()
    e2.record()
    e2.synchronize()
    return (e0.elapsed_time(e1), e1.elapsed_time(e2), out, geom, dict(imp.last_solve_info),
            xt.grad.clone())

  for _ in range(args.warmup):
    step(args.precision)
  clocks = ClockSampler(0)
  clocks.start()
  fw, bw = [], []
  for _ in range(args.steps):
    a_, b_, out, geom, info, grad = step(args.precision)
    fw.append(a_)
    bw.append(b_)
  clk = clocks.stop()
  fwd_s = statistics.median(fw) * 1e-3
  bwd_s = statistics.median(bw) * 1e-3
  pf, pb, pout, _, pinfo, pgrad = step("fp32")
  grad_diff = float((grad - pgrad).abs().max() / pgrad.abs().max())
  # the same backward with its MINRES steps replayed from a CUDA graph in
  # blocks of 4 instead of issued one by one from the host
  block = imp.MINRES_GRAPH_BLOCK
  imp.MINRES_GRAPH_BLOCK = 4
  try:
    gb = [step(args.precision)[1] for _ in range(max(1, min(args.steps, 3)))]
  finally:
    imp.MINRES_GRAPH_BLOCK = block
  bwd_graph_s = statistics.median(gb) * 1e-3
  # one single-vector product of the backward, timed alone, in both forms
  f, g = out.f.detach(), out.g.detach()
  vec = torch.randn(1, n, device="cuda")

  def time_app(prec, reps=20):
    for _ in range(3):
      geom._apply_raw(f, g, vec, 1, prec)
    e0, e1 = ev(), ev()
    e0.record()
    for _ in range(reps):
      geom._apply_raw(f, g, vec, 1, prec)
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / reps * 1e-3

  # the backward's own route: the sweep under the chosen precision at d >= 32
  # from 2^25 plan entries, FP32 products below
  tc = args.precision == "bf16_split3" or (
      args.precision == "auto" and d >= 32 and n * n >= imp.ImplicitDiff._TC_MIN_ENTRIES)
  t_app = time_app(args.precision if tc else "fp32")
  t_app32 = time_app("fp32")
  steps = int(info.get("steps", 0))
  n_app1 = 2 * steps + 4
  if tc:
    # two sweeps of n x m entries (v+ and v-), one exponential per entry
    ach = 2.0 * n * n / t_app / 1e9
    roof = {"bound": "mufu_ex2", "kernel": "sinkhorn persistent sweep (2 zero-iteration "
                                            "solves per product)",
            "achieved": ach, "peak": peaks["ex2_per_s"] / 1e9, "unit": "Gex2/s",
            "frac": ach / (peaks["ex2_per_s"] / 1e9),
            "work_per_launch": f"{2.0 * n * n:.4g} cost entries (2 sweeps of n*m)",
            "peak_source": "measured in bench.py (MUFU ex2 probe kernel)"}
  else:
    flops_app = float(n) * n * (2 * d + 2)
    roof = {"bound": "fp32_fma", "kernel": "apply_direct_kernel (one vector)",
            "achieved": flops_app / t_app / 1e12, "peak": 2 * peaks["ffma_per_s"] / 1e12,
            "unit": "TFLOP/s", "frac": flops_app / t_app / (2 * peaks["ffma_per_s"]),
            "work_per_launch": f"{flops_app:.4g} flops (n*m*(2d+2))",
            "peak_source": "measured in bench.py (FFMA probe kernel)"}
  flops32 = float(n) * n * (2 * d + 2)
  line = {
      "metric": "s per gradient through the Sinkhorn potentials (implicit differentiation)",
      "value": fwd_s + bwd_s, "unit": "s", "higher_is_better": False, "n_gpus": 1,
      "workload": "implicit",
      "dtype": ("bf16x3/f32" if (tc or (args.precision == "auto" and d >= 32)) else "f32"),
      "backward_products": "tensor-core sweep" if tc else "fp32",
      "data": "synthetic", "steps": args.steps, "warmup": args.warmup,
      "config": {"workload": f"grad of <w,f>+<v,g> through linear.solve, n=m={n} d={d} "
                             "x~N(0,I), y~N(0.5,diag(U[0.5,2])), uniform weights, "
                             "eps=0.01*mean(C), thr=1e-3",
                 "l2": "flushed before each step (256 MiB write)"},
      "forward_s": fwd_s, "backward_s": bwd_s, "n_iters": out.n_iters,
      "minres_graph_block": block, "backward_s_graph_replayed_blocks_of_4": bwd_graph_s,
      "minres_steps": steps, "minres_rel_residual": info.get("rel_residual"),
      "recomputed_rel_residual": info.get("true_rel_residual"),
      "single_vector_products": n_app1, "single_vector_product_s": t_app,
      "backward_share_in_single_vector_products": n_app1 * t_app / bwd_s,
      "plain_fp32": {"forward_s": pf * 1e-3, "backward_s": pb * 1e-3,
                     "minres_steps": int(pinfo.get("steps", 0)),
                     "single_vector_product_s": t_app32,
                     "single_vector_product_frac_of_ffma_peak":
                         flops32 / t_app32 / (2 * peaks["ffma_per_s"])},
      "grad_rel_diff_vs_fp32": grad_diff,
      "speedup_backward_vs_plain_fp32": pb * 1e-3 / bwd_s,
      "roofline": roof, "clocks": clk,
  }
  print(json.dumps(line))
  return 0


def run_sharded(args):
  """The headline problem (n = m = ``--n``, d = ``--d``, epsilon = 0.01 *
  mean(C), threshold 1e-3) row-sharded over the ranks (strong scaling: the
  problem is fixed, each rank holds n / N rows of x and all of y): per
  iteration two log-domain kernel applications per rank
  (``ottb_apply_lse_kernel``) and one all-gather of the column
  log-sum-exps. Time to threshold, max over ranks; against the one-launch
  persistent solve of the same problem on one GPU."""
  import torch
  import torch.distributed as dist
  from datetime import timedelta
  from ott_b200 import distributed as odist
  from ott_b200.geometry import pointcloud
  from ott_b200.solvers import linear
  from ott_b200.solvers.linear import sharded
  world = int(os.environ.get("WORLD_SIZE", "1"))
  rank = int(os.environ.get("RANK", "0"))
  local = int(os.environ.get("LOCAL_RANK", "0"))
  torch.cuda.set_device(local)
  if world > 1:
    dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                            device_id=torch.device("cuda", local))
  x, y, a, b = workload(args)
  lo, hi = odist.shard_bounds([1.0] * args.n, world)[rank]
  xd = torch.from_numpy(x[lo:hi]).cuda()
  yd = torch.from_numpy(y).cuda()
  ad = torch.from_numpy(a[lo:hi]).cuda()
  bd = torch.from_numpy(b).cuda()
  ev = lambda: torch.cuda.Event(enable_timing=True)

  def step():
    out = sharded.solve_sharded(xd, yd, ad, bd, epsilon=0.01, relative_epsilon="mean",
                                threshold=1e-3, precision=args.precision)
    return out

  for _ in range(args.warmup):
    step()
  if world > 1:
    dist.barrier()
  torch.cuda.synchronize()
  clocks = ClockSampler(local)
  clocks.start()
  e0, e1 = ev(), ev()
  e0.record()
  for _ in range(args.steps):
    out = step()
  e1.record()
  e1.synchronize()
  clk = clocks.stop()
  t = odist.max_over_ranks(e0.elapsed_time(e1) / args.steps * 1e-3)
  single = None
  if world == 1:
    geom = pointcloud.PointCloud(torch.from_numpy(x).cuda(), yd, epsilon=0.01,
                                 relative_epsilon="mean")
    for _ in range(2):
      linear.solve(geom, threshold=1e-3, precision=args.precision).n_iters
    e0, e1 = ev(), ev()
    e0.record()
    ref = linear.solve(geom, threshold=1e-3, precision=args.precision)
    e1.record()
    e1.synchronize()
    single = {"s": e0.elapsed_time(e1) * 1e-3, "n_iters": ref.n_iters,
              "reg_ot_cost": ref.reg_ot_cost}
  line = {
      "metric": "s to 1e-3 marginal err, one problem row-sharded over the ranks",
      "value": t, "unit": "s", "higher_is_better": False, "n_gpus": world,
      "scaling": "strong", "workload": "sharded", "data": "synthetic",
      "steps": args.steps, "warmup": args.warmup,
      "config": {"workload": f"sinkhorn sqeuclidean n=m={args.n} d={args.d} eps=0.01*mean(C) "
                             f"thr=1e-3, rows split over {world} rank(s)",
                 "parallelism": f"row shards x{world}, all-gather of m column LSEs per "
                                "iteration"},
      "n_iters": out.n_iters, "reg_ot_cost": out.reg_ot_cost, "converged": out.converged,
      "one_gpu_persistent_solve": single, "clocks": clk,
  }
  if rank == 0:
    print(json.dumps(line))
  if world > 1:
    dist.destroy_process_group()
  return 0


def main():
  args = parse_args()
  if args.warmup < 3:
    print("warning: fewer than 3 warm-up steps", file=sys.stderr)
  if args.impl == "reference":
    return run_reference(args)
  if args.workload == "warmstart":
    return run_warmstart(args)
  if args.workload == "batched":
    return run_batched(args)
  if args.workload == "anneal":
    return run_anneal(args)
  if args.workload == "divergence":
    return run_divergence(args)
  if args.workload == "implicit":
    return run_implicit(args)
  if args.workload == "sharded":
    return run_sharded(args)
  return run_ours(args)


if __name__ == "__main__":
  sys.exit(main())
