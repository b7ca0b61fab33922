"""Fits the polynomial p(f) ~ 2^f on f in [-1/2, 1/2] used by exp2_poly()
in engine_tc.cuh, minimising the maximum RELATIVE error (Remez exchange on
the weighted error (p - 2^f) / 2^f), then rounds the coefficients to float32
and reports the error of the float32 evaluation.

    python tests/exp2_poly_fit.py [degree]
"""
import sys

import numpy as np


def remez_relative(deg, lo=-0.5, hi=0.5, iters=30):
  target = lambda x: np.exp2(x)
  n = deg + 2
  # initial reference: Chebyshev extrema
  k = np.arange(n)
  xs = 0.5 * (lo + hi) + 0.5 * (hi - lo) * np.cos(np.pi * k[::-1] / (n - 1))
  grid = np.linspace(lo, hi, 200001)
  coef = None
  for _ in range(iters):
    # solve p(x_i) - 2^x_i = (-1)^i E 2^x_i for coefficients and E
    A = np.zeros((n, n))
    for i, x in enumerate(xs):
      A[i, :deg + 1] = x ** np.arange(deg + 1)
      A[i, deg + 1] = -((-1) ** i) * target(x)
    sol = np.linalg.solve(A, target(xs))
    coef = sol[:deg + 1]
    err = (np.polyval(coef[::-1], grid) - target(grid)) / target(grid)
    # new reference: extrema of the error between sign changes
    sgn = np.sign(err)
    idx = np.where(np.diff(sgn) != 0)[0]
    bounds = np.concatenate([[0], idx + 1, [len(grid)]])
    ext = [b0 + np.argmax(np.abs(err[b0:b1])) for b0, b1 in zip(bounds[:-1], bounds[1:])]
    if len(ext) < n:
      break
    # keep the n largest alternating extrema
    while len(ext) > n:
      if abs(err[ext[0]]) < abs(err[ext[-1]]):
        ext = ext[1:]
      else:
        ext = ext[:-1]
    xs = grid[ext]
  return coef, np.max(np.abs(err))


def eval_f32(coef32, f):
  p = np.float32(coef32[-1])
  for c in coef32[-2::-1]:
    p = np.float32(np.float32(p * f) + np.float32(c))
  return p


def main():
  deg = int(sys.argv[1]) if len(sys.argv) > 1 else 5
  coef, err = remez_relative(deg)
  c32 = coef.astype(np.float32)
  f = np.linspace(-0.5, 0.5, 100001).astype(np.float32)
  p = np.array([eval_f32(c32, v) for v in f[::50]])
  rel = np.abs(p.astype(np.float64) / np.exp2(f[::50].astype(np.float64)) - 1)
  print(f"degree {deg}: minimax relative error {err:.3e}, float32 evaluation {rel.max():.3e}")
  for i, c in enumerate(c32):
    print(f"  c{i} = {float(c):.9e}f  ({np.float32(c).view(np.uint32):#010x})")


if __name__ == "__main__":
  main()
