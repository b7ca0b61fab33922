"""Seeded synthetic problems shared by the tests, the smoke check and the
bench (numpy.random.default_rng; shapes and distributions of the workloads
the solver is measured on)."""
from __future__ import annotations

import numpy as np


def ref_test_problem(seed=0, n=17, m=29, d=4):
  """The reference tests' generic problem (sinkhorn_test.py:38-54): uniform
  points, uniform weights with a[0] = b[3] = 0, normalised."""
  rng = np.random.default_rng(seed)
  x = rng.uniform(size=(n, d)).astype(np.float32)
  y = rng.uniform(size=(m, d)).astype(np.float32)
  a = rng.uniform(size=n).astype(np.float32)
  b = rng.uniform(size=m).astype(np.float32)
  a[0] = 0
  if m > 3:
    b[3] = 0
  return x, y, (a / a.sum()).astype(np.float32), (b / b.sum()).astype(np.float32)


def uniform_cloud_problem(n, m, d, seed=0):
  """x, y ~ U[0,1]^d; a, b = U(0,1) + 0.2 normalised (the n=m=2048, d=2
  workload)."""
  rng = np.random.default_rng(seed)
  x = rng.uniform(size=(n, d)).astype(np.float32)
  y = rng.uniform(size=(m, d)).astype(np.float32)
  a = (rng.uniform(size=n) + 0.2).astype(np.float32)
  b = (rng.uniform(size=m) + 0.2).astype(np.float32)
  return x, y, (a / a.sum()).astype(np.float32), (b / b.sum()).astype(np.float32)


def gaussian_shift_problem(n, m, d, seed=0):
  """x ~ N(0, I_d), y ~ N(0.5 * 1, diag(U[0.5, 2])), uniform weights (the
  n=m=65536, d=64 workload)."""
  rng = np.random.default_rng(seed)
  x = rng.standard_normal((n, d)).astype(np.float32)
  var = rng.uniform(0.5, 2.0, size=d)
  y = (0.5 + rng.standard_normal((m, d)) * np.sqrt(var)).astype(np.float32)
  a = np.full(n, 1.0 / n, np.float32)
  b = np.full(m, 1.0 / m, np.float32)
  return x, y, a, b


def gmm_cloud(rng, n, d, k=4, mean_scale=2.0, std=0.5):
  """k-component Gaussian mixture in R^d: means N(0, mean_scale^2 I),
  covariance std^2 I, equal component probabilities."""
  means = rng.standard_normal((k, d)) * mean_scale
  comp = rng.integers(0, k, size=n)
  return (means[comp] + std * rng.standard_normal((n, d))).astype(np.float32)


def batched_uneven_problems(num, d=32, lo=128, hi=16384, seed=0):
  """num problems, n_k, m_k log-uniform in [lo, hi], 4-component GMM clouds
  (means N(0, 4I), covariance 0.25 I), Dirichlet(1) weights."""
  rng = np.random.default_rng(seed)
  out = []
  for _ in range(num):
    n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
    m = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
    x = gmm_cloud(rng, n, d)
    y = gmm_cloud(rng, m, d)
    a = rng.dirichlet(np.ones(n)).astype(np.float32)
    b = rng.dirichlet(np.ones(m)).astype(np.float32)
    out.append((x, y, a, b))
  return out


def grid_support(side=32):
  """side x side grid on [0, 1]^2 (the fixed support of the learned warm
  start workload), row-major."""
  t = np.linspace(0.0, 1.0, side)
  gx, gy = np.meshgrid(t, t, indexing="ij")
  return np.stack([gx.ravel(), gy.ravel()], axis=1).astype(np.float32)


def grid_mixture_weights(num, grid, seed=0, floor=1e-6, chunk=4096, device=None):
  """num measures on a fixed grid: each is a mixture of 1-5 isotropic
  Gaussians (means U[0,1]^2, std U[0.03, 0.2], mixture weights Dirichlet(1))
  evaluated at the grid points, normalised, plus a floor, renormalised.
  Returns [num, len(grid)] float32: numpy, or a torch tensor evaluated on
  ``device`` when one is given (same parameters, float64 evaluation)."""
  rng = np.random.default_rng(seed)
  if device is not None:
    import torch
    xp_g = torch.tensor(grid, dtype=torch.float64, device=device)
    out = torch.empty((num, len(grid)), dtype=torch.float32, device=device)
    conv = lambda v: torch.as_tensor(v, device=device)
    xp_exp = torch.exp
  else:
    xp_g = grid.astype(np.float64)
    out = np.empty((num, len(grid)), np.float32)
    conv = lambda v: v
    xp_exp = np.exp
  for s in range(0, num, chunk):
    c = min(chunk, num - s)
    k = rng.integers(1, 6, size=c)
    mu = rng.uniform(size=(c, 5, 2))
    sd = rng.uniform(0.03, 0.2, size=(c, 5))
    # Dirichlet(1) over the first k components: normalised exponentials
    e = rng.exponential(size=(c, 5)) * (np.arange(5)[None] < k[:, None])
    pi = e / e.sum(1, keepdims=True)
    mu, var, coef = conv(mu), conv(2 * sd * sd), conv(pi / (2 * np.pi * sd * sd))
    d2 = ((xp_g[None, :, None, :] - mu[:, None]) ** 2).sum(-1)          # [c, P, 5]
    dens = (coef[:, None] * xp_exp(-d2 / var[:, None])).sum(-1)
    w = dens / dens.sum(1, keepdims=True) + floor
    out[s:s + c] = w / w.sum(1, keepdims=True)
  return out


def gmm8_pair(n, m, d=128, seed=0):
  """Two independent 8-component Gaussian mixtures in R^d (means N(0, I),
  per-component std U[0.2, 1], equal component probabilities), uniform
  weights: the epsilon-annealing workload's clouds."""
  rng = np.random.default_rng(seed)

  def cloud(size):
    means = rng.standard_normal((8, d))
    std = rng.uniform(0.2, 1.0, size=8)
    comp = rng.integers(0, 8, size=size)
    return (means[comp] + std[comp, None] * rng.standard_normal((size, d))).astype(np.float32)

  x, y = cloud(n), cloud(m)
  return x, y, np.full(n, 1.0 / n, np.float32), np.full(m, 1.0 / m, np.float32)
