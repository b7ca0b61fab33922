/*
 * CPU oracle, C port (TEST INFRASTRUCTURE ONLY): the log-domain Sinkhorn of
 * ott-jax on a squared-Euclidean point cloud, restated in plain C with
 * OpenMP, in the float type of the reference's default (FP32) path.
 *
 * Used only by tests (as a second restatement checked against the NumPy
 * oracle) and by bench.py's CPU-baseline leg and `--impl reference` arm.
 * The ott_b200 package never links or loads it. Compiled with -DOTTB_TILED,
 * the kernel application is the tiled, vectorised one of lse_tiled.h (the
 * timed baseline); the loop around it is the same.
 *
 * Follows, in order:
 *   solvers/linear/sinkhorn.py:803-857  lse_step (g-update, then f-update)
 *   geometry/geometry.py:376-398       update_potential
 *   geometry/pointcloud.py:74-103      apply_lse_kernel, online (rows are
 *                                      recomputed block by block; the n x m
 *                                      cost is never stored)
 *   geometry/geometry.py:423-442       _center / _softmax: (f + g - C) / eps,
 *                                      max-shifted log-sum-exp
 *   solvers/linear/sinkhorn.py:191-221 marginal_error (p-norm)
 *   solvers/linear/sinkhorn.py:224-277 compute_kl_reg_cost (balanced)
 *   math/fixed_point_loop.py:23-93     blocks of inner_iterations, stop test
 *   solvers/linear/sinkhorn.py:914-953 error cadence, converged / diverged
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef float real;

/* C_ij = inv * (|x_i|^2 + |y_j|^2 + (-2 <x_i, y_j>)), costs.py:558-561. */
static inline real cost_ij(const real* xi, const real* yj, real nxi, real nyj, int d,
                           real inv) {
  real dot = 0;
  for (int k = 0; k < d; ++k) dot += xi[k] * yj[k];
  return inv * ((nxi + nyj) + (real)(-2.0) * dot);
}

#ifdef OTTB_TILED
#include "lse_tiled.h"

/* The tiled, vectorised row log-sum-exp of lse_tiled.h, with the roles of
 * the two point sets swapped for axis 0. */
static void apply_lse(const real* x, const real* y, const real* nx, const real* ny,
                      int64_t n, int64_t m, int d, real inv, const real* f,
                      const real* g, real eps, int axis, real* out) {
  if (axis == 0)
    lt_row_lse(y, x, ny, nx, m, n, d, inv, g, f, eps, out);
  else
    lt_row_lse(x, y, nx, ny, n, m, d, inv, f, g, eps, out);
}
#else
/* out[j] = eps * lse_i((f_i + g_j - C_ij) / eps) - finite(g_j)  (axis 0) or
 * out[i] = eps * lse_j((f_i + g_j - C_ij) / eps) - finite(f_i)  (axis 1). */
static void apply_lse(const real* x, const real* y, const real* nx, const real* ny,
                      int64_t n, int64_t m, int d, real inv, const real* f,
                      const real* g, real eps, int axis, real* out) {
  const int64_t R = axis == 0 ? m : n;
  const int64_t K = axis == 0 ? n : m;
#pragma omp parallel
  {
    real* buf = (real*)malloc(sizeof(real) * (size_t)K);
#pragma omp for schedule(static)
    for (int64_t r = 0; r < R; ++r) {
      real mx = -INFINITY;
      for (int64_t k = 0; k < K; ++k) {
        const int64_t i = axis == 0 ? k : r;
        const int64_t j = axis == 0 ? r : k;
        const real c = cost_ij(x + i * d, y + j * d, nx[i], ny[j], d, inv);
        const real v = ((f[i] + g[j]) - c) / eps;
        buf[k] = v;
        if (v > mx) mx = v;
      }
      if (!isfinite(mx)) mx = 0; /* shift replaced by 0 when not finite */
      real s = 0;
      for (int64_t k = 0; k < K; ++k) s += expf(buf[k] - mx);
      const real lse = logf(fabsf(s)) + mx;
      const real remove = axis == 0 ? g[r] : f[r];
      out[r] = eps * lse - (isfinite(remove) ? remove : (real)0);
    }
    free(buf);
  }
}
#endif

static void update_potential(const real* x, const real* y, const real* nx, const real* ny,
                             int64_t n, int64_t m, int d, real inv, const real* f,
                             const real* g, const real* logm, real eps, int axis,
                             real* out, real* tmp) {
  const int64_t R = axis == 0 ? m : n;
  apply_lse(x, y, nx, ny, n, m, d, inv, f, g, eps, axis, tmp);
  for (int64_t r = 0; r < R; ++r)
    out[r] = eps * logm[r] - (isfinite(tmp[r]) ? tmp[r] : (real)0);
}

/* Column marginal of (f, g): exp((apply_lse(axis 0) + g) / eps). */
static void col_marginal(const real* x, const real* y, const real* nx, const real* ny,
                         int64_t n, int64_t m, int d, real inv, const real* f,
                         const real* g, real eps, real* out) {
  apply_lse(x, y, nx, ny, n, m, d, inv, f, g, eps, 0, out);
  for (int64_t j = 0; j < m; ++j) out[j] = expf((out[j] + g[j]) / eps);
}

int oracle_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Full solve. f_init/g_init may be NULL (default init: 0, -inf at zero
 * weight). errors must hold ceil(max_it / inner) floats. Returns 0. */
int oracle_sinkhorn(const float* x, const float* y, const float* a, const float* b,
                    int64_t n, int64_t m, int d, float eps, float inv, float eps_init,
                    float eps_decay, float threshold, int norm_error, int inner,
                    int min_it, int max_it, const float* f_init, const float* g_init,
                    float* f, float* g, float* errors, double* reg_ot_cost,
                    int* n_iters, int* converged, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  real* nx = (real*)malloc(sizeof(real) * (size_t)n);
  real* ny = (real*)malloc(sizeof(real) * (size_t)m);
  real* loga = (real*)malloc(sizeof(real) * (size_t)n);
  real* logb = (real*)malloc(sizeof(real) * (size_t)m);
  real* tmp = (real*)malloc(sizeof(real) * (size_t)(n > m ? n : m));
  for (int64_t i = 0; i < n; ++i) {
    real s = 0;
    for (int k = 0; k < d; ++k) s += x[i * d + k] * x[i * d + k];
    nx[i] = s;
    loga[i] = logf(a[i]);
    f[i] = f_init ? f_init[i] : (a[i] > 0 ? 0.0f : -INFINITY);
  }
  for (int64_t j = 0; j < m; ++j) {
    real s = 0;
    for (int k = 0; k < d; ++k) s += y[j * d + k] * y[j * d + k];
    ny[j] = s;
    logb[j] = logf(b[j]);
    g[j] = g_init ? g_init[j] : (b[j] > 0 ? 0.0f : -INFINITY);
  }
  const int outer = (max_it + inner - 1) / inner;
  for (int k = 0; k < outer; ++k) errors[k] = -1.0f;
  const int force_scan = (min_it == max_it);
  const int scan_end = force_scan ? (max_it / inner) * inner : max_it;
  int it = 0;
  for (;;) {
    if (it > 0 && it % inner == 0) {
      const float err = errors[it / inner - 1];
      int cont;
      if (force_scan) {
        cont = it < scan_end;
      } else {
        const int conv = err < threshold;
        const int div = !isfinite(err);
        cont = it < max_it && (it < min_it || (!div && !conv));
      }
      if (!cont) break;
    } else if (it == 0 && scan_end == 0) {
      break;
    }
    for (int k = 0; k < inner; ++k, ++it) {
      const real mlt = fmaxf(eps_init * powf(eps_decay, (real)it), 1.0f);
      const real e = mlt * eps;
      update_potential(x, y, nx, ny, n, m, d, inv, f, g, logb, e, 0, g, tmp);
      update_potential(x, y, nx, ny, n, m, d, inv, f, g, loga, e, 1, f, tmp);
      float err = INFINITY;
      if (it == max_it - 1 || (k == inner - 1 && it >= min_it)) {
        col_marginal(x, y, nx, ny, n, m, d, inv, f, g, eps, tmp);
        double s = 0;
        for (int64_t j = 0; j < m; ++j) {
          const double dv = fabs((double)tmp[j] - (double)b[j]);
          s += norm_error == 1 ? dv : pow(dv, norm_error);
        }
        err = (float)(norm_error == 1 ? s : pow(s, 1.0 / norm_error));
      }
      errors[it / inner] = err;
    }
  }
  int valid = 0, any_nan = 0;
  for (int k = 0; k < outer; ++k) {
    if (errors[k] != -1.0f) ++valid;
    if (isnan(errors[k])) any_nan = 1;
  }
  *n_iters = valid * inner;
  *converged = (!any_nan && (outer > 0 ? errors[outer - 1] : -1.0f) < threshold) ? 1 : 0;
  /* compute_kl_reg_cost, balanced branch */
  col_marginal(x, y, nx, ny, n, m, d, inv, f, g, eps, tmp);
  double div_a = 0, div_b = 0, sa = 0, sb = 0, tot = 0;
  for (int64_t i = 0; i < n; ++i) {
    sa += a[i];
    if (a[i] > 0) div_a += (double)a[i] * ((double)f[i] - (double)eps * log((double)a[i]));
  }
  for (int64_t j = 0; j < m; ++j) {
    sb += b[j];
    tot += tmp[j];
    if (b[j] > 0) div_b += (double)b[j] * ((double)g[j] - (double)eps * log((double)b[j]));
  }
  *reg_ot_cost = div_a + div_b + (double)eps * (sa * sb - tot);
  free(nx); free(ny); free(loga); free(logb); free(tmp);
  return 0;
}
