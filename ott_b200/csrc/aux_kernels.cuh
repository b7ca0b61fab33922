// Non-persistent kernels around the solve: point preparation, potential
// initialisation, result finalisation and cost statistics.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "driver.cuh"

namespace ottb {

// Transposed, zero-padded copies xt[DP][n_pad], yt[DP][m_pad] and scaled
// squared norms (FP64 sums rounded once). blockIdx.y = problem,
// blockIdx.z = 0 for x, 1 for y.
struct PrepArgs {
  const float* const* src;  // [2 * P]: x_p, y_p (user pointers)
  ProbDev* probs;
  int d;
  int dp;
};

// Common centre of the two clouds: the midpoint of the means of strided
// samples (at most 256 points each) of x and y. C_ij = |x_i - y_j|^2 does
// not change under a common translation, but the terms of the expanded
// form |x|^2 + |y|^2 - 2 <x, y> shrink, and with them the FP32 rounding of
// every exponent. Deterministic: every CTA computes the same value.
__device__ void sample_center(const float* x, int64_t n, const float* y, int64_t m,
                              int d, float* center) {
  // thread t sums coordinate k = t % d over the samples q = t / d,
  // t / d + groups, ... of each side (consecutive threads read consecutive
  // coordinates of one sample row; 16 loads in flight per thread), then
  // thread k adds the groups' sums in a fixed order: the same value on
  // every call. Needs d <= 128 and blockDim.x >= d.
  __shared__ double part[2][256];
  const int t = threadIdx.x;
  const int groups = (blockDim.x < 256 ? blockDim.x : 256) / d;
  const int k = t % d, grp = t / d;
  int64_t ns_side[2];
  for (int side = 0; side < 2; ++side) {
    const float* src = side ? y : x;
    const int64_t cnt = side ? m : n;
    const int64_t ns = cnt < 256 ? cnt : 256;
    const int64_t stride = cnt / ns;
    ns_side[side] = ns;
    if (grp < groups) {
      double s = 0.0;
      for (int64_t q0 = grp; q0 < ns; q0 += 16 * (int64_t)groups) {
        float v[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) {
          const int64_t q = q0 + (int64_t)u * groups;
          v[u] = q < ns ? src[(q * stride) * d + k] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 16; ++u) s += (double)v[u];
      }
      part[side][t] = s;
    }
  }
  __syncthreads();
  if (t < d) {
    double a0 = 0.0, a1 = 0.0;
    for (int gi = 0; gi < groups; ++gi) {
      a0 += part[0][gi * d + t];
      a1 += part[1][gi * d + t];
    }
    center[t] = (float)(0.5 * (a0 / (double)ns_side[0] + a1 / (double)ns_side[1]));
  }
  __syncthreads();
}

// The common centre of problem blockIdx.x's two point sets, into its
// workspace slot (read by the preparation kernels that follow).
__global__ void center_kernel(PrepArgs args) {
  const int p = blockIdx.x;
  sample_center(args.src[2 * p], args.probs[p].n, args.src[2 * p + 1], args.probs[p].m,
                args.d, args.probs[p].center);
}

__global__ void prep_points_kernel(PrepArgs args) {
  __shared__ float center[128];
  const int p = blockIdx.y;
  const int side = blockIdx.z;
  const ProbDev& P = args.probs[p];
  const float* src = args.src[2 * p + side];
  const int64_t cnt = side ? P.m : P.n;
  const int64_t pad = side ? P.m_pad : P.n_pad;
  float* dst = const_cast<float*>(side ? P.yt : P.xt);
  float* nrm = const_cast<float*>(side ? P.ny : P.nx);
  const int d = args.d, dp = args.dp;
  for (int k = threadIdx.x; k < d; k += blockDim.x) center[k] = P.center[k];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < pad;
       i += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    if (i < cnt) {
      const float* row = src + i * d;
      for (int k = 0; k < d; ++k) {
        float v = row[k] - center[k];
        s += (double)v * (double)v;
        dst[(int64_t)k * pad + i] = v;
      }
      for (int k = d; k < dp; ++k) dst[(int64_t)k * pad + i] = 0.f;
    } else {
      for (int k = 0; k < dp; ++k) dst[(int64_t)k * pad + i] = 0.f;
    }
    nrm[i] = (float)((double)P.inv_scale * s);
  }
}

// Initial potentials (initializers.py:70-131 default, or the caller's init),
// written to the output buffers f and gbuf[0]. blockIdx.y = problem.
struct InitArgs {
  const float* const* init;  // [2 * P]: f_init_p, g_init_p (may be null)
  ProbDev* probs;
  int mask;                  // mask caller init with -inf at zero weights
};

__global__ void init_potentials_kernel(InitArgs args) {
  const int p = blockIdx.y;
  const ProbDev& P = args.probs[p];
  const float* fi = args.init[2 * p];
  const float* gi = args.init[2 * p + 1];
  const float wsh = P.ws_t;
  // f over n_pad, then g over both g buffers' m_pad rows (padding rows get
  // the -inf column shift of the tensor-core path)
  const int64_t tot = P.n_pad + 2 * P.m_pad;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < tot;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (i < P.n_pad) {
      float v = -INFINITY;
      if (i < P.n) {
        v = fi ? fi[i] : 0.f;
        if ((!fi || args.mask) && !(P.a[i] > 0.f)) v = -INFINITY;
        P.f[i] = v;
      }
      if (P.extx) write_ext_row((char*)P.extx + i * 16, i < P.n ? (v - P.nx[i]) * wsh : -INFINITY);
    } else {
      const int64_t k = i - P.n_pad;
      const int buf = (int)(k / P.m_pad);
      const int64_t j = k % P.m_pad;
      float v = -INFINITY;
      if (j < P.m && buf == 0) {
        v = gi ? gi[j] : 0.f;
        if ((!gi || args.mask) && !(P.b[j] > 0.f)) v = -INFINITY;
        P.gbuf[0][j] = v;
      }
      if (P.exty && (buf == 0 || j >= P.m))
        write_ext_row((char*)P.exty + k * 16, (j < P.m) ? (v - P.ny[j]) * wsh : -INFINITY);
    }
  }
}

// One CTA per problem: final g copy, reg_ot_cost (sinkhorn.py:224-277,
// balanced branch, FP64 sums), n_iters (:432-434), converged (:1020-1023).
struct FinalArgs {
  ProbDev* probs;
  ProbState* state;
  Sched* sched;
  ottb_result* results;
  ottb_solver_cfg cfg;
};

__device__ __forceinline__ double cta_sum(double v, double* red) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += red[i];
  }
  return r;
}

__global__ void finalize_kernel(FinalArgs args) {
  __shared__ double red[32];
  const int p = blockIdx.x;
  const ProbDev& P = args.probs[p];
  const ProbState& S = args.state[p];
  const int par = S.final_parity;
  const float* g = P.gbuf[par];
  const double eps = (double)P.eps_target;
  double da = 0.0, db = 0.0, sa = 0.0, sb = 0.0;
  for (int64_t i = threadIdx.x; i < P.n; i += blockDim.x) {
    const double a = (double)P.a[i];
    // a symmetric problem ends with f = g
    const float fv = P.symmetric ? g[i] : P.f[i];
    if (P.symmetric) P.f[i] = fv;
    sa += a;
    if (a > 0.0) da += a * ((double)fv - eps * log(a));
  }
  for (int64_t j = threadIdx.x; j < P.m; j += blockDim.x) {
    const double b = (double)P.b[j];
    const float gv = g[j];
    sb += b;
    if (b > 0.0) db += b * ((double)gv - eps * log(b));
    if (par == 1) P.gbuf[0][j] = gv;
  }
  da = cta_sum(da, red);
  db = cta_sum(db, red);
  sa = cta_sum(sa, red);
  sb = cta_sum(sb, red);
  __syncthreads();
  if (threadIdx.x == 0) {
    int valid = 0, any_nan = 0;
    for (int k = 0; k < P.outer; ++k) {
      const float e = P.errors[k];
      if (e != -1.f) ++valid;
      if (isnan(e)) any_nan = 1;
    }
    const float last = P.outer > 0 ? P.errors[P.outer - 1] : -1.f;
    ottb_result r;
    r.reg_ot_cost = da + db + eps * (sa * sb - S.msum);
    r.marginal_sum = S.msum;
    r.n_iters = valid * args.cfg.inner_iterations;
    r.converged = (!any_nan && last < args.cfg.threshold) ? 1 : 0;
    r.status = args.sched->status;
    r.reserved = 0;
    args.results[P.uid] = r;
  }
}

// Errors start at -1 (sinkhorn.py:964-972).
__global__ void fill_errors_kernel(ProbDev* probs) {
  const ProbDev& P = probs[blockIdx.y];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < P.outer;
       k += gridDim.x * blockDim.x)
    P.errors[k] = -1.f;
}

// FP64 moments for the cost statistics. Each CTA writes a partial vector
// [cnt, sum n, sum n^2, sum x (d), sum n x (d), sum x x^T (d*d, when
// second != 0)] for one point set, n = |x|^2; the reductions add partials in
// a fixed order, so the statistics are deterministic.
__host__ __device__ inline int moments_len(int d, int second) {
  return 3 + 2 * d + (second ? d * d : 0);
}

__global__ void moments_kernel(const float* pts, int64_t cnt, int d, int second, double* part) {
  extern __shared__ double sh[];
  const int K = moments_len(d, second);
  double* acc = sh;                                // [K] per-CTA accumulators
  float* tile = reinterpret_cast<float*>(sh + K);  // [64][d]
  double* nrm = sh + K + 32 * d;                   // [64] squared norms (tile is 64*d floats)
  for (int k = threadIdx.x; k < K; k += blockDim.x) acc[k] = 0.0;
  __syncthreads();
  const int64_t per = (cnt + gridDim.x - 1) / gridDim.x;
  const int64_t beg = (int64_t)blockIdx.x * per;
  const int64_t end = min(cnt, beg + per);
  for (int64_t c0 = beg; c0 < end; c0 += 64) {
    const int rows = (int)min((int64_t)64, end - c0);
    for (int idx = threadIdx.x; idx < rows * d; idx += blockDim.x)
      tile[idx] = pts[c0 * d + idx];
    __syncthreads();
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
      double s = 0.0;
      for (int k = 0; k < d; ++k) s += (double)tile[r * d + k] * tile[r * d + k];
      nrm[r] = s;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < K; e += blockDim.x) {
      double s = 0.0;
      if (e == 0) {
        s = rows;
      } else if (e <= 2) {
        for (int r = 0; r < rows; ++r) s += (e == 1) ? nrm[r] : nrm[r] * nrm[r];
      } else if (e < 3 + d) {
        const int k = e - 3;
        for (int r = 0; r < rows; ++r) s += tile[r * d + k];
      } else if (e < 3 + 2 * d) {
        const int k = e - 3 - d;
        for (int r = 0; r < rows; ++r) s += nrm[r] * tile[r * d + k];
      } else {
        const int q = e - 3 - 2 * d;
        const int k1 = q / d, k2 = q % d;
        for (int r = 0; r < rows; ++r) s += (double)tile[r * d + k1] * tile[r * d + k2];
      }
      acc[e] += s;
    }
    __syncthreads();
  }
  for (int k = threadIdx.x; k < K; k += blockDim.x) part[(int64_t)blockIdx.x * K + k] = acc[k];
}

// mom[k] = sum over the nblk partials of entry k, one thread per entry, for
// the concatenated x and y moment vectors.
__global__ void moments_reduce_kernel(const double* px, const double* py, int nblk, int K,
                                      double* mom) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 2 * K) return;
  const double* src = k < K ? px : py;
  const int e = k < K ? k : k - K;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += src[(int64_t)b * K + e];
  mom[k] = s;
}

// out[0] = mean(C), out[1] = mean(C^2) (when second != 0) from the moments.
__global__ void cost_stats_final_kernel(const double* mom, int d, int second, double inv,
                                        double* out) {
  const int K = moments_len(d, second);
  const double* X = mom;
  const double* Y = mom + K;
  const double n = X[0], m = Y[0];
  const double mnx = X[1] / n, mny = Y[1] / m;
  double xy = 0.0, nxy = 0.0, xny = 0.0;
  for (int k = 0; k < d; ++k) {
    xy += (X[3 + k] / n) * (Y[3 + k] / m);
    nxy += (X[3 + d + k] / n) * (Y[3 + k] / m);
    xny += (X[3 + k] / n) * (Y[3 + d + k] / m);
  }
  out[0] = inv * (mnx + mny - 2.0 * xy);
  if (second) {
    double tr = 0.0;
    for (int k1 = 0; k1 < d; ++k1)
      for (int k2 = 0; k2 < d; ++k2)
        tr += X[3 + 2 * d + k1 * d + k2] * Y[3 + 2 * d + k2 * d + k1];
    tr /= (n * m);
    const double mnx2 = X[2] / n, mny2 = Y[2] / m;
    out[1] = inv * inv *
             (mnx2 + mny2 + 2.0 * mnx * mny + 4.0 * tr - 4.0 * nxy - 4.0 * xny);
  } else {
    out[1] = NAN;
  }
}

}  // namespace ottb

namespace ottb {

// Tensor-core layout: centred points split into bf16 pairs, hi rows then lo
// rows, [2][pad][dk] (zero padded in both dimensions), and scaled squared
// norms of the centred FP32 points. The x side is multiplied by the exponent
// scale s = 2 inv log2(e) / eps_target before the split, so the products
// <x', y> come out in log2 units. blockIdx.y = problem, blockIdx.z = side.
__global__ void prep_points_tc_kernel(PrepArgs args) {
  __shared__ float center[128];
  const int p = blockIdx.y;
  const int side = blockIdx.z;
  const ProbDev& P = args.probs[p];
  const float* src = args.src[2 * p + side];
  const int64_t cnt = side ? P.m : P.n;
  const int64_t pad = side ? P.m_pad : P.n_pad;
  __nv_bfloat16* dst = (__nv_bfloat16*)(side ? P.yh : P.xh);
  float* nrm = const_cast<float*>(side ? P.ny : P.nx);
  const int d = args.d, dk = args.dp;
  const float scale = side ? 1.0f : 2.0f * P.inv_scale * P.ws_t;
  for (int k = threadIdx.x; k < d; k += blockDim.x) center[k] = P.center[k];
  __syncthreads();
  // one warp per row: lanes over the coordinates, so the bf16 stores of a
  // warp are contiguous; the squared norm is a fixed shuffle tree
  const int lane = threadIdx.x & 31;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < pad;
       i += warps) {
    __nv_bfloat16* hi = dst + i * dk;
    __nv_bfloat16* lo = dst + (pad + i) * dk;
    const float* row = src + i * d;
    double s = 0.0;
    for (int k = lane; k < dk; k += 32) {
      const float v = (i < cnt && k < d) ? row[k] - center[k] : 0.f;
      s += (double)v * (double)v;
      const float vs = v * scale;
      const __nv_bfloat16 h = __float2bfloat16_rn(vs);
      hi[k] = h;
      lo[k] = __float2bfloat16_rn(vs - __bfloat162float(h));
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) nrm[i] = (float)((double)P.inv_scale * s);
  }
}

}  // namespace ottb
