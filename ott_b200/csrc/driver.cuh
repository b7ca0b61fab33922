// Persistent Sinkhorn driver: the whole fixed-point loop of every problem of
// a call runs inside one cooperative launch.
//
// Mirrors ott/math/fixed_point_loop.py:23-93 (blocks of inner_iterations,
// stop test between blocks, scan mode when min == max) and
// ott/solvers/linear/sinkhorn.py:879-953 (g-update then f-update, the error
// of a block's last iteration, converged / diverged tests). The marginal
// error of the state after a block is read off the next g-sweep, which
// computes the same column log-sum-exp: b_hat_j = 2^(lse2_j + (g_j -
// inv |y_j|^2) log2(e) / eps). That sweep's new g goes to a second buffer
// and is dropped if the problem stops, so the returned (f, g) is exactly
// the state the reference returns.
#pragma once

#include "common.cuh"

namespace ottb {

struct KernelArgs {
  ProbDev* probs;
  ProbState* state;
  Sched* sched;
  Globals* gl;
  int* active_ids;   // [P] problems in schedule order
  int* prefix;       // [2][P + 1] unit prefix sums (g-sweep, f-sweep)
  int* eval_ids;     // [P]
  int* eval_prefix;  // [P + 1]
  int num_problems;
  unsigned expected_arrivals;
  uint64_t timeout_ns;
  ottb_solver_cfg cfg;
};

struct SweepParams {
  int kind;      // kSweepG / kSweepF
  float mult;    // epsilon multiplier of this sweep
  int eval;      // compute the column marginal (g-sweeps only)
  int write;     // write the new potential
  int final_eval;  // use the eval list and each problem's final parity
  int parity;    // g parity of active problems
  // tensor-core path: the rows' shifts may be bounded from their last sweep
  // (set by persistent_main: multiplier 1 now and then, not the final
  // evaluation); dkey slot this sweep reads, and slot of the other kind's
  // next sweep its potential changes go to
  int fast;
  int rslot;
  int wslot;
};

__device__ __forceinline__ float eps_mult(const ottb_solver_cfg& c, int it) {
  // epsilon_scheduler.py:47-60: max(init * decay^it, 1)
  float mlt = c.eps_init * powf(c.eps_decay, (float)it);
  return fmaxf(mlt, 1.0f);
}

// Exponent scale of a sweep, log2(e) / eps in FP32; the single source of
// this value for the sweep engines and the potential update.
__device__ __forceinline__ float sweep_wscale(const ProbDev& P, float mult) {
  return (float)(kLog2eD / ((double)P.eps_target * (double)mult));
}

__device__ __forceinline__ SweepOperands make_operands(const ProbDev& P, int kind,
                                                       const float* gcur) {
  SweepOperands op;
  if (kind == kSweepG) {
    op.At = P.yt; op.a_pad = P.m_pad; op.rows = P.m;
    op.Bt = P.xt; op.b_pad = P.n_pad; op.cols = P.n;
    op.potB = P.symmetric ? gcur : P.f; op.nb = P.nx;
  } else {
    op.At = P.xt; op.a_pad = P.n_pad; op.rows = P.n;
    op.Bt = P.yt; op.b_pad = P.m_pad; op.cols = P.m;
    op.potB = gcur; op.nb = P.ny;
  }
  return op;
}

// The thread group that runs the per-row-block steps of the CUDA-core
// engine (merges, potential updates): the whole CTA. tid() is the thread's
// index in the group; the rows of a row block are handled by tids
// 0..kBM-1 (whole warps).
struct CtaGroup {
  static __device__ __forceinline__ int tid() { return threadIdx.x; }
  static __device__ __forceinline__ int size() { return blockDim.x; }
  static __device__ __forceinline__ void sync() { __syncthreads(); }
};

// Group-wide sum of one double per thread (tids 0..kBM-1 contribute),
// fixed-order tree so the result is deterministic; tid 0 gets the sum.
template <class G>
__device__ __forceinline__ double group_sum_128(double v, double* red) {
  const int t = G::tid();
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if (t >= 0 && t < kBM && (t & 31) == 0) red[t >> 5] = v;
  G::sync();
  double r = 0.0;
  if (t == 0) r = (red[0] + red[1]) + (red[2] + red[3]);
  G::sync();
  return r;
}

__device__ __forceinline__ double block_sum_128(double v, double* red) {
  return group_sum_128<CtaGroup>(v, red);
}

// Potential update and (optionally) marginal of row r of a row block, from
// its base-2 LSE state (mv, lv). geometry.py:376-398 / :326-349. Folds the
// row's change of column shift into [dmin, dmax] and returns its error and
// marginal terms in err_t, msum_t.
__device__ __forceinline__ void finalize_row(const ProbDev& P, const SweepParams& sp, int parity,
                                             int64_t r, float mv, float lv, float ws, double eps,
                                             int norm_error, float& dmax, float& dmin,
                                             double& err_t, double& msum_t) {
  const bool isG = sp.kind == kSweepG;
  const float* marg = isG ? P.b : P.a;
  const float* na = isG ? P.ny : P.nx;
  const float* oldp = isG ? P.gbuf[parity] : P.f;
  float* outp = isG ? P.gbuf[parity ^ 1] : P.f;
  double lse2 = (lv > 0.f) ? (double)mv + log2((double)lv)
                           : (lv == 0.f ? -INFINITY : (double)NAN);
  const double nrm = (double)na[r];
  const double app = eps * kLn2 * lse2 - nrm;
  const double old = (double)__ldcg(oldp + r);
  const double mg = (double)marg[r];
  const double logm = log(mg);
  const bool keep = isfinite(old) && isfinite(app);
  double newp = eps * logm - (keep ? app : 0.0);
  // symmetric problem: Momentum(value=0.5) on the parallel update,
  // (1 - w) * where(isfinite(old), old, 0) + w * new (acceleration.py:168-170)
  if (P.symmetric) newp = 0.5 * (isfinite(old) ? old : 0.0) + 0.5 * newp;
  if (P.lprev) P.lprev[(isG ? P.n_pad : 0) + r] = (float)lse2;
  if (sp.write) {
    const float nf = (float)newp;
    outp[r] = nf;
    // tensor-core path: the updated point's column shift for the next sweep
    void* ext = isG ? P.exty : P.extx;
    if (ext) {
      const int64_t row = isG ? (int64_t)(parity ^ 1) * P.m_pad + r : r;
      write_ext_row((char*)ext + row * 16, (nf - na[r]) * P.ws_t);
    }
    if (isfinite(nf) && isfinite(old)) {
      const float dl = (nf - (float)old) * P.ws_t;
      dmax = fmaxf(dmax, dl);
      dmin = fminf(dmin, dl);
    } else if (isfinite(nf) != isfinite(old)) {
      // a potential became or stopped being -inf: no bound
      dmax = INFINITY;
      dmin = -INFINITY;
    }
  }
  err_t = 0.0;
  msum_t = 0.0;
  if (sp.eval) {
    double bh = 0.0;
    if (!(old == -INFINITY)) bh = exp2(lse2 + (old - nrm) * (double)ws);
    double dv = fabs(bh - mg);
    err_t = (norm_error == 1) ? dv : pow(dv, (double)norm_error);
    msum_t = bh;
    if (sp.final_eval && P.marg_out) P.marg_out[r] = (float)bh;
    if (sp.final_eval && P.lse_out) P.lse_out[r] = (float)app;  // eps LSE_i - |y_j|^2 term
  }
}

// The sweep scaled every exponent by the FP32 value ws = log2(e) / eps;
// the update uses the epsilon that ws stands for, eps = log2(e) / ws, in
// both of its terms. A mismatch between the two would bias the f- and
// g-updates differently, and such a bias accumulates along the neutral
// direction (f + c, g - c) of the iteration.
__device__ __forceinline__ double update_epsilon(float ws) { return kLog2eD / (double)ws; }

// One atomic each for a row block's extreme changes of column shift, into
// the other kind's slot (the bound of that kind's next sweep).
__device__ __forceinline__ void publish_shift_change(const ProbDev& P, const SweepParams& sp,
                                                     float mx, float mn) {
  int* slot = P.dkey + (((sp.kind == kSweepG ? kSweepF : kSweepG) * 2 + sp.wslot) * 2);
  if (mx > -INFINITY) atomicMax(slot, fkey(mx));
  if (mn < INFINITY) atomicMin(slot + 1, fkey(mn));
}

// Potential update and (optionally) marginal for the rows of one row block,
// one row per thread of group G (tids 0..kBM-1).
template <class G>
__device__ void finalize_rows_g(const ProbDev& P, const SweepParams& sp, int parity,
                                int rb, const float* rm, const float* rl,
                                int norm_error, double* red) {
  const int t = G::tid();
  const int64_t R = sp.kind == kSweepG ? P.m : P.n;
  const float ws = sweep_wscale(P, sp.mult);
  const double eps = update_epsilon(ws);
  double err_t = 0.0, msum_t = 0.0;
  float dmax = -INFINITY, dmin = INFINITY;
  const int64_t r = (int64_t)rb * kBM + t;
  if (t >= 0 && t < kBM && r < R)
    finalize_row(P, sp, parity, r, rm[t], rl[t], ws, eps, norm_error, dmax, dmin, err_t, msum_t);
  if (sp.write && P.dkey && !P.symmetric) {
    for (int off = 16; off > 0; off >>= 1) {
      dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, off));
      dmin = fminf(dmin, __shfl_xor_sync(0xffffffffu, dmin, off));
    }
    float* fr = reinterpret_cast<float*>(red);
    if (t >= 0 && t < kBM && (t & 31) == 0) {
      fr[t >> 5] = dmax;
      fr[4 + (t >> 5)] = dmin;
    }
    G::sync();
    if (t == 0)
      publish_shift_change(P, sp, fmaxf(fmaxf(fr[0], fr[1]), fmaxf(fr[2], fr[3])),
                           fminf(fminf(fr[4], fr[5]), fminf(fr[6], fr[7])));
    G::sync();
  }
  if (sp.eval) {
    double e = group_sum_128<G>(err_t, red);
    double s = group_sum_128<G>(msum_t, red);
    if (t == 0) {
      P.err_part[rb] = e;
      P.msum_part[rb] = s;
    }
  }
}

// The same for one warp: lane l holds rows l, l + 32, l + 64, l + 96 of the
// row block (mv[k], lv[k] for row l + 32 k). Reductions by shuffles only.
__device__ __forceinline__ void finalize_rows_warp(const ProbDev& P, const SweepParams& sp,
                                                   int parity, int rb, const float (&mv)[4],
                                                   const float (&lv)[4], int norm_error) {
  const int lane = threadIdx.x & 31;
  const int64_t R = sp.kind == kSweepG ? P.m : P.n;
  const float ws = sweep_wscale(P, sp.mult);
  const double eps = update_epsilon(ws);
  double err = 0.0, msum = 0.0;
  float dmax = -INFINITY, dmin = INFINITY;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int64_t r = (int64_t)rb * kBM + lane + 32 * k;
    if (r < R) {
      double e, m;
      finalize_row(P, sp, parity, r, mv[k], lv[k], ws, eps, norm_error, dmax, dmin, e, m);
      err += e;
      msum += m;
    }
  }
  if (sp.write && P.dkey && !P.symmetric) {
    for (int off = 16; off > 0; off >>= 1) {
      dmax = fmaxf(dmax, __shfl_xor_sync(0xffffffffu, dmax, off));
      dmin = fminf(dmin, __shfl_xor_sync(0xffffffffu, dmin, off));
    }
    if (lane == 0) publish_shift_change(P, sp, dmax, dmin);
  }
  if (sp.eval) {
    for (int off = 16; off > 0; off >>= 1) {
      err += __shfl_xor_sync(0xffffffffu, err, off);
      msum += __shfl_xor_sync(0xffffffffu, msum, off);
    }
    if (lane == 0) {
      P.err_part[rb] = err;
      P.msum_part[rb] = msum;
    }
  }
}

__device__ __forceinline__ void finalize_rows(const ProbDev& P, const SweepParams& sp,
                                              int parity, int rb, const float* rm,
                                              const float* rl, int norm_error, double* red) {
  finalize_rows_g<CtaGroup>(P, sp, parity, rb, rm, rl, norm_error, red);
}

}  // namespace ottb
