// One MINRES step (Paige and Saunders, SIAM J. Numer. Anal. 12, 1975) after
// the operator product, on the device: both Lanczos recurrences, the Givens
// rotation of the tridiagonal system, the stop test and the updates of the
// search direction, the iterate and the next Lanczos vector, in one launch.
// The solver's scalars live in a small device array, so the host issues the
// products of successive steps back to back and reads only the previous
// step's stop flag while the current step runs; with the step number kept
// on the device too (ottb_minres_step_next), a block of steps and their
// products is one fixed sequence of launches that a CUDA graph replays.
// Used by the implicit backward of the Sinkhorn potentials, whose
// linear system (implicit_differentiation.py:156-233) is solved here in a
// symmetric form.
//
// One CTA of 1024 threads: the vectors have the length of the smaller point
// set, and a step's 15 vector passes cost microseconds next to the two plan
// products of the same step. The two inner products are reduced in a fixed
// order (a strided per-thread sum, then a shuffle tree), so a step is
// deterministic.
#include <cuda_runtime.h>

#include <math.h>

#include "../../include/ott_b200.h"

namespace ottb {
namespace {

constexpr int kThreads = 1024;
constexpr int kWarps = kThreads / 32;

// state[] slots (float64)
enum : int {
  kBeta = 0,    // |r2|, the current Lanczos normaliser
  kOldBeta,     // the previous one
  kDbar,        // rotated entries of the tridiagonal column
  kEpsln,
  kPhibar,      // the residual norm estimate
  kCs,          // the last rotation
  kSn,
  kBeta1,       // |rhs|
  kRtol,
  kActive,      // 1 while iterating, 0 after the stop test fired
  kSteps,       // steps taken
};

__device__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (wid == 0) {
    double t = red[lane];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) red[kWarps] = t;
  }
  __syncthreads();
  const double r = red[kWarps];
  __syncthreads();  // red is reused by the next reduction
  return r;
}

// y holds op(v) on entry and the new Lanczos residual r2' on exit. w_prev
// holds the direction before w on entry and the new direction on exit.
// step == 0: the step number is state[steps] + 1, and a step past
// hist_len - 1 clears the active flag instead of running.
__global__ void __launch_bounds__(kThreads)
minres_step_kernel(double* __restrict__ st, int step, int window,
                   const double* __restrict__ v, double* __restrict__ y,
                   const double* __restrict__ r1, const double* __restrict__ r2,
                   const double* __restrict__ w, double* __restrict__ w_prev,
                   double* __restrict__ x, double* __restrict__ v_next,
                   double* __restrict__ hist, int64_t hist_len, int64_t s) {
  __shared__ double red[kWarps + 1];
  __shared__ double sc[5];
  // every thread reads the flag and the step count before thread 0 can
  // write them (it writes only after the reductions' barriers)
  if (st[kActive] == 0.0) return;
  if (step == 0) {
    const int64_t next = (int64_t)st[kSteps] + 1;
    if (next >= hist_len) {
      if (threadIdx.x == 0) st[kActive] = 0.0;  // the step cap: every thread returns here
      return;
    }
    step = (int)next;
  }
  const double beta = st[kBeta];
  // y = op(v) - (beta / oldb) r1 (not on the first step), alfa = <v, y>
  const double c1 = step >= 2 ? beta / st[kOldBeta] : 0.0;
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < s; i += kThreads) {
    double yi = y[i];
    if (step >= 2) yi -= c1 * r1[i];
    y[i] = yi;
    acc += v[i] * yi;
  }
  const double alfa = block_sum(acc, red);
  // y -= (alfa / beta) r2, beta' = |y|
  const double c2 = alfa / beta;
  acc = 0.0;
  for (int64_t i = threadIdx.x; i < s; i += kThreads) {
    const double yi = y[i] - c2 * r2[i];
    y[i] = yi;
    acc += yi * yi;
  }
  const double beta_n = sqrt(block_sum(acc, red));
  if (threadIdx.x == 0) {
    const double dbar = st[kDbar], epsln = st[kEpsln], cs = st[kCs], sn = st[kSn];
    const double phibar = st[kPhibar], beta1 = st[kBeta1];
    // the previous rotation applied to the new column
    const double delta = cs * dbar + sn * alfa;
    const double gbar = sn * dbar - cs * alfa;
    // the next rotation (gamma floored at the float64 epsilon)
    const double gamma = fmax(sqrt(gbar * gbar + beta_n * beta_n), 2.220446049250313e-16);
    const double cs_n = gbar / gamma, sn_n = beta_n / gamma;
    const double phibar_n = sn_n * phibar;
    sc[0] = epsln;
    sc[1] = delta;
    sc[2] = gamma;
    sc[3] = cs_n * phibar;
    sc[4] = beta_n > 0.0 ? beta_n : 1.0;
    st[kEpsln] = sn * beta_n;
    st[kDbar] = -cs * beta_n;
    st[kCs] = cs_n;
    st[kSn] = sn_n;
    st[kPhibar] = phibar_n;
    st[kOldBeta] = beta;
    st[kBeta] = beta_n;
    st[kSteps] = (double)step;
    hist[step] = phibar_n;
    // converged, the Krylov space closed, or `window` steps lowered the
    // estimate by less than 1 %
    bool stop = phibar_n <= st[kRtol] * beta1 || beta_n <= 1e-14 * beta1;
    if (step >= window && phibar_n > 0.99 * hist[step - window]) stop = true;
    if (stop) st[kActive] = 0.0;
  }
  __syncthreads();
  const double oldeps = sc[0], delta = sc[1], gamma = sc[2], phi = sc[3], bdiv = sc[4];
  // w' = (v - oldeps w_prev - delta w) / gamma, x += phi w', v' = y / beta'
  for (int64_t i = threadIdx.x; i < s; i += kThreads) {
    const double wn = (v[i] - oldeps * w_prev[i] - delta * w[i]) / gamma;
    w_prev[i] = wn;
    x[i] += phi * wn;
    v_next[i] = y[i] / bdiv;
  }
}

}  // namespace
}  // namespace ottb

extern "C" {

int32_t ottb_minres_step(double* state, int32_t step, int32_t window, const double* v,
                         double* y, const double* r1, const double* r2, const double* w,
                         double* w_prev, double* x, double* v_next, double* history,
                         int64_t history_len, int64_t s, void* stream) {
  if (!state || !v || !y || !r1 || !r2 || !w || !w_prev || !x || !v_next || !history)
    return OTTB_ERR_INVALID;
  if (s < 1 || step < 1 || window < 1 || step >= history_len) return OTTB_ERR_INVALID;
  ottb::minres_step_kernel<<<1, ottb::kThreads, 0, (cudaStream_t)stream>>>(
      state, step, window, v, y, r1, r2, w, w_prev, x, v_next, history, history_len, s);
  return cudaGetLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}

int32_t ottb_minres_step_next(double* state, int32_t window, const double* v, double* y,
                              const double* r1, const double* r2, const double* w,
                              double* w_prev, double* x, double* v_next, double* history,
                              int64_t history_len, int64_t s, void* stream) {
  if (!state || !v || !y || !r1 || !r2 || !w || !w_prev || !x || !v_next || !history)
    return OTTB_ERR_INVALID;
  if (s < 1 || window < 1 || history_len < 2 || history_len > (int64_t)INT32_MAX)
    return OTTB_ERR_INVALID;
  ottb::minres_step_kernel<<<1, ottb::kThreads, 0, (cudaStream_t)stream>>>(
      state, 0, window, v, y, r1, r2, w, w_prev, x, v_next, history, history_len, s);
  return cudaGetLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}

}  // extern "C"
