// Shared device-side definitions for the ott_b200 Sinkhorn kernels.
//
// Problem descriptors, the per-call schedule, a grid-wide barrier whose wait
// is bounded by %globaltimer, and small numeric helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ott_b200.h"

namespace ottb {

constexpr int kBM = 128;          // rows of A per work unit
constexpr int kBN = 128;          // columns of B per tile
constexpr float kLog2e = 1.4426950408889634f;
constexpr double kLn2 = 0.69314718055994530942;
constexpr double kLog2eD = 1.4426950408889634074;
// Running maxima start at a finite sentinel so that a chunk whose entries are
// all -inf (zero-weight potentials) gives 2^(-inf - sentinel) = 0, never NaN.
constexpr float kNegSentinel = -1.0e30f;
// Lazy rescaling: the running shift moves only when a new chunk maximum is
// more than kTau (log2 units) above it, so every term is at most 2^kTau.
constexpr float kTau = 8.0f;

// Sweep kinds. A "row LSE" over rows r of A against columns c of B:
//   lse2_r = log2 sum_c 2^(w_c + s * <A_r, B_c>),
//   w_c = (pot_c - inv * |B_c|^2) * log2(e) / eps,  s = 2 * inv * log2(e) / eps.
// kSweepG updates g (A = y, B = x, pot = f); kSweepF updates f (A = x,
// B = y, pot = g).
enum SweepKind : int { kSweepG = 0, kSweepF = 1 };

// Per-problem, per-call constants (device copy of the host plan).
struct ProbDev {
  // user buffers
  const float* a;
  const float* b;
  float* f;
  float* gbuf[2];  // gbuf[0] = user g, gbuf[1] = workspace copy
  float* errors;
  // workspace: transposed + zero-padded points [DP][pad] and scaled norms
  const float* xt;
  const float* yt;
  const float* nx;
  const float* ny;
  // workspace, tensor-core path: bf16 hi/lo copies [2][pad][DK] and the
  // TMA tensor maps over them (TcMaps, in the call header)
  const void* xh;
  const void* yh;
  const void* maps;
  // workspace: split partials (m, l) [S][rows] and per-row-block data
  float* part_m;
  float* part_l;
  int* arrive;         // [max(rb_f, rb_g)] arrival counters
  double* err_part;    // [rb_g]
  double* msum_part;   // [rb_g]
  int64_t n, m, n_pad, m_pad;
  int rb_f, rb_g;      // row blocks of the f- and g-sweeps
  int split_f, split_g;
  float eps_target;
  float inv_scale;
  int uid;             // index of the problem in the caller's array
  int outer;           // length of errors
};

// Operands of one sweep for one problem, resolved from the descriptor.
struct SweepOperands {
  const float* At;    // [DP][a_pad]
  const float* Bt;    // [DP][b_pad]
  const float* potB;  // potential of B's points
  const float* nb;    // scaled squared norms of B's points
  int64_t a_pad, b_pad;
  int64_t rows, cols;  // R (rows of A), C (columns of B)
};

// Mutable per-problem state, owned by CTA 0 between barriers.
struct ProbState {
  int active;        // still iterating
  int final_parity;  // g buffer holding the final g once stopped
  int msum_valid;    // msum holds the final state's marginal sum
  int stop_it;       // iteration count at stop
  double msum;
};

// Work schedule of the current sweep, rebuilt by CTA 0 at block boundaries.
struct Sched {
  int num_active;       // problems iterating
  int total_units[2];   // units of a g-sweep / f-sweep over active problems
  int num_eval;         // problems needing a final marginal sweep
  int eval_units;
  int commits;          // g commits so far (parity of active problems)
  int status;           // OTTB_OK or OTTB_ERR_TIMEOUT
};

struct Globals {
  unsigned int bar_count;
  unsigned int bar_gen;
  unsigned int unit_ctr[3];
  int pad_;
};

__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Compensated accumulation s + c += x (Knuth's TwoSum: c collects the exact
// rounding error of every addition). Each tile's terms are first summed in a
// short tree; adding that tile sum to a long-running FP32 total would
// otherwise drop every contribution below half an ulp of the total, a
// one-signed error that, at small epsilon (many negligible terms per row),
// biases the log-sum-exp low and, differing between the f- and g-sweeps,
// accumulates along the neutral direction (f + c, g - c) of the iteration.
__device__ __forceinline__ void two_sum_acc(float& s, float& c, float x) {
  const float t = s + x;
  const float bb = t - s;
  const float err = (s - (t - bb)) + (x - bb);
  s = t;
  c += err;
}

// Merge two (shift, sum) log-sum-exp states in base 2.
__device__ __forceinline__ void lse_merge(float& m, float& l, float m2, float l2) {
  float mx = fmaxf(m, m2);
  l = l * ex2_approx(m - mx) + l2 * ex2_approx(m2 - mx);
  m = mx;
}

// Grid-wide barrier for a cooperative (co-resident) grid. The wait is
// bounded: after deadline_ns of waiting the CTA records OTTB_ERR_TIMEOUT in
// *status and returns false. expected = gridDim.x + phantom arrivals.
__device__ __forceinline__ bool grid_barrier(Globals* gl, unsigned expected,
                                             uint64_t timeout_ns, int* status) {
  __syncthreads();
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = &gl->bar_gen;
    unsigned gen = *vgen;
    __threadfence();
    unsigned arrived = atomicAdd(&gl->bar_count, 1u);
    int ok = 1;
    if (arrived == expected - 1) {
      atomicExch(&gl->bar_count, 0u);
      __threadfence();
      atomicAdd(&gl->bar_gen, 1u);
    } else {
      uint64_t t0 = global_timer_ns();
      unsigned ns = 32;
      while (*vgen == gen) {
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
        if (global_timer_ns() - t0 > timeout_ns) {
          ok = 0;
          atomicExch(status, (int)OTTB_ERR_TIMEOUT);
          break;
        }
      }
    }
    __threadfence();
    if (ok && *((volatile int*)status) == OTTB_ERR_TIMEOUT) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

}  // namespace ottb
