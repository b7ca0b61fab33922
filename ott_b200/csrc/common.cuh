// Shared device-side definitions for the ott_b200 Sinkhorn kernels.
//
// Problem descriptors, the per-call schedule, a grid-wide barrier whose wait
// is bounded by %globaltimer, and small numeric helpers.
#pragma once

#include <cuda_bf16.h>
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
  // tensor-core path: column-shift rows [pad][8] bf16 of x and [2][pad][8]
  // of y (one per g buffer), written by every potential update
  void* extx;
  void* exty;
  // workspace: split partials (m, l) [S][rows] and per-row-block data
  float* part_m;
  float* part_l;
  int* arrive;         // [max(rb_f, rb_g)] arrival counters
  double* err_part;    // [rb_g]
  double* msum_part;   // [rb_g]
  int64_t n, m, n_pad, m_pad;
  int rb_f, rb_g;      // row blocks of the f- and g-sweeps
  int smax_f, smax_g;  // largest column split the workspace partials hold
  float eps_target;
  float inv_scale;
  int uid;             // index of the problem in the caller's array
  int outer;           // length of errors
  int symmetric;       // x == y, a == b: g-sweeps only, momentum 1/2, f = g
  float* marg_out;     // [m] column marginal of the final evaluation sweep, or null
  float* lse_out;      // [m] eps log sum_i exp((f_i + g_j - C_ij) / eps) - g_j of
                       // that sweep (apply_lse_kernel), or null
  float* center;       // [128] workspace: the common centre of the two point sets
  // tensor-core path: base-2 log-sum-exp of every row in its last sweep
  // ([n_pad] x rows from f-sweeps, then [m_pad] y rows from g-sweeps), and
  // this problem's ProbState::dkey (bounds of the column shifts' changes)
  float* lprev;
  int* dkey;
  float ws_t;          // log2(e) / eps_target in FP32 (sweep_wscale at multiplier 1)
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
  int split_f;       // column split of this problem's f- and g-sweeps (set
  int split_g;       // by the host, grown at schedule rebuilds)
  double msum;
  // Tensor-core path: order-preserving integer keys (fkey) of the largest
  // and smallest change of the column shifts w_c seen by the next sweep of
  // each kind, [consumer kind][slot][0 = max, 1 = min]; slot = parity of
  // the consumer's sweep count. Empty: kDkeyEmptyMax / kDkeyEmptyMin.
  int dkey[2][2][2];
};

// Work schedule of the current sweep, rebuilt by CTA 0 at block boundaries.
struct Sched {
  int num_active;       // problems iterating
  int total_units[2];   // units of a g-sweep / f-sweep over active problems
  int num_eval;         // problems needing a final marginal sweep
  int eval_units;
  int commits;          // g commits so far (parity of active problems)
  int status;           // OTTB_OK or OTTB_ERR_TIMEOUT
  int dynamic_units;    // 1: units dealt from an atomic queue, 0: round-robin
  int target_units;     // units per sweep the schedule rebuild aims for
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

// Coefficients of the degree-5 polynomial p(f) ~ 2^f on [-1/2, 1/2].
constexpr float kExp2C5 = 1.327647245e-03f;
constexpr float kExp2C4 = 9.675540961e-03f;
constexpr float kExp2C3 = 5.550713092e-02f;
constexpr float kExp2C2 = 2.402212024e-01f;
constexpr float kExp2C1 = 6.931469440e-01f;
constexpr float kExp2C0 = 1.000000119e+00f;
constexpr float kRoundShift = 12582912.0f;  // 1.5 * 2^23

// 2^x on the FMA pipe, to take part of the exponentials off the MUFU pipe.
// Range reduction x = n + f, n = rint(x), f in [-1/2, 1/2] (exact for
// |x| < 2^22: adding 1.5 * 2^23 rounds x to an integer in the low mantissa
// bits); 2^f by a degree-5 polynomial minimising the maximum relative error
// on [-1/2, 1/2], fitted by tests/exp2_poly_fit.py (Remez exchange; 7.5e-8
// minimax, 2.3e-7 evaluated in FP32); 2^n by adding n to the exponent
// field. Inputs below -126 are clamped (the result, < 2^-125, is negligible
// next to the running sum's leading term >= 1); callers keep x <= kTau + 1.
__device__ __forceinline__ float exp2_poly(float x) {
  x = fmaxf(x, -126.0f);
  const float t = x + kRoundShift;
  const float f = x - (t - kRoundShift);
  float p = kExp2C5;
  p = fmaf(p, f, kExp2C4);
  p = fmaf(p, f, kExp2C3);
  p = fmaf(p, f, kExp2C2);
  p = fmaf(p, f, kExp2C1);
  p = fmaf(p, f, kExp2C0);
  // t's bits are 0x4B400000 + n; shifted left by 23 they are n << 23.
  return __int_as_float(__float_as_int(p) + (__float_as_int(t) << 23));
}

// Packed pairs of FP32 values (sm_100 fma/add .f32x2: two lanes of FP32
// arithmetic per instruction, same IEEE rounding as the scalar forms).
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pack2(float a, float b) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void unpack2(f32x2 r, float& a, float& b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}

__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}

// exp2_poly on a pair, the range reduction and the polynomial in packed
// arithmetic (same operations, same results as two exp2_poly calls).
__device__ __forceinline__ f32x2 exp2_poly2(f32x2 xp) {
  float x0, x1;
  unpack2(xp, x0, x1);
  const f32x2 x = pack2(fmaxf(x0, -126.0f), fmaxf(x1, -126.0f));
  const f32x2 sh = pack2(kRoundShift, kRoundShift);
  const f32x2 t = add2(x, sh);
  const f32x2 f = sub2(x, sub2(t, sh));
  f32x2 p = pack2(kExp2C5, kExp2C5);
  p = fma2(p, f, pack2(kExp2C4, kExp2C4));
  p = fma2(p, f, pack2(kExp2C3, kExp2C3));
  p = fma2(p, f, pack2(kExp2C2, kExp2C2));
  p = fma2(p, f, pack2(kExp2C1, kExp2C1));
  p = fma2(p, f, pack2(kExp2C0, kExp2C0));
  float p0, p1, t0, t1;
  unpack2(p, p0, p1);
  unpack2(t, t0, t1);
  return pack2(__int_as_float(__float_as_int(p0) + (__float_as_int(t0) << 23)),
               __int_as_float(__float_as_int(p1) + (__float_as_int(t1) << 23)));
}

// Degree-4 polynomial 2^f on [-1/2, 1/2] (tests/exp2_poly_fit.py 4: 2.6e-6
// minimax relative error, 2.7e-6 evaluated in FP32), for the tensor-core
// epilogue, whose products carry ~1e-5 relative error already (BF16
// split-3 inner products scaled to exponents of tens).
constexpr float kExp2D4C4 = 9.570102207e-03f;
constexpr float kExp2D4C3 = 5.591785908e-02f;
constexpr float kExp2D4C2 = 2.402474433e-01f;
constexpr float kExp2D4C1 = 6.931217909e-01f;
constexpr float kExp2D4C0 = 9.999992847e-01f;

// exp2_poly2 with the degree-4 polynomial: one packed FMA fewer per pair.
__device__ __forceinline__ f32x2 exp2_poly2_d4(f32x2 xp) {
  float x0, x1;
  unpack2(xp, x0, x1);
  const f32x2 x = pack2(fmaxf(x0, -126.0f), fmaxf(x1, -126.0f));
  const f32x2 sh = pack2(kRoundShift, kRoundShift);
  const f32x2 t = add2(x, sh);
  const f32x2 f = sub2(x, sub2(t, sh));
  f32x2 p = pack2(kExp2D4C4, kExp2D4C4);
  p = fma2(p, f, pack2(kExp2D4C3, kExp2D4C3));
  p = fma2(p, f, pack2(kExp2D4C2, kExp2D4C2));
  p = fma2(p, f, pack2(kExp2D4C1, kExp2D4C1));
  p = fma2(p, f, pack2(kExp2D4C0, kExp2D4C0));
  float p0, p1, t0, t1;
  unpack2(p, p0, p1);
  unpack2(t, t0, t1);
  return pack2(__int_as_float(__float_as_int(p0) + (__float_as_int(t0) << 23)),
               __int_as_float(__float_as_int(p1) + (__float_as_int(t1) << 23)));
}

// Of every 8 exponentials, this many go to exp2_poly: in the CUDA-core
// engine at d <= 4, where the MUFU pipe binds (measured at n = m = 32768,
// d = 2: 2 of 8 is 2 % faster than 0, 3 of 8 slower); and in the
// tensor-core epilogue, which runs its arithmetic on packed pairs (measured
// in isolation, 16 warps per SM: 15.4 entries/clk/SM with scalar FP32 and
// every exponential on the MUFU, 18.9 packed with 2 of 8 on the
// polynomial, 15.6 with 4 of 8).
#ifndef OTTB_POLY_OF_8
#define OTTB_POLY_OF_8 2
#endif
#ifndef OTTB_POLY_OF_8_TC
#define OTTB_POLY_OF_8_TC 2
#endif

// Order-preserving map of non-NaN floats to ints (and back), for atomic
// maxima and minima of floats of either sign.
__host__ __device__ __forceinline__ int fkey_bits(int i) { return i >= 0 ? i : i ^ 0x7fffffff; }
__device__ __forceinline__ int fkey(float f) { return fkey_bits(__float_as_int(f)); }
__device__ __forceinline__ float fkey_value(int k) { return __int_as_float(fkey_bits(k)); }
constexpr int kDkeyEmptyMax = (int)0x807fffff;  // fkey(-inf)
constexpr int kDkeyEmptyMin = 0x7f800000;        // fkey(+inf)
// Largest spread (log2 units) of the column shifts' changes for which a
// sweep uses the bounded shift instead of running maxima: the row sums then
// stay within [2^-kMaxShiftSpread, m] (see tc_unit).
constexpr float kMaxShiftSpread = 60.0f;

// Three-input maximum (sm_100 max.f32 with three sources; NaN operands are
// ignored as by fmaxf).
__device__ __forceinline__ float fmax3(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
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

// One 16-byte column-shift row of the tensor-core path: the base-2 column
// shift w = (pot - inv |p|^2) log2(e) / eps_target as three bf16 terms
// w1 + w2 + w3 (~24 bits), then two ones (the factors of the row shift the
// A operand's extension block may carry) and three zeros. A non-finite w
// (zero-weight potentials, padding rows = -inf) is carried by w1 alone, so
// no inf - inf = NaN appears.
__device__ __forceinline__ void write_ext_row(void* row16, float w) {
  const bool fin = isfinite(w);
  const __nv_bfloat16 w1 = __float2bfloat16_rn(w);
  const float r1 = fin ? w - __bfloat162float(w1) : 0.f;
  const __nv_bfloat16 w2 = __float2bfloat16_rn(r1);
  const __nv_bfloat16 w3 = __float2bfloat16_rn(fin ? r1 - __bfloat162float(w2) : 0.f);
  uint4 v;
  const uint32_t one = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(1.f));
  v.x = (uint32_t)__bfloat16_as_ushort(w1) | ((uint32_t)__bfloat16_as_ushort(w2) << 16);
  v.y = (uint32_t)__bfloat16_as_ushort(w3) | (one << 16);
  v.z = one;
  v.w = 0u;
  *reinterpret_cast<uint4*>(row16) = v;
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
