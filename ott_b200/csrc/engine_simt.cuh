// FP32 CUDA-core sweep engine: one work unit = 128 rows of A against a
// contiguous range of 128-column tiles of B.
//
// The n x m cost never leaves registers. Each of the 256 threads owns an
// 8 x 8 micro-tile (rows ty*4+{0..3}, 64+ty*4+{0..3}; columns tx*4+{0..3},
// 64+tx*4+{0..3}) of
//   t_rc = w_c + s * <A_r, B_c>       (log2 units)
// from a d-step FFMA dot product over shared-memory tiles, scaled and
// shifted with one FFMA, followed by an online base-2 log-sum-exp with lazy
// rescaling and ex2.approx on the MUFU pipe.
#pragma once

#include "common.cuh"

namespace ottb {

template <int DP>
struct SimtSmem {
  float As[DP][kBM];
  float Bs[2][DP][kBN];
  float ws[2][kBN];
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::);
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <int DP>
__device__ __forceinline__ void simt_issue_tile(SimtSmem<DP>& sm, int buf,
                                                const SweepOperands& op,
                                                int64_t c0) {
  constexpr int kChunks = DP * (kBN / 4);
  for (int idx = threadIdx.x; idx < kChunks; idx += blockDim.x) {
    int k = idx / (kBN / 4);
    int c4 = idx % (kBN / 4);
    cp_async16(&sm.Bs[buf][k][c4 * 4], op.Bt + (int64_t)k * op.b_pad + c0 + c4 * 4);
  }
  cp_async_commit();
}

// Computes, for rows row0..row0+127 of A, the base-2 LSE state (rm, rl) of
// the columns in tiles [t0, t1). s scales <A, B>, wscale = log2(e) / eps.
template <int DP>
__device__ void simt_unit(SimtSmem<DP>& sm, const SweepOperands& op,
                          int64_t row0, int t0, int t1, float s, float wscale,
                          float* rm, float* rl) {
  const int tid = threadIdx.x;
  const int tx = tid & 15;
  const int ty = tid >> 4;
  // dot-product unrolling (registers are capped at 128 by two CTAs per SM)
  constexpr int kDotUnroll = DP <= 8 ? 2 : 4;

  // A tile.
  for (int idx = tid; idx < DP * kBM; idx += blockDim.x) {
    int k = idx / kBM, r = idx % kBM;
    sm.As[k][r] = op.At[(int64_t)k * op.a_pad + row0 + r];
  }

  float mrow[8], lrow[8], lcmp[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    mrow[i] = kNegSentinel;
    lrow[i] = 0.f;
    lcmp[i] = 0.f;
  }

  // Prologue: tile t0 into buffer 0 (points via cp.async, w computed here).
  if (t0 < t1) {
    int64_t c0 = (int64_t)t0 * kBN;
    simt_issue_tile<DP>(sm, 0, op, c0);
    if (tid < kBN) {
      int64_t c = c0 + tid;
      float w = -INFINITY;
      if (c < op.cols) w = (__ldcg(op.potB + c) - op.nb[c]) * wscale;
      sm.ws[0][tid] = w;
    }
  }

  for (int t = t0; t < t1; ++t) {
    const int buf = (t - t0) & 1;
    float wnext = -INFINITY;
    const bool has_next = (t + 1 < t1);
    if (has_next) {
      int64_t c0n = (int64_t)(t + 1) * kBN;
      simt_issue_tile<DP>(sm, buf ^ 1, op, c0n);
      if (tid < kBN) {
        int64_t c = c0n + tid;
        if (c < op.cols) wnext = (__ldcg(op.potB + c) - op.nb[c]) * wscale;
      }
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();

    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
#pragma unroll(kDotUnroll)
    for (int k = 0; k < DP; ++k) {
      float4 a0 = *reinterpret_cast<const float4*>(&sm.As[k][ty * 4]);
      float4 a1 = *reinterpret_cast<const float4*>(&sm.As[k][64 + ty * 4]);
      float4 b0 = *reinterpret_cast<const float4*>(&sm.Bs[buf][k][tx * 4]);
      float4 b1 = *reinterpret_cast<const float4*>(&sm.Bs[buf][k][64 + tx * 4]);
      float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
    }

    // t = s * <A_r, B_c> + w_c, one rounding. Seeding the FFMA chain with
    // w_c instead would round every one of the DP steps at the magnitude of
    // w_c (~|x|^2 / eps), an error 10x larger than the reference's FP32 path.
    {
      float4 w0 = *reinterpret_cast<const float4*>(&sm.ws[buf][tx * 4]);
      float4 w1 = *reinterpret_cast<const float4*>(&sm.ws[buf][64 + tx * 4]);
      float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(acc[i][j], s, wv[j]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const float cm = fmaxf(fmax3(acc[i][0], acc[i][1], acc[i][2]),
                             fmax3(acc[i][3], acc[i][4], fmax3(acc[i][5], acc[i][6], acc[i][7])));
      if (cm > mrow[i] + kTau) {
        const float sc = ex2_approx(mrow[i] - cm);
        lrow[i] *= sc;
        lcmp[i] *= sc;
        mrow[i] = cm;
      }
      float e[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const float xj = acc[i][j] - mrow[i];
        // small d is MUFU-bound: part of the exponentials on the FMA pipe
        e[j] = (DP <= 4 && j >= 8 - OTTB_POLY_OF_8) ? exp2_poly(xj) : ex2_approx(xj);
      }
      const float sum = ((e[0] + e[1]) + (e[2] + e[3])) + ((e[4] + e[5]) + (e[6] + e[7]));
      two_sum_acc(lrow[i], lcmp[i], sum);
    }
    __syncthreads();
    if (has_next && tid < kBN) sm.ws[buf ^ 1][tid] = wnext;
  }

  // Merge the 16 column-partial states of each row (lanes sharing ty).
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    lrow[i] += lcmp[i];
#pragma unroll
    for (int off = 1; off < 16; off <<= 1) {
      float m2 = __shfl_xor_sync(0xffffffffu, mrow[i], off);
      float l2 = __shfl_xor_sync(0xffffffffu, lrow[i], off);
      lse_merge(mrow[i], lrow[i], m2, l2);
    }
  }
  if (tx == 0) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      int r = (i < 4) ? (ty * 4 + i) : (64 + ty * 4 + (i - 4));
      rm[r] = mrow[i];
      rl[r] = lrow[i];
    }
  }
  __syncthreads();
}

}  // namespace ottb
