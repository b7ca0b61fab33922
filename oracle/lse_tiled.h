/*
 * Tiled, vectorised form of the C port's log-domain kernel application
 * (TEST INFRASTRUCTURE ONLY: the timed CPU baseline). Included by
 * sinkhorn_oracle.c when it is compiled with -DOTTB_TILED, in place of its
 * scalar apply_lse.
 *
 * Same function as the scalar apply_lse (geometry/geometry.py:260-299 with
 * pointcloud.py:74-103's online cost), organised the way an optimising CPU
 * backend runs it: the inner products <a_r, b_c> of a block of rows against
 * a chunk of columns as a register-blocked matrix product (6 rows x 32
 * columns of accumulators, the columns' coordinates packed in 16-wide
 * panels), then the cost, the centring (f + g) - C and the division by eps
 * in the reference's order, and a log-sum-exp over the row carried across
 * column chunks (running maximum; the sum rescaled when it moves). The
 * exponential is 2^(v log2 e) with the range reduction and degree-5
 * polynomial of tests/exp2_poly_fit.py (relative error 2.3e-7 in FP32);
 * the final logarithm is logf. Written with GCC vector extensions so one
 * source compiles to AVX-512 (-march=x86-64-v4) or AVX2 (x86-64-v3).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef float v16 __attribute__((vector_size(64)));
typedef int32_t vi16 __attribute__((vector_size(64)));

#define LT_MR 6      /* rows per micro-tile */
#define LT_NP 2      /* 16-column panels per micro-tile */
#define LT_CB 1024   /* columns per chunk (a multiple of 16 * LT_NP) */
#define LT_RB 96     /* rows per block (a multiple of LT_MR) */

static inline v16 lt_splat(float a) { return (v16){} + a; }

static inline v16 lt_select(vi16 mask, v16 a, v16 b) {
  return (v16)(((vi16)a & mask) | ((vi16)b & ~mask));
}

static inline float lt_hmax(v16 v) {
  float m = v[0];
  for (int i = 1; i < 16; ++i) m = v[i] > m ? v[i] : m;
  return m;
}

static inline float lt_hsum(v16 v) {
  float s8[8], s4[4];
  for (int i = 0; i < 8; ++i) s8[i] = v[i] + v[i + 8];
  for (int i = 0; i < 4; ++i) s4[i] = s8[i] + s8[i + 4];
  return (s4[0] + s4[2]) + (s4[1] + s4[3]);
}

/* e^v: 2^t, t = v log2 e = n + f (n = rint(t), |f| <= 1/2), 2^f by the
 * polynomial, 2^n added to the exponent field; exactly 0 for t < -126
 * (including v = -inf). Inputs here are <= 0 (centred by the running
 * maximum). */
static inline v16 lt_exp(v16 v) {
  const v16 t0 = v * 1.4426950408889634f;
  const vi16 under = t0 < -126.0f;
  const v16 t = lt_select(under, lt_splat(-126.0f), t0);
  const v16 shift = lt_splat(12582912.0f); /* 1.5 * 2^23: rounds to an integer */
  const v16 r = t + shift;
  const v16 f = t - (r - shift);
  v16 p = lt_splat(1.327647245e-03f);
  p = p * f + 9.675540961e-03f;
  p = p * f + 5.550713092e-02f;
  p = p * f + 2.402212024e-01f;
  p = p * f + 6.931469440e-01f;
  p = p * f + 1.000000119e+00f;
  const vi16 pi = (vi16)p + (((vi16)r) << 23);
  return (v16)(pi & ~under);
}

/* out[r] = eps * lse_c(((pa_r + pb_c) - C_rc) / eps) - finite(pa_r) over the
 * R rows of A against the K columns of B (C_rc = inv ((na_r + nb_c) - 2
 * <a_r, b_c>)). axis 1: A = x, B = y, pa = f, pb = g; axis 0: A = y,
 * B = x, pa = g, pb = f (the sums commute exactly, so both are the
 * reference's (f_i + g_j) - C_ij). */
static void lt_row_lse(const float* A, const float* B, const float* na, const float* nb,
                       int64_t R, int64_t K, int d, float inv, const float* pa,
                       const float* pb, float eps, float* out) {
  const int64_t kpad = (K + 16 * LT_NP - 1) / (16 * LT_NP) * (16 * LT_NP);
  const int64_t panels = kpad / 16;
  float* Bp = (float*)aligned_alloc(64, sizeof(float) * (size_t)(panels * d * 16));
  float* pbp = (float*)aligned_alloc(64, sizeof(float) * (size_t)kpad);
  float* nbp = (float*)aligned_alloc(64, sizeof(float) * (size_t)kpad);
  /* columns packed as [panel][k][16], padding columns at -inf potential */
#pragma omp parallel for schedule(static)
  for (int64_t p = 0; p < panels; ++p) {
    for (int k = 0; k < d; ++k)
      for (int l = 0; l < 16; ++l) {
        const int64_t c = p * 16 + l;
        Bp[(p * d + k) * 16 + l] = c < K ? B[c * d + k] : 0.0f;
      }
    for (int l = 0; l < 16; ++l) {
      const int64_t c = p * 16 + l;
      pbp[c] = c < K ? pb[c] : -INFINITY;
      nbp[c] = c < K ? nb[c] : 0.0f;
    }
  }
  const int64_t blocks = (R + LT_RB - 1) / LT_RB;
#pragma omp parallel
  {
    float* Ablk = (float*)aligned_alloc(64, sizeof(float) * (size_t)(LT_RB * d));
    float* vbuf = (float*)aligned_alloc(64, sizeof(float) * (size_t)(LT_MR * LT_CB));
    float mx[LT_RB], sm[LT_RB], pav[LT_RB], nav[LT_RB];
#pragma omp for schedule(dynamic, 1)
    for (int64_t blk = 0; blk < blocks; ++blk) {
      const int64_t r0 = blk * LT_RB;
      const int rows = (int)(R - r0 < LT_RB ? R - r0 : LT_RB);
      memset(Ablk, 0, sizeof(float) * (size_t)(LT_RB * d));
      memcpy(Ablk, A + r0 * d, sizeof(float) * (size_t)(rows * d));
      for (int i = 0; i < LT_RB; ++i) {
        mx[i] = -INFINITY;
        sm[i] = 0.0f;
        pav[i] = i < rows ? pa[r0 + i] : 0.0f;
        nav[i] = i < rows ? na[r0 + i] : 0.0f;
      }
      for (int64_t c0 = 0; c0 < kpad; c0 += LT_CB) {
        const int cw = (int)(kpad - c0 < LT_CB ? kpad - c0 : LT_CB);
        for (int mr = 0; mr < rows; mr += LT_MR) {
          const float* Am = Ablk + mr * d;
          for (int cc = 0; cc < cw; cc += 16 * LT_NP) {
            const float* bp = Bp + ((c0 + cc) / 16) * d * 16;
            v16 acc[LT_MR][LT_NP];
            for (int i = 0; i < LT_MR; ++i)
              for (int j = 0; j < LT_NP; ++j) acc[i][j] = lt_splat(0.0f);
            for (int k = 0; k < d; ++k) {
              v16 bv[LT_NP];
              for (int j = 0; j < LT_NP; ++j) bv[j] = *(const v16*)(bp + (j * d + k) * 16);
              for (int i = 0; i < LT_MR; ++i) {
                const float av = Am[i * d + k];
                for (int j = 0; j < LT_NP; ++j) acc[i][j] += bv[j] * av;
              }
            }
            for (int j = 0; j < LT_NP; ++j) {
              const int64_t c = c0 + cc + 16 * j;
              const v16 nbv = *(const v16*)(nbp + c);
              const v16 pbv = *(const v16*)(pbp + c);
              for (int i = 0; i < LT_MR; ++i) {
                const v16 cost = ((nav[mr + i] + nbv) + acc[i][j] * -2.0f) * inv;
                const v16 v = ((pav[mr + i] + pbv) - cost) / eps;
                *(v16*)(vbuf + i * LT_CB + cc + 16 * j) = v;
              }
            }
          }
          const int live = rows - mr < LT_MR ? rows - mr : LT_MR;
          for (int i = 0; i < live; ++i) {
            const float* vr = vbuf + i * LT_CB;
            v16 mv = *(const v16*)vr;
            for (int cc = 16; cc < cw; cc += 16) {
              const v16 x = *(const v16*)(vr + cc);
              mv = lt_select(x > mv, x, mv);
            }
            const float cm = lt_hmax(mv);
            float* m = &mx[mr + i];
            float* s = &sm[mr + i];
            if (cm > *m) {
              if (*s != 0.0f) *s *= expf(*m - cm);
              *m = cm;
            }
            const v16 sh = lt_splat(isfinite(*m) ? *m : 0.0f);
            v16 acc = lt_splat(0.0f);
            for (int cc = 0; cc < cw; cc += 16) acc += lt_exp(*(const v16*)(vr + cc) - sh);
            *s += lt_hsum(acc);
          }
        }
      }
      for (int i = 0; i < rows; ++i) {
        const float shift = isfinite(mx[i]) ? mx[i] : 0.0f;
        const float lse = logf(fabsf(sm[i])) + shift;
        const float rem = pa[r0 + i];
        out[r0 + i] = eps * lse - (isfinite(rem) ? rem : 0.0f);
      }
    }
    free(Ablk);
    free(vbuf);
  }
  free(Bp);
  free(pbp);
  free(nbp);
}
