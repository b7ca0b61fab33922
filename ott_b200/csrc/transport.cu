// Transport plan of a point-cloud problem applied to vectors, and the plan
// itself, from the dual potentials (geometry/geometry.py:361-365,
// transport_from_potentials; :444-486, apply_transport_from_potentials).
//
//   P_ij = exp((f_i + g_j - inv |x_i - y_j|^2) / eps)
//   axis 1: out[k][i] = sum_j P_ij vec[k][j]     axis 0: out[k][j] = sum_i P_ij vec[k][i]
//
// FP32 on the CUDA cores. One CTA takes 128 output rows (A = x for axis 1,
// y for axis 0) and a chunk of up to 64 vectors, and streams the other point
// set (B) in 128-point tiles: per tile the exponents z (log2 units) come
// from an 8 x 8 register micro-tile per thread (the solve's sweep
// arithmetic, on points translated by a common centre so the expanded
// |A|^2 + |B|^2 - 2 <A, B> stays small), a row maximum shared by the 16
// threads of a row rescales the running sums when it grows, and the tile's
// weights 2^(z - max) go through shared memory into O += P V on the same
// threads. Each tile's contribution is summed apart and added to the
// running sum once. P is never written to global memory. A CTA takes
// 16 * VT vectors (thread tx owns vectors tx + 16 j, j < VT); the host
// splits the vectors into the fewest such chunks (every chunk recomputes
// the cost tile). The P tile is stored as float4 row quads at slots
// XOR-swizzled by the column, so the quads written by a warp and the quads
// read back fall in distinct banks. When row blocks x vector chunks give
// fewer than two waves of CTAs, the B points are split too (blockIdx.z):
// each split writes its sums with its own row shift to the workspace and
// combine_splits_kernel merges them.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>

#include "../../include/ott_b200.h"
#include "common.cuh"

namespace ottb {
namespace {

constexpr int kTR = 128;   // output rows per CTA
constexpr int kTC = 128;   // B points per tile
constexpr int kSampleMax = 256;

// Vectors per thread: up to 5 (80 per CTA), 4 at DP = 128 (shared memory).
template <int DP>
constexpr int max_vt() { return DP == 128 ? 4 : 5; }

// Rows of the A and B tiles are padded by 4 floats (16-byte reads stay
// aligned, stores spread over 8 banks instead of 1) where it fits.
template <int DP, int VT>
struct ApplySmem {
  static constexpr int kPad = DP <= 64 ? 4 : 0;
  static constexpr int kKT = 16 * VT;
  float As[DP][kTR + kPad];   // A tile, transposed, centred
  float Bs[DP][kTC + kPad];   // B tile, transposed, centred
  float Ps[kTC][kTR];         // weights of the tile, [column][swizzled row quads]
  float Vs[kTC][kKT + 1];     // vectors of the tile, [column][k]
  float wb[kTC];              // (potB - inv |B|^2) * log2e / eps
  float center[DP];
};

// Float offset of row quad q (rows 4q .. 4q + 3, q < 32) of column c in Ps.
__device__ __forceinline__ int pquad(int c, int q) {
  return c * kTR + (q & 16) * 4 + (((q & 15) ^ ((c >> 2) & 7)) * 4);
}

struct ApplyArgs {
  const float* A;     // [R][d] output-side points
  const float* B;     // [C][d] summed-over points
  const float* potA;  // [R]
  const float* potB;  // [C]
  const float* vec;   // [K][C]
  float* out;         // [K][R]
  int64_t R, C;
  int d, K;
  float ws;           // log2(e) / eps
  float inv;          // inverse cost scale
  int splits;         // column splits (1: write out directly)
  float* part_o;      // [splits][K][R] sums of each split (splits > 1)
  float* part_m;      // [splits][R] their row shifts (log2 units)
  // operands prepared once per call for the pipelined kernel (null: the
  // tiles are transposed from A, B, vec inside the kernel)
  float* cen;         // [DP] common centre
  float* bt;          // [DP][c_pad] B transposed, centred, zero-padded
  float* wbv;         // [c_pad] (potB - inv |B - centre|^2) * ws, -inf padding
  float* vt;          // [c_pad][k_pad] vectors transposed, zero-padded
  int64_t c_pad, k_pad;
  int prepared;       // host only: cen, bt and wbv already hold this plan's values
};

// Common centre of both point sets: the mean of up to kSampleMax points of
// each, taken at a fixed stride (every CTA computes the same value).
template <int DP>
__device__ void apply_center(const ApplyArgs& p, float* center) {
  // warp w takes coordinates w, w + 8, ...; its lanes sum disjoint samples
  // and a fixed shuffle tree adds them (256 threads per CTA)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int warps = blockDim.x >> 5;
  const int64_t na = p.R < kSampleMax ? p.R : kSampleMax;
  const int64_t nb = p.C < kSampleMax ? p.C : kSampleMax;
  const int64_t sa = p.R / na, sb = p.C / nb;
  for (int k = warp; k < DP; k += warps) {
    float ma = 0.f, mb = 0.f;
    if (k < p.d) {
      for (int64_t i = lane; i < na; i += 32) ma += p.A[i * sa * p.d + k];
      for (int64_t i = lane; i < nb; i += 32) mb += p.B[i * sb * p.d + k];
    }
    for (int off = 16; off > 0; off >>= 1) {
      ma += __shfl_xor_sync(0xffffffffu, ma, off);
      mb += __shfl_xor_sync(0xffffffffu, mb, off);
    }
    if (lane == 0) center[k] = k < p.d ? 0.5f * (ma / (float)na + mb / (float)nb) : 0.f;
  }
}

// ---- pieces shared by the application kernels -----------------------------
// Rows of this thread's 8 x 8 micro-tile: ty*4 + {0..3}, 64 + ty*4 + {0..3};
// its columns are tx*4 + {0..3}, 64 + tx*4 + {0..3}.
__device__ __forceinline__ int tile_row(int ty, int i) {
  return (i < 4) ? (ty * 4 + i) : (64 + ty * 4 + (i - 4));
}

// The A tile (transposed, centred; rows beyond R are zero points), then the
// row terms u_r = (potA_r - inv |A_r|^2) * ws of this thread's 8 rows
// (-inf beyond R).
template <int DP, int LD>
__device__ __forceinline__ void load_rows(const ApplyArgs& p, float (*As)[LD],
                                          const float* center, int64_t row0, int ty,
                                          float u[8]) {
  for (int idx = threadIdx.x; idx < DP * kTR; idx += blockDim.x) {
    const int r = idx / DP, k = idx % DP;
    const int64_t gr = row0 + r;
    As[k][r] = (gr < p.R && k < p.d) ? p.A[gr * p.d + k] - center[k] : 0.f;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = tile_row(ty, i);
    const int64_t gr = row0 + r;
    float nrm = 0.f;
    for (int k = 0; k < DP; ++k) nrm = fmaf(As[k][r], As[k][r], nrm);
    u[i] = gr < p.R ? (__ldg(p.potA + gr) - p.inv * nrm) * p.ws : -INFINITY;
  }
}

// Exponents z = s <A_r, B_c> + wb_c + u_r (log2 units) of the micro-tile:
// an FFMA chain over the d coordinates, then one rounding for the scale and
// shift.
template <int DP, int LDA, int LDB>
__device__ __forceinline__ void cost_tile(const float (*As)[LDA], const float (*Bs)[LDB],
                                          const float* wb, float s, const float u[8], int tx,
                                          int ty, float z[8][8]) {
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) z[i][j] = 0.f;
#pragma unroll 4
  for (int k = 0; k < DP; ++k) {
    const float4 a0 = *reinterpret_cast<const float4*>(&As[k][ty * 4]);
    const float4 a1 = *reinterpret_cast<const float4*>(&As[k][64 + ty * 4]);
    const float4 b0 = *reinterpret_cast<const float4*>(&Bs[k][tx * 4]);
    const float4 b1 = *reinterpret_cast<const float4*>(&Bs[k][64 + tx * 4]);
    const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
    const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) z[i][j] = fmaf(av[i], bv[j], z[i][j]);
  }
  const float4 w0 = *reinterpret_cast<const float4*>(&wb[tx * 4]);
  const float4 w1 = *reinterpret_cast<const float4*>(&wb[64 + tx * 4]);
  const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) z[i][j] = fmaf(z[i][j], s, wv[j]) + u[i];
}

// Per row: the tile's maximum over the 16 threads of the row; when it grows
// the row's NA running sums are rescaled; then z = 2^(z - max).
template <int NA>
__device__ __forceinline__ void exp_rows(float z[8][8], float mrow[8], float o[8][NA]) {
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    float mx = fmaxf(fmax3(z[i][0], z[i][1], z[i][2]),
                     fmax3(z[i][3], z[i][4], fmax3(z[i][5], z[i][6], z[i][7])));
#pragma unroll
    for (int off = 1; off < 16; off <<= 1)
      mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    if (mx > mrow[i]) {
      const float sc = ex2_approx(mrow[i] - mx);
#pragma unroll
      for (int j = 0; j < NA; ++j) o[i][j] *= sc;
      mrow[i] = mx;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) z[i][j] = ex2_approx(z[i][j] - mrow[i]);
  }
}

// The weights of the micro-tile into the swizzled P tile: rows ty*4 .. +3
// (quad ty) and 64 + ty*4 .. +3 (quad 16 + ty) of each of its columns.
__device__ __forceinline__ void store_p_quads(float* Ps, const float z[8][8], int tx, int ty) {
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int c = (j < 4) ? (tx * 4 + j) : (64 + tx * 4 + (j - 4));
    *reinterpret_cast<float4*>(Ps + pquad(c, ty)) =
        make_float4(z[0][j], z[1][j], z[2][j], z[3][j]);
    *reinterpret_cast<float4*>(Ps + pquad(c, 16 + ty)) =
        make_float4(z[4][j], z[5][j], z[6][j], z[7][j]);
  }
}

// O[r][k] += sum_c P[r][c] V[c][k] for this thread's 8 rows and vectors
// tx + 16 j; the tile's contribution is summed apart, then added once.
template <int VT, int LDV>
__device__ __forceinline__ void pv_tile(const float* Ps, const float (*Vs)[LDV], int tx, int ty,
                                        float o[8][VT]) {
  float acc[8][VT];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < VT; ++j) acc[i][j] = 0.f;
#pragma unroll 4
  for (int c = 0; c < kTC; ++c) {
    const float4 p0 = *reinterpret_cast<const float4*>(Ps + pquad(c, ty));
    const float4 p1 = *reinterpret_cast<const float4*>(Ps + pquad(c, 16 + ty));
    const float pv[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
    float vv[VT];
#pragma unroll
    for (int j = 0; j < VT; ++j) vv[j] = Vs[c][tx + 16 * j];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < VT; ++j) acc[i][j] = fmaf(pv[i], vv[j], acc[i][j]);
  }
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < VT; ++j) o[i][j] += acc[i][j];
}

// Row r's sums times 2^max into out (a row whose weights are all zero gives
// 0), or with column splits this split's sums and shift into the workspace.
// Vector j of this thread is k0 + tx + 16 j (lane_stride 16), or k0 + j with
// the lanes of a row already reduced (lane_stride 0, thread tx == 0).
template <int NV>
__device__ __forceinline__ void store_rows(const ApplyArgs& p, const float o[8][NV],
                                           const float mrow[8], int64_t row0, int tx, int ty,
                                           int k0, int lane_stride) {
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int64_t gr = row0 + tile_row(ty, i);
    if (gr >= p.R) continue;
    const bool any = mrow[i] > kNegSentinel;
    if (p.splits > 1) {
      const int64_t sp = blockIdx.z;
      if (tx == 0 && blockIdx.y == 0) p.part_m[sp * p.R + gr] = any ? mrow[i] : -INFINITY;
#pragma unroll
      for (int j = 0; j < NV; ++j) {
        const int k = k0 + tx * (lane_stride ? 1 : 0) + (lane_stride ? 16 : 1) * j;
        if (k < p.K) p.part_o[(sp * p.K + k) * p.R + gr] = any ? o[i][j] : 0.f;
      }
      continue;
    }
    const float scale = any ? exp2f(mrow[i]) : 0.f;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      const int k = k0 + tx * (lane_stride ? 1 : 0) + (lane_stride ? 16 : 1) * j;
      if (k < p.K) p.out[(int64_t)k * p.R + gr] = any ? o[i][j] * scale : 0.f;
    }
  }
}

// The one- or two-vector products of the micro-tile: exponentials as in
// exp_rows, times the vectors' entries at this thread's 8 columns (the
// first k_valid vectors; the others are 0), added to the row sums.
template <int KD>
__device__ __forceinline__ void direct_tile(float z[8][8], float mrow[8], float o[8][KD],
                                            const float (*Vs)[kTC], int tx, int k_valid) {
  float vv[KD][8];
#pragma unroll
  for (int kk = 0; kk < KD; ++kk) {
    const float4 v0 = *reinterpret_cast<const float4*>(&Vs[kk][tx * 4]);
    const float4 v1 = *reinterpret_cast<const float4*>(&Vs[kk][64 + tx * 4]);
    const bool on = kk < k_valid;
    vv[kk][0] = on ? v0.x : 0.f; vv[kk][1] = on ? v0.y : 0.f;
    vv[kk][2] = on ? v0.z : 0.f; vv[kk][3] = on ? v0.w : 0.f;
    vv[kk][4] = on ? v1.x : 0.f; vv[kk][5] = on ? v1.y : 0.f;
    vv[kk][6] = on ? v1.z : 0.f; vv[kk][7] = on ? v1.w : 0.f;
  }
  exp_rows<KD>(z, mrow, o);
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int kk = 0; kk < KD; ++kk) {
      float part = z[i][0] * vv[kk][0];
#pragma unroll
      for (int j = 1; j < 8; ++j) part = fmaf(z[i][j], vv[kk][j], part);
      o[i][kk] += part;
    }
}

// The 16 threads of a row hold partial sums with the same shift: add them,
// and thread tx == 0 stores the row.
template <int KD>
__device__ __forceinline__ void direct_store(const ApplyArgs& p, float o[8][KD],
                                             const float mrow[8], int64_t row0, int tx, int ty) {
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int kk = 0; kk < KD; ++kk)
#pragma unroll
      for (int off = 1; off < 16; off <<= 1)
        o[i][kk] += __shfl_xor_sync(0xffffffffu, o[i][kk], off);
  if (tx == 0) store_rows<KD>(p, o, mrow, row0, 0, ty, 0, 0);
}

template <int DP, int VT>
__global__ void __launch_bounds__(256, 1) apply_transport_kernel(ApplyArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ApplySmem<DP, VT>& sm = *reinterpret_cast<ApplySmem<DP, VT>*>(smem_raw);
  constexpr int kKT = ApplySmem<DP, VT>::kKT;
  const int tid = threadIdx.x;
  const int tx = tid & 15;
  const int ty = tid >> 4;
  const int64_t row0 = (int64_t)blockIdx.x * kTR;
  const int k0 = blockIdx.y * kKT;
  const float s = 2.f * p.inv * p.ws;

  apply_center<DP>(p, sm.center);
  __syncthreads();
  float u[8];
  load_rows<DP>(p, sm.As, sm.center, row0, ty, u);
  float mrow[8];
  float o[8][VT];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    mrow[i] = kNegSentinel;
#pragma unroll
    for (int j = 0; j < VT; ++j) o[i][j] = 0.f;
  }

  const int64_t ntiles_all = (p.C + kTC - 1) / kTC;
  const int64_t t_begin = ntiles_all * blockIdx.z / p.splits;
  const int64_t t_end = ntiles_all * (blockIdx.z + 1) / p.splits;
  for (int64_t t = t_begin; t < t_end; ++t) {
    const int64_t c0 = t * kTC;
    __syncthreads();  // previous tile's Ps / Vs / Bs consumed
    for (int idx = tid; idx < DP * kTC; idx += blockDim.x) {
      const int c = idx / DP, k = idx % DP;
      const int64_t gc = c0 + c;
      sm.Bs[k][c] = (gc < p.C && k < p.d) ? p.B[gc * p.d + k] - sm.center[k] : 0.f;
    }
    for (int idx = tid; idx < kTC * kKT; idx += blockDim.x) {
      const int kk = idx / kTC, c = idx % kTC;
      const int64_t gc = c0 + c;
      sm.Vs[c][kk] = (gc < p.C && k0 + kk < p.K) ? __ldg(p.vec + (int64_t)(k0 + kk) * p.C + gc) : 0.f;
    }
    __syncthreads();
    if (tid < kTC) {
      const int64_t gc = c0 + tid;
      float nrm = 0.f;
      for (int k = 0; k < DP; ++k) nrm = fmaf(sm.Bs[k][tid], sm.Bs[k][tid], nrm);
      sm.wb[tid] = gc < p.C ? (__ldg(p.potB + gc) - p.inv * nrm) * p.ws : -INFINITY;
    }
    __syncthreads();
    float z[8][8];
    cost_tile<DP>(sm.As, sm.Bs, sm.wb, s, u, tx, ty, z);
    exp_rows<VT>(z, mrow, o);
    store_p_quads(&sm.Ps[0][0], z, tx, ty);
    __syncthreads();
    pv_tile<VT>(&sm.Ps[0][0], sm.Vs, tx, ty, o);
  }
  store_rows<VT>(p, o, mrow, row0, tx, ty, k0, 16);
}

__device__ __forceinline__ void tp_cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void tp_cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::);
}
template <int N>
__device__ __forceinline__ void tp_cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// The operands of the pipelined kernel, prepared once per call: the common
// centre (same sample as apply_center), B transposed and centred with its
// column terms, and the vectors transposed to [point][vector].
// One block per dimension (256 threads): the same samples as apply_center,
// summed by a fixed-order tree (any centre gives the same plan; this one is
// the sample mean of both sets).
__global__ void apply_prep_center_kernel(ApplyArgs p) {
  __shared__ float sa[256], sb[256];
  const int k = blockIdx.x, t = threadIdx.x;
  const int64_t na = p.R < kSampleMax ? p.R : kSampleMax;
  const int64_t nb = p.C < kSampleMax ? p.C : kSampleMax;
  const int64_t stra = p.R / na, strb = p.C / nb;
  sa[t] = (k < p.d && t < na) ? p.A[t * stra * p.d + k] : 0.f;
  sb[t] = (k < p.d && t < nb) ? p.B[t * strb * p.d + k] : 0.f;
  __syncthreads();
  for (int off = 128; off > 0; off >>= 1) {
    if (t < off) {
      sa[t] += sa[t + off];
      sb[t] += sb[t + off];
    }
    __syncthreads();
  }
  if (t == 0) p.cen[k] = k < p.d ? 0.5f * (sa[0] / (float)na + sb[0] / (float)nb) : 0.f;
}

__global__ void apply_prep_b_kernel(ApplyArgs p, int dp) {
  const int64_t total = (int64_t)dp * p.c_pad;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = idx / p.c_pad, c = idx % p.c_pad;
    p.bt[idx] = (c < p.C && k < p.d) ? p.B[c * p.d + k] - p.cen[k] : 0.f;
  }
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < p.c_pad;
       c += (int64_t)gridDim.x * blockDim.x) {
    float nrm = 0.f;
    if (c < p.C)
      for (int k = 0; k < p.d; ++k) {
        const float t = p.B[c * p.d + k] - p.cen[k];
        nrm = fmaf(t, t, nrm);
      }
    p.wbv[c] = c < p.C ? (__ldg(p.potB + c) - p.inv * nrm) * p.ws : -INFINITY;
  }
}

// vt[c][k] = vec[k][c] through 32 x 32 shared tiles (both sides coalesced).
__global__ void apply_prep_v_kernel(ApplyArgs p) {
  __shared__ float tile[32][33];
  const int64_t c0 = (int64_t)blockIdx.x * 32, k0 = (int64_t)blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const int64_t k = k0 + r, c = c0 + tx;
    tile[r][tx] = (k < p.K && c < p.C) ? p.vec[k * p.C + c] : 0.f;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int64_t c = c0 + r, k = k0 + tx;
    if (c < p.c_pad && k < p.k_pad) p.vt[c * p.k_pad + k] = tile[tx][r];
  }
}

// apply_transport_kernel with its B and vector tiles streamed by cp.async
// from the prepared operands: the next B tile (double-buffered) and this
// tile's vectors load while the cost tile is computed, instead of stalling
// the single 8-warp CTA of the SM on global loads at every tile. d <= 64
// (the double buffers fit in 227 KB with the P tile).
template <int DP, int VT>
struct PipeSmem {
  static constexpr int kKT = 16 * VT;
  float As[DP][kTR + 4];
  float Bs[2][DP][kTC + 4];
  float wb[2][kTC];
  float Ps[kTC][kTR];
  float Vs[kTC][kKT + 4];
  float center[DP];
};

template <int DP, int VT>
__global__ void __launch_bounds__(256, 1) apply_pipelined_kernel(ApplyArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PipeSmem<DP, VT>& sm = *reinterpret_cast<PipeSmem<DP, VT>*>(smem_raw);
  constexpr int kKT = PipeSmem<DP, VT>::kKT;
  const int tid = threadIdx.x;
  const int tx = tid & 15;
  const int ty = tid >> 4;
  const int64_t row0 = (int64_t)blockIdx.x * kTR;
  const int k0 = blockIdx.y * kKT;
  const float s = 2.f * p.inv * p.ws;

  for (int k = tid; k < DP; k += blockDim.x) sm.center[k] = p.cen[k];
  __syncthreads();
  float u[8];
  load_rows<DP>(p, sm.As, sm.center, row0, ty, u);
  float mrow[8];
  float o[8][VT];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    mrow[i] = kNegSentinel;
#pragma unroll
    for (int j = 0; j < VT; ++j) o[i][j] = 0.f;
  }

  // B tile t (DP rows of 128 floats) and its column terms into buffer buf
  auto issue_b = [&](int64_t t, int buf) {
    const int64_t c0 = t * kTC;
    for (int idx = tid; idx < DP * (kTC / 4); idx += blockDim.x) {
      const int k = idx / (kTC / 4), q = idx % (kTC / 4);
      tp_cp_async16(&sm.Bs[buf][k][q * 4], p.bt + (int64_t)k * p.c_pad + c0 + q * 4);
    }
    if (tid < kTC / 4) tp_cp_async16(&sm.wb[buf][tid * 4], p.wbv + c0 + tid * 4);
    tp_cp_async_commit();
  };
  // this chunk's vectors at tile t's points
  auto issue_v = [&](int64_t t) {
    const int64_t c0 = t * kTC;
    for (int idx = tid; idx < kTC * (kKT / 4); idx += blockDim.x) {
      const int c = idx / (kKT / 4), q = idx % (kKT / 4);
      tp_cp_async16(&sm.Vs[c][q * 4], p.vt + (c0 + c) * p.k_pad + k0 + q * 4);
    }
    tp_cp_async_commit();
  };

  const int64_t ntiles_all = (p.C + kTC - 1) / kTC;
  const int64_t t_begin = ntiles_all * blockIdx.z / p.splits;
  const int64_t t_end = ntiles_all * (blockIdx.z + 1) / p.splits;
  if (t_begin < t_end) issue_b(t_begin, 0);
  for (int64_t t = t_begin; t < t_end; ++t) {
    const int buf = (int)((t - t_begin) & 1);
    const bool has_next = t + 1 < t_end;
    __syncthreads();  // previous tile's Ps, Vs and B buffer consumed
    // commit order: B(t) (earlier), V(t), B(t + 1)
    issue_v(t);
    if (has_next) {
      issue_b(t + 1, buf ^ 1);
      tp_cp_async_wait<2>();  // B(t) landed
    } else {
      tp_cp_async_wait<1>();
    }
    __syncthreads();
    float z[8][8];
    cost_tile<DP>(sm.As, sm.Bs[buf], sm.wb[buf], s, u, tx, ty, z);
    exp_rows<VT>(z, mrow, o);
    store_p_quads(&sm.Ps[0][0], z, tx, ty);
    if (has_next)
      tp_cp_async_wait<1>();  // V(t) landed (B(t + 1) may still be in flight)
    else
      tp_cp_async_wait<0>();
    __syncthreads();
    pv_tile<VT>(&sm.Ps[0][0], sm.Vs, tx, ty, o);
  }
  store_rows<VT>(p, o, mrow, row0, tx, ty, k0, 16);
}

// One or two vectors (the conjugate-gradient steps of implicit
// differentiation apply the plan to one vector at a time): each thread
// multiplies its 8 x 8 weights by its 8 columns' vector entries in
// registers, and the 16 threads of a row add their partial sums at the
// end. No P tile goes through shared memory, so two CTAs share an SM up to
// d = 64 and one CTA's tile loads overlap the other's arithmetic.
template <int DP, int KD>
struct DirectSmem {
  static constexpr int kPad = DP <= 64 ? 4 : 0;
  float As[DP][kTR + kPad];   // A tile, transposed, centred
  float Bs[DP][kTC + kPad];   // B tile, transposed, centred
  float Vs[KD][kTC];          // vector entries of the tile's B points
  float wb[kTC];              // (potB - inv |B|^2) * log2e / eps
  float center[DP];
};

template <int DP, int KD>
__global__ void __launch_bounds__(256, (DP <= 64 ? 2 : 1)) apply_direct_kernel(ApplyArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  DirectSmem<DP, KD>& sm = *reinterpret_cast<DirectSmem<DP, KD>*>(smem_raw);
  const int tid = threadIdx.x;
  const int tx = tid & 15;
  const int ty = tid >> 4;
  const int64_t row0 = (int64_t)blockIdx.x * kTR;
  const float s = 2.f * p.inv * p.ws;

  apply_center<DP>(p, sm.center);
  __syncthreads();
  float u[8];
  load_rows<DP>(p, sm.As, sm.center, row0, ty, u);
  float mrow[8];
  float o[8][KD];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    mrow[i] = kNegSentinel;
#pragma unroll
    for (int j = 0; j < KD; ++j) o[i][j] = 0.f;
  }

  const int64_t ntiles_all = (p.C + kTC - 1) / kTC;
  const int64_t t_begin = ntiles_all * blockIdx.z / p.splits;
  const int64_t t_end = ntiles_all * (blockIdx.z + 1) / p.splits;
  for (int64_t t = t_begin; t < t_end; ++t) {
    const int64_t c0 = t * kTC;
    __syncthreads();  // previous tile's Bs / Vs / wb consumed
    for (int idx = tid; idx < DP * kTC; idx += blockDim.x) {
      const int c = idx / DP, k = idx % DP;
      const int64_t gc = c0 + c;
      sm.Bs[k][c] = (gc < p.C && k < p.d) ? p.B[gc * p.d + k] - sm.center[k] : 0.f;
    }
    for (int idx = tid; idx < KD * kTC; idx += blockDim.x) {
      const int kk = idx / kTC, c = idx % kTC;
      const int64_t gc = c0 + c;
      sm.Vs[kk][c] = (gc < p.C && kk < p.K) ? __ldg(p.vec + (int64_t)kk * p.C + gc) : 0.f;
    }
    __syncthreads();
    if (tid < kTC) {
      const int64_t gc = c0 + tid;
      float nrm = 0.f;
      for (int k = 0; k < DP; ++k) nrm = fmaf(sm.Bs[k][tid], sm.Bs[k][tid], nrm);
      sm.wb[tid] = gc < p.C ? (__ldg(p.potB + gc) - p.inv * nrm) * p.ws : -INFINITY;
    }
    __syncthreads();
    float z[8][8];
    cost_tile<DP>(sm.As, sm.Bs, sm.wb, s, u, tx, ty, z);
    direct_tile<KD>(z, mrow, o, sm.Vs, tx, KD);
  }
  direct_store<KD>(p, o, mrow, row0, tx, ty);
}

// out[k][r] = sum_s part_o[s][k][r] 2^(part_m[s][r] - M) 2^M, M = max_s part_m.
__global__ void combine_splits_kernel(ApplyArgs p) {
  const int64_t total = (int64_t)p.K * p.R;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx % p.R;
    float mx = -INFINITY;
    for (int sp = 0; sp < p.splits; ++sp) mx = fmaxf(mx, p.part_m[(int64_t)sp * p.R + r]);
    float acc = 0.f;
    if (mx > -INFINITY) {
      for (int sp = 0; sp < p.splits; ++sp) {
        const float ms = p.part_m[(int64_t)sp * p.R + r];
        if (ms > -INFINITY) acc += p.part_o[(int64_t)sp * total + idx] * exp2f(ms - mx);
      }
      acc *= exp2f(mx);
    }
    p.out[idx] = acc;
  }
}

// Dense plan P[i][j], one 32 x 32 block per CTA (for inspection of small
// problems: the plan is n x m floats).
__global__ void transport_matrix_kernel(const float* x, const float* y, int64_t n, int64_t m,
                                        int d, const float* f, const float* g, float eps,
                                        float inv, float* out) {
  __shared__ float xs[32][129];
  __shared__ float ys[32][129];
  const int64_t i0 = (int64_t)blockIdx.y * 32, j0 = (int64_t)blockIdx.x * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
  for (int idx = threadIdx.x; idx < 32 * d; idx += blockDim.x) {
    const int r = idx / d, k = idx % d;
    xs[r][k] = (i0 + r < n) ? x[(i0 + r) * d + k] : 0.f;
    ys[r][k] = (j0 + r < m) ? y[(j0 + r) * d + k] : 0.f;
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int64_t i = i0 + r, j = j0 + tx;
    if (i >= n || j >= m) continue;
    float c = 0.f;
    for (int k = 0; k < d; ++k) {
      const float t = xs[r][k] - ys[tx][k];
      c = fmaf(t, t, c);
    }
    out[i * m + j] = expf((f[i] + g[j] - inv * c) / eps);
  }
}

template <int DP, int VT>
int launch_apply_vt(const ApplyArgs& a, int chunks, cudaStream_t stream) {
  const size_t smem = sizeof(ApplySmem<DP, VT>);
  auto k = apply_transport_kernel<DP, VT>;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return OTTB_ERR_CUDA;
  dim3 grid((unsigned)((a.R + kTR - 1) / kTR), (unsigned)chunks, (unsigned)a.splits);
  k<<<grid, 256, smem, stream>>>(a);
  if (a.splits > 1) {
    const int64_t total = (int64_t)a.K * a.R;
    combine_splits_kernel<<<(unsigned)std::min<int64_t>((total + 255) / 256, 4096), 256, 0,
                            stream>>>(a);
  }
  return cudaGetLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}

// The one or two vectors zero-padded to c_pad columns (16-byte cp.async rows).
__global__ void apply_prep_vpad_kernel(ApplyArgs p) {
  const int64_t total = (int64_t)p.K * p.c_pad;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = idx / p.c_pad, c = idx % p.c_pad;
    p.vt[idx] = c < p.C ? p.vec[k * p.C + c] : 0.f;
  }
}

// apply_direct_kernel on the prepared operands: the next B tile, its column
// terms and vector entries stream in by cp.async (double-buffered) while the
// current tile is computed.
template <int DP, int KD>
struct DirectPipeSmem {
  float As[DP][kTR + 4];
  float Bs[2][DP][kTC + 4];
  float Vs[2][KD][kTC];
  float wb[2][kTC];
  float center[DP];
};

template <int DP, int KD>
__global__ void __launch_bounds__(256, (DP <= 64 ? 2 : 1))
apply_direct_pipelined_kernel(ApplyArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  DirectPipeSmem<DP, KD>& sm = *reinterpret_cast<DirectPipeSmem<DP, KD>*>(smem_raw);
  const int tid = threadIdx.x;
  const int tx = tid & 15;
  const int ty = tid >> 4;
  const int64_t row0 = (int64_t)blockIdx.x * kTR;
  const float s = 2.f * p.inv * p.ws;

  for (int k = tid; k < DP; k += blockDim.x) sm.center[k] = p.cen[k];
  __syncthreads();
  float u[8];
  load_rows<DP>(p, sm.As, sm.center, row0, ty, u);
  float mrow[8];
  float o[8][KD];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    mrow[i] = kNegSentinel;
#pragma unroll
    for (int j = 0; j < KD; ++j) o[i][j] = 0.f;
  }

  auto issue = [&](int64_t t, int buf) {
    const int64_t c0 = t * kTC;
    for (int idx = tid; idx < DP * (kTC / 4); idx += blockDim.x) {
      const int k = idx / (kTC / 4), q = idx % (kTC / 4);
      tp_cp_async16(&sm.Bs[buf][k][q * 4], p.bt + (int64_t)k * p.c_pad + c0 + q * 4);
    }
    if (tid < kTC / 4) tp_cp_async16(&sm.wb[buf][tid * 4], p.wbv + c0 + tid * 4);
    for (int idx = tid; idx < KD * (kTC / 4); idx += blockDim.x) {
      const int kk = idx / (kTC / 4), q = idx % (kTC / 4);
      if (kk < p.K)
        tp_cp_async16(&sm.Vs[buf][kk][q * 4], p.vt + (int64_t)kk * p.c_pad + c0 + q * 4);
    }
    tp_cp_async_commit();
  };

  const int64_t ntiles_all = (p.C + kTC - 1) / kTC;
  const int64_t t_begin = ntiles_all * blockIdx.z / p.splits;
  const int64_t t_end = ntiles_all * (blockIdx.z + 1) / p.splits;
  if (t_begin < t_end) issue(t_begin, 0);
  for (int64_t t = t_begin; t < t_end; ++t) {
    const int buf = (int)((t - t_begin) & 1);
    __syncthreads();  // the other buffer's previous tile consumed
    if (t + 1 < t_end) {
      issue(t + 1, buf ^ 1);
      tp_cp_async_wait<1>();
    } else {
      tp_cp_async_wait<0>();
    }
    __syncthreads();
    float z[8][8];
    cost_tile<DP>(sm.As, sm.Bs[buf], sm.wb[buf], s, u, tx, ty, z);
    direct_tile<KD>(z, mrow, o, sm.Vs[buf], tx, p.K);
  }
  direct_store<KD>(p, o, mrow, row0, tx, ty);
}

template <int DP, int KD>
int launch_direct_pipelined(const ApplyArgs& a, cudaStream_t stream);

template <int DP, int KD>
int launch_direct(const ApplyArgs& a, cudaStream_t stream) {
  if constexpr (DP <= 64) {
    if (a.bt) return launch_direct_pipelined<DP, KD>(a, stream);
  }
  const size_t smem = sizeof(DirectSmem<DP, KD>);
  auto k = apply_direct_kernel<DP, KD>;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return OTTB_ERR_CUDA;
  dim3 grid((unsigned)((a.R + kTR - 1) / kTR), 1u, (unsigned)a.splits);
  k<<<grid, 256, smem, stream>>>(a);
  if (a.splits > 1) {
    const int64_t total = (int64_t)a.K * a.R;
    combine_splits_kernel<<<(unsigned)std::min<int64_t>((total + 255) / 256, 4096), 256, 0,
                            stream>>>(a);
  }
  return cudaGetLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}

template <int DP, int KD>
int launch_direct_pipelined(const ApplyArgs& a, cudaStream_t stream) {
  {
    const size_t smem = sizeof(DirectPipeSmem<DP, KD>);
    auto k = apply_direct_pipelined_kernel<DP, KD>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return OTTB_ERR_CUDA;
    if (!a.prepared) {
      apply_prep_center_kernel<<<DP, 256, 0, stream>>>(a);
      const int64_t tot = (int64_t)DP * a.c_pad;
      apply_prep_b_kernel<<<(unsigned)std::min<int64_t>((tot + 255) / 256, 4096), 256, 0,
                            stream>>>(a, DP);
    }
    const int64_t vtot = (int64_t)a.K * a.c_pad;
    apply_prep_vpad_kernel<<<(unsigned)std::min<int64_t>((vtot + 255) / 256, 4096), 256, 0,
                             stream>>>(a);
    dim3 grid((unsigned)((a.R + kTR - 1) / kTR), 1u, (unsigned)a.splits);
    k<<<grid, 256, smem, stream>>>(a);
    if (a.splits > 1) {
      const int64_t total = (int64_t)a.K * a.R;
      combine_splits_kernel<<<(unsigned)std::min<int64_t>((total + 255) / 256, 4096), 256, 0,
                              stream>>>(a);
    }
    return cudaGetLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
  }
}

// Up to this many vectors take the register path (apply_direct_kernel).
constexpr int kDirectMax = 2;

// Vector chunks of a call: the fewest chunks of at most 16 * max_vt
// vectors (one for the register path).
int apply_chunks(int d, int K) {
  if (K <= kDirectMax) return 1;
  const int vm = d > 64 ? 4 : 5;
  return (K + 16 * vm - 1) / (16 * vm);
}

// Column splits (at most 16, at least one tile of B points each): the count
// that minimises waves x (tiles per CTA + 1), the launch's time when every
// CTA slot (two per SM on the register path up to d = 64, else one) runs
// at the same speed and a CTA's set-up (centre, A tile, norms, output)
// costs about one tile; more splits only for a 3 % gain. This fills the
// last wave: n = m = 65536 takes 4 splits (7 waves of 128 tiles) instead
// of 2 (4 waves of 256), n = m = 8192 takes 4 (one wave of 16 tiles).
int apply_splits(int64_t R, int64_t C, int d, int K, int sms) {
  const int64_t units = ((R + kTR - 1) / kTR) * apply_chunks(d, K);
  const int64_t per_sm = (K <= kDirectMax && d <= 64) ? 2 : 1;
  const int64_t slots = per_sm * (int64_t)sms;
  const int64_t tiles = (C + kTC - 1) / kTC;
  const int64_t smax = std::max<int64_t>(1, std::min<int64_t>(tiles, 16));
  int64_t best = 1, best_t = -1;
  for (int64_t s = 1; s <= smax; ++s) {
    const int64_t waves = (units * s + slots - 1) / slots;
    const int64_t t = waves * ((tiles + s - 1) / s + 1);
    if (best_t < 0 || 100 * t < 97 * best_t) {
      best_t = t;
      best = s;
    }
  }
  return (int)best;
}

size_t apply_workspace(int64_t R, int K, int splits) {
  return splits > 1 ? sizeof(float) * (size_t)splits * ((size_t)K + 1) * (size_t)R : 0;
}

// Vectors per thread and vector chunks of the many-vector kernels: the
// fewest chunks of at most 16 * max_vt vectors, then the smallest
// vectors-per-thread count that covers a chunk.
void apply_vt_chunks(int d, int K, int* vt, int* chunks) {
  const int vm = d > 64 ? 4 : 5;
  const int c0 = (K + 16 * vm - 1) / (16 * vm);
  const int per = (K + c0 - 1) / c0;
  *vt = std::min((per + 15) / 16, vm);
  *chunks = (K + 16 * *vt - 1) / (16 * *vt);
}

// Byte offsets of the pipelined kernel's prepared operands, which follow
// the split partials in the workspace (256-byte aligned).
struct PrepLayout {
  size_t cen = 0, bt = 0, wbv = 0, vt = 0, total = 0;
  int64_t c_pad = 0, k_pad = 0;
};

inline size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// Prepared operands for d <= 64: every vector count (the one- and two-vector
// register path included).
bool pipelined_path(int d, int K) { return d <= 64 && K >= 1; }

PrepLayout prep_layout(int64_t C, int d, int K, size_t base) {
  PrepLayout L;
  int vt = 1, chunks = 1;
  apply_vt_chunks(d, K, &vt, &chunks);
  const int dp = d <= 8 ? 8 : d <= 16 ? 16 : d <= 32 ? 32 : 64;
  L.c_pad = (C + kTC - 1) / kTC * kTC;
  // [c_pad][k_pad] for the many-vector kernel; [K][c_pad] on the register path
  L.k_pad = K <= 2 ? K : (int64_t)chunks * 16 * vt;
  size_t off = align256(base);
  L.cen = off;
  off = align256(off + sizeof(float) * 64);
  L.bt = off;
  off = align256(off + sizeof(float) * (size_t)dp * L.c_pad);
  L.wbv = off;
  off = align256(off + sizeof(float) * L.c_pad);
  L.vt = off;
  off = align256(off + sizeof(float) * (size_t)L.c_pad * L.k_pad);
  L.total = off;
  return L;
}

int device_sms() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 148;
  return sms > 0 ? sms : 148;
}

template <int DP, int VT>
int launch_pipelined_vt(const ApplyArgs& a, int chunks, cudaStream_t stream) {
  const size_t smem = sizeof(PipeSmem<DP, VT>);
  auto k = apply_pipelined_kernel<DP, VT>;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return OTTB_ERR_CUDA;
  if (!a.prepared) {
    apply_prep_center_kernel<<<DP, 256, 0, stream>>>(a);
    const int64_t tot = (int64_t)DP * a.c_pad;
    apply_prep_b_kernel<<<(unsigned)std::min<int64_t>((tot + 255) / 256, 4096), 256, 0,
                          stream>>>(a, DP);
  }
  {
    dim3 grid((unsigned)(a.c_pad / 32), (unsigned)((a.k_pad + 31) / 32));
    apply_prep_v_kernel<<<grid, 256, 0, stream>>>(a);
  }
  dim3 grid((unsigned)((a.R + kTR - 1) / kTR), (unsigned)chunks, (unsigned)a.splits);
  k<<<grid, 256, smem, stream>>>(a);
  if (a.splits > 1) {
    const int64_t total = (int64_t)a.K * a.R;
    combine_splits_kernel<<<(unsigned)std::min<int64_t>((total + 255) / 256, 4096), 256, 0,
                            stream>>>(a);
  }
  return cudaGetLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}

template <int DP>
int launch_apply(const ApplyArgs& a, cudaStream_t stream) {
  if (a.K == 1) return launch_direct<DP, 1>(a, stream);
  if (a.K == 2) return launch_direct<DP, 2>(a, stream);
  int vt = 1, chunks = 1;
  apply_vt_chunks(a.d, a.K, &vt, &chunks);
  if constexpr (DP <= 64) {
    if (a.bt) {
      switch (vt) {
        case 1: return launch_pipelined_vt<DP, 1>(a, chunks, stream);
        case 2: return launch_pipelined_vt<DP, 2>(a, chunks, stream);
        case 3: return launch_pipelined_vt<DP, 3>(a, chunks, stream);
        case 4: return launch_pipelined_vt<DP, 4>(a, chunks, stream);
        default: return launch_pipelined_vt<DP, 5>(a, chunks, stream);
      }
    }
  }
  switch (vt) {
    case 1: return launch_apply_vt<DP, 1>(a, chunks, stream);
    case 2: return launch_apply_vt<DP, 2>(a, chunks, stream);
    case 3: return launch_apply_vt<DP, 3>(a, chunks, stream);
    case 4: return launch_apply_vt<DP, 4>(a, chunks, stream);
    default: return launch_apply_vt<DP, (max_vt<DP>() > 4 ? 5 : 4)>(a, chunks, stream);
  }
}

}  // namespace
}  // namespace ottb

using namespace ottb;

extern "C" size_t ottb_apply_transport_workspace_size(int64_t n, int64_t m, int32_t d,
                                                     int32_t num_vec, int32_t axis) {
  if (n < 1 || m < 1 || d < 1 || d > 128 || num_vec < 1 || (axis != 0 && axis != 1)) return 0;
  const int64_t R = axis == 1 ? n : m, C = axis == 1 ? m : n;
  const size_t part = apply_workspace(R, num_vec, apply_splits(R, C, d, num_vec, device_sms()));
  return pipelined_path(d, num_vec) ? prep_layout(C, d, num_vec, part).total : part;
}

namespace {

// The launch arguments of one call (vec and out left to the caller).
int make_apply_args(const float* x, const float* y, int64_t n, int64_t m, int32_t d,
                    const float* f, const float* g, float epsilon, float inv_scale_cost,
                    int32_t num_vec, int32_t axis, void* workspace, size_t workspace_bytes,
                    ApplyArgs& a) {
  if (!x || !y || !f || !g || n < 1 || m < 1 || d < 1 || num_vec < 1) return OTTB_ERR_INVALID;
  if (axis != 0 && axis != 1) return OTTB_ERR_INVALID;
  if (!(epsilon > 0.f) || !(inv_scale_cost > 0.f)) return OTTB_ERR_INVALID;
  if (d > 128) return OTTB_ERR_UNSUPPORTED;
  a.A = axis == 1 ? x : y;
  a.B = axis == 1 ? y : x;
  a.potA = axis == 1 ? f : g;
  a.potB = axis == 1 ? g : f;
  a.R = axis == 1 ? n : m;
  a.C = axis == 1 ? m : n;
  a.vec = nullptr;
  a.out = nullptr;
  a.d = d;
  a.K = num_vec;
  a.ws = (float)(kLog2eD / (double)epsilon);
  a.inv = inv_scale_cost;
  // as many column splits as wanted and as the workspace holds
  a.splits = apply_splits(a.R, a.C, d, num_vec, device_sms());
  while (a.splits > 1 && (!workspace || apply_workspace(a.R, num_vec, a.splits) > workspace_bytes))
    --a.splits;
  a.part_o = (float*)workspace;
  a.part_m = a.splits > 1 ? a.part_o + (size_t)a.splits * num_vec * a.R : nullptr;
  a.cen = a.bt = a.wbv = a.vt = nullptr;
  a.c_pad = a.k_pad = 0;
  a.prepared = 0;
  if (pipelined_path(d, num_vec) && workspace) {
    // the prepared operands after the partials, when the workspace holds them
    const PrepLayout L = prep_layout(a.C, d, num_vec, apply_workspace(a.R, num_vec, a.splits));
    if (L.total <= workspace_bytes && ((uintptr_t)workspace) % 256 == 0) {
      char* w = (char*)workspace;
      a.cen = (float*)(w + L.cen);
      a.bt = (float*)(w + L.bt);
      a.wbv = (float*)(w + L.wbv);
      a.vt = (float*)(w + L.vt);
      a.c_pad = L.c_pad;
      a.k_pad = L.k_pad;
    }
  }
  return OTTB_OK;
}

int run_apply(const ApplyArgs& a, cudaStream_t s) {
  if (a.d <= 8) return launch_apply<8>(a, s);
  if (a.d <= 16) return launch_apply<16>(a, s);
  if (a.d <= 32) return launch_apply<32>(a, s);
  if (a.d <= 64) return launch_apply<64>(a, s);
  return launch_apply<128>(a, s);
}

}  // namespace

extern "C" int32_t ottb_apply_transport(const float* x, const float* y, int64_t n, int64_t m,
                                        int32_t d, const float* f, const float* g,
                                        float epsilon, float inv_scale_cost, const float* vec,
                                        int32_t num_vec, int32_t axis, float* out,
                                        void* workspace, size_t workspace_bytes,
                                        void* stream) {
  if (!vec || !out) return OTTB_ERR_INVALID;
  ApplyArgs a;
  const int st = make_apply_args(x, y, n, m, d, f, g, epsilon, inv_scale_cost, num_vec, axis,
                                 workspace, workspace_bytes, a);
  if (st != OTTB_OK) return st;
  a.vec = vec;
  a.out = out;
  return run_apply(a, (cudaStream_t)stream);
}

// A product planned once (ottb_apply_transport_plan) and run many times.
struct ottb_apply_product {
  ApplyArgs a;
};

extern "C" int32_t ottb_apply_transport_plan(const float* x, const float* y, int64_t n,
                                             int64_t m, int32_t d, const float* f,
                                             const float* g, float epsilon,
                                             float inv_scale_cost, int32_t num_vec,
                                             int32_t axis, void* workspace,
                                             size_t workspace_bytes, void* stream,
                                             ottb_apply_product** product) {
  if (!product) return OTTB_ERR_INVALID;
  *product = nullptr;
  ApplyArgs a;
  const int st = make_apply_args(x, y, n, m, d, f, g, epsilon, inv_scale_cost, num_vec, axis,
                                 workspace, workspace_bytes, a);
  if (st != OTTB_OK) return st;
  // the handle first, so that nothing is enqueued for a plan that cannot be kept
  ottb_apply_product* h = new (std::nothrow) ottb_apply_product;
  if (!h) return OTTB_ERR_HOST_MEMORY;
  if (a.bt) {
    // the centre, B transposed and the column terms, once (d <= 64 here)
    const int dp = d <= 8 ? 8 : d <= 16 ? 16 : d <= 32 ? 32 : 64;
    cudaStream_t s = (cudaStream_t)stream;
    (void)cudaGetLastError();  // clear an error left by earlier, unrelated work
    apply_prep_center_kernel<<<dp, 256, 0, s>>>(a);
    const int64_t tot = (int64_t)dp * a.c_pad;
    apply_prep_b_kernel<<<(unsigned)std::min<int64_t>((tot + 255) / 256, 4096), 256, 0, s>>>(
        a, dp);
    if (cudaGetLastError() != cudaSuccess) {
      delete h;
      return OTTB_ERR_CUDA;
    }
    a.prepared = 1;
  }
  h->a = a;
  *product = h;
  return OTTB_OK;
}

extern "C" int32_t ottb_apply_transport_run(const ottb_apply_product* product,
                                            const float* vec, float* out, void* stream) {
  if (!product || !vec || !out) return OTTB_ERR_INVALID;
  ApplyArgs a = product->a;
  a.vec = vec;
  a.out = out;
  return run_apply(a, (cudaStream_t)stream);
}

extern "C" void ottb_apply_transport_free(ottb_apply_product* product) { delete product; }

extern "C" int32_t ottb_transport_matrix(const float* x, const float* y, int64_t n, int64_t m,
                                         int32_t d, const float* f, const float* g,
                                         float epsilon, float inv_scale_cost, float* out,
                                         void* stream) {
  if (!x || !y || !f || !g || !out || n < 1 || m < 1 || d < 1) return OTTB_ERR_INVALID;
  if (!(epsilon > 0.f) || !(inv_scale_cost > 0.f)) return OTTB_ERR_INVALID;
  if (d > 128) return OTTB_ERR_UNSUPPORTED;
  dim3 grid((unsigned)((m + 31) / 32), (unsigned)((n + 31) / 32));
  transport_matrix_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(
      x, y, n, m, d, f, g, epsilon, inv_scale_cost, out);
  return cudaGetLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}
