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
// running sum once. P is never written to global memory.
#include <cuda_runtime.h>

#include "../../include/ott_b200.h"
#include "common.cuh"

namespace ottb {
namespace {

constexpr int kTR = 128;   // output rows per CTA
constexpr int kTC = 128;   // B points per tile
constexpr int kKT = 64;    // vectors per CTA
constexpr int kSampleMax = 256;

// Rows of the shared tiles are padded by 4 floats (16-byte reads stay
// aligned, stores spread over 8 banks instead of 1) where it fits: at
// DP = 128 the unpadded tiles already take 224 KB.
template <int DP>
struct ApplySmem {
  static constexpr int kPad = DP <= 64 ? 4 : 0;
  float As[DP][kTR + kPad];   // A tile, transposed, centred
  float Bs[DP][kTC + kPad];   // B tile, transposed, centred
  float Ps[kTC][kTR + kPad];  // weights of the tile, [column][row]
  float Vs[kTC][kKT + kPad];  // vectors of the tile, [column][k]
  float wb[kTC];              // (potB - inv |B|^2) * log2e / eps
  float center[DP];
};

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
};

// Common centre of both point sets: the mean of up to kSampleMax points of
// each, taken at a fixed stride (every CTA computes the same value).
template <int DP>
__device__ void apply_center(const ApplyArgs& p, float* center) {
  for (int k = threadIdx.x; k < DP; k += blockDim.x) {
    float s = 0.f;
    if (k < p.d) {
      const int64_t na = p.R < kSampleMax ? p.R : kSampleMax;
      const int64_t nb = p.C < kSampleMax ? p.C : kSampleMax;
      const int64_t sa = p.R / na, sb = p.C / nb;
      float ma = 0.f, mb = 0.f;
      for (int64_t i = 0; i < na; ++i) ma += p.A[i * sa * p.d + k];
      for (int64_t i = 0; i < nb; ++i) mb += p.B[i * sb * p.d + k];
      s = 0.5f * (ma / (float)na + mb / (float)nb);
    }
    center[k] = s;
  }
}

template <int DP>
__global__ void __launch_bounds__(256, 1) apply_transport_kernel(ApplyArgs p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ApplySmem<DP>& sm = *reinterpret_cast<ApplySmem<DP>*>(smem_raw);
  const int tid = threadIdx.x;
  const int tx = tid & 15;
  const int ty = tid >> 4;
  const int64_t row0 = (int64_t)blockIdx.x * kTR;
  const int k0 = blockIdx.y * kKT;
  const float s = 2.f * p.inv * p.ws;

  apply_center<DP>(p, sm.center);
  __syncthreads();
  // A tile (rows beyond R are zero points with potential -inf)
  for (int idx = tid; idx < DP * kTR; idx += blockDim.x) {
    const int r = idx / DP, k = idx % DP;
    const int64_t gr = row0 + r;
    sm.As[k][r] = (gr < p.R && k < p.d) ? p.A[gr * p.d + k] - sm.center[k] : 0.f;
  }
  __syncthreads();
  // row terms u_r = (potA_r - inv |A_r|^2) * ws of this thread's 8 rows
  float u[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = (i < 4) ? (ty * 4 + i) : (64 + ty * 4 + (i - 4));
    const int64_t gr = row0 + r;
    float nrm = 0.f;
    for (int k = 0; k < DP; ++k) nrm = fmaf(sm.As[k][r], sm.As[k][r], nrm);
    u[i] = gr < p.R ? (__ldg(p.potA + gr) - p.inv * nrm) * p.ws : -INFINITY;
  }

  float mrow[8];
  float o[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    mrow[i] = kNegSentinel;
#pragma unroll
    for (int j = 0; j < 4; ++j) o[i][j] = 0.f;
  }

  const int64_t ntiles = (p.C + kTC - 1) / kTC;
  for (int64_t t = 0; t < ntiles; ++t) {
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

    // exponents of the 8 x 8 micro-tile
    float z[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 8; ++j) z[i][j] = 0.f;
#pragma unroll 4
    for (int k = 0; k < DP; ++k) {
      const float4 a0 = *reinterpret_cast<const float4*>(&sm.As[k][ty * 4]);
      const float4 a1 = *reinterpret_cast<const float4*>(&sm.As[k][64 + ty * 4]);
      const float4 b0 = *reinterpret_cast<const float4*>(&sm.Bs[k][tx * 4]);
      const float4 b1 = *reinterpret_cast<const float4*>(&sm.Bs[k][64 + tx * 4]);
      const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
      const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) z[i][j] = fmaf(av[i], bv[j], z[i][j]);
    }
    {
      const float4 w0 = *reinterpret_cast<const float4*>(&sm.wb[tx * 4]);
      const float4 w1 = *reinterpret_cast<const float4*>(&sm.wb[64 + tx * 4]);
      const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) z[i][j] = fmaf(z[i][j], s, wv[j]) + u[i];
    }
    // row maxima over the tile (16 threads share a row), rescale the sums
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
        for (int j = 0; j < 4; ++j) o[i][j] *= sc;
        mrow[i] = mx;
      }
      const int r = (i < 4) ? (ty * 4 + i) : (64 + ty * 4 + (i - 4));
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int c = (j < 4) ? (tx * 4 + j) : (64 + tx * 4 + (j - 4));
        sm.Ps[c][r] = ex2_approx(z[i][j] - mrow[i]);
      }
    }
    __syncthreads();
    // O[r][k] += sum_c P[r][c] V[c][k]: rows of this thread's micro-tile,
    // vectors tx * 4 .. tx * 4 + 3
    float acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
#pragma unroll 4
    for (int c = 0; c < kTC; ++c) {
      const float4 p0 = *reinterpret_cast<const float4*>(&sm.Ps[c][ty * 4]);
      const float4 p1 = *reinterpret_cast<const float4*>(&sm.Ps[c][64 + ty * 4]);
      const float4 v = *reinterpret_cast<const float4*>(&sm.Vs[c][tx * 4]);
      const float pv[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
      const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(pv[i], vv[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) o[i][j] += acc[i][j];
  }

  // out = O * 2^max (a row whose weights are all zero gives 0)
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = (i < 4) ? (ty * 4 + i) : (64 + ty * 4 + (i - 4));
    const int64_t gr = row0 + r;
    if (gr >= p.R) continue;
    const bool any = mrow[i] > kNegSentinel;
    const float scale = any ? exp2f(mrow[i]) : 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int k = k0 + tx * 4 + j;
      if (k < p.K) p.out[(int64_t)k * p.R + gr] = any ? o[i][j] * scale : 0.f;
    }
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

template <int DP>
int launch_apply(const ApplyArgs& a, cudaStream_t stream) {
  const size_t smem = sizeof(ApplySmem<DP>);
  auto k = apply_transport_kernel<DP>;
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return OTTB_ERR_CUDA;
  dim3 grid((unsigned)((a.R + kTR - 1) / kTR), (unsigned)((a.K + kKT - 1) / kKT));
  k<<<grid, 256, smem, stream>>>(a);
  return cudaGetLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}

}  // namespace
}  // namespace ottb

using namespace ottb;

extern "C" int32_t ottb_apply_transport(const float* x, const float* y, int64_t n, int64_t m,
                                        int32_t d, const float* f, const float* g,
                                        float epsilon, float inv_scale_cost, const float* vec,
                                        int32_t num_vec, int32_t axis, float* out,
                                        void* stream) {
  if (!x || !y || !f || !g || !vec || !out || n < 1 || m < 1 || d < 1 || num_vec < 1)
    return OTTB_ERR_INVALID;
  if (axis != 0 && axis != 1) return OTTB_ERR_INVALID;
  if (!(epsilon > 0.f) || !(inv_scale_cost > 0.f)) return OTTB_ERR_INVALID;
  if (d > 128) return OTTB_ERR_UNSUPPORTED;
  ApplyArgs a;
  a.A = axis == 1 ? x : y;
  a.B = axis == 1 ? y : x;
  a.potA = axis == 1 ? f : g;
  a.potB = axis == 1 ? g : f;
  a.R = axis == 1 ? n : m;
  a.C = axis == 1 ? m : n;
  a.vec = vec;
  a.out = out;
  a.d = d;
  a.K = num_vec;
  a.ws = (float)(kLog2eD / (double)epsilon);
  a.inv = inv_scale_cost;
  cudaStream_t s = (cudaStream_t)stream;
  if (d <= 8) return launch_apply<8>(a, s);
  if (d <= 16) return launch_apply<16>(a, s);
  if (d <= 32) return launch_apply<32>(a, s);
  if (d <= 64) return launch_apply<64>(a, s);
  return launch_apply<128>(a, s);
}

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
