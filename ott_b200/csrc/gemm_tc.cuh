// BF16 GEMM on tcgen05 for the learned initializer's MLP:
//   D[M, N] = A[M, K] * B[N, K]^T  (A and B bf16, K contiguous; FP32 in TMEM)
// with the epilogues the MLP needs fused in:
//   kEpiHidden   Z = D + bias (bf16), H = GELU(Z) (bf16, row-major and
//                transposed)
//   kEpiOutput   Y = D + bias (fp32)
//   kEpiBackHid  dZ = D * GELU'(Zprev) (bf16, row-major and transposed)
//   kEpiWeight   G = D (fp32, weight gradient)
// One CTA per 128 x TN tile of D (TN = 128, 64 or 32; M a multiple of 128,
// N of TN, K of 64): the narrower tiles give small GEMMs (the batch-512
// layers: 32 tiles of 128 x 128 for 148 SMs) more CTAs. Warp 0 issues TMA
// loads of 64-wide K slabs of A and B through a 4-stage ring, warp 1 the
// MMAs (M = 128, N = TN, K = 16) into one TMEM accumulator, warps 2-5 read
// it back (warp w: TMEM lanes 32*(w%4)..) and run the epilogue, staging
// their rows in shared memory so the row-major outputs leave as whole rows.
// Waits are bounded; on a timeout the CTA sets *err and returns after
// draining.
#pragma once

#include <cuda_bf16.h>

#include "tc_ptx.cuh"

namespace ottb {

enum GemmEpi : int { kEpiHidden = 0, kEpiOutput = 1, kEpiBackHid = 2, kEpiWeight = 3 };

struct GemmArgs {
  int M, N, K;
  int epi;
  const float* bias;          // [N] (kEpiHidden, kEpiOutput)
  __nv_bfloat16* out_z;       // [M, N] pre-activation (kEpiHidden)
  __nv_bfloat16* out_h;       // [M, N] activation or dZ
  __nv_bfloat16* out_ht;      // [N, M] its transpose
  const __nv_bfloat16* zprev; // [M, N] pre-activation of the layer below (kEpiBackHid)
  float* out_f32;             // [M, N] (kEpiOutput, kEpiWeight)
  int* err;
  uint64_t timeout_ns;
};

constexpr int kGemmStages = 4;
constexpr int kGemmSlabBytes = 128 * 64 * 2;  // one [128][64] bf16 slab, 128-byte swizzle

// Epilogue staging, per epilogue warp (its 32 rows of the tile): an fp32
// [32][TN + 1] tile or two bf16-pair [32][TN / 2 + 1] tiles (the odd
// strides keep a warp's row-per-lane writes free of bank conflicts),
// written out as whole rows so every global store of a warp is contiguous.
template <int TN>
struct GemmSmem {
  static constexpr int kEpiWords = 32 * (TN + 2);
  uint8_t A[kGemmStages][kGemmSlabBytes];
  uint8_t B[kGemmStages][TN * 64 * 2];
  uint32_t epi[4][kEpiWords];
  uint64_t full[kGemmStages];
  uint64_t empty[kGemmStages];
  uint64_t done;
  uint32_t tmem_base;
  int err;
};

// tanh-form GELU, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), and its
// derivative.
__device__ __forceinline__ float gelu_tanh(float z) {
  const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
  return 0.5f * z * (1.0f + tanhf(u));
}
__device__ __forceinline__ float gelu_tanh_grad(float z) {
  const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
  const float t = tanhf(u);
  const float du = 0.7978845608028654f * (1.0f + 3.0f * 0.044715f * z * z);
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * du;
}

template <int TN>
__global__ void __launch_bounds__(192, 1)
gemm_bf16_tc_kernel(const __grid_constant__ CUtensorMap mapA,
                    const __grid_constant__ CUtensorMap mapB, GemmArgs g) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t base = tc::smem_u32(smem_raw);
  GemmSmem<TN>& sm =
      *reinterpret_cast<GemmSmem<TN>*>(smem_raw + ((1024u - (base & 1023u)) & 1023u));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * 128, n0 = blockIdx.x * TN;
  const int ksteps = g.K / 64;
  constexpr uint32_t kIdesc = tc::idesc_bf16_f32(128, TN);
  constexpr int S1 = TN / 2 + 1;  // bf16-pair staging stride (words)
  constexpr int SF = TN + 1;      // fp32 staging stride

  if (threadIdx.x == 0) {
    for (int i = 0; i < kGemmStages; ++i) {
      tc::mbar_init(&sm.full[i], 1);
      tc::mbar_init(&sm.empty[i], 1);
    }
    tc::mbar_init(&sm.done, 1);
    sm.err = 0;
    tc::fence_barrier_init();
  }
  if (warp == 1) {
    tc::tmem_alloc(&sm.tmem_base, TN);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();

  bool ok = true;
  if (warp == 0) {
    if (lane == 0) {
      for (int k = 0; k < ksteps; ++k) {
        const int st = k % kGemmStages;
        if (!tc::mbar_wait(&sm.empty[st], ((k / kGemmStages) & 1) ^ 1, g.timeout_ns)) {
          ok = false;
          break;
        }
        tc::mbar_arrive_expect_tx(&sm.full[st], kGemmSlabBytes + TN * 64 * 2);
        tc::tma_load_2d(sm.A[st], &mapA, &sm.full[st], 64 * k, m0);
        tc::tma_load_2d(sm.B[st], &mapB, &sm.full[st], 64 * k, n0);
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      for (int k = 0; k < ksteps; ++k) {
        const int st = k % kGemmStages;
        if (!tc::mbar_wait(&sm.full[st], (k / kGemmStages) & 1, g.timeout_ns)) {
          ok = false;
          break;
        }
        tc::fence_after_sync();
        const uint32_t a0 = tc::smem_u32(sm.A[st]), b0 = tc::smem_u32(sm.B[st]);
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
          tc::mma_bf16(sm.tmem_base, tc::sw128_kmajor_desc(a0 + 32 * kk),
                       tc::sw128_kmajor_desc(b0 + 32 * kk), kIdesc, (k | kk) ? 1u : 0u);
        tc::mma_commit(&sm.empty[st]);
      }
      tc::mma_commit(&sm.done);  // also issued after a timeout: drains the MMAs
    }
    __syncwarp();
  } else {
    // epilogue: row r of the tile (this warp's 32 rows, one per lane), 128
    // columns in 4 chunks of 32 from TMEM into the warp's staging tile,
    // then out by whole rows (the transposed outputs go straight out: a
    // column of the tile is contiguous there)
    const int q = warp & 3;
    const int r = 32 * q + lane;
    const int row = m0 + r;
    uint32_t* st = sm.epi[q];
    float* sf = reinterpret_cast<float*>(st);           // fp32 [32][TN + 1]
    uint32_t* s0 = st;                                   // bf16 pairs [32][TN / 2 + 1]
    uint32_t* s1 = st + 32 * S1;                         // bf16 pairs [32][TN / 2 + 1]
    if (!tc::mbar_wait(&sm.done, 0, g.timeout_ns)) ok = false;
    if (ok) {
      tc::fence_after_sync();
      if (g.epi == kEpiBackHid) {
        // the layer below's pre-activations of these rows, read as whole rows
        for (int i = 0; i < 32; ++i) {
          const uint32_t* src =
              reinterpret_cast<const uint32_t*>(g.zprev + (int64_t)(m0 + 32 * q + i) * g.N + n0);
          for (int w = lane; w < TN / 2; w += 32) s1[i * S1 + w] = src[w];
        }
        __syncwarp();
      }
      for (int c0 = 0; c0 < TN; c0 += 32) {
        float v[32];
        tc::tmem_ld32(sm.tmem_base + ((uint32_t)(32 * q) << 16) + c0, v);
        tc::tmem_ld_wait();
        const int col0 = n0 + c0;
        if (g.epi == kEpiHidden) {
#pragma unroll
          for (int j = 0; j < 32; j += 2) {
            const float z0 = v[j] + g.bias[col0 + j];
            const float z1 = v[j + 1] + g.bias[col0 + j + 1];
            const __nv_bfloat16 zb0 = __float2bfloat16_rn(z0), zb1 = __float2bfloat16_rn(z1);
            const __nv_bfloat16 hb0 = __float2bfloat16_rn(gelu_tanh(__bfloat162float(zb0)));
            const __nv_bfloat16 hb1 = __float2bfloat16_rn(gelu_tanh(__bfloat162float(zb1)));
            s0[lane * S1 + (c0 + j) / 2] =
                (uint32_t)__bfloat16_as_ushort(zb0) | ((uint32_t)__bfloat16_as_ushort(zb1) << 16);
            s1[lane * S1 + (c0 + j) / 2] =
                (uint32_t)__bfloat16_as_ushort(hb0) | ((uint32_t)__bfloat16_as_ushort(hb1) << 16);
            g.out_ht[(int64_t)(col0 + j) * g.M + row] = hb0;
            g.out_ht[(int64_t)(col0 + j + 1) * g.M + row] = hb1;
          }
        } else if (g.epi == kEpiBackHid) {
#pragma unroll
          for (int j = 0; j < 32; j += 2) {
            const uint32_t zw = s1[lane * S1 + (c0 + j) / 2];
            const float za = __bfloat162float(__ushort_as_bfloat16((unsigned short)(zw & 0xffffu)));
            const float zc = __bfloat162float(__ushort_as_bfloat16((unsigned short)(zw >> 16)));
            const __nv_bfloat16 d0 = __float2bfloat16_rn(v[j] * gelu_tanh_grad(za));
            const __nv_bfloat16 d1 = __float2bfloat16_rn(v[j + 1] * gelu_tanh_grad(zc));
            s0[lane * S1 + (c0 + j) / 2] =
                (uint32_t)__bfloat16_as_ushort(d0) | ((uint32_t)__bfloat16_as_ushort(d1) << 16);
            g.out_ht[(int64_t)(col0 + j) * g.M + row] = d0;
            g.out_ht[(int64_t)(col0 + j + 1) * g.M + row] = d1;
          }
        } else {
          const bool bias = g.epi == kEpiOutput;
#pragma unroll
          for (int j = 0; j < 32; ++j) sf[lane * SF + c0 + j] = v[j] + (bias ? g.bias[col0 + j] : 0.f);
        }
      }
      __syncwarp();
      // whole rows out: a warp store covers 32 consecutive words of a row
      // (bf16 pairs or floats), conflict-free shared-memory reads
      for (int i = 0; i < 32; ++i) {
        const int64_t grow = (int64_t)(m0 + 32 * q + i);
        if (g.epi == kEpiHidden) {
          uint32_t* dz = reinterpret_cast<uint32_t*>(g.out_z + grow * g.N + n0);
          uint32_t* dh = reinterpret_cast<uint32_t*>(g.out_h + grow * g.N + n0);
          for (int w = lane; w < TN / 2; w += 32) {
            dz[w] = s0[i * S1 + w];
            dh[w] = s1[i * S1 + w];
          }
        } else if (g.epi == kEpiBackHid) {
          uint32_t* dh = reinterpret_cast<uint32_t*>(g.out_h + grow * g.N + n0);
          for (int w = lane; w < TN / 2; w += 32) dh[w] = s0[i * S1 + w];
        } else {
          float* d = g.out_f32 + grow * g.N + n0;
#pragma unroll
          for (int k = 0; k < TN / 32; ++k) d[32 * k + lane] = sf[i * SF + 32 * k + lane];
        }
      }
    }
  }
  if (!ok) atomicExch(&sm.err, 1);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 1) {
    // after a timeout the MMA thread's final commit may not have landed yet
    if (sm.err && lane == 0) tc::mbar_wait(&sm.done, 0, 1000000000ull);
    __syncwarp();
    tc::fence_after_sync();
    tc::tmem_dealloc(sm.tmem_base, TN);
  }
  if (threadIdx.x == 0 && sm.err) atomicExch(g.err, 1);
}

// Column sums of a [rows, cols] bf16 matrix (bias gradients): out[c] =
// sum_r in[r, c]. One CTA of 8 warps per 64 columns: lane l of warp w sums
// columns 2l, 2l + 1 (one 4-byte pair) over rows w, w + 8, ..., eight loads
// in flight; the warps' sums are then added in a fixed order. cols must be
// even (the MLP's widths are multiples of 128).
__global__ void __launch_bounds__(256) colsum_bf16_kernel(const __nv_bfloat16* in, int rows,
                                                          int cols, float* out) {
  __shared__ float2 part[8][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = blockIdx.x * 64 + 2 * lane;
  float2 s = make_float2(0.f, 0.f);
  if (c < cols) {
    const __nv_bfloat162* src = reinterpret_cast<const __nv_bfloat162*>(in + c);
    const int64_t stride = cols / 2;  // bf16 pairs per row
    int r = warp;
    for (; r + 56 < rows; r += 64) {
      __nv_bfloat162 v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = src[(int64_t)(r + 8 * u) * stride];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        s.x += __low2float(v[u]);
        s.y += __high2float(v[u]);
      }
    }
    for (; r < rows; r += 8) {
      const __nv_bfloat162 v = src[(int64_t)r * stride];
      s.x += __low2float(v);
      s.y += __high2float(v);
    }
  }
  part[warp][lane] = s;
  __syncthreads();
  if (warp == 0 && c < cols) {
    float2 t = part[0][lane];
    for (int w = 1; w < 8; ++w) {
      t.x += part[w][lane].x;
      t.y += part[w][lane].y;
    }
    out[c] = t.x;
    out[c + 1] = t.y;
  }
}

// Centred squared error per sample, optionally weighted:
//   loss_b = sum_j w_j ((y_j - t_j) - s)^2 / sum_j w_j,
//   s = sum_j w_j (y_j - t_j) / sum_j w_j
// (potentials are defined up to a constant, so only the best-aligned
// difference is penalised; w = 1 when weight is null). The residual
// r = y - t - s has zero weighted mean, so d loss_b / d y_j = 2 w_j r_j /
// sum w; dY (that over the batch size) goes out as bf16, row-major and
// transposed, for the backward GEMMs. One CTA per sample, blockDim a
// multiple of 32 up to 1024.
__device__ __forceinline__ float block_sum_f32(float v, float* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float tot = 0.f;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) tot += red[i];
  return tot;
}

__global__ void centred_mse_kernel(const float* y, const float* t, const float* weight,
                                   int batch, int m, __nv_bfloat16* dy, __nv_bfloat16* dyt,
                                   float* loss_per) {
  __shared__ float red[32];
  const int b = blockIdx.x;
  const float* yb = y + (int64_t)b * m;
  const float* tb = t + (int64_t)b * m;
  const float* wb = weight ? weight + (int64_t)b * m : nullptr;
  float s = 0.f, sw = 0.f;
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    const float w = wb ? wb[j] : 1.f;
    s += w * (yb[j] - tb[j]);
    sw += w;
  }
  const float wsum = block_sum_f32(sw, red);
  const float shift = block_sum_f32(s, red) / wsum;
  float l = 0.f;
  const float scale = 2.0f / (wsum * (float)batch);
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    const float w = wb ? wb[j] : 1.f;
    const float r = yb[j] - tb[j] - shift;
    l += w * r * r;
    const __nv_bfloat16 g = __float2bfloat16_rn(scale * w * r);
    dy[(int64_t)b * m + j] = g;
    dyt[(int64_t)j * batch + b] = g;
  }
  const float tot = block_sum_f32(l, red);
  if (threadIdx.x == 0) loss_per[b] = tot / wsum;
}

// Adam (Kingma & Ba) on FP32 master weights [rows, cols]; writes the bf16
// copies used by the GEMMs, row-major and transposed [cols, rows] (wt may
// be null, e.g. for biases). One CTA of 32 x 8 threads per 32 x 32 tile:
// the row-major arrays are read and written along rows, the transposed
// copy goes out through a shared-memory tile along its own rows. lr and the
// bias corrections c1 = 1 - beta1^t, c2 = 1 - beta2^t come from hyper (device,
// {lr, c1, c2}) when it is given, else from the arguments.
__global__ void __launch_bounds__(256) adam_kernel(float* w, float* mom, float* vel,
                                                   const float* grad, int rows, int cols,
                                                   float lr, float b1, float b2, float eps,
                                                   float c1, float c2, const float* hyper,
                                                   __nv_bfloat16* wb, __nv_bfloat16* wt) {
  __shared__ __nv_bfloat16 tile[32][34];
  if (hyper) {
    lr = hyper[0];
    c1 = hyper[1];
    c2 = hyper[2];
  }
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int r = r0 + ty + 8 * k, c = c0 + tx;
    if (r < rows && c < cols) {
      const int64_t i = (int64_t)r * cols + c;
      const float gr = grad[i];
      const float m1 = b1 * mom[i] + (1.f - b1) * gr;
      const float v1 = b2 * vel[i] + (1.f - b2) * gr * gr;
      mom[i] = m1;
      vel[i] = v1;
      const float nw = w[i] - lr * (m1 / c1) / (sqrtf(v1 / c2) + eps);
      w[i] = nw;
      const __nv_bfloat16 h = __float2bfloat16_rn(nw);
      if (wb) wb[i] = h;
      tile[ty + 8 * k][tx] = h;
    }
  }
  if (!wt) return;
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int c = c0 + ty + 8 * k, r = r0 + tx;
    if (r < rows && c < cols) wt[(int64_t)c * rows + r] = tile[tx][ty + 8 * k];
  }
}

// f32 -> bf16 (row-major and optionally transposed) for the network input.
__global__ void to_bf16_kernel(const float* in, int64_t rows, int cols, __nv_bfloat16* out,
                               __nv_bfloat16* outt) {
  const int64_t count = rows * cols;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x) {
    const __nv_bfloat16 h = __float2bfloat16_rn(in[i]);
    out[i] = h;
    if (outt) outt[(i % cols) * rows + i / cols] = h;
  }
}

}  // namespace ottb
