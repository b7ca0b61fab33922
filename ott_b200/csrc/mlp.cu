// C-ABI entry points of the learned initializer's MLP (declared in
// include/ott_b200.h): forward, gradients of the centred squared error, and
// Adam. Layers are Dense (y = x W^T + b) with tanh-GELU between them and a
// linear last layer, the shape of the meta model of
// initializers/neural/meta_initializer.py (flax Dense layers, optax Adam).
// All arithmetic is in the kernels of gemm_tc.cuh: bf16 operands, FP32
// accumulation, FP32 master weights. Nothing here allocates device memory.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/ott_b200.h"
#include "gemm_tc.cuh"
#include "launch.cuh"
#include "tmap.cuh"

using namespace ottb;

namespace {

constexpr size_t kAlign = 256;
inline size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// [rows][cols] bf16, K = cols contiguous: boxes of 64 x box_rows, 128-byte swizzle.
bool operand_map(CUtensorMap* map, const void* base, int64_t rows, int64_t cols,
                 uint32_t box_rows = 128) {
  return encode_bf16_2d(map, const_cast<void*>(base), rows, cols, 64, box_rows,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B);
}

template <int TN>
size_t gemm_smem() { return sizeof(GemmSmem<TN>) + 1024; }

template <int TN>
int launch_gemm(const CUtensorMap& ma, const CUtensorMap& mb, const GemmArgs& g,
                cudaStream_t stream) {
  if (!ensure_dynamic_smem((const void*)gemm_bf16_tc_kernel<TN>, gemm_smem<TN>()))
    return OTTB_ERR_CUDA;
  gemm_bf16_tc_kernel<TN><<<dim3(g.N / TN, g.M / 128), 192, gemm_smem<TN>(), stream>>>(ma, mb, g);
  return cudaGetLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}

// D[M, N] = A[M, K] B[N, K]^T with the given epilogue. The tile width is
// the widest of 128, 64, 32 columns that still gives 96 or more CTAs (all
// three when M N is small), since one 128 x 128 tile per CTA leaves most
// of the 148 SMs idle on the batch-512 layers.
int gemm(const void* A, const void* B, GemmArgs g, cudaStream_t stream) {
  if (g.M % 128 || g.N % 128 || g.K % 64 || g.K < 64) return OTTB_ERR_UNSUPPORTED;
  const int64_t tiles128 = (int64_t)(g.M / 128) * (g.N / 128);
  const int tn = tiles128 >= 96 ? 128 : tiles128 * 2 >= 96 ? 64 : 32;
  CUtensorMap ma, mb;
  if (!operand_map(&ma, A, g.M, g.K) || !operand_map(&mb, B, g.N, g.K, (uint32_t)tn))
    return OTTB_ERR_CUDA;
  if (tn == 128) return launch_gemm<128>(ma, mb, g, stream);
  if (tn == 64) return launch_gemm<64>(ma, mb, g, stream);
  return launch_gemm<32>(ma, mb, g, stream);
}

// Workspace layout of one batch: input, activations, gradients.
struct MlpPlan {
  int L = 0;
  int dims[OTTB_MLP_MAX_LAYERS + 1];
  size_t xb = 0, xbt = 0, z[OTTB_MLP_MAX_LAYERS], h[OTTB_MLP_MAX_LAYERS],
         ht[OTTB_MLP_MAX_LAYERS], y = 0, dy = 0, dyt = 0, dz[OTTB_MLP_MAX_LAYERS],
         dzt[OTTB_MLP_MAX_LAYERS], total = 0;
};

int plan_mlp(const ottb_mlp* net, int batch, MlpPlan& p) {
  if (!net || net->num_layers < 1 || net->num_layers > OTTB_MLP_MAX_LAYERS) return OTTB_ERR_INVALID;
  if (batch < 128 || batch % 128) return OTTB_ERR_UNSUPPORTED;
  p.L = net->num_layers;
  for (int l = 0; l < p.L; ++l) {
    const ottb_mlp_layer& ly = net->layers[l];
    if (ly.in < 1 || ly.out < 1) return OTTB_ERR_INVALID;
    if (ly.in % 128 || ly.out % 128) return OTTB_ERR_UNSUPPORTED;
    if (l > 0 && ly.in != net->layers[l - 1].out) return OTTB_ERR_INVALID;
    p.dims[l] = ly.in;
    p.dims[l + 1] = ly.out;
  }
  size_t off = 0;
  const size_t B = (size_t)batch;
  p.xb = off; off = align_up(off + 2 * B * p.dims[0]);
  p.xbt = off; off = align_up(off + 2 * B * p.dims[0]);
  for (int l = 0; l + 1 < p.L; ++l) {
    const size_t w = (size_t)p.dims[l + 1];
    p.z[l] = off; off = align_up(off + 2 * B * w);
    p.h[l] = off; off = align_up(off + 2 * B * w);
    p.ht[l] = off; off = align_up(off + 2 * B * w);
    p.dz[l] = off; off = align_up(off + 2 * B * w);
    p.dzt[l] = off; off = align_up(off + 2 * B * w);
  }
  const size_t o = (size_t)p.dims[p.L];
  p.y = off; off = align_up(off + 4 * B * o);
  p.dy = off; off = align_up(off + 2 * B * o);
  p.dyt = off; off = align_up(off + 2 * B * o);
  p.total = off;
  return OTTB_OK;
}

GemmArgs base_args(int M, int N, int K, int epi, int* status, int timeout_ms) {
  GemmArgs g;
  std::memset(&g, 0, sizeof(g));
  g.M = M;
  g.N = N;
  g.K = K;
  g.epi = epi;
  g.err = status;
  g.timeout_ns = (uint64_t)(timeout_ms > 0 ? timeout_ms : 10000) * 1000000ull;
  return g;
}

// Forward pass into the workspace; the output goes to ws + p.y (fp32).
int forward(const ottb_mlp* net, const float* x, int batch, char* ws, const MlpPlan& p,
            int* status, cudaStream_t stream) {
  const int L = p.L;
  const int64_t count = (int64_t)batch * p.dims[0];
  to_bf16_kernel<<<(unsigned)std::min<int64_t>((count + 255) / 256, 4096), 256, 0, stream>>>(
      x, batch, p.dims[0], (__nv_bfloat16*)(ws + p.xb), (__nv_bfloat16*)(ws + p.xbt));
  const void* in = ws + p.xb;
  for (int l = 0; l < L; ++l) {
    const ottb_mlp_layer& ly = net->layers[l];
    const bool last = l + 1 == L;
    GemmArgs g = base_args(batch, ly.out, ly.in, last ? kEpiOutput : kEpiHidden, status, 0);
    g.bias = ly.b;
    if (last) {
      g.out_f32 = (float*)(ws + p.y);
    } else {
      g.out_z = (__nv_bfloat16*)(ws + p.z[l]);
      g.out_h = (__nv_bfloat16*)(ws + p.h[l]);
      g.out_ht = (__nv_bfloat16*)(ws + p.ht[l]);
    }
    const int st = gemm(in, ly.w_bf16, g, stream);
    if (st != OTTB_OK) return st;
    in = ws + (last ? 0 : p.h[l]);
  }
  return OTTB_OK;
}

}  // namespace

extern "C" {

size_t ottb_mlp_workspace_size(const ottb_mlp* net, int32_t batch) {
  MlpPlan p;
  return plan_mlp(net, batch, p) == OTTB_OK ? p.total : 0;
}

int32_t ottb_mlp_forward(const ottb_mlp* net, const float* x, int32_t batch, float* y,
                         int32_t* status, void* workspace, size_t workspace_bytes,
                         void* stream_ptr) {
  MlpPlan p;
  int st = plan_mlp(net, batch, p);
  if (st != OTTB_OK) return st;
  if (!x || !y || !status) return OTTB_ERR_INVALID;
  if (!workspace || workspace_bytes < p.total) return OTTB_ERR_WORKSPACE;
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  char* ws = (char*)workspace;
  st = forward(net, x, batch, ws, p, status, stream);
  if (st != OTTB_OK) return st;
  const size_t bytes = 4 * (size_t)batch * p.dims[p.L];
  return cudaMemcpyAsync(y, ws + p.y, bytes, cudaMemcpyDeviceToDevice, stream) == cudaSuccess
             ? OTTB_OK
             : OTTB_ERR_CUDA;
}

int32_t ottb_mlp_gradients(const ottb_mlp* net, const float* x, const float* target,
                           const float* weight, int32_t batch, float* loss_per,
                           int32_t* status, void* workspace, size_t workspace_bytes,
                           void* stream_ptr) {
  MlpPlan p;
  int st = plan_mlp(net, batch, p);
  if (st != OTTB_OK) return st;
  if (!x || !target || !loss_per || !status) return OTTB_ERR_INVALID;
  for (int l = 0; l < p.L; ++l)
    if (!net->layers[l].w_grad || !net->layers[l].b_grad) return OTTB_ERR_INVALID;
  if (!workspace || workspace_bytes < p.total) return OTTB_ERR_WORKSPACE;
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  char* ws = (char*)workspace;
  st = forward(net, x, batch, ws, p, status, stream);
  if (st != OTTB_OK) return st;
  const int L = p.L;
  const int out = p.dims[L];
  centred_mse_kernel<<<batch, 256, 0, stream>>>((const float*)(ws + p.y), target, weight,
                                                batch, out,
                                                (__nv_bfloat16*)(ws + p.dy),
                                                (__nv_bfloat16*)(ws + p.dyt), loss_per);
  // walk back: dz_l (row-major) and dz_l^T for l = L-1 (the output) .. 0
  const void* dz = ws + p.dy;
  const void* dzt = ws + p.dyt;
  for (int l = L - 1; l >= 0; --l) {
    const ottb_mlp_layer& ly = net->layers[l];
    // dW_l[out, in] = dz_l^T [out, B] x act_{l-1}^T [in, B]^T
    const void* actt = l == 0 ? (const void*)(ws + p.xbt) : (const void*)(ws + p.ht[l - 1]);
    GemmArgs gw = base_args(ly.out, ly.in, batch, kEpiWeight, status, 0);
    gw.out_f32 = ly.w_grad;
    st = gemm(dzt, actt, gw, stream);
    if (st != OTTB_OK) return st;
    colsum_bf16_kernel<<<(ly.out + 63) / 64, 256, 0, stream>>>(
        (const __nv_bfloat16*)dz, batch, ly.out, ly.b_grad);
    if (l == 0) break;
    // dz_{l-1}[B, in] = (dz_l [B, out] x W_l^T ... as A B^T with B = W_l^T [in, out])
    //                   * GELU'(z_{l-1})
    GemmArgs gb = base_args(batch, ly.in, ly.out, kEpiBackHid, status, 0);
    gb.zprev = (const __nv_bfloat16*)(ws + p.z[l - 1]);
    gb.out_h = (__nv_bfloat16*)(ws + p.dz[l - 1]);
    gb.out_ht = (__nv_bfloat16*)(ws + p.dzt[l - 1]);
    st = gemm(dz, ly.wt_bf16, gb, stream);
    if (st != OTTB_OK) return st;
    dz = ws + p.dz[l - 1];
    dzt = ws + p.dzt[l - 1];
  }
  return cudaGetLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}

}  // extern "C"

namespace {

int adam_all(const ottb_mlp* net, float lr, float beta1, float beta2, float eps, float c1,
             float c2, const float* hyper, cudaStream_t stream) {
  if (!net || net->num_layers < 1 || net->num_layers > OTTB_MLP_MAX_LAYERS)
    return OTTB_ERR_INVALID;
  for (int l = 0; l < net->num_layers; ++l) {
    const ottb_mlp_layer& ly = net->layers[l];
    if (!ly.w || !ly.w_m || !ly.w_v || !ly.w_grad || !ly.b || !ly.b_m || !ly.b_v || !ly.b_grad)
      return OTTB_ERR_INVALID;
    const dim3 block(32, 8);
    adam_kernel<<<dim3((ly.in + 31) / 32, (ly.out + 31) / 32), block, 0, stream>>>(
        ly.w, ly.w_m, ly.w_v, ly.w_grad, ly.out, ly.in, lr, beta1, beta2, eps, c1, c2, hyper,
        (__nv_bfloat16*)ly.w_bf16, (__nv_bfloat16*)ly.wt_bf16);
    adam_kernel<<<dim3((ly.out + 31) / 32, 1), block, 0, stream>>>(
        ly.b, ly.b_m, ly.b_v, ly.b_grad, 1, ly.out, lr, beta1, beta2, eps, c1, c2, hyper,
        nullptr, nullptr);
  }
  return cudaGetLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}

}  // namespace

extern "C" {

int32_t ottb_mlp_adam(const ottb_mlp* net, float lr, float beta1, float beta2, float eps,
                      int32_t step, void* stream_ptr) {
  if (step < 1) return OTTB_ERR_INVALID;
  // bias corrections in double, rounded once
  const float c1 = (float)(1.0 - pow((double)beta1, (double)step));
  const float c2 = (float)(1.0 - pow((double)beta2, (double)step));
  return adam_all(net, lr, beta1, beta2, eps, c1, c2, nullptr, (cudaStream_t)stream_ptr);
}

int32_t ottb_mlp_adam_device(const ottb_mlp* net, const float* hyper, float beta1, float beta2,
                             float eps, void* stream_ptr) {
  if (!hyper) return OTTB_ERR_INVALID;
  return adam_all(net, 0.f, beta1, beta2, eps, 1.f, 1.f, hyper, (cudaStream_t)stream_ptr);
}

int32_t ottb_mlp_sync_bf16(const ottb_mlp* net, void* stream_ptr) {
  if (!net || net->num_layers < 1 || net->num_layers > OTTB_MLP_MAX_LAYERS) return OTTB_ERR_INVALID;
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  for (int l = 0; l < net->num_layers; ++l) {
    const ottb_mlp_layer& ly = net->layers[l];
    if (!ly.w || !ly.w_bf16 || !ly.wt_bf16) return OTTB_ERR_INVALID;
    const int64_t nw = (int64_t)ly.out * ly.in;
    to_bf16_kernel<<<(unsigned)std::min<int64_t>((nw + 255) / 256, 4096), 256, 0, stream>>>(
        ly.w, ly.out, ly.in, (__nv_bfloat16*)ly.w_bf16, (__nv_bfloat16*)ly.wt_bf16);
  }
  return cudaGetLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}

}  // extern "C"
