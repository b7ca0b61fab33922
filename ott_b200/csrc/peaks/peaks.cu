// Throughput probes for the roofline denominators that have no driver-
// measured figure: FP32 FMA and MUFU ex2 issue rates. Used by bench.py; not
// part of the Sinkhorn C ABI. Every thread runs 8 independent dependency
// chains so the pipe, not latency, bounds the loop.
#include <cuda_runtime.h>
#include <stdint.h>

__global__ void ffma_probe(float* out, int iters) {
  float v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = (float)(threadIdx.x + k) * 1e-3f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = fmaf(v[k], 0.999f, 1e-3f);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += v[k];
  if (s == 12345.f) out[blockIdx.x] = s;
}

__global__ void ex2_probe(float* out, int iters) {
  float v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = -(float)(threadIdx.x + k) * 1e-3f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      float y;
      asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(v[k]));
      v[k] = -y;
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += v[k];
  if (s == 12345.f) out[blockIdx.x] = s;
}

extern "C" {
// kind 0: FFMA, kind 1: ex2. Returns 0 on success. Work = blocks * 256 *
// iters * 8 operations.
int ottb_peaks_launch(int kind, int blocks, int iters, float* out, void* stream) {
  cudaStream_t s = (cudaStream_t)stream;
  if (kind == 0)
    ffma_probe<<<blocks, 256, 0, s>>>(out, iters);
  else
    ex2_probe<<<blocks, 256, 0, s>>>(out, iters);
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}
}
