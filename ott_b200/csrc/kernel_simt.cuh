// Persistent Sinkhorn kernel on the FP32 CUDA-core engine.
#pragma once

#include "engine_simt.cuh"
#include "persistent.cuh"

namespace ottb {

template <int DP>
struct SimtKernelSmem {
  SimtSmem<DP> tiles;
  float rm[kBM];
  float rl[kBM];
  double red[8];
  int unit;
  int last;
};

// Two CTAs per SM up to DP = 64 (128 registers and < 114 KB of shared
// memory each): one CTA's tile barriers and epilogue overlap the other's
// FMAs. Measured against one CTA per SM: n = m = 65536, d = 64: 3 % faster;
// n = m = 16384, d = 16: 14 %; n = m = 32768, d = 8: 13 % (with the dot
// product unrolled by 2 there).
template <int DP>
__global__ void __launch_bounds__(256, (DP <= 64 ? 2 : 1))
sinkhorn_simt_kernel(KernelArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SimtKernelSmem<DP>& sm = *reinterpret_cast<SimtKernelSmem<DP>*>(smem_raw);
  const CommonSmem cs{sm.rm, sm.rl, sm.red, &sm.unit, &sm.last};
  auto sweep = [&](const SweepParams& sp, unsigned idx) -> bool {
    auto unit = [&](const ProbDev& P, const float* gcur, int parity, int rb, int t0, int t1,
                    float s, float wscale) -> bool {
      const SweepOperands op = make_operands(P, sp.kind, gcur);
      simt_unit<DP>(sm.tiles, op, (int64_t)rb * kBM, t0, t1, s, wscale, sm.rm, sm.rl);
      return true;
    };
    return sweep_units<kBN>(A, sp, idx, cs, unit);
  };
  persistent_main(A, sweep);
}

}  // namespace ottb
