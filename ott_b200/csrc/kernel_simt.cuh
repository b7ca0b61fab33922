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

template <int DP>
__global__ void __launch_bounds__(256, (DP <= 2 ? 2 : 1))
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
