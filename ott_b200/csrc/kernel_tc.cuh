// Persistent Sinkhorn kernel on the tensor-core (tcgen05, BF16 split-3)
// engine. One CTA per SM (its shared memory exceeds half an SM), so the
// 256-column TMEM allocation never waits on another CTA.
#pragma once

#include "engine_tc.cuh"
#include "persistent.cuh"

namespace ottb {

__device__ __forceinline__ TcOperands make_tc_operands(const ProbDev& P, int kind,
                                                       int parity) {
  const TcMaps* maps = reinterpret_cast<const TcMaps*>(P.maps);
  TcOperands op;
  if (kind == kSweepG) {
    op.mapA = &maps->y; op.padA = (int32_t)P.m_pad; op.rows = P.m;
    op.mapB = &maps->x; op.padB = (int32_t)P.n_pad; op.cols = P.n;
    // symmetric problem: the columns' potential is the current g, whose
    // shift rows the g-updates write into y's buffers (y's points are x's)
    op.mapBext = P.symmetric ? &maps->exty : &maps->extx;
    op.extRow0 = P.symmetric ? (int32_t)(parity * P.m_pad) : 0;
  } else {
    op.mapA = &maps->x; op.padA = (int32_t)P.n_pad; op.rows = P.n;
    op.mapB = &maps->y; op.padB = (int32_t)P.m_pad; op.cols = P.m;
    op.mapBext = &maps->exty; op.extRow0 = (int32_t)(parity * P.m_pad);
  }
  return op;
}

// Whether this problem's units of the sweep use the bounded row shift, and
// the bound: D = the largest change of a column shift since the rows' last
// sweep (0 when no potential changed), usable while the spread of those
// changes stays within kMaxShiftSpread.
__device__ __forceinline__ RowShift bounded_row_shift(const ProbDev& P, const SweepParams& sp) {
  RowShift rs{nullptr, 0.f, 0, false};
  if (!sp.fast || P.symmetric || !P.lprev || !P.dkey) return rs;
  const int* slot = P.dkey + ((sp.kind * 2 + sp.rslot) * 2);
  const int kmax = __ldcg(slot), kmin = __ldcg(slot + 1);
  float dmax = 0.f, spread = 0.f;
  if (kmax != kDkeyEmptyMax) {
    if (kmin == kDkeyEmptyMin) return rs;
    dmax = fkey_value(kmax);
    spread = dmax - fkey_value(kmin);
  }
  if (!(spread <= kMaxShiftSpread) || !isfinite(dmax)) return rs;
  rs.lprev = P.lprev + (sp.kind == kSweepG ? P.n_pad : 0);
  rs.dmax = dmax;
  rs.rows = sp.kind == kSweepG ? P.m : P.n;
  rs.on = true;
  return rs;
}

template <int DK, int TN>
__global__ void __launch_bounds__(TcCfg<DK, TN>::kThreads, 1)
sinkhorn_tc_kernel(KernelArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // The 128-byte swizzled operand tiles need 1024-byte alignment.
  const uint32_t base = tc::smem_u32(smem_raw);
  unsigned char* aligned = smem_raw + ((1024u - (base & 1023u)) & 1023u);
  TcSmem<DK, TN>& sm = *reinterpret_cast<TcSmem<DK, TN>*>(aligned);
  constexpr int NS = TcCfg<DK, TN>::kStages;
  constexpr int NB = TcCfg<DK, TN>::kTmemBufs;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    constexpr int NE = TcCfg<DK, TN>::kEpiWarps;
    for (int i = 0; i < NS; ++i) {
      tc::mbar_init(&sm.full[i], 1);   // producer arrival + TMA bytes
      tc::mbar_init(&sm.empty[i], 1);  // MMA commit
    }
    for (int i = 0; i < NB; ++i) {
      tc::mbar_init(&sm.tfull[i], 1);
      tc::mbar_init(&sm.tempty[i], NE);
    }
    tc::mbar_init(&sm.a_full, 1);
    tc::mbar_init(&sm.a_empty, 1);
    tc::mbar_init(&sm.drain, 1);
    sm.err = 0;
    tc::fence_barrier_init();
  }
  if (warp == 1) {
    tc::tmem_alloc(&sm.tmem_base, TcCfg<DK, TN>::kTmemCols);
    tc::tmem_relinquish();
  }
  // Extension blocks: zero everywhere; A's first 3 K columns are ones.
  {
    uint32_t* a32 = reinterpret_cast<uint32_t*>(sm.Aext);
    for (int i = threadIdx.x; i < TcCfg<DK, TN>::kAExtBytes / 4; i += blockDim.x) a32[i] = 0u;
    for (int st = 0; st < NS; ++st) {
      uint32_t* b32 = reinterpret_cast<uint32_t*>(sm.Bext[st]);
      for (int i = threadIdx.x; i < TcCfg<DK, TN>::kBExtBytes / 4; i += blockDim.x) b32[i] = 0u;
    }
    __syncthreads();
    if (threadIdx.x < kBM) {
      const __nv_bfloat16 one = __float2bfloat16_rn(1.f);
      for (int k = 0; k < 3; ++k)
        reinterpret_cast<__nv_bfloat16*>(sm.Aext + threadIdx.x * 16)[k] = one;
    }
    tc::fence_proxy_async_smem();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();

  TcPipe pp{0u, 0u, 0u, 0u, 0u, 0};
  const CommonSmem cs{sm.rm, sm.rl, sm.red, &sm.unit, &sm.last};
  auto sweep = [&](const SweepParams& sp, unsigned idx) -> bool {
    auto unit = [&](const ProbDev& P, const float* gcur, int parity, int rb, int t0, int t1,
                    float s, float wscale) -> bool {
      const TcOperands op = make_tc_operands(P, sp.kind, parity);
      // The x layout carries the exponent scale of the target epsilon; a
      // sweep at another epsilon scales the accumulator by ws / ws_t.
      const float r = wscale / P.ws_t;
      RowShift rs = bounded_row_shift(P, sp);
      return tc_unit<DK, TN>(sm, pp, op, rb * kBM, t0, t1, r, rs, A.timeout_ns);
    };
    return sweep_units<TcCfg<DK, TN>::kTileN>(A, sp, idx, cs, unit);
  };
  persistent_main(A, sweep);

  // Teardown. After a timeout, wait (bounded) for this CTA's own MMAs and
  // TMA loads still in flight before the TMEM and shared memory go away.
  __syncthreads();
  if (sm.err) {
    const uint64_t limit = 1000000000ull;  // 1 s
    if (warp == 1 && lane == 0) {
      tc::mma_commit(&sm.drain);
      tc::mbar_wait(&sm.drain, 0, limit);
    }
    if (warp == 0 && lane == 0 && pp.issued)
      tc::mbar_wait(&sm.full[pp.last_full_stage], pp.last_full_parity, limit);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 1) tc::tmem_dealloc(sm.tmem_base, TcCfg<DK, TN>::kTmemCols);
}

}  // namespace ottb
