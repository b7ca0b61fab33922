// Persistent Sinkhorn kernel on the tensor-core (tcgen05, BF16 split-3)
// engine. One CTA per SM (its shared memory exceeds half an SM), so the
// 512-column TMEM allocation never waits on another CTA.
//
// A sweep's work units run pipelined across units: the epilogue warps deal
// the units (round-robin or from the sweep's atomic queue) and publish each
// as a descriptor in a two-slot ring in shared memory; the producer and MMA
// warps consume the descriptors in order, so they load the next unit's A
// tile and B tiles and issue its MMAs while the epilogue warps still finish
// the current unit (its last tiles, the column-group merge, the split
// combine and the potential update, synchronised among the epilogue warps
// by named barrier 1). Only the sweep's end, a grid barrier, joins all
// warps.
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

// One sweep on the tensor cores (see the file comment). Returns false,
// uniformly over the CTA, if any wait timed out.
template <int DK, int TN>
__device__ bool tc_sweep(const KernelArgs& A, const SweepParams& sp, unsigned sweep_idx,
                         TcSmem<DK, TN>& sm, TcPipe& pp) {
  constexpr int kEpiThreads = TcCfg<DK, TN>::kEpiWarps * 32;
  constexpr int CG = TcCfg<DK, TN>::kColGroups;
  using G = WarpGroup<64, kEpiThreads>;
  const int warp = threadIdx.x >> 5;
  const volatile int* err = &sm.err;
  const uint64_t tmo = A.timeout_ns;

  if (warp < 2) {
    // producer (warp 0) and MMA issuer (warp 1): consume unit descriptors
    // until this sweep's end marker
    const int lane = threadIdx.x & 31;
    bool ok = true;
    while (ok) {
      const uint32_t d = pp.desc++;
      const int slot = d & 1;
      ok = __all_sync(0xffffffffu, tc::mbar_wait(&sm.unit_full[slot], (d >> 1) & 1, tmo));
      if (!ok) break;
      // read in place: the dealer rewrites this slot only after both warps
      // arrive on unit_empty, which they do once they are done with the unit
      const TcUnit& u = sm.units[slot];
      bool stop = u.end || *err;
      if (!stop) {
        const bool r = warp == 0 ? tc_produce<DK, TN>(sm, pp, u, tmo)
                                 : tc_mma<DK, TN>(sm, pp, u, tmo);
        ok = __all_sync(0xffffffffu, r);
      }
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&sm.unit_empty[slot]);
      if (stop) break;
    }
    if (!ok) atomicExch(&sm.err, 1);
  } else {
    // epilogue warps: deal the units, reduce their tiles, finish each unit
    const int t = G::tid();
    const bool leader = t == 0;
    // Writes the next descriptor into its ring slot (leader only; its
    // round-robin position and end flag live in shared memory).
    auto deal = [&]() -> bool {
      if (sm.deal_ended) return true;
      const int* ids = sp.final_eval ? A.eval_ids : A.active_ids;
      const int* pre = sp.final_eval ? A.eval_prefix
                                     : (A.prefix + (sp.kind == kSweepG ? 0 : A.num_problems + 1));
      const int count = sp.final_eval ? ld_sched(&A.sched->num_eval)
                                      : ld_sched(&A.sched->num_active);
      const int total = sp.final_eval
                            ? ld_sched(&A.sched->eval_units)
                            : ld_sched(&A.sched->total_units[sp.kind == kSweepG ? 0 : 1]);
      const uint32_t w = pp.wdesc;
      const int slot = w & 1;
      if (w >= 2 && !tc::mbar_wait(&sm.unit_empty[slot], ((w - 2) >> 1) & 1, tmo)) return false;
      TcUnit& u = sm.units[slot];
      const int ui = ld_sched(&A.sched->dynamic_units) != 0
                         ? (int)atomicAdd(&A.gl->unit_ctr[sweep_idx % 3], 1u)
                         : sm.deal_rr;
      sm.deal_rr += gridDim.x;
      if (ui >= total) {
        u.end = 1;
        sm.deal_ended = 1;
      } else {
        const int q = find_problem(pre, count, ui);
        const int p = __ldcg(ids + q);
        const ProbDev& P = A.probs[p];
        const int local = ui - __ldcg(pre + q);
        const int S = split_of(A.state[p], sp.kind);
        u.end = 0;
        u.p = p;
        u.S = S;
        u.rb = local / S;
        u.sidx = local % S;
        u.parity = sp.final_eval ? __ldcg(&A.state[p].final_parity) : sp.parity;
        const int64_t cols = sp.kind == kSweepG ? P.n : P.m;
        const int ntiles = (int)((cols + TN - 1) / TN);
        u.t0 = (int)(((int64_t)ntiles * u.sidx) / S);
        u.t1 = (int)(((int64_t)ntiles * (u.sidx + 1)) / S);
        // The x layout carries the exponent scale of the target epsilon; a
        // sweep at another epsilon scales the accumulator by ws / ws_t.
        u.r = sweep_wscale(P, sp.mult) / P.ws_t;
        u.op = make_tc_operands(P, sp.kind, u.parity);
        u.rs = bounded_row_shift(P, sp);
      }
      ++pp.wdesc;
      tc::mbar_arrive(&sm.unit_full[slot]);
      return true;
    };
    if (leader) {
      if (blockIdx.x == 0) A.gl->unit_ctr[(sweep_idx + 1) % 3] = 0u;
      sm.deal_rr = blockIdx.x;
      sm.deal_ended = 0;
      if (!deal() || !deal()) atomicExch(&sm.err, 1);
    }
    while (true) {
      const uint32_t d = pp.desc++;
      const int slot = d & 1;
      if (!tc::mbar_wait(&sm.unit_full[slot], (d >> 1) & 1, tmo)) atomicExch(&sm.err, 1);
      // read in place: the dealer rewrites this slot only after this unit
      const TcUnit& u = sm.units[slot];
      // err may be set by the producer or MMA warp at any time: the group
      // decides together whether to stop
      if (G::sync_or(*err != 0 || u.end != 0)) break;
      tc_epilogue<DK, TN>(sm, pp, u, tmo);
      if (G::sync_or(*err != 0)) break;
      // the column groups' (shift, sum) of each row merged
      if (t < kBM) {
        float mv = sm.part_m[0][t], lv = sm.part_l[0][t];
#pragma unroll
        for (int k = 1; k < CG; ++k) lse_merge(mv, lv, sm.part_m[k][t], sm.part_l[k][t]);
        sm.rm[t] = mv;
        sm.rl[t] = lv;
      }
      G::sync();
      // a row block split over S column ranges is finished by the CTA that
      // completes its last range (as sweep_units)
      const ProbDev& P = A.probs[u.p];
      const int64_t R = sp.kind == kSweepG ? P.m : P.n;
      bool do_final = true;
      if (u.S > 1) {
        const int64_t rbase = (int64_t)u.rb * kBM;
        for (int i = t; i < kBM; i += kEpiThreads) {
          if (rbase + i < R) {
            P.part_m[(int64_t)u.sidx * R + rbase + i] = sm.rm[i];
            P.part_l[(int64_t)u.sidx * R + rbase + i] = sm.rl[i];
          }
        }
        __threadfence();
        G::sync();
        if (leader) {
          const int prev = atomicAdd(&P.arrive[u.rb], 1);
          sm.last = (prev == u.S - 1);
          if (sm.last) atomicExch(&P.arrive[u.rb], 0);
        }
        G::sync();
        do_final = sm.last != 0;
        if (do_final) {
          __threadfence();
          for (int i = t; i < kBM; i += kEpiThreads) {
            float mv = kNegSentinel, lv = 0.f;
            if (rbase + i < R) {
              for (int k = 0; k < u.S; ++k) {
                const float m2 = __ldcg(P.part_m + (int64_t)k * R + rbase + i);
                const float l2 = __ldcg(P.part_l + (int64_t)k * R + rbase + i);
                lse_merge(mv, lv, m2, l2);
              }
            }
            sm.rm[i] = mv;
            sm.rl[i] = lv;
          }
          G::sync();
        }
      }
      if (do_final)
        finalize_rows_g<G>(P, sp, u.parity, u.rb, sm.rm, sm.rl, A.cfg.norm_error, sm.red);
      G::sync();
      if (leader && !deal()) atomicExch(&sm.err, 1);
    }
  }
  __syncthreads();
  return *err == 0;
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
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(&sm.unit_full[i], 1);   // the dealer
      tc::mbar_init(&sm.unit_empty[i], 2);  // producer and MMA warps
    }
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

  TcPipe pp{0u, 0u, 0u, 0u, 0u, 0, 0u, 0u};
  auto sweep = [&](const SweepParams& sp, unsigned idx) -> bool {
    return tc_sweep<DK, TN>(A, sp, idx, sm, pp);
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
