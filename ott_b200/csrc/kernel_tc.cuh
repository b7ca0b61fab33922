// Persistent Sinkhorn kernel on the tensor-core (tcgen05, BF16 split-3)
// engine. One CTA per SM (its shared memory exceeds half an SM), so the
// 512-column TMEM allocation never waits on another CTA.
//
// A sweep's work units run pipelined across units and roles: the dealer
// warp takes the units (round-robin or from the sweep's atomic queue) and
// publishes each as a descriptor in a ring of four slots in shared memory;
// the producer and MMA warps consume the descriptors in order, so they load
// the next unit's A tile and B tiles and issue its MMAs while the epilogue
// warps still reduce the current unit's last tiles; the finalizer warp
// merges, combines and applies each unit's row results while the epilogue
// warps reduce the next one. Only the sweep's end, a grid barrier, joins
// all warps.
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

// The problem of unit u in a sweep's unit list: the last q with
// prefix[q] <= u (prefix[count] = total > u), by a 32-way search over the
// warp's lanes (two rounds for up to 1024 problems).
__device__ __forceinline__ int warp_find_problem(const int* prefix, int count, int u) {
  const int lane = threadIdx.x & 31;
  int lo = 0, hi = count;
  while (hi - lo > 1) {
    const int step = (hi - lo + 31) >> 5;
    const int idx = lo + lane * step;
    const bool le = idx < hi && __ldcg(prefix + idx) <= u;
    const unsigned bal = __ballot_sync(0xffffffffu, le);  // lane 0 (idx = lo) is set
    lo += (31 - __clz(bal)) * step;
    hi = min(hi, lo + step);
  }
  return lo;
}

// One sweep on the tensor cores (see the file comment). Returns false,
// uniformly over the CTA, if any wait timed out.
template <int DK, int TN>
__device__ bool tc_sweep(const KernelArgs& A, const SweepParams& sp, unsigned sweep_idx,
                         TcSmem<DK, TN>& sm, TcPipe& pp) {
  constexpr int CG = TcCfg<DK, TN>::kColGroups;
  constexpr uint32_t NSLOT = TcCfg<DK, TN>::kDescSlots;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const volatile int* err = &sm.err;
  const uint64_t tmo = A.timeout_ns;

  if (warp == 2) {
    // dealer: every unit of this CTA, then the end marker
    const int* ids = sp.final_eval ? A.eval_ids : A.active_ids;
    const int* pre = sp.final_eval ? A.eval_prefix
                                   : (A.prefix + (sp.kind == kSweepG ? 0 : A.num_problems + 1));
    const int count = sp.final_eval ? ld_sched(&A.sched->num_eval)
                                    : ld_sched(&A.sched->num_active);
    const int total = sp.final_eval ? ld_sched(&A.sched->eval_units)
                                    : ld_sched(&A.sched->total_units[sp.kind == kSweepG ? 0 : 1]);
    const bool dynamic = ld_sched(&A.sched->dynamic_units) != 0;
    unsigned* ctr = &A.gl->unit_ctr[sweep_idx % 3];
    if (blockIdx.x == 0 && lane == 0) A.gl->unit_ctr[(sweep_idx + 1) % 3] = 0u;
    int rr = blockIdx.x;
    bool ended = false;
    while (!ended) {
      const uint32_t w = pp.wdesc++;
      const uint32_t slot = w % NSLOT;
      bool ok = w < NSLOT || tc::mbar_wait(&sm.unit_empty[slot], ((w - NSLOT) / NSLOT) & 1, tmo);
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) atomicExch(&sm.err, 1);
        break;
      }
      TcUnit& u = sm.units[slot];
      int ui = 0;
      if (lane == 0) ui = dynamic ? (int)atomicAdd(ctr, 1u) : rr;
      ui = __shfl_sync(0xffffffffu, ui, 0);
      rr += gridDim.x;
      // after an error the end marker lets the other roles unwind at once
      if (ui >= total || __any_sync(0xffffffffu, *err != 0)) {
        ended = true;
        if (lane == 0) u.end = 1;
      } else {
        const int q = warp_find_problem(pre, count, ui);
        if (lane == 0) {
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
      }
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&sm.unit_full[slot]);
    }
  } else if (warp == 3) {
    // finalizer: per unit, merge the column groups' (shift, sum) of each row
    // (lane l: rows l + 32 k), combine the column splits of a row block
    // (the CTA that completes its last split finishes it, as sweep_units)
    // and update the rows' potentials
    while (true) {
      const uint32_t d = pp.desc++;
      const uint32_t slot = d % NSLOT;
      bool ok = tc::mbar_wait(&sm.unit_full[slot], (d / NSLOT) & 1, tmo);
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) atomicExch(&sm.err, 1);
        break;
      }
      const TcUnit& u = sm.units[slot];
      const bool stop = u.end != 0 || __any_sync(0xffffffffu, *err != 0);
      if (!stop) {
        const uint32_t pb = pp.unit & 1;
        ok = __all_sync(0xffffffffu, tc::mbar_wait(&sm.epi_done[pb], (pp.unit >> 1) & 1, tmo));
        ++pp.unit;
        if (!ok) {
          if (lane == 0) atomicExch(&sm.err, 1);
          break;
        }
        float mv[4], lv[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int r = lane + 32 * k;
          mv[k] = sm.part_m[pb][0][r];
          lv[k] = sm.part_l[pb][0][r];
#pragma unroll
          for (int c = 1; c < CG; ++c) lse_merge(mv[k], lv[k], sm.part_m[pb][c][r], sm.part_l[pb][c][r]);
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&sm.part_free[pb]);
        const ProbDev& P = A.probs[u.p];
        const int64_t R = sp.kind == kSweepG ? P.m : P.n;
        const int64_t rbase = (int64_t)u.rb * kBM;
        bool do_final = true;
        if (u.S > 1) {
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int64_t row = rbase + lane + 32 * k;
            if (row < R) {
              P.part_m[(int64_t)u.sidx * R + row] = mv[k];
              P.part_l[(int64_t)u.sidx * R + row] = lv[k];
            }
          }
          __threadfence();
          __syncwarp();
          int last = 0;
          if (lane == 0) {
            const int prev = atomicAdd(&P.arrive[u.rb], 1);
            last = prev == u.S - 1;
            if (last) atomicExch(&P.arrive[u.rb], 0);
          }
          do_final = __shfl_sync(0xffffffffu, last, 0) != 0;
          if (do_final) {
            __threadfence();
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const int64_t row = rbase + lane + 32 * k;
              mv[k] = kNegSentinel;
              lv[k] = 0.f;
              if (row < R) {
                for (int j = 0; j < u.S; ++j)
                  lse_merge(mv[k], lv[k], __ldcg(P.part_m + (int64_t)j * R + row),
                            __ldcg(P.part_l + (int64_t)j * R + row));
              }
            }
          }
        }
        if (do_final) finalize_rows_warp(P, sp, u.parity, u.rb, mv, lv, A.cfg.norm_error);
      }
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&sm.unit_empty[slot]);
      if (stop) break;
    }
  } else if (warp < 2) {
    // producer (warp 0) and MMA issuer (warp 1)
    while (true) {
      const uint32_t d = pp.desc++;
      const uint32_t slot = d % NSLOT;
      bool ok = __all_sync(0xffffffffu, tc::mbar_wait(&sm.unit_full[slot], (d / NSLOT) & 1, tmo));
      if (!ok) {
        if (lane == 0) atomicExch(&sm.err, 1);
        break;
      }
      // read in place: the dealer rewrites this slot only after this warp,
      // the other control warp and the finalizer have arrived on unit_empty
      const TcUnit& u = sm.units[slot];
      const bool stop = u.end != 0 || __any_sync(0xffffffffu, *err != 0);
      if (!stop) {
        const bool r = warp == 0 ? tc_produce<DK, TN>(sm, pp, u, tmo)
                                 : tc_mma<DK, TN>(sm, pp, u, tmo);
        ok = __all_sync(0xffffffffu, r);
      }
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&sm.unit_empty[slot]);
      if (stop || !ok) break;
    }
  } else {
    // epilogue warps, each on its own: reduce every unit's tiles into the
    // part buffers
    while (true) {
      const uint32_t d = pp.desc++;
      const uint32_t slot = d % NSLOT;
      bool ok = __all_sync(0xffffffffu, tc::mbar_wait(&sm.unit_full[slot], (d / NSLOT) & 1, tmo));
      if (!ok) {
        if (lane == 0) atomicExch(&sm.err, 1);
        break;
      }
      const TcUnit& u = sm.units[slot];
      if (u.end != 0 || __any_sync(0xffffffffu, *err != 0)) break;
      if (!__all_sync(0xffffffffu, tc_epilogue<DK, TN>(sm, pp, u, tmo))) break;
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
    for (int i = 0; i < TcCfg<DK, TN>::kDescSlots; ++i) {
      tc::mbar_init(&sm.unit_full[i], 1);   // the dealer
      tc::mbar_init(&sm.unit_empty[i], 3);  // producer, MMA and finalizer warps
    }
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(&sm.epi_done[i], NE);   // one arrival per epilogue warp
      tc::mbar_init(&sm.part_free[i], 1);   // the finalizer
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
