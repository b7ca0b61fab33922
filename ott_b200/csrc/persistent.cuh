// The persistent cooperative kernel: control flow of the fixed-point loop,
// work distribution over (problem, row block, column split) units, split
// combination by the last-arriving CTA, and the per-block stop test.
#pragma once

#include "common.cuh"
#include "driver.cuh"

namespace ottb {

// Locates unit u in a prefix-summed list of problems.
__device__ __forceinline__ int find_problem(const int* prefix, int count, int u) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= u) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int split_of(const ProbState& S, int kind) {
  return kind == kSweepG ? __ldcg(&S.split_g) : __ldcg(&S.split_f);
}

// A symmetric problem has no f-sweep (f = g).
__device__ __forceinline__ int units_of(const ProbDev& P, const ProbState& S, int kind) {
  if (kind == kSweepF && P.symmetric) return 0;
  return kind == kSweepG ? P.rb_g * split_of(S, kSweepG) : P.rb_f * split_of(S, kSweepF);
}

// CTA 0 only: rebuild the active list and unit prefix sums. When the
// active problems (fewer as problems converge) no longer offer
// sched->target_units units per sweep, their column splits grow, each up to the
// largest split its workspace partials hold, so the remaining problems
// still spread over the whole grid. Splits never shrink.
__device__ void rebuild_schedule(const KernelArgs& A) {
  if (threadIdx.x == 0) {
    int ug = 0, uf = 0, rg = 0, rf = 0;
    for (int p = 0; p < A.num_problems; ++p) {
      if (!A.state[p].active) continue;
      ug += units_of(A.probs[p], A.state[p], kSweepG);
      uf += units_of(A.probs[p], A.state[p], kSweepF);
      rg += A.probs[p].rb_g;
      rf += A.probs[p].rb_f;
    }
    const int tgt = A.sched->target_units;
    if (rg > 0 && (ug < tgt || uf < tgt)) {
      const int kg = (tgt + rg - 1) / rg, kf = (tgt + rf - 1) / rf;
      for (int p = 0; p < A.num_problems; ++p) {
        ProbState& S = A.state[p];
        if (!S.active) continue;
        const ProbDev& P = A.probs[p];
        S.split_g = max(S.split_g, min(kg, P.smax_g));
        S.split_f = max(S.split_f, min(kf, P.smax_f));
      }
    }
    int na = 0;
    ug = 0;
    uf = 0;
    for (int p = 0; p < A.num_problems; ++p) {
      if (!A.state[p].active) continue;
      A.active_ids[na] = p;
      A.prefix[na] = ug;
      A.prefix[A.num_problems + 1 + na] = uf;
      ug += units_of(A.probs[p], A.state[p], kSweepG);
      uf += units_of(A.probs[p], A.state[p], kSweepF);
      ++na;
    }
    A.prefix[na] = ug;
    A.prefix[A.num_problems + 1 + na] = uf;
    A.sched->num_active = na;
    A.sched->total_units[0] = ug;
    A.sched->total_units[1] = uf;
    int ne = 0, ue = 0;
    for (int p = 0; p < A.num_problems; ++p) {
      if (A.state[p].active || A.state[p].msum_valid) continue;
      A.eval_ids[ne] = p;
      A.eval_prefix[ne] = ue;
      ue += units_of(A.probs[p], A.state[p], kSweepG);
      ++ne;
    }
    A.eval_prefix[ne] = ue;
    A.sched->num_eval = ne;
    A.sched->eval_units = ue;
    __threadfence();
  }
  __syncthreads();
}

// Deterministic reduction of the per-row-block marginal partials of one
// problem (one warp per problem, fixed lane assignment and shuffle tree).
__device__ __forceinline__ void reduce_marginals(const ProbDev& P, int lane,
                                                double& err, double& msum) {
  double e = 0.0, s = 0.0;
  for (int i = lane; i < P.rb_g; i += 32) {
    e += __ldcg(P.err_part + i);
    s += __ldcg(P.msum_part + i);
  }
  for (int off = 16; off > 0; off >>= 1) {
    e += __shfl_xor_sync(0xffffffffu, e, off);
    s += __shfl_xor_sync(0xffffffffu, s, off);
  }
  err = e;
  msum = s;
}

// CTA 0, at the end of a block (it = iterations done, a multiple of inner):
// record the block error, apply fixed_point_loop's stop test, update state.
__device__ void block_boundary(const KernelArgs& A, int it, bool need_err,
                               bool may_continue, int parity) {
  const ottb_solver_cfg& c = A.cfg;
  const bool force_scan = c.min_iterations == c.max_iterations;
  const int blk = (it - 1) / c.inner_iterations;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  for (int q = warp; q < A.sched->num_active; q += nwarps) {
    const int p = A.active_ids[q];
    const ProbDev& P = A.probs[p];
    double err = INFINITY, msum = 0.0;
    if (need_err) {
      reduce_marginals(P, lane, err, msum);
      if (c.norm_error != 1) err = pow(err, 1.0 / (double)c.norm_error);
      // parallel updates: the error of both marginals (sinkhorn.py:168-188),
      // equal for a symmetric problem
      if (P.symmetric) err *= 2.0;
    }
    if (lane == 0) {
      const float errf = (float)err;
      P.errors[blk] = errf;
      bool cont;
      if (force_scan) {
        cont = may_continue;
      } else {
        // sinkhorn.py:940-953 inside fixed_point_loop.py:63-70
        const bool converged = (it > 0) && (errf < c.threshold);
        const bool diverged = !isfinite(errf);
        cont = may_continue && ((it < c.min_iterations) || (!diverged && !converged));
      }
      ProbState& S = A.state[p];
      if (!cont) {
        S.active = 0;
        S.final_parity = parity;
        S.stop_it = it;
        S.msum_valid = need_err ? 1 : 0;
        S.msum = msum;
      }
    }
  }
  __syncthreads();
  __threadfence();
  rebuild_schedule(A);
}


__device__ __forceinline__ int ld_sched(const int* p) { return *(const volatile int*)p; }

// Shared-memory words every engine provides to the unit loop.
struct CommonSmem {
  float* rm;    // [kBM] row shift (base-2) of the current unit
  float* rl;    // [kBM] row sum
  double* red;  // [8] reduction scratch
  int* unit;    // dealt unit index broadcast
  int* last;    // last-arriver flag broadcast
};

// One sweep over the units of the scheduled problems, common to both
// engines (tiles of TILE_N columns: 128 on the CUDA cores, 256 on the tensor
// cores). unit_fn(P, gcur, parity, rb, t0, t1, s, wscale) computes the (shift, sum)
// state of the 128 rows of row block rb over column tiles [t0, t1) into
// cs.rm / cs.rl and returns false on a device-side timeout. Units are dealt
// round-robin (one problem) or from an atomic queue (several problems, in
// decreasing-work order). A row block split over S column ranges is
// combined by the CTA that finishes its last range.
template <int TILE_N, class UnitFn>
__device__ bool sweep_units(const KernelArgs& A, const SweepParams& sp, unsigned sweep_idx,
                            const CommonSmem& cs, UnitFn&& unit_fn) {
  const int* ids = sp.final_eval ? A.eval_ids : A.active_ids;
  const int* pre = sp.final_eval ? A.eval_prefix
                                 : (A.prefix + (sp.kind == kSweepG ? 0 : A.num_problems + 1));
  const int count = sp.final_eval ? ld_sched(&A.sched->num_eval)
                                  : ld_sched(&A.sched->num_active);
  const int total = sp.final_eval ? ld_sched(&A.sched->eval_units)
                                  : ld_sched(&A.sched->total_units[sp.kind == kSweepG ? 0 : 1]);
  unsigned* ctr = &A.gl->unit_ctr[sweep_idx % 3];
  if (blockIdx.x == 0 && threadIdx.x == 0) A.gl->unit_ctr[(sweep_idx + 1) % 3] = 0u;

  const bool dynamic = ld_sched(&A.sched->dynamic_units) != 0;
  int u = blockIdx.x;
  if (dynamic) {
    if (threadIdx.x == 0) *cs.unit = (int)atomicAdd(ctr, 1u);
    __syncthreads();
    u = *cs.unit;
    __syncthreads();
  }
  while (u < total) {
    const int q = find_problem(pre, count, u);
    const int p = __ldcg(ids + q);
    const ProbDev& P = A.probs[p];
    const int local = u - __ldcg(pre + q);
    const int S = split_of(A.state[p], sp.kind);
    const int rb = local / S;
    const int sidx = local % S;
    const int parity = sp.final_eval ? __ldcg(&A.state[p].final_parity) : sp.parity;
    const float* gcur = P.gbuf[parity];
    const int64_t R = sp.kind == kSweepG ? P.m : P.n;
    const int64_t Ccols = sp.kind == kSweepG ? P.n : P.m;
    const int ntiles = (int)((Ccols + TILE_N - 1) / TILE_N);
    const int t0 = (int)(((int64_t)ntiles * sidx) / S);
    const int t1 = (int)(((int64_t)ntiles * (sidx + 1)) / S);
    const float wscale = sweep_wscale(P, sp.mult);
    const float s = 2.0f * P.inv_scale * wscale;

    if (!unit_fn(P, gcur, parity, rb, t0, t1, s, wscale)) return false;

    bool do_final = true;
    if (S > 1) {
      const int64_t rbase = (int64_t)rb * kBM;
      for (int t = threadIdx.x; t < kBM; t += blockDim.x) {
        if (rbase + t < R) {
          P.part_m[(int64_t)sidx * R + rbase + t] = cs.rm[t];
          P.part_l[(int64_t)sidx * R + rbase + t] = cs.rl[t];
        }
      }
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) {
        int prev = atomicAdd(&P.arrive[rb], 1);
        *cs.last = (prev == S - 1);
        if (*cs.last) atomicExch(&P.arrive[rb], 0);
      }
      __syncthreads();
      do_final = *cs.last != 0;
      if (do_final) {
        __threadfence();
        for (int t = threadIdx.x; t < kBM; t += blockDim.x) {
          float mv = kNegSentinel, lv = 0.f;
          if (rbase + t < R) {
            for (int k = 0; k < S; ++k) {
              float m2 = __ldcg(P.part_m + (int64_t)k * R + rbase + t);
              float l2 = __ldcg(P.part_l + (int64_t)k * R + rbase + t);
              lse_merge(mv, lv, m2, l2);
            }
          }
          cs.rm[t] = mv;
          cs.rl[t] = lv;
        }
        __syncthreads();
      }
    }
    if (do_final) finalize_rows(P, sp, parity, rb, cs.rm, cs.rl, A.cfg.norm_error, cs.red);
    __syncthreads();

    if (dynamic) {
      if (threadIdx.x == 0) *cs.unit = (int)atomicAdd(ctr, 1u);
      __syncthreads();
      u = *cs.unit;
      __syncthreads();
    } else {
      u += gridDim.x;
    }
  }
  return true;
}

// The fixed-point loop of every problem of the call, run by every CTA of
// the cooperative grid. sweep(sp, idx) runs one sweep and returns false on a
// device-side timeout. Mirrors fixed_point_loop.py:23-93 (blocks of
// inner_iterations, stop test between blocks, scan mode when min == max)
// with sinkhorn.py:879-953 (g- then f-update, block error, converged /
// diverged).
template <class SweepFn>
__device__ void persistent_main(const KernelArgs& A, SweepFn&& sweep) {
  const ottb_solver_cfg& c = A.cfg;
  const int inner = c.inner_iterations;
  const bool force_scan = c.min_iterations == c.max_iterations;
  const int scan_end = force_scan ? (c.max_iterations / inner) * inner : c.max_iterations;
  int* status = &A.sched->status;
  unsigned sweep_idx = 0;
  int it = 0;
  int commits = 0;  // committed g-sweeps; identical in every CTA
  // Per sweep kind: sweeps begun, and whether the last one ran at
  // multiplier 1 (its row log-sum-exps, stored by finalize_rows, then bound
  // the next one's rows; see tc_unit).
  int nsw[2] = {0, 0};
  int prev_one[2] = {0, 0};
  auto begin_sweep = [&](SweepParams& sp) {
    const int K = sp.kind;
    sp.rslot = nsw[K] & 1;
    sp.wslot = nsw[K ^ 1] & 1;
    sp.fast = (!sp.final_eval && sp.mult == 1.0f && prev_one[K]) ? 1 : 0;
    // The slot the sweep after next of this kind reads is free now (its
    // previous reader has finished, its writers come after this sweep).
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      const int nxt = (nsw[K] + 1) & 1;
      for (int p = 0; p < A.num_problems; ++p) {
        A.state[p].dkey[K][nxt][0] = kDkeyEmptyMax;
        A.state[p].dkey[K][nxt][1] = kDkeyEmptyMin;
      }
    }
    prev_one[K] = (!sp.final_eval && sp.mult == 1.0f) ? 1 : 0;
    ++nsw[K];
  };

#define OTTB_SWEEP(sp)                                                           \
  do {                                                                           \
    begin_sweep(sp);                                                             \
    if (!sweep((sp), sweep_idx++)) {                                             \
      if (threadIdx.x == 0) atomicExch(status, (int)OTTB_ERR_TIMEOUT);           \
      grid_barrier(A.gl, A.expected_arrivals, A.timeout_ns, status);             \
      return;                                                                    \
    }                                                                            \
  } while (0)
#define OTTB_BARRIER()                                                          \
  do {                                                                          \
    if (!grid_barrier(A.gl, A.expected_arrivals, A.timeout_ns, status)) return; \
  } while (0)

  if (c.init_f_from_g && scan_end > 0) {
    // f = update_potential(., g_init, log a, 0, axis=1): the c-transform of
    // an initializer's g, so that g is not discarded by the first g-update.
    SweepParams sp{kSweepF, eps_mult(c, 0), 0, 1, 0, 0};
    OTTB_SWEEP(sp);
    OTTB_BARRIER();
  }
  while (true) {
    bool fused = false;
    if (it > 0 && it % inner == 0) {
      const int last = it - 1;
      const bool need_err = (last == c.max_iterations - 1) || (last >= c.min_iterations);
      const bool may_continue = it < scan_end;
      const float mlt = may_continue ? eps_mult(c, it) : 1.0f;
      fused = need_err && may_continue && (mlt == 1.0f);
      const int parity = commits & 1;
      if (need_err) {
        SweepParams sp{kSweepG, fused ? mlt : 1.0f, 1, fused ? 1 : 0, 0, parity};
        OTTB_SWEEP(sp);
        OTTB_BARRIER();
      }
      if (blockIdx.x == 0) block_boundary(A, it, need_err, may_continue, parity);
      OTTB_BARRIER();
      if (ld_sched(&A.sched->num_active) == 0) break;
      if (fused) ++commits;
    } else if (it == 0 && scan_end == 0) {
      // max_iterations == 0, or a scan with fewer iterations than one block:
      // the loop body never runs (fixed_point_loop.py:63-93).
      break;
    }
    const float mlt = eps_mult(c, it);
    if (!fused) {
      SweepParams sp{kSweepG, mlt, 0, 1, 0, commits & 1};
      OTTB_SWEEP(sp);
      OTTB_BARRIER();
      ++commits;
    }
    {
      SweepParams sp{kSweepF, mlt, 0, 1, 0, commits & 1};
      OTTB_SWEEP(sp);
      OTTB_BARRIER();
    }
    ++it;
  }
  // Problems whose final state has no marginal sum yet (their last block
  // recorded no error, or they never iterated): one marginal sweep with the
  // target epsilon, needed by reg_ot_cost.
  if (blockIdx.x == 0) {
    if (it == 0 && threadIdx.x == 0) {
      // No iteration ran: every problem stops in its initial state.
      for (int p = 0; p < A.num_problems; ++p) {
        A.state[p].active = 0;
        A.state[p].final_parity = 0;
        A.state[p].msum_valid = 0;
        A.state[p].stop_it = 0;
      }
      __threadfence();
    }
    __syncthreads();
    rebuild_schedule(A);
  }
  OTTB_BARRIER();
  if (ld_sched(&A.sched->num_eval) > 0) {
    SweepParams sp{kSweepG, 1.0f, 1, 0, 1, 0};
    OTTB_SWEEP(sp);
    OTTB_BARRIER();
    if (blockIdx.x == 0) {
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int ne = ld_sched(&A.sched->num_eval);
      for (int q = warp; q < ne; q += (blockDim.x >> 5)) {
        const int p = A.eval_ids[q];
        double err, msum;
        reduce_marginals(A.probs[p], lane, err, msum);
        if (lane == 0) {
          A.state[p].msum = msum;
          A.state[p].msum_valid = 1;
        }
      }
    }
  }
#undef OTTB_BARRIER
#undef OTTB_SWEEP
}

}  // namespace ottb
