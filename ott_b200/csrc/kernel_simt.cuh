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

__device__ __forceinline__ int ld_sched(const int* p) { return *(const volatile int*)p; }

// Runs one sweep over the units of the scheduled problems. Every CTA calls
// it; units are dealt round-robin (one problem) or from an atomic queue.
template <int DP>
__device__ void simt_sweep(const KernelArgs& A, SimtKernelSmem<DP>& sm,
                           const SweepParams& sp, unsigned sweep_idx) {
  const int* ids = sp.final_eval ? A.eval_ids : A.active_ids;
  const int* pre = sp.final_eval ? A.eval_prefix
                                 : (A.prefix + (sp.kind == kSweepG ? 0 : A.num_problems + 1));
  const int count = sp.final_eval ? ld_sched(&A.sched->num_eval)
                                  : ld_sched(&A.sched->num_active);
  const int total = sp.final_eval ? ld_sched(&A.sched->eval_units)
                                  : ld_sched(&A.sched->total_units[sp.kind == kSweepG ? 0 : 1]);
  unsigned* ctr = &A.gl->unit_ctr[sweep_idx % 3];
  if (blockIdx.x == 0 && threadIdx.x == 0) A.gl->unit_ctr[(sweep_idx + 1) % 3] = 0u;

  int u = blockIdx.x;
  if (A.dynamic_units) {
    if (threadIdx.x == 0) sm.unit = (int)atomicAdd(ctr, 1u);
    __syncthreads();
    u = sm.unit;
    __syncthreads();
  }
  while (u < total) {
    const int q = find_problem(pre, count, u);
    const int p = __ldcg(ids + q);
    const ProbDev& P = A.probs[p];
    const int local = u - __ldcg(pre + q);
    const int S = sp.kind == kSweepG ? P.split_g : P.split_f;
    const int rb = local / S;
    const int sidx = local % S;
    const int parity = sp.final_eval ? __ldcg(&A.state[p].final_parity) : sp.parity;
    const float* gcur = P.gbuf[parity];
    SweepOperands op = make_operands(P, sp.kind, gcur);
    const int ntiles = (int)((op.cols + kBN - 1) / kBN);
    const int t0 = (int)(((int64_t)ntiles * sidx) / S);
    const int t1 = (int)(((int64_t)ntiles * (sidx + 1)) / S);
    const float wscale = sweep_wscale(P, sp.mult);
    const float s = 2.0f * P.inv_scale * wscale;

    simt_unit<DP>(sm.tiles, op, (int64_t)rb * kBM, t0, t1, s, wscale, sm.rm, sm.rl);

    bool do_final = true;
    if (S > 1) {
      const int64_t R = op.rows;
      const int64_t rbase = (int64_t)rb * kBM;
      for (int t = threadIdx.x; t < kBM; t += blockDim.x) {
        if (rbase + t < R) {
          P.part_m[(int64_t)sidx * R + rbase + t] = sm.rm[t];
          P.part_l[(int64_t)sidx * R + rbase + t] = sm.rl[t];
        }
      }
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) {
        int prev = atomicAdd(&P.arrive[rb], 1);
        sm.last = (prev == S - 1);
        if (sm.last) atomicExch(&P.arrive[rb], 0);
      }
      __syncthreads();
      do_final = sm.last != 0;
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
          sm.rm[t] = mv;
          sm.rl[t] = lv;
        }
        __syncthreads();
      }
    }
    if (do_final) finalize_rows(P, sp, parity, rb, sm.rm, sm.rl, A.cfg.norm_error, sm.red);
    __syncthreads();

    if (A.dynamic_units) {
      if (threadIdx.x == 0) sm.unit = (int)atomicAdd(ctr, 1u);
      __syncthreads();
      u = sm.unit;
      __syncthreads();
    } else {
      u += gridDim.x;
    }
  }
}

template <int DP>
__global__ void __launch_bounds__(256, (DP <= 2 ? 2 : 1))
sinkhorn_simt_kernel(KernelArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SimtKernelSmem<DP>& sm = *reinterpret_cast<SimtKernelSmem<DP>*>(smem_raw);
  const ottb_solver_cfg& c = A.cfg;
  const int inner = c.inner_iterations;
  const bool force_scan = c.min_iterations == c.max_iterations;
  const int scan_end = force_scan ? (c.max_iterations / inner) * inner : c.max_iterations;
  int* status = &A.sched->status;
  unsigned sweep_idx = 0;
  int it = 0;
  int commits = 0;  // committed g-sweeps; identical in every CTA

#define OTTB_BARRIER()                                                          \
  do {                                                                          \
    if (!grid_barrier(A.gl, A.expected_arrivals, A.timeout_ns, status)) return; \
  } while (0)

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
        simt_sweep<DP>(A, sm, sp, sweep_idx++);
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
      simt_sweep<DP>(A, sm, sp, sweep_idx++);
      OTTB_BARRIER();
      ++commits;
    }
    {
      SweepParams sp{kSweepF, mlt, 0, 1, 0, commits & 1};
      simt_sweep<DP>(A, sm, sp, sweep_idx++);
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
    simt_sweep<DP>(A, sm, sp, sweep_idx++);
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
}

}  // namespace ottb
