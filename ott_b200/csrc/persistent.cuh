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

__device__ __forceinline__ int units_of(const ProbDev& P, int kind) {
  return kind == kSweepG ? P.rb_g * P.split_g : P.rb_f * P.split_f;
}

// CTA 0 only: rebuild the active list and unit prefix sums.
__device__ void rebuild_schedule(const KernelArgs& A) {
  if (threadIdx.x == 0) {
    int na = 0, ug = 0, uf = 0;
    for (int p = 0; p < A.num_problems; ++p) {
      if (!A.state[p].active) continue;
      A.active_ids[na] = p;
      A.prefix[na] = ug;
      A.prefix[A.num_problems + 1 + na] = uf;
      ug += units_of(A.probs[p], kSweepG);
      uf += units_of(A.probs[p], kSweepF);
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
      ue += units_of(A.probs[p], kSweepG);
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

}  // namespace ottb
