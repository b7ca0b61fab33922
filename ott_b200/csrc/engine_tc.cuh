// Tensor-core sweep engine (sm_100a): BF16 split-3 inner products on tcgen05
// with FP32 accumulators in TMEM, followed by the same online base-2
// log-sum-exp as the CUDA-core engine.
//
// Points are stored as bf16 pairs v = hi + lo (hi = bf16(v), lo =
// bf16(v - hi)), rows of DK (64 or 128) elements, hi rows then lo rows. For a
// 128 x 128 tile the three products hi*hi + hi*lo + lo*hi accumulate into one
// TMEM tile (3 * DK / 16 MMAs of M = N = 128, K = 16); lo*lo (~2^-16
// relative) is dropped.
//
// Warp roles in the 320-thread CTA:
//   warp 0      TMA producer: A tile once per unit, B tiles through a ring of
//               kStages shared-memory stages (no multicast).
//   warp 1      TMEM owner and MMA issuer (lane 0): two 128-column
//               accumulators, so MMAs of tile t+1 overlap the epilogue of t.
//   warps 2-9   epilogue: warp w reads TMEM lanes 32*(w%4).. (its rows) and
//               the column half (w-2)/4 of each tile, computes
//               t = s*acc + w_c, and keeps a running (max, sum) per row.
// Every wait is bounded; a timeout marks the CTA and unwinds.
#pragma once

#include "common.cuh"
#include "tc_ptx.cuh"

namespace ottb {

template <int DK>
struct TcCfg {
  static constexpr int kChunks = DK / 64;                 // 128-byte swizzle atoms along K
  static constexpr int kBlockBytes = 128 * 64 * 2;        // one [128][64] bf16 block
  static constexpr int kOperandBytes = 2 * kChunks * kBlockBytes;  // hi + lo
  static constexpr int kStages = DK <= 64 ? 4 : 2;
  static constexpr int kTmemBufs = 2;
  static constexpr int kTmemCols = 256;
  static constexpr int kThreads = 320;
  static constexpr int kEpiThreads = 256;
  static constexpr uint32_t kIdesc = tc::idesc_bf16_f32(128, 128);
};

template <int DK>
struct TcSmem {
  // operand tiles first: the struct is placed at a 1024-byte boundary
  uint8_t A[TcCfg<DK>::kOperandBytes];
  uint8_t B[TcCfg<DK>::kStages][TcCfg<DK>::kOperandBytes];
  float ws[2][kBN];
  float part_m[2][kBM];
  float part_l[2][kBM];
  float rm[kBM];
  float rl[kBM];
  double red[8];
  uint64_t full[TcCfg<DK>::kStages];
  uint64_t empty[TcCfg<DK>::kStages];
  uint64_t tfull[TcCfg<DK>::kTmemBufs];
  uint64_t tempty[TcCfg<DK>::kTmemBufs];
  uint64_t a_full;
  uint64_t a_empty;
  uint64_t drain;
  uint32_t tmem_base;
  int unit;
  int last;
  int err;
};

// Pipeline positions, one copy per thread, advanced identically by every
// role over the same sequence of tiles and units.
struct TcPipe {
  uint32_t tile;   // tiles processed so far (all units, all sweeps)
  uint32_t unit;   // units processed so far
  uint32_t last_full_stage;  // producer: most recent stage issued
  uint32_t last_full_parity;
  int issued;
};

// Tensor maps of a problem's point sets, [2 * pad][DK] bf16 (hi rows, then
// lo rows), box 64 x 128, 128-byte swizzle. Stored in global memory.
struct TcMaps {
  CUtensorMap x;
  CUtensorMap y;
};

template <int DK>
__device__ __forceinline__ void tc_load_operand(uint8_t* dst, const CUtensorMap* map,
                                                uint64_t* bar, int32_t row, int32_t pad) {
  constexpr int C = TcCfg<DK>::kChunks;
#pragma unroll
  for (int part = 0; part < 2; ++part)
#pragma unroll
    for (int c = 0; c < C; ++c)
      tc::tma_load_2d(dst + (part * C + c) * TcCfg<DK>::kBlockBytes, map, bar, 64 * c,
                      row + part * pad);
}

// Issues the 3 * DK / 16 MMAs of one tile into the TMEM accumulator d_tmem.
template <int DK>
__device__ __forceinline__ void tc_issue_tile(uint32_t d_tmem, const uint8_t* A, const uint8_t* B) {
  constexpr int C = TcCfg<DK>::kChunks;
  constexpr int BB = TcCfg<DK>::kBlockBytes;
  const uint32_t a0 = tc::smem_u32(A), b0 = tc::smem_u32(B);
  // (A part, B part): hi*hi, hi*lo, lo*hi
  const int pa[3] = {0, 0, 1};
  const int pb[3] = {0, 1, 0};
  uint32_t acc = 0;
#pragma unroll
  for (int prod = 0; prod < 3; ++prod)
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const uint64_t ad = tc::sw128_kmajor_desc(a0 + (pa[prod] * C + c) * BB + kk * 32);
        const uint64_t bd = tc::sw128_kmajor_desc(b0 + (pb[prod] * C + c) * BB + kk * 32);
        tc::mma_bf16(d_tmem, ad, bd, TcCfg<DK>::kIdesc, acc);
        acc = 1;
      }
}

// Operands of one tensor-core sweep for one problem.
struct TcOperands {
  const CUtensorMap* mapA;
  const CUtensorMap* mapB;
  int32_t padA, padB;
  const float* potB;
  const float* nb;
  int64_t rows, cols;
};

// One work unit: rows row0..row0+127 of A against B tiles [t0, t1).
// Leaves the per-row base-2 LSE state in sm.rm / sm.rl. Returns false if a
// wait timed out.
template <int DK>
__device__ bool tc_unit(TcSmem<DK>& sm, TcPipe& pp, const TcOperands& op, int32_t row0,
                        int t0, int t1, float s, float wscale, uint64_t timeout_ns) {
  constexpr int NS = TcCfg<DK>::kStages;
  constexpr int NB = TcCfg<DK>::kTmemBufs;
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int ntiles = t1 - t0;
  bool ok = true;

  if (warp == 0) {
    if (lane == 0) {
      // A tile: wait until the previous unit's MMAs released it.
      if (!tc::mbar_wait(&sm.a_empty, (pp.unit & 1) ^ 1, timeout_ns)) ok = false;
      if (ok) {
        tc::mbar_arrive_expect_tx(&sm.a_full, TcCfg<DK>::kOperandBytes);
        tc_load_operand<DK>(sm.A, op.mapA, &sm.a_full, row0, op.padA);
      }
      for (int i = 0; ok && i < ntiles; ++i) {
        const uint32_t g = pp.tile + i;
        const uint32_t st = g % NS;
        if (!tc::mbar_wait(&sm.empty[st], ((g / NS) & 1) ^ 1, timeout_ns)) { ok = false; break; }
        tc::mbar_arrive_expect_tx(&sm.full[st], TcCfg<DK>::kOperandBytes);
        tc_load_operand<DK>(sm.B[st], op.mapB, &sm.full[st], (t0 + i) * kBN, op.padB);
        pp.last_full_stage = st;
        pp.last_full_parity = (g / NS) & 1;
        pp.issued = 1;
      }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      if (!tc::mbar_wait(&sm.a_full, pp.unit & 1, timeout_ns)) ok = false;
      for (int i = 0; ok && i < ntiles; ++i) {
        const uint32_t g = pp.tile + i;
        const uint32_t st = g % NS;
        const uint32_t b = g % NB;
        if (!tc::mbar_wait(&sm.full[st], (g / NS) & 1, timeout_ns)) { ok = false; break; }
        if (!tc::mbar_wait(&sm.tempty[b], ((g / NB) & 1) ^ 1, timeout_ns)) { ok = false; break; }
        tc::fence_after_sync();
        tc_issue_tile<DK>(sm.tmem_base + b * 128, sm.A, sm.B[st]);
        tc::mma_commit(&sm.empty[st]);
        tc::mma_commit(&sm.tfull[b]);
      }
      if (ok) tc::mma_commit(&sm.a_empty);
    }
    __syncwarp();
  } else {
    // epilogue
    const int e = warp - 2;          // 0..7
    const int q = warp & 3;          // TMEM lane quarter this warp may access
    const int h = e >> 2;            // column half of each tile
    const int etid = threadIdx.x - 64;
    const int r = 32 * q + lane;     // row within the unit
    float mrun = kNegSentinel, lrun = 0.f, lcmp = 0.f;
    float wnext = -INFINITY;
    if (etid < kBN) {
      const int64_t c = (int64_t)t0 * kBN + etid;
      if (c < op.cols) wnext = (__ldcg(op.potB + c) - op.nb[c]) * wscale;
    }
    for (int i = 0; i < ntiles; ++i) {
      const uint32_t g = pp.tile + i;
      const uint32_t b = g % NB;
      const int wslot = i & 1;
      if (etid < kBN) sm.ws[wslot][etid] = wnext;
      asm volatile("bar.sync 1, 256;" ::: "memory");
      if (etid < kBN && i + 1 < ntiles) {
        const int64_t c = (int64_t)(t0 + i + 1) * kBN + etid;
        wnext = c < op.cols ? (__ldcg(op.potB + c) - op.nb[c]) * wscale : -INFINITY;
      }
      if (ok && !tc::mbar_wait(&sm.tfull[b], (g / NB) & 1, timeout_ns)) ok = false;
      if (ok) {
        tc::fence_after_sync();
        const uint32_t taddr = sm.tmem_base + ((uint32_t)(32 * q) << 16) + b * 128 + 64 * h;
        float v0[32], v1[32];
        tc::tmem_ld32(taddr, v0);
        tc::tmem_ld32(taddr + 32, v1);
        tc::tmem_ld_wait();
        const float* wv = &sm.ws[wslot][64 * h];
        float cm = kNegSentinel;
#pragma unroll
        for (int j = 0; j < 32; j += 4) {
          const float4 w4 = *reinterpret_cast<const float4*>(wv + j);
          v0[j] = fmaf(v0[j], s, w4.x);
          v0[j + 1] = fmaf(v0[j + 1], s, w4.y);
          v0[j + 2] = fmaf(v0[j + 2], s, w4.z);
          v0[j + 3] = fmaf(v0[j + 3], s, w4.w);
          cm = fmaxf(cm, fmaxf(fmaxf(v0[j], v0[j + 1]), fmaxf(v0[j + 2], v0[j + 3])));
        }
#pragma unroll
        for (int j = 0; j < 32; j += 4) {
          const float4 w4 = *reinterpret_cast<const float4*>(wv + 32 + j);
          v1[j] = fmaf(v1[j], s, w4.x);
          v1[j + 1] = fmaf(v1[j + 1], s, w4.y);
          v1[j + 2] = fmaf(v1[j + 2], s, w4.z);
          v1[j + 3] = fmaf(v1[j + 3], s, w4.w);
          cm = fmaxf(cm, fmaxf(fmaxf(v1[j], v1[j + 1]), fmaxf(v1[j + 2], v1[j + 3])));
        }
        // The accumulator buffer can be refilled once every warp has read it.
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&sm.tempty[b]);
        if (cm > mrun + kTau) {
          const float sc = ex2_approx(mrun - cm);
          lrun *= sc;
          lcmp *= sc;
          mrun = cm;
        }
        // 64 terms: 8 accumulators of 8 terms, then a tree.
        float acc8[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) acc8[k] = 0.f;
#pragma unroll
        for (int j = 0; j < 32; j += 4) {
          acc8[0] += ex2_approx(v0[j] - mrun);
          acc8[1] += ex2_approx(v0[j + 1] - mrun);
          acc8[2] += ex2_approx(v0[j + 2] - mrun);
          acc8[3] += ex2_approx(v0[j + 3] - mrun);
          acc8[4] += ex2_approx(v1[j] - mrun);
          acc8[5] += ex2_approx(v1[j + 1] - mrun);
          acc8[6] += ex2_approx(v1[j + 2] - mrun);
          acc8[7] += ex2_approx(v1[j + 3] - mrun);
        }
        const float tile_sum = ((acc8[0] + acc8[1]) + (acc8[2] + acc8[3])) +
                               ((acc8[4] + acc8[5]) + (acc8[6] + acc8[7]));
        two_sum_acc(lrun, lcmp, tile_sum);
      }
    }
    sm.part_m[h][r] = mrun;
    sm.part_l[h][r] = lrun + lcmp;
  }
  pp.tile += ntiles;
  pp.unit += 1;
  if (!ok) atomicExch(&sm.err, 1);
  __syncthreads();
  if (threadIdx.x < kBM) {
    float mv = sm.part_m[0][threadIdx.x], lv = sm.part_l[0][threadIdx.x];
    lse_merge(mv, lv, sm.part_m[1][threadIdx.x], sm.part_l[1][threadIdx.x]);
    sm.rm[threadIdx.x] = mv;
    sm.rl[threadIdx.x] = lv;
  }
  __syncthreads();
  return sm.err == 0;
}

}  // namespace ottb
