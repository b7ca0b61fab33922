// Tensor-core sweep engine (sm_100a): BF16 split-3 inner products on tcgen05
// with FP32 accumulators in TMEM, followed by the same online base-2
// log-sum-exp as the CUDA-core engine.
//
// Points are stored as bf16 pairs v = hi + lo (hi = bf16(v), lo =
// bf16(v - hi)), rows of DK (64 or 128) elements, hi rows then lo rows. For a
// 128 x 128 tile the three products hi*hi + hi*lo + lo*hi accumulate into one
// TMEM tile (3 * DK / 16 MMAs of M = N = 128, K = 16); lo*lo (~2^-16
// relative) is dropped. One more K = 16 MMA adds the column shift: A's
// extension block holds ones in its first 3 K columns, B's holds
// w'_c = (pot_c - inv |B_c|^2) / (2 inv) as 3 bf16 terms (~24 bits), so the
// accumulator is acc = <a_r, b_c> + w'_c and the exponent is s * acc,
// s = 2 inv log2(e) / eps. The epilogue needs no per-column data.
//
// Warp roles in the 576-thread CTA:
//   warp 0      producer: A tile once per unit; B tiles through a ring of
//               kStages shared-memory stages (TMA, no multicast), and each
//               stage's w' extension block.
//   warp 1      TMEM owner and MMA issuer (lane 0): two 128-column
//               accumulators, so MMAs of tile t+1 overlap the epilogue of t.
//   warps 2-17  epilogue: warp w reads TMEM lanes 32*(w%4).. (its rows) and
//               the 32-column group (w-2)/4 of each tile and keeps a running
//               (max, sum) of 2^(s * acc) per row.
// Every wait is bounded; a timeout marks the CTA and unwinds.
#pragma once

#include <cuda_bf16.h>

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
  static constexpr int kColGroups = 4;    // epilogue warps per TMEM lane quarter
  static constexpr int kEpiWarps = 4 * kColGroups;
  static constexpr int kThreads = 64 + 32 * kEpiWarps;
  static constexpr uint32_t kIdesc = tc::idesc_bf16_f32(128, 128);
  // extension block: 128 rows x 16 bf16, 8-row groups 256 B apart, K halves
  // 128 B apart, rows 16 B apart
  static constexpr int kExtBytes = 128 * 16 * 2;
  static constexpr uint32_t kExtLbo = 128;
  static constexpr uint32_t kExtSbo = 256;
};

// Byte offset of element (row, k) in an extension block.
__device__ __forceinline__ int ext_offset(int row, int k) {
  return (row >> 3) * 256 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

template <int DK>
struct TcSmem {
  // operand tiles first: the struct is placed at a 1024-byte boundary
  uint8_t A[TcCfg<DK>::kOperandBytes];
  uint8_t B[TcCfg<DK>::kStages][TcCfg<DK>::kOperandBytes];
  // K = 16 extension blocks, no swizzle: [16 row groups][2 K halves][8 rows][8]
  uint8_t Aext[TcCfg<DK>::kExtBytes];
  uint8_t Bext[TcCfg<DK>::kStages][TcCfg<DK>::kExtBytes];
  float part_m[TcCfg<DK>::kColGroups][kBM];
  float part_l[TcCfg<DK>::kColGroups][kBM];
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

// The column-shift MMA: D += Aext * Bext^T over K = 16.
template <int DK>
__device__ __forceinline__ void tc_issue_ext(uint32_t d_tmem, const uint8_t* Aext,
                                             const uint8_t* Bext) {
  const uint64_t ad = tc::plain_kmajor_desc(tc::smem_u32(Aext), TcCfg<DK>::kExtLbo,
                                            TcCfg<DK>::kExtSbo);
  const uint64_t bd = tc::plain_kmajor_desc(tc::smem_u32(Bext), TcCfg<DK>::kExtLbo,
                                            TcCfg<DK>::kExtSbo);
  tc::mma_bf16(d_tmem, ad, bd, TcCfg<DK>::kIdesc, 1);
}

// w' split into three bf16 terms, written at K = 0, 1, 2 of row `row`
// (K = 3..15 stay zero).
// A non-finite w' (padding columns and zero-weight potentials are -inf) is
// carried by the first term alone, so no inf - inf = NaN appears.
__device__ __forceinline__ void write_ext_shift(uint8_t* blk, int row, float w) {
  const bool fin = isfinite(w);
  const __nv_bfloat16 w1 = __float2bfloat16_rn(w);
  const float r1 = fin ? w - __bfloat162float(w1) : 0.f;
  const __nv_bfloat16 w2 = __float2bfloat16_rn(r1);
  const __nv_bfloat16 w3 = __float2bfloat16_rn(fin ? r1 - __bfloat162float(w2) : 0.f);
  __nv_bfloat162 p01;
  p01.x = w1;
  p01.y = w2;
  __nv_bfloat162 p23;
  p23.x = w3;
  p23.y = __float2bfloat16_rn(0.f);
  *reinterpret_cast<__nv_bfloat162*>(blk + ext_offset(row, 0)) = p01;
  *reinterpret_cast<__nv_bfloat162*>(blk + ext_offset(row, 2)) = p23;
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
//
// Per ring stage st the producer warp fills B's hi/lo tiles (TMA) and the
// stage's w' extension block (plain loads of pot and |B|^2 one tile ahead in
// registers, generic stores, then an async-proxy fence); full[st] completes
// on the TMA bytes plus 32 lane arrivals, empty[st] on the MMA commit.
// wshift = 1 / (2 inv).
template <int DK>
__device__ bool tc_unit(TcSmem<DK>& sm, TcPipe& pp, const TcOperands& op, int32_t row0,
                        int t0, int t1, float s, float wshift, uint64_t timeout_ns) {
  constexpr int NS = TcCfg<DK>::kStages;
  constexpr int NB = TcCfg<DK>::kTmemBufs;
  constexpr int CG = TcCfg<DK>::kColGroups;
  constexpr int CW = kBN / CG;  // columns per epilogue warp per tile
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const int ntiles = t1 - t0;
  bool ok = true;

  if (warp == 0) {
    // w' of the first tile, 4 columns per lane
    float wreg[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int64_t c = (int64_t)t0 * kBN + lane + 32 * k;
      wreg[k] = c < op.cols ? (__ldcg(op.potB + c) - op.nb[c]) * wshift : -INFINITY;
    }
    if (lane == 0) {
      // A tile: wait until the previous unit's MMAs released it.
      if (!tc::mbar_wait(&sm.a_empty, (pp.unit & 1) ^ 1, timeout_ns)) ok = false;
      if (ok) {
        tc::mbar_arrive_expect_tx(&sm.a_full, TcCfg<DK>::kOperandBytes);
        tc_load_operand<DK>(sm.A, op.mapA, &sm.a_full, row0, op.padA);
      }
    }
    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    for (int i = 0; ok && i < ntiles; ++i) {
      const uint32_t g = pp.tile + i;
      const uint32_t st = g % NS;
      const bool got = tc::mbar_wait(&sm.empty[st], ((g / NS) & 1) ^ 1, timeout_ns);
      if (!__all_sync(0xffffffffu, got)) {
        ok = false;
        break;
      }
      if (lane == 0) {
        tc::mbar_expect_tx(&sm.full[st], TcCfg<DK>::kOperandBytes);
        tc_load_operand<DK>(sm.B[st], op.mapB, &sm.full[st], (t0 + i) * kBN, op.padB);
        pp.last_full_stage = st;
        pp.last_full_parity = (g / NS) & 1;
        pp.issued = 1;
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) write_ext_shift(sm.Bext[st], lane + 32 * k, wreg[k]);
      tc::fence_proxy_async_smem();
      tc::mbar_arrive(&sm.full[st]);
      if (i + 1 < ntiles) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int64_t c = (int64_t)(t0 + i + 1) * kBN + lane + 32 * k;
          wreg[k] = c < op.cols ? (__ldcg(op.potB + c) - op.nb[c]) * wshift : -INFINITY;
        }
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
        const uint32_t d = sm.tmem_base + b * 128;
        tc_issue_tile<DK>(d, sm.A, sm.B[st]);
        tc_issue_ext<DK>(d, sm.Aext, sm.Bext[st]);
        tc::mma_commit(&sm.empty[st]);
        tc::mma_commit(&sm.tfull[b]);
      }
      if (ok) tc::mma_commit(&sm.a_empty);
    }
    __syncwarp();
  } else {
    // epilogue: warp e reads TMEM lane quarter q (its 32 rows) and column
    // group cg (CW columns) of every tile
    const int e = warp - 2;
    const int q = warp & 3;
    const int cg = e >> 2;
    const int r = 32 * q + lane;
    float mrun = kNegSentinel, lrun = 0.f, lcmp = 0.f;
    for (int i = 0; ok && i < ntiles; ++i) {
      const uint32_t g = pp.tile + i;
      const uint32_t b = g % NB;
      if (!tc::mbar_wait(&sm.tfull[b], (g / NB) & 1, timeout_ns)) {
        ok = false;
        break;
      }
      tc::fence_after_sync();
      float v[CW];
      tc::tmem_ld32(sm.tmem_base + ((uint32_t)(32 * q) << 16) + b * 128 + CW * cg, v);
      tc::tmem_ld_wait();
      // The accumulator buffer can be refilled once every warp has read it.
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&sm.tempty[b]);
      float amax = v[0];
#pragma unroll
      for (int j = 1; j < CW; ++j) amax = fmaxf(amax, v[j]);
      const float cm = amax * s;  // s > 0
      if (cm > mrun + kTau) {
        const float sc = ex2_approx(mrun - cm);
        lrun *= sc;
        lcmp *= sc;
        mrun = cm;
      }
      const float negm = -mrun;
      float acc4[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int j = 0; j < CW; j += 4) {
        acc4[0] += ex2_approx(fmaf(v[j], s, negm));
        acc4[1] += ex2_approx(fmaf(v[j + 1], s, negm));
        acc4[2] += ex2_approx(fmaf(v[j + 2], s, negm));
        acc4[3] += ex2_approx(fmaf(v[j + 3], s, negm));
      }
      two_sum_acc(lrun, lcmp, (acc4[0] + acc4[1]) + (acc4[2] + acc4[3]));
    }
    sm.part_m[cg][r] = mrun;
    sm.part_l[cg][r] = lrun + lcmp;
  }
  pp.tile += ntiles;
  pp.unit += 1;
  if (!ok) atomicExch(&sm.err, 1);
  __syncthreads();
  if (threadIdx.x < kBM) {
    float mv = sm.part_m[0][threadIdx.x], lv = sm.part_l[0][threadIdx.x];
#pragma unroll
    for (int k = 1; k < CG; ++k) lse_merge(mv, lv, sm.part_m[k][threadIdx.x], sm.part_l[k][threadIdx.x]);
    sm.rm[threadIdx.x] = mv;
    sm.rl[threadIdx.x] = lv;
  }
  __syncthreads();
  return sm.err == 0;
}

}  // namespace ottb
