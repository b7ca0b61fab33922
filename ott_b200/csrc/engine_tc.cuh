// Tensor-core sweep engine (sm_100a): BF16 split-3 inner products on tcgen05
// with FP32 accumulators in TMEM, followed by the same online base-2
// log-sum-exp as the CUDA-core engine.
//
// Points are stored as bf16 pairs v = hi + lo (hi = bf16(v), lo =
// bf16(v - hi)), rows of DK (64 or 128) elements, hi rows then lo rows; the
// x points carry the exponent scale s = 2 inv log2(e) / eps_target (x' =
// s x before the split), so <x', y> is already in log2 units. A tile is 128
// rows of A by TN = 256 (or 128) columns of B: the three products hi*hi +
// hi*lo + lo*hi accumulate into one TMEM tile (3 * DK / 16 MMAs of M = 128,
// N = TN, K = 16); lo*lo (~2^-16 relative) is dropped. TN = 256 is the
// default because an N = 128 MMA takes ~84 cycles on B200 where an N = 256
// one takes 128 (the full rate; measured with back-to-back MMAs, A in
// shared or tensor memory alike); TN = 128 gives four accumulators instead
// of two and a 4-stage ring, and the autotuner times both. One more K = 16
// MMA adds the shifts: B's extension rows hold the
// column shift w_c = (pot_c - inv |B_c|^2) log2(e) / eps_target as 3 bf16
// terms (~24 bits) and two ones, A's hold three ones and -sigma_r as two
// bf16 terms, so acc = s <a_r, b_c> + w_c - sigma_r, the base-2 exponent of
// the entry less a row shift. w is computed once per point per sweep: every
// potential update writes its point's row of the global extension array
// (write_ext_row), which the producer loads by TMA with the B tile.
//
// Row shifts. A row's log-sum-exp changes between two sweeps of its kind by
// at most D = max_c (change of w_c) (each term moves by its column's change),
// and by at least the smallest change. So when the last sweep of the kind
// ran at the same epsilon and its row log-sum-exps L_r are stored, sigma_r =
// L_r + D bounds every exponent of the row from above (terms <= 1, sums
// <= m), and while the spread of the changes is at most kMaxShiftSpread the
// row sum stays >= 2^-kMaxShiftSpread: the epilogue needs no maxima and no
// rescaling, only 2^acc and the sums. Otherwise (first sweeps, epsilon
// decay, large moves) sigma_r = 0 and the epilogue keeps running maxima.
//
// Warp roles in the 640-thread CTA:
//   warp 0      producer: the row shifts of a unit into A's extension block
//               (all lanes), then (lane 0) the A tile once per unit; B tiles,
//               one 64-wide K chunk (hi and lo) per shared-memory stage, and
//               their column-shift rows with the last chunk, through a ring
//               of kStages stages (TMA, no multicast).
//   warp 1      TMEM owner and MMA issuer (lane 0): two 256-column
//               accumulators (all of TMEM), so MMAs of tile t+1 overlap the
//               epilogue of t.
//   warp 2      dealer: takes the sweep's work units (round-robin or from
//               the sweep's atomic queue) and publishes each as a descriptor
//               in a ring of kDescSlots slots in shared memory.
//   warp 3      finalizer: merges the epilogue's per-row (shift, sum) of a
//               unit, combines column splits and updates the rows'
//               potentials, while the epilogue warps reduce the next unit.
//   warps 4-19  epilogue: warp w reads TMEM lanes 32*(w%4).. (its rows) and
//               the column group (w-4)/4 of each tile and keeps a running
//               (shift, sum) of 2^acc per row.
// Every wait is bounded; a timeout marks the CTA and unwinds.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "tc_ptx.cuh"

namespace ottb {

template <int DK, int TN>
struct TcCfg {
  static constexpr int kChunks = DK / 64;           // 64-wide K chunks (128-byte swizzle atoms)
  static constexpr int kTileN = TN;                 // columns of B per tile (MMA N): 256 or 128
  static constexpr int kABlockBytes = 128 * 64 * 2;    // one [128][64] bf16 block
  static constexpr int kBBlockBytes = kTileN * 64 * 2; // one [256][64] bf16 block
  static constexpr int kABytes = 2 * kChunks * kABlockBytes;  // hi + lo, every chunk
  static constexpr int kStageBytes = 2 * kBBlockBytes;        // hi + lo of one chunk
  static constexpr int kStages = 2 * 256 / TN;      // a 128 KB ring either way
  static constexpr int kTmemBufs = 512 / TN;        // accumulators filling the 512 columns
  static constexpr int kTmemCols = 512;
  static constexpr int kColGroups = 4;    // epilogue warps per TMEM lane quarter
  static constexpr int kColsPerWarp = kTileN / kColGroups;
  static constexpr int kEpiWarps = 4 * kColGroups;
  static constexpr int kCtrlWarps = 4;    // producer, MMA, dealer, finalizer
  static constexpr int kEpiWarp0 = kCtrlWarps;
  static constexpr int kThreads = 32 * (kCtrlWarps + kEpiWarps);
  static constexpr int kDescSlots = 4;    // unit descriptors in flight
  static constexpr uint32_t kIdesc = tc::idesc_bf16_f32(128, kTileN);
  // extension blocks: R rows x 16 bf16, K-major without swizzle: K half 0
  // (elements 0-7) of all rows first, rows 16 B apart (8-row groups 128 B
  // apart), then K half 1 (all zeros) 16 * R bytes on
  static constexpr int kAExtBytes = 128 * 16 * 2;
  static constexpr uint32_t kAExtLbo = 128 * 16;
  static constexpr int kBExtBytes = kTileN * 16 * 2;
  static constexpr int kBExtHalfBytes = kTileN * 16;  // the TMA-loaded K half
  static constexpr uint32_t kBExtLbo = kTileN * 16;
  static constexpr uint32_t kExtSbo = 128;
};

// The bounded row shift of one problem's units in a sweep (see the file
// comment); on = false: sigma = 0 and running maxima.
struct RowShift {
  const float* lprev;  // the rows' log-sum-exps from their last sweep
  float dmax;          // D
  int64_t rows;        // rows of A (padding rows get sigma = 0)
  bool on;
};

// Operands of one tensor-core sweep for one problem.
struct TcOperands {
  const CUtensorMap* mapA;
  const CUtensorMap* mapB;
  const CUtensorMap* mapBext;
  int32_t padA, padB;
  int32_t extRow0;  // first row of B's column-shift rows (g buffer of y)
  int64_t rows, cols;
};

// One work unit of a tensor-core sweep as the epilogue warps deal it to the
// producer and MMA warps: problem (table index), row block, column split
// and tile range, g parity, accumulator scale, operands and row shift; end
// marks the end of the sweep's units for this CTA.
struct TcUnit {
  TcOperands op;
  RowShift rs;
  int p, rb, sidx, S, parity, t0, t1, end;
  float r;
};

template <int DK, int TN>
struct TcSmem {
  // operand tiles first: the struct is placed at a 1024-byte boundary
  uint8_t A[TcCfg<DK, TN>::kABytes];
  uint8_t B[TcCfg<DK, TN>::kStages][TcCfg<DK, TN>::kStageBytes];
  // K = 16 extension blocks, no swizzle: [row groups][2 K halves][8 rows][8]
  uint8_t Aext[TcCfg<DK, TN>::kAExtBytes];
  uint8_t Bext[TcCfg<DK, TN>::kStages][TcCfg<DK, TN>::kBExtBytes];
  TcUnit units[TcCfg<DK, TN>::kDescSlots];  // ring of unit descriptors
  // per-row (shift, sum) of each column group, epilogue -> finalizer,
  // double-buffered by unit
  float part_m[2][TcCfg<DK, TN>::kColGroups][kBM];
  float part_l[2][TcCfg<DK, TN>::kColGroups][kBM];
  uint64_t full[TcCfg<DK, TN>::kStages];
  uint64_t empty[TcCfg<DK, TN>::kStages];
  uint64_t tfull[TcCfg<DK, TN>::kTmemBufs];
  uint64_t tempty[TcCfg<DK, TN>::kTmemBufs];
  uint64_t a_full;
  uint64_t a_empty;
  uint64_t drain;
  uint64_t unit_full[TcCfg<DK, TN>::kDescSlots];   // descriptor written (dealer)
  uint64_t unit_empty[TcCfg<DK, TN>::kDescSlots];  // producer, MMA and finalizer done with it
  uint64_t epi_done[2];   // the epilogue warps wrote part buffer b
  uint64_t part_free[2];  // the finalizer has read part buffer b
  uint32_t tmem_base;
  int err;
};

// Pipeline positions, one copy per thread, advanced identically by every
// role over the same sequence of tiles, K chunks and units.
struct TcPipe {
  uint32_t tile;   // tiles processed so far (all units, all sweeps)
  uint32_t chunk;  // ring stages consumed so far (kChunks per tile)
  uint32_t unit;   // units processed so far
  uint32_t last_full_stage;  // producer: most recent stage issued
  uint32_t last_full_parity;
  int issued;
  uint32_t desc;   // unit descriptors consumed so far (end markers included)
  uint32_t wdesc;  // dealer: unit descriptors written so far
};

// Tensor maps of a problem, stored in global memory: the point sets
// [2 * pad][DK] bf16 (hi rows, then lo rows; box 64 x 128, 128-byte swizzle)
// and their column-shift rows [pad][8] and [2 * pad][8] bf16 (box 8 x 128,
// no swizzle). pad is a multiple of 256, so a B tile never crosses from the
// hi rows into the lo rows.
struct TcMaps {
  CUtensorMap x;
  CUtensorMap y;
  CUtensorMap extx;
  CUtensorMap exty;
};

// A tile: 128 rows, every K chunk, hi and lo ([part][chunk] blocks).
template <int DK, int TN>
__device__ __forceinline__ void tc_load_a(uint8_t* dst, const CUtensorMap* map, uint64_t* bar,
                                          int32_t row, int32_t pad) {
  constexpr int C = TcCfg<DK, TN>::kChunks;
#pragma unroll
  for (int part = 0; part < 2; ++part)
#pragma unroll
    for (int c = 0; c < C; ++c)
      tc::tma_load_2d(dst + (part * C + c) * TcCfg<DK, TN>::kABlockBytes, map, bar, 64 * c,
                      row + part * pad);
}

// One ring stage: K chunk c of 256 B rows from row, hi and lo ([part] blocks
// of 256 rows, each loaded as two 128-row boxes).
template <int DK, int TN>
__device__ __forceinline__ void tc_load_b_chunk(uint8_t* dst, const CUtensorMap* map,
                                                uint64_t* bar, int c, int32_t row, int32_t pad) {
#pragma unroll
  for (int part = 0; part < 2; ++part)
#pragma unroll
    for (int h = 0; h < TN / 128; ++h)
      tc::tma_load_2d(dst + part * TcCfg<DK, TN>::kBBlockBytes + h * TcCfg<DK, TN>::kABlockBytes, map,
                      bar, 64 * c, row + 128 * h + part * pad);
}

// Issues the 3 * 4 MMAs of K chunk c of one tile into the TMEM accumulator
// d_tmem (first = the tile's first MMA, which overwrites the accumulator).
template <int DK, int TN>
__device__ __forceinline__ void tc_issue_chunk(uint32_t d_tmem, const uint8_t* A,
                                               const uint8_t* Bst, int c, bool first) {
  constexpr int C = TcCfg<DK, TN>::kChunks;
  const uint32_t a0 = tc::smem_u32(A), b0 = tc::smem_u32(Bst);
  // (A part, B part): hi*hi, hi*lo, lo*hi
  const int pa[3] = {0, 0, 1};
  const int pb[3] = {0, 1, 0};
  uint32_t acc = first ? 0u : 1u;
#pragma unroll
  for (int prod = 0; prod < 3; ++prod)
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
      const uint64_t ad =
          tc::sw128_kmajor_desc(a0 + (pa[prod] * C + c) * TcCfg<DK, TN>::kABlockBytes + kk * 32);
      const uint64_t bd = tc::sw128_kmajor_desc(b0 + pb[prod] * TcCfg<DK, TN>::kBBlockBytes + kk * 32);
      tc::mma_bf16(d_tmem, ad, bd, TcCfg<DK, TN>::kIdesc, acc);
      acc = 1;
    }
}

// The column-shift MMA: D += Aext * Bext^T over K = 16.
template <int DK, int TN>
__device__ __forceinline__ void tc_issue_ext(uint32_t d_tmem, const uint8_t* Aext,
                                             const uint8_t* Bext) {
  const uint64_t ad = tc::plain_kmajor_desc(tc::smem_u32(Aext), TcCfg<DK, TN>::kAExtLbo,
                                            TcCfg<DK, TN>::kExtSbo);
  const uint64_t bd = tc::plain_kmajor_desc(tc::smem_u32(Bext), TcCfg<DK, TN>::kBExtLbo,
                                            TcCfg<DK, TN>::kExtSbo);
  tc::mma_bf16(d_tmem, ad, bd, TcCfg<DK, TN>::kIdesc, 1);
}


// sigma_r = L_r + D as two bf16 terms (sigma = p1 + p2 exactly in FP32), 0
// for padding rows, rows whose L_r is not finite, or without a bound.
__device__ __forceinline__ float row_shift(const RowShift& rs, int64_t row,
                                           __nv_bfloat16& p1, __nv_bfloat16& p2) {
  float sg = 0.f;
  if (rs.on && row < rs.rows) {
    const float lp = __ldcg(rs.lprev + row);
    if (isfinite(lp)) sg = lp + rs.dmax;
  }
  p1 = __float2bfloat16_rn(sg);
  p2 = __float2bfloat16_rn(sg - __bfloat162float(p1));
  return __bfloat162float(p1) + __bfloat162float(p2);
}

// Of every 8 exponentials of a bounded-shift chunk, this many (even) go to
// exp2_poly2_d4 (FMA pipe), the rest to ex2.approx (MUFU); measured in an
// epilogue-only kernel, 4 of 8 (2019 cycles per tile) is slower than 2
// (1841): the polynomial's issue slots then bind.
#ifndef OTTB_POLY_OF_8_TC_FAST
#define OTTB_POLY_OF_8_TC_FAST 2
#endif



// The three roles of one work unit: rows row0 = u.rb * 128 .. +127 of A
// against B tiles [u.t0, u.t1) of TN columns. Each role advances its own
// copy of the pipeline positions pp over the same sequence of units and
// returns false if one of its waits timed out (after marking sm.err).
//
// Per ring stage st the producer fills one K chunk of B's hi/lo tiles (and,
// with the last chunk, the first K half of B's extension block) by TMA;
// full[st] completes on those bytes, empty[st] on the MMA commit.
// Producer (warp 0, all lanes; lane 0 issues the copies).
template <int DK, int TN>
__device__ bool tc_produce(TcSmem<DK, TN>& sm, TcPipe& pp, const TcUnit& u, uint64_t timeout_ns) {
  constexpr int NS = TcCfg<DK, TN>::kStages;
  constexpr int C = TcCfg<DK, TN>::kChunks;
  const int lane = threadIdx.x & 31;
  const TcOperands& op = u.op;
  const int32_t row0 = u.rb * kBM;
  const int t0 = u.t0;
  const int ntiles = u.t1 - u.t0;
  bool ok = true;
  // A tile and its extension block: wait until the previous unit's MMAs
  // released them, then write the rows' -sigma terms (K columns 3, 4).
  const bool freed = tc::mbar_wait(&sm.a_empty, (pp.unit & 1) ^ 1, timeout_ns);
  if (freed) {
    for (int i = lane; i < kBM; i += 32) {
      __nv_bfloat16 p1, p2;
      row_shift(u.rs, (int64_t)row0 + i, p1, p2);
      __nv_bfloat16* e = reinterpret_cast<__nv_bfloat16*>(sm.Aext + i * 16);
      e[3] = __hneg(p1);
      e[4] = __hneg(p2);
    }
    tc::fence_proxy_async_smem();
  }
  __syncwarp();
  if (lane == 0) {
    if (!freed) ok = false;
    if (ok) {
      tc::mbar_arrive_expect_tx(&sm.a_full, TcCfg<DK, TN>::kABytes);
      tc_load_a<DK, TN>(sm.A, op.mapA, &sm.a_full, row0, op.padA);
    }
    for (int i = 0; ok && i < ntiles; ++i) {
      const int32_t brow = (t0 + i) * TN;
      for (int c = 0; c < C; ++c) {
        const uint32_t g = pp.chunk + i * C + c;
        const uint32_t st = g % NS;
        if (!tc::mbar_wait(&sm.empty[st], ((g / NS) & 1) ^ 1, timeout_ns)) { ok = false; break; }
        const bool last = c == C - 1;
        tc::mbar_arrive_expect_tx(&sm.full[st], TcCfg<DK, TN>::kStageBytes +
                                                    (last ? TcCfg<DK, TN>::kBExtHalfBytes : 0));
        tc_load_b_chunk<DK, TN>(sm.B[st], op.mapB, &sm.full[st], c, brow, op.padB);
        if (last) {
#pragma unroll
          for (int h = 0; h < TN / 128; ++h)
            tc::tma_load_2d(sm.Bext[st] + h * 128 * 16, op.mapBext, &sm.full[st], 0,
                            op.extRow0 + brow + 128 * h);
        }
        pp.last_full_stage = st;
        pp.last_full_parity = (g / NS) & 1;
        pp.issued = 1;
      }
    }
  }
  __syncwarp();
  pp.tile += ntiles;
  pp.chunk += ntiles * C;
  pp.unit += 1;
  if (!ok) atomicExch(&sm.err, 1);
  return ok;
}

// MMA issuer (warp 1, all lanes; lane 0 issues).
template <int DK, int TN>
__device__ bool tc_mma(TcSmem<DK, TN>& sm, TcPipe& pp, const TcUnit& u, uint64_t timeout_ns) {
  constexpr int NS = TcCfg<DK, TN>::kStages;
  constexpr int NB = TcCfg<DK, TN>::kTmemBufs;
  constexpr int C = TcCfg<DK, TN>::kChunks;
  const int lane = threadIdx.x & 31;
  const int ntiles = u.t1 - u.t0;
  bool ok = true;
  if (lane == 0) {
    if (!tc::mbar_wait(&sm.a_full, pp.unit & 1, timeout_ns)) ok = false;
    for (int i = 0; ok && i < ntiles; ++i) {
      const uint32_t gt = pp.tile + i;
      const uint32_t b = gt % NB;
      if (!tc::mbar_wait(&sm.tempty[b], ((gt / NB) & 1) ^ 1, timeout_ns)) { ok = false; break; }
      const uint32_t d = sm.tmem_base + b * TN;
      for (int c = 0; c < C; ++c) {
        const uint32_t g = pp.chunk + i * C + c;
        const uint32_t st = g % NS;
        if (!tc::mbar_wait(&sm.full[st], (g / NS) & 1, timeout_ns)) { ok = false; break; }
        tc::fence_after_sync();
        tc_issue_chunk<DK, TN>(d, sm.A, sm.B[st], c, c == 0);
        if (c == C - 1) tc_issue_ext<DK, TN>(d, sm.Aext, sm.Bext[st]);
        tc::mma_commit(&sm.empty[st]);
      }
      if (!ok) break;
      tc::mma_commit(&sm.tfull[b]);
    }
    if (ok) tc::mma_commit(&sm.a_empty);
  }
  __syncwarp();
  pp.tile += ntiles;
  pp.chunk += ntiles * C;
  pp.unit += 1;
  if (!ok) atomicExch(&sm.err, 1);
  return ok;
}

// Epilogue (warps 4-19): each warp's rows and column group of every tile
// into part buffer (units so far) & 1 of sm.part_m / sm.part_l, handed to
// the finalizer by epi_done.
template <int DK, int TN>
__device__ bool tc_epilogue(TcSmem<DK, TN>& sm, TcPipe& pp, const TcUnit& u,
                            uint64_t timeout_ns) {
  constexpr int NB = TcCfg<DK, TN>::kTmemBufs;
  constexpr int C = TcCfg<DK, TN>::kChunks;
  constexpr int CW = TcCfg<DK, TN>::kColsPerWarp;  // columns per epilogue warp per tile
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  const RowShift& rs = u.rs;
  const int32_t row0 = u.rb * kBM;
  const int ntiles = u.t1 - u.t0;
  const float s = u.r;
  bool ok = true;
  // epilogue: warp e reads TMEM lane quarter q (its 32 rows) and column
  // group cg (CW columns, two 32-column loads) of every tile
  const int e = warp - TcCfg<DK, TN>::kEpiWarp0;
  const int q = warp & 3;
  const int cg = e >> 2;
  const int r = 32 * q + lane;
  float mrun = kNegSentinel, lrun = 0.f, lcmp = 0.f;
  __nv_bfloat16 p1, p2;
  const float sigma = row_shift(rs, (int64_t)row0 + r, p1, p2);
  const bool fast = rs.on;
  for (int i = 0; ok && i < ntiles; ++i) {
    const uint32_t g = pp.tile + i;
    const uint32_t b = g % NB;
    if (!tc::mbar_wait(&sm.tfull[b], (g / NB) & 1, timeout_ns)) {
      ok = false;
      break;
    }
    tc::fence_after_sync();
    if (fast) {
      // acc is the exponent less sigma_r: every term <= 1, no maxima.
      // 16-column loads, the next issued before the current one is
      // reduced; scalar sums into 8 accumulators; the polynomial pairs in
      // packed arithmetic. Measured per 128 x 256 tile in the solve at
      // n = m = 65536: 1808 cycles (2026 with two 32-column loads per
      // tile and packed sums, 2059 before that).
      const uint32_t tb = sm.tmem_base + ((uint32_t)(32 * q) << 16) + b * TN + CW * cg;
      float acc[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) acc[k] = 0.f;
      auto reduce16 = [&](const float (&v)[16]) {
#pragma unroll
        for (int j = 0; j < 16; j += 8) {
#pragma unroll
          for (int k = 0; k < 8; k += 2) {
            if (k >= 8 - OTTB_POLY_OF_8_TC_FAST) {
              float e0, e1;
              unpack2(exp2_poly2_d4(pack2(v[j + k], v[j + k + 1])), e0, e1);
              acc[k] += e0;
              acc[k + 1] += e1;
            } else {
              acc[k] += ex2_approx(v[j + k]);
              acc[k + 1] += ex2_approx(v[j + k + 1]);
            }
          }
        }
      };
      constexpr int NCH = CW / 16;  // 16-column loads per warp and tile (4 or 2)
      static_assert(NCH >= 2 && CW % 16 == 0, "at least two 16-column loads per tile");
      float va[16], vb[16];
      tc::tmem_ld16(tb, va);
      tc::tmem_ld_wait();
#pragma unroll
      for (int c = 0; c + 1 < NCH; ++c) {
        float(&cur)[16] = (c & 1) ? vb : va;
        float(&nxt)[16] = (c & 1) ? va : vb;
        tc::tmem_ld16(tb + 16 * (c + 1), nxt);
        reduce16(cur);
        tc::tmem_ld_wait();
      }
      // The accumulator buffer can be refilled once every warp has read it.
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&sm.tempty[b]);
      reduce16(((NCH - 1) & 1) ? vb : va);
      two_sum_acc(lrun, lcmp,
                  ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7])));
      continue;
    }
#pragma unroll 1
    for (int h = 0; h < CW / 32; ++h) {
      float v[32];
      tc::tmem_ld32(sm.tmem_base + ((uint32_t)(32 * q) << 16) + b * TN + CW * cg + 32 * h, v);
      tc::tmem_ld_wait();
      if (h == CW / 32 - 1) {
        // The accumulator buffer can be refilled once every warp has read it.
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&sm.tempty[b]);
      }
      // tree maximum (depth 4) instead of a 31-step dependent chain
      float t11[11];
#pragma unroll
      for (int j = 0; j < 10; ++j) t11[j] = fmax3(v[3 * j], v[3 * j + 1], v[3 * j + 2]);
      t11[10] = fmaxf(v[30], v[31]);
      const float u0 = fmax3(t11[0], t11[1], t11[2]);
      const float u1 = fmax3(t11[3], t11[4], t11[5]);
      const float u2 = fmax3(t11[6], t11[7], t11[8]);
      const float amax = fmaxf(fmax3(u0, u1, u2), fmaxf(t11[9], t11[10]));
      const float cm = amax * s;  // s > 0
      if (cm > mrun + kTau) {
        const float sc = ex2_approx(mrun - cm);
        lrun *= sc;
        lcmp *= sc;
        mrun = cm;
      }
      const float negm = -mrun;
      // Packed pairs (v[j + 2k], v[j + 2k + 1]) in 4 accumulator pairs; of
      // every 8 columns the last OTTB_POLY_OF_8_TC go to exp2_poly2 (FMA
      // pipe), the rest to ex2.approx (MUFU).
      const f32x2 s2 = pack2(s, s), m2 = pack2(negm, negm);
      f32x2 acc[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) acc[k] = 0ull;
#pragma unroll
      for (int j = 0; j < 32; j += 8) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const f32x2 x = fma2(pack2(v[j + 2 * k], v[j + 2 * k + 1]), s2, m2);
          f32x2 e;
          if (2 * k >= 8 - OTTB_POLY_OF_8_TC) {
            e = exp2_poly2(x);
          } else {
            float x0, x1;
            unpack2(x, x0, x1);
            e = pack2(ex2_approx(x0), ex2_approx(x1));
          }
          acc[k] = add2(acc[k], e);
        }
      }
      float ta, tb;
      unpack2(add2(add2(acc[0], acc[1]), add2(acc[2], acc[3])), ta, tb);
      two_sum_acc(lrun, lcmp, ta + tb);
    }
  }
  // the part buffer is free once the finalizer has read it two units ago
  const uint32_t pb = pp.unit & 1;
  if (ok && pp.unit >= 2 &&
      !tc::mbar_wait(&sm.part_free[pb], ((pp.unit - 2) >> 1) & 1, timeout_ns))
    ok = false;
  sm.part_m[pb][cg][r] = fast ? sigma : mrun;
  sm.part_l[pb][cg][r] = lrun + lcmp;
  __syncwarp();
  if (ok && lane == 0) tc::mbar_arrive(&sm.epi_done[pb]);
  pp.tile += ntiles;
  pp.chunk += ntiles * C;
  pp.unit += 1;
  if (!ok) atomicExch(&sm.err, 1);
  return ok;
}

}  // namespace ottb
