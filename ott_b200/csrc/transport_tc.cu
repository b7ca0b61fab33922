// Transport plan applied to many vectors on the tensor cores
// (geometry/geometry.py:444-486, apply_transport_from_potentials):
//
//   P_ij = exp((f_i + g_j - inv |x_i - y_j|^2) / eps)
//   axis 1: out[k][i] = sum_j P_ij vec[k][j]     axis 0: out[k][j] = sum_i P_ij vec[k][i]
//
// A is the output side (x for axis 1), B the summed side. Both products of
// the application are tcgen05 MMAs with FP32 accumulators in TMEM, in BF16
// split-3 form (v = hi + lo, hi*hi + hi*lo + lo*hi):
//   S = s <A_r, B_c> + w_c - sigma_r      (M = 128 rows, N = 128 columns, K = d,
//                                          + one K = 16 MMA for the shifts)
//   O += 2^S V^T                           (M = 128 rows, N = vectors, K = 128 columns)
// The second product's split is two MMAs per K slab, not three: the hi and
// lo rows of V are stacked along N, so P_hi [V_hi | V_lo] fills two
// accumulator halves at once, P_lo V_hi adds into the first, and O is the
// sum of the halves (an MMA costs about the same from N = 16 to N = 128).
// with s = 2 inv log2(e) / eps on A's centred points, w_c = (g_c - inv |B_c|^2)
// log2(e) / eps and sigma_r the row's largest exponent s <A_r, B_c> + w_c,
// which a first pass of the same kernel provides (MAXP: the hi*hi product
// and the shift block only, 5 MMAs a tile instead of 13 at d <= 64, row
// maxima instead of weights, combined across column splits with an integer
// atomicMax). Its products drop the hi*lo and lo*hi terms, so its maxima
// are good to about one log2 unit; the weights need no more: with that
// shift every weight 2^S of a row is at most a few units, no row sum
// overflows, no running maximum or rescale is needed, and out =
// 2^(u_r + sigma_r) O_r with u_r = (f_r - inv |A_r|^2) log2(e) / eps,
// applied once per row with the sigma_r the weights were formed with.
//
// The weights never leave the SM: each epilogue thread owns one TMEM lane
// (one row), reads its 32 columns of S, and writes 2^S back into the same
// 32 columns as bf16 pairs, hi then lo (the 16-column K slab j of the tile
// in columns 32 (j / 2) + 8 (j % 2) (hi) and + 16 (lo)), so the second MMA
// takes P straight from tensor memory as its A operand. Two S/P buffers
// (TMEM columns 0-255) let the MMAs of tile t + 1 run while the epilogue
// turns tile t into weights; O's two halves take columns 256 up to 256 +
// 2 * 96. (Measured at n = m = 65536, d = 64, 65 vectors: a third S/P
// buffer, or loading the next tile's S before forming the current tile's
// weights, made the kernel slower; stacking V's hi and lo rows saved a
// quarter of its time.)
//
// Warp roles in the 608-thread CTA (one work unit: a 128-row block, a
// range of 128-column tiles, a chunk of up to 96 vectors):
//   warp 0      producer of the rows' shift block, the A tile and per tile
//               B (one 64-wide K chunk, hi and lo, per ring stage) with its
//               shift rows (TMA, no multicast).
//   warp 1      TMEM owner and MMA issuer (lane 0): S of tile t, then the
//               P V MMAs of tile t - 1.
//   warp 2      producer of V's hi and lo rows of the vector chunk, per tile.
//   warps 3-18  epilogue: warp w reads TMEM lanes 32 (w % 4).. and the
//               column group (w - 3) / 4 of each tile; at the end the same
//               warps scale O and write it out (or a column split's part).
// Every wait is bounded; a timeout sets the error flag, the producers wait
// (again bounded) for their copies in flight, and the CTA unwinds.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../../include/ott_b200.h"
#include "common.cuh"
#include "launch.cuh"
#include "tc_ptx.cuh"
#include "tmap.cuh"

namespace ottb {
namespace {

constexpr int kAtcRows = 128;      // output rows per unit (MMA M)
constexpr int kAtcCols = 128;      // summed columns per tile (S's N, P V's K)
constexpr int kAtcWarps = 19;
constexpr int kAtcThreads = 32 * kAtcWarps;
constexpr int kAtcEpiWarp0 = 3;
constexpr int kAtcSBufs = 2;       // S/P buffers in TMEM (128 columns each)
constexpr int kAtcStages = 2;      // B ring (one 64-wide K chunk per stage)
constexpr int kAtcVStages = 2;     // V ring (one tile per stage)
constexpr int kAtcSplitsMax = 32;
constexpr int64_t kAtcAlign = 256;

template <int DK>
struct AtcCfg {
  static constexpr int kChunks = DK / 64;
  static constexpr int kKvMax = DK == 64 ? 96 : 64;     // vectors per unit (MMA N)
  static constexpr int kBlock = 128 * 64 * 2;          // [128][64] bf16, 128-byte swizzle
  static constexpr int kABytes = 2 * kChunks * kBlock;  // hi + lo, every chunk
  static constexpr int kStageBytes = 2 * kBlock;        // hi + lo of one chunk of 128 B rows
  static constexpr int kVBlock = kKvMax * 128;          // [kv][64] bf16 (one column half)
  static constexpr int kVStageBytes = 4 * kVBlock;      // [half][part], KVP rows each
  static constexpr int kExtBytes = 128 * 16 * 2;        // K = 16 shift block, 128 rows
  static constexpr int kExtHalf = 128 * 16;             // its TMA-loaded K half
};

template <int DK>
struct AtcSmem {
  uint8_t A[AtcCfg<DK>::kABytes];
  uint8_t B[kAtcStages][AtcCfg<DK>::kStageBytes];
  uint8_t V[kAtcVStages][AtcCfg<DK>::kVStageBytes];
  uint8_t Aext[AtcCfg<DK>::kExtBytes];
  uint8_t Bext[kAtcStages][AtcCfg<DK>::kExtBytes];
  uint64_t bfull[kAtcStages], bempty[kAtcStages];
  uint64_t vfull[kAtcVStages], vempty[kAtcVStages];
  uint64_t sfull[kAtcSBufs], pfull[kAtcSBufs];
  uint64_t a_full, ofull;
  uint32_t tmem_base;
  int err;
};

struct AtcArgs {
  int64_t R, C, R_pad, C_pad;
  int K;            // vectors
  int KV;           // vectors per chunk
  int KVP;          // padded to a multiple of 16 (the P V MMA's N)
  int nch;          // vector chunks
  int64_t Kpad;     // nch * KVP: rows of each V part
  int splits;       // column splits (1: write out directly)
  int nt;           // 128-column tiles of B
  const float* potA;
  int* smax;            // [R_pad] order-preserving keys (fkey) of the rows' largest exponent
  const double* nrmA;   // [R_pad] |A_r - centre|^2
  float lf;             // log2(e) / eps (FP32)
  float inv;
  float* out;           // [K][R]
  float* part;          // [splits][K][R]
  int* err;
  uint64_t timeout_ns;
};

// Row shift sigma_r = the first pass's max_c (w_c + s <A_r, B_c>) as two
// bf16 terms (sigma = p1 + p2 exactly in FP32); 0 for padding rows, rows
// whose maximum is not finite, and in the first pass itself.
template <bool MAXP>
__device__ __forceinline__ float atc_sigma(const AtcArgs& a, int64_t row, __nv_bfloat16& p1,
                                           __nv_bfloat16& p2) {
  float sg = 0.f;
  if (!MAXP && row < a.R) {
    const float mx = fkey_value(__ldcg(a.smax + row));
    if (isfinite(mx)) sg = mx;
  }
  p1 = __float2bfloat16_rn(sg);
  p2 = __float2bfloat16_rn(sg - __bfloat162float(p1));
  return __bfloat162float(p1) + __bfloat162float(p2);
}

template <int DK, bool MAXP>
__global__ void __launch_bounds__(kAtcThreads, 1)
apply_tc_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                const __grid_constant__ CUtensorMap mapBext,
                const __grid_constant__ CUtensorMap mapV, AtcArgs a) {
  using Cfg = AtcCfg<DK>;
  constexpr int C = Cfg::kChunks;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const uint32_t base = tc::smem_u32(smem_raw);
  AtcSmem<DK>& sm =
      *reinterpret_cast<AtcSmem<DK>*>(smem_raw + ((1024u - (base & 1023u)) & 1023u));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // unit: (row block, vector chunk, column split)
  const int u = blockIdx.x;
  const int sp = u % a.splits;
  const int ch = (u / a.splits) % a.nch;
  const int rb = u / (a.splits * a.nch);
  const int t0 = (int)((int64_t)a.nt * sp / a.splits);
  const int t1 = (int)((int64_t)a.nt * (sp + 1) / a.splits);
  const int T = t1 - t0;
  const int kv = min(a.KV, a.K - ch * a.KV);  // vectors of this chunk
  const uint32_t idesc_s = tc::idesc_bf16_f32(128, kAtcCols);
  const uint32_t idesc_o = tc::idesc_bf16_f32(128, a.KVP);
  const uint32_t idesc_o2 = tc::idesc_bf16_f32(128, 2 * a.KVP);
  const uint32_t vbytes = 4u * (uint32_t)a.KVP * 128u;

  if (threadIdx.x == 0) {
    for (int i = 0; i < kAtcStages; ++i) {
      tc::mbar_init(&sm.bfull[i], 1);
      tc::mbar_init(&sm.bempty[i], 1);
    }
    for (int i = 0; i < kAtcVStages; ++i) {
      tc::mbar_init(&sm.vfull[i], 1);
      tc::mbar_init(&sm.vempty[i], 1);
    }
    for (int i = 0; i < kAtcSBufs; ++i) {
      tc::mbar_init(&sm.sfull[i], 1);
      tc::mbar_init(&sm.pfull[i], kAtcWarps - kAtcEpiWarp0);
    }
    tc::mbar_init(&sm.a_full, 1);
    tc::mbar_init(&sm.ofull, 1);
    sm.err = 0;
    tc::fence_barrier_init();
  }
  // the shift blocks' second K half (elements 8-15) is zero throughout
  for (int i = threadIdx.x; i < (1 + kAtcStages) * 128; i += blockDim.x) {
    uint8_t* blk = i < 128 ? sm.Aext : sm.Bext[i / 128 - 1];
    *reinterpret_cast<uint4*>(blk + Cfg::kExtHalf + (i % 128) * 16) = make_uint4(0, 0, 0, 0);
  }
  tc::fence_proxy_async_smem();
  if (warp == 1) {
    tc::tmem_alloc(&sm.tmem_base, 512);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = sm.tmem_base;
  const uint32_t tO = tbase + kAtcSBufs * kAtcCols;

  bool ok = true;
  if (warp == 0) {
    // ---- producer
    if (lane == 0) {
      tc::prefetch_tensormap(&mapA);
      tc::prefetch_tensormap(&mapB);
      tc::prefetch_tensormap(&mapBext);
      tc::prefetch_tensormap(&mapV);
    }
    // the rows' shift block: [1, 1, 1, -sigma_1, -sigma_2, 0, 0, 0]
    const uint32_t one = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(1.f));
    for (int i = lane; i < kAtcRows; i += 32) {
      __nv_bfloat16 p1, p2;
      atc_sigma<MAXP>(a, (int64_t)rb * kAtcRows + i, p1, p2);
      uint4 v;
      v.x = one | (one << 16);
      v.y = one | ((uint32_t)__bfloat16_as_ushort(__hneg(p1)) << 16);
      v.z = (uint32_t)__bfloat16_as_ushort(__hneg(p2));
      v.w = 0u;
      *reinterpret_cast<uint4*>(sm.Aext + i * 16) = v;
    }
    tc::fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) {
      tc::mbar_arrive_expect_tx(&sm.a_full, Cfg::kABytes);
      for (int part = 0; part < 2; ++part)
        for (int c = 0; c < C; ++c)
          tc::tma_load_2d(sm.A + (part * C + c) * Cfg::kBlock, &mapA, &sm.a_full, 64 * c,
                          (int32_t)(rb * kAtcRows + part * a.R_pad));
      int issued = -1;  // the last ring stage given a copy
      for (int i = 0; ok && i < T; ++i) {
        const int32_t col = (t0 + i) * kAtcCols;
        for (int c = 0; c < C; ++c) {
          const uint32_t g = i * C + c;
          const uint32_t st = g % kAtcStages;
          if (!tc::mbar_wait(&sm.bempty[st], ((g / kAtcStages) & 1) ^ 1, a.timeout_ns)) {
            ok = false;
            break;
          }
          const bool last = c == C - 1;
          tc::mbar_arrive_expect_tx(&sm.bfull[st],
                                    Cfg::kStageBytes + (last ? Cfg::kExtHalf : 0));
          for (int part = 0; part < 2; ++part)
            tc::tma_load_2d(sm.B[st] + part * Cfg::kBlock, &mapB, &sm.bfull[st], 64 * c,
                            (int32_t)(col + part * a.C_pad));
          if (last) tc::tma_load_2d(sm.Bext[st], &mapBext, &sm.bfull[st], 0, col);
          issued = (int)g;
        }
      }
      // after a timeout: wait (bounded) for this warp's copies in flight
      if (!ok) {
        tc::mbar_wait(&sm.a_full, 0, 1000000000ull);
        for (int g = issued - kAtcStages + 1; g <= issued; ++g)
          if (g >= 0) tc::mbar_wait(&sm.bfull[g % kAtcStages], (g / kAtcStages) & 1, 1000000000ull);
      }
    }
    __syncwarp();
  } else if (warp == 2) {
    // ---- producer of the vector tiles
    if (!MAXP && lane == 0) {
      int issued = -1;  // the last vector tile given a copy
      for (int i = 0; ok && i < T; ++i) {
        const int32_t col = (t0 + i) * kAtcCols;
        const uint32_t vs = i % kAtcVStages;
        if (!tc::mbar_wait(&sm.vempty[vs], ((i / kAtcVStages) & 1) ^ 1, a.timeout_ns)) {
          ok = false;
          break;
        }
        tc::mbar_arrive_expect_tx(&sm.vfull[vs], vbytes);
        // block (column half h, part): the hi and lo rows of a half adjacent
        for (int h = 0; h < 2; ++h)
          for (int part = 0; part < 2; ++part)
            tc::tma_load_2d(sm.V[vs] + (h * 2 + part) * a.KVP * 128, &mapV, &sm.vfull[vs],
                            col + 64 * h, (int32_t)(part * a.Kpad + (int64_t)ch * a.KVP));
        issued = i;
      }
      if (!ok)
        for (int i = issued - kAtcVStages + 1; i <= issued; ++i)
          if (i >= 0)
            tc::mbar_wait(&sm.vfull[i % kAtcVStages], (i / kAtcVStages) & 1, 1000000000ull);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ---- MMA issuer
    if (lane == 0) {
      if (!tc::mbar_wait(&sm.a_full, 0, a.timeout_ns)) ok = false;
      const uint32_t a0 = tc::smem_u32(sm.A);
      for (int i = 0; ok && i < T + kAtcSBufs - 1; ++i) {
        if (i < T) {
          // S of tile i into buffer i % 2 (its P was consumed by the P V
          // MMAs of tile i - 2, issued before these; in the first pass the
          // epilogue releases the buffer once it has read tile i - 2)
          if (MAXP && i >= kAtcSBufs) {
            const int j = i - kAtcSBufs;
            if (!tc::mbar_wait(&sm.pfull[j % kAtcSBufs], (j / kAtcSBufs) & 1, a.timeout_ns)) {
              ok = false;
              break;
            }
            tc::fence_after_sync();
          }
          const uint32_t d = tbase + (i % kAtcSBufs) * kAtcCols;
          for (int c = 0; ok && c < C; ++c) {
            const uint32_t g = i * C + c;
            const uint32_t st = g % kAtcStages;
            if (!tc::mbar_wait(&sm.bfull[st], (g / kAtcStages) & 1, a.timeout_ns)) {
              ok = false;
              break;
            }
            tc::fence_after_sync();
            const uint32_t b0 = tc::smem_u32(sm.B[st]);
            // (A part, B part): hi*hi, hi*lo, lo*hi
            const int pa[3] = {0, 0, 1};
            const int pb[3] = {0, 1, 0};
            for (int prod = 0; prod < (MAXP ? 1 : 3); ++prod)
              for (int kk = 0; kk < 4; ++kk)
                tc::mma_bf16(d,
                             tc::sw128_kmajor_desc(a0 + (pa[prod] * C + c) * Cfg::kBlock + kk * 32),
                             tc::sw128_kmajor_desc(b0 + pb[prod] * Cfg::kBlock + kk * 32), idesc_s,
                             (c | prod | kk) ? 1u : 0u);
            if (c == C - 1)
              tc::mma_bf16(d, tc::plain_kmajor_desc(tc::smem_u32(sm.Aext), Cfg::kExtHalf, 128),
                           tc::plain_kmajor_desc(tc::smem_u32(sm.Bext[st]), Cfg::kExtHalf, 128),
                           idesc_s, 1u);
            tc::mma_commit(&sm.bempty[st]);
          }
          if (!ok) break;
          tc::mma_commit(&sm.sfull[i % kAtcSBufs]);
        }
        if (!MAXP && i >= kAtcSBufs - 1) {
          // O += P V^T for tile j = i - 1: P from TMEM, V from the ring
          const int j = i - (kAtcSBufs - 1);
          const uint32_t b = j % kAtcSBufs, vs = j % kAtcVStages;
          if (!tc::mbar_wait(&sm.pfull[b], (j / kAtcSBufs) & 1, a.timeout_ns) ||
              !tc::mbar_wait(&sm.vfull[vs], (j / kAtcVStages) & 1, a.timeout_ns)) {
            ok = false;
            break;
          }
          tc::fence_after_sync();
          const uint32_t v0 = tc::smem_u32(sm.V[vs]);
          for (int s = 0; s < kAtcCols / 16; ++s) {
            const uint32_t ahi = tbase + b * kAtcCols + 32 * (s >> 1) + 8 * (s & 1);
            // V_hi rows of the slab's column half, its V_lo rows right after
            const uint32_t vhi = v0 + (s >> 2) * 2 * a.KVP * 128 + (s & 3) * 32;
            tc::mma_bf16_ts(tO, ahi, tc::sw128_kmajor_desc(vhi), idesc_o2, (j | s) ? 1u : 0u);
            tc::mma_bf16_ts(tO, ahi + 16, tc::sw128_kmajor_desc(vhi), idesc_o, 1u);
          }
          tc::mma_commit(&sm.vempty[vs]);
        }
      }
      // issued after a timeout too: its arrival drains the MMAs in flight
      tc::mma_commit(&sm.ofull);
    }
    __syncwarp();
  } else {
    // ---- epilogue: weights of every tile, then the output rows
    const int e = warp - kAtcEpiWarp0;
    const int q = warp & 3;
    const int cg = e >> 2;
    const int64_t row = (int64_t)rb * kAtcRows + 32 * q + lane;
    const uint32_t lane_off = (uint32_t)(32 * q) << 16;
    float rmax = -INFINITY;  // first pass: this row's largest exponent so far
    for (int i = 0; ok && i < T; ++i) {
      const uint32_t b = i % kAtcSBufs;
      if (!tc::mbar_wait(&sm.sfull[b], (i / kAtcSBufs) & 1, a.timeout_ns)) {
        ok = false;
        break;
      }
      tc::fence_after_sync();
      const uint32_t ta = tbase + lane_off + b * kAtcCols + 32 * cg;
      float v[32];
      tc::tmem_ld32(ta, v);
      tc::tmem_ld_wait();
      if (MAXP) {
        // the buffer is free once read
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&sm.pfull[b]);
        float t11[11];
#pragma unroll
        for (int j = 0; j < 10; ++j) t11[j] = fmax3(v[3 * j], v[3 * j + 1], v[3 * j + 2]);
        t11[10] = fmaxf(v[30], v[31]);
        rmax = fmaxf(rmax, fmax3(fmax3(t11[0], t11[1], t11[2]), fmax3(t11[3], t11[4], t11[5]),
                                 fmaxf(fmax3(t11[6], t11[7], t11[8]), fmaxf(t11[9], t11[10]))));
        continue;
      }
      uint32_t hi[16], lo[16];
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        const float p0 = ex2_approx(v[2 * t]);
        const float p1 = ex2_approx(v[2 * t + 1]);
        const __nv_bfloat162 h = __floats2bfloat162_rn(p0, p1);
        const __nv_bfloat162 l =
            __floats2bfloat162_rn(p0 - __low2float(h), p1 - __high2float(h));
        hi[t] = *reinterpret_cast<const uint32_t*>(&h);
        lo[t] = *reinterpret_cast<const uint32_t*>(&l);
      }
      tc::tmem_st16(ta, hi);
      tc::tmem_st16(ta + 16, lo);
      tc::tmem_st_wait();
      tc::fence_before_sync();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&sm.pfull[b]);
    }
    if (MAXP) {
      // every column group's maximum of the row into the row's key (the
      // column splits' CTAs combine there too)
      if (ok && row < a.R && rmax > -INFINITY) atomicMax(a.smax + row, fkey(rmax));
    } else if (ok && !tc::mbar_wait(&sm.ofull, 0, a.timeout_ns)) {
      ok = false;
    }
    if (!MAXP && ok) {
      tc::fence_after_sync();
      // the row's scale 2^(u_r + sigma_r), u_r = (potA_r - inv |A_r|^2) lf
      double sc = 0.0;
      if (row < a.R) {
        __nv_bfloat16 p1, p2;
        const float sig = atc_sigma<false>(a, row, p1, p2);
        const double pa = (double)__ldg(a.potA + row);
        const double ex =
            (pa - (double)a.inv * a.nrmA[row]) * (double)a.lf + (double)sig;
        sc = (ex == -INFINITY) ? 0.0 : exp2(ex);
      }
      const float scf = (float)sc;
      for (int jc = cg; jc < a.KVP / 16; jc += 4) {
        // O = its first half (P_hi V_hi + P_lo V_hi) + its second (P_hi V_lo)
        float o[16], o2[16];
        tc::tmem_ld16(tO + lane_off + 16 * jc, o);
        tc::tmem_ld16(tO + lane_off + a.KVP + 16 * jc, o2);
        tc::tmem_ld_wait();
#pragma unroll
        for (int t = 0; t < 16; ++t) o[t] += o2[t];
        if (row < a.R) {
#pragma unroll
          for (int t = 0; t < 16; ++t) {
            const int kk = 16 * jc + t;
            if (kk < kv) {
              const int64_t k = (int64_t)ch * a.KV + kk;
              const float val = o[t] * scf;
              if (a.splits == 1)
                a.out[k * a.R + row] = val;
              else
                a.part[((int64_t)sp * a.K + k) * a.R + row] = val;
            }
          }
        }
      }
    }
  }
  if (!ok) atomicExch(&sm.err, 1);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 1) {
    // after a timeout the final commit may not have landed yet
    if (sm.err && lane == 0) tc::mbar_wait(&sm.ofull, 0, 1000000000ull);
    __syncwarp();
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, 512);
  }
  if (threadIdx.x == 0 && sm.err) atomicExch(a.err, 1);
}

// ---------------------------------------------------------------- preparation
struct AtcPrep {
  const float* A;
  const float* B;
  const float* potB;
  const float* vec;
  int64_t R, C, R_pad, C_pad;
  int d, DK;
  int K, KV, KVP;
  int64_t Kpad;
  float s;      // 2 inv lf
  float lf;
  float inv;
  float* cen;               // [DK]
  __nv_bfloat16* abuf;      // [2 R_pad][DK]
  __nv_bfloat16* bbuf;      // [2 C_pad][DK]
  uint8_t* bext;            // [C_pad][16 bytes]
  double* nrmA;             // [R_pad]
  __nv_bfloat16* vbuf;      // [2 Kpad][C_pad]
};

// Common centre of both point sets: the mean of up to 256 points of each
// at a fixed stride (any centre gives the same plan; a central one keeps
// the expanded |a|^2 + |b|^2 - 2 <a, b> small). One CTA per coordinate,
// one sample per thread, a fixed-order tree sum.
__global__ void atc_center_kernel(AtcPrep p) {
  __shared__ float red[2][8];
  const int k = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int64_t na = p.R < 256 ? p.R : 256, nb = p.C < 256 ? p.C : 256;
  const int64_t sa = p.R / na, sb = p.C / nb;
  float ma = 0.f, mb = 0.f;
  if (k < p.d) {
    if (t < na) ma = p.A[t * sa * p.d + k];
    if (t < nb) mb = p.B[t * sb * p.d + k];
  }
  for (int off = 16; off > 0; off >>= 1) {
    ma += __shfl_xor_sync(0xffffffffu, ma, off);
    mb += __shfl_xor_sync(0xffffffffu, mb, off);
  }
  if (lane == 0) {
    red[0][warp] = ma;
    red[1][warp] = mb;
  }
  __syncthreads();
  if (t == 0) {
    float sa2 = 0.f, sb2 = 0.f;
    for (int w = 0; w < 8; ++w) {
      sa2 += red[0][w];
      sb2 += red[1][w];
    }
    p.cen[k] = k < p.d ? 0.5f * (sa2 / (float)na + sb2 / (float)nb) : 0.f;
  }
}

// One warp per point: centred coordinates, their bf16 hi/lo split (A's
// scaled by s), A's squared norms, B's shift rows.
__global__ void atc_prep_points_kernel(AtcPrep p) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const bool isA = blockIdx.y == 0;
  const int64_t n = isA ? p.R : p.C, npad = isA ? p.R_pad : p.C_pad;
  const float* src = isA ? p.A : p.B;
  if (wid >= npad) return;
  __nv_bfloat16* dst = isA ? p.abuf : p.bbuf;
  double nrm = 0.0;
  for (int k = lane; k < p.DK; k += 32) {
    float c = 0.f;
    if (wid < n && k < p.d) c = src[wid * p.d + k] - p.cen[k];
    nrm += (double)c * (double)c;
    const float v = isA ? c * p.s : c;
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    dst[wid * p.DK + k] = h;
    dst[(npad + wid) * p.DK + k] = l;
  }
  for (int off = 16; off > 0; off >>= 1) nrm += __shfl_xor_sync(0xffffffffu, nrm, off);
  if (lane == 0) {
    if (isA) {
      p.nrmA[wid] = nrm;
    } else {
      const float w = wid < n ? (__ldg(p.potB + wid) - p.inv * (float)nrm) * p.lf : -INFINITY;
      write_ext_row(p.bext + wid * 16, w);
    }
  }
}

// The vectors as bf16 hi and lo rows, chunk ch's vector kk in row
// ch * KVP + kk of each part, zero beyond the vectors and columns.
__global__ void atc_prep_vec_kernel(AtcPrep p) {
  const int64_t total = p.Kpad * p.C_pad;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx / p.C_pad, c = idx % p.C_pad;
    const int ch = (int)(r / p.KVP), kk = (int)(r % p.KVP);
    const int64_t k = (int64_t)ch * p.KV + kk;
    float v = 0.f;
    if (kk < p.KV && k < p.K && c < p.C) v = p.vec[k * p.C + c];
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    p.vbuf[idx] = h;
    p.vbuf[total + idx] = __float2bfloat16_rn(v - __bfloat162float(h));
  }
}

// Every row's key of its largest exponent starts as fkey(-inf).
__global__ void atc_fill_keys_kernel(int* keys, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) keys[i] = kDkeyEmptyMax;
}

// out[k][r] = sum over the column splits of their parts (fixed order).
__global__ void atc_combine_kernel(const float* part, int splits, int64_t KR, float* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < KR;
       i += (int64_t)gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int t = 0; t < splits; ++t) s += part[(int64_t)t * KR + i];
    out[i] = s;
  }
}

// ---------------------------------------------------------------- host side
inline size_t align_up(size_t v) { return (v + kAtcAlign - 1) / kAtcAlign * kAtcAlign; }
inline int64_t round_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

int device_sm_count() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
}

struct AtcLayout {
  int DK;
  int64_t R, C, R_pad, C_pad;
  int K, KV, KVP, nch;
  int64_t Kpad;
  int splits, nt;
  size_t status, cen, abuf, bbuf, bext, nrmA, smax, vbuf, part, total;
};

// Column splits: the fewest waves x (tiles per unit + 2 for the pipeline's
// fill and drain) over the SMs.
int atc_splits(int64_t units0, int nt, int sms) {
  int best = 1;
  double best_cost = 1e300;
  for (int s = 1; s <= std::min(nt, kAtcSplitsMax); ++s) {
    const int64_t units = units0 * s;
    const double waves = (double)((units + sms - 1) / sms);
    const double cost = waves * ((double)((nt + s - 1) / s) + 2.0);
    if (cost < best_cost - 1e-9) {
      best_cost = cost;
      best = s;
    }
  }
  return best;
}

int atc_layout(int64_t n, int64_t m, int d, int K, int axis, AtcLayout& L) {
  if (n < 1 || m < 1 || d < 1 || K < 1 || (axis != 0 && axis != 1)) return OTTB_ERR_INVALID;
  if (d > 128) return OTTB_ERR_UNSUPPORTED;
  L.DK = d <= 64 ? 64 : 128;
  L.R = axis == 1 ? n : m;
  L.C = axis == 1 ? m : n;
  if (L.R > (int64_t)1 << 30 || L.C > (int64_t)1 << 30) return OTTB_ERR_UNSUPPORTED;
  L.R_pad = round_up(L.R, kAtcRows);
  L.C_pad = round_up(L.C, kAtcCols);
  const int kvmax = L.DK == 64 ? AtcCfg<64>::kKvMax : AtcCfg<128>::kKvMax;
  L.K = K;
  L.nch = (K + kvmax - 1) / kvmax;
  L.KV = (K + L.nch - 1) / L.nch;
  L.KVP = (int)round_up(L.KV, 16);
  L.Kpad = (int64_t)L.nch * L.KVP;
  L.nt = (int)(L.C_pad / kAtcCols);
  L.splits = atc_splits((L.R_pad / kAtcRows) * L.nch, L.nt, device_sm_count());
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += align_up(bytes);
    return o;
  };
  L.status = take(sizeof(int32_t));
  L.cen = take(sizeof(float) * L.DK);
  L.abuf = take(2 * (size_t)L.R_pad * L.DK * 2);
  L.bbuf = take(2 * (size_t)L.C_pad * L.DK * 2);
  L.bext = take((size_t)L.C_pad * 16);
  L.nrmA = take(sizeof(double) * (size_t)L.R_pad);
  L.smax = take(sizeof(int32_t) * (size_t)L.R_pad);
  L.vbuf = take(2 * (size_t)L.Kpad * L.C_pad * 2);
  L.part = take(L.splits > 1 ? sizeof(float) * (size_t)L.splits * K * L.R : 0);
  L.total = off;
  return OTTB_OK;
}

template <int DK, bool MAXP>
int atc_launch(const CUtensorMap* maps, const AtcArgs& args, int units, cudaStream_t stream) {
  const size_t smem = sizeof(AtcSmem<DK>) + 1024;
  if (!ensure_dynamic_smem((const void*)apply_tc_kernel<DK, MAXP>, smem)) return OTTB_ERR_CUDA;
  apply_tc_kernel<DK, MAXP><<<units, kAtcThreads, smem, stream>>>(maps[0], maps[1], maps[2],
                                                                   maps[3], args);
  return cudaPeekAtLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}

}  // namespace
}  // namespace ottb

using namespace ottb;

extern "C" size_t ottb_apply_transport_tc_workspace_size(int64_t n, int64_t m, int32_t d,
                                                         int32_t num_vec, int32_t axis) {
  AtcLayout L;
  if (atc_layout(n, m, d, num_vec, axis, L) != OTTB_OK) return 0;
  return L.total;
}

extern "C" int32_t ottb_apply_transport_tc(const float* x, const float* y, int64_t n, int64_t m,
                                           int32_t d, const float* f, const float* g,
                                           float epsilon, float inv_scale_cost,
                                           const float* vec, int32_t num_vec, int32_t axis,
                                           float* out, void* workspace, size_t workspace_bytes,
                                           void* stream_ptr) {
  if (!x || !y || !f || !g || !vec || !out) return OTTB_ERR_INVALID;
  if (!(epsilon > 0.f) || !(inv_scale_cost > 0.f)) return OTTB_ERR_INVALID;
  AtcLayout L;
  int st = atc_layout(n, m, d, num_vec, axis, L);
  if (st != OTTB_OK) return st;
  if (!workspace || workspace_bytes < L.total || ((uintptr_t)workspace) % kAtcAlign != 0)
    return OTTB_ERR_WORKSPACE;
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  char* ws = (char*)workspace;
  (void)cudaGetLastError();  // clear an error left by earlier, unrelated work
  int32_t* status = (int32_t*)(ws + L.status);
  if (cudaMemsetAsync(status, 0, sizeof(int32_t), stream) != cudaSuccess) return OTTB_ERR_CUDA;

  AtcPrep p;
  p.A = axis == 1 ? x : y;
  p.B = axis == 1 ? y : x;
  p.potB = axis == 1 ? g : f;
  p.vec = vec;
  p.R = L.R;
  p.C = L.C;
  p.R_pad = L.R_pad;
  p.C_pad = L.C_pad;
  p.d = d;
  p.DK = L.DK;
  p.K = num_vec;
  p.KV = L.KV;
  p.KVP = L.KVP;
  p.Kpad = L.Kpad;
  p.lf = (float)(kLog2eD / (double)epsilon);
  p.inv = inv_scale_cost;
  p.s = 2.f * inv_scale_cost * p.lf;
  p.cen = (float*)(ws + L.cen);
  p.abuf = (__nv_bfloat16*)(ws + L.abuf);
  p.bbuf = (__nv_bfloat16*)(ws + L.bbuf);
  p.bext = (uint8_t*)(ws + L.bext);
  p.nrmA = (double*)(ws + L.nrmA);
  p.vbuf = (__nv_bfloat16*)(ws + L.vbuf);

  atc_center_kernel<<<L.DK, 256, 0, stream>>>(p);
  {
    const int64_t warps = std::max(L.R_pad, L.C_pad);
    dim3 grid((unsigned)((warps * 32 + 255) / 256), 2);
    atc_prep_points_kernel<<<grid, 256, 0, stream>>>(p);
  }
  {
    const int64_t total = L.Kpad * L.C_pad;
    atc_prep_vec_kernel<<<(unsigned)std::min<int64_t>((total + 255) / 256, 4096), 256, 0,
                          stream>>>(p);
  }
  if (cudaPeekAtLastError() != cudaSuccess) return OTTB_ERR_CUDA;

  // tensor maps: A and B [2 pad][DK] (64 x 128 boxes), B's shift rows
  // [C_pad][8] (8 x 128), V [2 Kpad][C_pad] (64 x KVP boxes)
  CUtensorMap maps[4];
  if (!encode_bf16_2d(&maps[0], p.abuf, 2 * L.R_pad, L.DK, 64, 128, CU_TENSOR_MAP_SWIZZLE_128B,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B) ||
      !encode_bf16_2d(&maps[1], p.bbuf, 2 * L.C_pad, L.DK, 64, 128, CU_TENSOR_MAP_SWIZZLE_128B,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B) ||
      !encode_bf16_2d(&maps[2], p.bext, L.C_pad, 8, 8, 128, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B) ||
      !encode_bf16_2d(&maps[3], p.vbuf, 2 * L.Kpad, L.C_pad, 64, (uint32_t)L.KVP,
                      CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B))
    return OTTB_ERR_CUDA;

  AtcArgs a;
  a.R = L.R;
  a.C = L.C;
  a.R_pad = L.R_pad;
  a.C_pad = L.C_pad;
  a.K = num_vec;
  a.KV = L.KV;
  a.KVP = L.KVP;
  a.nch = L.nch;
  a.Kpad = L.Kpad;
  a.splits = L.splits;
  a.nt = L.nt;
  a.potA = axis == 1 ? f : g;
  a.smax = (int*)(ws + L.smax);
  a.nrmA = p.nrmA;
  a.lf = p.lf;
  a.inv = inv_scale_cost;
  a.out = out;
  a.part = L.splits > 1 ? (float*)(ws + L.part) : nullptr;
  a.err = status;
  a.timeout_ns = 20ull * 1000000000ull;
  // first pass: the rows' largest exponents (one vector chunk's worth of
  // units), then the product
  {
    AtcArgs a1 = a;
    a1.nch = 1;
    const int units1 = (int)((L.R_pad / kAtcRows) * L.splits);
    atc_fill_keys_kernel<<<(unsigned)((L.R_pad + 255) / 256), 256, 0, stream>>>(a.smax, L.R_pad);
    st = L.DK == 64 ? atc_launch<64, true>(maps, a1, units1, stream)
                    : atc_launch<128, true>(maps, a1, units1, stream);
    if (st != OTTB_OK) return st;
  }
  const int units = (int)((L.R_pad / kAtcRows) * L.nch * L.splits);
  st = L.DK == 64 ? atc_launch<64, false>(maps, a, units, stream)
                  : atc_launch<128, false>(maps, a, units, stream);
  if (st != OTTB_OK) return st;
  if (L.splits > 1) {
    const int64_t KR = (int64_t)num_vec * L.R;
    atc_combine_kernel<<<(unsigned)std::min<int64_t>((KR + 255) / 256, 4096), 256, 0, stream>>>(
        a.part, L.splits, KR, out);
  }
  return cudaPeekAtLastError() == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}
