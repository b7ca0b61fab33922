// C-ABI entry points of libottb200 (declared in include/ott_b200.h).
//
// Host side of the solve: argument checks, the work plan (padding, column
// splits, workspace layout), the device tables and the launch sequence
//   fill errors -> prep points -> init potentials -> persistent loop
//   (cooperative) -> finalize.
// Nothing here allocates device memory: all scratch lives in the caller's
// workspace.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <tuple>
#include <vector>

#include <cuda.h>

#include "aux_kernels.cuh"
#include "kernel_simt.cuh"
#include "kernel_tc.cuh"
#include "tmap.cuh"

using namespace ottb;

namespace {

constexpr size_t kAlign = 256;
inline size_t align_up(size_t v, size_t a = kAlign) { return (v + a - 1) / a * a; }
inline int64_t round_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

struct DeviceInfo {
  int sms = 0;
  int major = 0;
  int minor = 0;
};

DeviceInfo device_info() {
  static std::mutex mu;
  static DeviceInfo cache[64];
  static bool have[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DeviceInfo{};
  std::lock_guard<std::mutex> lock(mu);
  if (!have[dev]) {
    DeviceInfo di;
    cudaDeviceGetAttribute(&di.sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&di.major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&di.minor, cudaDevAttrComputeCapabilityMinor, dev);
    cache[dev] = di;
    have[dev] = true;
  }
  return cache[dev];
}

int simt_dp(int d) {
  int dp = 2;
  while (dp < d) dp <<= 1;
  return dp;
}

// Kernel table for the CUDA-core engine.
template <int DP>
struct SimtKernel {
  static void* fn() { return (void*)&sinkhorn_simt_kernel<DP>; }
  static size_t smem() { return sizeof(SimtKernelSmem<DP>); }
};

struct KernelChoice {
  void* fn = nullptr;
  size_t smem = 0;
  int threads = 256;
};

KernelChoice pick_simt(int dp) {
  KernelChoice k;
  switch (dp) {
    case 2: k.fn = SimtKernel<2>::fn(); k.smem = SimtKernel<2>::smem(); break;
    case 4: k.fn = SimtKernel<4>::fn(); k.smem = SimtKernel<4>::smem(); break;
    case 8: k.fn = SimtKernel<8>::fn(); k.smem = SimtKernel<8>::smem(); break;
    case 16: k.fn = SimtKernel<16>::fn(); k.smem = SimtKernel<16>::smem(); break;
    case 32: k.fn = SimtKernel<32>::fn(); k.smem = SimtKernel<32>::smem(); break;
    case 64: k.fn = SimtKernel<64>::fn(); k.smem = SimtKernel<64>::smem(); break;
    case 128: k.fn = SimtKernel<128>::fn(); k.smem = SimtKernel<128>::smem(); break;
    default: break;
  }
  return k;
}

// Tensor-core engine: DK = 64 or 128 (d padded with zeros), tiles of TN =
// 256 or 128 columns.
template <int DK, int TN>
struct TcKernel {
  static void* fn() { return (void*)&sinkhorn_tc_kernel<DK, TN>; }
  static size_t smem() { return sizeof(TcSmem<DK, TN>) + 1024; }  // + alignment slack
};

// Points of the tensor-core layout are padded to this many (either tile
// width divides it), so the workspace layout does not depend on the tile.
constexpr int64_t kTcPad = 256;

KernelChoice pick_tc(int dk, int tn) {
  KernelChoice k;
  k.threads = TcCfg<64, 256>::kThreads;
  if (dk == 64 && tn == 256) { k.fn = TcKernel<64, 256>::fn(); k.smem = TcKernel<64, 256>::smem(); }
  if (dk == 64 && tn == 128) { k.fn = TcKernel<64, 128>::fn(); k.smem = TcKernel<64, 128>::smem(); }
  if (dk == 128 && tn == 256) { k.fn = TcKernel<128, 256>::fn(); k.smem = TcKernel<128, 256>::smem(); }
  if (dk == 128 && tn == 128) { k.fn = TcKernel<128, 128>::fn(); k.smem = TcKernel<128, 128>::smem(); }
  return k;
}

// Tensor map over a [2 * pad][dk] bf16 array (hi rows, then lo rows): boxes
// of 64 elements (128 bytes) x 128 rows, 128-byte swizzle.
bool encode_points_map(CUtensorMap* map, void* base, int64_t pad, int dk) {
  return encode_bf16_2d(map, base, 2 * pad, dk, 64, 128, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B);
}

// Tensor map over column-shift rows [rows][8] bf16: boxes of 8 x 128, no
// swizzle (the K-major core-matrix layout of an MMA extension block).
bool encode_ext_map(CUtensorMap* map, void* base, int64_t rows) {
  return encode_bf16_2d(map, base, rows, 8, 8, 128, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B);
}

// Grid size of the persistent launch: all CTAs co-resident. Computed once
// per kernel and device (the attribute and occupancy queries then stay out
// of later calls, which may be under stream capture).
int persistent_grid(const KernelChoice& k, int sms) {
  static std::mutex mu;
  static std::map<std::pair<int, void*>, int> cache;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find({dev, k.fn});
  if (it != cache.end()) return it->second;
  if (cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)k.smem) != cudaSuccess)
    return 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, k.threads, k.smem) !=
      cudaSuccess)
    return 0;
  cache[{dev, k.fn}] = per_sm * sms;
  return per_sm * sms;
}

// Work schedule knobs of a call: the autotuner's search space.
//   split_scale  the initial column split of a single problem is the
//                heuristic choice (choose_split; choose_split_tc on the
//                tensor cores) times split_scale / 4
//   waves        the kernel grows the splits of the still-active problems
//                whenever they offer fewer than waves * grid units per sweep
//                (0: never; without a tuned or pinned schedule a single
//                problem takes 0: on B200 growth cost a single FP32 solve
//                1.42x at n = m = 4096 and 1.24x at 8192, nothing at 2048
//                and 16384)
//   dynamic      work units dealt from an atomic queue (1) or round-robin
//                (0); calls with several problems always use the queue
//   tile_n       columns of a tensor-core tile (256: two accumulators, full
//                MMA rate; 128: four accumulators, smaller last tiles)
struct Schedule {
  int split_scale = 4;
  int waves = 2;
  int dynamic = 0;
  int tile_n = 256;  // tensor-core tile width (256 or 128); the CUDA-core engine ignores it
};

// Column splits of one sweep: enough units to keep every CTA busy with
// little tail (efficiency = units / (waves * grid)).
int choose_split(int rb, int ntiles, int grid, int num_problems) {
  if (num_problems > 1 || grid <= 0) return 1;
  int best = 1;
  double best_score = -1.0;
  const int smax = std::max(1, std::min(ntiles, 32));
  for (int s = 1; s <= smax; ++s) {
    const double units = (double)rb * s;
    const double waves = std::ceil(units / grid);
    const double eff = units / (waves * grid);
    const double score = eff - 0.004 * s;
    if (score > best_score + 1e-9) {
      best_score = score;
      best = s;
    }
  }
  return best;
}

// Column splits of a single problem on the tensor cores: the split that
// minimises a cost model of one sweep, in units of one 128 x 256 tile's
// time (about 1.5 us at the power-capped clock). A work unit costs about
// 4.2 tiles beyond its own tiles (filling the TMA/MMA pipeline, the first
// accumulator round trip through tensor memory, handing its row results to
// the merge), units run in waves of the grid, and merging s splits of a row
// block adds about 0.33 s tiles per unit. Fitted to B200 sweeps of the
// split at d = 64 (n = m = 2048 ... 65536): it keeps the splits of 32768
// and 65536 (4 and 2) and takes fewer, longer units from 2048 to 16384,
// where more units than one wave cost up to twice the time (n = m = 8192:
// 2 splits, 3.5 ms to 1e-3, against 6.9 ms with 9).
int choose_split_tc(int rb, int ntiles, int grid) {
  if (grid <= 0) return 1;
  int best = 1;
  double best_t = -1.0;
  const int smax = std::max(1, std::min(ntiles, 32));
  for (int s = 1; s <= smax; ++s) {
    const double units = (double)rb * s;
    const double waves = std::ceil(units / grid);
    const double t = waves * (4.2 + std::ceil((double)ntiles / s)) + 0.33 * units * s / grid;
    if (best_t < 0.0 || t < best_t - 1e-9) {
      best_t = t;
      best = s;
    }
  }
  return best;
}

// Largest column split the workspace is sized for: 32 for a single
// problem, 8 per problem in calls with several (splits there only grow once
// problems have converged).
constexpr int kMaxSplitSingle = 32;
constexpr int kMaxSplitBatch = 8;

struct ProbPlan {
  int64_t n, m, n_pad, m_pad;
  int rb_f, rb_g, split_f, split_g, smax_f, smax_g;
  size_t off_xt, off_yt, off_nx, off_ny, off_galt, off_pm, off_pl, off_arr, off_err,
      off_msum, off_extx, off_exty, off_cen, off_lprev;
};

// BF16 split-3 on tcgen05 when asked for, and by default where the inner
// product is a real contraction (d >= 32); FP32 CUDA-core FMAs below.
bool wants_tc(const ottb_solver_cfg* cfg, int d) {
  if (cfg->precision == OTTB_PRECISION_BF16_SPLIT3) return true;
  return cfg->precision == OTTB_PRECISION_AUTO && d >= 32;
}

struct Plan {
  int num = 0;
  int dp = 0;        // FP32 engine: padded dimension; tensor cores: DK
  bool tc = false;
  int grid = 0;
  KernelChoice kern;
  Schedule sched;
  size_t off_globals = 0, off_sched = 0, off_probs = 0, off_state = 0, off_ids = 0,
         off_prefix = 0, off_eval_ids = 0, off_eval_prefix = 0, off_ptrs = 0, off_maps = 0;
  size_t header_bytes = 0;
  size_t off_pristine = 0;  // unmodified copy of the header, restored by every launch
  size_t total = 0;
  std::vector<ProbPlan> probs;
  std::vector<int> order;  // table position -> caller index
};

// ---------------------------------------------------------------- autotune cache
// Key of a call's shape: device, engine, padded dimension, grid, number of
// problems and a hash of the (n, m) list.
struct TuneKey {
  int dev, tc, dp, grid, num;
  uint64_t hash;
  bool operator<(const TuneKey& o) const {
    return std::tie(dev, tc, dp, grid, num, hash) < std::tie(o.dev, o.tc, o.dp, o.grid, o.num, o.hash);
  }
};

std::mutex g_tune_mu;
std::map<TuneKey, Schedule>& tune_cache() {
  static std::map<TuneKey, Schedule> cache;
  return cache;
}

TuneKey tune_key(const ottb_problem* probs, int num, const Plan& plan) {
  TuneKey k;
  k.dev = -1;
  cudaGetDevice(&k.dev);
  k.tc = plan.tc ? 1 : 0;
  k.dp = plan.dp;
  k.grid = plan.grid;
  k.num = num;
  uint64_t h = 1469598103934665603ull;  // FNV-1a over the sizes
  for (int i = 0; i < num; ++i) {
    const uint64_t v[2] = {(uint64_t)probs[i].n, (uint64_t)probs[i].m};
    for (uint64_t x : v)
      for (int b = 0; b < 8; ++b) {
        h ^= (x >> (8 * b)) & 0xffu;
        h *= 1099511628211ull;
      }
  }
  k.hash = h;
  return k;
}

bool tuned_schedule(const TuneKey& key, Schedule* out) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto it = tune_cache().find(key);
  if (it == tune_cache().end()) return false;
  *out = it->second;
  return true;
}

int validate_cfg(const ottb_solver_cfg* cfg) {
  if (!cfg) return OTTB_ERR_INVALID;
  if (cfg->inner_iterations < 1 || cfg->max_iterations < 0 || cfg->min_iterations < 0)
    return OTTB_ERR_INVALID;
  if (cfg->norm_error < 1) return OTTB_ERR_UNSUPPORTED;
  if (!(cfg->eps_decay <= 1.0f) || !(cfg->eps_init > 0.0f)) return OTTB_ERR_INVALID;
  return OTTB_OK;
}

// The work plan of a call. sched_override (or else the autotune cache, or
// else the defaults) sets the schedule knobs; the workspace layout does not
// depend on them.
int make_plan(const ottb_problem* probs, int num, int d, const ottb_solver_cfg* cfg,
              bool need_grid, Plan& plan, const Schedule* sched_override = nullptr) {
  if (!probs || num < 1 || d < 1) return OTTB_ERR_INVALID;
  int st = validate_cfg(cfg);
  if (st != OTTB_OK) return st;
  if (d > 128) return OTTB_ERR_UNSUPPORTED;
  plan.num = num;
  plan.tc = wants_tc(cfg, d);
  if (plan.tc) {
    plan.dp = d <= 64 ? 64 : 128;
    plan.kern = pick_tc(plan.dp, 256);
  } else {
    plan.dp = simt_dp(d);
    plan.kern = pick_simt(plan.dp);
  }
  if (!plan.kern.fn) return OTTB_ERR_UNSUPPORTED;
  if (need_grid) {
    DeviceInfo di = device_info();
    if (di.sms <= 0) return OTTB_ERR_NO_DEVICE;
    if (di.major < 10) return OTTB_ERR_NO_DEVICE;
    plan.grid = persistent_grid(plan.kern, di.sms);
    if (plan.grid <= 0) return OTTB_ERR_CUDA;
  } else {
    plan.grid = 148;
  }
  // Problems ordered by decreasing work so the atomic queue deals the
  // largest units first.
  plan.order.resize(num);
  for (int i = 0; i < num; ++i) {
    if (probs[i].n < 1 || probs[i].m < 1) return OTTB_ERR_INVALID;
    if (probs[i].n > (int64_t)1 << 31 || probs[i].m > (int64_t)1 << 31) return OTTB_ERR_UNSUPPORTED;
    plan.order[i] = i;
  }
  std::stable_sort(plan.order.begin(), plan.order.end(), [&](int a, int b) {
    return (double)probs[a].n * probs[a].m > (double)probs[b].n * probs[b].m;
  });
  if (sched_override) {
    plan.sched = *sched_override;
  } else if (need_grid) {
    Schedule t;
    if (tuned_schedule(tune_key(probs, num, plan), &t))
      plan.sched = t;
    else if (num == 1)
      plan.sched.waves = 0;  // a single problem keeps its first split
  }
  if (num > 1) plan.sched.dynamic = 1;
  if (plan.tc) {
    if (plan.sched.tile_n != 256 && plan.sched.tile_n != 128) return OTTB_ERR_INVALID;
    plan.kern = pick_tc(plan.dp, plan.sched.tile_n);
    if (!plan.kern.fn) return OTTB_ERR_UNSUPPORTED;
    if (need_grid) {
      DeviceInfo di = device_info();
      plan.grid = persistent_grid(plan.kern, di.sms);
      if (plan.grid <= 0) return OTTB_ERR_CUDA;
    }
  }
  size_t off = 0;
  plan.off_globals = off; off = align_up(off + sizeof(Globals));
  plan.off_sched = off; off = align_up(off + sizeof(Sched));
  plan.off_probs = off; off = align_up(off + sizeof(ProbDev) * num);
  plan.off_state = off; off = align_up(off + sizeof(ProbState) * num);
  plan.off_ids = off; off = align_up(off + sizeof(int) * num);
  plan.off_prefix = off; off = align_up(off + sizeof(int) * 2 * (num + 1));
  plan.off_eval_ids = off; off = align_up(off + sizeof(int) * num);
  plan.off_eval_prefix = off; off = align_up(off + sizeof(int) * (num + 1));
  plan.off_ptrs = off; off = align_up(off + sizeof(float*) * 4 * num);
  plan.off_maps = off; off = align_up(off + (plan.tc ? sizeof(TcMaps) * num : 0));
  plan.header_bytes = off;
  plan.probs.resize(num);
  for (int t = 0; t < num; ++t) {
    const ottb_problem& q = probs[plan.order[t]];
    ProbPlan& pp = plan.probs[t];
    pp.n = q.n;
    pp.m = q.m;
    // Points are padded to whole column tiles (128 columns on the CUDA
    // cores, 256 on the tensor cores); row blocks of 128 cover the real rows.
    const int64_t tile_n = plan.tc ? kTcPad : kBN;
    pp.n_pad = round_up(q.n, tile_n);
    pp.m_pad = round_up(q.m, tile_n);
    pp.rb_f = (int)((q.n + kBM - 1) / kBM);
    pp.rb_g = (int)((q.m + kBM - 1) / kBM);
    const int cap = num > 1 ? kMaxSplitBatch : kMaxSplitSingle;
    pp.smax_f = (int)std::max<int64_t>(1, std::min<int64_t>(cap, pp.m_pad / tile_n));
    pp.smax_g = (int)std::max<int64_t>(1, std::min<int64_t>(cap, pp.n_pad / tile_n));
    auto scaled = [&](int s0, int smax) {
      return std::max(1, std::min(smax, (s0 * plan.sched.split_scale + 2) / 4));
    };
    auto base = [&](int rb, int64_t pad) {
      const int nt = (int)(pad / tile_n);
      return plan.tc && num == 1 ? choose_split_tc(rb, nt, plan.grid)
                                 : choose_split(rb, nt, plan.grid, num);
    };
    pp.split_f = scaled(base(pp.rb_f, pp.m_pad), pp.smax_f);
    pp.split_g = scaled(base(pp.rb_g, pp.n_pad), pp.smax_g);
    const size_t fsz = sizeof(float);
    // FP32 engine: transposed [DP][pad] floats; tensor cores: [2][pad][DK] bf16
    const size_t elt = plan.tc ? 2 * 2 : fsz;
    pp.off_xt = off; off = align_up(off + elt * plan.dp * pp.n_pad);
    pp.off_yt = off; off = align_up(off + elt * plan.dp * pp.m_pad);
    pp.off_nx = off; off = align_up(off + fsz * pp.n_pad);
    pp.off_ny = off; off = align_up(off + fsz * pp.m_pad);
    pp.off_galt = off; off = align_up(off + fsz * pp.m);
    // Partials of split sweeps, sized for the largest split (smax_f for the
    // f-sweep over n rows, smax_g for the g-sweep over m rows).
    const int64_t parts = std::max((int64_t)pp.smax_f * pp.n, (int64_t)pp.smax_g * pp.m);
    const bool split = pp.smax_f > 1 || pp.smax_g > 1;
    pp.off_pm = off; off = align_up(off + (split ? fsz * parts : 0));
    pp.off_pl = off; off = align_up(off + (split ? fsz * parts : 0));
    pp.off_arr = off; off = align_up(off + sizeof(int) * std::max(pp.rb_f, pp.rb_g));
    pp.off_err = off; off = align_up(off + sizeof(double) * pp.rb_g);
    pp.off_msum = off; off = align_up(off + sizeof(double) * pp.rb_g);
    // tensor-core path: column-shift rows, 16 bytes per point (y: per g buffer)
    pp.off_extx = off; off = align_up(off + (plan.tc ? 16 * pp.n_pad : 0));
    pp.off_exty = off; off = align_up(off + (plan.tc ? 16 * 2 * pp.m_pad : 0));
    pp.off_cen = off; off = align_up(off + fsz * 128);
    // tensor-core path: the rows' log-sum-exps of their last sweep
    pp.off_lprev = off; off = align_up(off + (plan.tc ? fsz * (pp.n_pad + pp.m_pad) : 0));
  }
  plan.off_pristine = off; off = align_up(off + plan.header_bytes);
  plan.total = off;
  return OTTB_OK;
}

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA; }

int check_problems(const ottb_problem* problems, int num_problems) {
  for (int i = 0; i < num_problems && problems; ++i) {
    const ottb_problem& q = problems[i];
    if (!q.x || !q.y || !q.a || !q.b || !q.f || !q.g || !q.errors) return OTTB_ERR_INVALID;
    if (!(q.epsilon > 0.0f) || !std::isfinite(q.epsilon)) return OTTB_ERR_INVALID;
    if (!(q.inv_scale_cost > 0.0f) || !std::isfinite(q.inv_scale_cost)) return OTTB_ERR_INVALID;
    if (q.symmetric != 0 && (q.symmetric != 1 || q.x != q.y || q.a != q.b || q.n != q.m))
      return OTTB_ERR_INVALID;
  }
  return OTTB_OK;
}

int outer_of(const ottb_solver_cfg* cfg) {
  return (int)std::ceil((double)cfg->max_iterations / cfg->inner_iterations);
}

// Writes the call header (tables, tensor maps, schedule, initial state)
// into the pristine region of the workspace: one host-to-device copy.
int write_header(const ottb_problem* problems, int num_problems, const ottb_solver_cfg* cfg,
                 const Plan& plan, char* ws, cudaStream_t stream,
                 float* const* marg_out = nullptr, float* const* lse_out = nullptr) {
  const int outer = outer_of(cfg);
  std::vector<char> host(plan.header_bytes, 0);
  Sched* sched = (Sched*)(host.data() + plan.off_sched);
  ProbDev* pd = (ProbDev*)(host.data() + plan.off_probs);
  ProbState* ps = (ProbState*)(host.data() + plan.off_state);
  int* ids = (int*)(host.data() + plan.off_ids);
  int* prefix = (int*)(host.data() + plan.off_prefix);
  const float** ptrs = (const float**)(host.data() + plan.off_ptrs);
  int ug = 0, uf = 0;
  for (int t = 0; t < num_problems; ++t) {
    const ottb_problem& q = problems[plan.order[t]];
    const ProbPlan& pp = plan.probs[t];
    ProbDev P;
    std::memset(&P, 0, sizeof(P));
    P.a = q.a;
    P.b = q.b;
    P.f = q.f;
    P.gbuf[0] = q.g;
    P.gbuf[1] = (float*)(ws + pp.off_galt);
    P.errors = q.errors;
    if (plan.tc) {
      P.xh = ws + pp.off_xt;
      P.yh = ws + pp.off_yt;
      TcMaps maps;  // 64-byte aligned, then copied into the header image
      if (!encode_points_map(&maps.x, ws + pp.off_xt, pp.n_pad, plan.dp) ||
          !encode_points_map(&maps.y, ws + pp.off_yt, pp.m_pad, plan.dp) ||
          !encode_ext_map(&maps.extx, ws + pp.off_extx, pp.n_pad) ||
          !encode_ext_map(&maps.exty, ws + pp.off_exty, 2 * pp.m_pad))
        return OTTB_ERR_CUDA;
      P.extx = ws + pp.off_extx;
      P.exty = ws + pp.off_exty;
      P.lprev = (float*)(ws + pp.off_lprev);
      P.dkey = &((ProbState*)(ws + plan.off_state))[t].dkey[0][0][0];
      std::memcpy(host.data() + plan.off_maps + sizeof(TcMaps) * t, &maps, sizeof(TcMaps));
      P.maps = ws + plan.off_maps + sizeof(TcMaps) * t;
    } else {
      P.xt = (const float*)(ws + pp.off_xt);
      P.yt = (const float*)(ws + pp.off_yt);
    }
    P.nx = (const float*)(ws + pp.off_nx);
    P.ny = (const float*)(ws + pp.off_ny);
    P.center = (float*)(ws + pp.off_cen);
    P.part_m = (float*)(ws + pp.off_pm);
    P.part_l = (float*)(ws + pp.off_pl);
    P.arrive = (int*)(ws + pp.off_arr);
    P.err_part = (double*)(ws + pp.off_err);
    P.msum_part = (double*)(ws + pp.off_msum);
    P.n = pp.n;
    P.m = pp.m;
    P.n_pad = pp.n_pad;
    P.m_pad = pp.m_pad;
    P.rb_f = pp.rb_f;
    P.rb_g = pp.rb_g;
    P.smax_f = pp.smax_f;
    P.smax_g = pp.smax_g;
    P.eps_target = q.epsilon;
    P.inv_scale = q.inv_scale_cost;
    // sweep_wscale at multiplier 1, the same FP32 value the kernels derive
    P.ws_t = (float)(kLog2eD / ((double)q.epsilon * 1.0));
    P.uid = plan.order[t];
    P.outer = outer;
    P.symmetric = q.symmetric;
    P.marg_out = marg_out ? marg_out[plan.order[t]] : nullptr;
    P.lse_out = lse_out ? lse_out[plan.order[t]] : nullptr;
    pd[t] = P;
    ps[t].active = 1;
    for (int k = 0; k < 2; ++k)
      for (int sl = 0; sl < 2; ++sl) {
        ps[t].dkey[k][sl][0] = kDkeyEmptyMax;
        ps[t].dkey[k][sl][1] = kDkeyEmptyMin;
      }
    ps[t].split_f = pp.split_f;
    ps[t].split_g = pp.split_g;
    ids[t] = t;
    prefix[t] = ug;
    prefix[num_problems + 1 + t] = uf;
    ug += pp.rb_g * pp.split_g;
    uf += q.symmetric ? 0 : pp.rb_f * pp.split_f;
    ptrs[2 * t] = q.x;
    ptrs[2 * t + 1] = q.y;
    ptrs[2 * num_problems + 2 * t] = q.f_init;
    ptrs[2 * num_problems + 2 * t + 1] = q.g_init;
  }
  prefix[num_problems] = ug;
  prefix[2 * num_problems + 1] = uf;
  sched->num_active = num_problems;
  sched->total_units[0] = ug;
  sched->total_units[1] = uf;
  sched->status = OTTB_OK;
  sched->dynamic_units = plan.sched.dynamic;
  sched->target_units = plan.sched.waves * plan.grid;
  // Pageable source: the copy is staged before cudaMemcpyAsync returns.
  const cudaError_t e = cudaMemcpyAsync(ws + plan.off_pristine, host.data(), plan.header_bytes,
                                        cudaMemcpyHostToDevice, stream);
  return e == cudaSuccess ? OTTB_OK : OTTB_ERR_CUDA;
}

// The device side of a solve: restore the header from its pristine copy,
// clear the split-arrival counters, then fill errors -> prep points -> init
// potentials -> persistent loop (cooperative) -> finalize. Stream
// operations only (a device-to-device copy, memsets, kernel launches).
// finalize = false leaves out finalize_kernel (the result records, the
// user g copy): for zero-iteration solves whose only output is marg_out or
// lse_out, written by the persistent kernel itself.
int launch_solve(int num_problems, int d, const ottb_solver_cfg* cfg, ottb_result* results,
                 const Plan& plan, char* ws, cudaStream_t stream, bool finalize = true) {
  cudaError_t e;
  e = cudaMemcpyAsync(ws, ws + plan.off_pristine, plan.header_bytes, cudaMemcpyDeviceToDevice,
                      stream);
  if (e != cudaSuccess) return OTTB_ERR_CUDA;
  for (int t = 0; t < num_problems; ++t) {
    const ProbPlan& pp = plan.probs[t];
    e = cudaMemsetAsync(ws + pp.off_arr, 0, sizeof(int) * std::max(pp.rb_f, pp.rb_g), stream);
    if (e != cudaSuccess) return OTTB_ERR_CUDA;
  }
  ProbDev* d_probs = (ProbDev*)(ws + plan.off_probs);
  const float* const* d_ptrs = (const float* const*)(ws + plan.off_ptrs);
  int64_t maxpts = 1;
  for (const ProbPlan& pp : plan.probs) maxpts = std::max(maxpts, pp.n_pad + 2 * pp.m_pad);
  const int outer = outer_of(cfg);
  {
    dim3 grid(std::max(1, (outer + 255) / 256), num_problems);
    fill_errors_kernel<<<grid, 256, 0, stream>>>(d_probs);
  }
  {
    PrepArgs pa{d_ptrs, d_probs, d, plan.dp};
    // the common centre once per problem, then the points
    center_kernel<<<num_problems, 256, 0, stream>>>(pa);
    int64_t mx = 1;
    for (const ProbPlan& pp : plan.probs) mx = std::max(mx, std::max(pp.n_pad, pp.m_pad));
    // one thread per row (FP32 layout) or one warp per row, 8 rows a warp
    // (tensor-core layout)
    const int64_t per_cta = plan.tc ? 64 : 256;
    dim3 grid((unsigned)std::min<int64_t>((mx + per_cta - 1) / per_cta, 1024), num_problems, 2);
    if (plan.tc)
      prep_points_tc_kernel<<<grid, 256, 0, stream>>>(pa);
    else
      prep_points_kernel<<<grid, 256, 0, stream>>>(pa);
  }
  {
    InitArgs ia{d_ptrs + 2 * num_problems, d_probs, cfg->mask_init};
    dim3 grid((unsigned)std::min<int64_t>((maxpts + 255) / 256, 1024), num_problems);
    init_potentials_kernel<<<grid, 256, 0, stream>>>(ia);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return OTTB_ERR_CUDA;

  KernelArgs ka;
  std::memset(&ka, 0, sizeof(ka));
  ka.probs = d_probs;
  ka.state = (ProbState*)(ws + plan.off_state);
  ka.sched = (Sched*)(ws + plan.off_sched);
  ka.gl = (Globals*)(ws + plan.off_globals);
  ka.active_ids = (int*)(ws + plan.off_ids);
  ka.prefix = (int*)(ws + plan.off_prefix);
  ka.eval_ids = (int*)(ws + plan.off_eval_ids);
  ka.eval_prefix = (int*)(ws + plan.off_eval_prefix);
  ka.num_problems = num_problems;
  ka.expected_arrivals = (unsigned)plan.grid + (unsigned)std::max(0, cfg->phantom_arrivals);
  const int tmo = cfg->timeout_ms > 0 ? cfg->timeout_ms : 60000;
  ka.timeout_ns = (uint64_t)tmo * 1000000ull;
  ka.cfg = *cfg;
  // Cooperative launch (all CTAs co-resident for the grid barrier), through
  // cudaLaunchKernelEx so that it can be captured into a CUDA graph.
  cudaLaunchConfig_t lc;
  std::memset(&lc, 0, sizeof(lc));
  lc.gridDim = dim3(plan.grid);
  lc.blockDim = dim3(plan.kern.threads);
  lc.dynamicSmemBytes = plan.kern.smem;
  lc.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  lc.attrs = attr;
  lc.numAttrs = 1;
  void* kargs[] = {&ka};
  e = cudaLaunchKernelExC(&lc, plan.kern.fn, kargs);
  if (e != cudaSuccess) return OTTB_ERR_CUDA;
  if (!finalize) return OTTB_OK;

  FinalArgs fa{d_probs, ka.state, ka.sched, results, *cfg};
  finalize_kernel<<<num_problems, 512, 0, stream>>>(fa);
  return cuda_status(cudaGetLastError());
}

int plan_for_call(const ottb_problem* problems, int32_t num_problems, int32_t d,
                  const ottb_solver_cfg* cfg, void* workspace, size_t workspace_bytes,
                  Plan& plan, const Schedule* sched_override = nullptr) {
  int st = check_problems(problems, num_problems);
  if (st != OTTB_OK) return st;
  st = make_plan(problems, num_problems, d, cfg, true, plan, sched_override);
  if (st != OTTB_OK) return st;
  if (!workspace || workspace_bytes < plan.total) return OTTB_ERR_WORKSPACE;
  if (((uintptr_t)workspace) % kAlign != 0) return OTTB_ERR_WORKSPACE;
  return OTTB_OK;
}

// ---------------------------------------------------------------------------
// The plan applied to vectors through the solver's sweep engine.
//
// A solve with max_iterations = 0 keeps its initial potentials and runs one
// evaluation sweep, whose column marginal is
//   sum_i exp((f'_i + g_j - C_ij) / eps).
// With f'_i = f_i + eps log v_i that is (P^T v)_j for a vector v >= 0, so a
// signed vector is two such problems (v+ and v-), and K vectors are 2K
// problems in one launch. Axis 1 (P v over the columns) swaps the roles of
// the point sets. The sweep is the solver's: tcgen05 BF16 split-3 for d >= 32
// under OTTB_PRECISION_AUTO / BF16_SPLIT3, FP32 otherwise.
// ---------------------------------------------------------------------------
struct SweepApply {
  int64_t R = 0;  // points summed over (rows of each problem's x)
  int64_t C = 0;  // points of the output (each problem's y)
  int K = 0;
  ottb_solver_cfg cfg{};
  Plan plan;
  size_t off_fp = 0, off_fo = 0, off_go = 0, off_wa = 0, off_wb = 0, off_err = 0,
         off_marg = 0, off_res = 0, off_gz = 0, total = 0;
};

__global__ void sweep_apply_potential_kernel(const float* pot, const float* vec, int64_t R,
                                             int K, float eps, float* fp) {
  const int64_t total = (int64_t)2 * K * R;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t q = idx / R, i = idx % R;
    const int k = (int)(q >> 1);
    const float v = vec[(int64_t)k * R + i];
    const float w = (q & 1) ? -v : v;
    fp[idx] = w > 0.f ? pot[i] + eps * logf(w) : -INFINITY;
  }
}

__global__ void fill_kernel(float* p, int64_t n, float v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

__global__ void sweep_apply_diff_kernel(const float* marg, int64_t C, int K, float* out) {
  const int64_t total = (int64_t)K * C;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = idx / C, j = idx % C;
    out[idx] = marg[(2 * k) * C + j] - marg[(2 * k + 1) * C + j];
  }
}

// Problem records, configuration and workspace layout; with ws null only
// the sizes are meaningful.
int sweep_apply_setup(const float* x, const float* y, int64_t n, int64_t m, int d,
                      const float* f, const float* g, float eps, float inv, int K, int axis,
                      int precision, char* ws, bool need_grid, SweepApply& S,
                      std::vector<ottb_problem>& probs, std::vector<float*>& marg) {
  S.R = axis == 0 ? n : m;
  S.C = axis == 0 ? m : n;
  S.K = K;
  ottb_solver_cfg& c = S.cfg;
  std::memset(&c, 0, sizeof(c));
  c.threshold = 1e-3f;
  c.norm_error = 1;
  c.inner_iterations = 1;
  c.min_iterations = 0;
  c.max_iterations = 0;
  c.eps_init = 1.f;
  c.eps_decay = 1.f;
  c.precision = precision;
  const int np = 2 * K;
  probs.assign(np, ottb_problem{});
  marg.assign(np, nullptr);
  for (int q = 0; q < np; ++q) {
    ottb_problem& P = probs[q];
    P.x = axis == 0 ? x : y;
    P.y = axis == 0 ? y : x;
    P.n = S.R;
    P.m = S.C;
    P.epsilon = eps;
    P.inv_scale_cost = inv;
  }
  int st = make_plan(probs.data(), np, d, &c, need_grid, S.plan);
  if (st != OTTB_OK) return st;
  size_t off = align_up(S.plan.total);
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = align_up(off + bytes);
    return o;
  };
  S.off_fp = take(sizeof(float) * np * S.R);
  S.off_fo = take(sizeof(float) * np * S.R);
  S.off_go = take(sizeof(float) * np * S.C);
  S.off_wa = take(sizeof(float) * S.R);
  S.off_wb = take(sizeof(float) * S.C);
  S.off_err = take(sizeof(float) * np);
  S.off_marg = take(sizeof(float) * np * S.C);
  S.off_res = take(sizeof(ottb_result) * np);
  S.off_gz = take(sizeof(float) * S.C);
  S.total = off;
  if (!ws) return OTTB_OK;
  for (int q = 0; q < np; ++q) {
    ottb_problem& P = probs[q];
    P.a = (const float*)(ws + S.off_wa);
    P.b = (const float*)(ws + S.off_wb);
    P.f_init = (const float*)(ws + S.off_fp) + (int64_t)q * S.R;
    P.g_init = axis == 0 ? g : f;
    P.f = (float*)(ws + S.off_fo) + (int64_t)q * S.R;
    P.g = (float*)(ws + S.off_go) + (int64_t)q * S.C;
    P.errors = (float*)(ws + S.off_err) + q;
    marg[q] = (float*)(ws + S.off_marg) + (int64_t)q * S.C;
  }
  return OTTB_OK;
}

// The part of a sweep product fixed by its sizes, points, the potential of
// the output side and the workspace: the layout, the uniform weights and the
// problem header (whose pristine copy every launch restores).
int sweep_product_plan(const float* x, const float* y, int64_t n, int64_t m, int32_t d,
                       const float* f, const float* g, float epsilon, float inv_scale_cost,
                       int32_t num_vec, int32_t axis, int32_t precision, char* ws,
                       size_t workspace_bytes, cudaStream_t stream, SweepApply& S) {
  std::vector<ottb_problem> probs;
  std::vector<float*> marg;
  int st = sweep_apply_setup(x, y, n, m, d, f, g, epsilon, inv_scale_cost, num_vec, axis,
                             precision, ws, true, S, probs, marg);
  if (st != OTTB_OK) return st;
  if (workspace_bytes < S.total) return OTTB_ERR_WORKSPACE;
  fill_kernel<<<(unsigned)std::min<int64_t>((S.R + 255) / 256, 1024), 256, 0, stream>>>(
      (float*)(ws + S.off_wa), S.R, 1.f / (float)S.R);
  fill_kernel<<<(unsigned)std::min<int64_t>((S.C + 255) / 256, 1024), 256, 0, stream>>>(
      (float*)(ws + S.off_wb), S.C, 1.f / (float)S.C);
  if (cudaGetLastError() != cudaSuccess) return OTTB_ERR_CUDA;
  return write_header(probs.data(), 2 * num_vec, &S.cfg, S.plan, ws, stream, marg.data());
}

// One planned product: stream operations only. pot is the summed side's
// potential (f for axis 0, g for axis 1).
int sweep_product_run(const SweepApply& S, int32_t d, float epsilon, char* ws,
                      const float* pot, const float* vec, float* out, cudaStream_t stream) {
  const int np = 2 * S.K;
  const int64_t fp_n = (int64_t)np * S.R;
  sweep_apply_potential_kernel<<<(unsigned)std::min<int64_t>((fp_n + 255) / 256, 4096), 256, 0,
                                 stream>>>(pot, vec, S.R, S.K, epsilon,
                                           (float*)(ws + S.off_fp));
  if (cudaGetLastError() != cudaSuccess) return OTTB_ERR_CUDA;
  const int st =
      launch_solve(np, d, &S.cfg, (ottb_result*)(ws + S.off_res), S.plan, ws, stream, false);
  if (st != OTTB_OK) return st;
  const int64_t tot = (int64_t)S.K * S.C;
  sweep_apply_diff_kernel<<<(unsigned)std::min<int64_t>((tot + 255) / 256, 4096), 256, 0,
                            stream>>>((const float*)(ws + S.off_marg), S.C, S.K, out);
  return cuda_status(cudaGetLastError());
}

}  // namespace

// A sweep product planned once (ottb_apply_transport_sweep_plan) and run
// many times on its workspace.
struct ottb_sweep_product {
  SweepApply S;
  int32_t d = 0;
  float epsilon = 0.f;
  char* ws = nullptr;
};

extern "C" {

const char* ottb_version(void) { return "0.2.0"; }

const char* ottb_status_string(int32_t status) {
  switch (status) {
    case OTTB_OK: return "ok";
    case OTTB_ERR_INVALID: return "invalid argument";
    case OTTB_ERR_UNSUPPORTED: return "unsupported configuration";
    case OTTB_ERR_CUDA: return "CUDA runtime error";
    case OTTB_ERR_TIMEOUT: return "device wait timed out";
    case OTTB_ERR_WORKSPACE: return "workspace missing or too small";
    case OTTB_ERR_NO_DEVICE: return "no sm_100 device";
    case OTTB_ERR_HOST_MEMORY: return "host memory allocation failed";
    default: return "unknown status";
  }
}

size_t ottb_sinkhorn_workspace_size(const ottb_problem* problems, int32_t num_problems,
                                    int32_t d, const ottb_solver_cfg* cfg) {
  Plan plan;
  // The layout does not depend on the grid or the schedule; without a
  // device the plan is made for a 148-SM grid.
  if (make_plan(problems, num_problems, d, cfg, true, plan) != OTTB_OK) {
    if (make_plan(problems, num_problems, d, cfg, false, plan) != OTTB_OK) return 0;
  }
  return plan.total;
}

int32_t ottb_sinkhorn_prepare(const ottb_problem* problems, int32_t num_problems, int32_t d,
                              const ottb_solver_cfg* cfg, void* workspace,
                              size_t workspace_bytes, void* stream_ptr) {
  Plan plan;
  int st = plan_for_call(problems, num_problems, d, cfg, workspace, workspace_bytes, plan);
  if (st != OTTB_OK) return st;
  return write_header(problems, num_problems, cfg, plan, (char*)workspace,
                      (cudaStream_t)stream_ptr);
}

int32_t ottb_sinkhorn_launch(const ottb_problem* problems, int32_t num_problems, int32_t d,
                             const ottb_solver_cfg* cfg, ottb_result* results,
                             void* workspace, size_t workspace_bytes, void* stream_ptr) {
  if (!results) return OTTB_ERR_INVALID;
  Plan plan;
  int st = plan_for_call(problems, num_problems, d, cfg, workspace, workspace_bytes, plan);
  if (st != OTTB_OK) return st;
  return launch_solve(num_problems, d, cfg, results, plan, (char*)workspace,
                      (cudaStream_t)stream_ptr);
}

int32_t ottb_sinkhorn_pointcloud(const ottb_problem* problems, int32_t num_problems,
                                 int32_t d, const ottb_solver_cfg* cfg,
                                 ottb_result* results, void* workspace,
                                 size_t workspace_bytes, void* stream_ptr) {
  if (!results) return OTTB_ERR_INVALID;
  Plan plan;
  int st = plan_for_call(problems, num_problems, d, cfg, workspace, workspace_bytes, plan);
  if (st != OTTB_OK) return st;
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  st = write_header(problems, num_problems, cfg, plan, (char*)workspace, stream);
  if (st != OTTB_OK) return st;
  return launch_solve(num_problems, d, cfg, results, plan, (char*)workspace, stream);
}

int32_t ottb_sinkhorn_autotune(const ottb_problem* problems, int32_t num_problems, int32_t d,
                               const ottb_solver_cfg* cfg, ottb_result* results,
                               void* workspace, size_t workspace_bytes, void* stream_ptr,
                               int32_t force) {
  if (!results) return OTTB_ERR_INVALID;
  Plan base;
  int st = plan_for_call(problems, num_problems, d, cfg, workspace, workspace_bytes, base);
  if (st != OTTB_OK) return st;
  const TuneKey key = tune_key(problems, num_problems, base);
  Schedule cached;
  if (!force && tuned_schedule(key, &cached)) return OTTB_OK;
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) return OTTB_ERR_CUDA;
  if (cap != cudaStreamCaptureStatusNone) return OTTB_ERR_INVALID;  // trials synchronise
  // Candidate schedules: initial split of a single problem (x1/2, x1, x2;
  // round-robin or queued units; the split stays as chosen); for several
  // problems, how far the splits of the problems still
  // iterating may grow (0, 1, 2, 4 waves of units). On the tensor cores each
  // of these with 256- and with 128-column tiles.
  std::vector<Schedule> cands;
  for (int tile : {256, 128}) {
    if (tile != 256 && !base.tc) break;
    if (num_problems == 1) {
      for (int scale : {4, 2, 8})
        for (int dyn : {0, 1}) {
          Schedule c;
          c.split_scale = scale;
          c.dynamic = dyn;
          c.tile_n = tile;
          c.waves = 0;
          cands.push_back(c);
        }
    } else {
      for (int w : {2, 0, 1, 4}) {
        Schedule c;
        c.waves = w;
        c.dynamic = 1;
        c.tile_n = tile;
        cands.push_back(c);
      }
    }
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return OTTB_ERR_CUDA;
  }
  float best_ms = 0.f;
  Schedule best = cands[0];
  for (size_t i = 0; i < cands.size() && st == OTTB_OK; ++i) {
    Plan plan;
    st = plan_for_call(problems, num_problems, d, cfg, workspace, workspace_bytes, plan,
                       &cands[i]);
    if (st != OTTB_OK) break;
    st = write_header(problems, num_problems, cfg, plan, (char*)workspace, stream);
    // one untimed run, then one timed run of the whole solve
    for (int rep = 0; rep < 2 && st == OTTB_OK; ++rep) {
      if (rep == 1 && cudaEventRecord(e0, stream) != cudaSuccess) st = OTTB_ERR_CUDA;
      if (st == OTTB_OK)
        st = launch_solve(num_problems, d, cfg, results, plan, (char*)workspace, stream);
      if (rep == 1 && st == OTTB_OK && cudaEventRecord(e1, stream) != cudaSuccess)
        st = OTTB_ERR_CUDA;
    }
    if (st != OTTB_OK) break;
    if (cudaEventSynchronize(e1) != cudaSuccess) { st = OTTB_ERR_CUDA; break; }
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) { st = OTTB_ERR_CUDA; break; }
    if (i == 0 || ms < best_ms) {
      best_ms = ms;
      best = cands[i];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != OTTB_OK) return st;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  tune_cache()[key] = best;
  return OTTB_OK;
}

int32_t ottb_sinkhorn_set_schedule(const ottb_problem* problems, int32_t num_problems,
                                   int32_t d, const ottb_solver_cfg* cfg, int32_t split_scale,
                                   int32_t waves, int32_t dynamic, int32_t tile_n) {
  if (split_scale < 1 || split_scale > 128 || waves < 0 || waves > 64) return OTTB_ERR_INVALID;
  if (dynamic != 0 && dynamic != 1) return OTTB_ERR_INVALID;
  if (tile_n != 256 && tile_n != 128) return OTTB_ERR_INVALID;
  int st = check_problems(problems, num_problems);
  if (st != OTTB_OK) return st;
  Plan base;
  st = make_plan(problems, num_problems, d, cfg, true, base);
  if (st != OTTB_OK) return st;
  Schedule sc;
  sc.split_scale = split_scale;
  sc.waves = waves;
  sc.dynamic = dynamic;
  sc.tile_n = tile_n;
  Plan check;  // the schedule must give a valid plan (and a launchable kernel)
  st = make_plan(problems, num_problems, d, cfg, true, check, &sc);
  if (st != OTTB_OK) return st;
  const TuneKey key = tune_key(problems, num_problems, base);
  std::lock_guard<std::mutex> lock(g_tune_mu);
  tune_cache()[key] = sc;
  return OTTB_OK;
}

size_t ottb_apply_transport_sweep_workspace_size(int64_t n, int64_t m, int32_t d,
                                                 int32_t num_vec, int32_t axis,
                                                 int32_t precision) {
  if (n < 1 || m < 1 || d < 1 || num_vec < 1 || (axis != 0 && axis != 1)) return 0;
  SweepApply S;
  std::vector<ottb_problem> probs;
  std::vector<float*> marg;
  if (sweep_apply_setup(nullptr, nullptr, n, m, d, nullptr, nullptr, 1.f, 1.f, num_vec, axis,
                        precision, nullptr, false, S, probs, marg) != OTTB_OK)
    return 0;
  return S.total;
}

int32_t ottb_apply_transport_sweep(const float* x, const float* y, int64_t n, int64_t m,
                                   int32_t d, const float* f, const float* g, float epsilon,
                                   float inv_scale_cost, const float* vec, int32_t num_vec,
                                   int32_t axis, int32_t precision, float* out,
                                   void* workspace, size_t workspace_bytes, void* stream_ptr) {
  if (!x || !y || !f || !g || !vec || !out || n < 1 || m < 1 || d < 1 || num_vec < 1)
    return OTTB_ERR_INVALID;
  if (axis != 0 && axis != 1) return OTTB_ERR_INVALID;
  if (!(epsilon > 0.f) || !(inv_scale_cost > 0.f)) return OTTB_ERR_INVALID;
  if (!workspace || ((uintptr_t)workspace) % kAlign != 0) return OTTB_ERR_WORKSPACE;
  char* ws = (char*)workspace;
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  SweepApply S;
  int st = sweep_product_plan(x, y, n, m, d, f, g, epsilon, inv_scale_cost, num_vec, axis,
                              precision, ws, workspace_bytes, stream, S);
  if (st != OTTB_OK) return st;
  return sweep_product_run(S, d, epsilon, ws, axis == 0 ? f : g, vec, out, stream);
}

int32_t ottb_apply_transport_sweep_plan(const float* x, const float* y, int64_t n, int64_t m,
                                        int32_t d, const float* f, const float* g,
                                        float epsilon, float inv_scale_cost, int32_t num_vec,
                                        int32_t axis, int32_t precision, void* workspace,
                                        size_t workspace_bytes, void* stream_ptr,
                                        ottb_sweep_product** product) {
  if (!product) return OTTB_ERR_INVALID;
  *product = nullptr;
  if (axis != 0 && axis != 1) return OTTB_ERR_INVALID;
  // the output side's potential is bound here; the summed side's comes with each run
  if (!x || !y || !(axis == 0 ? g : f) || n < 1 || m < 1 || d < 1 || num_vec < 1)
    return OTTB_ERR_INVALID;
  if (!(epsilon > 0.f) || !(inv_scale_cost > 0.f)) return OTTB_ERR_INVALID;
  if (!workspace || ((uintptr_t)workspace) % kAlign != 0) return OTTB_ERR_WORKSPACE;
  ottb_sweep_product* h = new (std::nothrow) ottb_sweep_product;
  if (!h) return OTTB_ERR_HOST_MEMORY;
  const int st = sweep_product_plan(x, y, n, m, d, f, g, epsilon, inv_scale_cost, num_vec, axis,
                                    precision, (char*)workspace, workspace_bytes,
                                    (cudaStream_t)stream_ptr, h->S);
  if (st != OTTB_OK) {
    delete h;
    return st;
  }
  h->d = d;
  h->epsilon = epsilon;
  h->ws = (char*)workspace;
  *product = h;
  return OTTB_OK;
}

int32_t ottb_apply_transport_sweep_run(const ottb_sweep_product* product, const float* pot,
                                       const float* vec, float* out, void* stream_ptr) {
  if (!product || !pot || !vec || !out) return OTTB_ERR_INVALID;
  return sweep_product_run(product->S, product->d, product->epsilon, product->ws, pot, vec, out,
                           (cudaStream_t)stream_ptr);
}

void ottb_apply_transport_sweep_free(ottb_sweep_product* product) { delete product; }

size_t ottb_apply_lse_kernel_workspace_size(int64_t n, int64_t m, int32_t d, int32_t axis,
                                            int32_t precision) {
  if (n < 1 || m < 1 || d < 1 || (axis != 0 && axis != 1)) return 0;
  SweepApply S;
  std::vector<ottb_problem> probs;
  std::vector<float*> marg;
  // one problem: the layout of a one-vector application holds it
  if (sweep_apply_setup(nullptr, nullptr, n, m, d, nullptr, nullptr, 1.f, 1.f, 1, axis,
                        precision, nullptr, false, S, probs, marg) != OTTB_OK)
    return 0;
  return S.total;
}

int32_t ottb_apply_lse_kernel(const float* x, const float* y, int64_t n, int64_t m,
                              int32_t d, const float* pot, float epsilon,
                              float inv_scale_cost, int32_t axis, int32_t precision,
                              float* out, void* workspace, size_t workspace_bytes,
                              void* stream_ptr) {
  if (!x || !y || !pot || !out || n < 1 || m < 1 || d < 1) return OTTB_ERR_INVALID;
  if (axis != 0 && axis != 1) return OTTB_ERR_INVALID;
  if (!(epsilon > 0.f) || !(inv_scale_cost > 0.f)) return OTTB_ERR_INVALID;
  if (!workspace || ((uintptr_t)workspace) % kAlign != 0) return OTTB_ERR_WORKSPACE;
  char* ws = (char*)workspace;
  SweepApply S;
  std::vector<ottb_problem> probs;
  std::vector<float*> marg;
  int st = sweep_apply_setup(x, y, n, m, d, pot, pot, epsilon, inv_scale_cost, 1, axis,
                             precision, ws, true, S, probs, marg);
  if (st != OTTB_OK) return st;
  if (workspace_bytes < S.total) return OTTB_ERR_WORKSPACE;
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  // one zero-iteration problem: row potential pot, column potential 0; the
  // final sweep's log-sum-exp goes to out
  probs.resize(1);
  probs[0].f_init = pot;
  probs[0].g_init = (const float*)(ws + S.off_gz);
  if (cudaMemsetAsync(ws + S.off_gz, 0, sizeof(float) * S.C, stream) != cudaSuccess)
    return OTTB_ERR_CUDA;
  fill_kernel<<<(unsigned)std::min<int64_t>((S.R + 255) / 256, 1024), 256, 0, stream>>>(
      (float*)(ws + S.off_wa), S.R, 1.f / (float)S.R);
  fill_kernel<<<(unsigned)std::min<int64_t>((S.C + 255) / 256, 1024), 256, 0, stream>>>(
      (float*)(ws + S.off_wb), S.C, 1.f / (float)S.C);
  if (cudaGetLastError() != cudaSuccess) return OTTB_ERR_CUDA;
  Plan plan1;
  st = make_plan(probs.data(), 1, d, &S.cfg, true, plan1);
  if (st != OTTB_OK) return st;
  if (plan1.total > S.off_fp) return OTTB_ERR_WORKSPACE;  // the solver region of the layout
  float* lse[1] = {out};
  st = write_header(probs.data(), 1, &S.cfg, plan1, ws, stream, nullptr, lse);
  if (st != OTTB_OK) return st;
  return launch_solve(1, d, &S.cfg, (ottb_result*)(ws + S.off_res), plan1, ws, stream, false);
}

size_t ottb_cost_stats_workspace_size(int64_t n, int64_t m, int32_t d) {
  if (n < 1 || m < 1 || d < 1 || d > 128) return 0;
  const size_t K = (size_t)moments_len(d, 1);
  return align_up(sizeof(double) * K * 2 * 148) + align_up(sizeof(double) * 2 * K);
}

int32_t ottb_cost_stats(const float* x, const float* y, int64_t n, int64_t m, int32_t d,
                        float inv_scale_cost, int32_t second, double* out, void* workspace,
                        size_t workspace_bytes, void* stream_ptr) {
  if (!x || !y || !out || n < 1 || m < 1 || d < 1) return OTTB_ERR_INVALID;
  if (d > 128) return OTTB_ERR_UNSUPPORTED;
  const size_t need = ottb_cost_stats_workspace_size(n, m, d);
  if (!workspace || workspace_bytes < need) return OTTB_ERR_WORKSPACE;
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  second = second ? 1 : 0;
  const int K = moments_len(d, second);
  const int64_t pts = std::max(n, m);
  const int nblk = (int)std::min<int64_t>(148, (pts + 255) / 256);
  double* px = (double*)workspace;
  double* py = px + (size_t)K * nblk;
  double* mom = (double*)((char*)workspace + align_up(sizeof(double) * moments_len(d, 1) * 2 * 148));
  const size_t smem = sizeof(double) * (K + 64) + sizeof(float) * 64 * d;
  static std::mutex mu;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (cudaFuncSetAttribute((void*)moments_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(sizeof(double) * (moments_len(128, 1) + 64) +
                                   sizeof(float) * 64 * 128)) != cudaSuccess)
      return OTTB_ERR_CUDA;
  }
  moments_kernel<<<nblk, 256, smem, stream>>>(x, n, d, second, px);
  moments_kernel<<<nblk, 256, smem, stream>>>(y, m, d, second, py);
  moments_reduce_kernel<<<(2 * K + 255) / 256, 256, 0, stream>>>(px, py, nblk, K, mom);
  cost_stats_final_kernel<<<1, 1, 0, stream>>>(mom, d, second, (double)inv_scale_cost, out);
  return cuda_status(cudaGetLastError());
}

}  // extern "C"
