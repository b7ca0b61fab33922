/*
 * ott_b200 C ABI: log-domain Sinkhorn on squared-Euclidean point clouds for
 * NVIDIA B200 (sm_100a).
 *
 * Plain C: pointers, sizes and an int status; no C++ or torch types cross the
 * boundary, nothing throws, and the library allocates no device memory. The
 * caller owns every buffer, including a workspace sized by
 * ottb_sinkhorn_workspace_size(). Every call is stream-ordered on the stream
 * it is given; calls on different streams with distinct buffers may overlap.
 *
 * Reference interfaces replaced (paths inside the ott-jax source tree):
 *   ottb_sinkhorn_pointcloud  <- ott/solvers/linear/_solve.py:29-64 (solve)
 *                                -> sinkhorn.py:782-801 (Sinkhorn.__call__),
 *                                sinkhorn.py:1052-1099 (run / iterations),
 *                                math/fixed_point_loop.py:23-93 (fixpoint_iter),
 *                                geometry/geometry.py:376-398 (update_potential),
 *                                geometry/pointcloud.py:74-103 (apply_lse_kernel),
 *                                sinkhorn.py:191-221 (marginal_error),
 *                                sinkhorn.py:224-277 (compute_kl_reg_cost)
 *   ottb_cost_stats           <- geometry/geometry.py:113-135
 *                                (mean_cost_matrix / std_cost_matrix) through
 *                                geometry/pointcloud.py:170-186 (sqeucl form)
 */
#ifndef OTT_B200_H_
#define OTT_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes returned by every entry point. */
enum {
  OTTB_OK = 0,
  OTTB_ERR_INVALID = 1,     /* bad argument (null pointer, size, config)   */
  OTTB_ERR_UNSUPPORTED = 2, /* valid in the reference, not on this path    */
  OTTB_ERR_CUDA = 3,        /* a CUDA runtime call failed                  */
  OTTB_ERR_TIMEOUT = 4,     /* a device-side wait hit its time limit       */
  OTTB_ERR_WORKSPACE = 5,   /* workspace missing or too small              */
  OTTB_ERR_NO_DEVICE = 6,   /* no sm_100 device visible                    */
  OTTB_ERR_HOST_MEMORY = 7  /* a host-side allocation (a plan handle) failed */
};

/* Arithmetic used for the inner products <x_i, y_j>. */
enum {
  OTTB_PRECISION_AUTO = -1,       /* BF16 split-3 for d >= 32, else FP32   */
  OTTB_PRECISION_FP32 = 0,        /* FP32 FMAs on the CUDA cores           */
  OTTB_PRECISION_BF16_SPLIT3 = 1  /* tcgen05 BF16 hi/lo, 3 products, TMEM  */
};

/* One point-cloud problem. All pointers are device pointers. */
typedef struct ottb_problem {
  const float* x;      /* [n, d] row-major                                  */
  const float* y;      /* [m, d] row-major                                  */
  const float* a;      /* [n] first marginal (>= 0)                         */
  const float* b;      /* [m] second marginal (>= 0)                        */
  const float* f_init; /* [n] initial f, or NULL                            */
  const float* g_init; /* [m] initial g, or NULL                            */
  float* f;            /* [n] out: first potential                          */
  float* g;            /* [m] out: second potential                         */
  float* errors;       /* [ceil(max_iterations / inner_iterations)] out     */
  int64_t n;
  int64_t m;
  float epsilon;        /* target epsilon (already resolved)                */
  float inv_scale_cost; /* cost multiplier, 1 / scale_cost                  */
  int32_t symmetric;    /* 1: x == y and a == b (same pointers); the update is
                           sinkhorn.py:836-855 with parallel_dual_updates and
                           Momentum(start=0, value=0.5) (acceleration.py:
                           164-172), which keeps f == g: one sweep per
                           iteration, g <- (fin(g) + T(g)) / 2, the error of
                           both marginals (sinkhorn.py:168-188), f = g at the
                           end. 0: the default sequential update.           */
  int32_t reserved;     /* 0                                                */
} ottb_problem;

/* Solver configuration shared by every problem of one call
 * (sinkhorn.py:718-780 defaults: threshold 1e-3, norm_error 1,
 * inner_iterations 10, min_iterations 0, max_iterations 2000). */
typedef struct ottb_solver_cfg {
  float threshold;
  int32_t norm_error;       /* p of the p-norm marginal error (>= 1)        */
  int32_t inner_iterations;
  int32_t min_iterations;
  int32_t max_iterations;
  float eps_init;           /* epsilon_scheduler.py:43-60 (init, decay)     */
  float eps_decay;
  int32_t precision;        /* OTTB_PRECISION_*                             */
  int32_t mask_init;        /* 1: f_init/g_init set to -inf where weight 0  */
  int32_t timeout_ms;       /* device wait limit, 0 = default (60 s)        */
  int32_t phantom_arrivals; /* extra grid-barrier arrivals to wait for; 0 in
                               normal use, > 0 only to exercise the timeout */
  int32_t init_f_from_g;    /* 1: before the loop, f = the f-update of the
                               initial g (the initializer predicted g; the
                               first g-update would otherwise discard it)  */
} ottb_solver_cfg;

/* Per-problem scalar results, written to device memory. */
typedef struct ottb_result {
  double reg_ot_cost;  /* sinkhorn.py:224-277, FP64 sums                    */
  double marginal_sum; /* sum_j of the column marginal of the final state   */
  int32_t n_iters;     /* sinkhorn.py:432-434                               */
  int32_t converged;   /* sinkhorn.py:1020-1023                             */
  int32_t status;      /* OTTB_OK or OTTB_ERR_TIMEOUT                       */
  int32_t reserved;
} ottb_result;

/* Bytes of workspace ottb_sinkhorn_pointcloud needs for these problems.
 * Only n, m of each problem are read. Returns 0 on invalid input. */
size_t ottb_sinkhorn_workspace_size(const ottb_problem* problems,
                                    int32_t num_problems, int32_t d,
                                    const ottb_solver_cfg* cfg);

/* Solve num_problems independent problems of dimension d in one persistent
 * launch. problems and cfg are host memory; results is a device array of
 * num_problems ottb_result. Returns OTTB_OK once the work is enqueued;
 * per-problem device-side status is in results[k].status. */
int32_t ottb_sinkhorn_pointcloud(const ottb_problem* problems,
                                 int32_t num_problems, int32_t d,
                                 const ottb_solver_cfg* cfg,
                                 ottb_result* results, void* workspace,
                                 size_t workspace_bytes, void* stream);

/* ottb_sinkhorn_pointcloud in two halves, for callers that repeat a solve
 * on the same buffers (the role jax.jit plays for ott/solvers/linear/
 * _solve.py:29-64: compile once per shape, then re-run the executable).
 *
 * ottb_sinkhorn_prepare: the host half. Plans the call and writes its
 * header (problem table, tensor maps, work schedule, initial state) into
 * the workspace with one host-to-device copy on stream.
 *
 * ottb_sinkhorn_launch: the device half, called with the same arguments as
 * the prepare that filled this workspace. Issues stream operations only (a
 * device-to-device copy that restores the header, memsets and kernel
 * launches; no host memory and no synchronisation), so it can be captured
 * into a CUDA graph and replayed. Every launch or replay solves again from
 * the current contents of the problems' x, y, a, b, f_init and g_init;
 * sizes, epsilon and buffer addresses are those given to prepare.
 * ottb_sinkhorn_pointcloud is prepare followed by launch. */
int32_t ottb_sinkhorn_prepare(const ottb_problem* problems, int32_t num_problems,
                              int32_t d, const ottb_solver_cfg* cfg, void* workspace,
                              size_t workspace_bytes, void* stream);
int32_t ottb_sinkhorn_launch(const ottb_problem* problems, int32_t num_problems,
                             int32_t d, const ottb_solver_cfg* cfg,
                             ottb_result* results, void* workspace,
                             size_t workspace_bytes, void* stream);

/* No counterpart in the reference (XLA picks its own kernel schedules).
 * Times candidate work schedules of a solve with these shapes and this
 * configuration and records the fastest in a process-wide cache (guarded by
 * a mutex) that every later plan with the same shapes on this device uses:
 * for one problem, the column split of each sweep (the heuristic choice
 * x1/2, x1, x2) and round-robin or queued dealing of work units; for
 * several problems, how far the column splits of the problems still
 * iterating may grow as others converge; on the tensor cores each of those
 * with tiles of 256 and of 128 columns. Each candidate runs the whole
 * solve twice (one untimed, one timed with CUDA events), writing the
 * problems' outputs and results; the call blocks until the trials finish
 * and refuses a stream under capture (OTTB_ERR_INVALID). Returns at once if
 * the shape is already tuned, unless force != 0. */
int32_t ottb_sinkhorn_autotune(const ottb_problem* problems, int32_t num_problems,
                               int32_t d, const ottb_solver_cfg* cfg,
                               ottb_result* results, void* workspace,
                               size_t workspace_bytes, void* stream, int32_t force);

/* Records a work schedule for calls with these shapes and this
 * configuration on the current device, in the cache ottb_sinkhorn_autotune
 * fills (no counterpart in the reference, where XLA schedules the loop):
 * later plans of such calls use it without timing trials. split_scale: a
 * single problem's column split is the heuristic one times split_scale / 4;
 * waves: the splits of problems still iterating grow while fewer than
 * waves x grid units remain (0: never; unpinned, a single problem runs
 * with 0, on the tensor cores with its split from a cost model of one
 * sweep);
 * dynamic: 1 deals work units from an
 * atomic queue, 0 round-robin (calls with several problems always queue);
 * tile_n: columns of a tensor-core tile, 256 or 128 (ignored by the
 * CUDA-core engine). OTTB_ERR_INVALID for values outside those ranges. */
int32_t ottb_sinkhorn_set_schedule(const ottb_problem* problems, int32_t num_problems,
                                   int32_t d, const ottb_solver_cfg* cfg,
                                   int32_t split_scale, int32_t waves, int32_t dynamic,
                                   int32_t tile_n);

/* Transport plan of a point-cloud problem applied to num_vec vectors, from
 * its dual potentials, without materialising the plan
 * (geometry/geometry.py:444-486, apply_transport_from_potentials; through
 * sinkhorn.py:458-469, SinkhornOutput.apply):
 *   P_ij = exp((f_i + g_j - inv_scale_cost |x_i - y_j|^2) / epsilon),
 *   axis 1: out[k][i] = sum_j P_ij vec[k][j]   (vec [num_vec][m], out [num_vec][n])
 *   axis 0: out[k][j] = sum_i P_ij vec[k][i]   (vec [num_vec][n], out [num_vec][m]).
 * x [n][d], y [m][d], f [n], g [m] (entries may be -inf), vec and out are
 * device arrays; FP32 with a running row maximum. The summed-over points
 * are split across CTAs when the output rows alone would leave SMs idle;
 * the splits' partial sums then go through the workspace (size from
 * ottb_apply_transport_workspace_size). For d <= 64 the workspace also
 * holds the operands prepared once per call for the pipelined kernels (the
 * summed-over points transposed and centred, their column terms, the
 * vectors transposed). A smaller workspace, or none, gives fewer splits and
 * the kernels that transpose their tiles themselves; the results agree up
 * to FP32 summation order. */
size_t ottb_apply_transport_workspace_size(int64_t n, int64_t m, int32_t d, int32_t num_vec,
                                           int32_t axis);
int32_t ottb_apply_transport(const float* x, const float* y, int64_t n, int64_t m,
                             int32_t d, const float* f, const float* g, float epsilon,
                             float inv_scale_cost, const float* vec, int32_t num_vec,
                             int32_t axis, float* out, void* workspace,
                             size_t workspace_bytes, void* stream);

/* The same application (geometry/geometry.py:444-486) on the tensor cores,
 * for many vectors at once (the Danskin gradients' [1, y^T] products,
 * sinkhorn.py:779-780, and the implicit pullback's plan products,
 * implicit_differentiation.py:262-287): both products are tcgen05 BF16
 * split-3 MMAs with FP32 accumulation, S = <x, y> (+ the potentials) into
 * tensor memory, its weights 2^S written back there as bf16 hi/lo pairs and
 * O += P V^T taken with P straight from tensor memory. A first pass of the
 * same kernel (the hi*hi product only) gives every output row its largest
 * exponent, so the weights need no running maximum. d <= 128; the
 * workspace (ottb_apply_transport_tc_workspace_size bytes, 256-byte
 * aligned) holds the bf16 operands, the rows' maxima and the column
 * splits' partial sums. Its first int32 is a status word, 0 after the call's
 * kernels complete normally and 1 if one of the kernel's bounded waits gave
 * up (the output is then not valid). */
size_t ottb_apply_transport_tc_workspace_size(int64_t n, int64_t m, int32_t d, int32_t num_vec,
                                              int32_t axis);
int32_t ottb_apply_transport_tc(const float* x, const float* y, int64_t n, int64_t m,
                                int32_t d, const float* f, const float* g, float epsilon,
                                float inv_scale_cost, const float* vec, int32_t num_vec,
                                int32_t axis, float* out, void* workspace,
                                size_t workspace_bytes, void* stream);

/* ottb_apply_transport planned once for fixed points and potentials and
 * run for many vectors (the implicit backward's one-vector products below
 * the tensor-core route). _plan takes the workspace
 * (ottb_apply_transport_workspace_size bytes, 256-byte aligned for the
 * prepared path) and, where the call takes the prepared path (d <= 64),
 * writes the common centre, B transposed and the column terms into it
 * once; _run takes num_vec vectors and the output. x, y, f, g and the
 * workspace must stay allocated and unchanged until _free. */
typedef struct ottb_apply_product ottb_apply_product;
int32_t ottb_apply_transport_plan(const float* x, const float* y, int64_t n, int64_t m,
                                  int32_t d, const float* f, const float* g, float epsilon,
                                  float inv_scale_cost, int32_t num_vec, int32_t axis,
                                  void* workspace, size_t workspace_bytes, void* stream,
                                  ottb_apply_product** product);
int32_t ottb_apply_transport_run(const ottb_apply_product* product, const float* vec,
                                 float* out, void* stream);
void ottb_apply_transport_free(ottb_apply_product* product);

/* The same application (geometry/geometry.py:444-486) on the solver's sweep
 * engine: tcgen05 BF16 split-3 products for d >= 32 under
 * OTTB_PRECISION_AUTO or _BF16_SPLIT3, FP32 otherwise. Each vector becomes two
 * zero-iteration solves whose final marginal sweep sums
 * exp((f_i + eps log(+-v_i) + g_j - C_ij) / eps) over i (axis 0; axis 1 swaps
 * the point sets); all 2 * num_vec run in one persistent launch and the two
 * sums are subtracted. Used for the one-vector products of the implicit
 * backward (implicit_differentiation.py:173-185, app_transport) when the
 * solve ran on the tensor cores. The workspace (size from
 * ottb_apply_transport_sweep_workspace_size, 256-byte aligned) is required. */
size_t ottb_apply_transport_sweep_workspace_size(int64_t n, int64_t m, int32_t d,
                                                 int32_t num_vec, int32_t axis,
                                                 int32_t precision);
int32_t ottb_apply_transport_sweep(const float* x, const float* y, int64_t n, int64_t m,
                                   int32_t d, const float* f, const float* g, float epsilon,
                                   float inv_scale_cost, const float* vec, int32_t num_vec,
                                   int32_t axis, int32_t precision, float* out,
                                   void* workspace, size_t workspace_bytes, void* stream);

/* The same product planned once and run many times (the implicit
 * backward's MINRES steps apply the plan to a new vector at every step,
 * with the points and potentials fixed). _plan lays out the workspace
 * (ottb_apply_transport_sweep_workspace_size bytes), writes the uniform
 * weights and the problem header into it and binds x, y and the output
 * side's potential (g for axis 0, f for axis 1; the other may be NULL);
 * it returns a handle in *product. _run takes the summed side's potential
 * (f for axis 0, g for axis 1), num_vec vectors and the output, and issues
 * stream operations only. The workspace must stay allocated and untouched
 * by anything else, and the bound buffers allocated, until _free; their
 * contents may change between runs. */
typedef struct ottb_sweep_product ottb_sweep_product;
int32_t ottb_apply_transport_sweep_plan(const float* x, const float* y, int64_t n, int64_t m,
                                        int32_t d, const float* f, const float* g,
                                        float epsilon, float inv_scale_cost, int32_t num_vec,
                                        int32_t axis, int32_t precision, void* workspace,
                                        size_t workspace_bytes, void* stream,
                                        ottb_sweep_product** product);
int32_t ottb_apply_transport_sweep_run(const ottb_sweep_product* product, const float* pot,
                                       const float* vec, float* out, void* stream);
void ottb_apply_transport_sweep_free(ottb_sweep_product* product);

/* The log-domain kernel application (geometry/geometry.py:259-299,
 * apply_lse_kernel, vec = None) on the solver's sweep engine: axis 0
 * out[j] = eps log sum_i exp((pot_i - C_ij) / eps) over x (pot = f, out over
 * y); axis 1 the same over y (pot = g, out over x). One zero-iteration solve
 * whose final sweep's log-sum-exp is written out; the per-shard step of a
 * row-sharded solve, whose column log-sum-exps are combined across ranks.
 * Workspace from ottb_apply_lse_kernel_workspace_size (256-byte aligned). */
size_t ottb_apply_lse_kernel_workspace_size(int64_t n, int64_t m, int32_t d, int32_t axis,
                                            int32_t precision);
int32_t ottb_apply_lse_kernel(const float* x, const float* y, int64_t n, int64_t m,
                              int32_t d, const float* pot, float epsilon,
                              float inv_scale_cost, int32_t axis, int32_t precision,
                              float* out, void* workspace, size_t workspace_bytes,
                              void* stream);

/* The plan itself, out [n][m] row-major (geometry/geometry.py:361-365,
 * transport_from_potentials; sinkhorn.py:346-349, SinkhornOutput.matrix). */
int32_t ottb_transport_matrix(const float* x, const float* y, int64_t n, int64_t m,
                              int32_t d, const float* f, const float* g, float epsilon,
                              float inv_scale_cost, float* out, void* stream);

/* Fixed device scratch of ottb_sinkhorn_pointcloud_noalloc, per device. */
#define OTTB_NOALLOC_SCRATCH_BYTES (16u << 20)

/* No counterpart in the reference: ott-jax runs inside XLA, which owns all
 * device memory. This is ottb_sinkhorn_pointcloud for callers that cannot
 * allocate device memory where they call the solver (a handler inside a host
 * framework that only passes it the input and output buffers, or a service
 * whose GPU memory budget is fixed at start-up). It allocates nothing: its
 * workspace is a 16 MiB (OTTB_NOALLOC_SCRATCH_BYTES) array compiled into the
 * library, held in every GPU that loads the library until the process exits.
 * Calls whose scratch need (ottb_sinkhorn_workspace_size) exceeds that return
 * OTTB_ERR_WORKSPACE before enqueuing anything. A call outside stream capture
 * looks up the array's device address on the current device; a call under
 * capture reuses the address of the last uncaptured call on that device, so
 * make one call on each device before capturing (a first call under capture
 * returns OTTB_ERR_INVALID). All calls share the array: calls whose work
 * overlaps on the GPU race, so order them (one stream). Inputs, outputs and
 * status as for ottb_sinkhorn_pointcloud. */
int32_t ottb_sinkhorn_pointcloud_noalloc(const ottb_problem* problems,
                                         int32_t num_problems, int32_t d,
                                         const ottb_solver_cfg* cfg,
                                         ottb_result* results, void* stream);

/* Bytes of workspace ottb_cost_stats needs. */
size_t ottb_cost_stats_workspace_size(int64_t n, int64_t m, int32_t d);

/* Cost-matrix statistics of one problem without materialising it.
 * out (device, 2 doubles): mean(C) and, when second != 0, mean(C^2) of
 * C_ij = inv_scale_cost * |x_i - y_j|^2 over uniform weights (out[1] is NaN
 * otherwise), from FP64 moments of x and y (fixed-order reductions,
 * deterministic). mean(C) needs O((n + m) d) work, mean(C^2) O((n + m) d^2). */
int32_t ottb_cost_stats(const float* x, const float* y, int64_t n, int64_t m,
                        int32_t d, float inv_scale_cost, int32_t second,
                        double* out, void* workspace, size_t workspace_bytes,
                        void* stream);

/* ---------------------------------------------------------------------
 * Learned initializer network (replaces the meta model of
 * ott/initializers/neural/meta_initializer.py:36-213: flax Dense layers
 * applied to concat(a, b) in _compute_f :192-207, trained with optax Adam in
 * update :101-135). Dense layers y = x W^T + b, tanh-GELU between layers,
 * linear last layer; bf16 operands on tcgen05 tensor cores with FP32
 * accumulation and FP32 master weights. Every width and the batch must be a
 * multiple of 128. All pointers are device pointers owned by the caller.
 * --------------------------------------------------------------------- */
#define OTTB_MLP_MAX_LAYERS 8

typedef struct ottb_mlp_layer {
  int32_t in;        /* input width                                      */
  int32_t out;       /* output width                                     */
  float* w;          /* [out, in] FP32 master weights                    */
  void* w_bf16;      /* [out, in] bf16 copy (GEMM operand)               */
  void* wt_bf16;     /* [in, out] bf16 transposed copy                   */
  float* b;          /* [out] bias                                       */
  float* w_m;        /* Adam first / second moments of w and b           */
  float* w_v;
  float* b_m;
  float* b_v;
  float* w_grad;     /* [out, in] written by ottb_mlp_gradients          */
  float* b_grad;     /* [out]                                            */
} ottb_mlp_layer;

typedef struct ottb_mlp {
  int32_t num_layers;
  ottb_mlp_layer layers[OTTB_MLP_MAX_LAYERS];
} ottb_mlp;

/* Workspace bytes for activations and gradients of one batch. */
size_t ottb_mlp_workspace_size(const ottb_mlp* net, int32_t batch);

/* y[batch, out] = net(x[batch, in]). *status (device int) receives
 * OTTB_ERR_TIMEOUT if a device wait gave up. */
int32_t ottb_mlp_forward(const ottb_mlp* net, const float* x, int32_t batch,
                         float* y, int32_t* status, void* workspace,
                         size_t workspace_bytes, void* stream);

/* Gradients of the batch mean of the centred squared error
 *   loss_b = sum_j w_j ((y_j - t_j) - s_b)^2 / sum_j w_j,
 *   s_b = sum_j w_j (y_j - t_j) / sum_j w_j
 * into every layer's w_grad / b_grad; weight [batch, out] (> 0) or NULL for
 * w = 1; loss_per[batch] receives each sample's loss. */
int32_t ottb_mlp_gradients(const ottb_mlp* net, const float* x,
                           const float* target, const float* weight,
                           int32_t batch, float* loss_per, int32_t* status,
                           void* workspace, size_t workspace_bytes,
                           void* stream);

/* One Adam step (bias-corrected, step >= 1) on every layer from its
 * gradients; refreshes the bf16 copies. */
int32_t ottb_mlp_adam(const ottb_mlp* net, float lr, float beta1, float beta2,
                      float eps, int32_t step, void* stream);

/* The same step with the learning rate and the bias corrections read from
 * device memory, hyper = {lr, 1 - beta1^step, 1 - beta2^step}, so that a
 * training step can be captured once in a CUDA graph and replayed with a
 * different row of a schedule each time (meta_initializer.py:101-135,
 * the update). */
int32_t ottb_mlp_adam_device(const ottb_mlp* net, const float* hyper, float beta1,
                             float beta2, float eps, void* stream);

/* Refreshes the bf16 copies (w_bf16, wt_bf16) from the FP32 weights. */
int32_t ottb_mlp_sync_bf16(const ottb_mlp* net, void* stream);

/* One MINRES step (Paige and Saunders 1975) after the operator product, for
 * the symmetric linear system of the implicit backward of the potentials
 * (implicit_differentiation.py:156-233, solved there by lineax CG /
 * NormalCG; lineax_implicit.py:49-101). On entry y = op(v); the kernel
 * finishes the Lanczos step (y -= (beta/oldb) r1 for step >= 2,
 * alfa = <v, y>, y -= (alfa/beta) r2, beta' = |y|), applies and updates the
 * Givens rotation, writes the new direction into w_prev
 * ((v - oldeps w_prev - delta w) / gamma), adds phi times it to x, writes
 * v_next = y / beta', and stores the residual estimate in history[step].
 * state[16] (float64, device): beta, oldb, dbar, epsln, phibar, cs, sn,
 * beta1, rtol, active, steps; the host sets it to beta1, 0, 0, 0, beta1,
 * -1, 0, beta1, rtol, 1, 0 and history[0] = beta1 before step 1. The stop
 * test (phibar <= rtol beta1, beta' <= 1e-14 beta1, or phibar above
 * 0.99 history[step - window]) clears active, after which later calls
 * return at once. All vectors hold s float64 values on the device;
 * 1 <= step < history_len. */
int32_t ottb_minres_step(double* state, int32_t step, int32_t window, const double* v,
                         double* y, const double* r1, const double* r2, const double* w,
                         double* w_prev, double* x, double* v_next, double* history,
                         int64_t history_len, int64_t s, void* stream);

/* ottb_minres_step with the step number kept on the device: the step run is
 * state[steps] + 1, and a call once that would reach history_len clears
 * active (the step cap) instead. The launch then has no host-side
 * argument that changes from step to step, so a fixed sequence of steps
 * and their operator products can be captured into a CUDA graph and
 * replayed; calls after the stop return at once. Same state layout and
 * initial values as ottb_minres_step; history_len >= 2. Replaces the same
 * reference solve as ottb_minres_step (implicit_differentiation.py:156-233,
 * lineax_implicit.py:49-101). */
int32_t ottb_minres_step_next(double* state, int32_t window, const double* v, double* y,
                              const double* r1, const double* r2, const double* w,
                              double* w_prev, double* x, double* v_next, double* history,
                              int64_t history_len, int64_t s, void* stream);

/* Human-readable text of a status code. */
const char* ottb_status_string(int32_t status);

/* Library version, e.g. "0.1.0". */
const char* ottb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* OTT_B200_H_ */
