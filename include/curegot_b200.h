/*
 * curegot_b200.h -- C ABI of the B200-native entropic optimal-transport engine.
 *
 * Every entry point takes plain device pointers, sizes and an explicit CUDA
 * stream, returns an int status (CG_OK == 0) and never calls exit().  Inputs
 * and outputs are owned by the caller; the library allocates its own
 * workspace (stream-ordered) and releases it before returning, except for
 * objects it hands back (backward contexts, engines), which the caller frees
 * with the matching *_destroy call.
 *
 * Each declaration cites the reference interface it replaces
 * (benben-cd/curegot_backward, paths relative to that project).
 */
#ifndef CUREGOT_B200_H
#define CUREGOT_B200_H

#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference prints and calls exit(EXIT_FAILURE) on CUDA
 * and cuDSS errors (e.g. src/sinkhorn_bcd_kernel.cu:20-27,
 * src/linsolve.cu:19-26); here every failure is returned to the caller. */
enum {
  CG_OK = 0,
  CG_ERR_INVALID_ARG = 1,      /* bad shape, pointer or parameter            */
  CG_ERR_CUDA = 2,             /* CUDA runtime / launch error                */
  CG_ERR_NOT_SPD = 3,          /* direction-solve factorization failed       */
  CG_ERR_OOM = 4,              /* device allocation failed                   */
  CG_ERR_TIMEOUT = 5,          /* bounded device wait expired                */
  CG_ERR_NONFINITE = 6,        /* non-finite state where one is not allowed  */
  CG_ERR_INVALID_CONTEXT = 7,  /* backward context missing or invalid        */
  CG_ERR_SOLVER = 8,           /* linear-solver library error                */
  CG_ERR_ADMISSION = 9,        /* request does not fit the engine budget     */
  CG_ERR_CANCELLED = 10        /* engine request cancelled by the caller     */
};

/* Human-readable text of the last error raised on the calling thread. */
const char* cg_last_error(void);
/* Library version string. */
const char* cg_version(void);
/* Kernel launches issued by the library since load / last reset (graph
 * replays count the kernels they run). */
long long cg_launch_count(void);
void cg_launch_count_reset(void);

/* The library's stream-ordered memory pool on `device` (a cudaMemPool_t),
 * created on first use.  Solver workspaces come from it; it keeps freed
 * blocks mapped (release threshold = max) so repeated solves of similar sizes
 * reuse memory without remapping.  cg_memory_pool_trim releases unused memory
 * above keep_bytes back to the driver.  No reference counterpart (the
 * reference calls cudaMalloc/cudaFree inside its loops). */
int cg_memory_pool(int device, void** pool);
int cg_memory_pool_trim(int device, size_t keep_bytes);

/* ------------------------------------------------------------------------ */
/* Sinkhorn block-coordinate descent (log-domain Sinkhorn).                  */
/* ------------------------------------------------------------------------ */

/*
 * Plain FP64 BCD.  Replaces cuda_sinkhorn_bcd (src/solvers.h:4-9,
 * src/sinkhorn_bcd_kernel.cu:429-634) with input_on_device = output_on_device
 * = true.  M is row-major n x m; a[n], b[m]; x0 (nullable) = [alpha; beta];
 * P (nullable: skip the plan) is n x m; dual (nullable) = [alpha; beta].
 * Same stopping rule and niter semantics as the reference: gauge-normalised
 * iterate difference until it drops below 10*tol, then the row-marginal
 * error ||rowsum(P) - a||_2 < tol.
 */
int cg_bcd_f64(const double* M, const double* a, const double* b, double* P, double reg,
               int max_iter, double tol, int n, int m, int* niter, const double* x0,
               double* dual, cudaStream_t stream);

/*
 * Allocation-free FP64 BCD.  No counterpart in the reference: an addition
 * for callers that must not allocate device memory at call time -- a host
 * framework that owns HBM (a preallocating allocator, or a caching allocator
 * that has reserved nearly all of it), where a stream-ordered allocation
 * inside the call can fail with out-of-memory or grow a second pool beside
 * the framework's.  Same arguments and stopping rule as cg_bcd_f64, and the same
 * kernels and results as cg_bcd_f64 takes with the cluster path disabled
 * (cg_bcd_set_cluster_path(0)): this entry point always runs the multi-CTA
 * row/column passes, so for small problems that cg_bcd_f64 would solve in
 * one cluster launch the two can differ in rounding (and, rarely, niter by
 * one).  The scratch is a 4 MiB file-scope device array inside this library
 * instead of a cudaMallocAsync block, and nothing else is allocated.
 *   - n and m must each be <= 16384, otherwise CG_ERR_INVALID_ARG (before any
 *     launch; cg_last_error() says why).
 *   - Nothing has to start at zero: every call initialises the state, the
 *     counters and the duals it uses.
 *   - The first call on each device resolves the array's address
 *     (cudaGetSymbolAddress, which may load the module): make it before any
 *     stream capture.  The call reads its state back with a stream
 *     synchronize, like cg_bcd_f64.
 *   - One array per device: calls on the same device must not overlap.  The
 *     plan/dual kernels of a call still read the array after it returns, so
 *     issue calls on one stream or synchronize between them; overlapping
 *     calls race on the scratch.
 */
int cg_bcd_f64_noalloc(const double* M, const double* a, const double* b, double* P,
                       double reg, int max_iter, double tol, int n, int m, int* niter,
                       const double* x0, double* dual, cudaStream_t stream);

/*
 * Sinkhorn path selection (process-wide; default on).  When enabled,
 * cg_bcd_f64 / cg_bcd_mixed solve problems whose cost matrix fits the shared
 * memory of one thread-block cluster (up to 16 CTAs, ~3 MB of M) in a single
 * cluster-resident launch; larger problems, and all problems when disabled,
 * use the multi-CTA row/column passes.  Same stopping rule and niter
 * semantics either way.  No reference counterpart.
 */
int cg_bcd_set_cluster_path(int enable);

/*
 * Memory pipeline of the multi-CTA Sinkhorn passes (process-wide; default
 * off: on B200 the register path measured 10-18% faster).  When enabled, rows and column strips long enough to stream are
 * brought into per-warp shared-memory rings by bulk asynchronous copies
 * (three 2 KB stages per warp, completion on mbarriers with bounded waits)
 * and read from there; disabled, the passes load M straight into registers.
 * Same arithmetic in the same order: results are bitwise identical.  A
 * staging wait that gives up ends the solve with CG_ERR_TIMEOUT.  No
 * reference counterpart.
 */
int cg_bcd_set_staging(int enable);

/*
 * Shifted log-sum-exp in the Sinkhorn row / column passes (default on).  The
 * first pass of a solve keeps a running maximum per row / column.  Later
 * passes sum 2^(x - k) with k the previous LSE of the same row (column),
 * recovered from the current dual, whenever the other side's duals moved by
 * less than 40 (base-2 exponent units) since: every term is then at most
 * 2^41 and the sum at least 2^-41, so no maximum is needed.  This removes
 * the per-element maximum and shift from the passes.  Results agree with the
 * running-maximum passes to rounding (a few ulp per LSE).  enable = 0 keeps
 * the running maximum in every pass.  Process-wide; captured engine graphs
 * keep the setting they were captured with.  No reference counterpart.
 */
int cg_bcd_set_shifted_lse(int enable);

/*
 * L2 prefetch distance of the Sinkhorn row / column passes (register path),
 * in chunks of one warp's loop step (0 = off, at most 64; default below in
 * the implementation).  Each warp sends a bulk L2 prefetch hint for the chunk
 * `chunks` steps ahead of the one it reads, so more of M is in flight than
 * the registers hold.  A hint only: results are bitwise identical for every
 * setting.  Process-wide; the serving engine's captured batch graphs keep the
 * setting they were captured with.  No reference counterpart.
 */
int cg_bcd_set_l2_prefetch(int chunks);

/*
 * Mixed-precision BCD: M stored in FP32, duals and all reductions in FP64.
 * Same contract as cg_bcd_f64; P (nullable) is written in FP64.  The
 * FP32-M form of cuda_sinkhorn_bcd; the stopping rule is evaluated with the
 * same FP64 formulas on the FP32-valued M.
 */
int cg_bcd_mixed(const float* M, const double* a, const double* b, double* P, double reg,
                 int max_iter, double tol, int n, int m, int* niter, const double* x0,
                 double* dual, cudaStream_t stream);

/* Transport plan P = exp((alpha_i + beta_j - M_ij) / reg).  Replaces
 * compute_transport_plan (src/sinkhorn_bcd_kernel.cu:383-424). */
int cg_transport_plan_f64(const double* M, const double* alpha, const double* beta,
                          double* P, double reg, int n, int m, cudaStream_t stream);
int cg_transport_plan_mixed(const float* M, const double* alpha, const double* beta,
                            double* P, double reg, int n, int m, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* SPLR (sparse-plus-low-rank quasi-Newton) and its backward context.        */
/* ------------------------------------------------------------------------ */

/* Opaque backward context: the sparsified Hessian A_k of the last forward
 * direction solve with its factorization, the secant pair (s, y), A_k^{-1} y
 * and ys.  Replaces SPLRBackwardContext (src/backward_context.h:83-376). */
typedef struct cg_ctx_s cg_ctx;

typedef struct {
  int n, m, dim;          /* dim = n + m - 1 (reduced dual)                  */
  long long nnz;          /* entries of the context CSR                      */
  double reg, ys;
  int low_rank;           /* rank-2 correction active                         */
  int fallback;           /* immediate convergence: factor at the final point */
  int valid;              /* forward state finite; usable for backward        */
  int has_diag;           /* diagonal preconditioner set up                   */
  int has_point;          /* context point available                          */
  int adopted;            /* forward factorization adopted (not a fallback)   */
} cg_ctx_info_t;

enum { CG_PRECOND_NONE = 0, CG_PRECOND_DIAG = 1, CG_PRECOND_SPLR = 2 };
enum {
  CG_CTX_CSR_VALUES = 0, CG_CTX_CSR_COLIND = 1, CG_CTX_CSR_ROWPTR = 2, CG_CTX_SECANT_S = 3,
  CG_CTX_SECANT_Y = 4, CG_CTX_INV_DIAG = 5, CG_CTX_POINT = 6, CG_CTX_INVA_Y = 7
};

/*
 * Plain FP64 SPLR.  Replaces cuda_sinkhorn_splr / cuda_sinkhorn_splr_bwd
 * (src/solvers.h:11-33; src/sinkhorn_splr.cu:1064-1611) on device pointers.
 * density_max, shift_max, sparsity_pattern_cycle and candidate_sinkhorn_iter
 * mean what the reference's kwargs mean (src/solvers_torch.cpp:212-243).
 * ctx_out (nullable): export the backward context (adopt semantics; fallback
 * factorization when niter == 0).  converged (nullable): the reference's
 * converged flag.  trace (nullable, HOST, 8 doubles x max_iter): per
 * iteration f, ||g||, step, K, low_rank, recompute_fg, candidate accepted,
 * line-search trials.  The direction solve is an exact FP64 solve with the
 * sparsified Hessian (Schur complement + cuSOLVER Cholesky) in place of cuDSS.
 */
int cg_splr_f64(const double* M, const double* a, const double* b, double* P, double reg,
                int max_iter, double tol, int n, int m, int* niter, double density_max,
                double shift_max, int sparsity_pattern_cycle, int candidate_sinkhorn_iter,
                int verbose, const double* x0, double* dual, cg_ctx** ctx_out, int* converged,
                double* trace, cudaStream_t stream);
/* Same with M in FP32 (all arithmetic, duals, line search and solve in FP64).
 * Stopping test: the full marginal error ||(T1 - a, T^T 1 - b)||_2 < tol,
 * i.e. the reference's ||g|| plus the gauge column's error, so every column
 * meets tol too (the reference's test leaves column m-1 out). */
int cg_splr_mixed(const float* M, const double* a, const double* b, double* P, double reg,
                  int max_iter, double tol, int n, int m, int* niter, double density_max,
                  double shift_max, int sparsity_pattern_cycle, int candidate_sinkhorn_iter,
                  int verbose, const double* x0, double* dual, cg_ctx** ctx_out,
                  int* converged, double* trace, cudaStream_t stream);

/*
 * Direction-solve path of the SPLR Newton step (process-wide setting).  The
 * reference always calls cuDSS sparse Cholesky (src/linsolve.cu:159-268);
 * here the same A^{-1}[g, y] is computed either by
 *   CG_DIRSOLVE_DENSE : exact elimination of the larger diagonal block and a
 *                       dense FP64 Cholesky (cuSOLVER potrf) of the Schur
 *                       complement, or
 *   CG_DIRSOLVE_SPARSE: cuSOLVER sparse Cholesky of the full A in an AMD order
 *                       computed on the host on every pattern update;
 *   CG_DIRSOLVE_PEEL  : LDL^T elimination of the nodes outside the graph's
 *                       2-core (degree <= 1, no fill), planned on the host on
 *                       every pattern update, then the dense Schur path on
 *                       the 2-core only;
 *   CG_DIRSOLVE_AUTO  : (default) per pattern, PEEL when the 2-core's Schur
 *                       complement is at most half the dense one, else DENSE.
 * cg_splr_last_direction_solver() returns the path of the last direction
 * solve issued by the calling thread (0 dense, 1 sparse, 2 peel, -1 none).
 */
enum { CG_DIRSOLVE_AUTO = 0, CG_DIRSOLVE_DENSE = 1, CG_DIRSOLVE_SPARSE = 2, CG_DIRSOLVE_PEEL = 3 };
int cg_splr_set_direction_solver(int mode);
int cg_splr_last_direction_solver(void);


/* Context properties (reg, dim, low_rank_enabled, is_fallback, ...;
 * src/solvers_torch.cpp:691-696). */
int cg_ctx_info(const cg_ctx* ctx, cg_ctx_info_t* out);
/* One-time D_A^{-1} extraction, validated (backward_context.cu:616-640). */
int cg_ctx_setup_diag(cg_ctx* ctx, cudaStream_t stream);
/* z = B^{-1} r (mode CG_PRECOND_SPLR: factor solve + rank-2 Woodbury,
 * backward_context.cu:543-581) or z = D_A^{-1} r (CG_PRECOND_DIAG,
 * backward_context.cu:642-655).  r, z: device [dim]. */
int cg_ctx_apply(cg_ctx* ctx, const double* r, double* z, int mode, cudaStream_t stream);
/* Copies a context array (CG_CTX_*) to device memory dst
 * (csr_values/csr_colind/csr_rowptr/secant_s/secant_y/inv_diag/ctx_point,
 * src/solvers_torch.cpp:583-647). */
int cg_ctx_copy(const cg_ctx* ctx, int what, void* dst, cudaStream_t stream);
/* Releases the context (factorization first, then its buffers). */
int cg_ctx_destroy(cg_ctx* ctx);

/*
 * Implicit backward: solves Q(T) lambda = mu with PCG and assembles
 * dL/dM = T * (lambda_a 1^T + 1 lambda_b^T - G) / eta.  Replaces
 * solve_backward / pcg / q_matvec / rhs_Q_scale / assemble_grad
 * (curegot/backward.py:72-144, curegot/_backward_core.py:31-83).
 * precond: CG_PRECOND_NONE | CG_PRECOND_DIAG | CG_PRECOND_SPLR (ctx may be
 * NULL for NONE).  T, G: device n x m; lambda: device [n+m-1]; grad: device
 * n x m.  iterations / converged: host.  A PCG breakdown (p^T A p <= 0)
 * returns CG_ERR_NOT_SPD.
 */
int cg_backward_f64(const double* T, const double* G, cg_ctx* ctx, double eta, int precond,
                    double tol, int max_iter, int n, int m, double* lambda, double* grad,
                    int* iterations, int* converged, cudaStream_t stream);

/*
 * The same backward for B problems of one shape in one call: T, G, grad are
 * [B, n, m] (contiguous), lambda [B, n + m - 1], iterations / converged host
 * [B]; ctxs: B contexts (CG_PRECOND_DIAG) or NULL (CG_PRECOND_NONE; the SPLR
 * preconditioner is not batched).  One launch per PCG iteration covers every
 * unfinished problem and the host reads the B states once per chunk of
 * iterations; each problem's values are those of cg_backward_f64.  Replaces
 * the per-problem backward of splr_ot_batch (curegot/autograd.py:340-367).
 */
int cg_backward_batch_f64(const double* T, const double* G, cg_ctx* const* ctxs, double eta,
                          int precond, double tol, int max_iter, int B, int n, int m,
                          double* lambda, double* grad, int* iterations, int* converged,
                          cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Continuous-batching serving engine (no reference counterpart: the         */
/* reference solves one problem per blocking call and batches only with a    */
/* Python loop, curegot/autograd.py:340-367).                                */
/* ------------------------------------------------------------------------ */

typedef struct cg_engine_s cg_engine;

enum { CG_ALGO_BCD = 0, CG_ALGO_SPLR = 1 };

typedef struct {
  int algo;            /* CG_ALGO_BCD | CG_ALGO_SPLR                                  */
  int n, m;
  int m_f32;           /* 1: M is float (mixed precision), 0: double                 */
  int host_inputs;     /* 1: M, a, b, dual_out are host pointers (copied by the engine) */
  int max_iter;
  double eta, tol;
  const void* M;       /* row-major n x m                                             */
  const double* a;     /* [n] */
  const double* b;     /* [m] */
  double* dual_out;    /* [n + m] (nullable)                                          */
  uint64_t tag;        /* caller's tag, returned with the result                      */
} cg_request_t;

typedef struct {
  uint64_t id, tag;
  int status, niter, converged, fast_iters;
  double last_err;                 /* last stop-test value (Sinkhorn)             */
  double t_submit, t_admit, t_done; /* cg_engine_clock() seconds                  */
} cg_result_t;

typedef struct {
  size_t in_use_bytes, budget_bytes;
  long long queued, active_bcd, active_splr, completed;
  double bcd_bytes;      /* algorithmic bytes streamed by the Sinkhorn passes   */
  double bcd_gpu_ms;     /* device time of the Sinkhorn chunks                  */
  long long chunks, graph_builds;
} cg_engine_stats_t;

/* Starts the engine on the current device: a Sinkhorn batch scheduler and
 * splr_workers SPLR worker threads.  budget_bytes bounds the device memory
 * of admitted requests; max_batch bounds the Sinkhorn batch; chunk = ticks
 * (row + column pass) per captured graph launch. */
int cg_engine_create(size_t budget_bytes, int max_batch, int splr_workers, int chunk,
                     cg_engine** out);
/* Enqueues a request (non-blocking).  Input buffers must stay valid until its
 * result is polled. */
int cg_engine_submit(cg_engine* eng, const cg_request_t* req, uint64_t* id);
/* Moves up to capacity finished results into results (waits up to wait_ms
 * for the first one). */
int cg_engine_poll(cg_engine* eng, cg_result_t* results, int capacity, int wait_ms, int* count);
int cg_engine_stats(cg_engine* eng, cg_engine_stats_t* out);
/* The engine's clock (seconds, monotonic), for latency accounting. */
double cg_engine_clock(void);
/* Cancels a request: a queued one ends at once, an admitted Sinkhorn one at
 * the end of its batch's current chunk, an admitted SPLR one at its next
 * iteration.  Its result (status CG_ERR_CANCELLED, no duals written) is
 * returned by cg_engine_poll like any other.  CG_ERR_INVALID_ARG when the id
 * is unknown or already finished.  No reference counterpart. */
int cg_engine_cancel(cg_engine* eng, uint64_t id);
/* Stops the engine (admitted work finishes; queued requests are dropped). */
int cg_engine_destroy(cg_engine* eng);

/* ------------------------------------------------------------------------ */
/* Test hooks of the reference (curegot.tests, src/tests.cpp:36-200).        */
/* ------------------------------------------------------------------------ */

/* T_t values and flat Hsl indices (i*(m-1)+j -> (n+j)*(n+m-1)+i); the
 * Tvalues / Tflatind outputs of T_computation_sparsify_host. */
int cg_t_values_f64(const double* alpha, const double* beta, const double* M, int n, int m,
                    double reg, double* Tvalues, int* Tflatind, cudaStream_t stream);
/* T pass + objective/gradient + top-K sparsification into CSR
 * (T_computation_sparsify_host, src/sinkhorn_splr_kernel.cu:909-1032).
 * Device arrays; objfn_gnorm: device [2]; k_actual: host. */
int cg_test_t_sparsify_f64(const double* alpha, const double* beta, const double* M,
                           const double* a, const double* b, double reg, double shift, int K,
                           int n, int m, double* rows, double* cols, double* grad,
                           double* objfn_gnorm, double* csr_val, int* csr_colind,
                           int* csr_rowptr, long long* k_actual, cudaStream_t stream);
/* Host-side failure injection for tests (process-wide).  what =
 * CG_INJECT_DIRECTION_SOLVE: the next `count` SPLR direction solves report a
 * failed factorization, as a non-positive pivot would, so the solve returns
 * CG_ERR_NOT_SPD (the reference exits the process on a cuDSS failure,
 * src/linsolve.cu:19-26).  Nothing on the device is altered; count = 0
 * clears it. */
enum { CG_INJECT_DIRECTION_SOLVE = 1 };
int cg_test_inject_failure(int what, int count);

/* SPD solve with a CSR matrix (full or lower storage, lower triangle read)
 * (sparse_cholesky_solve_host, src/linsolve.cu:312-350).  Device arrays. */
int cg_test_spd_solve_f64(const double* values, const int* colind, const int* rowptr, int n,
                          const double* rhs, double* x, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Cost recomputed from point clouds on the tensor cores.                    */
/* ------------------------------------------------------------------------ */
/*
 * No reference counterpart (the reference always takes a materialised M,
 * src/solvers.h:4-9); this is the BF16-input / FP32-compute cost variant of
 * the differentiation configuration.  X (n x d) and Y (m x d) are row-major
 * BF16 device arrays (raw 16-bit patterns), 1 <= d <= 64.  The cost is
 *   M_ij = max(0, s * ((|x_i|^2 + |y_j|^2) - 2 x_i . y_j))       (FP32)
 * with x_i . y_j accumulated in FP32 by tcgen05 MMAs and the squared norms
 * summed in FP32 (s = cost_scale, e.g. 1/d for the mean over features).
 *
 * cg_points_cost_bf16 writes M (n x m FP32, row-major, device).
 * cg_bcd_points_bf16 runs Sinkhorn BCD on that cost without storing it:
 * alpha, beta updates as cg_bcd_f64 (src/sinkhorn_bcd_kernel.cu:35-634),
 * stopping when the row-marginal error ||T 1 - a||_2 of an iterate is below
 * tol (checked for every iterate).  precision CG_POINTS_FP64: FP64
 * exponentials; CG_POINTS_MIXED: SFU exponentials until the estimate is
 * below tol/2, then FP64 passes confirm.  dual: device [n + m] (alpha, beta);
 * niter, fast_iters: host (nullable).
 */
enum { CG_POINTS_FP64 = 0, CG_POINTS_MIXED = 1 };
int cg_points_cost_bf16(const uint16_t* X, const uint16_t* Y, int n, int m, int d,
                        double cost_scale, float* M, cudaStream_t stream);
int cg_bcd_points_bf16(const uint16_t* X, const uint16_t* Y, int n, int m, int d,
                       double cost_scale, const double* a, const double* b, double reg,
                       int max_iter, double tol, int precision, int* niter, double* dual,
                       int* fast_iters, cudaStream_t stream);
/*
 * Normalisers of the cost on the tensor-core tiles, without storing it:
 * *max_out = the largest and *median_out = the lower median (the
 * ceil(nm/2)-th smallest) of c_ij = max(0, |x_i|^2 + |y_j|^2 - 2 x_i . y_j),
 * the FP32 values cg_points_cost_bf16 writes at cost_scale 1.  Three passes
 * recompute the tiles and histogram the FP32 bit patterns digit by digit
 * (12, 12, 8 bits); the maximum comes with the first.  The configurations'
 * "M / max" and "M / median" are cost_scale = 1 / max or 1 / median.
 * Outputs are host doubles (exactly the FP32 values).
 */
int cg_points_cost_stats_bf16(const uint16_t* X, const uint16_t* Y, int n, int m, int d,
                              double* max_out, double* median_out, cudaStream_t stream);
/* Poll limit of the first wait for each tile's tensor-core MMAs in the
 * functions above (process-wide; polls < 0 restores the default of 2^24).
 * When a wait gives up, the kernel waits once more at the full limit for the
 * MMAs to drain, frees its tensor memory and flags the error: the call
 * returns CG_ERR_TIMEOUT and the device stays usable.  polls = 0 makes every
 * first wait give up at once -- the way tests exercise that path without a
 * fault.  No reference counterpart. */
int cg_points_set_wait_limit(long long polls);

/* ------------------------------------------------------------------------ */
/* Diagnostics (no reference counterpart).                                   */
/* ------------------------------------------------------------------------ */

/* Evaluates the library's own base-2 exponentials on x[0..n): mode 0 = the
 * FP64 table-driven exp2 used by FP64 passes, mode 1 = the mixed-precision
 * SFU exp2 used by FP32-M passes (x <= 0 only).  Lets tests bound their
 * error against CUDA's exp2. */
int cg_diag_exp2(const double* x, double* y, int n, int mode, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* CUREGOT_B200_H */
