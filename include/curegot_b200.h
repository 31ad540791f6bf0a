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
  CG_ERR_ADMISSION = 9         /* request does not fit the engine budget     */
};

/* Human-readable text of the last error raised on the calling thread. */
const char* cg_last_error(void);
/* Library version string. */
const char* cg_version(void);

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
