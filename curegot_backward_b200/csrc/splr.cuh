// SPLR solver internals shared by the driver, the backward context and the
// adjoint (PCG) solver.
#pragma once

#include <atomic>

#include "schur.cuh"
#include "peel.cuh"
#include "spchol.cuh"

struct cg_ctx_s;

namespace cg {

// Small device-side results of the direction step.
struct DirRes {
  double ys, yy, dg_init;
  int low_rank;
  int pad;
};

// Direction-solve choice (process-wide): 0 auto -- per sparsity pattern, leaf
// peeling + core Schur complement when the core Schur complement is at most
// half the dense one, else the dense Schur path; 1 always dense Schur;
// 2 always cuSOLVER sparse Cholesky; 3 always leaf peeling (unless the
// pattern needs more peel rounds than the solver allows).
enum DirSolveMode { kDirAuto = 0, kDirDense = 1, kDirSparse = 2, kDirPeel = 3 };

struct SplrParams {
  double reg, tol;
  int max_iter;
  double density_max, shift_max;
  int cycle, cand_iter, verbose;
  // 0: stop on ||g|| < tol with g over the first n + m - 1 dual entries (the
  // reference's test, sinkhorn_splr.cu:1128-1132); 1: stop on the full
  // marginal error ||(T1 - a, T^T 1 - b)||_2 < tol, which adds the gauge
  // column's error (the serving engine's per-result accuracy guarantee).
  int full_stop = 0;
  // with full_stop: once the reference's test passes, also accept the point
  // whose gauge column m - 1 is made exact (beta_{m-1} moved, then the gauge
  // shifted back) when that gives a full marginal error below tol; the
  // returned duals then carry the correction.  Without a context only.
  int gauge_fix = 0;
  // set by another thread to stop the solve at the next iteration with
  // CG_ERR_CANCELLED (the serving engine's request cancellation); may be null
  const std::atomic<bool>* cancel = nullptr;
};

struct TaskIO;
struct SolveTask;

// The SPLR solve as a resumable task on io->st (task.cuh; splr.cu).
template <typename TM>
SolveTask splr_task(TaskIO* io, const TM* M, const double* a, const double* b, double* Pout,
                    int n, int m, SplrParams prm, const double* x0, double* dual,
                    int* niter_out, int* converged_out, cg_ctx_s** ctx_out, double* trace);

// The SPLR solve (splr.cu), driven to completion on the calling thread.  M is
// float (mixed) or double; everything else FP64.
template <typename TM>
int splr_solve(const TM* M, const double* a, const double* b, double* Pout, int n, int m,
               const SplrParams& prm, const double* x0, double* dual, int* niter_out,
               int* converged_out, cg_ctx_s** ctx_out, double* trace, cudaStream_t st);

}  // namespace cg

// Backward context (opaque to C callers).  Owns the sparsified Hessian A_k of
// the last forward direction solve (CSR + per-row lists), its Schur factor,
// the secant pair and A_k^{-1} y_k -- the state the reference's
// SPLRBackwardContext adopts from the forward solver
// (src/backward_context.h:83-376).
struct cg_ctx_s {
  int device = 0;
  int n = 0, m = 0, H = 0;
  double reg = 0.0, ys = 0.0;
  bool low_rank = false, fallback = false, valid = false, has_point = false;
  bool diag_ready = false;
  long long nnz = 0;
  void* block = nullptr;  // single allocation owning every device buffer below
  cg::SpHess A;
  cg::SchurFactor F;
  cg::SparseChol* sc = nullptr;  // sparse Cholesky factor (owned) when path == 1
  cg::PeelFactor* pf = nullptr;  // leaf-peeling factor (owned) when path == 2
  int path = 0;                  // factor of the last direction solve: 0 F, 1 sc, 2 pf
  double* s = nullptr;
  double* y = nullptr;
  double* u = nullptr;  // A^{-1} y
  double* inv_diag = nullptr;
  double* point = nullptr;
  double* tmp = nullptr;  // [k] solve scratch
  double* xtmp = nullptr; // [H] solve scratch
  cg::DirRes* dres = nullptr;
  int* err = nullptr;
};
