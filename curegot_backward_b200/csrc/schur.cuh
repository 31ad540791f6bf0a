// Direction solve with the sparsified Hessian: block elimination of the larger
// diagonal block, dense FP64 Cholesky (cuSOLVER) of the Schur complement.
#pragma once

#include <cusolverDn.h>

#include "sparsify.cuh"

namespace cg {

struct SchurFactor {
  int n = 0, m = 0, H = 0;
  int k = 0;               // Schur dimension: m-1 (alpha block eliminated) or n
  bool big_alpha = true;   // eliminate the alpha block (n >= m-1)
  double* S = nullptr;     // [k*k] factor (in place)
  int* info = nullptr;     // [1] potrf info (device)
  int* solve_info = nullptr;  // [1] potrs info (kept apart so potrf's survives)
  double* work = nullptr;  // potrf workspace
  int lwork = 0;
};

// Schur dimension and potrf workspace size (doubles) for an (n, m) problem.
void schur_dims(int n, int m, int& k, bool& big_alpha);
int schur_lwork(cusolverDnHandle_t h, int k, int& lwork);

// cuSOLVER handle for the calling thread and current device (created once).
int solver_handle(cusolverDnHandle_t* out);

// Assemble S from the CSR / per-row lists of A and factor it (async; the
// potrf status lands in F.info).
// assembled = true: F.S already holds the Schur complement (factor only).
int schur_factor(cusolverDnHandle_t h, const SpHess& A, SchurFactor& F, cudaStream_t st,
                 bool assembled = false);

// x = A^{-1} rhs for nrhs column-major right-hand sides (leading dim H).
// tmp: [k * nrhs] scratch.
int schur_solve(cusolverDnHandle_t h, const SpHess& A, const SchurFactor& F, const double* rhs,
                double* x, int nrhs, double* tmp, cudaStream_t st);

}  // namespace cg
