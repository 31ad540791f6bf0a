// Dense FP64 Cholesky factor / solve for mid-size SPD matrices (dense.cu).
#pragma once

#include "common.cuh"

namespace cg {

// Largest k the cluster factorization takes (a 32-column panel of k - 32
// rows stays in one CTA's shared memory).
constexpr int kDenseMaxK = 768;

bool dense_chol_fits(int k);

// In-place lower Cholesky of the column-major k x k matrix S (cuSOLVER potrf
// layout, lower triangle); dinv[j] <- 1 / L_jj; *info <- 0, or column + 1 of
// a pivot that was not positive and finite.  One cluster launch on st.
int dense_chol_factor(double* S, int k, double* dinv, int* info, cudaStream_t st);

// In-place solve (L L^T) X = B for nrhs <= 2 columns of B (ldb = k) with the
// factor of dense_chol_factor.
int dense_chol_solve(const double* S, int k, const double* dinv, double* B, int nrhs,
                     cudaStream_t st);

}  // namespace cg
