// Sparse Cholesky direction solve: cuSOLVER's sparse Cholesky of the full
// symmetric A = Hsl + shift I, in a fill-reducing order computed on the host
// whenever the sparsity pattern changes.
#pragma once

#include <cusolverSp.h>
#include <cusolverSp_LOWLEVEL_PREVIEW.h>
#include <cusparse.h>

#include <vector>

#include "sparsify.cuh"

namespace cg {

struct SparseChol {
  int H = 0;
  long long nnz = 0;           // entries of the permuted full pattern
  double flops = 0.0;          // sum over columns of L of count^2 (inf: above the budget)
  long long nnz_L = 0;         // entries of L below the diagonal (when counted)
  // host copy of the permuted pattern (pattern phase -> device upload)
  std::vector<int> h_rowptr, h_col, h_map, h_perm;
  csrcholInfo_t info = nullptr;
  void* dblock = nullptr;      // rowptr / col / map / perm / values / rhs scratch
  size_t dblock_bytes = 0;
  int* d_rowptr = nullptr;
  int* d_col = nullptr;
  int* d_map = nullptr;        // permuted entry -> index into the lower CSR values
  int* d_perm = nullptr;       // new index -> original index
  double* d_val = nullptr;
  double* d_b = nullptr;       // [H] permuted rhs
  double* d_x = nullptr;       // [H] permuted solution
  void* buffer = nullptr;
  size_t buffer_bytes = 0;
  bool analyzed = false;
  // allocate/free with cudaMallocAsync/cudaFreeAsync on this stream (a solve-owned
  // factor); plain cudaMalloc when a backward context may outlive the stream
  bool stream_ordered = false;
  cudaStream_t alloc_stream = nullptr;
};

// Pattern phase, host part: copy A's pattern to the host, order it (AMD) and
// count the factor (nnz(L), flops), stopping early once flops exceed
// flop_budget (then C.flops = +inf).  Synchronizes the stream.
int spchol_order(SparseChol& C, const SpHess& A, double flop_budget, cudaStream_t st);
// Pattern phase, device part: upload the permuted pattern, symbolic analysis.
int spchol_analyze(SparseChol& C, cudaStream_t st);
// Numeric phase: current values of A into the permuted pattern, factor.
// *zero_pivot (host) receives the first non-positive pivot or -1.
int spchol_factor(SparseChol& C, const SpHess& A, cudaStream_t st, int* zero_pivot);
// x = A^{-1} rhs for nrhs column-major right-hand sides (leading dim H).
int spchol_solve(SparseChol& C, const double* rhs, double* x, int nrhs, cudaStream_t st);
void spchol_release(SparseChol& C);

}  // namespace cg
