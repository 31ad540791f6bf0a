// Exact direction solve A x = b for the SPLR sparsified Hessian.
//
// Replaces the cuDSS sparse Cholesky of the reference (benben-cd/curegot_backward
// src/linsolve.cu:159-268, called from compute_search_direc,
// src/sinkhorn_splr.cu:538-649).  cuDSS is not available in this image, so
// the structure of A is used instead: with the reference's Hsl layout
//     A = [ D1   B^T ]      D1 = diag(r) + shift   (n x n)
//         [ B    D2  ]      D2 = diag(c_t) + shift ((m-1) x (m-1)),
// one diagonal block is purely diagonal.  The larger one is eliminated
// exactly and the Schur complement (size min(n, m-1)) is factored densely:
//     S = D2 - B D1^{-1} B^T   (n >= m-1)   or   S = D1 - B^T D2^{-1} B.
// S is assembled deterministically (one CTA per row of S, contributions in
// CSR order, distinct targets per step) and factored with cuSOLVER potrf in
// FP64; the solves are potrs plus two sparse sweeps.  The result is the same
// linear-algebra object the reference computes (A^{-1} b), to rounding.
#include <mutex>
#include <unordered_map>

#include "schur.cuh"

namespace cg {

void schur_dims(int n, int m, int& k, bool& big_alpha) {
  big_alpha = (n >= m - 1);
  k = big_alpha ? (m - 1) : n;
}

int schur_lwork(cusolverDnHandle_t h, int k, int& lwork) {
  lwork = 0;
  if (k <= 0) return CG_OK;
  if (cusolverDnDpotrf_bufferSize(h, CUBLAS_FILL_MODE_LOWER, k, nullptr, k, &lwork) !=
      CUSOLVER_STATUS_SUCCESS) {
    set_last_error("cusolverDnDpotrf_bufferSize failed", __FILE__, __LINE__);
    return CG_ERR_SOLVER;
  }
  return CG_OK;
}

int solver_handle(cusolverDnHandle_t* out) {
  thread_local std::unordered_map<int, cusolverDnHandle_t> handles;
  int dev = 0;
  CG_TRY_CUDA(cudaGetDevice(&dev));
  auto it = handles.find(dev);
  if (it == handles.end()) {
    cusolverDnHandle_t h = nullptr;
    if (cusolverDnCreate(&h) != CUSOLVER_STATUS_SUCCESS) {
      set_last_error("cusolverDnCreate failed", __FILE__, __LINE__);
      return CG_ERR_SOLVER;
    }
    it = handles.emplace(dev, h).first;
  }
  *out = it->second;
  return CG_OK;
}

namespace {

// Row j of S (alpha block eliminated): D2_j e_j - sum_{i in row n+j} (T_ij / D1_i) T_i,:
__global__ void assemble_big_alpha(const double* __restrict__ val, const int* __restrict__ col,
                                   const int* __restrict__ rowptr, const int* __restrict__ ipt,
                                   const int* __restrict__ ij, const double* __restrict__ iv,
                                   int n, int k, double* __restrict__ S) {
  const int j = blockIdx.x;
  double* __restrict__ Sr = S + (size_t)j * k;
  const int r = n + j;
  for (int c = threadIdx.x; c < k; c += blockDim.x) Sr[c] = 0.0;
  __syncthreads();
  if (threadIdx.x == 0) Sr[j] = val[rowptr[r + 1] - 1];
  __syncthreads();
  for (int q = rowptr[r]; q < rowptr[r + 1] - 1; ++q) {
    const int i = col[q];
    const double w = val[q] / val[i];  // row i < n holds only its diagonal, at position i
    for (int p = ipt[i] + threadIdx.x; p < ipt[i + 1]; p += blockDim.x) Sr[ij[p]] -= w * iv[p];
    __syncthreads();
  }
}

// Row i of S (beta block eliminated): D1_i e_i - sum_{j in list i} (T_ij / D2_j) T_:,j
__global__ void assemble_big_beta(const double* __restrict__ val, const int* __restrict__ col,
                                  const int* __restrict__ rowptr, const int* __restrict__ ipt,
                                  const int* __restrict__ ij, const double* __restrict__ iv,
                                  int n, int k, double* __restrict__ S) {
  const int i = blockIdx.x;
  double* __restrict__ Sr = S + (size_t)i * k;
  for (int c = threadIdx.x; c < k; c += blockDim.x) Sr[c] = 0.0;
  __syncthreads();
  if (threadIdx.x == 0) Sr[i] = val[i];
  __syncthreads();
  for (int p = ipt[i]; p < ipt[i + 1]; ++p) {
    const int j = ij[p];
    const int r = n + j;
    const double w = iv[p] / val[rowptr[r + 1] - 1];
    for (int q = rowptr[r] + threadIdx.x; q < rowptr[r + 1] - 1; q += blockDim.x)
      Sr[col[q]] -= w * val[q];
    __syncthreads();
  }
}

// Warp-per-row sparse sweeps (fixed-order lane partials + shfl_down tree).
// mode 0 (big alpha):  rs_j = b_{n+j} - sum_{q in row n+j} (v_q / D1_{i_q}) b_{i_q}
// mode 1 (big beta):   rs_i = b_i - sum_{p in list i} (v_p / D2_{j_p}) b_{n+j_p}
__global__ void reduce_rhs_kernel(int mode, const double* __restrict__ val,
                                  const int* __restrict__ col, const int* __restrict__ rowptr,
                                  const int* __restrict__ ipt, const int* __restrict__ ij,
                                  const double* __restrict__ iv, int n, int H, int k,
                                  const double* __restrict__ rhs, int nrhs,
                                  double* __restrict__ rs) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int t = blockIdx.x * (blockDim.x >> 5) + warp; t < k; t += gridDim.x * (blockDim.x >> 5)) {
    for (int c = 0; c < nrhs; ++c) {
      const double* b = rhs + (size_t)c * H;
      double acc = 0.0;
      double self;
      if (mode == 0) {
        const int r = n + t;
        self = b[r];
        for (int q = rowptr[r] + lane; q < rowptr[r + 1] - 1; q += 32) {
          const int i = col[q];
          acc += val[q] / val[i] * b[i];
        }
      } else {
        self = b[t];
        for (int p = ipt[t] + lane; p < ipt[t + 1]; p += 32) {
          const int j = ij[p];
          acc += iv[p] / val[rowptr[n + j + 1] - 1] * b[n + j];
        }
      }
      acc = warp_sum_down(acc);
      if (lane == 0) rs[(size_t)c * k + t] = self - acc;
    }
  }
}

// Back substitution of the eliminated block and scatter of the Schur part.
// mode 0: x_i = (b_i - sum_{p in list i} v_p xs_{j_p}) / D1_i ; x_{n+j} = xs_j
// mode 1: x_{n+j} = (b_{n+j} - sum_{q in row n+j} v_q xs_{i_q}) / D2_j ; x_i = xs_i
__global__ void back_kernel(int mode, const double* __restrict__ val, const int* __restrict__ col,
                            const int* __restrict__ rowptr, const int* __restrict__ ipt,
                            const int* __restrict__ ij, const double* __restrict__ iv, int n,
                            int m, int H, int k, const double* __restrict__ rhs,
                            const double* __restrict__ xs, int nrhs, double* __restrict__ x) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int big = (mode == 0) ? n : (m - 1);
  for (int t = blockIdx.x * (blockDim.x >> 5) + warp; t < big; t += gridDim.x * (blockDim.x >> 5)) {
    for (int c = 0; c < nrhs; ++c) {
      const double* b = rhs + (size_t)c * H;
      const double* s = xs + (size_t)c * k;
      double* xo = x + (size_t)c * H;
      double acc = 0.0;
      if (mode == 0) {
        for (int p = ipt[t] + lane; p < ipt[t + 1]; p += 32) acc += iv[p] * s[ij[p]];
      } else {
        const int r = n + t;
        for (int q = rowptr[r] + lane; q < rowptr[r + 1] - 1; q += 32) acc += val[q] * s[col[q]];
      }
      acc = warp_sum_down(acc);
      if (lane == 0) {
        if (mode == 0) xo[t] = (b[t] - acc) / val[t];
        else xo[n + t] = (b[n + t] - acc) / val[rowptr[n + t + 1] - 1];
      }
    }
  }
  // scatter the Schur-block solution
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < k * nrhs; q += gridDim.x * blockDim.x) {
    const int c = q / k, t = q - c * k;
    x[(size_t)c * H + (mode == 0 ? n + t : t)] = xs[(size_t)c * k + t];
  }
}

}  // namespace

int schur_factor(cusolverDnHandle_t h, const SpHess& A, SchurFactor& F, cudaStream_t st,
                 bool assembled) {
  if (F.k <= 0) return CG_OK;
  if (assembled) {
    // S assembled by the caller
  } else if (F.big_alpha)
    { assemble_big_alpha<<<F.k, 256, 0, st>>>(A.val, A.col, A.rowptr, A.ipt, A.ij, A.iv, A.n, F.k,
                                            F.S); cg::count_launch(); }
  else
    { assemble_big_beta<<<F.k, 256, 0, st>>>(A.val, A.col, A.rowptr, A.ipt, A.ij, A.iv, A.n, F.k,
                                           F.S); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  if (cusolverDnSetStream(h, st) != CUSOLVER_STATUS_SUCCESS) return CG_ERR_SOLVER;
  if (cusolverDnDpotrf(h, CUBLAS_FILL_MODE_LOWER, F.k, F.S, F.k, F.work, F.lwork, F.info) !=
      CUSOLVER_STATUS_SUCCESS) {
    set_last_error("cusolverDnDpotrf failed to launch", __FILE__, __LINE__);
    return CG_ERR_SOLVER;
  }
  return CG_OK;
}

int schur_solve(cusolverDnHandle_t h, const SpHess& A, const SchurFactor& F, const double* rhs,
                double* x, int nrhs, double* tmp, cudaStream_t st) {
  const int mode = F.big_alpha ? 0 : 1;
  const int k = F.k;
  if (k > 0) {
    { reduce_rhs_kernel<<<std::max(1, std::min((k + 7) / 8, 148 * 8)), 256, 0, st>>>(
        mode, A.val, A.col, A.rowptr, A.ipt, A.ij, A.iv, A.n, A.H, k, rhs, nrhs, tmp); cg::count_launch(); }
    CG_TRY_CUDA(cudaGetLastError());
    if (cusolverDnSetStream(h, st) != CUSOLVER_STATUS_SUCCESS) return CG_ERR_SOLVER;
    if (cusolverDnDpotrs(h, CUBLAS_FILL_MODE_LOWER, k, nrhs, F.S, k, tmp, k, F.solve_info) !=
        CUSOLVER_STATUS_SUCCESS) {
      set_last_error("cusolverDnDpotrs failed to launch", __FILE__, __LINE__);
      return CG_ERR_SOLVER;
    }
  }
  const int big = F.big_alpha ? A.n : (A.m - 1);
  const int work = std::max(big, k * nrhs);
  { back_kernel<<<std::max(1, std::min((work + 7) / 8, 148 * 8)), 256, 0, st>>>(
      mode, A.val, A.col, A.rowptr, A.ipt, A.ij, A.iv, A.n, A.m, A.H, k, rhs, tmp, nrhs, x); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // namespace cg
