// Dense FP64 Cholesky factor and solve of mid-size SPD matrices (the Schur
// complements of the SPLR direction solve), replacing cuSOLVER potrf/potrs
// there.  At k of a few hundred those calls are latency-bound chains of
// small kernels (hundreds of microseconds per factor-solve).
//
// Storage: the cuSOLVER convention -- column-major k x k, lower triangle
// (element (i, j) at S[j * k + i], i >= j), so the factor is interchangeable
// with potrf's.
//
// Factor: ONE cluster of kDnCtas CTAs, right-looking by panels of 32
// columns, two cluster barriers per panel:
//   B. the panel below the diagonal block, L21 = S21 L11^{-T}: one thread per
//      row, the row's 32 entries in registers, solved left-looking against
//      L11 (shared memory), rows spread over every thread of the cluster;
//   C. the trailing update S22 -= L21 L21^T (lower triangle) by 32 x 32 tiles
//      spread over the CTAs, every CTA holding the whole L21 panel in shared
//      memory; rank 0 computes tile (0, 0) -- the next diagonal block -- and
//      factors it at once (one warp, warp_block_cholesky), so the diagonal
//      factorization needs no barrier of its own.
// k <= kDenseMaxK keeps a whole panel in shared memory.
//
// Solve (nrhs <= 2 columns, in place): one 1024-thread CTA, blocks of 32:
// the 32 x 32 diagonal block is solved by one warp in shared memory, the
// other blocks' contributions are column sweeps (forward) or dot products
// along columns (backward) spread over the CTA.
//
// A pivot that is not positive and finite sets info = column + 1 and the
// factorization continues with pivot 1 (the caller reads info != 0 as "not
// SPD"; potrf reports the first such column, this the last).
#include <algorithm>

#include <cooperative_groups.h>

#include "chol.cuh"
#include "dense.cuh"

namespace cg {

namespace {

namespace cgx = cooperative_groups;

constexpr int kDnCtas = 8;      // cluster size (portable)
constexpr int kDnThreads = 256;
constexpr int kNB = 32;
constexpr int kLd = kNB + 1;    // shared row stride of 32-wide blocks

__global__ void __cluster_dims__(kDnCtas, 1, 1) __launch_bounds__(kDnThreads)
    dense_chol_kernel(double* __restrict__ S, int k, double* __restrict__ dinv,
                      int* __restrict__ info) {
  extern __shared__ double dsm[];
  __shared__ double A[kNB][kLd];   // diagonal block / L11
  __shared__ double dv[kNB];       // 1 / L_jj of the panel
  double* P = dsm;                 // L21 panel: row r at P[r * kLd]
  cgx::cluster_group cl = cgx::this_cluster();
  const int rank = (int)cl.block_rank();
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto at = [&](int i, int j) -> double& { return S[(size_t)j * k + i]; };

  if (rank == 0) {
    if (tid == 0) *info = 0;
    const int bw = min(kNB, k);
    for (int e = tid; e < bw * bw; e += blockDim.x) {
      const int r = e % bw, c = e / bw;
      A[r][c] = at(r, c);
    }
    __syncthreads();
    if (warp == 0) warp_block_cholesky(&A[0][0], kLd, bw, dinv, 0, info);
    __syncthreads();
    for (int e = tid; e < bw * bw; e += blockDim.x) {
      const int r = e % bw, c = e / bw;
      if (c <= r) at(r, c) = A[r][c];
    }
  }
  cl.sync();

  for (int j0 = 0; j0 < k; j0 += kNB) {
    const int bw = min(kNB, k - j0);
    const int r0 = j0 + bw, w = k - r0;
    if (w <= 0) break;
    // ---- B: L21 rows, one thread per row ----------------------------------
    for (int e = tid; e < bw * bw; e += blockDim.x) {
      const int r = e % bw, c = e / bw;
      A[r][c] = (c <= r) ? at(j0 + r, j0 + c) : 0.0;
    }
    if (tid < bw) dv[tid] = dinv[j0 + tid];
    __syncthreads();
    for (int i = r0 + rank * kDnThreads + tid; i < k; i += kDnCtas * kDnThreads) {
      double x[kNB];
#pragma unroll
      for (int c = 0; c < kNB; ++c) x[c] = (c < bw) ? at(i, j0 + c) : 0.0;
#pragma unroll
      for (int kk = 0; kk < kNB; ++kk) {
        if (kk < bw) {
          double a0 = x[kk], a1 = 0.0;
#pragma unroll
          for (int c = 0; c < kk; c += 2) {
            a0 = fma(-x[c], A[kk][c], a0);
            if (c + 1 < kk) a1 = fma(-x[c + 1], A[kk][c + 1], a1);
          }
          x[kk] = (a0 + a1) * dv[kk];
        }
      }
#pragma unroll
      for (int c = 0; c < kNB; ++c)
        if (c < bw) at(i, j0 + c) = x[c];
    }
    cl.sync();
    // ---- C: trailing update; rank 0 also factors the next diagonal block ---
    for (int e = tid; e < w * bw; e += blockDim.x) {
      const int r = e % w, c = e / w;
      P[(size_t)r * kLd + c] = at(r0 + r, j0 + c);
    }
    __syncthreads();
    const int nt = (w + kNB - 1) / kNB;
    const int ntiles = nt * (nt + 1) / 2;
    for (int t = rank; t < ntiles; t += kDnCtas) {
      int ti = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
      while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
      while (ti * (ti + 1) / 2 > t) --ti;
      const int tc = t - ti * (ti + 1) / 2;
      const int ib = ti * kNB, cb = tc * kNB;  // offsets from r0
      const int i = ib + lane;                 // this thread's row
      const int c0 = cb + warp * 4;            // its four columns
      double acc[4] = {0.0, 0.0, 0.0, 0.0};
      if (i < w) {
        for (int kk = 0; kk < bw; ++kk) {
          const double a = P[(size_t)i * kLd + kk];
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (c0 + q < w) acc[q] = fma(a, P[(size_t)(c0 + q) * kLd + kk], acc[q]);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (c0 + q < w && c0 + q <= i) at(r0 + i, r0 + c0 + q) -= acc[q];
      }
      if (t == 0) {
        // tile (0, 0) is the next diagonal block: factor it now
        __syncthreads();
        const int bn = min(kNB, w);
        for (int e = tid; e < bn * bn; e += blockDim.x) {
          const int r = e % bn, c = e / bn;
          A[r][c] = at(r0 + r, r0 + c);
        }
        __syncthreads();
        if (warp == 0) warp_block_cholesky(&A[0][0], kLd, bn, dinv + r0, r0, info);
        __syncthreads();
        for (int e = tid; e < bn * bn; e += blockDim.x) {
          const int r = e % bn, c = e / bn;
          if (c <= r) at(r0 + r, r0 + c) = A[r][c];
        }
      }
    }
    cl.sync();
  }
}

// In-place solve S S^T X = B for nrhs <= 2 columns of B (ldb = k).
__global__ void __launch_bounds__(1024) dense_solve_kernel(const double* __restrict__ S, int k,
                                                           const double* __restrict__ dinv,
                                                           double* __restrict__ B, int nrhs) {
  __shared__ double D[kNB][kLd];
  __shared__ double zb[2][kNB];
  __shared__ double part[2][kNB];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  auto at = [&](int i, int j) -> double { return S[(size_t)j * k + i]; };
  // forward: L y = b
  for (int j0 = 0; j0 < k; j0 += kNB) {
    const int bw = min(kNB, k - j0);
    for (int e = tid; e < bw * bw; e += blockDim.x) {
      const int r = e % bw, c = e / bw;
      D[r][c] = (c <= r) ? at(j0 + r, j0 + c) : 0.0;
    }
    __syncthreads();
    if (warp < nrhs) {
      double* b = B + (size_t)warp * k;
      double zr = (lane < bw) ? b[j0 + lane] : 0.0;
      for (int jj = 0; jj < bw; ++jj) {
        const double zj = __shfl_sync(0xffffffffu, zr, jj) * dinv[j0 + jj];
        if (lane == jj) zr = zj;
        if (lane > jj && lane < bw) zr = fma(-D[lane][jj], zj, zr);
      }
      if (lane < bw) {
        b[j0 + lane] = zr;
        zb[warp][lane] = zr;
      }
    }
    __syncthreads();
    for (int i = j0 + bw + tid; i < k; i += blockDim.x) {
      double a0 = 0.0, a1 = 0.0;
      for (int c = 0; c < bw; ++c) {
        const double l = at(i, j0 + c);
        a0 = fma(l, zb[0][c], a0);
        if (nrhs > 1) a1 = fma(l, zb[1][c], a1);
      }
      B[i] -= a0;
      if (nrhs > 1) B[(size_t)k + i] -= a1;
    }
    __syncthreads();
  }
  // backward: L^T x = y, blocks from the bottom
  for (int j1 = k; j1 > 0; j1 -= kNB) {
    const int j0 = max(0, j1 - kNB), bw = j1 - j0;
    // contributions of the solved rows i >= j1 to column j0 + c: warp w
    // takes columns c = w (32 warps, 32 columns), lanes stride the rows
    {
      const int c = warp;
      double a0 = 0.0, a1 = 0.0;
      if (c < bw) {
        for (int i = j1 + lane; i < k; i += 32) {
          const double l = at(i, j0 + c);
          a0 = fma(l, B[i], a0);
          if (nrhs > 1) a1 = fma(l, B[(size_t)k + i], a1);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
      }
      if (lane == 0 && c < bw) {
        part[0][c] = a0;
        part[1][c] = a1;
      }
    }
    for (int e = tid; e < bw * bw; e += blockDim.x) {
      const int r = e % bw, c = e / bw;
      D[r][c] = (c <= r) ? at(j0 + r, j0 + c) : 0.0;
    }
    __syncthreads();
    if (warp < nrhs) {
      double* b = B + (size_t)warp * k;
      double zr = (lane < bw) ? b[j0 + lane] - part[warp][lane] : 0.0;
      for (int jj = bw - 1; jj >= 0; --jj) {
        const double zj = __shfl_sync(0xffffffffu, zr, jj) * dinv[j0 + jj];
        if (lane == jj) zr = zj;
        if (lane < jj) zr = fma(-D[jj][lane], zj, zr);
      }
      if (lane < bw) b[j0 + lane] = zr;
    }
    __syncthreads();
  }
}

size_t dense_smem(int k) {
  const int w = std::max(k - kNB, 1);
  return (size_t)w * kLd * sizeof(double);
}

}  // namespace

bool dense_chol_fits(int k) { return k > 0 && k <= kDenseMaxK; }

int dense_chol_factor(double* S, int k, double* dinv, int* info, cudaStream_t st) {
  if (!dense_chol_fits(k)) return CG_ERR_INVALID_ARG;
  static const int ok = [] {
    return cudaFuncSetAttribute(dense_chol_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dense_smem(kDenseMaxK)) == cudaSuccess;
  }();
  if (!ok) {
    set_last_error("dense_chol: shared-memory attribute refused", __FILE__, __LINE__);
    return CG_ERR_CUDA;
  }
  { dense_chol_kernel<<<kDnCtas, kDnThreads, dense_smem(k), st>>>(S, k, dinv, info); count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

int dense_chol_solve(const double* S, int k, const double* dinv, double* B, int nrhs,
                     cudaStream_t st) {
  if (!dense_chol_fits(k) || nrhs < 1 || nrhs > 2) return CG_ERR_INVALID_ARG;
  { dense_solve_kernel<<<1, 1024, 0, st>>>(S, k, dinv, B, nrhs); count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // namespace cg
