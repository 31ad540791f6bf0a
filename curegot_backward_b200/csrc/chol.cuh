// Warp-level Cholesky of a small diagonal block, used by the in-shared-
// memory factorization of the small peel cores (peel.cu).
#pragma once

#include "common.cuh"

namespace cg {

// Left-looking (Crout) Cholesky of the bw x bw block A (bw <= 32, row-major
// in shared memory with row stride lda, lower triangle) by ONE warp; lane r
// computes row r.  Step k: every lane forms the pivot d = A_kk - sum_c L_kc^2
// from row k (broadcast reads), lane r > k forms L_rk = (A_rk - sum_c L_rc
// L_kc) / L_kk from its own row -- dot products of loads only, so the loads
// pipeline -- and one rsqrt gives both 1 / L_kk and L_kk = d / sqrt(d).
// dinv[k] <- 1 / L_kk.  A pivot that is not positive and finite sets *info =
// col0 + k + 1 and continues with d = 1.
__device__ __forceinline__ void warp_block_cholesky(double* __restrict__ A, int lda, int bw,
                                                    double* __restrict__ dinv, int col0,
                                                    int* __restrict__ info) {
  const int lane = threadIdx.x & 31;
  double* Lr = A + (size_t)min(lane, bw - 1) * lda;  // this lane's row
  for (int k = 0; k < bw; ++k) {
    const double* Lk = A + (size_t)k * lda;
    double p0 = Lk[k], p1 = 0.0;
    double a0 = Lr[k], a1 = 0.0;
    int c = 0;
    // unrolled by 4 (8 columns per trip): the loads of a trip issue back to
    // back; this cut the per-block cycles by about a third on B200, while
    // the fully unrolled form spills under the 64-register cap of a
    // 1024-thread block and was slower
#pragma unroll 4
    for (; c + 1 < k; c += 2) {
      const double x0 = Lk[c], x1 = Lk[c + 1];
      p0 = fma(-x0, x0, p0);
      p1 = fma(-x1, x1, p1);
      a0 = fma(-Lr[c], x0, a0);
      a1 = fma(-Lr[c + 1], x1, a1);
    }
    if (c < k) {
      const double x0 = Lk[c];
      p0 = fma(-x0, x0, p0);
      a0 = fma(-Lr[c], x0, a0);
    }
    double d = p0 + p1;
    if (!(d > 0.0) || !isfinite(d)) {
      if (lane == 0) *info = col0 + k + 1;
      d = 1.0;
    }
    const double inv = rsqrt(d);
    __syncwarp();  // every lane has read A_kk and its own A_rk
    if (lane > k && lane < bw) Lr[k] = (a0 + a1) * inv;
    if (lane == k) {
      Lr[k] = d * inv;
      dinv[k] = inv;
    }
    __syncwarp();
  }
}

}  // namespace cg
