// Leaf-peeling LDL^T + 2-core Schur complement direction solve.
//
// Host (on every sparsity-pattern update, every `cycle` SPLR iterations):
//   the pattern of A's lower CSR (the reference Hsl layout: row i < n holds
//   only its diagonal; row n + j holds the alpha columns of beta node j in
//   ascending order, then its diagonal) is copied to the host and peeled:
//   round after round, every alive node of degree <= 1 whose single
//   neighbour is not itself eliminated in the same round is eliminated.
//   Each eliminated node remembers its parent (the neighbour still alive)
//   and each node the list of its eliminated children.  The nodes never
//   eliminated form the 2-core; its larger side is eliminated exactly and
//   the smaller side carries the dense Schur complement.
// Device (every iteration): one CTA computes the pivots round by round (a
//   node's pivot pulls its children's contributions in a fixed order, so
//   the result is deterministic), one CTA per Schur row assembles the core
//   Schur complement, cuSOLVER potrf factors it.  The solve is a forward
//   sweep over the rounds with the core's triangular solves in the same
//   single-CTA kernel (potrs above kPeelTriMax), and a backward sweep.
// Small cores (kc <= kPeelSmallCore = 160, 204 KB of shared memory for the
//   dense core factor): the whole factorization and solve run in
//   ONE single-CTA kernel -- pivots and forward values in the same rounds,
//   the core Schur complement assembled and Cholesky-factored in shared
//   memory, the triangular solves and the backward sweep -- instead of ~6
//   launches with cuSOLVER calls that cost tens of microseconds each at
//   these sizes.  The factor L is also written out for later solves
//   (backward-context applies).
#include <algorithm>
#include <cmath>

#include "chol.cuh"
#include "peel.cuh"

namespace cg {

namespace {

constexpr int kMaxPeelRounds = 512;
#ifndef CG_PEEL_THREADS
#define CG_PEEL_THREADS 1024
#endif
constexpr int kPeelThreads = CG_PEEL_THREADS;  // threads of the single-CTA peel kernels
#ifndef CG_PEEL_MINB
#define CG_PEEL_MINB 1
#endif
constexpr int kPeelMinBlocks = CG_PEEL_MINB;  // launch-bounds residency hint
constexpr int kSmallCore = kPeelSmallCore;  // in-shared-memory Cholesky

struct PeelPtrs {
  // order: nodes round by round; per order position k: cpos[k]..cpos[k+1]
  // its children (child node, value index of the edge), dqo[k] the value
  // index of its diagonal, ppar[k] / pparq[k] its parent and the edge's
  // value index (-1: none).  diagq: diagonal value index by node id.
  const int *order, *rptr, *hcnt, *diagq, *cpos, *child, *childq, *dqo, *ppar, *pparq;
  const int *snodes, *enodes, *sptr, *sadj, *sq, *eptr, *eadj, *eq;
  // contribution lists of the core Schur complement (entry t * kc + t2):
  // eliminated node ce, E-list position cw of the edge (ce, t) (its weight
  // W[cw] = a / d_ce), value index cq2 of the edge (ce, t2)
  const int *ccp, *ce, *cw, *cq2;
};

constexpr int kContribMax = kPeelContribMax;

PeelPtrs ptrs_of(const PeelFactor& P) {
  const int* b = P.ints;
  PeelPtrs p;
  p.order = b + P.off_order;
  p.rptr = b + P.off_rptr;
  p.hcnt = b + P.off_hcnt;
  p.diagq = b + P.off_diagq;
  p.cpos = b + P.off_cpos;
  p.child = b + P.off_child;
  p.childq = b + P.off_childq;
  p.dqo = b + P.off_dqo;
  p.ppar = b + P.off_ppar;
  p.pparq = b + P.off_pparq;
  p.snodes = b + P.off_snodes;
  p.enodes = b + P.off_enodes;
  p.sptr = b + P.off_sptr;
  p.sadj = b + P.off_sadj;
  p.sq = b + P.off_sq;
  p.eptr = b + P.off_eptr;
  p.eadj = b + P.off_eadj;
  p.eq = b + P.off_eq;
  p.ccp = P.contrib ? b + P.off_ccp : nullptr;
  p.ce = P.contrib ? b + P.off_ce : nullptr;
  p.cw = P.contrib ? b + P.off_cq1 : nullptr;
  p.cq2 = P.contrib ? b + P.off_cq2 : nullptr;
  return p;
}

// Threads per node for a block-wide step over cnt nodes: the largest power
// of two g <= 32 with cnt * g <= blockDim.x (1 once the nodes fill the
// block).  A node's list (children, S-list, E-list) is then split over its g
// lanes -- lane `sub` takes entries sub, sub + g, ... -- and the partial
// sums meet in a shuffle tree, so a round with few nodes but long lists
// (the core round: beta nodes holding dozens of peeled alpha leaves) does
// not wait on one thread walking a list serially.  g depends only on cnt,
// so the summation order is fixed for a given plan.
__device__ __forceinline__ int group_width(int cnt) {
  int g = 1;
  while (g < 32 && cnt * (g * 2) <= (int)blockDim.x) g *= 2;
  return g;
}

// Sum over the g lanes of a group (g a power of two <= 32; every lane of the
// warp calls it).
__device__ __forceinline__ double group_sum(double v, int g) {
  for (int o = g >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Pivot (with_d) and forward values y = L^{-1} rhs (nrhs columns, stride H)
// of node v at order position k (k < 0: none), its child list split over
// the g lanes of a group (this lane is `sub`; every lane of the warp calls
// it).  The child range and the diagonal index are read by position, in
// parallel with order[k], not after it.  Node v's pivot is
//   d_v = A_vv - sum over children ch of (a_ch,v / d_ch) a_ch,v
// and its forward value y_v = rhs_v - sum (a_ch,v / d_ch) y_ch.
// nrhs <= 2 is handled in one pass over the children.
__device__ __forceinline__ void node_step(const double* __restrict__ val, const PeelPtrs& p,
                                          int k, int sub, int g, bool with_d,
                                          double* __restrict__ d, const double* __restrict__ rhs,
                                          int nrhs, int H, double* __restrict__ y,
                                          int* __restrict__ info) {
  const int v = k >= 0 ? p.order[k] : -1;
  const int q0 = k >= 0 ? p.cpos[k] : 0, q1 = k >= 0 ? p.cpos[k + 1] : 0;
  if (nrhs <= 2) {
    double sd = 0.0, s0 = 0.0, s1 = 0.0;
    for (int q = q0 + sub; q < q1; q += g) {
      const int ch = p.child[q];
      const double a = val[p.childq[q]];
      const double w = a / d[ch];
      sd = fma(w, a, sd);
      if (nrhs > 0) s0 = fma(w, y[ch], s0);
      if (nrhs > 1) s1 = fma(w, y[(size_t)H + ch], s1);
    }
    if (with_d) sd = group_sum(sd, g);
    if (nrhs > 0) s0 = group_sum(s0, g);
    if (nrhs > 1) s1 = group_sum(s1, g);
    if (v >= 0 && sub == 0) {
      if (with_d) {
        const double dv = val[p.dqo[k]] - sd;
        d[v] = dv;
        if (!(dv > 0.0) || !isfinite(dv)) info[1] = 1;
      }
      if (nrhs > 0) y[v] = rhs[v] - s0;
      if (nrhs > 1) y[(size_t)H + v] = rhs[(size_t)H + v] - s1;
    }
  } else {
    for (int c = 0; c < nrhs; ++c) {
      const double* yc = y + (size_t)c * H;
      double s = 0.0;
      for (int q = q0 + sub; q < q1; q += g) {
        const int ch = p.child[q];
        s = fma(val[p.childq[q]] / d[ch], yc[ch], s);
      }
      s = group_sum(s, g);
      if (v >= 0 && sub == 0) y[(size_t)c * H + v] = rhs[(size_t)c * H + v] - s;
    }
  }
}

// One round (every thread of the block calls it; the caller puts the round's
// barrier after it).  The plan lists a round's nodes by descending child
// count and marks the first hcnt[r] as heavy: those take one warp each
// (lanes over the children), the others a lane group sized by their number.
// The host picks hcnt[r] from the child counts so that neither the few
// long lists (a core beta node holding dozens of peeled alpha leaves) nor
// the many short ones set the round's latency alone.
__device__ __forceinline__ void round_step(const double* __restrict__ val, const PeelPtrs& p,
                                           int r, bool with_d, double* __restrict__ d,
                                           const double* __restrict__ rhs, int nrhs, int H,
                                           double* __restrict__ y, int* __restrict__ info) {
  const int r0 = p.rptr[r], cnt = p.rptr[r + 1] - r0, nh = p.hcnt[r];
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k0 = 0; k0 < nh; k0 += nw) {
    const int k = k0 + warp;
    node_step(val, p, k < nh ? r0 + k : -1, threadIdx.x & 31, 32, with_d, d, rhs, nrhs, H, y,
              info);
  }
  const int nl = cnt - nh, l0 = r0 + nh;
  const int g = group_width(nl), per = blockDim.x / g, sub = threadIdx.x & (g - 1);
  for (int k0 = 0; k0 < nl; k0 += per) {
    const int k = k0 + (int)threadIdx.x / g;
    node_step(val, p, k < nl ? l0 + k : -1, sub, g, with_d, d, rhs, nrhs, H, y, info);
  }
}

// Core right-hand side reduced to the Schur side (kc core nodes t):
//   z[c * kc + t] = y_{s_t} - sum over the S-list of t of (a_q / d_e) y_e.
// Every thread calls it; no barrier inside.
__device__ __forceinline__ void core_rhs_step(const double* __restrict__ val, const PeelPtrs& p,
                                              const double* __restrict__ d,
                                              const double* __restrict__ y, int nrhs, int H,
                                              int kc, double* __restrict__ z) {
  const int g = group_width(kc), per = blockDim.x / g, sub = threadIdx.x & (g - 1);
  for (int k0 = 0; k0 < kc; k0 += per) {
    const int t = k0 + (int)threadIdx.x / g;
    const int q0 = t < kc ? p.sptr[t] : 0, q1 = t < kc ? p.sptr[t + 1] : 0;
    for (int c = 0; c < nrhs; ++c) {
      const double* yc = y + (size_t)c * H;
      double s = 0.0;
      for (int q = q0 + sub; q < q1; q += g) {
        const int ev = p.enodes[p.sadj[q]];
        s = fma(val[p.sq[q]] / d[ev], yc[ev], s);
      }
      s = group_sum(s, g);
      if (t < kc && sub == 0) z[(size_t)c * kc + t] = yc[p.snodes[t]] - s;
    }
  }
}

// Core E-side back-substitution from the Schur-side solution zs (stride kc):
//   x_e = (y_e - sum over the E-list of e of a_q zs_t) / d_e.
// Every thread calls it; no barrier inside.
__device__ __forceinline__ void core_back_step(const double* __restrict__ val, const PeelPtrs& p,
                                               const double* __restrict__ d,
                                               const double* __restrict__ y,
                                               const double* __restrict__ zs, int nrhs, int H,
                                               int kc, int ke, double* __restrict__ x) {
  const int g = group_width(ke), per = blockDim.x / g, sub = threadIdx.x & (g - 1);
  for (int k0 = 0; k0 < ke; k0 += per) {
    const int e = k0 + (int)threadIdx.x / g;
    const int q0 = e < ke ? p.eptr[e] : 0, q1 = e < ke ? p.eptr[e + 1] : 0;
    for (int c = 0; c < nrhs; ++c) {
      double s = 0.0;
      for (int q = q0 + sub; q < q1; q += g) s = fma(val[p.eq[q]], zs[(size_t)c * kc + p.eadj[q]], s);
      s = group_sum(s, g);
      if (e < ke && sub == 0) {
        const int ev = p.enodes[e];
        x[(size_t)c * H + ev] = (y[(size_t)c * H + ev] - s) / d[ev];
      }
    }
  }
}


// Pivots of every node, round by round; the core nodes come last (one round)
// and receive their diagonal updated by their peeled children.
__global__ void __launch_bounds__(kPeelThreads, kPeelMinBlocks) peel_factor_kernel(
    const double* __restrict__ val, PeelPtrs p, int rounds, double* __restrict__ d,
    int* __restrict__ info) {
  for (int r = 0; r <= rounds; ++r) {
    round_step(val, p, r, true, d, nullptr, 0, 0, nullptr, info);
    __syncthreads();
  }
}

// Row t of the core Schur complement:
//   S_t,: = d_{s_t} e_t - sum_{(e, q) in S-list t} (a_q / d_e) * (a_q' over E-list e)
__global__ void peel_assemble_kernel(const double* __restrict__ val, PeelPtrs p,
                                     const double* __restrict__ d, int kc,
                                     double* __restrict__ S) {
  const int t = blockIdx.x;
  double* __restrict__ Sr = S + (size_t)t * kc;
  for (int c = threadIdx.x; c < kc; c += blockDim.x) Sr[c] = 0.0;
  __syncthreads();
  if (threadIdx.x == 0) Sr[t] = d[p.snodes[t]];
  __syncthreads();
  for (int q = p.sptr[t]; q < p.sptr[t + 1]; ++q) {
    const int e = p.sadj[q];
    const double w = val[p.sq[q]] / d[p.enodes[e]];
    for (int q2 = p.eptr[e] + threadIdx.x; q2 < p.eptr[e + 1]; q2 += blockDim.x)
      Sr[p.eadj[q2]] -= w * val[p.eq[q2]];
    __syncthreads();
  }
}

// Core Schur complement from the contribution lists: one thread per entry.
__global__ void peel_contrib_kernel(const double* __restrict__ val, PeelPtrs p,
                                    const double* __restrict__ d, const double* __restrict__ W,
                                    int kc, double* __restrict__ S) {
  const long long total = (long long)kc * kc;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(idx / kc), t2 = (int)(idx - (long long)t * kc);
    double acc = (t == t2) ? d[p.snodes[t]] : 0.0;
    for (int q = p.ccp[idx]; q < p.ccp[idx + 1]; ++q) acc -= W[p.cw[q]] * val[p.cq2[q]];
    S[idx] = acc;
  }
}

// Edge weights of the core: W[pos] = a_{e,t} / d_e for every E-list entry
// (pivots d of the peel path, or A's own diagonal when d == nullptr).
__global__ void peel_weights_kernel(const double* __restrict__ val, PeelPtrs p,
                                    const double* __restrict__ d, int ke, double* __restrict__ W) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ke; e += gridDim.x * blockDim.x) {
    const int ev = p.enodes[e];
    const double de = d ? d[ev] : val[p.diagq[ev]];
    for (int q = p.eptr[e]; q < p.eptr[e + 1]; ++q) W[q] = val[p.eq[q]] / de;
  }
}

// Dense Schur complement of the whole graph from a no-peel plan: the pivots
// of both sides are A's own diagonal entries.
__global__ void dense_contrib_kernel(const double* __restrict__ val, PeelPtrs p,
                                     const double* __restrict__ W, int kc,
                                     double* __restrict__ S) {
  const long long total = (long long)kc * kc;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int t = (int)(idx / kc), t2 = (int)(idx - (long long)t * kc);
    double acc = (t == t2) ? val[p.diagq[p.snodes[t]]] : 0.0;
    for (int q = p.ccp[idx]; q < p.ccp[idx + 1]; ++q) acc -= W[p.cw[q]] * val[p.cq2[q]];
    S[idx] = acc;
  }
}

// z <- (L L^T)^{-1} z in shared memory (nrhs <= 2 columns of kc entries),
// with L the potrf factor in global memory (column-major kc x kc, lower:
// L(i, j) = L[j * kc + i]), by the whole block, 32-row blocks at a time:
//   - a block's diagonal 32 x 32 part of L is staged in shared memory
//     (coalesced over rows; double-buffered: the next block's is staged
//     while the current block's contribution is applied) and solved by one
//     warp per right-hand side with shuffles (lane r holds z_r);
//   - forward: the rows below take the block's contribution, one thread per
//     row (loads coalesced over rows for each column of the block);
//   - backward: the rows above take it, one thread per row (a row's 32
//     entries are contiguous in its column of L).
// Two block barriers per 32-row block.  idiag[kc] and blk[2 * 32 * 33] are
// shared scratch.  Replaces cuSOLVER potrs, whose two trsm launches took
// 90-450 us each at these sizes (latency-bound).
__device__ void dev_trisolve_cm(const double* __restrict__ L, int kc, double* __restrict__ z,
                                int nrhs, double* __restrict__ idiag, double* __restrict__ blk) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* z0 = z;
  double* z1 = z + kc;
  for (int t = threadIdx.x; t < kc; t += blockDim.x) idiag[t] = 1.0 / L[(size_t)t * kc + t];
  auto stage = [&](double* B, int j0, int bw) {  // B[r * 33 + c] = L(j0 + r, j0 + c)
    for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
      const int c = e >> 5, r = e & 31;
      if (r < bw && c < bw) B[r * 33 + c] = L[(size_t)(j0 + c) * kc + j0 + r];
    }
  };
  const int nb = (kc + 31) / 32;
  stage(blk, 0, min(32, kc));
  __syncthreads();
  for (int b = 0; b < nb; ++b) {  // L y = z
    const int j0 = b * 32, bw = min(32, kc - j0);
    const double* B = blk + (b & 1) * (32 * 33);
    if (warp < nrhs) {
      double* zc = z + (size_t)warp * kc;
      double zr = lane < bw ? zc[j0 + lane] : 0.0;
      for (int jj = 0; jj < bw; ++jj) {
        const double zj = __shfl_sync(0xffffffffu, zr, jj) * idiag[j0 + jj];
        if (lane == jj) zr = zj;
        else if (lane > jj && lane < bw) zr = fma(-B[lane * 33 + jj], zj, zr);
      }
      if (lane < bw) zc[j0 + lane] = zr;
    }
    __syncthreads();
    if (b + 1 < nb) stage(blk + ((b + 1) & 1) * (32 * 33), j0 + 32, min(32, kc - j0 - 32));
    // (unrolled: the block's L loads of a row are independent and must be in
    // flight together -- one at a time, each waited ~L2 latency)
    for (int i = j0 + bw + threadIdx.x; i < kc; i += blockDim.x) {
      double a0 = z0[i], a1 = nrhs > 1 ? z1[i] : 0.0;
#pragma unroll 8
      for (int c = 0; c < bw; ++c) {
        const double l = L[(size_t)(j0 + c) * kc + i];
        a0 = fma(-l, z0[j0 + c], a0);
        if (nrhs > 1) a1 = fma(-l, z1[j0 + c], a1);
      }
      z0[i] = a0;
      if (nrhs > 1) z1[i] = a1;
    }
    __syncthreads();
  }
  // L^T x = y, blocks from the last; the last block's diagonal part is
  // staged again into the buffer the forward sweep ends on
  {
    const int j0 = (nb - 1) * 32;
    stage(blk + (nb & 1) * (32 * 33), j0, kc - j0);
  }
  __syncthreads();
  for (int q = 0; q < nb; ++q) {
    const int b = nb - 1 - q, j0 = b * 32, bw = min(32, kc - j0);
    const double* B = blk + ((nb + q) & 1) * (32 * 33);
    if (warp < nrhs) {
      double* zc = z + (size_t)warp * kc;
      double zr = lane < bw ? zc[j0 + lane] : 0.0;
      for (int jj = bw - 1; jj >= 0; --jj) {
        const double zj = __shfl_sync(0xffffffffu, zr, jj) * idiag[j0 + jj];
        if (lane == jj) zr = zj;
        else if (lane < jj) zr = fma(-B[jj * 33 + lane], zj, zr);
      }
      if (lane < bw) zc[j0 + lane] = zr;
    }
    __syncthreads();
    if (b > 0) stage(blk + ((nb + q + 1) & 1) * (32 * 33), j0 - 32, 32);
    for (int j = threadIdx.x; j < j0; j += blockDim.x) {
      const double* Lj = L + (size_t)j * kc + j0;  // L(j0 + c, j)
      double a0 = z0[j], a1 = nrhs > 1 ? z1[j] : 0.0;
#pragma unroll 8
      for (int c = 0; c < bw; ++c) {
        const double l = Lj[c];
        a0 = fma(-l, z0[j0 + c], a0);
        if (nrhs > 1) a1 = fma(-l, z1[j0 + c], a1);
      }
      z0[j] = a0;
      if (nrhs > 1) z1[j] = a1;
    }
    __syncthreads();
  }
}

// Forward sweep (y = L^{-1} b over the peeled rounds and the core's own
// children), then the reduction of the core right-hand side to the Schur
// side, rs.  With Lcm (the core's potrf factor, kc <= kPeelTriMax) the core
// solve rs <- S^{-1} rs runs here too, in shared memory (dynamic shared
// memory: tri_smem(kc)); without it the caller runs potrs.
__global__ void __launch_bounds__(kPeelThreads, kPeelMinBlocks) peel_forward_kernel(
    const double* __restrict__ val, PeelPtrs p, int rounds, const double* __restrict__ d,
    const double* __restrict__ rhs, int nrhs, int H, int kc, double* __restrict__ y,
    double* __restrict__ rs, const double* __restrict__ Lcm) {
  extern __shared__ double tsm[];
  for (int r = 0; r <= rounds; ++r) {
    round_step(val, p, r, false, const_cast<double*>(d), rhs, nrhs, H, y, nullptr);
    __syncthreads();
  }
  if (Lcm == nullptr) {
    core_rhs_step(val, p, d, y, nrhs, H, kc, rs);
    return;
  }
  double* z = tsm;                // [2 kc]
  double* idiag = tsm + 2 * kc;   // [kc]
  double* blk = idiag + kc;       // [2 * 32 * 33]
  core_rhs_step(val, p, d, y, nrhs, H, kc, z);
  __syncthreads();
  dev_trisolve_cm(Lcm, kc, z, nrhs, idiag, blk);
  for (int e = threadIdx.x; e < nrhs * kc; e += blockDim.x) rs[e] = z[e];
}

// Core back-substitution, then the backward sweep over the peeled rounds.
__global__ void __launch_bounds__(kPeelThreads, kPeelMinBlocks) peel_backward_kernel(
    const double* __restrict__ val, PeelPtrs p, int rounds, const double* __restrict__ d,
    const double* __restrict__ y, const double* __restrict__ rs, int nrhs, int H, int kc,
    int ke, double* __restrict__ x) {
  for (int t = threadIdx.x; t < kc; t += blockDim.x)
    for (int c = 0; c < nrhs; ++c) x[(size_t)c * H + p.snodes[t]] = rs[(size_t)c * kc + t];
  core_back_step(val, p, d, y, rs, nrhs, H, kc, ke, x);
  __syncthreads();
  for (int r = rounds - 1; r >= 0; --r) {
    for (int idx = p.rptr[r] + threadIdx.x; idx < p.rptr[r + 1]; idx += blockDim.x) {
      const int v = p.order[idx];
      const int u = p.ppar[idx];
      for (int c = 0; c < nrhs; ++c) {
        double xv = y[(size_t)c * H + v];
        if (u >= 0) xv -= val[p.pparq[idx]] * x[(size_t)c * H + u];
        x[(size_t)c * H + v] = xv / d[v];
      }
    }
    __syncthreads();
  }
}

// ---- small-core path: everything in one CTA --------------------------------
// Forward values of the peeled rounds and the core (pivots d already known).
__device__ void dev_forward(const double* __restrict__ val, const PeelPtrs& p, int rounds,
                            const double* __restrict__ d, const double* __restrict__ rhs,
                            int nrhs, int H, double* __restrict__ y) {
  for (int r = 0; r <= rounds; ++r) {
    round_step(val, p, r, false, const_cast<double*>(d), rhs, nrhs, H, y, nullptr);
    __syncthreads();
  }
}

// Core right-hand side reduced to the Schur side, into z[c * kc + t].
__device__ void dev_core_rhs(const double* __restrict__ val, const PeelPtrs& p,
                             const double* __restrict__ d, const double* __restrict__ y,
                             int nrhs, int H, int kc, double* __restrict__ z) {
  core_rhs_step(val, p, d, y, nrhs, H, kc, z);
  __syncthreads();
}

// Row stride of the in-shared-memory core matrix: odd, so that a warp reading
// one column (consecutive rows) touches distinct bank pairs.
__host__ __device__ __forceinline__ int core_ld(int kc) { return kc | 1; }

// z <- (L L^T)^{-1} z for nrhs columns; L lower, row-major kc x kc with row
// stride ld (shared), idiag[j] = 1 / L_jj.  One warp per right-hand side,
// blocks of 32 rows: the diagonal block is solved in registers (lane r holds
// z_r; the solved value is broadcast by a shuffle), the rows below (forward)
// or the block's own entries (backward) take the other blocks' contributions
// as dot products.  __syncwarp only.
__device__ void dev_trisolve(const double* __restrict__ L, const double* __restrict__ idiag,
                             int kc, int ld, double* __restrict__ z, int nrhs) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < nrhs) {
    double* zc = z + (size_t)warp * kc;
    for (int j0 = 0; j0 < kc; j0 += 32) {  // L y = z
      const int bw = min(32, kc - j0);
      double zr = (lane < bw) ? zc[j0 + lane] : 0.0;
      for (int jj = 0; jj < bw; ++jj) {
        const double zj = __shfl_sync(0xffffffffu, zr, jj) * idiag[j0 + jj];
        if (lane == jj) zr = zj;
        if (lane > jj && lane < bw) zr = fma(-L[(size_t)(j0 + lane) * ld + j0 + jj], zj, zr);
      }
      if (lane < bw) zc[j0 + lane] = zr;
      __syncwarp();
      for (int i = j0 + bw + lane; i < kc; i += 32) {
        const double* Li = L + (size_t)i * ld + j0;
        double a0 = zc[i], a1 = 0.0;
        int c = 0;
        for (; c + 1 < bw; c += 2) {
          a0 = fma(-Li[c], zc[j0 + c], a0);
          a1 = fma(-Li[c + 1], zc[j0 + c + 1], a1);
        }
        if (c < bw) a0 = fma(-Li[c], zc[j0 + c], a0);
        zc[i] = a0 + a1;
      }
      __syncwarp();
    }
    for (int j1 = kc; j1 > 0; j1 -= 32) {  // L^T x = y
      const int j0 = max(0, j1 - 32), bw = j1 - j0;
      double zr = 0.0;
      if (lane < bw) {
        double a0 = zc[j0 + lane], a1 = 0.0;
        int i = j1;
        for (; i + 1 < kc; i += 2) {
          a0 = fma(-L[(size_t)i * ld + j0 + lane], zc[i], a0);
          a1 = fma(-L[(size_t)(i + 1) * ld + j0 + lane], zc[i + 1], a1);
        }
        if (i < kc) a0 = fma(-L[(size_t)i * ld + j0 + lane], zc[i], a0);
        zr = a0 + a1;
      }
      for (int jj = bw - 1; jj >= 0; --jj) {
        const double zj = __shfl_sync(0xffffffffu, zr, jj) * idiag[j0 + jj];
        if (lane == jj) zr = zj;
        if (lane < jj) zr = fma(-L[(size_t)(j0 + jj) * ld + j0 + lane], zj, zr);
      }
      if (lane < bw) zc[j0 + lane] = zr;
      __syncwarp();
    }
  }
  __syncthreads();
}

// In-place Cholesky S = L L^T of the lower triangle (row-major kc x kc, row
// stride ld, shared), blocked by panels of 32 columns, three block barriers
// per panel; idiag[j] <- 1 / L_jj.
//   1. the 32 x 32 diagonal block, by warp 0 alone (warp_block_cholesky:
//      left-looking, lane r computes row r of the block);
//   2. the panel below it, L21 = S21 L11^{-T}: one warp per two rows, a
//      row's 32 entries in the lanes, each solved column broadcast by a
//      shuffle and subtracted from the later lanes (32 short steps instead of
//      a thread walking 528 dependent multiply-adds per row);
//   3. the trailing update S22 -= L21 L21^T on the lower triangle: a work
//      item is one column c of a 4-row tile (rows i0..i0+3, c <= i), its
//      four dot products over the panel accumulated in registers.
// A pivot that is not positive and finite sets info = column + 1 and
// continues with d = 1 (the last such column is reported).
__device__ void dev_cholesky(double* __restrict__ S, double* __restrict__ idiag, int kc, int ld,
                             int* __restrict__ info) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int j0 = 0; j0 < kc; j0 += 32) {
    const int bw = min(32, kc - j0);
    if (warp == 0) warp_block_cholesky(S + (size_t)j0 * ld + j0, ld, bw, idiag + j0, j0, info);
    __syncthreads();
    const int r0 = j0 + bw;  // first row below the block
    // panel rows, two per warp: lane k holds entry k of each row; column jj
    // is final once the earlier columns are subtracted, is broadcast by a
    // shuffle and subtracted from the lanes k > jj (L11[k][jj] read by lane
    // k: consecutive rows, distinct banks under the odd row stride)
    {
      const int nw = blockDim.x >> 5;
      const double* L11 = S + (size_t)j0 * ld + j0;
      for (int i = r0 + 2 * warp; i < kc; i += 2 * nw) {
        const bool two = i + 1 < kc;
        double* Si = S + (size_t)i * ld + j0;
        double* Sj = Si + ld;
        double s0 = lane < bw ? Si[lane] : 0.0;
        double s1 = (two && lane < bw) ? Sj[lane] : 0.0;
        for (int jj = 0; jj < bw; ++jj) {
          const double l = (lane > jj && lane < bw) ? L11[(size_t)lane * ld + jj] : 0.0;
          const double dj = idiag[j0 + jj];
          const double x0 = __shfl_sync(0xffffffffu, s0, jj) * dj;
          const double x1 = __shfl_sync(0xffffffffu, s1, jj) * dj;
          if (lane == jj) {
            s0 = x0;
            s1 = x1;
          } else if (lane > jj) {
            s0 = fma(-l, x0, s0);
            s1 = fma(-l, x1, s1);
          }
        }
        if (lane < bw) {
          Si[lane] = s0;
          if (two) Sj[lane] = s1;
        }
      }
    }
    __syncthreads();
    const int w = kc - r0;
    if (w > 0) {
      // items: row tile ti (rows r0 + 4 ti .. + 3) has 4 (ti + 1) columns
      // c = r0 .. r0 + 4 ti + 3; items before tile ti: 2 ti (ti + 1)
      const int nt = (w + 3) >> 2;
      const int items = 2 * nt * (nt + 1);
      for (int e = threadIdx.x; e < items; e += blockDim.x) {
        int ti = (int)((sqrt(2.0 * e + 1.0) - 1.0) * 0.5);
        while (2 * (ti + 1) * (ti + 2) <= e) ++ti;
        while (2 * ti * (ti + 1) > e) --ti;
        const int c = r0 + (e - 2 * ti * (ti + 1));
        const int i0 = r0 + 4 * ti;
        if (c >= kc) continue;
        const double* Sc = S + (size_t)c * ld + j0;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        const int nr = min(4, kc - i0);
        for (int k = 0; k < bw; ++k) {
          const double b = Sc[k];
#pragma unroll
          for (int r = 0; r < 4; ++r)
            if (r < nr) acc[r] = fma(S[(size_t)(i0 + r) * ld + j0 + k], b, acc[r]);
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
          if (r < nr && c <= i0 + r) S[(size_t)(i0 + r) * ld + c] -= acc[r];
      }
    }
    __syncthreads();
  }
}

// Core back-substitution from the Schur-side solution zc, then the backward
// sweep over the peeled rounds.
__device__ void dev_backward(const double* __restrict__ val, const PeelPtrs& p, int rounds,
                             const double* __restrict__ d, const double* __restrict__ y,
                             const double* __restrict__ zc, int nrhs, int H, int kc, int ke,
                             double* __restrict__ x) {
  for (int t = threadIdx.x; t < kc; t += blockDim.x)
    for (int c = 0; c < nrhs; ++c) x[(size_t)c * H + p.snodes[t]] = zc[(size_t)c * kc + t];
  core_back_step(val, p, d, y, zc, nrhs, H, kc, ke, x);
  __syncthreads();
  for (int r = rounds - 1; r >= 0; --r) {
    for (int idx = p.rptr[r] + threadIdx.x; idx < p.rptr[r + 1]; idx += blockDim.x) {
      const int v = p.order[idx];
      const int u = p.ppar[idx];
      for (int c = 0; c < nrhs; ++c) {
        double xv = y[(size_t)c * H + v];
        if (u >= 0) xv -= val[p.pparq[idx]] * x[(size_t)c * H + u];
        x[(size_t)c * H + v] = xv / d[v];
      }
    }
    __syncthreads();
  }
}

// Factorization (pivots d, core factor L -> Lout) and, for nrhs > 0, the
// solve x = A^{-1} rhs.  Dynamic shared memory: kc*ld + 3*kc doubles (ld =
// core_ld(kc), the shared row stride of the core matrix; then 2 kc for the
// reduced right-hand sides and kc for the inverse diagonal of the factor).
__global__ void __launch_bounds__(kPeelThreads, kPeelMinBlocks) peel_fused_kernel(
    const double* __restrict__ val, PeelPtrs p, int rounds, int kc, int ke, int H,
    const double* __restrict__ rhs, int nrhs, double* __restrict__ x, double* __restrict__ d,
    double* __restrict__ y, double* __restrict__ Lout, int* __restrict__ info,
    double* __restrict__ W) {
  extern __shared__ double sm[];
  const int ld = core_ld(kc);
  double* S = sm;
  double* z = sm + (size_t)kc * ld;
  double* idiag = z + 2 * (size_t)kc;
  // pivots and forward values, round by round (core last)
  for (int r = 0; r <= rounds; ++r) {
    round_step(val, p, r, true, d, rhs, nrhs, H, y, info);
    __syncthreads();
  }
  if (kc > 0 && p.ccp != nullptr) {
    // edge weights (a node's E-list split over a lane group), then the core
    // Schur complement from the contribution lists, one thread per entry
    {
      const int g = group_width(ke), per = blockDim.x / g, sub = threadIdx.x & (g - 1);
      for (int e = (int)threadIdx.x / g; e < ke; e += per) {
        const double rde = 1.0 / d[p.enodes[e]];
        for (int q = p.eptr[e] + sub; q < p.eptr[e + 1]; q += g) W[q] = val[p.eq[q]] * rde;
      }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < kc * kc; idx += blockDim.x) {
      const int t = idx / kc, t2 = idx - t * kc;
      double acc = (t == t2) ? d[p.snodes[t]] : 0.0;
#pragma unroll 4
      for (int q = p.ccp[idx]; q < p.ccp[idx + 1]; ++q) acc -= W[p.cw[q]] * val[p.cq2[q]];
      S[(size_t)t * ld + t2] = acc;
    }
    __syncthreads();
  } else if (kc > 0) {
    // core Schur complement, one warp per row (same order as the multi-CTA path)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int t = warp; t < kc; t += nw) {
      double* Sr = S + (size_t)t * ld;
      for (int c = lane; c < kc; c += 32) Sr[c] = 0.0;
      __syncwarp();
      if (lane == 0) Sr[t] = d[p.snodes[t]];
      __syncwarp();
      for (int q = p.sptr[t]; q < p.sptr[t + 1]; ++q) {
        const int e = p.sadj[q];
        const double w = val[p.sq[q]] / d[p.enodes[e]];
        for (int q2 = p.eptr[e] + lane; q2 < p.eptr[e + 1]; q2 += 32)
          Sr[p.eadj[q2]] -= w * val[p.eq[q2]];
        __syncwarp();
      }
    }
    __syncthreads();
  }
  if (kc > 0) {
    dev_cholesky(S, idiag, kc, ld, info);
    for (int e = threadIdx.x; e < kc * kc; e += blockDim.x) {
      const int t = e / kc;
      Lout[e] = S[(size_t)t * ld + (e - t * kc)];
    }
  }
  if (nrhs == 0) return;
  if (kc > 0) {
    dev_core_rhs(val, p, d, y, nrhs, H, kc, z);
    dev_trisolve(S, idiag, kc, ld, z, nrhs);
  }
  dev_backward(val, p, rounds, d, y, z, nrhs, H, kc, ke, x);
}

// Solve with a stored small-core factor (pivots d, L in global memory).
__global__ void __launch_bounds__(kPeelThreads, kPeelMinBlocks) peel_small_solve_kernel(
    const double* __restrict__ val, PeelPtrs p, int rounds, int kc, int ke, int H,
    const double* __restrict__ rhs, int nrhs, double* __restrict__ x,
    const double* __restrict__ d, double* __restrict__ y, const double* __restrict__ Lin) {
  extern __shared__ double sm[];
  const int ld = core_ld(kc);
  double* S = sm;
  double* z = sm + (size_t)kc * ld;
  double* idiag = z + 2 * (size_t)kc;
  for (int e = threadIdx.x; e < kc * kc; e += blockDim.x) {
    const int t = e / kc;
    S[(size_t)t * ld + (e - t * kc)] = Lin[e];
  }
  for (int t = threadIdx.x; t < kc; t += blockDim.x) idiag[t] = 1.0 / Lin[(size_t)t * kc + t];
  dev_forward(val, p, rounds, d, rhs, nrhs, H, y);  // its round barriers also publish S
  if (kc > 0) {
    dev_core_rhs(val, p, d, y, nrhs, H, kc, z);
    dev_trisolve(S, idiag, kc, ld, z, nrhs);
  }
  dev_backward(val, p, rounds, d, y, z, nrhs, H, kc, ke, x);
}

size_t tri_smem(int kc) { return ((size_t)3 * std::max(kc, 1) + 2 * 32 * 33) * sizeof(double); }

size_t small_smem(int kc) {
  return ((size_t)kc * core_ld(kc) + 3 * (size_t)std::max(kc, 1)) * sizeof(double);
}

int ensure_small_smem() {
  static thread_local int done_dev = -1;
  int dev = 0;
  CG_TRY_CUDA(cudaGetDevice(&dev));
  if (done_dev == dev) return CG_OK;
  const int bytes = (int)small_smem(kSmallCore);
  CG_TRY_CUDA(cudaFuncSetAttribute(peel_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CG_TRY_CUDA(cudaFuncSetAttribute(peel_small_solve_kernel,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  CG_TRY_CUDA(cudaFuncSetAttribute(peel_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)tri_smem(kPeelTriMax)));
  done_dev = dev;
  return CG_OK;
}

int alloc_dev(PeelFactor& P, void** ptr, size_t bytes) {
  if (P.stream_ordered) CG_TRY(pool_alloc_async(ptr, bytes, P.alloc_stream));
  else CG_TRY_CUDA(cudaMalloc(ptr, bytes));
  return CG_OK;
}

void free_dev(PeelFactor& P, void* ptr) {
  if (!ptr) return;
  if (P.stream_ordered) cudaFreeAsync(ptr, P.alloc_stream);
  else cudaFree(ptr);
}

}  // namespace

void peel_release(PeelFactor& P) {
  free_dev(P, P.block);
  P.block = nullptr;
  P.block_bytes = 0;
  P.ready = false;
}

int peel_plan(PeelFactor& P, const SpHess& A, cudaStream_t st, bool no_peel) {
  const int H = A.H;
  // pattern to the host through pinned memory (pageable copies serialise
  // with the other streams' work)
  std::vector<int> rp(H + 1);
  CG_TRY(read_device_bulk(rp.data(), A.rowptr, (H + 1) * sizeof(int), st));
  const int nl = rp[H];
  std::vector<int> cl(std::max(nl, 1));
  CG_TRY(read_device_bulk(cl.data(), A.col, (size_t)nl * sizeof(int), st));
  return peel_plan_host(P, A.n, A.m, rp, cl, no_peel);
}

int peel_plan_host(PeelFactor& P, int n, int m, const std::vector<int>& rp,
                   const std::vector<int>& cl, bool no_peel) {
  const int H = n + m - 1;
  P.ready = false;
  P.n = n;
  P.m = m;
  P.H = H;

  // diagonal positions and the bipartite adjacency (neighbour, value index)
  std::vector<int> diagq(H);
  std::vector<int> deg(H, 0);
  for (int i = 0; i < n; ++i) diagq[i] = rp[i];
  for (int j = 0; j < m - 1; ++j) {
    const int r = n + j;
    diagq[r] = rp[r + 1] - 1;
    for (int q = rp[r]; q < rp[r + 1] - 1; ++q) {
      deg[r]++;
      deg[cl[q]]++;
    }
  }
  std::vector<int> aptr(H + 1, 0);
  for (int v = 0; v < H; ++v) aptr[v + 1] = aptr[v] + deg[v];
  std::vector<int> adj(std::max(aptr[H], 1)), adjq(std::max(aptr[H], 1));
  {
    std::vector<int> fill(aptr.begin(), aptr.end() - 1);
    for (int j = 0; j < m - 1; ++j) {
      const int r = n + j;
      for (int q = rp[r]; q < rp[r + 1] - 1; ++q) {
        const int i = cl[q];
        adj[fill[r]] = i;
        adjq[fill[r]++] = q;
        adj[fill[i]] = r;
        adjq[fill[i]++] = q;
      }
    }
  }

  // synchronous peeling
  std::vector<char> alive(H, 1), taken(H, 0);
  std::vector<int> par(H, -1), parq(H, -1);
  std::vector<int> order;
  order.reserve(H);
  std::vector<int> rptr(1, 0);
  std::vector<int> cur, next;
  for (int v = 0; v < H; ++v)
    if (!no_peel && deg[v] <= 1) cur.push_back(v);
  int rounds = 0;
  while (!cur.empty()) {
    if (rounds >= kMaxPeelRounds) {
      P.rounds = rounds + 1;  // over the limit: the caller keeps the dense path
      P.kc = H;
      P.ke = 0;
      return CG_OK;
    }
    next.clear();
    std::vector<int> sel;
    for (int v : cur) {
      if (!alive[v] || deg[v] > 1) continue;
      int u = -1, uq = -1;
      if (deg[v] == 1)
        for (int q = aptr[v]; q < aptr[v + 1]; ++q)
          if (alive[adj[q]]) {
            u = adj[q];
            uq = adjq[q];
            break;
          }
      if (u >= 0 && taken[u]) {  // its neighbour goes this round: v waits
        next.push_back(v);
        continue;
      }
      taken[v] = 1;
      par[v] = u;
      parq[v] = uq;
      sel.push_back(v);
    }
    for (int v : sel) {
      alive[v] = 0;
      order.push_back(v);
    }
    for (int v : sel) {
      const int u = par[v];
      if (u >= 0) {
        deg[u]--;
        if (deg[u] <= 1) next.push_back(u);
      }
    }
    for (int v : sel) taken[v] = 0;
    std::sort(next.begin(), next.end());
    next.erase(std::unique(next.begin(), next.end()), next.end());
    cur.swap(next);
    rptr.push_back((int)order.size());
    ++rounds;
  }
  const int npeel = (int)order.size();
  // core nodes (one final round) and the sides of the core
  std::vector<int> core_a, core_b;
  for (int v = 0; v < H; ++v)
    if (alive[v]) {
      order.push_back(v);
      (v < n ? core_a : core_b).push_back(v);
    }
  rptr.push_back((int)order.size());
  // child counts; each round's nodes by descending count, the first hcnt[r]
  // of them heavy (one warp each on the device).  hcnt[r] minimises an
  // estimate of the round's latency in dependent child steps: a pass of
  // kWarps heavy nodes costs 1.5 + ceil(c_first / 32), a pass of the light
  // nodes (lane groups of g, as group_width sizes them) 1 + ceil(c_max / g),
  // plus 0.5 for the shuffle reduction when g > 1.
  std::vector<int> ccount(H, 0);
  for (int k = 0; k < npeel; ++k)
    if (par[order[k]] >= 0) ccount[par[order[k]]]++;
  std::vector<int> hcnt(rounds + 1, 0);
  {
    constexpr int kWarps = kPeelThreads / 32;
    for (int r = 0; r <= rounds; ++r) {
      const int b0 = rptr[r], cnt = rptr[r + 1] - b0;
      std::stable_sort(order.begin() + b0, order.begin() + b0 + cnt,
                       [&](int x, int y) { return ccount[x] > ccount[y]; });
      double best = 0.0, heavy = 0.0;
      int bnh = 0;
      for (int nh = 0; nh <= cnt; ++nh) {
        if (nh > 0 && (nh - 1) % kWarps == 0) heavy += 1.5 + (ccount[order[b0 + nh - 1]] + 31) / 32;
        const int nl = cnt - nh;
        double light = 0.0;
        if (nl > 0) {
          int g = 1;
          while (g < 32 && nl * (g * 2) <= kPeelThreads) g *= 2;
          const int per = kPeelThreads / g, passes = (nl + per - 1) / per;
          light = passes * (1.0 + (ccount[order[b0 + nh]] + g - 1) / g + (g > 1 ? 0.5 : 0.0));
        }
        if (nh == 0 || heavy + light < best) {
          best = heavy + light;
          bnh = nh;
        }
      }
      hcnt[r] = bnh;
    }
  }
  const bool elim_a = core_a.size() >= core_b.size();
  const std::vector<int>& snodes = elim_a ? core_b : core_a;
  const std::vector<int>& enodes = elim_a ? core_a : core_b;
  const int kc = (int)snodes.size(), ke = (int)enodes.size();
  std::vector<int> loc(H, -1);
  for (int t = 0; t < kc; ++t) loc[snodes[t]] = t;
  for (int e = 0; e < ke; ++e) loc[enodes[e]] = e;
  // children lists (eliminated neighbours of every node), in round order
  // children by order position: the children of the node at position k
  // occupy [cpos[k], cpos[k + 1]), in round order; per position also the
  // diagonal value index and the parent edge
  const int npos = (int)order.size();  // every node: peeled rounds + core
  std::vector<int> posof(H, -1);
  for (int k = 0; k < npos; ++k) posof[order[k]] = k;
  std::vector<int> cpos(npos + 1, 0);
  for (int k = 0; k < npos; ++k) cpos[k + 1] = cpos[k] + ccount[order[k]];
  std::vector<int> child(std::max(cpos[npos], 1)), childq(std::max(cpos[npos], 1));
  {
    std::vector<int> fill(cpos.begin(), cpos.end() - 1);
    for (int k = 0; k < npeel; ++k) {
      const int v = order[k], u = par[v];
      if (u < 0) continue;
      const int pu = posof[u];
      child[fill[pu]] = v;
      childq[fill[pu]++] = parq[v];
    }
  }
  std::vector<int> dqo(npos), ppar(npos), pparq(npos);
  for (int k = 0; k < npos; ++k) {
    const int v = order[k];
    dqo[k] = diagq[v];
    ppar[k] = par[v];
    pparq[k] = parq[v];
  }
  // core adjacency restricted to alive neighbours, as local indices
  auto core_lists = [&](const std::vector<int>& nodes, std::vector<int>& ptr, std::vector<int>& ladj,
                        std::vector<int>& lq) {
    ptr.assign(nodes.size() + 1, 0);
    ladj.clear();
    lq.clear();
    for (size_t t = 0; t < nodes.size(); ++t) {
      const int v = nodes[t];
      for (int q = aptr[v]; q < aptr[v + 1]; ++q)
        if (alive[adj[q]]) {
          ladj.push_back(loc[adj[q]]);
          lq.push_back(adjq[q]);
        }
      ptr[t + 1] = (int)ladj.size();
    }
  };
  std::vector<int> sptr, sadj, sq, eptr, eadj, eq;
  core_lists(snodes, sptr, sadj, sq);
  core_lists(enodes, eptr, eadj, eq);

  // pack
  std::vector<int>& I = P.h_ints;
  I.clear();
  auto put = [&I](const std::vector<int>& v, size_t count) {
    const size_t off = I.size();
    I.insert(I.end(), v.begin(), v.begin() + count);
    while (I.size() % 64) I.push_back(0);  // 256-byte alignment of every array
    return off;
  };
  P.off_order = put(order, order.size());
  P.off_rptr = put(rptr, rptr.size());
  P.off_hcnt = put(hcnt, hcnt.size());
  P.off_diagq = put(diagq, H);
  P.off_cpos = put(cpos, npos + 1);
  P.off_child = put(child, cpos[npos]);
  P.off_childq = put(childq, cpos[npos]);
  P.off_dqo = put(dqo, npos);
  P.off_ppar = put(ppar, npos);
  P.off_pparq = put(pparq, npos);
  P.off_snodes = put(snodes, kc);
  P.off_enodes = put(enodes, ke);
  P.off_sptr = put(sptr, kc + 1);
  P.off_sadj = put(sadj, sadj.size());
  P.off_sq = put(sq, sq.size());
  P.off_eptr = put(eptr, ke + 1);
  P.off_eadj = put(eadj, eadj.size());
  P.off_eq = put(eq, eq.size());
  // contribution lists: every pair of S-neighbours (t, t2) of an eliminated
  // core node e adds (a_{t,e} / d_e) a_{e,t2} to entry (t, t2); listed per
  // entry in ascending e, the order of the row-wise assembly
  P.contrib = kc > 0 && kc <= kContribMax;
  if (P.contrib) {
    std::vector<int> ccnt((size_t)kc * kc + 1, 0);
    for (int e = 0; e < ke; ++e)
      for (int p1 = eptr[e]; p1 < eptr[e + 1]; ++p1)
        for (int p2 = eptr[e]; p2 < eptr[e + 1]; ++p2) ccnt[(size_t)eadj[p1] * kc + eadj[p2] + 1]++;
    for (size_t k2 = 0; k2 < (size_t)kc * kc; ++k2) ccnt[k2 + 1] += ccnt[k2];
    const size_t nc = (size_t)ccnt[(size_t)kc * kc];
    std::vector<int> ce(std::max<size_t>(nc, 1)), cq1(std::max<size_t>(nc, 1)), cq2(std::max<size_t>(nc, 1));
    std::vector<int> fill(ccnt.begin(), ccnt.end() - 1);
    for (int e = 0; e < ke; ++e)
      for (int p1 = eptr[e]; p1 < eptr[e + 1]; ++p1)
        for (int p2 = eptr[e]; p2 < eptr[e + 1]; ++p2) {
          const int pos = fill[(size_t)eadj[p1] * kc + eadj[p2]]++;
          ce[pos] = e;
          cq1[pos] = p1;  // E-list position: weight index
          cq2[pos] = eq[p2];
        }
    P.off_ccp = put(ccnt, ccnt.size());
    P.off_ce = put(ce, nc);
    P.off_cq1 = put(cq1, nc);
    P.off_cq2 = put(cq2, nc);
  }
  P.rounds = rounds;
  P.npeel = npeel;
  P.kc = kc;
  P.ke = ke;
  P.nchild = cpos[npos];
  P.ns_adj = (long long)sadj.size();
  P.ne_adj = (long long)eadj.size();
  return CG_OK;
}

int peel_upload(PeelFactor& P, cusolverDnHandle_t h, cudaStream_t st, bool plan_only) {
  const int H = P.H, kc = P.kc;
  int lwork = 0;
  if (!plan_only && kc > kSmallCore &&
      cusolverDnDpotrf_bufferSize(h, CUBLAS_FILL_MODE_LOWER, kc, nullptr, kc, &lwork) !=
          CUSOLVER_STATUS_SUCCESS) {
    set_last_error("cusolverDnDpotrf_bufferSize failed", __FILE__, __LINE__);
    return CG_ERR_SOLVER;
  }
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t ib = al(P.h_ints.size() * sizeof(int));
  const size_t wb = al((size_t)std::max<long long>(P.ne_adj, 1) * 8);
  const size_t bytes = plan_only ? ib + wb : ib + wb + al((size_t)H * 8) + al((size_t)kc * kc * 8) +
                       al((size_t)std::max(lwork, 1) * 8) + al(3 * sizeof(int)) +
                       al((size_t)2 * H * 8) + al((size_t)2 * std::max(kc, 1) * 8);
  if (bytes > P.block_bytes) {
    free_dev(P, P.block);
    P.block = nullptr;
    P.block_bytes = 0;
    CG_TRY(alloc_dev(P, &P.block, bytes));
    P.block_bytes = bytes;
  }
  char* p = static_cast<char*>(P.block);
  P.ints = reinterpret_cast<int*>(p); p += ib;
  P.W = reinterpret_cast<double*>(p); p += wb;
  if (plan_only) {
    P.d = P.S = P.work = P.y = P.rs = nullptr;
    P.info = nullptr;
    P.lwork = 0;
    CG_TRY_CUDA(cudaMemcpyAsync(P.ints, P.h_ints.data(), P.h_ints.size() * sizeof(int),
                                cudaMemcpyHostToDevice, st));
    P.ready = true;
    return CG_OK;
  }
  P.d = reinterpret_cast<double*>(p); p += al((size_t)H * 8);
  P.S = reinterpret_cast<double*>(p); p += al((size_t)kc * kc * 8);
  P.work = reinterpret_cast<double*>(p); p += al((size_t)std::max(lwork, 1) * 8);
  P.info = reinterpret_cast<int*>(p); p += al(3 * sizeof(int));
  P.y = reinterpret_cast<double*>(p); p += al((size_t)2 * H * 8);
  P.rs = reinterpret_cast<double*>(p);
  P.lwork = lwork;
  CG_TRY_CUDA(cudaMemcpyAsync(P.ints, P.h_ints.data(), P.h_ints.size() * sizeof(int),
                              cudaMemcpyHostToDevice, st));
  // the pageable source is staged before cudaMemcpyAsync returns
  P.ready = true;
  return CG_OK;
}

int peel_factor(PeelFactor& P, const SpHess& A, cusolverDnHandle_t h, cudaStream_t st) {
  if (!P.ready) {
    set_last_error("peel factor: no plan for the current pattern", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  const PeelPtrs pp = ptrs_of(P);
  CG_TRY_CUDA(cudaMemsetAsync(P.info, 0, 3 * sizeof(int), st));
  if (P.kc <= kSmallCore) return peel_factor_solve(P, A, h, nullptr, nullptr, 0, st);
  { peel_factor_kernel<<<1, kPeelThreads, 0, st>>>(A.val, pp, P.rounds, P.d, P.info); count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  if (P.kc > 0) {
    if (P.contrib) {
      const long long total = (long long)P.kc * P.kc;
      const int grid = (int)std::min<long long>((total + 255) / 256, 148 * 8);
      { peel_weights_kernel<<<std::max(1, std::min((P.ke + 255) / 256, 148 * 4)), 256, 0, st>>>(A.val, pp, P.d, P.ke, P.W); count_launch(); }
      { peel_contrib_kernel<<<grid, 256, 0, st>>>(A.val, pp, P.d, P.W, P.kc, P.S); count_launch(); }
    } else {
      { peel_assemble_kernel<<<P.kc, 256, 0, st>>>(A.val, pp, P.d, P.kc, P.S); count_launch(); }
    }
    CG_TRY_CUDA(cudaGetLastError());
    if (cusolverDnSetStream(h, st) != CUSOLVER_STATUS_SUCCESS) return CG_ERR_SOLVER;
    if (cusolverDnDpotrf(h, CUBLAS_FILL_MODE_LOWER, P.kc, P.S, P.kc, P.work, P.lwork, P.info) !=
        CUSOLVER_STATUS_SUCCESS) {
      set_last_error("cusolverDnDpotrf failed to launch", __FILE__, __LINE__);
      return CG_ERR_SOLVER;
    }
  }
  return CG_OK;
}

int peel_info_async(const PeelFactor& P, int* host2, cudaStream_t st) {
  CG_TRY_CUDA(cudaMemcpyAsync(host2, P.info, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  return CG_OK;
}

int peel_solve(PeelFactor& P, const SpHess& A, cusolverDnHandle_t h, const double* rhs,
               double* x, int nrhs, cudaStream_t st) {
  if (nrhs < 1 || nrhs > 2) return CG_ERR_INVALID_ARG;
  const PeelPtrs pp = ptrs_of(P);
  if (P.kc <= kSmallCore) {
    CG_TRY(ensure_small_smem());
    { peel_small_solve_kernel<<<1, kPeelThreads, small_smem(P.kc), st>>>(
        A.val, pp, P.rounds, P.kc, P.ke, P.H, rhs, nrhs, x, P.d, P.y, P.S); count_launch(); }
    CG_TRY_CUDA(cudaGetLastError());
    return CG_OK;
  }
  // cores up to kPeelTriMax: the triangular solves with the potrf factor in
  // the forward kernel; larger ones: potrs
  const bool tri = P.kc > 0 && P.kc <= kPeelTriMax;
  if (tri) CG_TRY(ensure_small_smem());
  { peel_forward_kernel<<<1, kPeelThreads, tri ? tri_smem(P.kc) : 0, st>>>(
        A.val, pp, P.rounds, P.d, rhs, nrhs, P.H, P.kc, P.y, P.rs, tri ? P.S : nullptr);
    count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  if (P.kc > 0 && !tri) {
    if (cusolverDnSetStream(h, st) != CUSOLVER_STATUS_SUCCESS) return CG_ERR_SOLVER;
    if (cusolverDnDpotrs(h, CUBLAS_FILL_MODE_LOWER, P.kc, nrhs, P.S, P.kc, P.rs, P.kc,
                         P.info + 2) != CUSOLVER_STATUS_SUCCESS) {
      set_last_error("cusolverDnDpotrs failed to launch", __FILE__, __LINE__);
      return CG_ERR_SOLVER;
    }
  }
  { peel_backward_kernel<<<1, kPeelThreads, 0, st>>>(A.val, pp, P.rounds, P.d, P.y, P.rs, nrhs,
                                                     P.H, P.kc, P.ke, x); count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

int peel_factor_solve(PeelFactor& P, const SpHess& A, cusolverDnHandle_t h, const double* rhs,
                      double* x, int nrhs, cudaStream_t st) {
  if (!P.ready) {
    set_last_error("peel factor: no plan for the current pattern", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  if (nrhs < 0 || nrhs > 2) return CG_ERR_INVALID_ARG;
  if (P.kc > kSmallCore) {
    CG_TRY(peel_factor(P, A, h, st));
    return nrhs > 0 ? peel_solve(P, A, h, rhs, x, nrhs, st) : CG_OK;
  }
  CG_TRY(ensure_small_smem());
  const PeelPtrs pp = ptrs_of(P);
  CG_TRY_CUDA(cudaMemsetAsync(P.info, 0, 3 * sizeof(int), st));
  { peel_fused_kernel<<<1, kPeelThreads, small_smem(P.kc), st>>>(
      A.val, pp, P.rounds, P.kc, P.ke, P.H, rhs, nrhs, x, P.d, P.y, P.S, P.info, P.W); count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

int peel_assemble_dense(const PeelFactor& P, const SpHess& A, double* S, int k, cudaStream_t st) {
  if (!P.ready || !P.contrib || P.rounds != 0 || P.kc != k) {
    set_last_error("dense Schur assembly: no matching contribution plan", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  const PeelPtrs pp = ptrs_of(P);
  const long long total = (long long)k * k;
  const int grid = (int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148 * 8));
  { peel_weights_kernel<<<std::max(1, std::min((P.ke + 255) / 256, 148 * 4)), 256, 0, st>>>(A.val, pp, nullptr, P.ke, P.W); count_launch(); }
  { dense_contrib_kernel<<<grid, 256, 0, st>>>(A.val, pp, P.W, k, S); count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // namespace cg
