// Fused plan pass (SPLR objective / gradient / line-search trials).
//
// Replaces, in one kernel per evaluation (reference benben-cd/curegot_backward):
//   T_fused_kernel + obj_grad_kernel + launch_T_objfn_grad
//                                       src/sinkhorn_splr_kernel.cu:214-546
//   line_search_fused_kernel1/2/3 + launch_line_search_computation
//                                       src/sinkhorn_splr_kernel_line_search.cu:93-458
//
// One CTA = one tile of 256 columns x a range of rows.  Lanes own 8 columns
// (16-byte vectors), warps own rows: row sums come from one warp reduction
// per (row, strip) and column sums from registers merged across warps in
// shared memory.  Partials are merged by the last CTA of each row split and
// of each column strip (fixed order), and the last of those finishers
// assembles f, ||g|| and <g, d>: no host reduction, no double atomics, bitwise
// reproducible.  In trial mode the point gamma_prev + step * direc is formed
// on the fly (gamma_{n+m-1} = 0) and written out by the finishers.
// The exponent is evaluated in base 2 with the FP64 table-driven exp2_f64;
// overflow gives +inf and NaN propagates, as the reference's exp() does.
#include <algorithm>

#include "bcd.cuh"
#include "bulk.cuh"
#include "lse.cuh"
#include "tpass.cuh"

namespace cg {

namespace {

template <typename TM>
struct TLayout;
template <>
struct TLayout<double> {
  static constexpr int VN = 2, NV = 4;  // 4 x double2 per lane, stride 64 columns
};
template <>
struct TLayout<float> {
  static constexpr int VN = 4, NV = 2;  // 2 x float4 per lane, stride 128 columns
};

__device__ __forceinline__ double point_alpha(const TPassArgs& A, int i, double step) {
  return A.trial ? fma(step, A.direc[i], A.gamma_prev[i]) : A.gamma[i];
}
__device__ __forceinline__ double point_beta(const TPassArgs& A, int j, double step) {
  const int k = A.n + j;
  if (j == A.m - 1 && A.trial) return 0.0;
  return A.trial ? fma(step, A.direc[k], A.gamma_prev[k]) : A.gamma[k];
}

// Slot k's view of the outputs and workspace (see TPassArgs).
struct Slot {
  double *gamma, *rows, *cols, *grad, *rowpart, *colpart, *scal;
  TResult* res;
  double step;
};
__device__ __forceinline__ Slot slot_of(const TPassArgs& A, int k) {
  const size_t n = A.n, m = A.m;
  Slot o;
  o.gamma = A.gamma + k * (n + m);
  o.rows = A.rows + k * n;
  o.cols = A.cols + k * m;
  o.grad = A.grad + k * (n + m - 1);
  o.rowpart = A.rowpart + k * (size_t)A.strips * n;
  o.colpart = A.colpart + k * (size_t)A.splits * m;
  o.scal = A.scal + k * (size_t)(A.splits + A.strips) * kTScal;
  o.res = A.res + k;
  o.step = (k == 0) ? A.step : A.steps[k];
  return o;
}

}  // namespace

// K trial points per pass (K = 1: the plain pass).  Every element of M is
// loaded once; for each point k the exponent, the row / column sums and the
// finishers' reductions are exactly those of a one-point pass at step k, in
// the same order, so slot k is bitwise what a one-point pass would give.
template <typename TM, int K>
__global__ void __launch_bounds__(kThreads, 2) tpass_kernel(const TPassArgs A) {
  constexpr int VN = TLayout<TM>::VN, NV = TLayout<TM>::NV;
  constexpr int VS = 32 * VN;  // column stride between a lane's vectors
  __shared__ double tab[kExp2TableSize];
  __shared__ double sm_col[kWarps][kTStrip];
  __shared__ double red[kWarps];
  load_exp2_table(tab);
  __syncthreads();

  const int n = A.n, m = A.m;
  const int strip = blockIdx.x % A.strips;
  const int split = blockIdx.x / A.strips;
  const int rows_per = (n + A.splits - 1) / A.splits;
  const int r0 = split * rows_per, r1 = min(n, r0 + rows_per);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c0 = strip * kTStrip;
  const TM* __restrict__ M = static_cast<const TM*>(A.M);
  const double s2 = A.s2;
  const bool vec_ok = (m % VN) == 0 && (reinterpret_cast<uintptr_t>(M) % 16) == 0;
  double stp[K];
#pragma unroll
  for (int p = 0; p < K; ++p) stp[p] = (p == 0) ? A.step : A.steps[p];

  // this lane's columns and their scaled beta
  double bs[K][NV * VN];
  bool cin[NV * VN];
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int k = 0; k < VN; ++k) {
      const int j = c0 + v * VS + lane * VN + k;
      cin[v * VN + k] = j < m;
#pragma unroll
      for (int p = 0; p < K; ++p)
        bs[p][v * VN + k] = (j < m) ? point_beta(A, j, stp[p]) * s2 : 0.0;
    }
  double cacc[K][NV * VN];
#pragma unroll
  for (int p = 0; p < K; ++p)
#pragma unroll
    for (int q = 0; q < NV * VN; ++q) cacc[p][q] = 0.0;

  // L2 prefetch (lane 0, one bulk hint per row segment) of the warp's rows
  // pf steps ahead, when the segments are 16-byte aligned
  const int pf = vec_ok ? A.l2pf : 0;
  const uint32_t seg_bytes = (uint32_t)(min(kTStrip, m - c0) * (int)sizeof(TM));
  if (pf > 0 && lane == 0)
    for (int k = 1; k < pf; ++k) {
      const int ip = r0 + warp + k * kWarps;
      if (ip < r1) prefetch_l2_bulk(M + (size_t)ip * m + c0, seg_bytes);
    }
  // One row's contribution: T for this lane's columns and every point, the
  // row sums reduced over the warp, the column sums kept in registers.
  // full: every column of the strip exists (no per-column predicate).
  auto row_body = [&](int i, const double (&mv)[NV][VN], bool full) {
    double as[K], rsum[K];
#pragma unroll
    for (int p = 0; p < K; ++p) {
      as[p] = point_alpha(A, i, stp[p]) * s2;
      rsum[p] = 0.0;
    }
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int k = 0; k < VN; ++k) {
        const int q = v * VN + k;
#pragma unroll
        for (int p = 0; p < K; ++p) {
          const double e = exp2_f64_clamped(fma(-mv[v][k], s2, as[p] + bs[p][q]), tab);
          const double T = (full || cin[q]) ? e : 0.0;
          rsum[p] += T;
          cacc[p][q] += T;
        }
      }
#pragma unroll
    for (int p = 0; p < K; ++p) {
      const double r = warp_sum_down(rsum[p]);
      if (lane == 0) slot_of(A, p).rowpart[(size_t)strip * n + i] = r;
    }
  };
  if (vec_ok && c0 + kTStrip <= m) {
    // full strip, aligned vectors: the next row's vectors are loaded before
    // this row is processed (two rows of M in flight per warp)
    using RT = typename Raw<TM>::T;
    RT nxt[NV];
    auto load_row = [&](int i) {
      const TM* __restrict__ Mi = M + (size_t)i * m + c0 + lane * VN;
#pragma unroll
      for (int v = 0; v < NV; ++v) nxt[v] = Raw<TM>::load(Mi + v * VS);
    };
    int i = r0 + warp;
    if (i < r1) load_row(i);
    for (; i < r1; i += kWarps) {
      if (pf > 0 && lane == 0) {
        const int ip = i + pf * kWarps;
        if (ip < r1) prefetch_l2_bulk(M + (size_t)ip * m + c0, seg_bytes);
      }
      double mv[NV][VN];
#pragma unroll
      for (int v = 0; v < NV; ++v)
#pragma unroll
        for (int k = 0; k < VN; ++k) mv[v][k] = Raw<TM>::get(nxt[v], k);
      if (i + kWarps < r1) load_row(i + kWarps);
      row_body(i, mv, true);
    }
  } else {
    for (int i = r0 + warp; i < r1; i += kWarps) {
      const TM* __restrict__ Mi = M + (size_t)i * m;
      double mv[NV][VN];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const int jb = c0 + v * VS + lane * VN;
        if (vec_ok && jb + VN <= m) {
          Vec<TM>::load(Mi + jb, mv[v]);
        } else {
#pragma unroll
          for (int k = 0; k < VN; ++k) mv[v][k] = (jb + k < m) ? ld1(Mi + jb + k) : 0.0;
        }
      }
      row_body(i, mv, false);
    }
  }
#pragma unroll
  for (int p = 0; p < K; ++p) {
    if (p > 0) __syncthreads();  // sm_col reused
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int k = 0; k < VN; ++k) sm_col[warp][v * VS + lane * VN + k] = cacc[p][v * VN + k];
    __syncthreads();
    const int c = threadIdx.x;
    const int j = c0 + c;
    if (j < m) {
      double s = 0.0;
      for (int w = 0; w < kWarps; ++w) s += sm_col[w][c];
      slot_of(A, p).colpart[(size_t)split * m + j] = s;
    }
  }

  const unsigned int nfin = (unsigned)(A.splits + A.strips);
  unsigned int* cnt_split = A.counters;               // [splits]
  unsigned int* cnt_strip = A.counters + A.splits;    // [strips]
  unsigned int* cnt_all = A.counters + A.splits + A.strips;
  bool final_role = false;

  // Row finisher: rows [r0, r1) of this split, every slot.
  if (elect_last(&cnt_split[split], (unsigned)A.strips)) {
    for (int p = 0; p < K; ++p) {
      const Slot S = slot_of(A, p);
      double s_r = 0, s_aa = 0, s_g2 = 0, s_gd = 0;
      for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
        double r = 0.0;
        for (int s = 0; s < A.strips; ++s) r += ldcg(S.rowpart + (size_t)s * n + i);
        const double al = point_alpha(A, i, S.step);
        if (A.trial) S.gamma[i] = al;
        const double g = r - A.ab[i];
        S.rows[i] = r;
        S.grad[i] = g;
        s_r += r;
        s_aa += A.ab[i] * al;
        s_g2 += g * g;
        if (A.direc) s_gd += g * A.direc[i];
      }
      s_r = cta_sum(s_r, red);
      s_aa = cta_sum(s_aa, red);
      s_g2 = cta_sum(s_g2, red);
      s_gd = cta_sum(s_gd, red);
      if (threadIdx.x == 0) {
        double* o = S.scal + (size_t)split * kTScal;
        o[0] = s_r;
        o[1] = s_aa;
        o[2] = s_g2;
        o[3] = s_gd;
        o[4] = 0.0;
      }
    }
    if (elect_last(cnt_all, nfin)) final_role = true;
  }
  // Column finisher: columns of this strip, every slot.
  if (elect_last(&cnt_strip[strip], (unsigned)A.splits)) {
    for (int p = 0; p < K; ++p) {
      const Slot S = slot_of(A, p);
      double s_bb = 0, s_g2 = 0, s_gd = 0, s_gl = 0;
      const int j = c0 + threadIdx.x;
      if (j < m) {
        double c = 0.0;
        for (int s = 0; s < A.splits; ++s) c += ldcg(S.colpart + (size_t)s * m + j);
        const double be = point_beta(A, j, S.step);
        if (A.trial) S.gamma[n + j] = be;
        S.cols[j] = c;
        s_bb = A.ab[n + j] * be;
        const double g = c - A.ab[n + j];
        if (j < m - 1) {
          S.grad[n + j] = g;
          s_g2 = g * g;
          if (A.direc) s_gd = g * A.direc[n + j];
        } else {
          s_gl = g * g;  // the gauge column: outside g, inside the full marginal error
        }
      }
      s_bb = cta_sum(s_bb, red);
      s_g2 = cta_sum(s_g2, red);
      s_gd = cta_sum(s_gd, red);
      s_gl = cta_sum(s_gl, red);
      if (threadIdx.x == 0) {
        double* o = S.scal + (size_t)(A.splits + strip) * kTScal;
        o[0] = 0.0;
        o[1] = s_bb;
        o[2] = s_g2;
        o[3] = s_gd;
        o[4] = s_gl;
      }
    }
    if (elect_last(cnt_all, nfin)) final_role = true;
  }
  if (!final_role) return;
  if (threadIdx.x < K) {
    const Slot S = slot_of(A, threadIdx.x);
    double tsum = 0, dot = 0, g2 = 0, gd = 0, gl = 0;
    for (int q = 0; q < A.splits + A.strips; ++q) {
      const double* o = S.scal + (size_t)q * kTScal;
      tsum += ldcg(o);
      dot += ldcg(o + 1);
      g2 += ldcg(o + 2);
      gd += ldcg(o + 3);
      gl += ldcg(o + 4);
    }
    S.res->f = A.eta * tsum - dot;
    S.res->gnorm = sqrt(g2);
    S.res->dg = gd;
    S.res->tsum = tsum;
    S.res->gfull = sqrt(g2 + gl);
  }
}

// strips x splits CTAs, at most 2 per SM (the two-point trial kernel's
// occupancy): one full wave.  Rounding the split count up instead left a few
// CTAs for a second wave, which doubled the pass time (e.g. 16 strips x 19
// splits = 304 CTAs on 296 slots).
void tpass_geometry(int n, int m, int sm_count, int& strips, int& splits) {
  strips = (m + kTStrip - 1) / kTStrip;
  int s = (2 * sm_count) / strips;
  s = std::max(1, std::min(s, std::max(1, n / 64)));
  splits = s;
}

size_t tpass_workspace_doubles(int n, int m, int strips, int splits) {
  return (size_t)strips * n + (size_t)splits * m + (size_t)(splits + strips) * kTScal;
}

int launch_tpass(bool f32, const TPassArgs& a_in, cudaStream_t stream) {
  TPassArgs a = a_in;
  a.l2pf = bcd_l2_prefetch();
  const int grid = a.strips * a.splits;
  const bool multi = a.trial && a.nsteps > 1;
  if (f32 && multi)
    { tpass_kernel<float, 2><<<grid, kThreads, 0, stream>>>(a); cg::count_launch(); }
  else if (f32)
    { tpass_kernel<float, 1><<<grid, kThreads, 0, stream>>>(a); cg::count_launch(); }
  else if (multi)
    { tpass_kernel<double, 2><<<grid, kThreads, 0, stream>>>(a); cg::count_launch(); }
  else
    { tpass_kernel<double, 1><<<grid, kThreads, 0, stream>>>(a); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // namespace cg
