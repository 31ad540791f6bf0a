// Fused plan pass (SPLR objective / gradient / line-search trial).
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

__device__ __forceinline__ double point_alpha(const TPassArgs& A, int i) {
  return A.trial ? fma(A.step, A.direc[i], A.gamma_prev[i]) : A.gamma[i];
}
__device__ __forceinline__ double point_beta(const TPassArgs& A, int j) {
  const int k = A.n + j;
  if (j == A.m - 1 && A.trial) return 0.0;
  return A.trial ? fma(A.step, A.direc[k], A.gamma_prev[k]) : A.gamma[k];
}

}  // namespace

template <typename TM>
__global__ void __launch_bounds__(kThreads, 3) tpass_kernel(const TPassArgs A) {
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

  // this lane's columns and their scaled beta
  double bs[NV * VN];
  bool cin[NV * VN];
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int k = 0; k < VN; ++k) {
      const int j = c0 + v * VS + lane * VN + k;
      cin[v * VN + k] = j < m;
      bs[v * VN + k] = (j < m) ? point_beta(A, j) * s2 : 0.0;
    }
  double cacc[NV * VN];
#pragma unroll
  for (int q = 0; q < NV * VN; ++q) cacc[q] = 0.0;

  for (int i = r0 + warp; i < r1; i += kWarps) {
    const double as = point_alpha(A, i) * s2;
    const TM* __restrict__ Mi = M + (size_t)i * m;
    double rsum = 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const int jb = c0 + v * VS + lane * VN;
      double mv[VN];
      if (vec_ok && jb + VN <= m) {
        Vec<TM>::load(Mi + jb, mv);
      } else {
#pragma unroll
        for (int k = 0; k < VN; ++k) mv[k] = (jb + k < m) ? ld1(Mi + jb + k) : 0.0;
      }
#pragma unroll
      for (int k = 0; k < VN; ++k) {
        const int q = v * VN + k;
        const double T = cin[q] ? exp2_f64(fma(-mv[k], s2, as + bs[q]), tab) : 0.0;
        rsum += T;
        cacc[q] += T;
      }
    }
    rsum = warp_sum_down(rsum);
    if (lane == 0) A.rowpart[(size_t)strip * n + i] = rsum;
  }
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int k = 0; k < VN; ++k) sm_col[warp][v * VS + lane * VN + k] = cacc[v * VN + k];
  __syncthreads();
  {
    const int c = threadIdx.x;
    const int j = c0 + c;
    if (j < m) {
      double s = 0.0;
      for (int w = 0; w < kWarps; ++w) s += sm_col[w][c];
      A.colpart[(size_t)split * m + j] = s;
    }
  }

  const unsigned int nfin = (unsigned)(A.splits + A.strips);
  unsigned int* cnt_split = A.counters;               // [splits]
  unsigned int* cnt_strip = A.counters + A.splits;    // [strips]
  unsigned int* cnt_all = A.counters + A.splits + A.strips;
  const int H = n + m - 1;
  bool final_role = false;

  // Row finisher: rows [r0, r1) of this split.
  if (elect_last(&cnt_split[split], (unsigned)A.strips)) {
    double s_r = 0, s_aa = 0, s_g2 = 0, s_gd = 0;
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      double r = 0.0;
      for (int s = 0; s < A.strips; ++s) r += ldcg(A.rowpart + (size_t)s * n + i);
      const double al = point_alpha(A, i);
      if (A.trial) A.gamma[i] = al;
      const double g = r - A.ab[i];
      A.rows[i] = r;
      A.grad[i] = g;
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
      double* o = A.scal + (size_t)split * kTScal;
      o[0] = s_r;
      o[1] = s_aa;
      o[2] = s_g2;
      o[3] = s_gd;
      o[4] = 0.0;
    }
    if (elect_last(cnt_all, nfin)) final_role = true;
  }
  // Column finisher: columns of this strip.
  if (elect_last(&cnt_strip[strip], (unsigned)A.splits)) {
    double s_bb = 0, s_g2 = 0, s_gd = 0, s_gl = 0;
    const int j = c0 + threadIdx.x;
    if (j < m) {
      double c = 0.0;
      for (int s = 0; s < A.splits; ++s) c += ldcg(A.colpart + (size_t)s * m + j);
      const double be = point_beta(A, j);
      if (A.trial) A.gamma[n + j] = be;
      A.cols[j] = c;
      s_bb = A.ab[n + j] * be;
      const double g = c - A.ab[n + j];
      if (j < m - 1) {
        A.grad[n + j] = g;
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
      double* o = A.scal + (size_t)(A.splits + strip) * kTScal;
      o[0] = 0.0;
      o[1] = s_bb;
      o[2] = s_g2;
      o[3] = s_gd;
      o[4] = s_gl;
    }
    if (elect_last(cnt_all, nfin)) final_role = true;
  }
  if (!final_role) return;
  if (threadIdx.x == 0) {
    double tsum = 0, dot = 0, g2 = 0, gd = 0, gl = 0;
    for (int q = 0; q < A.splits + A.strips; ++q) {
      const double* o = A.scal + (size_t)q * kTScal;
      tsum += ldcg(o);
      dot += ldcg(o + 1);
      g2 += ldcg(o + 2);
      gd += ldcg(o + 3);
      gl += ldcg(o + 4);
    }
    A.res->f = A.eta * tsum - dot;
    A.res->gnorm = sqrt(g2);
    A.res->dg = gd;
    A.res->tsum = tsum;
    A.res->gfull = sqrt(g2 + gl);
  }
  (void)H;
}

void tpass_geometry(int n, int m, int sm_count, int& strips, int& splits) {
  strips = (m + kTStrip - 1) / kTStrip;
  int s = (2 * sm_count + strips - 1) / strips;
  s = std::max(1, std::min(s, std::max(1, n / 64)));
  splits = s;
}

size_t tpass_workspace_doubles(int n, int m, int strips, int splits) {
  return (size_t)strips * n + (size_t)splits * m + (size_t)(splits + strips) * kTScal;
}

int launch_tpass(bool f32, const TPassArgs& a, cudaStream_t stream) {
  const int grid = a.strips * a.splits;
  if (f32)
    { tpass_kernel<float><<<grid, kThreads, 0, stream>>>(a); cg::count_launch(); }
  else
    { tpass_kernel<double><<<grid, kThreads, 0, stream>>>(a); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // namespace cg
