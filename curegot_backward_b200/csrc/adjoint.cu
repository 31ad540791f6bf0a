// Implicit backward of the entropic-OT plan: PCG on the reduced Hessian.
//
// Replaces (reference benben-cd/curegot_backward):
//   q_matvec / rhs_Q_scale / assemble_grad / pcg   curegot/_backward_core.py:31-83
//   solve_backward                                 curegot/backward.py:72-144
//
// Q(T) z = [ r * z_a + T_t z_b ;  T_t^T z_a + c_t * z_b ]  (r = T 1, c = T^T 1).
// The reference evaluates it with two GEMVs plus two full sums over T per PCG
// iteration and synchronises with the host every iteration.  Here:
//   * one RHS pass over (T, G) gives mu and caches r and c;
//   * every PCG iteration is ONE pass over T computing both T_t z_b (row
//     reductions) and T_t^T z_a (column reductions); the last CTA of that pass
//     performs the whole PCG vector update (dots, axpys, diagonal
//     preconditioner, convergence / breakdown test) on the device;
//   * the host queues iterations in chunks and reads a 64-byte state per chunk.
// Tiles, finishers and reduction orders follow the plan pass (tpass.cu):
// deterministic, no atomics on values.
#include <algorithm>
#include <cmath>
#include <vector>

#include "splr.cuh"
#include "tpass.cuh"
#include "workspace.cuh"

namespace cg {

int ctx_apply_full(cg_ctx_s* c, const double* r, double* z, cudaStream_t st);
int ctx_setup_diag(cg_ctx_s* c, cudaStream_t st);

namespace {

struct PcgState {
  int k, done, converged, breakdown;
  int max_iter, precond, allzero, pad;
  double rz, bnorm, tol, rnorm;
};

struct AdjArgs {
  const double* T;
  const double* G;
  int n, m;
  // vectors (H = n + m - 1 unless noted)
  double* rows;   // [n]  T 1
  double* cols;   // [m]  T^T 1
  double* x;      // lambda
  double* r;
  double* z;
  double* p;
  double* w;
  const double* inv_diag;  // null: no diagonal
  PcgState* st;
  // tiles
  int strips, splits;
  double* rowpart;  // [2 * strips * n]
  double* colpart;  // [2 * splits * m]
  double* scal;     // [(splits + strips) * 2]
  unsigned int* counters;
};

constexpr int VN = 2, NV = 4, VS = 64;  // 4 x double2 per lane, 256-column strips

// Final CTA: PCG vector work after w = Q p is complete.  Part 1 through the
// convergence test; part 2 (preconditioner, new direction) when fused.
__device__ void pcg_update(const AdjArgs& A, bool part2, double* red) {
  PcgState* st = A.st;
  const int H = A.n + A.m - 1;
  __shared__ double sh_alpha, sh_beta;
  __shared__ int sh_stop;
  double pw = 0.0;
  for (int k = threadIdx.x; k < H; k += blockDim.x) pw += A.p[k] * ldcg(A.w + k);
  pw = cta_sum(pw, red);
  if (threadIdx.x == 0) {
    sh_stop = 0;
    if (pw <= 0.0) {  // reference: raise on p^T A p <= 0
      st->breakdown = 1;
      st->done = 1;
      sh_stop = 1;
    } else {
      sh_alpha = st->rz / pw;
    }
  }
  __syncthreads();
  if (sh_stop) return;
  const double alpha = sh_alpha;
  double rn2 = 0.0;
  for (int k = threadIdx.x; k < H; k += blockDim.x) {
    A.x[k] += alpha * A.p[k];
    const double rv = A.r[k] - alpha * ldcg(A.w + k);
    A.r[k] = rv;
    rn2 += rv * rv;
  }
  rn2 = cta_sum(rn2, red);
  if (threadIdx.x == 0) {
    const double rnorm = sqrt(rn2);
    st->rnorm = rnorm;
    if (rnorm < st->tol * st->bnorm) {
      st->converged = 1;
      st->done = 1;
      st->k = st->k + 1;
      sh_stop = 1;
    }
  }
  __syncthreads();
  if (sh_stop || !part2) return;
  double rz = 0.0;
  for (int k = threadIdx.x; k < H; k += blockDim.x) {
    const double zv = A.inv_diag ? A.inv_diag[k] * A.r[k] : A.r[k];
    A.z[k] = zv;
    rz += A.r[k] * zv;
  }
  rz = cta_sum(rz, red);
  if (threadIdx.x == 0) {
    sh_beta = rz / st->rz;
    st->rz = rz;
  }
  __syncthreads();
  const double beta = sh_beta;
  for (int k = threadIdx.x; k < H; k += blockDim.x) A.p[k] = A.z[k] + beta * A.p[k];
  if (threadIdx.x == 0) {
    st->k = st->k + 1;
    if (st->k >= st->max_iter) st->done = 1;
  }
}

// mode 0: RHS pass (row/col sums of T and of G*T, then PCG init)
// mode 1: Q p pass (then the PCG update)
// cta: this CTA's index within the problem's tile grid.
template <int MODE>
__device__ __forceinline__ void adj_pass_body(const AdjArgs& A, int fused, int cta) {
  __shared__ double sm_col[2][kWarps][kTStrip];
  __shared__ double red[kWarps];
  const int n = A.n, m = A.m;
  if (MODE == 1 && ldcg(&A.st->done)) return;
  const int strip = cta % A.strips;
  const int split = cta / A.strips;
  const int rows_per = (n + A.splits - 1) / A.splits;
  const int r0 = split * rows_per, r1 = min(n, r0 + rows_per);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c0 = strip * kTStrip;
  const bool vec_ok = (m % VN) == 0 && (reinterpret_cast<uintptr_t>(A.T) % 16) == 0 &&
                      (MODE == 1 || (reinterpret_cast<uintptr_t>(A.G) % 16) == 0);
  // per-lane column data
  double pb[NV * VN];
  bool cin[NV * VN];
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int k = 0; k < VN; ++k) {
      const int j = c0 + v * VS + lane * VN + k;
      cin[v * VN + k] = j < m;
      pb[v * VN + k] = (MODE == 1 && j < m - 1) ? A.p[n + j] : 0.0;
    }
  double ca0[NV * VN], ca1[NV * VN];
#pragma unroll
  for (int q = 0; q < NV * VN; ++q) ca0[q] = ca1[q] = 0.0;

  for (int i = r0 + warp; i < r1; i += kWarps) {
    const double* Ti = A.T + (size_t)i * m;
    const double* Gi = (MODE == 0) ? A.G + (size_t)i * m : nullptr;
    const double pa = (MODE == 1) ? A.p[i] : 0.0;
    double rs0 = 0.0, rs1 = 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const int jb = c0 + v * VS + lane * VN;
      double tv[VN], gv[VN];
      if (vec_ok && jb + VN <= m) {
        Vec<double>::load(Ti + jb, tv);
        if (MODE == 0) Vec<double>::load(Gi + jb, gv);
      } else {
#pragma unroll
        for (int k = 0; k < VN; ++k) {
          tv[k] = (jb + k < m) ? Ti[jb + k] : 0.0;
          if (MODE == 0) gv[k] = (jb + k < m) ? Gi[jb + k] : 0.0;
        }
      }
#pragma unroll
      for (int k = 0; k < VN; ++k) {
        const int q = v * VN + k;
        if (!cin[q]) continue;
        if (MODE == 0) {
          const double gt = gv[k] * tv[k];
          rs0 += tv[k];
          rs1 += gt;
          ca0[q] += tv[k];
          ca1[q] += gt;
        } else {
          rs1 += tv[k] * pb[q];
          ca1[q] += tv[k] * pa;
        }
      }
    }
    if (MODE == 0) rs0 = warp_sum_down(rs0);
    rs1 = warp_sum_down(rs1);
    if (lane == 0) {
      if (MODE == 0) A.rowpart[(size_t)strip * n + i] = rs0;
      A.rowpart[(size_t)(A.strips + strip) * n + i] = rs1;
    }
  }
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int k = 0; k < VN; ++k) {
      sm_col[0][warp][v * VS + lane * VN + k] = ca0[v * VN + k];
      sm_col[1][warp][v * VS + lane * VN + k] = ca1[v * VN + k];
    }
  __syncthreads();
  {
    const int c = threadIdx.x, j = c0 + c;
    if (j < m) {
      double s0 = 0.0, s1 = 0.0;
      for (int w = 0; w < kWarps; ++w) {
        s0 += sm_col[0][w][c];
        s1 += sm_col[1][w][c];
      }
      if (MODE == 0) A.colpart[(size_t)split * m + j] = s0;
      A.colpart[(size_t)(A.splits + split) * m + j] = s1;
    }
  }
  const unsigned int nfin = (unsigned)(A.splits + A.strips);
  unsigned int* cnt_split = A.counters;
  unsigned int* cnt_strip = A.counters + A.splits;
  unsigned int* cnt_all = A.counters + A.splits + A.strips;
  bool final_role = false;
  if (elect_last(&cnt_split[split], (unsigned)A.strips)) {
    double b2 = 0.0, nz = 0.0;
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      double s1 = 0.0;
      for (int s = 0; s < A.strips; ++s) s1 += ldcg(A.rowpart + (size_t)(A.strips + s) * n + i);
      if (MODE == 0) {
        double s0 = 0.0;
        for (int s = 0; s < A.strips; ++s) s0 += ldcg(A.rowpart + (size_t)s * n + i);
        A.rows[i] = s0;
        A.r[i] = s1;  // mu_a
        b2 += s1 * s1;
        nz += (s1 != 0.0);
      } else {
        A.w[i] = A.rows[i] * A.p[i] + s1;
      }
    }
    if (MODE == 0) {
      b2 = cta_sum(b2, red);
      nz = cta_sum(nz, red);
      if (threadIdx.x == 0) {
        A.scal[(size_t)split * 2] = b2;
        A.scal[(size_t)split * 2 + 1] = nz;
      }
    }
    if (elect_last(cnt_all, nfin)) final_role = true;
  }
  if (elect_last(&cnt_strip[strip], (unsigned)A.splits)) {
    double b2 = 0.0, nz = 0.0;
    const int j = c0 + threadIdx.x;
    if (j < m) {
      double s1 = 0.0;
      for (int s = 0; s < A.splits; ++s) s1 += ldcg(A.colpart + (size_t)(A.splits + s) * m + j);
      if (MODE == 0) {
        double s0 = 0.0;
        for (int s = 0; s < A.splits; ++s) s0 += ldcg(A.colpart + (size_t)s * m + j);
        A.cols[j] = s0;
        if (j < m - 1) {
          A.r[n + j] = s1;  // mu_b
          b2 = s1 * s1;
          nz = (s1 != 0.0);
        }
      } else if (j < m - 1) {
        A.w[n + j] = s1 + A.cols[j] * A.p[n + j];
      }
    }
    if (MODE == 0) {
      b2 = cta_sum(b2, red);
      nz = cta_sum(nz, red);
      if (threadIdx.x == 0) {
        A.scal[(size_t)(A.splits + strip) * 2] = b2;
        A.scal[(size_t)(A.splits + strip) * 2 + 1] = nz;
      }
    }
    if (elect_last(cnt_all, nfin)) final_role = true;
  }
  if (!final_role) return;
  if (MODE == 1) {
    pcg_update(A, fused != 0, red);
    return;
  }
  // RHS finalize + PCG init: x = 0, r = mu, z = P(r), p = z, rz = r.z
  __shared__ int sh_zero;
  __shared__ double sh_b2;
  if (threadIdx.x == 0) {
    double b2 = 0.0, nz = 0.0;
    for (int q = 0; q < A.splits + A.strips; ++q) {
      b2 += ldcg(A.scal + (size_t)q * 2);
      nz += ldcg(A.scal + (size_t)q * 2 + 1);
    }
    sh_zero = (nz == 0.0);
    sh_b2 = b2;
  }
  __syncthreads();
  const int H = n + m - 1;
  double rz = 0.0;
  for (int k = threadIdx.x; k < H; k += blockDim.x) {
    const double rv = ldcg(A.r + k);
    A.x[k] = 0.0;
    const double zv = A.inv_diag ? A.inv_diag[k] * rv : rv;
    A.z[k] = zv;
    A.p[k] = zv;
    rz += rv * zv;
  }
  rz = cta_sum(rz, red);
  if (threadIdx.x == 0) {
    PcgState* st = A.st;
    st->k = 0;
    st->converged = sh_zero;
    st->breakdown = 0;
    st->allzero = sh_zero;
    st->done = sh_zero;
    st->bnorm = sqrt(sh_b2);
    st->rz = rz;
    st->rnorm = st->bnorm;
  }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, 3) adj_pass_kernel(const AdjArgs A, int fused) {
  adj_pass_body<MODE>(A, fused, (int)blockIdx.x);
}

// B problems of one shape in one launch: CTAs [b * per, (b + 1) * per) are
// problem b's tile grid.  Each problem's arithmetic is adj_pass_kernel's.
template <int MODE>
__global__ void __launch_bounds__(kThreads, 3) adj_pass_batch_kernel(const AdjArgs* __restrict__ probs,
                                                                     int per, int fused) {
  const int b = blockIdx.x / per;
  adj_pass_body<MODE>(probs[b], fused, (int)blockIdx.x - b * per);
}

// Second half of a PCG step when the preconditioner runs outside the pass.
__global__ void __launch_bounds__(1024) pcg_update2_kernel(double* r, double* z, double* p,
                                                           int H, PcgState* st) {
  __shared__ double red[32];
  __shared__ double sh_beta;
  if (ldcg(&st->done)) return;
  double rz = 0.0;
  for (int k = threadIdx.x; k < H; k += blockDim.x) rz += r[k] * z[k];
  rz = warp_sum_down(rz);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = rz;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    sh_beta = t / st->rz;
    st->rz = t;
  }
  __syncthreads();
  const double beta = sh_beta;
  for (int k = threadIdx.x; k < H; k += blockDim.x) p[k] = z[k] + beta * p[k];
  if (threadIdx.x == 0) {
    st->k = st->k + 1;
    if (st->k >= st->max_iter) st->done = 1;
  }
}

// SPLR-preconditioned start: p = z = B^{-1} r (z computed outside), rz = r.z
__global__ void __launch_bounds__(1024) pcg_splr_init_kernel(const double* r, const double* z,
                                                             double* p, int H, PcgState* st) {
  __shared__ double red[32];
  double rz = 0.0;
  for (int k = threadIdx.x; k < H; k += blockDim.x) {
    p[k] = z[k];
    rz += r[k] * z[k];
  }
  rz = warp_sum_down(rz);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = rz;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    st->rz = t;
  }
}

// dL/dM = T * (lambda_a + lambda_b - G) / eta, lambda_b[m-1] = 0
__global__ void assemble_grad_kernel(const double* __restrict__ T, const double* __restrict__ G,
                                     const double* __restrict__ lam, int n, int m, double inv_eta,
                                     double* __restrict__ grad) {
  const size_t total = (size_t)n * m;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(q / m);
    const int j = (int)(q - (size_t)i * m);
    const double lb = (j < m - 1) ? lam[n + j] : 0.0;
    grad[q] = (T[q] * (lam[i] + lb - G[q])) * inv_eta;
  }
}

__global__ void pcg_state_init(PcgState* st, int max_iter, int precond, double tol, int count) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < count; b += gridDim.x * blockDim.x) {
    st[b].k = 0;
    st[b].done = 0;
    st[b].converged = 0;
    st[b].breakdown = 0;
    st[b].max_iter = max_iter;
    st[b].precond = precond;
    st[b].allzero = 0;
    st[b].tol = tol;
  }
}

// dL/dM of B problems (T, G, grad: [B, n, m]; lam: [B, n + m - 1]).
__global__ void assemble_grad_batch_kernel(const double* __restrict__ T,
                                           const double* __restrict__ G,
                                           const double* __restrict__ lam, int B, int n, int m,
                                           double inv_eta, double* __restrict__ grad) {
  const size_t nm = (size_t)n * m, total = nm * B;
  const int H = n + m - 1;
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (size_t)gridDim.x * blockDim.x) {
    const size_t b = q / nm, e = q - b * nm;
    const int i = (int)(e / m);
    const int j = (int)(e - (size_t)i * m);
    const double* lb_ = lam + b * H;
    const double lb = (j < m - 1) ? lb_[n + j] : 0.0;
    grad[q] = (T[q] * (lb_[i] + lb - G[q])) * inv_eta;
  }
}

}  // namespace

int backward_solve(const double* T, const double* G, cg_ctx_s* ctx, double eta, int precond,
                   double tol, int max_iter, int n, int m, double* lambda, double* grad,
                   int* iterations, int* converged, cudaStream_t st) {
  if (!T || !G || !lambda || n <= 0 || m <= 0 || !(eta > 0.0) || max_iter <= 0) {
    set_last_error("cg_backward: invalid argument", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  const int H = n + m - 1;
  if (precond != CG_PRECOND_NONE) {
    if (!ctx || !ctx->valid) {
      set_last_error("cg_backward: preconditioner needs a valid backward context", __FILE__,
                     __LINE__);
      return CG_ERR_INVALID_CONTEXT;
    }
    if (ctx->H != H) {
      set_last_error("cg_backward: context dimension mismatch", __FILE__, __LINE__);
      return CG_ERR_INVALID_ARG;
    }
    if (precond == CG_PRECOND_DIAG) CG_TRY(ctx_setup_diag(ctx, st));
  }
  const int sms = sm_count_current();
  int strips = 1, splits = 1;
  tpass_geometry(n, m, sms, strips, splits);
  Workspace ws(st);
  const size_t o_rows = ws.reserve<double>(n), o_cols = ws.reserve<double>(m);
  const size_t o_r = ws.reserve<double>(H), o_z = ws.reserve<double>(H);
  const size_t o_p = ws.reserve<double>(H), o_w = ws.reserve<double>(H);
  const size_t o_rp = ws.reserve<double>(2 * (size_t)strips * n);
  const size_t o_cp = ws.reserve<double>(2 * (size_t)splits * m);
  const size_t o_sc = ws.reserve<double>(2 * (size_t)(splits + strips));
  const size_t o_cnt = ws.reserve<unsigned int>(splits + strips + 1);
  const size_t o_st = ws.reserve<PcgState>(1);
  CG_TRY(ws.allocate());
  AdjArgs A{};
  A.T = T;
  A.G = G;
  A.n = n;
  A.m = m;
  A.rows = ws.at<double>(o_rows);
  A.cols = ws.at<double>(o_cols);
  A.x = lambda;
  A.r = ws.at<double>(o_r);
  A.z = ws.at<double>(o_z);
  A.p = ws.at<double>(o_p);
  A.w = ws.at<double>(o_w);
  A.inv_diag = (precond == CG_PRECOND_DIAG) ? ctx->inv_diag : nullptr;
  A.st = ws.at<PcgState>(o_st);
  A.strips = strips;
  A.splits = splits;
  A.rowpart = ws.at<double>(o_rp);
  A.colpart = ws.at<double>(o_cp);
  A.scal = ws.at<double>(o_sc);
  A.counters = ws.at<unsigned int>(o_cnt);
  CG_TRY_CUDA(cudaMemsetAsync(A.counters, 0, (splits + strips + 1) * sizeof(unsigned int), st));
  { pcg_state_init<<<1, 32, 0, st>>>(A.st, max_iter, precond, tol, 1); cg::count_launch(); }
  const int grid = strips * splits;
  const bool splr = (precond == CG_PRECOND_SPLR);
  if (splr) {
    // RHS pass without preconditioner; then z = B^{-1} r, p = z, rz = r.z
    AdjArgs A0 = A;
    A0.inv_diag = nullptr;
    { adj_pass_kernel<0><<<grid, kThreads, 0, st>>>(A0, 0); cg::count_launch(); }
  } else {
    { adj_pass_kernel<0><<<grid, kThreads, 0, st>>>(A, 0); cg::count_launch(); }
  }
  CG_TRY_CUDA(cudaGetLastError());
  PcgState hs{};
  CG_TRY(read_device(&hs, A.st, sizeof(PcgState), st));
  if (!hs.allzero && splr) {
    // z = B^{-1} r, p = z, rz = r.z
    CG_TRY(ctx_apply_full(ctx, A.r, A.z, st));
    { pcg_splr_init_kernel<<<1, 1024, 0, st>>>(A.r, A.z, A.p, H, A.st); cg::count_launch(); }
    CG_TRY_CUDA(cudaGetLastError());
  }
  if (!hs.allzero) {
    int chunk = 4;
    while (!hs.done) {
      for (int c = 0; c < chunk; ++c) {
        { adj_pass_kernel<1><<<grid, kThreads, 0, st>>>(A, splr ? 0 : 1); cg::count_launch(); }
        if (splr) {
          CG_TRY(ctx_apply_full(ctx, A.r, A.z, st));
          { pcg_update2_kernel<<<1, 1024, 0, st>>>(A.r, A.z, A.p, H, A.st); cg::count_launch(); }
        }
      }
      CG_TRY_CUDA(cudaGetLastError());
      CG_TRY(read_device(&hs, A.st, sizeof(PcgState), st));
      chunk = std::min(chunk * 2, 64);
    }
  }
  if (iterations) *iterations = hs.allzero ? 0 : (hs.converged ? hs.k : max_iter);
  if (converged) *converged = hs.converged;
  if (grad) {
    const size_t total = (size_t)n * m;
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((total + 255) / 256, sms * 16));
    { assemble_grad_kernel<<<blocks, 256, 0, st>>>(T, G, lambda, n, m, 1.0 / eta, grad); cg::count_launch(); }
    CG_TRY_CUDA(cudaGetLastError());
  }
  ws.release();
  if (hs.breakdown) {
    set_last_error("PCG breakdown: p^T A p <= 0 (matrix not SPD?)", __FILE__, __LINE__);
    return CG_ERR_NOT_SPD;
  }
  return CG_OK;
}

// B problems of one shape with the diagonal preconditioner (or none): every
// PCG iteration of all unfinished problems is one launch, and the host reads
// the B states once per chunk of iterations.  Per problem, the values are
// those of backward_solve.
int backward_solve_batch(const double* T, const double* G, cg_ctx_s* const* ctxs, double eta,
                         int precond, double tol, int max_iter, int B, int n, int m,
                         double* lambda, double* grad, int* iterations, int* converged,
                         cudaStream_t st) {
  if (!T || !G || !lambda || B <= 0 || n <= 0 || m <= 0 || !(eta > 0.0) || max_iter <= 0 ||
      (precond != CG_PRECOND_NONE && precond != CG_PRECOND_DIAG)) {
    set_last_error("cg_backward_batch: invalid argument (precond must be NONE or DIAG)", __FILE__,
                   __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  const int H = n + m - 1;
  if (precond == CG_PRECOND_DIAG) {
    if (!ctxs) {
      set_last_error("cg_backward_batch: DIAG needs one backward context per problem", __FILE__,
                     __LINE__);
      return CG_ERR_INVALID_CONTEXT;
    }
    for (int b = 0; b < B; ++b) {
      cg_ctx_s* c = ctxs[b];
      if (!c || !c->valid) {
        set_last_error("cg_backward_batch: invalid backward context", __FILE__, __LINE__);
        return CG_ERR_INVALID_CONTEXT;
      }
      if (c->H != H) {
        set_last_error("cg_backward_batch: context dimension mismatch", __FILE__, __LINE__);
        return CG_ERR_INVALID_ARG;
      }
      CG_TRY(ctx_setup_diag(c, st));
    }
  }
  const int sms = sm_count_current();
  int strips = 1, splits = 1;
  tpass_geometry(n, m, sms, strips, splits);
  const int per = strips * splits;
  const size_t nc = (size_t)splits + strips + 1;
  Workspace ws(st);
  const size_t o_rows = ws.reserve<double>((size_t)B * n), o_cols = ws.reserve<double>((size_t)B * m);
  const size_t o_r = ws.reserve<double>((size_t)B * H), o_z = ws.reserve<double>((size_t)B * H);
  const size_t o_p = ws.reserve<double>((size_t)B * H), o_w = ws.reserve<double>((size_t)B * H);
  const size_t o_rp = ws.reserve<double>((size_t)B * 2 * strips * n);
  const size_t o_cp = ws.reserve<double>((size_t)B * 2 * splits * m);
  const size_t o_sc = ws.reserve<double>((size_t)B * 2 * (splits + strips));
  const size_t o_cnt = ws.reserve<unsigned int>((size_t)B * nc);
  const size_t o_st = ws.reserve<PcgState>(B);
  const size_t o_args = ws.reserve<AdjArgs>(B);
  CG_TRY(ws.allocate());
  std::vector<AdjArgs> hA(B);
  PcgState* dst = ws.at<PcgState>(o_st);
  for (int b = 0; b < B; ++b) {
    AdjArgs& A = hA[b];
    A = AdjArgs{};
    A.T = T + (size_t)b * n * m;
    A.G = G + (size_t)b * n * m;
    A.n = n;
    A.m = m;
    A.rows = ws.at<double>(o_rows) + (size_t)b * n;
    A.cols = ws.at<double>(o_cols) + (size_t)b * m;
    A.x = lambda + (size_t)b * H;
    A.r = ws.at<double>(o_r) + (size_t)b * H;
    A.z = ws.at<double>(o_z) + (size_t)b * H;
    A.p = ws.at<double>(o_p) + (size_t)b * H;
    A.w = ws.at<double>(o_w) + (size_t)b * H;
    A.inv_diag = (precond == CG_PRECOND_DIAG) ? ctxs[b]->inv_diag : nullptr;
    A.st = dst + b;
    A.strips = strips;
    A.splits = splits;
    A.rowpart = ws.at<double>(o_rp) + (size_t)b * 2 * strips * n;
    A.colpart = ws.at<double>(o_cp) + (size_t)b * 2 * splits * m;
    A.scal = ws.at<double>(o_sc) + (size_t)b * 2 * (splits + strips);
    A.counters = ws.at<unsigned int>(o_cnt) + (size_t)b * nc;
  }
  AdjArgs* dA = ws.at<AdjArgs>(o_args);
  CG_TRY_CUDA(cudaMemcpyAsync(dA, hA.data(), B * sizeof(AdjArgs), cudaMemcpyHostToDevice, st));
  CG_TRY_CUDA(cudaMemsetAsync(ws.at<unsigned int>(o_cnt), 0, B * nc * sizeof(unsigned int), st));
  { pcg_state_init<<<std::max(1, (B + 127) / 128), 128, 0, st>>>(dst, max_iter, precond, tol, B); cg::count_launch(); }
  { adj_pass_batch_kernel<0><<<B * per, kThreads, 0, st>>>(dA, per, 0); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  std::vector<PcgState> hs(B);
  auto all_done = [&]() {
    for (const PcgState& x : hs)
      if (!x.done) return false;
    return true;
  };
  // B states are read through a pinned bounce buffer in pieces of 4 KB
  auto read_states = [&]() -> int {
    const int per_read = (int)(4096 / sizeof(PcgState));
    for (int b0 = 0; b0 < B; b0 += per_read) {
      const int cnt = std::min(per_read, B - b0);
      CG_TRY(read_device(hs.data() + b0, dst + b0, cnt * sizeof(PcgState), st));
    }
    return CG_OK;
  };
  CG_TRY(read_states());
  int chunk = 4;
  while (!all_done()) {
    for (int c = 0; c < chunk; ++c)
      { adj_pass_batch_kernel<1><<<B * per, kThreads, 0, st>>>(dA, per, 1); cg::count_launch(); }
    CG_TRY_CUDA(cudaGetLastError());
    CG_TRY(read_states());
    chunk = std::min(chunk * 2, 64);
  }
  int broke = -1;
  for (int b = 0; b < B; ++b) {
    if (iterations) iterations[b] = hs[b].allzero ? 0 : (hs[b].converged ? hs[b].k : max_iter);
    if (converged) converged[b] = hs[b].converged;
    if (hs[b].breakdown && broke < 0) broke = b;
  }
  if (grad) {
    const size_t total = (size_t)B * n * m;
    const int blocks = (int)std::max<size_t>(1, std::min<size_t>((total + 255) / 256, sms * 16));
    { assemble_grad_batch_kernel<<<blocks, 256, 0, st>>>(T, G, lambda, B, n, m, 1.0 / eta, grad); cg::count_launch(); }
    CG_TRY_CUDA(cudaGetLastError());
  }
  ws.release();
  if (broke >= 0) {
    set_last_error("PCG breakdown: p^T A p <= 0 (matrix not SPD?) in a problem of the batch",
                   __FILE__, __LINE__);
    return CG_ERR_NOT_SPD;
  }
  return CG_OK;
}

}  // namespace cg

extern "C" int cg_backward_batch_f64(const double* T, const double* G, cg_ctx* const* ctxs,
                                     double eta, int precond, double tol, int max_iter, int B,
                                     int n, int m, double* lambda, double* grad, int* iterations,
                                     int* converged, cudaStream_t stream) {
  return cg::backward_solve_batch(T, G, reinterpret_cast<cg_ctx_s* const*>(ctxs), eta, precond,
                                  tol, max_iter, B, n, m, lambda, grad, iterations, converged,
                                  stream);
}

extern "C" int cg_backward_f64(const double* T, const double* G, cg_ctx* ctx, double eta,
                               int precond, double tol, int max_iter, int n, int m,
                               double* lambda, double* grad, int* iterations, int* converged,
                               cudaStream_t stream) {
  return cg::backward_solve(T, G, reinterpret_cast<cg_ctx_s*>(ctx), eta, precond, tol, max_iter,
                            n, m, lambda, grad, iterations, converged, stream);
}
