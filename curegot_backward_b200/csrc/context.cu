// C ABI: SPLR solver entry points, backward-context operations and the
// reference's test hooks.
//
// Context semantics follow SPLRBackwardContext (reference
// benben-cd/curegot_backward src/backward_context.{h,cu}):
//   apply_preconditioner           backward_context.cu:543-581
//   setup / apply diagonal         backward_context.cu:591-655
//   adopt / fallback export        sinkhorn_splr.cu:1566-1601
#include <climits>
#include <cstring>

#include "splr.cuh"
#include "tpass.cuh"
#include "workspace.cuh"

namespace cg {

namespace {

__global__ void scale_kernel(const double* inv, const double* r, double* z, int H) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < H; k += gridDim.x * blockDim.x)
    z[k] = inv[k] * r[k];
}

__global__ void inv_diag_ctx_kernel(const double* val, const int* rowptr, int n, int H,
                                    double* inv, int* err) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < H; r += gridDim.x * blockDim.x) {
    const double v = (r < n) ? val[r] : val[rowptr[r + 1] - 1];
    if (!(v > 0.0) || !isfinite(v)) {
      atomicMin(err, r);
      inv[r] = 0.0;
    } else {
      inv[r] = 1.0 / v;
    }
  }
}

// Woodbury correction without the -reg scaling (context apply).
__global__ void __launch_bounds__(1024) ctx_woodbury_kernel(double* x, const double* u,
                                                            const double* r, const double* y,
                                                            const double* s, int H, double reg,
                                                            double ys) {
  __shared__ double sh[32];
  auto bsum = [&](double v) {
    v = warp_sum_down(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double q = 0.0;
    if (threadIdx.x < 32) q = warp_sum_down(sh[threadIdx.x]);
    __syncthreads();
    if (threadIdx.x == 0) sh[0] = q;
    __syncthreads();
    const double out = sh[0];
    __syncthreads();
    return out;
  };
  double sg = 0, yu = 0, yx = 0;
  for (int k = threadIdx.x; k < H; k += blockDim.x) {
    sg += s[k] * r[k];
    yu += y[k] * u[k];
    yx += y[k] * x[k];
  }
  sg = bsum(sg);
  yu = bsum(yu);
  yx = bsum(yx);
  const double sg_ys = sg / ys;
  const double term1 = (1.0 / reg + yu / ys) * sg_ys - yx / ys;
  for (int k = threadIdx.x; k < H; k += blockDim.x) x[k] += (term1 * s[k] - sg_ys * u[k]);
}

__global__ void t_values_kernel(const double* alpha, const double* beta, const double* M, int n,
                                int m, double inv_reg, double* tv, int* ti) {
  const long long Te = (long long)n * (m - 1);
  const int H = n + m - 1;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < Te;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / (m - 1));
    const int j = (int)(q - (long long)i * (m - 1));
    tv[q] = exp((alpha[i] + beta[j] - M[(size_t)i * m + j]) * inv_reg);
    ti[q] = (n + j) * H + i;
  }
}

__global__ void densify_lower_kernel(const double* val, const int* col, const int* rowptr, int n,
                                     double* S) {
  for (int r = blockIdx.x; r < n; r += gridDim.x)
    for (int q = rowptr[r] + threadIdx.x; q < rowptr[r + 1]; q += blockDim.x) {
      const int c = col[q];
      if (c <= r) {
        S[(size_t)r * n + c] = val[q];
        S[(size_t)c * n + r] = val[q];
      }
    }
}

}  // namespace

int ctx_apply_full(cg_ctx_s* c, const double* r, double* z, cudaStream_t st) {
  if (c->path == 1) {
    CG_TRY(spchol_solve(*c->sc, r, c->xtmp, 1, st));
  } else {
    cusolverDnHandle_t h = nullptr;
    CG_TRY(solver_handle(&h));
    if (c->path == 2) CG_TRY(peel_solve(*c->pf, c->A, h, r, c->xtmp, 1, st));
    else CG_TRY(schur_solve(h, c->A, c->F, r, c->xtmp, 1, c->tmp, st));
  }
  if (c->low_rank)
    { ctx_woodbury_kernel<<<1, 1024, 0, st>>>(c->xtmp, c->u, r, c->y, c->s, c->H, c->reg, c->ys); cg::count_launch(); }
  CG_TRY_CUDA(cudaMemcpyAsync(z, c->xtmp, c->H * sizeof(double), cudaMemcpyDeviceToDevice, st));
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

int ctx_setup_diag(cg_ctx_s* c, cudaStream_t st) {
  if (c->diag_ready) return CG_OK;
  const int init = INT_MAX;
  CG_TRY_CUDA(cudaMemcpyAsync(c->err, &init, sizeof(int), cudaMemcpyHostToDevice, st));
  { inv_diag_ctx_kernel<<<std::max(1, std::min((c->H + 255) / 256, 1024)), 256, 0, st>>>(
      c->A.val, c->A.rowptr, c->n, c->H, c->inv_diag, c->err); cg::count_launch(); }
  int bad = INT_MAX;
  CG_TRY_CUDA(cudaMemcpyAsync(&bad, c->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CG_TRY_CUDA(cudaStreamSynchronize(st));
  if (bad != INT_MAX) {
    set_last_error("backward context: CSR diagonal missing, non-positive or non-finite",
                   __FILE__, __LINE__);
    return CG_ERR_NONFINITE;
  }
  c->diag_ready = true;
  return CG_OK;
}

}  // namespace cg

extern "C" {

static int splr_entry(bool f32, const void* M, const double* a, const double* b, double* P,
                      double reg, int max_iter, double tol, int n, int m, int* niter,
                      double density_max, double shift_max, int cycle, int cand_iter,
                      int verbose, const double* x0, double* dual, cg_ctx** ctx_out,
                      int* converged, double* trace, cudaStream_t stream) {
  // FP64: the reference's stopping test (parity).  Mixed precision (an
  // addition of this library): the full marginal error, gauge column included.
  cg::SplrParams prm{reg, tol, max_iter, density_max, shift_max, cycle, cand_iter, verbose,
                     f32 ? 1 : 0};
  cg_ctx_s* c = nullptr;
  int rc;
  if (f32)
    rc = cg::splr_solve<float>(static_cast<const float*>(M), a, b, P, n, m, prm, x0, dual, niter,
                               converged, ctx_out ? &c : nullptr, trace, stream);
  else
    rc = cg::splr_solve<double>(static_cast<const double*>(M), a, b, P, n, m, prm, x0, dual,
                                niter, converged, ctx_out ? &c : nullptr, trace, stream);
  if (ctx_out) *ctx_out = reinterpret_cast<cg_ctx*>(c);
  return rc;
}

int cg_splr_f64(const double* M, const double* a, const double* b, double* P, double reg,
                int max_iter, double tol, int n, int m, int* niter, double density_max,
                double shift_max, int sparsity_pattern_cycle, int candidate_sinkhorn_iter,
                int verbose, const double* x0, double* dual, cg_ctx** ctx_out, int* converged,
                double* trace, cudaStream_t stream) {
  return splr_entry(false, M, a, b, P, reg, max_iter, tol, n, m, niter, density_max, shift_max,
                    sparsity_pattern_cycle, candidate_sinkhorn_iter, verbose, x0, dual, ctx_out,
                    converged, trace, stream);
}

int cg_splr_mixed(const float* M, const double* a, const double* b, double* P, double reg,
                  int max_iter, double tol, int n, int m, int* niter, double density_max,
                  double shift_max, int sparsity_pattern_cycle, int candidate_sinkhorn_iter,
                  int verbose, const double* x0, double* dual, cg_ctx** ctx_out,
                  int* converged, double* trace, cudaStream_t stream) {
  return splr_entry(true, M, a, b, P, reg, max_iter, tol, n, m, niter, density_max, shift_max,
                    sparsity_pattern_cycle, candidate_sinkhorn_iter, verbose, x0, dual, ctx_out,
                    converged, trace, stream);
}

int cg_ctx_info(const cg_ctx* ctx, cg_ctx_info_t* out) {
  if (!ctx || !out) return CG_ERR_INVALID_ARG;
  const cg_ctx_s* c = reinterpret_cast<const cg_ctx_s*>(ctx);
  out->n = c->n;
  out->m = c->m;
  out->dim = c->H;
  out->nnz = c->nnz;
  out->reg = c->reg;
  out->ys = c->ys;
  out->low_rank = c->low_rank;
  out->fallback = c->fallback;
  out->valid = c->valid;
  out->has_diag = c->diag_ready;
  out->has_point = c->has_point;
  out->adopted = !c->fallback;
  return CG_OK;
}

int cg_ctx_setup_diag(cg_ctx* ctx, cudaStream_t stream) {
  if (!ctx) return CG_ERR_INVALID_ARG;
  cg_ctx_s* c = reinterpret_cast<cg_ctx_s*>(ctx);
  if (!c->valid) return CG_ERR_INVALID_CONTEXT;
  return cg::ctx_setup_diag(c, stream);
}

int cg_ctx_apply(cg_ctx* ctx, const double* r, double* z, int mode, cudaStream_t stream) {
  if (!ctx || !r || !z) return CG_ERR_INVALID_ARG;
  cg_ctx_s* c = reinterpret_cast<cg_ctx_s*>(ctx);
  if (!c->valid) return CG_ERR_INVALID_CONTEXT;
  if (mode == CG_PRECOND_DIAG) {
    if (!c->diag_ready) {
      cg::set_last_error("diagonal preconditioner not set up", __FILE__, __LINE__);
      return CG_ERR_INVALID_CONTEXT;
    }
    { cg::scale_kernel<<<std::max(1, std::min((c->H + 255) / 256, 1024)), 256, 0, stream>>>(
        c->inv_diag, r, z, c->H); cg::count_launch(); }
    CG_TRY_CUDA(cudaGetLastError());
    return CG_OK;
  }
  if (mode == CG_PRECOND_SPLR) return cg::ctx_apply_full(c, r, z, stream);
  return CG_ERR_INVALID_ARG;
}

int cg_ctx_copy(const cg_ctx* ctx, int what, void* dst, cudaStream_t stream) {
  if (!ctx || !dst) return CG_ERR_INVALID_ARG;
  const cg_ctx_s* c = reinterpret_cast<const cg_ctx_s*>(ctx);
  const void* src = nullptr;
  size_t bytes = 0;
  switch (what) {
    case CG_CTX_CSR_VALUES: src = c->A.val; bytes = c->nnz * sizeof(double); break;
    case CG_CTX_CSR_COLIND: src = c->A.col; bytes = c->nnz * sizeof(int); break;
    case CG_CTX_CSR_ROWPTR: src = c->A.rowptr; bytes = (c->H + 1) * sizeof(int); break;
    case CG_CTX_SECANT_S: src = c->s; bytes = c->H * sizeof(double); break;
    case CG_CTX_SECANT_Y: src = c->y; bytes = c->H * sizeof(double); break;
    case CG_CTX_INV_DIAG:
      if (!c->diag_ready) return CG_ERR_INVALID_CONTEXT;
      src = c->inv_diag; bytes = c->H * sizeof(double); break;
    case CG_CTX_POINT:
      if (!c->has_point) return CG_ERR_INVALID_CONTEXT;
      src = c->point; bytes = c->H * sizeof(double); break;
    case CG_CTX_INVA_Y: src = c->u; bytes = c->H * sizeof(double); break;
    default: return CG_ERR_INVALID_ARG;
  }
  CG_TRY_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream));
  return CG_OK;
}

int cg_ctx_destroy(cg_ctx* ctx) {
  if (!ctx) return CG_OK;
  cg_ctx_s* c = reinterpret_cast<cg_ctx_s*>(ctx);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  if (c->block) cudaFree(c->block);
  if (c->sc) {
    cg::spchol_release(*c->sc);
    delete c->sc;
  }
  if (c->pf) {
    cg::peel_release(*c->pf);
    delete c->pf;
  }
  cudaSetDevice(prev);
  delete c;
  return CG_OK;
}

int cg_t_values_f64(const double* alpha, const double* beta, const double* M, int n, int m,
                    double reg, double* Tvalues, int* Tflatind, cudaStream_t stream) {
  if (!alpha || !beta || !M || n <= 0 || m <= 0 || !(reg > 0)) return CG_ERR_INVALID_ARG;
  if (m == 1) return CG_OK;
  const long long Te = (long long)n * (m - 1);
  const int blocks = (int)std::max<long long>(1, std::min<long long>((Te + 255) / 256, 148 * 16));
  { cg::t_values_kernel<<<blocks, 256, 0, stream>>>(alpha, beta, M, n, m, 1.0 / reg, Tvalues,
                                                  Tflatind); cg::count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

int cg_test_t_sparsify_f64(const double* alpha, const double* beta, const double* M,
                           const double* a, const double* b, double reg, double shift, int K,
                           int n, int m, double* rows, double* cols, double* grad,
                           double* objfn_gnorm, double* csr_val, int* csr_colind,
                           int* csr_rowptr, long long* k_actual, cudaStream_t stream) {
  using namespace cg;
  if (!alpha || !beta || !M || !a || !b || n <= 0 || m <= 0 || !(reg > 0))
    return CG_ERR_INVALID_ARG;
  const int H = n + m - 1;
  const long long Te = (long long)n * (m - 1);
  long long Ks = std::min<long long>(std::max(K, 1), Te);
  const long long kcap = std::max<long long>(Ks, 1);
  const int sms = sm_count_current();
  int strips = 1, splits = 1;
  tpass_geometry(n, m, sms, strips, splits);
  Workspace ws(stream);
  const size_t o_g = ws.reserve<double>(n + m), o_ab = ws.reserve<double>(n + m);
  const size_t o_res = ws.reserve<TResult>(1);
  const size_t o_tw = ws.reserve<double>(tpass_workspace_doubles(n, m, strips, splits));
  const size_t o_tc = ws.reserve<unsigned int>(splits + strips + 1);
  const size_t o_sw = ws.reserve<char>(sparsify_work_bytes(n, m));
  const size_t o_ipt = ws.reserve<int>(n + 1), o_ij = ws.reserve<int>(kcap);
  const size_t o_iv = ws.reserve<double>(kcap);
  CG_TRY(ws.allocate());
  double* gamma = ws.at<double>(o_g);
  double* ab = ws.at<double>(o_ab);
  CG_TRY_CUDA(cudaMemcpyAsync(gamma, alpha, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  CG_TRY_CUDA(cudaMemcpyAsync(gamma + n, beta, m * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  CG_TRY_CUDA(cudaMemcpyAsync(ab, a, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  CG_TRY_CUDA(cudaMemcpyAsync(ab + n, b, m * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  unsigned int* tc = ws.at<unsigned int>(o_tc);
  CG_TRY_CUDA(cudaMemsetAsync(tc, 0, (splits + strips + 1) * sizeof(unsigned int), stream));
  double* tw = ws.at<double>(o_tw);
  TPassArgs x{};
  x.M = M;
  x.n = n;
  x.m = m;
  x.eta = reg;
  x.s2 = kLog2e / reg;
  x.ab = ab;
  x.gamma = gamma;
  x.rows = rows;
  x.cols = cols;
  x.grad = grad;
  x.res = ws.at<TResult>(o_res);
  x.strips = strips;
  x.splits = splits;
  x.rowpart = tw;
  x.colpart = tw + (size_t)strips * n;
  x.scal = tw + (size_t)strips * n + (size_t)splits * m;
  x.counters = tc;
  CG_TRY(launch_tpass(false, x, stream));
  TResult tr{};
  CG_TRY_CUDA(cudaMemcpyAsync(&tr, x.res, sizeof(TResult), cudaMemcpyDeviceToHost, stream));
  SparsifyWork sw;
  sparsify_work_carve(ws.at<char>(o_sw), n, m, sw);
  SpHess h;
  h.n = n;
  h.m = m;
  h.H = H;
  h.kcap = kcap;
  h.val = csr_val;
  h.col = csr_colind;
  h.rowptr = csr_rowptr;
  h.ipt = ws.at<int>(o_ipt);
  h.ij = ws.at<int>(o_ij);
  h.iv = ws.at<double>(o_iv);
  CG_TRY(sparsify_select_and_build(false, M, gamma, rows, cols, n, m, x.s2, shift, Ks, h, sw,
                                   stream));
  CG_TRY_CUDA(cudaStreamSynchronize(stream));
  if (objfn_gnorm) {
    const double fg[2] = {tr.f, tr.gnorm};
    CG_TRY_CUDA(cudaMemcpyAsync(objfn_gnorm, fg, sizeof(fg), cudaMemcpyHostToDevice, stream));
    CG_TRY_CUDA(cudaStreamSynchronize(stream));
  }
  if (k_actual) *k_actual = Ks;
  ws.release();
  return CG_OK;
}

int cg_test_spd_solve_f64(const double* values, const int* colind, const int* rowptr, int n,
                          const double* rhs, double* x, cudaStream_t stream) {
  using namespace cg;
  if (!values || !colind || !rowptr || !rhs || !x || n <= 0) return CG_ERR_INVALID_ARG;
  cusolverDnHandle_t h = nullptr;
  CG_TRY(solver_handle(&h));
  int lwork = 0;
  CG_TRY(schur_lwork(h, n, lwork));
  Workspace ws(stream);
  const size_t o_S = ws.reserve<double>((size_t)n * n), o_w = ws.reserve<double>(std::max(lwork, 1));
  const size_t o_info = ws.reserve<int>(2);  // potrf, potrs
  CG_TRY(ws.allocate());
  double* S = ws.at<double>(o_S);
  CG_TRY_CUDA(cudaMemsetAsync(S, 0, (size_t)n * n * sizeof(double), stream));
  { densify_lower_kernel<<<std::min(n, 4096), 256, 0, stream>>>(values, colind, rowptr, n, S); cg::count_launch(); }
  CG_TRY_CUDA(cudaMemcpyAsync(x, rhs, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  if (cusolverDnSetStream(h, stream) != CUSOLVER_STATUS_SUCCESS) return CG_ERR_SOLVER;
  int* info = ws.at<int>(o_info);
  if (cusolverDnDpotrf(h, CUBLAS_FILL_MODE_LOWER, n, S, n, ws.at<double>(o_w), lwork, info) !=
      CUSOLVER_STATUS_SUCCESS)
    return CG_ERR_SOLVER;
  if (cusolverDnDpotrs(h, CUBLAS_FILL_MODE_LOWER, n, 1, S, n, x, n, info + 1) !=
      CUSOLVER_STATUS_SUCCESS)
    return CG_ERR_SOLVER;
  int hinfo = 0;
  CG_TRY_CUDA(cudaMemcpyAsync(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost, stream));
  CG_TRY_CUDA(cudaStreamSynchronize(stream));
  ws.release();
  if (hinfo != 0) {
    set_last_error("matrix is not symmetric positive definite", __FILE__, __LINE__);
    return CG_ERR_NOT_SPD;
  }
  return CG_OK;
}

}  // extern "C"
