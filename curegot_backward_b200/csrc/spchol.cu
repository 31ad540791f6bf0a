// Sparse Cholesky direction solve with the SPLR sparsified Hessian.
//
// The reference factors A = Hsl + shift I with cuDSS (src/linsolve.cu:159-268):
// reorder + symbolic on pattern updates, numeric factorization every
// iteration, then the solve.  cuDSS is not in this image; cuSOLVER's sparse
// Cholesky provides the same phases:
//   pattern update : copy the kernel-built CSR pattern (lower view) to the
//                    host, build the full symmetric pattern, AMD ordering
//                    (cusolverSpXcsrsymamdHost; the reorder runs on the CPU
//                    as cuDSS's does), permuted pattern + value map, and a
//                    count of the factor (elimination tree + row subtrees)
//                    so the caller can choose between this solve and the
//                    dense Schur-complement one; then the symbolic analysis
//                    on the device (cusolverSpXcsrcholAnalysis);
//   every iteration: gather the current values into the permuted pattern
//                    (one kernel), numeric factorization on the device;
//   solve          : permute, cusolverSpDcsrcholSolve, un-permute.
// At low Hessian density the SPLR graph is close to a forest and the factor
// has about as many entries as A; at ~1 % density on unstructured point
// clouds it fills in to a nearly dense matrix, where the dense Schur path is
// the faster one.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <unordered_map>

#include "spchol.cuh"

namespace cg {

namespace {

__global__ void gather_vals_kernel(const double* __restrict__ src, const int* __restrict__ map,
                                   long long nnz, double* __restrict__ dst) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nnz;
       e += (long long)gridDim.x * blockDim.x)
    dst[e] = src[map[e]];
}

__global__ void permute_kernel(const double* __restrict__ src, const int* __restrict__ perm,
                               int H, double* __restrict__ dst, int forward) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < H; k += gridDim.x * blockDim.x) {
    if (forward) dst[k] = src[perm[k]];   // new <- old
    else dst[perm[k]] = src[k];           // old <- new
  }
}

int grid_for(long long work, int per_block, int cap) {
  long long g = (work + per_block - 1) / per_block;
  return (int)std::max<long long>(1, std::min<long long>(g, cap));
}

int sp_status(cusolverStatus_t s, const char* what) {
  if (s == CUSOLVER_STATUS_SUCCESS) return CG_OK;
  set_last_error(what, __FILE__, __LINE__);
  return (s == CUSOLVER_STATUS_ALLOC_FAILED) ? CG_ERR_OOM : CG_ERR_SOLVER;
}

struct SpHandles {
  cusolverSpHandle_t sp = nullptr;
  cusparseMatDescr_t descr = nullptr;
};

// cuSOLVER-sparse handle + general zero-based descriptor for the calling
// thread and current device (created once).
int sp_handles(SpHandles* out) {
  thread_local std::unordered_map<int, SpHandles> handles;
  int dev = 0;
  CG_TRY_CUDA(cudaGetDevice(&dev));
  auto it = handles.find(dev);
  if (it == handles.end()) {
    SpHandles h;
    CG_TRY(sp_status(cusolverSpCreate(&h.sp), "cusolverSpCreate failed"));
    if (cusparseCreateMatDescr(&h.descr) != CUSPARSE_STATUS_SUCCESS) {
      set_last_error("cusparseCreateMatDescr failed", __FILE__, __LINE__);
      return CG_ERR_SOLVER;
    }
    cusparseSetMatType(h.descr, CUSPARSE_MATRIX_TYPE_GENERAL);
    cusparseSetMatIndexBase(h.descr, CUSPARSE_INDEX_BASE_ZERO);
    it = handles.emplace(dev, h).first;
  }
  *out = it->second;
  return CG_OK;
}

// Elimination tree of the permuted pattern, then for every row the subtree
// of the etree it reaches: each visited node is one entry of L (Liu's
// row-subtree count).  Accumulates flops = sum_j colcount_j^2 and stops once
// it passes the budget.
void count_factor(int H, const std::vector<int>& rp, const std::vector<int>& col,
                  double budget, double& flops, long long& nnz_L) {
  std::vector<int> parent(H, -1), anc(H, -1), mark(H, -1);
  std::vector<long long> cc(H, 0);
  for (int i = 0; i < H; ++i)
    for (int q = rp[i]; q < rp[i + 1]; ++q) {
      int r = col[q];
      if (r >= i) continue;
      while (anc[r] != -1 && anc[r] != i) {
        const int nx = anc[r];
        anc[r] = i;
        r = nx;
      }
      if (anc[r] == -1) {
        anc[r] = i;
        parent[r] = i;
      }
    }
  double f = 0.0;
  long long cnt = 0;
  for (int i = 0; i < H; ++i) {
    mark[i] = i;
    for (int q = rp[i]; q < rp[i + 1]; ++q) {
      int r = col[q];
      if (r >= i) continue;
      while (r != -1 && mark[r] != i) {
        mark[r] = i;
        // column r gains row i: (c+1)^2 - c^2
        f += 2.0 * (double)cc[r] + 1.0;
        ++cc[r];
        ++cnt;
        r = parent[r];
      }
    }
    if (f > budget) {
      flops = INFINITY;
      nnz_L = cnt;
      return;
    }
  }
  flops = f;
  nnz_L = cnt;
}

}  // namespace

namespace {
int dev_alloc(SparseChol& C, void** p, size_t bytes) {
  if (C.stream_ordered) CG_TRY(pool_alloc_async(p, bytes, C.alloc_stream));
  else CG_TRY_CUDA(cudaMalloc(p, bytes));
  return CG_OK;
}
void dev_free(SparseChol& C, void* p) {
  if (!p) return;
  if (C.stream_ordered) cudaFreeAsync(p, C.alloc_stream);
  else cudaFree(p);
}
}  // namespace

void spchol_release(SparseChol& C) {
  if (C.info) cusolverSpDestroyCsrcholInfo(C.info);
  C.info = nullptr;
  dev_free(C, C.buffer);
  C.buffer = nullptr;
  C.buffer_bytes = 0;
  dev_free(C, C.dblock);
  C.dblock = nullptr;
  C.dblock_bytes = 0;
  C.analyzed = false;
}

int spchol_order(SparseChol& C, const SpHess& A, double flop_budget, cudaStream_t st) {
  const int H = A.H;
  SpHandles hd;
  CG_TRY(sp_handles(&hd));
  C.analyzed = false;
  // lower pattern -> host
  std::vector<int> rp(H + 1);
  CG_TRY(read_device_bulk(rp.data(), A.rowptr, (H + 1) * sizeof(int), st));
  const int nl = rp[H];
  std::vector<int> cl(std::max(nl, 1));
  CG_TRY(read_device_bulk(cl.data(), A.col, (size_t)nl * sizeof(int), st));
  // full symmetric pattern + value map; rows are filled in increasing row
  // order of the lower view, so every row of the full pattern comes out with
  // ascending columns (upper part first from earlier rows, then the lower)
  std::vector<int> cnt(H, 0);
  for (int r = 0; r < H; ++r)
    for (int q = rp[r]; q < rp[r + 1]; ++q) {
      cnt[r]++;
      if (cl[q] != r) cnt[cl[q]]++;
    }
  std::vector<int> frp(H + 1, 0);
  for (int r = 0; r < H; ++r) frp[r + 1] = frp[r] + cnt[r];
  const int nf = frp[H];
  std::vector<int> fcol(nf), fmap(nf), fill(frp.begin(), frp.end() - 1);
  // entries (r, c) with c < r, placed as (r, c) and (c, r): visit rows in
  // order so row c receives its upper entries (c, r) with r ascending after
  // its own lower entries.  Sort per row afterwards to be safe.
  for (int r = 0; r < H; ++r)
    for (int q = rp[r]; q < rp[r + 1]; ++q) {
      const int c = cl[q];
      int k = fill[r]++;
      fcol[k] = c;
      fmap[k] = q;
      if (c != r) {
        k = fill[c]++;
        fcol[k] = r;
        fmap[k] = q;
      }
    }
  {
    std::vector<std::pair<int, int>> row;
    for (int r = 0; r < H; ++r) {
      row.clear();
      for (int k = frp[r]; k < frp[r + 1]; ++k) row.emplace_back(fcol[k], fmap[k]);
      std::sort(row.begin(), row.end());
      for (int k = frp[r]; k < frp[r + 1]; ++k) {
        fcol[k] = row[k - frp[r]].first;
        fmap[k] = row[k - frp[r]].second;
      }
    }
  }
  std::vector<int>& perm = C.h_perm;
  perm.assign(H, 0);
  CG_TRY(sp_status(cusolverSpXcsrsymamdHost(hd.sp, H, nf, hd.descr, frp.data(), fcol.data(),
                                            perm.data()),
                   "cusolverSpXcsrsymamdHost failed"));
  std::vector<int> inv(H);
  for (int k = 0; k < H; ++k) inv[perm[k]] = k;
  // permuted pattern: row inv[r] holds inv[c] for every (r, c)
  std::vector<int>& prp = C.h_rowptr;
  prp.assign(H + 1, 0);
  for (int r = 0; r < H; ++r) prp[inv[r] + 1] = frp[r + 1] - frp[r];
  for (int r = 0; r < H; ++r) prp[r + 1] += prp[r];
  C.h_col.assign(nf, 0);
  C.h_map.assign(nf, 0);
  {
    std::vector<std::pair<int, int>> row;
    for (int r = 0; r < H; ++r) {
      const int nr = inv[r];
      row.clear();
      for (int k = frp[r]; k < frp[r + 1]; ++k) row.emplace_back(inv[fcol[k]], fmap[k]);
      std::sort(row.begin(), row.end());
      for (size_t t = 0; t < row.size(); ++t) {
        C.h_col[prp[nr] + t] = row[t].first;
        C.h_map[prp[nr] + t] = row[t].second;
      }
    }
  }
  C.H = H;
  C.nnz = nf;
  count_factor(H, prp, C.h_col, flop_budget, C.flops, C.nnz_L);
  return CG_OK;
}

int spchol_analyze(SparseChol& C, cudaStream_t st) {
  const int H = C.H;
  const long long nf = C.nnz;
  SpHandles hd;
  CG_TRY(sp_handles(&hd));
  CG_TRY(sp_status(cusolverSpSetStream(hd.sp, st), "cusolverSpSetStream failed"));
  auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
  const size_t bytes = al((H + 1) * 4) + 2 * al(nf * 4) + al(H * 4) + al(nf * 8) + 2 * al(H * 8);
  if (bytes > C.dblock_bytes) {
    dev_free(C, C.dblock);
    C.dblock = nullptr;
    C.dblock_bytes = 0;
    CG_TRY(dev_alloc(C, &C.dblock, bytes));
    C.dblock_bytes = bytes;
  }
  char* p = static_cast<char*>(C.dblock);
  C.d_rowptr = reinterpret_cast<int*>(p); p += al((H + 1) * 4);
  C.d_col = reinterpret_cast<int*>(p); p += al(nf * 4);
  C.d_map = reinterpret_cast<int*>(p); p += al(nf * 4);
  C.d_perm = reinterpret_cast<int*>(p); p += al(H * 4);
  C.d_val = reinterpret_cast<double*>(p); p += al(nf * 8);
  C.d_b = reinterpret_cast<double*>(p); p += al(H * 8);
  C.d_x = reinterpret_cast<double*>(p);
  CG_TRY_CUDA(cudaMemcpyAsync(C.d_rowptr, C.h_rowptr.data(), (H + 1) * 4, cudaMemcpyHostToDevice, st));
  CG_TRY_CUDA(cudaMemcpyAsync(C.d_col, C.h_col.data(), nf * 4, cudaMemcpyHostToDevice, st));
  CG_TRY_CUDA(cudaMemcpyAsync(C.d_map, C.h_map.data(), nf * 4, cudaMemcpyHostToDevice, st));
  CG_TRY_CUDA(cudaMemcpyAsync(C.d_perm, C.h_perm.data(), H * 4, cudaMemcpyHostToDevice, st));
  if (C.info) cusolverSpDestroyCsrcholInfo(C.info);
  C.info = nullptr;
  CG_TRY(sp_status(cusolverSpCreateCsrcholInfo(&C.info), "cusolverSpCreateCsrcholInfo failed"));
  CG_TRY(sp_status(cusolverSpXcsrcholAnalysis(hd.sp, H, (int)nf, hd.descr, C.d_rowptr, C.d_col,
                                              C.info),
                   "cusolverSpXcsrcholAnalysis failed"));
  size_t internal = 0, work = 0;
  CG_TRY(sp_status(cusolverSpDcsrcholBufferInfo(hd.sp, H, (int)nf, hd.descr, C.d_val, C.d_rowptr,
                                                C.d_col, C.info, &internal, &work),
                   "cusolverSpDcsrcholBufferInfo failed"));
  work = std::max<size_t>(work, 256);
  if (work > C.buffer_bytes) {
    dev_free(C, C.buffer);
    C.buffer = nullptr;
    C.buffer_bytes = 0;
    CG_TRY(dev_alloc(C, &C.buffer, work));
    C.buffer_bytes = work;
  }
  C.analyzed = true;
  return CG_OK;
}

int spchol_factor(SparseChol& C, const SpHess& A, cudaStream_t st, int* zero_pivot) {
  if (!C.analyzed) {
    set_last_error("sparse Cholesky: factor before analysis", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  SpHandles hd;
  CG_TRY(sp_handles(&hd));
  CG_TRY(sp_status(cusolverSpSetStream(hd.sp, st), "cusolverSpSetStream failed"));
  { gather_vals_kernel<<<grid_for(C.nnz, 256, 148 * 8), 256, 0, st>>>(A.val, C.d_map, C.nnz, C.d_val); count_launch(); }
  CG_TRY_CUDA(cudaGetLastError());
  CG_TRY(sp_status(cusolverSpDcsrcholFactor(hd.sp, C.H, (int)C.nnz, hd.descr, C.d_val, C.d_rowptr,
                                            C.d_col, C.info, C.buffer),
                   "cusolverSpDcsrcholFactor failed"));
  if (zero_pivot) {
    int pos = -1;
    CG_TRY(sp_status(cusolverSpDcsrcholZeroPivot(hd.sp, C.info, 0.0, &pos),
                     "cusolverSpDcsrcholZeroPivot failed"));
    *zero_pivot = pos;
  }
  return CG_OK;
}

int spchol_solve(SparseChol& C, const double* rhs, double* x, int nrhs, cudaStream_t st) {
  SpHandles hd;
  CG_TRY(sp_handles(&hd));
  CG_TRY(sp_status(cusolverSpSetStream(hd.sp, st), "cusolverSpSetStream failed"));
  const int H = C.H;
  for (int c = 0; c < nrhs; ++c) {
    { permute_kernel<<<grid_for(H, 256, 1024), 256, 0, st>>>(rhs + (size_t)c * H, C.d_perm, H, C.d_b, 1); count_launch(); }
    CG_TRY(sp_status(cusolverSpDcsrcholSolve(hd.sp, H, C.d_b, C.d_x, C.info, C.buffer),
                     "cusolverSpDcsrcholSolve failed"));
    { permute_kernel<<<grid_for(H, 256, 1024), 256, 0, st>>>(C.d_x, C.d_perm, H, x + (size_t)c * H, 0); count_launch(); }
  }
  CG_TRY_CUDA(cudaGetLastError());
  return CG_OK;
}

}  // namespace cg
