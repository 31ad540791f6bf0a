// CPU oracle for the entropic-OT hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain FP64 C++ on the
// host, the algorithms of the reference solver (benben-cd/curegot_backward)
// so that tests can check the CUDA product path against it.  Only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference leg
// may load it.  The product library never links or calls it.
//
// Every function names the reference file:line it follows.  Reduction order
// differs from the reference GPU kernels (they use atomics and block trees);
// results agree to rounding, which is what the parity tolerances allow.
//
// Deliberate, documented choices where the reference is unspecified:
//   * top-K ties (the reference's cub::DeviceTopK runs with
//     determinism::not_guaranteed, sinkhorn_splr_kernel.cu:625-628): values
//     are ordered by value descending, then by flat Hsl index ascending.
//   * the direction solve (a cuDSS sparse Cholesky in the reference,
//     linsolve.cu:159-268) is an exact direct solve here as well: block
//     elimination of the larger diagonal block followed by a dense Cholesky
//     of the Schur complement.
//   * a negative candidate_sinkhorn_iter (the reference's timing-dependent
//     "fill idle time" mode, sinkhorn_splr.cu:500-526) runs 3 iterations.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kInf = std::numeric_limits<double>::infinity();

// ---------------------------------------------------------------------------
// BCD building blocks
// ---------------------------------------------------------------------------

// alpha_i = reg * (log a_i - LSE_j((beta_j - M_ij) / reg)), two passes (max,
// then sum of shifted exps) as in sinkhorn_bcd_kernel.cu:115-192.
void opt_alpha(const double* M, const double* beta, const double* loga,
               double* alpha, double reg, int n, int m) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    const double* Mi = M + (size_t)i * m;
    double mx = -kInf;
    for (int j = 0; j < m; ++j) mx = std::fmax(mx, (beta[j] - Mi[j]) / reg);
    double s = 0.0;
    for (int j = 0; j < m; ++j) s += std::exp((beta[j] - Mi[j]) / reg - mx);
    alpha[i] = reg * (loga[i] - (mx + std::log(s)));
  }
}

// beta_j = reg * (log b_j - LSE_i((alpha_i - M_ij) / reg)), two passes, as in
// sinkhorn_bcd_kernel.cu:35-112.  Traversed row-major per column block for
// cache locality; each column's max and sum are accumulated in i order.
void opt_beta(const double* M, const double* alpha, const double* logb,
              double* beta, double reg, int n, int m) {
  const int CB = 256;
  const int nblk = (m + CB - 1) / CB;
#pragma omp parallel for schedule(static)
  for (int blk = 0; blk < nblk; ++blk) {
    const int j0 = blk * CB, j1 = std::min(m, j0 + CB);
    double mx[CB], s[CB];
    for (int j = j0; j < j1; ++j) mx[j - j0] = -kInf;
    for (int i = 0; i < n; ++i) {
      const double* Mi = M + (size_t)i * m;
      for (int j = j0; j < j1; ++j)
        mx[j - j0] = std::fmax(mx[j - j0], (alpha[i] - Mi[j]) / reg);
    }
    for (int j = j0; j < j1; ++j) s[j - j0] = 0.0;
    for (int i = 0; i < n; ++i) {
      const double* Mi = M + (size_t)i * m;
      for (int j = j0; j < j1; ++j)
        s[j - j0] += std::exp((alpha[i] - Mi[j]) / reg - mx[j - j0]);
    }
    for (int j = j0; j < j1; ++j)
      beta[j] = reg * (logb[j] - (mx[j - j0] + std::log(s[j - j0])));
  }
}

// Gauge-normalised distance between (alpha, beta) and the previous iterate,
// sinkhorn_bcd_kernel.cu:280-326.
double iter_difference(const double* al, const double* be, const double* alp,
                       const double* bep, int n, int m) {
  double sa = 0, sb = 0, sap = 0, sbp = 0;
  for (int i = 0; i < n; ++i) { sa += al[i]; sap += alp[i]; }
  for (int j = 0; j < m; ++j) { sb += be[j]; sbp += bep[j]; }
  const double c = (sb - sa) / (n + m);
  const double d = (sbp - sap) / (n + m);
  const double K = c - d;
  double acc = 0.0;
  for (int i = 0; i < n; ++i) { double t = (al[i] - alp[i]) + K; acc += t * t; }
  for (int j = 0; j < m; ++j) { double t = (be[j] - bep[j]) - K; acc += t * t; }
  return std::sqrt(acc);
}

// ||rowsum(T) - a||_2 with T = exp((alpha + beta - M) / reg),
// sinkhorn_bcd_kernel.cu:329-353 and utils.cu:104-128.
double marginal_error(const double* M, const double* al, const double* be,
                      const double* a, double reg, int n, int m) {
  std::vector<double> r(n);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    const double* Mi = M + (size_t)i * m;
    double s = 0.0;
    for (int j = 0; j < m; ++j) s += std::exp((al[i] + be[j] - Mi[j]) / reg);
    r[i] = s;
  }
  double acc = 0.0;
  for (int i = 0; i < n; ++i) { double t = r[i] - a[i]; acc += t * t; }
  return std::sqrt(acc);
}

void transport_plan(const double* M, const double* al, const double* be,
                    double* P, double reg, int n, int m) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < m; ++j)
      P[(size_t)i * m + j] = std::exp((al[i] + be[j] - M[(size_t)i * m + j]) / reg);
}

// ---------------------------------------------------------------------------
// SPLR building blocks
// ---------------------------------------------------------------------------

// gamma -> (alpha + beta_{m-1}, beta - beta_{m-1}, 0); sinkhorn_splr_kernel.cu:156-197.
void shift_gamma(double* g, int n, int m) {
  const int last = n + m - 1;
  const double sh = g[last];
  for (int i = 0; i < last; ++i) g[i] += (i < n) ? sh : -sh;
  g[last] = 0.0;
}

struct TEval {
  double f = 0.0, gnorm = 0.0, dg = 0.0;
};

// T = exp((alpha + beta - M)/reg), row/col sums, f = reg*sum(T) - <gamma,ab>,
// g = (r - a, c_{:m-1} - b_{:m-1}); sinkhorn_splr_kernel.cu:214-546.  When
// direc != nullptr also returns <g, direc> (line-search variant,
// sinkhorn_splr_kernel_line_search.cu:277-370).
TEval t_objfn_grad(const double* gamma, const double* M, const double* ab,
                   double reg, int n, int m, double* rows, double* cols,
                   double* grad, const double* direc) {
  const double* al = gamma;
  const double* be = gamma + n;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i) {
    const double* Mi = M + (size_t)i * m;
    double s = 0.0;
    for (int j = 0; j < m; ++j) s += std::exp((al[i] + be[j] - Mi[j]) / reg);
    rows[i] = s;
  }
  const int CB = 256;
  const int nblk = (m + CB - 1) / CB;
#pragma omp parallel for schedule(static)
  for (int blk = 0; blk < nblk; ++blk) {
    const int j0 = blk * CB, j1 = std::min(m, j0 + CB);
    double acc[CB];
    for (int j = j0; j < j1; ++j) acc[j - j0] = 0.0;
    for (int i = 0; i < n; ++i) {
      const double* Mi = M + (size_t)i * m;
      for (int j = j0; j < j1; ++j) acc[j - j0] += std::exp((al[i] + be[j] - Mi[j]) / reg);
    }
    for (int j = j0; j < j1; ++j) cols[j] = acc[j - j0];
  }
  TEval e;
  double tsum = 0.0, dot = 0.0, g2 = 0.0, dg = 0.0;
  const int H = n + m - 1;
  for (int k = 0; k < n + m; ++k) {
    dot += ab[k] * gamma[k];
    if (k < H) {
      double gv;
      if (k < n) { tsum += rows[k]; gv = rows[k] - ab[k]; }
      else gv = cols[k - n] - ab[k];
      grad[k] = gv;
      g2 += gv * gv;
      if (direc) dg += gv * direc[k];
    }
  }
  e.f = reg * tsum - dot;
  e.gnorm = std::sqrt(g2);
  e.dg = dg;
  return e;
}

// Sparsified, shifted, scaled lower Hessian Hsl in CSR form
// (sinkhorn_splr_kernel.cu:38-100 layout; :554-675 top-K + diagonal + sort;
// :681-734 fixed-pattern refresh; :741-820 CSR conversion).
struct Csr {
  int H = 0;
  std::vector<double> val;
  std::vector<int> col;
  std::vector<int> rowptr;
  // pattern of the selected T_t entries, as (i, j) pairs in CSR order
  std::vector<int> sel_i, sel_j;
};

void build_csr_from_selection(Csr& A, const std::vector<int64_t>& flat, const double* gamma,
                              const double* M, const double* rows, const double* cols,
                              double reg, double shift, int n, int m) {
  const int H = n + m - 1;
  A.H = H;
  A.rowptr.assign(H + 1, 0);
  // count entries per Hsl row: rows < n hold only the diagonal.
  std::vector<int> cnt(H, 1);
  for (int64_t f : flat) cnt[(int)(f / H)] += 1;
  for (int r = 0; r < H; ++r) A.rowptr[r + 1] = A.rowptr[r] + cnt[r];
  const int nnz = A.rowptr[H];
  A.val.assign(nnz, 0.0);
  A.col.assign(nnz, 0);
  A.sel_i.clear();
  A.sel_j.clear();
  std::vector<int> fill(A.rowptr.begin(), A.rowptr.end() - 1);
  // flat indices are sorted ascending: row-major over Hsl, off-diagonals of
  // row n+j (cols i < n) come before its diagonal (col n+j).
  size_t p = 0;
  for (int r = 0; r < H; ++r) {
    if (r >= n) {
      while (p < flat.size() && flat[p] / H == r) {
        const int i = (int)(flat[p] % H);
        const int j = r - n;
        const int k = fill[r]++;
        A.col[k] = i;
        A.val[k] = std::exp((gamma[i] + gamma[n + j] - M[(size_t)i * m + j]) / reg);
        A.sel_i.push_back(i);
        A.sel_j.push_back(j);
        ++p;
      }
    }
    const int k = fill[r]++;
    A.col[k] = r;
    A.val[k] = (r < n) ? rows[r] + shift : cols[r - n] + shift;
  }
}

// Top-K over T_t (i < n, j < m-1), Hsl flat index (n+j)*H + i.
std::vector<int64_t> select_topk(const double* gamma, const double* M, double reg,
                                 int n, int m, int64_t Ks) {
  const int H = n + m - 1;
  const int64_t Te = (int64_t)n * (m - 1);
  std::vector<std::pair<double, int64_t>> items((size_t)Te);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < m - 1; ++j) {
      const double t = std::exp((gamma[i] + gamma[n + j] - M[(size_t)i * m + j]) / reg);
      items[(size_t)i * (m - 1) + j] = {t, (int64_t)(n + j) * H + i};
    }
  auto better = [](const std::pair<double, int64_t>& x, const std::pair<double, int64_t>& y) {
    if (x.first != y.first) return x.first > y.first;
    return x.second < y.second;
  };
  if (Ks < Te) std::nth_element(items.begin(), items.begin() + Ks, items.end(), better);
  std::vector<int64_t> flat((size_t)Ks);
  for (int64_t k = 0; k < Ks; ++k) flat[(size_t)k] = items[(size_t)k].second;
  std::sort(flat.begin(), flat.end());
  return flat;
}

void refresh_values(Csr& A, const double* gamma, const double* M, const double* rows,
                    const double* cols, double reg, double shift, int n, int m) {
  const int H = n + m - 1;
  size_t p = 0;
  for (int r = 0; r < H; ++r) {
    for (int k = A.rowptr[r]; k < A.rowptr[r + 1]; ++k) {
      const int c = A.col[k];
      if (c == r) {
        A.val[k] = (r < n) ? rows[r] + shift : cols[r - n] + shift;
      } else {
        const int i = A.sel_i[p], j = A.sel_j[p];
        ++p;
        A.val[k] = std::exp((gamma[i] + gamma[n + j] - M[(size_t)i * m + j]) / reg);
      }
    }
  }
}

// Dense Cholesky (lower) in place, row-major k x k; returns false if not SPD.
bool cholesky(std::vector<double>& S, int k) {
  for (int c = 0; c < k; ++c) {
    double d = S[(size_t)c * k + c];
    for (int t = 0; t < c; ++t) d -= S[(size_t)c * k + t] * S[(size_t)c * k + t];
    if (!(d > 0.0) || !std::isfinite(d)) return false;
    d = std::sqrt(d);
    S[(size_t)c * k + c] = d;
#pragma omp parallel for schedule(static) if (k - c > 256)
    for (int r = c + 1; r < k; ++r) {
      double v = S[(size_t)r * k + c];
      const double* Lr = &S[(size_t)r * k];
      const double* Lc = &S[(size_t)c * k];
      for (int t = 0; t < c; ++t) v -= Lr[t] * Lc[t];
      S[(size_t)r * k + c] = v / d;
    }
  }
  return true;
}

void chol_solve(const std::vector<double>& L, int k, double* x) {
  for (int r = 0; r < k; ++r) {
    double v = x[r];
    for (int t = 0; t < r; ++t) v -= L[(size_t)r * k + t] * x[t];
    x[r] = v / L[(size_t)r * k + r];
  }
  for (int r = k - 1; r >= 0; --r) {
    double v = x[r];
    for (int t = r + 1; t < k; ++t) v -= L[(size_t)t * k + r] * x[t];
    x[r] = v / L[(size_t)r * k + r];
  }
}

// Exact solve with the Hsl-structured matrix A = [D1, B^T; B, D2] (lower CSR
// with rows < n diagonal-only).  The larger diagonal block is eliminated and
// the Schur complement is factored densely.
struct SchurFactor {
  int n = 0, m = 0, H = 0;
  bool big_is_alpha = true;  // eliminate the alpha (n) block
  int k = 0;                 // Schur dimension
  std::vector<double> Dbig, Dsmall;
  // entries of the coupling block C (k x p): small index, big index, value
  std::vector<int> cs, cb;
  std::vector<double> cv;
  std::vector<double> L;     // k x k Cholesky factor
  bool ok = false;
};

bool schur_factor(SchurFactor& F, const Csr& A, int n, int m) {
  const int H = n + m - 1;
  F.n = n; F.m = m; F.H = H;
  std::vector<double> D(H, 0.0);
  F.cs.clear(); F.cb.clear(); F.cv.clear();
  F.big_is_alpha = (n >= m - 1);
  for (int r = 0; r < H; ++r)
    for (int q = A.rowptr[r]; q < A.rowptr[r + 1]; ++q) {
      const int c = A.col[q];
      if (c == r) D[r] = A.val[q];
      else {
        // row r = n + j (beta block), col c = i (alpha block)
        if (F.big_is_alpha) { F.cs.push_back(r - n); F.cb.push_back(c); }
        else { F.cs.push_back(c); F.cb.push_back(r - n); }
        F.cv.push_back(A.val[q]);
      }
    }
  if (F.big_is_alpha) {
    F.Dbig.assign(D.begin(), D.begin() + n);
    F.Dsmall.assign(D.begin() + n, D.end());
  } else {
    F.Dbig.assign(D.begin() + n, D.end());
    F.Dsmall.assign(D.begin(), D.begin() + n);
  }
  const int k = (int)F.Dsmall.size();
  F.k = k;
  F.L.assign((size_t)k * k, 0.0);
  for (int s = 0; s < k; ++s) F.L[(size_t)s * k + s] = F.Dsmall[s];
  // group entries by big index
  const int p = (int)F.Dbig.size();
  std::vector<int> start(p + 1, 0);
  for (int b : F.cb) start[b + 1]++;
  for (int b = 0; b < p; ++b) start[b + 1] += start[b];
  std::vector<int> order(F.cb.size());
  {
    std::vector<int> fill(start.begin(), start.end() - 1);
    for (size_t e = 0; e < F.cb.size(); ++e) order[fill[F.cb[e]]++] = (int)e;
  }
  for (int b = 0; b < p; ++b) {
    const double inv = 1.0 / F.Dbig[b];
    for (int u = start[b]; u < start[b + 1]; ++u) {
      const int eu = order[u];
      for (int w = start[b]; w < start[b + 1]; ++w) {
        const int ew = order[w];
        F.L[(size_t)F.cs[eu] * k + F.cs[ew]] -= F.cv[eu] * F.cv[ew] * inv;
      }
    }
  }
  F.ok = cholesky(F.L, k);
  return F.ok;
}

// x = A^{-1} rhs (length H, alpha block first).
void schur_solve(const SchurFactor& F, const double* rhs, double* x) {
  const int n = F.n, H = F.H;
  const int p = (int)F.Dbig.size(), k = F.k;
  std::vector<double> rb(p), rs(k);
  if (F.big_is_alpha) {
    for (int i = 0; i < n; ++i) rb[i] = rhs[i];
    for (int j = 0; j < k; ++j) rs[j] = rhs[n + j];
  } else {
    for (int j = 0; j < p; ++j) rb[j] = rhs[n + j];
    for (int i = 0; i < k; ++i) rs[i] = rhs[i];
  }
  // rs -= C Dbig^{-1} rb
  for (size_t e = 0; e < F.cv.size(); ++e) rs[F.cs[e]] -= F.cv[e] * rb[F.cb[e]] / F.Dbig[F.cb[e]];
  chol_solve(F.L, k, rs.data());
  // xb = Dbig^{-1}(rb - C^T xs)
  std::vector<double> t(rb);
  for (size_t e = 0; e < F.cv.size(); ++e) t[F.cb[e]] -= F.cv[e] * rs[F.cs[e]];
  for (int b = 0; b < p; ++b) t[b] /= F.Dbig[b];
  if (F.big_is_alpha) {
    for (int i = 0; i < n; ++i) x[i] = t[i];
    for (int j = 0; j < k; ++j) x[n + j] = rs[j];
  } else {
    for (int j = 0; j < p; ++j) x[n + j] = t[j];
    for (int i = 0; i < k; ++i) x[i] = rs[i];
  }
  (void)H;
}

// ---------------------------------------------------------------------------
// Moré-Thuente style line-search helpers, utils.h:76-230.
// ---------------------------------------------------------------------------
double quad_min_fg(double a, double b, double fa, double ga, double fb) {
  const double ba = b - a;
  const double w = 0.5 * ba * ga / (fa - fb + ba * ga);
  return a + w * ba;
}
double quad_min_gg(double a, double b, double ga, double gb) {
  const double w = ga / (ga - gb);
  return a + w * (b - a);
}
double cubic_min(double a, double b, double fa, double fb, double ga, double gb, bool& exists) {
  const double apb = a + b, ba = b - a, ba2 = ba * ba;
  const double fba = fb - fa, gba = gb - ga;
  const double z3 = (ga + gb) * ba - 2.0 * fba;
  const double z2 = 0.5 * (gba * ba2 - 3.0 * apb * z3);
  const double z1 = fba * ba2 - apb * z2 - (a * apb + b * b) * z3;
  const double eps = std::numeric_limits<double>::epsilon();
  if (std::fabs(z3) < eps * std::fabs(z2) || std::fabs(z3) < eps * std::fabs(z1)) {
    exists = (z2 * ba > 0.0);
    return exists ? (-0.5 * z1 / z2) : b;
  }
  const double u = z2 / (3.0 * z3), v = z1 / z2;
  const double vu = v / u;
  exists = (vu <= 1.0);
  if (!exists) return b;
  double r1, r2;
  if (std::fabs(u) >= std::fabs(v)) {
    const double w = 1.0 + std::sqrt(1.0 - vu);
    r1 = -u * w;
    r2 = -v / w;
  } else {
    const double sqrtd = std::sqrt(std::fabs(u)) * std::sqrt(std::fabs(v)) * std::sqrt(1 - u / v);
    r1 = -u - sqrtd;
    r2 = -u + sqrtd;
  }
  return (z3 * ba > 0.0) ? std::max(r1, r2) : std::min(r1, r2);
}
double step_selection(double al, double au, double at, double fl, double fu, double ft,
                      double gl, double gu, double gt) {
  if (al == au) return al;
  if (!std::isfinite(ft) || !std::isfinite(gt)) return (al + at) / 2.0;
  bool ac_exists;
  const double ac = cubic_min(al, at, fl, ft, gl, gt, ac_exists);
  const double aq = quad_min_fg(al, at, fl, gl, ft);
  if (ft > fl) {
    if (!ac_exists) return aq;
    return (std::fabs(ac - al) < std::fabs(aq - al)) ? ac : ((aq + ac) / 2.0);
  }
  const double as = quad_min_gg(al, at, gl, gt);
  if (gt * gl < 0.0) return (std::fabs(ac - at) >= std::fabs(as - at)) ? ac : as;
  const double deltal = 1.1, deltau = 0.66;
  if (std::fabs(gt) < std::fabs(gl)) {
    const bool choose_ac = ac_exists && ((ac - at) * (at - al) > 0.0) &&
                           (std::fabs(ac - at) < std::fabs(as - at));
    const double res = choose_ac ? ac : as;
    return (at > al) ? std::min(at + deltau * (au - at), res)
                     : std::max(at + deltau * (au - at), res);
  }
  if (!std::isfinite(au) || !std::isfinite(fu) || !std::isfinite(gu))
    return at + deltal * (at - al);
  bool ae_exists;
  const double ae = cubic_min(at, au, ft, fu, gt, gu, ae_exists);
  return (at > al) ? std::min(at + deltau * (au - at), ae)
                   : std::max(at + deltau * (au - at), ae);
}

}  // namespace

extern "C" {

int oracle_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_set_num_threads(int t) {
#ifdef _OPENMP
  if (t > 0) omp_set_num_threads(t);
#else
  (void)t;
#endif
}

// cuda_sinkhorn_bcd, sinkhorn_bcd_kernel.cu:429-634.
int oracle_bcd(const double* M, const double* a, const double* b, int n, int m, double reg,
               double tol, int max_iter, const double* x0, double* P, double* dual, int* niter,
               double* trace, int trace_cap) {
  std::vector<double> loga(n), logb(m), al(n, 0.0), be(m, 0.0), alp(n), bep(m);
  for (int i = 0; i < n; ++i) loga[i] = std::log(a[i]);
  for (int j = 0; j < m; ++j) logb[j] = std::log(b[j]);
  if (x0) {
    std::copy(x0, x0 + n, al.begin());
    std::copy(x0 + n, x0 + n + m, be.begin());
  }
  bool use_marginal = false;
  *niter = 0;
  for (int iter = 0; iter < max_iter; ++iter) {
    alp = al;
    bep = be;
    opt_alpha(M, be.data(), loga.data(), al.data(), reg, n, m);
    opt_beta(M, al.data(), logb.data(), be.data(), reg, n, m);
    if (!use_marginal) {
      const double diff = iter_difference(al.data(), be.data(), alp.data(), bep.data(), n, m);
      if (trace && iter < trace_cap) trace[iter] = diff;
      if (diff < tol * 10) use_marginal = true;
    } else {
      const double err = marginal_error(M, al.data(), be.data(), a, reg, n, m);
      if (trace && iter < trace_cap) trace[iter] = -err;
      if (err < tol) {
        *niter = iter + 1;
        break;
      }
    }
    *niter = iter + 1;
  }
  if (P) transport_plan(M, al.data(), be.data(), P, reg, n, m);
  if (dual) {
    std::copy(al.begin(), al.end(), dual);
    std::copy(be.begin(), be.end(), dual + n);
  }
  return 0;
}

// Fixed number of BCD half-steps from a given (alpha, beta): used by tests
// that compare a single alpha or beta update.
int oracle_bcd_half_steps(const double* M, const double* a, const double* b, int n, int m,
                          double reg, double* alpha, double* beta, int which) {
  std::vector<double> loga(n), logb(m);
  for (int i = 0; i < n; ++i) loga[i] = std::log(a[i]);
  for (int j = 0; j < m; ++j) logb[j] = std::log(b[j]);
  if (which == 0) opt_alpha(M, beta, loga.data(), alpha, reg, n, m);
  else opt_beta(M, alpha, logb.data(), beta, reg, n, m);
  return 0;
}

// T pass + objective/gradient, sinkhorn_splr_kernel.cu:461-546.
int oracle_t_objfn_grad(const double* gamma, const double* M, const double* a, const double* b,
                        int n, int m, double reg, double* rows, double* cols, double* grad,
                        double* out3 /* f, gnorm */) {
  std::vector<double> ab(n + m);
  std::copy(a, a + n, ab.begin());
  std::copy(b, b + m, ab.begin() + n);
  TEval e = t_objfn_grad(gamma, M, ab.data(), reg, n, m, rows, cols, grad, nullptr);
  out3[0] = e.f;
  out3[1] = e.gnorm;
  return 0;
}

// T pass + top-K + CSR (T_computation_sparsify_host, sinkhorn_splr_kernel.cu:909-1032).
// val/colind sized >= Ks + H, rowptr sized H + 1.  Returns Ks via *k_actual.
int oracle_t_sparsify(const double* alpha, const double* beta, const double* M,
                      const double* a, const double* b, int n, int m, double reg, double shift,
                      int K, double* rows, double* cols, double* grad, double* out2,
                      double* val, int* colind, int* rowptr, long* k_actual) {
  const int H = n + m - 1;
  std::vector<double> gamma(n + m), ab(n + m);
  std::copy(alpha, alpha + n, gamma.begin());
  std::copy(beta, beta + m, gamma.begin() + n);
  std::copy(a, a + n, ab.begin());
  std::copy(b, b + m, ab.begin() + n);
  TEval e = t_objfn_grad(gamma.data(), M, ab.data(), reg, n, m, rows, cols, grad, nullptr);
  out2[0] = e.f;
  out2[1] = e.gnorm;
  const int64_t Te = (int64_t)n * (m - 1);
  int64_t Ks = std::max(K, 1);
  Ks = std::min<int64_t>(Ks, Te);
  auto flat = select_topk(gamma.data(), M, reg, n, m, Ks);
  Csr A;
  build_csr_from_selection(A, flat, gamma.data(), M, rows, cols, reg, shift, n, m);
  std::copy(A.val.begin(), A.val.end(), val);
  std::copy(A.col.begin(), A.col.end(), colind);
  std::copy(A.rowptr.begin(), A.rowptr.end(), rowptr);
  *k_actual = (long)Ks;
  (void)H;
  return 0;
}

// Solve with a general SPD CSR matrix (full or lower storage; only the lower
// triangle is read, as cuDSS with CUDSS_MVIEW_LOWER does in linsolve.cu:159).
// Dense Cholesky: test-size matrices only.
int oracle_csr_spd_solve(const double* val, const int* colind, const int* rowptr, int n,
                         const double* rhs, double* x) {
  std::vector<double> S((size_t)n * n, 0.0);
  for (int r = 0; r < n; ++r)
    for (int q = rowptr[r]; q < rowptr[r + 1]; ++q) {
      const int c = colind[q];
      if (c <= r) {
        S[(size_t)r * n + c] = val[q];
        S[(size_t)c * n + r] = val[q];
      }
    }
  if (!cholesky(S, n)) return 1;
  std::copy(rhs, rhs + n, x);
  chol_solve(S, n, x);
  return 0;
}

// cuda_sinkhorn_splr_bwd, sinkhorn_splr.cu:1305-1611 (the iterate sequence is
// identical to cuda_sinkhorn_splr, sinkhorn_splr.cu:1064-1279).
//
// ctx_* outputs describe the backward context the reference exports:
//   ctx_val/ctx_col/ctx_rowptr : CSR of the matrix A_k of the last direction
//                                solve (or, with niter == 0, of the initial
//                                sparsified Hessian: the fallback path)
//   ctx_s, ctx_y               : last secant pair (valid when low_rank)
//   ctx_scalars[0..4]          : ys, low_rank, fallback, valid, nnz
// trace (optional, 8 doubles per iteration): f, gnorm, step, K, low_rank,
// recompute_fg, candidate accepted, line-search trials.
int oracle_splr(const double* M, const double* a, const double* b, int n, int m, double reg,
                double tol, int max_iter, double density_max, double shift_max, int cycle,
                int cand_iter, const double* x0, double* P, double* dual, int* niter_out,
                int* converged_out, double* ctx_val, int* ctx_col, int* ctx_rowptr, long ctx_cap,
                double* ctx_s, double* ctx_y, double* ctx_scalars, double* trace,
                int trace_cap) {
  const int H = n + m - 1;
  const int64_t Te = (int64_t)n * (m - 1);
  if (cand_iter < 0) cand_iter = 3;
  density_max = std::min(density_max, 1.0);
  density_max = std::max(density_max, 0.0);
  const double density_min = 0.01 * density_max;
  double density = 0.1 * density_max;
  double shift;
  size_t Kmax = (size_t)(density_max * n * (m - 1));
  Kmax = std::max(Kmax, (size_t)1);

  std::vector<double> ab(n + m), logab(n + m);
  std::copy(a, a + n, ab.begin());
  std::copy(b, b + m, ab.begin() + n);
  for (int k = 0; k < n + m; ++k) logab[k] = std::log(ab[k]);
  std::vector<double> gamma(n + m, 0.0), gamma_prev(n + m, 0.0), gamma_bcd(n + m, 0.0);
  std::vector<double> grad(H, 0.0), grad_prev(H, 0.0), grad_bcd(H, 0.0);
  std::vector<double> rows(n), cols(m), rows_bcd(n), cols_bcd(m);
  std::vector<double> y(H, 0.0), s(H, 0.0), direc(H, 0.0), u(H, 0.0);

  // init_dual, sinkhorn_splr.cu:330-359
  if (x0) {
    std::copy(x0, x0 + n + m, gamma.begin());
    shift_gamma(gamma.data(), n, m);
  } else {
    std::fill(gamma.begin() + n, gamma.end(), 0.0);
    opt_alpha(M, gamma.data() + n, logab.data(), gamma.data(), reg, n, m);
  }

  auto T_eval = [&](std::vector<double>& g, std::vector<double>& gr, std::vector<double>& r,
                    std::vector<double>& c, const double* d) {
    return t_objfn_grad(g.data(), M, ab.data(), reg, n, m, r.data(), c.data(), gr.data(), d);
  };

  TEval ev = T_eval(gamma, grad, rows, cols, nullptr);
  double objfn = ev.f, gnorm = ev.gnorm;
  const double gnorm_init = gnorm;
  shift = std::min(gnorm, shift_max);

  Csr A;
  int64_t Kcur = 0;
  auto dual_sphess = [&](double dens, double sh, bool fixed) {
    dens = std::min(dens, 1.0);
    dens = std::max(dens, 0.0);
    size_t K = (size_t)(dens * (double)Te);
    K = std::min(K, Kmax);
    K = std::max(K, (size_t)1);
    int64_t Ks = std::max<int64_t>((int64_t)K, 1);
    Ks = std::min<int64_t>(Ks, Te);
    if (fixed) {
      refresh_values(A, gamma.data(), M, rows.data(), cols.data(), reg, sh, n, m);
    } else {
      auto flat = select_topk(gamma.data(), M, reg, n, m, Ks);
      build_csr_from_selection(A, flat, gamma.data(), M, rows.data(), cols.data(), reg, sh, n, m);
    }
    Kcur = Ks;
  };
  dual_sphess(density, shift * reg, false);

  double alpha_step = 1.0;
  double ys = 0.0, yy = 0.0;
  bool low_rank = false, converged = false, invalid_state = false;
  int niter = 0;
  SchurFactor F;

  for (int iter = 0; iter < max_iter; ++iter) {
    if (gnorm < tol) { converged = true; break; }
    if (!std::isfinite(objfn)) break;

    // launch_low_rank, sinkhorn_splr_kernel_low_rank.cu:92-206
    ys = yy = 0.0;
    for (int k = 0; k < H; ++k) {
      y[k] = grad[k] - grad_prev[k];
      s[k] = gamma[k] - gamma_prev[k];
      ys += y[k] * s[k];
      yy += y[k] * y[k];
    }
    low_rank = (iter > 0) && (ys > 1e-6 * yy);
    const bool analyze = (iter % cycle == 0);
    const bool update = (iter % cycle == (cycle - 1));

    // candidate Sinkhorn iterate, sinkhorn_splr.cu:441-526 (run from the
    // current beta, before the line search moves gamma)
    double f_bcd = 0.0, g_bcd = 0.0;
    const bool use_cand = analyze && (cand_iter != 0);
    if (use_cand) {
      opt_alpha(M, gamma.data() + n, logab.data(), gamma_bcd.data(), reg, n, m);
      for (int t = 0; t < cand_iter; ++t) {
        opt_beta(M, gamma_bcd.data(), logab.data() + n, gamma_bcd.data() + n, reg, n, m);
        opt_alpha(M, gamma_bcd.data() + n, logab.data(), gamma_bcd.data(), reg, n, m);
      }
      shift_gamma(gamma_bcd.data(), n, m);
      TEval eb = T_eval(gamma_bcd, grad_bcd, rows_bcd, cols_bcd, nullptr);
      f_bcd = eb.f;
      g_bcd = eb.gnorm;
    }

    // compute_search_direc, sinkhorn_splr.cu:538-649
    schur_factor(F, A, n, m);
    schur_solve(F, grad.data(), direc.data());
    if (low_rank) {
      schur_solve(F, y.data(), u.data());
      double sg = 0, yinvAy = 0, yinvAg = 0;
      for (int k = 0; k < H; ++k) {
        sg += s[k] * grad[k];
        yinvAy += y[k] * u[k];
        yinvAg += y[k] * direc[k];
      }
      const double sg_ys = sg / ys;
      const double term1 = (1.0 / reg + yinvAy / ys) * sg_ys - yinvAg / ys;
      const double term2 = sg_ys;
      for (int k = 0; k < H; ++k) direc[k] += (term1 * s[k] - term2 * u[k]);
    }
    for (int k = 0; k < H; ++k) direc[k] *= -reg;

    // save_history, sinkhorn_splr.cu:652-664 (first H entries)
    std::copy(gamma.begin(), gamma.begin() + H, gamma_prev.begin());
    std::copy(grad.begin(), grad.end(), grad_prev.begin());

    // line_search_wolfe, sinkhorn_splr.cu:667-920
    bool recompute_fg = false;
    int trials = 0;
    double step_out;
    {
      const double c1 = 1e-4, c2 = 0.9;
      const int ls_max = 20;
      const double step_min = 1e-10, step_max = 2.0;
      double init_step = std::min(1.0, 1.5 * alpha_step);
      init_step = std::max(init_step, step_min);
      init_step = std::min(init_step, step_max);
      double step = init_step;
      double dg = 0.0;
      for (int k = 0; k < H; ++k) dg += grad_prev[k] * direc[k];
      double fx = objfn;
      const double fx_init = objfn;
      const double dg_init = dg;
      bool done = false;
      if (dg_init > 0.0) {
        recompute_fg = true;
        step_out = init_step;
        done = true;
      }
      if (!done) {
        const double test_decr = c1 * dg_init;
        const double test_curv = -c2 * dg_init;
        double I_lo = 0.0, I_hi = kInf;
        double fI_lo = 0.0, fI_hi = kInf;
        double gI_lo = (1.0 - c1) * dg_init, gI_hi = kInf;
        double psiI_lo = fI_lo;
        bool bracketed = false;
        const bool f_is_psi = true;
        bool use_step_min_safeguard = (step_min > 0.0);
        double I_width = kInf, I_width_prev = kInf;
        int I_shrink_fail_count = 0;
        const double delta_max = 1.1, delta_min = 7.0 / 12, shrink = 0.66;
        for (int it = 0; it < ls_max && !done; ++it) {
          // launch_line_search_computation
          for (int k = 0; k < H; ++k) gamma[k] = gamma_prev[k] + step * direc[k];
          gamma[H] = 0.0;
          TEval et = T_eval(gamma, grad, rows, cols, direc.data());
          ++trials;
          fx = et.f;
          dg = et.dg;
          objfn = fx;  // new_obj
          const double psit = fx - fx_init - step * test_decr;
          const double dpsit = dg - test_decr;
          if (psit <= 0.0 && std::fabs(dg) <= test_curv) { step_out = step; done = true; break; }
          if (step <= step_min && (psit > 0.0 || dpsit >= 0.0)) { step_out = step; done = true; break; }
          if (step >= step_max && (psit <= 0.0 && dpsit < 0.0)) { step_out = step; done = true; break; }
          const double ft = f_is_psi ? psit : fx;
          const double gt = f_is_psi ? dpsit : dg;
          if (use_step_min_safeguard && (psit <= 0.0 && dpsit < 0.0)) use_step_min_safeguard = false;
          double new_step;
          const bool in_case_2 = (psit <= psiI_lo) && (dpsit * (I_lo - step) > 0.0);
          if (in_case_2) {
            new_step = std::min(step_max, step + delta_max * (step - I_lo));
          } else {
            new_step = step_selection(I_lo, I_hi, step, fI_lo, fI_hi, ft, gI_lo, gI_hi, gt);
            new_step = std::max(new_step, step_min);
            new_step = std::min(new_step, step_max);
            if (use_step_min_safeguard) {
              const double lower = step_min;
              const double upper = std::max(step_min, delta_min * step);
              new_step = std::max(new_step, lower);
              new_step = std::min(new_step, upper);
            }
          }
          if (psit > psiI_lo) {
            I_hi = step; fI_hi = ft; gI_hi = gt;
          } else if (in_case_2) {
            I_lo = step; fI_lo = ft; gI_lo = gt; psiI_lo = psit;
          } else {
            I_hi = I_lo; fI_hi = fI_lo; gI_hi = gI_lo;
            I_lo = step; fI_lo = ft; gI_lo = gt; psiI_lo = psit;
          }
          if (!bracketed && !in_case_2) {
            const double I_left = std::min(I_lo, I_hi);
            const double I_right = std::max(I_lo, I_hi);
            bracketed = (I_left >= step_min && I_right <= step_max);
          }
          if (bracketed) {
            I_width_prev = I_width;
            I_width = std::fabs(I_hi - I_lo);
            if (I_width_prev < kInf && I_width > shrink * I_width_prev) I_shrink_fail_count += 1;
            else I_shrink_fail_count = 0;
            if (I_shrink_fail_count >= 2) {
              new_step = (I_lo + I_hi) / 2.0;
              I_shrink_fail_count = 0;
            }
          }
          step = new_step;
        }
        if (!done) {
          const double psit = fx - fx_init - step * test_decr;
          if (psit <= psiI_lo) {
            step_out = step;
          } else if (I_lo <= 0.0) {
            recompute_fg = true;
            step_out = init_step;
          } else {
            recompute_fg = true;
            step_out = I_lo;
          }
        }
      }
    }
    alpha_step = step_out;

    const double gnorm_pre = gnorm;
    if (recompute_fg) {
      for (int k = 0; k < H; ++k) gamma[k] = gamma_prev[k] + alpha_step * direc[k];
      ev = T_eval(gamma, grad, rows, cols, nullptr);
      objfn = ev.f;
      gnorm = ev.gnorm;
    } else {
      double g2 = 0.0;
      for (int k = 0; k < H; ++k) g2 += grad[k] * grad[k];
      gnorm = std::sqrt(g2);
    }

    bool cand_accepted = false;
    if (use_cand) {
      if ((f_bcd < objfn) && (g_bcd < 10 * gnorm)) {
        cand_accepted = true;
        std::copy(gamma_bcd.begin(), gamma_bcd.begin() + H, gamma.begin());
        ev = T_eval(gamma, grad, rows, cols, nullptr);
        objfn = ev.f;
        gnorm = ev.gnorm;
      }
    }

    if (update) {
      const bool bad_move = (gnorm_pre < gnorm_init) && (gnorm > gnorm_pre);
      density *= (bad_move ? 1.1 : 0.99);
      density = std::min(density_max, std::max(density_min, density));
    }

    if (trace && iter < trace_cap) {
      double* tr = trace + (size_t)iter * 8;
      tr[0] = objfn; tr[1] = gnorm; tr[2] = alpha_step; tr[3] = (double)Kcur;
      tr[4] = low_rank; tr[5] = recompute_fg; tr[6] = cand_accepted; tr[7] = trials;
    }

    const bool converged_after = std::isfinite(gnorm) && (gnorm < tol);
    const bool max_iter_reached = (iter + 1 >= max_iter);
    const bool invalid_after = !std::isfinite(objfn) || !std::isfinite(gnorm);
    const bool stop_after = converged_after || max_iter_reached || invalid_after;
    if (!stop_after) {
      shift = std::min(gnorm, shift_max);
      dual_sphess(density, shift * reg, !update);
    }
    niter = iter + 1;
    if (stop_after) {
      if (invalid_after) invalid_state = true;
      if (!max_iter_reached && converged_after) converged = true;
      break;
    }
  }

  *niter_out = niter;
  *converged_out = converged ? 1 : 0;
  if (P) transport_plan(M, gamma.data(), gamma.data() + n, P, reg, n, m);
  if (dual) std::copy(gamma.begin(), gamma.end(), dual);

  if (ctx_scalars) {
    const bool valid = !(invalid_state || !std::isfinite(objfn));
    const bool fallback = (niter == 0);
    ctx_scalars[0] = fallback ? 0.0 : ys;
    ctx_scalars[1] = (fallback ? false : low_rank) ? 1.0 : 0.0;
    ctx_scalars[2] = fallback ? 1.0 : 0.0;
    ctx_scalars[3] = valid ? 1.0 : 0.0;
    ctx_scalars[4] = (double)A.val.size();
    if (ctx_val && (long)A.val.size() <= ctx_cap) {
      std::copy(A.val.begin(), A.val.end(), ctx_val);
      std::copy(A.col.begin(), A.col.end(), ctx_col);
      std::copy(A.rowptr.begin(), A.rowptr.end(), ctx_rowptr);
    }
    if (ctx_s) std::copy(s.begin(), s.end(), ctx_s);
    if (ctx_y) std::copy(y.begin(), y.end(), ctx_y);
  }
  return 0;
}

}  // extern "C"
