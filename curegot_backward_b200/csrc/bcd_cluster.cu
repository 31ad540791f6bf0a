// Cluster-resident Sinkhorn BCD: one thread-block cluster solves one problem
// from start to finish in a single launch.
//
// Same iteration, stopping rule and niter semantics as the multi-CTA passes
// (bcd.cu; reference cuda_sinkhorn_bcd, src/sinkhorn_bcd_kernel.cu:429-634):
// gauge-normalised iterate difference until < 10 tol, then the row-marginal
// test of the current iterate, folded into the next row pass.
//
// Design (used for cost matrices of up to 768 KB, which fit the shared memory
// of one cluster of up to 16 CTAs; larger ones run faster on the multi-CTA
// passes, which spread each pass over every SM):
// * CTA r of the cluster owns a band of rows of M, copied once into its
//   shared memory; M is never read from HBM/L2 again.
// * Row pass: local to each CTA (warp per row, or several warps per row for
//   short bands), against a full local copy of the scaled beta.
// * Column pass: each CTA folds its band into per-column (max, sum) partials
//   in its shared memory; after a cluster barrier, CTA r merges the partials
//   of its slice of columns from all CTAs through distributed shared memory
//   (fixed rank order), and every CTA then pulls the new beta slices of the
//   others.
// * Stop test: every CTA publishes its partials (Chan statistics of the dual
//   changes, squared marginal errors) in its own shared memory; after a
//   barrier each CTA reads all of them in rank order and runs the control
//   logic itself, so every copy of the decision is identical and nothing is
//   broadcast.  The marginal test runs before the column pass, so a switch
//   from SFU to FP64 exponentials applies to that column pass already and
//   the last iteration skips it, as in the multi-CTA passes.
// Three cluster barriers per iteration and no global-memory traffic besides
// the first read of M and the final duals: small problems run in a few
// microseconds per iteration instead of two grid launches each.
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "bcd.cuh"
#include "lse.cuh"
#include "workspace.cuh"

namespace cg {

namespace cgx = cooperative_groups;

namespace {

constexpr int kCT = 512;        // threads per CTA
constexpr int kCW = kCT / 32;   // warps per CTA
constexpr int kMaxCluster = 16;
constexpr size_t kSmemMax = 225 * 1024;   // dynamic shared memory per CTA (opt-in)
constexpr size_t kBandTarget = 48 * 1024; // preferred bytes of M per CTA
// Largest M taken by the single-problem cluster path: above this the
// multi-CTA passes, which spread a pass over every SM, were as fast or faster
// on B200 (measured with profile_cases bcd).
constexpr size_t kClusterMaxBytes = 768 * 1024;

struct Ctrl {
  int iter, phase, check_pending, done, niter, fast, stall, fast_iters, nonfinite;
  double best_est, last_err, stat_a[3];
};

// Shared-memory layout of one CTA (identical on host and device).
struct CLayout {
  int nr, ldm, sl;
  size_t o_M, o_betas, o_colmx, o_cols, o_alpha, o_alphas, o_loga, o_bsl, o_logb, o_scr, o_wst,
      o_rowslot, o_colslot, o_ctrl, o_tab, o_stage, o_gath, total;
};

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~size_t(15); }

__host__ __device__ inline CLayout clayout(int n, int m, int C, int es) {
  CLayout L;
  const int vn = 16 / es;
  L.nr = (n + C - 1) / C;
  L.ldm = ((m + vn - 1) / vn) * vn;
  L.sl = (m + C - 1) / C;
  size_t o = 0;
  L.o_M = o;        o += al16((size_t)L.nr * L.ldm * es);
  L.o_betas = o;    o += al16((size_t)m * 8);
  L.o_colmx = o;    o += al16((size_t)m * 8);
  L.o_cols = o;     o += al16((size_t)m * 8);
  L.o_alpha = o;    o += al16((size_t)2 * L.nr * 8);
  L.o_alphas = o;   o += al16((size_t)2 * L.nr * 8);
  L.o_loga = o;     o += al16((size_t)L.nr * 8);
  L.o_bsl = o;      o += al16((size_t)2 * L.sl * 8);
  L.o_logb = o;     o += al16((size_t)L.sl * 8);
  L.o_scr = o;      o += al16((size_t)3 * kCT * 8);
  L.o_wst = o;      o += al16((size_t)kCW * 4 * 8);
  L.o_rowslot = o;  o += al16((size_t)kMaxCluster * 4 * 8);
  L.o_colslot = o;  o += al16((size_t)kMaxCluster * 3 * 8);
  L.o_ctrl = o;     o += al16(sizeof(Ctrl));
  L.o_tab = o;      o += al16(kExp2TableSize * 8);
  L.o_stage = o;    o += al16((size_t)2 * C * L.sl * 8);   // remote (max, sum) of the slice
  L.o_gath = o;     o += al16((size_t)kMaxCluster * 4 * 8); // remote row / column statistics
  L.total = o;
  return L;
}

__device__ __forceinline__ void welford(double& cnt, double& mean, double& m2, double x) {
  cnt += 1.0;
  const double d = x - mean;
  mean += d / cnt;
  m2 += d * (x - mean);
}

// Row segment [c0, c1) of one row held in shared memory.
template <typename TM, bool FAST>
__device__ __forceinline__ void row_seg_smem(const TM* __restrict__ Mrow,
                                             const double* __restrict__ betas, double s2, int c0,
                                             int c1, int lane, const double* tab, double& mx,
                                             double& s) {
  constexpr int VN = Vec<TM>::N;
  constexpr int U = (VN == 4) ? 2 : 4;
  using RT = typename Raw<TM>::T;
  for (int j0 = c0 + lane * VN; j0 < c1; j0 += 32 * VN * U) {
    double d[U * VN];
    bool ok[U * VN];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int j = j0 + u * 32 * VN;
      RT v;
      if (j < c1) v = *reinterpret_cast<const RT*>(Mrow + j);
#pragma unroll
      for (int k = 0; k < VN; ++k) {
        const bool in = (j + k) < c1;
        ok[u * VN + k] = in;
        d[u * VN + k] = in ? fma(-Raw<TM>::get(v, k), s2, betas[j + k]) : kNegInf;
      }
    }
    lse_chunk<FAST, U * VN>(d, ok, mx, s, tab);
  }
}

// Column partials over the CTA's band: (colmx[j], cols[j]) for all m columns.
template <typename TM, bool FAST>
__device__ void col_partials(const TM* __restrict__ Mb, int ldm, int nrr, int m,
                             const double* __restrict__ alphas, double s2, const double* tab,
                             double* __restrict__ colmx, double* __restrict__ cols,
                             double* __restrict__ scr) {
  int G = 1;
  while (G * 2 * m <= kCT && G * 2 <= nrr) G *= 2;
  const int cpr = kCT / G;
  const int g = threadIdx.x / cpr, c = threadIdx.x % cpr;
  for (int jb = 0; jb < m; jb += cpr) {
    const int j = jb + c;
    double mx = kNegInf, s = 0.0;
    if (j < m) {
      for (int i0 = g; i0 < nrr; i0 += 4 * G) {
        double d[4];
        bool ok[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int i = i0 + u * G;
          ok[u] = i < nrr;
          d[u] = ok[u] ? fma(-(double)Mb[(size_t)i * ldm + j], s2, alphas[i]) : kNegInf;
        }
        lse_chunk<FAST, 4>(d, ok, mx, s, tab);
      }
    }
    if (G == 1) {
      if (j < m) {
        colmx[j] = mx;
        cols[j] = s;
      }
    } else {
      scr[2 * threadIdx.x] = mx;
      scr[2 * threadIdx.x + 1] = s;
      __syncthreads();
      if (g == 0 && j < m) {
        for (int q = 1; q < G; ++q)
          lse2_merge(mx, s, scr[2 * (q * cpr + c)], scr[2 * (q * cpr + c) + 1], tab);
        colmx[j] = mx;
        cols[j] = s;
      }
      __syncthreads();
    }
  }
}

template <typename TM>
__global__ void __launch_bounds__(kCT, 1) bcd_cluster_kernel(const ClusterProb* __restrict__ probs,
                                                            int C) {
  extern __shared__ __align__(16) unsigned char smem[];
  cgx::cluster_group cluster = cgx::this_cluster();
  const int rank = (int)cluster.block_rank();
  const ClusterProb& P = probs[blockIdx.x / C];
  const int n = P.n, m = P.m;
  const CLayout L = clayout(n, m, C, (int)sizeof(TM));
  TM* Mb = reinterpret_cast<TM*>(smem + L.o_M);
  double* betas = reinterpret_cast<double*>(smem + L.o_betas);
  double* colmx = reinterpret_cast<double*>(smem + L.o_colmx);
  double* cols = reinterpret_cast<double*>(smem + L.o_cols);
  double* alpha = reinterpret_cast<double*>(smem + L.o_alpha);    // [2][nr]
  double* alphas = reinterpret_cast<double*>(smem + L.o_alphas);  // [2][nr]
  double* loga = reinterpret_cast<double*>(smem + L.o_loga);
  double* bsl = reinterpret_cast<double*>(smem + L.o_bsl);        // [2][sl]
  double* logb = reinterpret_cast<double*>(smem + L.o_logb);
  double* scr = reinterpret_cast<double*>(smem + L.o_scr);
  double* wst = reinterpret_cast<double*>(smem + L.o_wst);        // [kCW][4]
  double* rowslot = reinterpret_cast<double*>(smem + L.o_rowslot);
  double* colslot = reinterpret_cast<double*>(smem + L.o_colslot);
  Ctrl* ctrl = reinterpret_cast<Ctrl*>(smem + L.o_ctrl);
  double* tab = reinterpret_cast<double*>(smem + L.o_tab);
  double* stage = reinterpret_cast<double*>(smem + L.o_stage);  // [2][C][sl]
  double* gath = reinterpret_cast<double*>(smem + L.o_gath);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = rank * L.nr;
  const int nrr = max(0, min(L.nr, n - r0));
  const int j0 = rank * L.sl;
  const int nsl = max(0, min(L.sl, m - j0));
  const double s2 = P.s2, eta = P.eta;
  const TM* __restrict__ Mg = static_cast<const TM*>(P.M);

  // ---- set-up: band of M, marginal logs, initial duals, control ----------
  load_exp2_table(tab);
  bool nan_seen = false;
  for (size_t e = tid; e < (size_t)nrr * m; e += kCT) {
    const int i = (int)(e / m), j = (int)(e - (size_t)i * m);
    const TM v = Mg[(size_t)(r0 + i) * m + j];
    nan_seen |= (v != v);
    Mb[(size_t)i * L.ldm + j] = v;
  }
  // A NaN cost must not drop out of the sums like an infinite one (the
  // exponent clamp ignores NaN): the band's rows get a NaN log-marginal, so
  // the first iterate difference is NaN and every rank stops with
  // `nonfinite` on the same gathered values.
  nan_seen = __syncthreads_or(nan_seen) != 0;
  for (int i = tid; i < nrr; i += kCT) {
    loga[i] = nan_seen ? __longlong_as_double(0x7ff8000000000000LL) : log(P.a[r0 + i]);
    const double v = P.x0 ? P.x0[r0 + i] : 0.0;
    alpha[i] = v;
    alphas[i] = v * s2;
  }
  for (int j = tid; j < m; j += kCT) betas[j] = (P.x0 ? P.x0[n + j] : 0.0) * s2;
  for (int jj = tid; jj < nsl; jj += kCT) {
    logb[jj] = log(P.b[j0 + jj]);
    bsl[jj] = P.x0 ? P.x0[n + j0 + jj] : 0.0;
  }
  if (tid == 0) {
    Ctrl c{};
    c.iter = 0;
    c.phase = 1;
    c.check_pending = 0;
    c.done = (P.max_iter <= 0) ? 1 : 0;
    c.niter = 0;
    c.fast = (sizeof(TM) == 4) ? 1 : 0;
    c.stall = 0;
    c.fast_iters = 0;
    c.nonfinite = 0;
    c.best_est = INFINITY;
    c.last_err = 0.0;
    c.stat_a[0] = c.stat_a[1] = c.stat_a[2] = 0.0;
    *ctrl = c;
  }
  cluster.sync();

  // row-pass geometry: wpr warps per row
  int wpr = 1;
  while (wpr * 2 <= kCW && wpr * 2 * max(nrr, 1) <= kCW) wpr *= 2;
  const int slots = kCW / wpr;
  const int slot = warp / wpr, seg = warp % wpr;
  constexpr int VN = Vec<TM>::N;
  int chunk = (m + wpr - 1) / wpr;
  chunk = ((chunk + 32 * VN - 1) / (32 * VN)) * (32 * VN);
  const int c0 = seg * chunk, c1 = min(m, c0 + chunk);

  // Every rank keeps its own copy of the control state and updates it with
  // the same arithmetic on the same (remote-read) partials, in rank order, so
  // all copies stay identical and no rank has to broadcast a decision.
  while (true) {
    if (ctrl->done) break;
    const int t = ctrl->iter;
    const bool fast_row = ctrl->fast != 0;
    const bool check = ctrl->check_pending != 0;
    const int phase = ctrl->phase;
    const int cb = t & 1, nb = (t + 1) & 1;

    // ---- A: row pass (alpha^{t+1} of the band) ----------------------------
    double w_cnt = 0.0, w_mean = 0.0, w_m2 = 0.0, w_err = 0.0;
    for (int base = 0; base < nrr; base += slots) {
      const int i = base + slot;
      double mx = kNegInf, s = 0.0;
      if (i < nrr) {
        const TM* Mrow = Mb + (size_t)i * L.ldm;
        if (fast_row) row_seg_smem<TM, true>(Mrow, betas, s2, c0, c1, lane, tab, mx, s);
        else row_seg_smem<TM, false>(Mrow, betas, s2, c0, c1, lane, tab, mx, s);
      }
      double wmx = mx;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) wmx = fmax(wmx, __shfl_xor_sync(0xffffffffu, wmx, o));
      double sc = (s != 0.0) ? s * exp2_f64(mx - wmx, tab) : 0.0;
      sc = warp_sum_down(sc);
      if (wpr > 1) {
        if (lane == 0) {
          scr[2 * warp] = wmx;
          scr[2 * warp + 1] = sc;
        }
        __syncthreads();
      }
      if (lane == 0 && seg == 0 && i < nrr) {
        double M0 = wmx, S0 = sc;
        for (int q = 1; q < wpr; ++q) lse2_merge(M0, S0, scr[2 * (warp + q)], scr[2 * (warp + q) + 1], tab);
        const double a_new = eta * loga[i] - (eta * kLn2) * (M0 + log2(S0));
        const double as_new = a_new * s2;
        if (check) {
          const double ai = P.a[r0 + i];
          const double e = ai * exp2_f64(alphas[cb * L.nr + i] - as_new, tab) - ai;
          w_err += e * e;
        }
        welford(w_cnt, w_mean, w_m2, a_new - alpha[cb * L.nr + i]);
        alpha[nb * L.nr + i] = a_new;
        alphas[nb * L.nr + i] = as_new;
      }
      if (wpr > 1) __syncthreads();
    }
    if (lane == 0) {
      wst[warp * 4 + 0] = w_cnt;
      wst[warp * 4 + 1] = w_mean;
      wst[warp * 4 + 2] = w_m2;
      wst[warp * 4 + 3] = w_err;
    }
    __syncthreads();
    if (tid == 0) {
      double cn = 0, cmu = 0, cm2 = 0, ce = 0;
      for (int w = 0; w < kCW; ++w) {
        chan_combine(cn, cmu, cm2, wst[w * 4], wst[w * 4 + 1], wst[w * 4 + 2]);
        ce += wst[w * 4 + 3];
      }
      rowslot[0] = cn;
      rowslot[1] = cmu;
      rowslot[2] = cm2;
      rowslot[3] = ce;
    }
    cluster.sync();  // #1: row partials of every rank visible

    // ---- marginal test of iterate t, same decision on every rank ------------
    if (tid < 4 * C) gath[tid] = cluster.map_shared_rank(rowslot, tid >> 2)[tid & 3];
    __syncthreads();
    if (tid == 0) {
      const double* rp = gath;
      Ctrl c = *ctrl;
      if (phase == 1) {
        double an = 0, amu = 0, am2 = 0;
        for (int q = 0; q < C; ++q) chan_combine(an, amu, am2, rp[q * 4], rp[q * 4 + 1], rp[q * 4 + 2]);
        c.stat_a[0] = an;
        c.stat_a[1] = amu;
        c.stat_a[2] = am2;
      }
      if (check) {
        double tot = 0.0;
        for (int q = 0; q < C; ++q) tot += rp[q * 4 + 3];
        const double err = sqrt(tot);
        c.last_err = err;
        c.check_pending = 0;
        if (!isfinite(err)) {
          c.done = 1;
          c.nonfinite = 1;
          c.niter = t;
        } else if (!fast_row) {
          if (err < P.tol) {
            c.done = 1;
            c.niter = t;
          }
        } else if (err < 0.5 * P.tol) {
          c.fast = 0;
        } else if (err < 0.9 * c.best_est) {
          c.best_est = err;
          c.stall = 0;
        } else if (++c.stall >= 8) {
          c.fast = 0;
        }
      }
      *ctrl = c;
    }
    __syncthreads();
    if (ctrl->done) break;
    const bool fast_col = ctrl->fast != 0;

    // ---- B: column partials over the band with alpha^{t+1} ----------------
    if (fast_col)
      col_partials<TM, true>(Mb, L.ldm, nrr, m, alphas + nb * L.nr, s2, tab, colmx, cols, scr);
    else
      col_partials<TM, false>(Mb, L.ldm, nrr, m, alphas + nb * L.nr, s2, tab, colmx, cols, scr);
    cluster.sync();  // #2: column partials visible

    // ---- D: merge this CTA's column slice -> beta^{t+1} --------------------
    double b_cnt = 0.0, b_mean = 0.0, b_m2 = 0.0;
    // stage the slice's partials of every rank locally (all threads load)
    for (int e = tid; e < C * nsl; e += kCT) {
      const int q = e / nsl, jj = e - q * nsl;
      stage[e] = cluster.map_shared_rank(colmx, q)[j0 + jj];
      stage[C * nsl + e] = cluster.map_shared_rank(cols, q)[j0 + jj];
    }
    __syncthreads();
    for (int jj = tid; jj < nsl; jj += kCT) {
      const int j = j0 + jj;
      // max over ranks, then one sum of rescaled partials (rank order)
      double M0 = kNegInf;
      for (int q = 0; q < C; ++q)
        if (stage[C * nsl + q * nsl + jj] != 0.0) M0 = fmax(M0, stage[q * nsl + jj]);
      double S0 = 0.0;
      for (int q = 0; q < C; ++q) {
        const double sq = stage[C * nsl + q * nsl + jj];
        if (sq != 0.0) S0 += sq * exp2_f64(stage[q * nsl + jj] - M0, tab);
      }
      const double b_new = eta * logb[jj] - (eta * kLn2) * (M0 + log2(S0));
      welford(b_cnt, b_mean, b_m2, b_new - bsl[cb * L.sl + jj]);
      bsl[nb * L.sl + jj] = b_new;
      betas[j] = b_new * s2;
    }
    // warp Chan combine (fixed shuffle order), then the warps by thread 0
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double on = __shfl_down_sync(0xffffffffu, b_cnt, o);
      const double omu = __shfl_down_sync(0xffffffffu, b_mean, o);
      const double om2 = __shfl_down_sync(0xffffffffu, b_m2, o);
      if (lane + o < 32) chan_combine(b_cnt, b_mean, b_m2, on, omu, om2);
    }
    if (lane == 0) {
      wst[warp * 4 + 0] = b_cnt;
      wst[warp * 4 + 1] = b_mean;
      wst[warp * 4 + 2] = b_m2;
    }
    __syncthreads();
    if (tid == 0) {
      double bn = 0, bmu = 0, bm2 = 0;
      for (int w = 0; w < kCW; ++w) chan_combine(bn, bmu, bm2, wst[w * 4], wst[w * 4 + 1], wst[w * 4 + 2]);
      colslot[0] = bn;
      colslot[1] = bmu;
      colslot[2] = bm2;
    }
    cluster.sync();  // #3: new beta slices and column statistics visible

    // ---- F: gather beta; iterate-difference test, bookkeeping --------------
    for (int j = tid; j < m; j += kCT) {
      const int owner = j / L.sl;
      if (owner != rank) betas[j] = cluster.map_shared_rank(betas, owner)[j];
    }
    if (phase == 1 && tid < 3 * C) gath[tid] = cluster.map_shared_rank(colslot, tid / 3)[tid % 3];
    __syncthreads();
    if (tid == 0) {
      Ctrl c = *ctrl;
      const int tn = t + 1;
      if (phase == 1) {
        const double* cp = gath;
        double bn = 0, bmu = 0, bm2 = 0;
        for (int q = 0; q < C; ++q) chan_combine(bn, bmu, bm2, cp[q * 3], cp[q * 3 + 1], cp[q * 3 + 2]);
        const double an = c.stat_a[0], amu = c.stat_a[1], am2 = c.stat_a[2];
        const double K = (bn * bmu - an * amu) / (double)(n + m);
        const double ea = amu + K, eb = bmu - K;
        const double diff = sqrt(am2 + an * ea * ea + bm2 + bn * eb * eb);
        c.last_err = diff;
        if (diff < P.tol * 10) c.phase = 2;
        if (!isfinite(diff)) {
          c.done = 1;
          c.nonfinite = 1;
        }
      } else if (phase == 2) {
        c.check_pending = 1;
      }
      c.iter = tn;
      c.niter = tn;
      if (fast_col) c.fast_iters += 1;
      if (tn >= P.max_iter) c.done = 1;
      *ctrl = c;
    }
    __syncthreads();
  }
  cluster.sync();  // no CTA leaves while another may still read its shared memory

  // ---- outputs: iterate niter ----------------------------------------------
  const int ob = ctrl->niter & 1;
  if (P.dual) {
    for (int i = tid; i < nrr; i += kCT) P.dual[r0 + i] = alpha[ob * L.nr + i];
    for (int jj = tid; jj < nsl; jj += kCT) P.dual[n + j0 + jj] = bsl[ob * L.sl + jj];
  }
  if (rank == 0 && tid == 0) {
    BcdState* st = P.st;
    const Ctrl& c = *ctrl;
    st->iter = c.iter;
    st->phase = c.phase;
    st->check_pending = c.check_pending;
    st->done = 1;
    st->niter = c.niter;
    st->max_iter = P.max_iter;
    st->fast = c.fast;
    st->stall = c.stall;
    st->tol = P.tol;
    st->last_err = c.last_err;
    st->best_est = c.best_est;
    st->stat_a[0] = c.stat_a[0];
    st->stat_a[1] = c.stat_a[1];
    st->stat_a[2] = c.stat_a[2];
    st->fast_iters = c.fast_iters;
    st->nonfinite = c.nonfinite;
  }
}

std::atomic<int> g_cluster_enabled{1};

struct ClusterSupport {
  bool checked = false;
  int max_c = 0;  // largest supported cluster size at kSmemMax
};

template <typename TM>
int cluster_setup(int* max_c) {
  static std::mutex mu;
  static ClusterSupport sup[64];
  int dev = 0;
  CG_TRY_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return CG_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(mu);
  ClusterSupport& s = sup[dev];
  if (!s.checked) {
    s.checked = true;
    s.max_c = 0;
    auto fn = bcd_cluster_kernel<TM>;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemMax) !=
            cudaSuccess ||
        cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess) {
      cudaGetLastError();
    } else {
      for (int c = kMaxCluster; c >= 1; c /= 2) {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3(c, 1, 1);
        cfg.blockDim = dim3(kCT, 1, 1);
        cfg.dynamicSmemBytes = kSmemMax;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = c;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg) == cudaSuccess && nclusters > 0) {
          s.max_c = c;
          break;
        }
        cudaGetLastError();
      }
    }
  }
  *max_c = s.max_c;
  return CG_OK;
}

}  // namespace

int bcd_cluster_plan(int n, int m, int elem_bytes, int max_c) {
  if (n <= 0 || m <= 0) return 0;
  if ((size_t)n * m * elem_bytes > kClusterMaxBytes) return 0;
  int best = 0;
  for (int c = 1; c <= max_c && c <= n; c *= 2) {
    const CLayout L = clayout(n, m, c, elem_bytes);
    if (L.total > kSmemMax) continue;
    if (!best) best = c;
    const size_t band = (size_t)L.nr * L.ldm * elem_bytes;
    if (band <= kBandTarget) return c;
    best = c;
  }
  return best;
}

template <typename TM>
int bcd_cluster_eligible(int n, int m) {
  if (!g_cluster_enabled.load()) return 0;
  int max_c = 0;
  if (cluster_setup<TM>(&max_c) != CG_OK || max_c == 0) return 0;
  return bcd_cluster_plan(n, m, (int)sizeof(TM), max_c);
}

template <typename TM>
int launch_bcd_cluster(const ClusterProb* d_probs, int nprob, int C, cudaStream_t st) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(C * nprob), 1, 1);
  cfg.blockDim = dim3(kCT, 1, 1);
  cfg.dynamicSmemBytes = kSmemMax;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  CG_TRY_CUDA(cudaLaunchKernelEx(&cfg, bcd_cluster_kernel<TM>, d_probs, C));
  count_launch();
  return CG_OK;
}

bool bcd_cluster_enabled() { return g_cluster_enabled.load() != 0; }

int bcd_cluster_max(bool f32) {
  int max_c = 0;
  const int rc = f32 ? cluster_setup<float>(&max_c) : cluster_setup<double>(&max_c);
  return rc == CG_OK ? max_c : 0;
}

template int bcd_cluster_eligible<double>(int, int);
template int bcd_cluster_eligible<float>(int, int);
template int launch_bcd_cluster<double>(const ClusterProb*, int, int, cudaStream_t);
template int launch_bcd_cluster<float>(const ClusterProb*, int, int, cudaStream_t);

}  // namespace cg

extern "C" int cg_bcd_set_cluster_path(int enable) {
  cg::g_cluster_enabled.store(enable ? 1 : 0);
  return CG_OK;
}
