// Sinkhorn BCD on sm_100a: streaming row / column log-sum-exp passes with
// fused stop tests, batched over problems.
//
// Reference behaviour followed (benben-cd/curegot_backward):
//   optimal_alpha_kernel / optimal_beta_kernel  src/sinkhorn_bcd_kernel.cu:35-192
//   compute_iter_difference                     src/sinkhorn_bcd_kernel.cu:280-326
//   compute_marginal_a_kernel + l2 distance     src/sinkhorn_bcd_kernel.cu:329-353
//   cuda_sinkhorn_bcd loop                      src/sinkhorn_bcd_kernel.cu:532-592
//
// Design
// * Each half-step reads M exactly once, coalesced, in 16-byte vectors.  The
//   row pass is warp-per-row (up to 8 warps per row for short-n problems);
//   the column pass streams 512-byte column strips down the rows with one
//   online (max, sum) pair per column per lane, split over row ranges whose
//   partials are merged by the last CTA of each strip.
// * LSEs run in the base-2 exponent domain (duals are also kept scaled by
//   log2(e)/eta) with a running max updated once per 4-vector chunk, so the
//   exponentials are branch-free.  FP64 passes use exp2_f64 (table-driven,
//   ~2 ulp); mixed-precision passes round the max-shifted exponent (<= 0)
//   to FP32 once and evaluate it on the SFU (ex2.approx.ftz.f32).
// * The reference's third pass over M (row marginal for the stop test) is
//   folded into the next row pass:
//     rowsum_i(alpha^t, beta^t) = a_i * 2^(s2 * (alpha_i^t - alpha_i^{t+1})),
//   and the duals are double-buffered so the iterate that passes the test is
//   the one returned.
// * The gauge-normalised iterate difference is assembled from per-CTA
//   (count, mean, M2) statistics combined with Chan's formula (no
//   cancellation), so no pass needs a second sweep over the duals.
// * Every reduction has a fixed order: results are bitwise reproducible.
#include <algorithm>
#include <atomic>
#include <mutex>

#include "bcd.cuh"
#include "bulk.cuh"
#include "lse.cuh"

#ifndef CG_BCD_MINB
#define CG_BCD_MINB 3
#endif
// Resident CTAs per SM the row/column passes are compiled for (register cap).
constexpr int kBcdMinBlocks = CG_BCD_MINB;
// FP32-M vectors per lane per loop step of the row pass and rows per step of
// the column pass (4-float vectors; FP64 M takes 4 two-double vectors / rows).
#ifndef CG_F32_ROW_U
#define CG_F32_ROW_U 2
#endif
#ifndef CG_F32_COL_U
#define CG_F32_COL_U 4
#endif

namespace cg {

namespace {
// Elements per lane per step: 8 (two float4 or four double2 vectors).
template <typename TM>
struct RowU {
  static constexpr int U = (Vec<TM>::N == 4) ? CG_F32_ROW_U : 4;
};

// L2 bulk prefetch of the chunk [pos, min(pos + span, c1)) of a row whose
// 16-byte vectors are aligned (c1 is a multiple of the vector width).
template <typename TM>
__device__ __forceinline__ void prefetch_row_chunk(const TM* Mrow, int pos, int c1, int span) {
  if (pos < c1) prefetch_l2_bulk(Mrow + pos, (uint32_t)(min(span, c1 - pos) * (int)sizeof(TM)));
}

// One warp's segment [c0, c1) of row `row`: LSE over j of (betas_j - s2*M_ij).
// Full chunks run predicate-free with the next chunk's M vectors prefetched.
// CHECK (first pass of a solve): a NaN exponent (NaN in M or the duals) makes
// the row's sum NaN.  Without it a NaN entry would drop out of the sum like
// an infinite cost: the exponent clamp of the exponential ignores NaN.
// Float-pair form of a row chunk (FP32 M, SFU, shifted): U float4 vectors of
// M and their columns' (hi, lo) beta pairs at bp + u * step; k = the row's
// shift, s2 = s2h + s2l.  Same grouping as the FP64-argument chunk: one FP32
// partial per chunk, added to s.
template <int U>
__device__ __forceinline__ void split_chunk_row(const float4 (&mv)[U], const float2* __restrict__ bp,
                                                int step, float k, float s2h, float s2l,
                                                double& s) {
  float acc = 0.0f;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const float4 b01 = *reinterpret_cast<const float4*>(bp + u * step);
    const float4 b23 = *reinterpret_cast<const float4*>(bp + u * step + 2);
    acc += split_term(mv[u].x, b01.x, b01.y, k, s2h, s2l);
    acc += split_term(mv[u].y, b01.z, b01.w, k, s2h, s2l);
    acc += split_term(mv[u].z, b23.x, b23.y, k, s2h, s2l);
    acc += split_term(mv[u].w, b23.z, b23.w, k, s2h, s2l);
  }
  s += static_cast<double>(acc);
}

// Float pair (hi, lo) of a scaled dual; false when |v| >= kSplitMax or v is
// not finite (the pair is then unusable).
__device__ __forceinline__ bool split_of(double v, float2& out) {
  if (!(fabs(v) < kSplitMax)) {
    out = make_float2(0.0f, 0.0f);
    return false;
  }
  const double hi = rint(v * 512.0) * (1.0 / 512.0);
  out = make_float2(static_cast<float>(hi), static_cast<float>(v - hi));
  return true;
}

// SPLIT (FP32 M, FAST and SHIFT only): the full vector chunks take their
// exponents from the float-pair betas bsplit (split_chunk_row); the tail
// keeps the FP64-argument form.
template <typename TM, bool FAST, bool CHECK, bool SHIFT, bool SPLIT = false>
__device__ __forceinline__ void row_segment(const TM* __restrict__ Mrow,
                                            const double* __restrict__ betas, double s2, int c0,
                                            int c1, int lane, bool vec_ok, const double* tab,
                                            int pf, double& mx, double& s,
                                            const float2* __restrict__ bsplit = nullptr,
                                            float s2h = 0.0f, float s2l = 0.0f) {
  bool bad = false;
  constexpr int VN = Vec<TM>::N;
  if (vec_ok) {
    constexpr int U = RowU<TM>::U;
    constexpr int step = 32 * VN;
    constexpr int span = step * U;
    using RT = typename Raw<TM>::T;
    int cb = c0;
    RT nxt[U];
    if (cb + span <= c1) {
#pragma unroll
      for (int u = 0; u < U; ++u) nxt[u] = Raw<TM>::load(Mrow + cb + lane * VN + u * step);
    }
    // L2 prefetch pf chunks ahead (lane 0, one bulk hint per chunk); chunks
    // 0 and 1 are already on their way through the register prefetch.
    if (pf > 0 && lane == 0)
      for (int k = 2; k < pf; ++k) prefetch_row_chunk(Mrow, cb + k * span, c1, span);
    for (; cb + span <= c1; cb += span) {
      if (pf > 0 && lane == 0) prefetch_row_chunk(Mrow, cb + pf * span, c1, span);
      RT cur[U];
#pragma unroll
      for (int u = 0; u < U; ++u) cur[u] = nxt[u];
      if (cb + 2 * span <= c1) {
#pragma unroll
        for (int u = 0; u < U; ++u) nxt[u] = Raw<TM>::load(Mrow + cb + span + lane * VN + u * step);
      }
      if constexpr (SPLIT) {
        split_chunk_row<U>(cur, bsplit + cb + lane * VN, step, static_cast<float>(mx), s2h, s2l,
                           s);
      } else {
        double d[U * VN];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          double bv[VN];
          ld_duals<VN>(betas + cb + lane * VN + u * step, bv);
#pragma unroll
          for (int k = 0; k < VN; ++k) d[u * VN + k] = fma(-Raw<TM>::get(cur[u], k), s2, bv[k]);
        }
        if (CHECK)
#pragma unroll
          for (int q = 0; q < U * VN; ++q) bad |= (d[q] != d[q]);
        lse_chunk_full<FAST, U * VN, SHIFT>(d, mx, s, tab);
      }
    }
    // tail (vectors that are in range, then nothing: c1 is a multiple of VN)
    for (int j = cb + lane * VN; j < c1; j += step) {
      double d[VN];
      bool ok[VN];
      double mv[VN], bv[VN];
      Vec<TM>::load(Mrow + j, mv);
      ld_duals<VN>(betas + j, bv);
#pragma unroll
      for (int k = 0; k < VN; ++k) {
        ok[k] = true;
        d[k] = fma(-mv[k], s2, bv[k]);
      }
      if (CHECK)
#pragma unroll
        for (int q = 0; q < VN; ++q) bad |= (d[q] != d[q]);
      lse_chunk<FAST, VN, SHIFT>(d, ok, mx, s, tab);
    }
  } else {
    for (int j0 = c0 + lane; j0 < c1; j0 += 32 * kUnroll) {
      double d[kUnroll];
      bool ok[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const int j = j0 + u * 32;
        ok[u] = j < c1;
        d[u] = ok[u] ? fma(-ld1(Mrow + j), s2, betas[j]) : kNegInf;
      }
      if (CHECK)
#pragma unroll
        for (int q = 0; q < kUnroll; ++q) bad |= (ok[q] && d[q] != d[q]);
      lse_chunk<FAST, kUnroll, SHIFT>(d, ok, mx, s, tab);
    }
  }
  if (CHECK && bad) s = __longlong_as_double(0x7ff8000000000000LL);
}

// row_segment for rows whose 16-byte vectors are aligned (vec_ok) and long
// enough to stream: the whole spans of [c0, c1) reach shared memory through
// the warp's ring (bulk copies issued kRingStages chunks ahead, so the HBM
// latency is covered without registers held by in-flight loads), then each
// span is processed exactly like row_segment's loop body -- same grouping,
// same order, bitwise the same (mx, s).  The tail (< one span) is read as in
// row_segment.  A ring wait that gives up leaves ring.failed set.
template <typename TM, bool FAST, bool CHECK, bool SHIFT, bool SPLIT = false>
__device__ __forceinline__ void row_segment_staged(const TM* __restrict__ Mrow,
                                                   const double* __restrict__ betas, double s2,
                                                   int c0, int c1, int lane, const double* tab,
                                                   WarpRing& ring, double& mx, double& s,
                                                   const float2* __restrict__ bsplit = nullptr,
                                                   float s2h = 0.0f, float s2l = 0.0f) {
  bool bad = false;
  constexpr int VN = Vec<TM>::N;
  constexpr int U = RowU<TM>::U;
  constexpr int step = 32 * VN;
  constexpr int span = step * U;
  constexpr int span_bytes = span * (int)sizeof(TM);
  constexpr int SPC = kRingBytes / span_bytes;  // spans per ring chunk
  static_assert(SPC >= 1 && kRingBytes % span_bytes == 0, "ring chunk size");
  using RT = typename Raw<TM>::T;
  const int nspans = (c1 - c0) / span;
  const int nchunks = (nspans + SPC - 1) / SPC;
  const uint32_t g0 = ring.issued;
  auto issue = [&](int k) {  // lane 0
    const int sp0 = k * SPC;
    const uint32_t bytes = (uint32_t)min(SPC, nspans - sp0) * span_bytes;
    const uint32_t g = g0 + (uint32_t)k;
    mbar_expect_tx(ring.barrier(g), bytes);
    bulk_g2s(ring.stage(g), Mrow + c0 + (size_t)sp0 * span, bytes, ring.barrier(g));
  };
  const int pre = min(nchunks, kRingStages);
  if (lane == 0)
    for (int k = 0; k < pre; ++k) issue(k);
  ring.issued = g0 + (uint32_t)pre;
  for (int k = 0; k < nchunks; ++k) {
    if (!ring.wait_next()) {
      ring.drain();
      return;
    }
    const RT* chunk = reinterpret_cast<const RT*>(ring.stage(ring.consumed));
    const int sp0 = k * SPC, nsp = min(SPC, nspans - sp0);
    for (int q = 0; q < nsp; ++q) {
      const int cb = c0 + (sp0 + q) * span;
      if constexpr (SPLIT) {
        RT v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) v[u] = chunk[q * (span / VN) + u * 32 + lane];
        split_chunk_row<U>(v, bsplit + cb + lane * VN, step, static_cast<float>(mx), s2h, s2l, s);
      } else {
        double d[U * VN];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const RT v = chunk[q * (span / VN) + u * 32 + lane];
          double bv[VN];
          ld_duals<VN>(betas + cb + lane * VN + u * step, bv);
#pragma unroll
          for (int kk = 0; kk < VN; ++kk) d[u * VN + kk] = fma(-Raw<TM>::get(v, kk), s2, bv[kk]);
        }
        if (CHECK)
#pragma unroll
          for (int q = 0; q < U * VN; ++q) bad |= (d[q] != d[q]);
        lse_chunk_full<FAST, U * VN, SHIFT>(d, mx, s, tab);
      }
    }
    ring.consumed++;
    __syncwarp();
    if (k + kRingStages < nchunks) {
      if (lane == 0) {
        fence_proxy_async_smem();  // this stage's reads before the copy that refills it
        issue(k + kRingStages);
      }
      ring.issued++;
    }
  }
  for (int j = c0 + nspans * span + lane * VN; j < c1; j += step) {
    double d[VN];
    bool ok[VN];
    double mv[VN], bv[VN];
    Vec<TM>::load(Mrow + j, mv);
    ld_duals<VN>(betas + j, bv);
#pragma unroll
    for (int k = 0; k < VN; ++k) {
      ok[k] = true;
      d[k] = fma(-mv[k], s2, bv[k]);
    }
    if (CHECK)
#pragma unroll
      for (int q = 0; q < VN; ++q) bad |= (d[q] != d[q]);
    lse_chunk<FAST, VN, SHIFT>(d, ok, mx, s, tab);
  }
  if (CHECK && bad) s = __longlong_as_double(0x7ff8000000000000LL);
}

// CTA-wide Chan combine; thread 0 ends with the total.  sh: 3 * kThreads.
__device__ __forceinline__ void cta_chan(double& n, double& mu, double& m2, double* sh) {
  const int t = threadIdx.x;
  __syncthreads();
  sh[t] = n;
  sh[kThreads + t] = mu;
  sh[2 * kThreads + t] = m2;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (t < w) {
      double a = sh[t], b = sh[kThreads + t], c = sh[2 * kThreads + t];
      chan_combine(a, b, c, sh[t + w], sh[kThreads + t + w], sh[2 * kThreads + t + w]);
      sh[t] = a;
      sh[kThreads + t] = b;
      sh[2 * kThreads + t] = c;
    }
    __syncthreads();
  }
  n = sh[0];
  mu = sh[kThreads];
  m2 = sh[2 * kThreads];
}

// Two-pass (count, mean, M2) of v over the CTA (invalid entries skipped).
__device__ __forceinline__ void cta_stats(double v, bool valid, double* red, double& n,
                                          double& mu, double& m2) {
  __shared__ double sh_mu;
  const double cnt = cta_sum(valid ? 1.0 : 0.0, red);
  const double sum = cta_sum(valid ? v : 0.0, red);
  if (threadIdx.x == 0) sh_mu = (cnt > 0) ? sum / cnt : 0.0;
  __syncthreads();
  const double mean = sh_mu;
  const double dv = valid ? (v - mean) : 0.0;
  const double q = cta_sum(dv * dv, red);
  n = cnt;
  mu = mean;
  m2 = q;
}
}  // namespace

template <typename TM, bool FAST, bool CHECK, bool SHIFT, bool SPLIT = false>
__device__ __forceinline__ void row_any(bool use_ring, const TM* __restrict__ Mrow,
                                        const double* __restrict__ betas, double s2, int c0,
                                        int c1, int lane, bool vec_ok, const double* tab, int pf,
                                        WarpRing& ring, double& mx, double& s,
                                        const float2* __restrict__ bsplit = nullptr,
                                        float s2h = 0.0f, float s2l = 0.0f) {
  if (use_ring)
    row_segment_staged<TM, FAST, CHECK, SHIFT, SPLIT>(Mrow, betas, s2, c0, c1, lane, tab, ring,
                                                      mx, s, bsplit, s2h, s2l);
  else
    row_segment<TM, FAST, CHECK, SHIFT, SPLIT>(Mrow, betas, s2, c0, c1, lane, vec_ok, tab, pf,
                                               mx, s, bsplit, s2h, s2l);
}

// ---------------------------------------------------------------------------
// Row pass: alpha^{t+1}_i = eta * (log a_i - LSE_j((beta^t_j - M_ij) / eta))
// ---------------------------------------------------------------------------
// One virtual CTA (index vb) of the row pass.
template <typename TM>
__device__ __forceinline__ void row_block(const BcdProb* __restrict__ probs,
                                          const int* __restrict__ cta_prob,
                                          const int* __restrict__ cta_start, int vb,
                                          int flags, WarpRing& ring) {
  const bool staged = (flags & kPassStaged) != 0;
  const bool online = (flags & kPassOnline) != 0;
  const int pf = flags >> kPassPrefetchShift;
  __shared__ double tab[kExp2TableSize];
  __shared__ double sm_mx[kWarps], sm_s[kWarps];
  __shared__ double sm_v[kWarps][2];
  __shared__ double red[kWarps];
  __shared__ double shc[3 * kThreads];
  load_exp2_table(tab);

  const int pidx = cta_prob ? cta_prob[vb] : 0;
  const int cta = cta_prob ? vb - cta_start[pidx] : vb;
  const BcdProb& P = probs[pidx];
  BcdState* st = P.st;
  if (ldcg(&st->done)) return;
  const int t = ldcg(&st->iter);
  const bool check = ldcg(&st->check_pending) != 0;
  const bool fast = ldcg(&st->fast) != 0;
  const int phase = ldcg(&st->phase);
  const double drift_b = ldcg(&st->drift_b);
  const bool split_ok = P.bsplit != nullptr && ldcg(&st->split_bad_b) == 0;
  __syncthreads();

  const int n = P.n, m = P.m;
  const TM* __restrict__ M = static_cast<const TM*>(P.M);
  const double* __restrict__ betas = P.betas[t & 1];
  const double* __restrict__ alphas_cur = P.alphas[t & 1];
  const double* __restrict__ alpha_cur = P.alpha[t & 1];
  const double s2 = P.s2;
  const float s2h = static_cast<float>(s2);
  const float s2l = static_cast<float>(s2 - static_cast<double>(s2h));

  const int R = P.rows_per_cta;
  const int wpr = kWarps / R;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int rloc = warp / wpr, seg = warp % wpr;
  const int row = cta * R + rloc;

  constexpr int VN = Vec<TM>::N;
  const bool vec_ok = (m % VN) == 0 && (reinterpret_cast<uintptr_t>(M) % 16) == 0;

  double mx = kNegInf, s = 0.0;
  if (row < n) {
    const int step = 32 * VN;
    int chunk = (m + wpr - 1) / wpr;
    chunk = ((chunk + step - 1) / step) * step;
    const int c0 = seg * chunk;
    const int c1 = min(m, c0 + chunk);
    const TM* __restrict__ Mrow = M + (size_t)row * m;
    // stream through the ring when the segment holds at least two chunks
    const bool use_ring = staged && vec_ok && (c1 - c0) * (int)sizeof(TM) >= 2 * kRingBytes;
    // Mode: the first pass also flags NaN exponents (online maximum); later
    // passes sum relative to the row's previous LSE, log2 a_i - alphas^t_i,
    // when the column duals moved by less than kShiftDrift since it was taken.
    // With FP32 M, SFU passes and float-pair betas in range, the shifted
    // exponents are formed in FP32 from the pairs (mode 3).
    int mode = 1;
    if (t == 0) {
      mode = 0;
    } else if (!online && drift_b < kShiftDrift) {
      const double sh = rint(P.loga[row] * kLog2e - alphas_cur[row]);
      if (fabs(sh) < 1.0e6) {
        mx = sh;
        mode = 2;
        if (sizeof(TM) == 4 && fast && split_ok && fabs(sh) < kSplitMax) mode = 3;
      }
    }
    if (fast) {
      if (mode == 0) row_any<TM, true, true, false>(use_ring, Mrow, betas, s2, c0, c1, lane, vec_ok, tab, pf, ring, mx, s);
      else if (mode == 1) row_any<TM, true, false, false>(use_ring, Mrow, betas, s2, c0, c1, lane, vec_ok, tab, pf, ring, mx, s);
      else if (mode == 2) row_any<TM, true, false, true>(use_ring, Mrow, betas, s2, c0, c1, lane, vec_ok, tab, pf, ring, mx, s);
      else row_any<TM, true, false, true, sizeof(TM) == 4>(use_ring, Mrow, betas, s2, c0, c1, lane, vec_ok, tab, pf, ring, mx, s, P.bsplit, s2h, s2l);
    } else {
      if (mode == 0) row_any<TM, false, true, false>(use_ring, Mrow, betas, s2, c0, c1, lane, vec_ok, tab, pf, ring, mx, s);
      else if (mode == 1) row_any<TM, false, false, false>(use_ring, Mrow, betas, s2, c0, c1, lane, vec_ok, tab, pf, ring, mx, s);
      else row_any<TM, false, false, true>(use_ring, Mrow, betas, s2, c0, c1, lane, vec_ok, tab, pf, ring, mx, s);
    }
  }
  if (ring.failed && lane == 0) {
    // a staging wait gave up: the problem ends with an error status
    atomicExch(&st->error, 1);
    atomicExch(&st->done, 1);
  }
  // warp combine: exact max by butterfly, then one rescale and a sum tree
  double wmx = mx;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) wmx = fmax(wmx, __shfl_xor_sync(0xffffffffu, wmx, o));
  double sc = (s != 0.0) ? s * exp2_f64(mx - wmx, tab) : 0.0;
  sc = warp_sum_down(sc);
  if (lane == 0) {
    sm_mx[warp] = wmx;
    sm_s[warp] = sc;
  }
  __syncthreads();
  if (lane == 0 && seg == 0) {
    double err2 = 0.0, da = 0.0;
    if (row < n) {
      double M0 = sm_mx[warp], S0 = sm_s[warp];
      for (int q = 1; q < wpr; ++q) lse2_merge(M0, S0, sm_mx[warp + q], sm_s[warp + q], tab);
      const double a_new = P.eta * P.loga[row] - (P.eta * kLn2) * (M0 + log2(S0));
      const double as_new = a_new * s2;
      P.alpha[(t + 1) & 1][row] = a_new;
      P.alphas[(t + 1) & 1][row] = as_new;
      if (P.asplit != nullptr && !split_of(as_new, P.asplit[row])) atomicOr(&st->split_bad_a, 1);
      if (check) {
        const double ai = P.a[row];
        const double e = ai * exp2_f64(alphas_cur[row] - as_new, tab) - ai;
        err2 = e * e;
      }
      da = a_new - alpha_cur[row];
    }
    sm_v[rloc][0] = err2;
    sm_v[rloc][1] = da;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double acc = 0.0, cnt = 0.0, sum = 0.0;
    for (int q = 0; q < R; ++q) {
      acc += sm_v[q][0];
      if (cta * R + q < n) {
        cnt += 1.0;
        sum += sm_v[q][1];
      }
    }
    const double mean = cnt > 0 ? sum / cnt : 0.0;
    double m2 = 0.0;
    for (int q = 0; q < R; ++q)
      if (cta * R + q < n) {
        const double dd = sm_v[q][1] - mean;
        m2 += dd * dd;
      }
    double* out = P.row_part + (size_t)cta * 4;
    out[0] = cnt;
    out[1] = mean;
    out[2] = m2;
    out[3] = acc;
    // largest |alphas change| of the CTA's rows (NaN orders above +inf)
    unsigned long long dbits = 0ull;
    for (int q = 0; q < R; ++q)
      if (cta * R + q < n) {
        const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(sm_v[q][1] * s2));
        dbits = b > dbits ? b : dbits;
      }
    atomicMax(&st->acc_a, dbits);
  }
  if (!elect_last(&P.counters[0], (unsigned)P.row_ctas)) return;
  if (threadIdx.x == 0) {
    st->drift_a = __longlong_as_double((long long)atomicExch(&st->acc_a, 0ull));
    st->split_bad_b = 0;  // every CTA of this pass has read it
  }

  // Last CTA of the row pass.
  if (phase == 1) {
    double cn = 0, cmu = 0, cm2 = 0;
    for (int q0 = threadIdx.x; q0 < P.row_ctas; q0 += 4 * blockDim.x) {
      double bn[4], bmu[4], bm2[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int q = q0 + u * blockDim.x;
        const bool in = q < P.row_ctas;
        bn[u] = in ? ldcg(P.row_part + (size_t)q * 4) : 0.0;
        bmu[u] = in ? ldcg(P.row_part + (size_t)q * 4 + 1) : 0.0;
        bm2[u] = in ? ldcg(P.row_part + (size_t)q * 4 + 2) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) chan_combine(cn, cmu, cm2, bn[u], bmu[u], bm2[u]);
    }
    cta_chan(cn, cmu, cm2, shc);
    if (threadIdx.x == 0) {
      st->stat_a[0] = cn;
      st->stat_a[1] = cmu;
      st->stat_a[2] = cm2;
    }
  }
  if (check) {
    double v = 0.0;
    for (int q = threadIdx.x; q < P.row_ctas; q += blockDim.x) v += ldcg(P.row_part + (size_t)q * 4 + 3);
    const double tot = cta_sum(v, red);
    if (threadIdx.x == 0) {
      // Marginal test of iterate t (reference :568-589).
      const double err = sqrt(tot);
      st->last_err = err;
      st->check_pending = 0;
      if (!isfinite(err)) {
        // non-finite marginal: no later iterate can pass the test
        st->done = 1;
        st->nonfinite = 1;
        st->niter = t;
      } else if (!fast) {
        if (err < st->tol) {
          st->done = 1;
          st->niter = t;
        }
      } else {
        // Mixed precision: the SFU estimate only decides when to switch to
        // FP64 passes; convergence is always confirmed by an FP64 test.
        if (err < 0.5 * st->tol) {
          st->fast = 0;
        } else if (err < 0.9 * st->best_est) {
          st->best_est = err;
          st->stall = 0;
        } else if (++st->stall >= 8) {
          st->fast = 0;
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Column pass: beta^{t+1}_j = eta * (log b_j - LSE_i((alpha^{t+1}_i - M_ij)/eta))
// ---------------------------------------------------------------------------
// pf > 0: lanes 0..U-1 also send the strip segments of the rows pf steps
// ahead to L2 (one bulk hint of strip_bytes per row, from column strip_c0).
// Float-pair form of a column group (FP32 M, SFU, shifted): U rows' float4
// vectors, the rows' (hi, lo) alpha pairs, this lane's column shifts k[].
// Same grouping as the FP64-argument group: per column one FP32 partial over
// the U rows, added to s[column].
template <int U>
__device__ __forceinline__ void split_group_col(const float4 (&mv)[U], const float2 (&ap)[U],
                                                const float (&k)[4], float s2h, float s2l,
                                                double* s) {
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int u = 0; u < U; ++u) {
    acc[0] += split_term(mv[u].x, ap[u].x, ap[u].y, k[0], s2h, s2l);
    acc[1] += split_term(mv[u].y, ap[u].x, ap[u].y, k[1], s2h, s2l);
    acc[2] += split_term(mv[u].z, ap[u].x, ap[u].y, k[2], s2h, s2l);
    acc[3] += split_term(mv[u].w, ap[u].x, ap[u].y, k[3], s2h, s2l);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) s[q] += static_cast<double>(acc[q]);
}

// SPLIT (FP32 M, FAST and SHIFT only): the full row groups take their
// exponents from the float-pair alphas asplit (split_group_col); the
// remaining rows keep the FP64-argument form.
template <typename TM, bool FAST, bool SHIFT, bool SPLIT = false>
__device__ __forceinline__ void col_rows(const TM* __restrict__ M, const double* __restrict__ alphas,
                                         double s2, int m, int jb, int r0, int r1, int warp,
                                         bool vec_ok, const double* tab, int pf, int strip_c0,
                                         int strip_bytes, double* mx, double* s,
                                         const float2* __restrict__ asplit = nullptr,
                                         float s2h = 0.0f, float s2l = 0.0f) {
  constexpr int VN = Vec<TM>::N;
  constexpr int U = (VN == 4) ? CG_F32_COL_U : 4;  // rows per lane per step
  constexpr int rstep = kWarps * U;
  const int lane = threadIdx.x & 31;
  if (vec_ok) {
    using RT = typename Raw<TM>::T;
    int i0 = r0 + warp;
    RT nxt[U];
    if (i0 + (U - 1) * kWarps < r1) {
#pragma unroll
      for (int u = 0; u < U; ++u) nxt[u] = Raw<TM>::load(M + (size_t)(i0 + u * kWarps) * m + jb);
    }
    if (pf > 0 && lane < U)
      for (int k = 2; k < pf; ++k) {
        const int i = i0 + k * rstep + lane * kWarps;
        if (i < r1) prefetch_l2_bulk(M + (size_t)i * m + strip_c0, (uint32_t)strip_bytes);
      }
    for (; i0 + (U - 1) * kWarps < r1; i0 += rstep) {
      if (pf > 0 && lane < U) {
        const int i = i0 + pf * rstep + lane * kWarps;
        if (i < r1) prefetch_l2_bulk(M + (size_t)i * m + strip_c0, (uint32_t)strip_bytes);
      }
      RT cur[U];
#pragma unroll
      for (int u = 0; u < U; ++u) cur[u] = nxt[u];
      if (i0 + rstep + (U - 1) * kWarps < r1) {
#pragma unroll
        for (int u = 0; u < U; ++u)
          nxt[u] = Raw<TM>::load(M + (size_t)(i0 + rstep + u * kWarps) * m + jb);
      }
      if constexpr (SPLIT) {
        float2 ap[U];
#pragma unroll
        for (int u = 0; u < U; ++u) ap[u] = asplit[i0 + u * kWarps];
        const float kf[4] = {static_cast<float>(mx[0]), static_cast<float>(mx[1]),
                             static_cast<float>(mx[2]), static_cast<float>(mx[3])};
        split_group_col<U>(cur, ap, kf, s2h, s2l, s);
      } else {
        double ai[U];
#pragma unroll
        for (int u = 0; u < U; ++u) ai[u] = alphas[i0 + u * kWarps];
#pragma unroll
        for (int k = 0; k < VN; ++k) {
          double d[U];
#pragma unroll
          for (int u = 0; u < U; ++u) d[u] = fma(-Raw<TM>::get(cur[u], k), s2, ai[u]);
          lse_chunk_full<FAST, U, SHIFT>(d, mx[k], s[k], tab);
        }
      }
    }
    // remaining rows of this warp (fewer than U)
    for (int i = i0; i < r1; i += kWarps) {
      const double ai = alphas[i];
      double mv[VN];
      Vec<TM>::load(M + (size_t)i * m + jb, mv);
#pragma unroll
      for (int k = 0; k < VN; ++k) {
        double d[1] = {fma(-mv[k], s2, ai)};
        bool ok[1] = {true};
        lse_chunk<FAST, 1, SHIFT>(d, ok, mx[k], s[k], tab);
      }
    }
  } else {
    for (int i = r0 + warp; i < r1; i += kWarps) {
      const double ai = alphas[i];
      const TM* p = M + (size_t)i * m + jb;
#pragma unroll
      for (int k = 0; k < VN; ++k) {
        double d[1];
        bool ok[1] = {jb + k < m};
        d[0] = ok[0] ? fma(-ld1(p + k), s2, ai) : kNegInf;
        lse_chunk<FAST, 1, SHIFT>(d, ok, mx[k], s[k], tab);
      }
    }
  }
}

// col_rows for strips whose 16-byte vectors are aligned (vec_ok): the warp's
// full U-row groups reach shared memory through its ring, kRingBytes / 512
// rows (one 512-byte strip segment each) per chunk, and are processed
// exactly like col_rows's loop body -- same groups, same order, bitwise the
// same (mx, s).  The remaining rows (fewer than U) are read as in col_rows.
// lane_in: this lane's columns exist (the last strip may be partial);
// strip_bytes: bytes of the strip in one row.
template <typename TM, bool FAST, bool SHIFT, bool SPLIT = false>
__device__ __forceinline__ void col_rows_staged(const TM* __restrict__ M,
                                                const double* __restrict__ alphas, double s2,
                                                int m, int strip_c0, int strip_bytes, int jb,
                                                bool lane_in, int r0, int r1, int warp, int lane,
                                                const double* tab, WarpRing& ring, double* mx,
                                                double* s, const float2* __restrict__ asplit = nullptr,
                                                float s2h = 0.0f, float s2l = 0.0f) {
  constexpr int VN = Vec<TM>::N;
  constexpr int U = (VN == 4) ? CG_F32_COL_U : 4;
  constexpr int RPC = kRingBytes / 512;  // warp rows per ring chunk
  static_assert(RPC % U == 0, "ring chunk must hold whole row groups");
  using RT = typename Raw<TM>::T;
  const int i_first = r0 + warp;
  const int nr = (r1 > i_first) ? (r1 - i_first + kWarps - 1) / kWarps : 0;
  const int grouped = (nr / U) * U;  // rows taken in full groups
  const int nchunks = (grouped + RPC - 1) / RPC;
  const uint32_t g0 = ring.issued;
  auto issue = [&](int k) {  // lane 0
    const int q0 = k * RPC, nq = min(RPC, grouped - q0);
    const uint32_t g = g0 + (uint32_t)k;
    mbar_expect_tx(ring.barrier(g), (uint32_t)(nq * strip_bytes));
    unsigned char* dst = ring.stage(g);
    for (int q = 0; q < nq; ++q)
      bulk_g2s(dst + q * 512, M + (size_t)(i_first + (q0 + q) * kWarps) * m + strip_c0,
               (uint32_t)strip_bytes, ring.barrier(g));
  };
  const int pre = min(nchunks, kRingStages);
  if (lane == 0)
    for (int k = 0; k < pre; ++k) issue(k);
  ring.issued = g0 + (uint32_t)pre;
  for (int k = 0; k < nchunks; ++k) {
    if (!ring.wait_next()) {
      ring.drain();
      return;
    }
    const unsigned char* chunk = ring.stage(ring.consumed);
    const int q0 = k * RPC, nq = min(RPC, grouped - q0);
    if (lane_in) {
      for (int qg = 0; qg < nq; qg += U) {
        RT cur[U];
#pragma unroll
        for (int u = 0; u < U; ++u) cur[u] = reinterpret_cast<const RT*>(chunk + (qg + u) * 512)[lane];
        if constexpr (SPLIT) {
          float2 ap[U];
#pragma unroll
          for (int u = 0; u < U; ++u) ap[u] = asplit[i_first + (q0 + qg + u) * kWarps];
          const float kf[4] = {static_cast<float>(mx[0]), static_cast<float>(mx[1]),
                               static_cast<float>(mx[2]), static_cast<float>(mx[3])};
          split_group_col<U>(cur, ap, kf, s2h, s2l, s);
        } else {
          double ai[U];
#pragma unroll
          for (int u = 0; u < U; ++u) ai[u] = alphas[i_first + (q0 + qg + u) * kWarps];
#pragma unroll
          for (int kk = 0; kk < VN; ++kk) {
            double d[U];
#pragma unroll
            for (int u = 0; u < U; ++u) d[u] = fma(-Raw<TM>::get(cur[u], kk), s2, ai[u]);
            lse_chunk_full<FAST, U, SHIFT>(d, mx[kk], s[kk], tab);
          }
        }
      }
    }
    ring.consumed++;
    __syncwarp();
    if (k + kRingStages < nchunks) {
      if (lane == 0) {
        fence_proxy_async_smem();  // this stage's reads before the copy that refills it
        issue(k + kRingStages);
      }
      ring.issued++;
    }
  }
  if (!lane_in) return;
  for (int i = i_first + grouped * kWarps; i < r1; i += kWarps) {
    const double ai = alphas[i];
    double mv[VN];
    Vec<TM>::load(M + (size_t)i * m + jb, mv);
#pragma unroll
    for (int kk = 0; kk < VN; ++kk) {
      double d[1] = {fma(-mv[kk], s2, ai)};
      bool ok[1] = {true};
      lse_chunk<FAST, 1, SHIFT>(d, ok, mx[kk], s[kk], tab);
    }
  }
}

// One virtual CTA (index vb) of the column pass.
template <typename TM>
__device__ __forceinline__ void col_block(const BcdProb* __restrict__ probs,
                                          const int* __restrict__ cta_prob,
                                          const int* __restrict__ cta_start, int vb,
                                          int flags, WarpRing& ring) {
  const bool staged = (flags & kPassStaged) != 0;
  const bool online = (flags & kPassOnline) != 0;
  const int pf = flags >> kPassPrefetchShift;
  constexpr int VN = Vec<TM>::N;
  constexpr int W = 32 * VN;
  constexpr int G = kThreads / W;  // merge groups per column
  __shared__ double tab[kExp2TableSize];
  __shared__ double sm_mx[kWarps][W];
  __shared__ double sm_s[kWarps][W];
  __shared__ double red[kWarps];
  __shared__ double shc[3 * kThreads];
  load_exp2_table(tab);

  const int pidx = cta_prob ? cta_prob[vb] : 0;
  const int cta = cta_prob ? vb - cta_start[pidx] : vb;
  const BcdProb& P = probs[pidx];
  BcdState* st = P.st;
  if (ldcg(&st->done)) return;
  const int t = ldcg(&st->iter);
  const bool fast = ldcg(&st->fast) != 0;
  const int phase = ldcg(&st->phase);
  const double drift_a = ldcg(&st->drift_a);
  const bool split_a_ok = P.asplit != nullptr && ldcg(&st->split_bad_a) == 0;
  __syncthreads();

  const int n = P.n, m = P.m;
  const TM* __restrict__ M = static_cast<const TM*>(P.M);
  const double* __restrict__ alphas = P.alphas[(t + 1) & 1];
  const double s2 = P.s2;

  const int strip = cta % P.col_strips;
  const int split = cta / P.col_strips;
  const int rows_per = (n + P.col_splits - 1) / P.col_splits;
  const int r0 = split * rows_per, r1 = min(n, r0 + rows_per);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int jb = strip * W + lane * VN;
  const bool vec_ok = (m % VN) == 0 && (reinterpret_cast<uintptr_t>(M) % 16) == 0;

  // Mode: from the second pass on, each column sums relative to its previous
  // LSE, log2 b_j - betas^t_j, when the row duals of this iteration moved by
  // less than kShiftDrift; the CTA takes the online maximum if any of its
  // columns has no usable shift.
  const double* __restrict__ betas_cur = P.betas[t & 1];
  double mx[VN], s[VN];
  bool no_shift = online || !(t >= 1 && drift_a < kShiftDrift);
#pragma unroll
  for (int k = 0; k < VN; ++k) {
    mx[k] = kNegInf;
    s[k] = 0.0;
    if (!no_shift && jb + k < m) {
      const double sh = rint(P.logb[jb + k] * kLog2e - betas_cur[jb + k]);
      if (fabs(sh) < 1.0e6) mx[k] = sh;
      else no_shift = true;
    }
  }
  const bool shift = !__syncthreads_or(no_shift ? 1 : 0);
  if (!shift)
#pragma unroll
    for (int k = 0; k < VN; ++k) mx[k] = kNegInf;
  // FP32 M with SFU passes: exponents from the float-pair alphas when they
  // and every column shift of the CTA are in range
  bool fsplit = false;
  if (sizeof(TM) == 4 && fast && shift && split_a_ok) {
    bool bad = false;
#pragma unroll
    for (int k = 0; k < VN; ++k) bad |= (jb + k < m) && !(fabs(mx[k]) < kSplitMax);
    fsplit = !__syncthreads_or(bad ? 1 : 0);
  }
  const float s2h = static_cast<float>(s2);
  const float s2l = static_cast<float>(s2 - static_cast<double>(s2h));
  // stream through the ring when every warp has at least two chunks of rows
  const bool use_ring = staged && vec_ok && (r1 - r0) >= 2 * kWarps * (kRingBytes / 512);
  if (use_ring) {
    const int strip_c0 = strip * W;
    const int strip_bytes = min(W, m - strip_c0) * (int)sizeof(TM);
    if (fast && fsplit)
      col_rows_staged<TM, true, true, sizeof(TM) == 4>(M, alphas, s2, m, strip_c0, strip_bytes,
                                                       jb, jb < m, r0, r1, warp, lane, tab, ring,
                                                       mx, s, P.asplit, s2h, s2l);
    else if (fast && shift)
      col_rows_staged<TM, true, true>(M, alphas, s2, m, strip_c0, strip_bytes, jb, jb < m, r0,
                                      r1, warp, lane, tab, ring, mx, s);
    else if (fast)
      col_rows_staged<TM, true, false>(M, alphas, s2, m, strip_c0, strip_bytes, jb, jb < m, r0,
                                       r1, warp, lane, tab, ring, mx, s);
    else if (shift)
      col_rows_staged<TM, false, true>(M, alphas, s2, m, strip_c0, strip_bytes, jb, jb < m, r0,
                                       r1, warp, lane, tab, ring, mx, s);
    else
      col_rows_staged<TM, false, false>(M, alphas, s2, m, strip_c0, strip_bytes, jb, jb < m, r0,
                                        r1, warp, lane, tab, ring, mx, s);
    if (ring.failed && lane == 0) {
      // a staging wait gave up: the problem ends with an error status
      atomicExch(&st->error, 1);
      atomicExch(&st->done, 1);
    }
  } else if (jb < m) {
    const int strip_c0 = strip * W;
    const int strip_bytes = min(W, m - strip_c0) * (int)sizeof(TM);
    if (fast && fsplit)
      col_rows<TM, true, true, sizeof(TM) == 4>(M, alphas, s2, m, jb, r0, r1, warp, vec_ok, tab,
                                                pf, strip_c0, strip_bytes, mx, s, P.asplit, s2h,
                                                s2l);
    else if (fast && shift)
      col_rows<TM, true, true>(M, alphas, s2, m, jb, r0, r1, warp, vec_ok, tab, pf, strip_c0,
                               strip_bytes, mx, s);
    else if (fast)
      col_rows<TM, true, false>(M, alphas, s2, m, jb, r0, r1, warp, vec_ok, tab, pf, strip_c0,
                                strip_bytes, mx, s);
    else if (shift)
      col_rows<TM, false, true>(M, alphas, s2, m, jb, r0, r1, warp, vec_ok, tab, pf, strip_c0,
                                strip_bytes, mx, s);
    else
      col_rows<TM, false, false>(M, alphas, s2, m, jb, r0, r1, warp, vec_ok, tab, pf, strip_c0,
                                 strip_bytes, mx, s);
  }
#pragma unroll
  for (int k = 0; k < VN; ++k) {
    sm_mx[warp][lane * VN + k] = mx[k];
    sm_s[warp][lane * VN + k] = s[k];
  }
  __syncthreads();
  const int c = threadIdx.x % W;  // column within the strip
  const int g = threadIdx.x / W;  // merge group
  const int j = strip * W + c;
  double Mc = kNegInf, Sc = 0.0;
  if (g == 0 && j < m) {
    Mc = sm_mx[0][c];
    Sc = sm_s[0][c];
    for (int w = 1; w < kWarps; ++w) lse2_merge(Mc, Sc, sm_mx[w][c], sm_s[w][c], tab);
  }
  if (P.col_splits > 1) {
    if (g == 0 && j < m) {
      P.col_m[(size_t)split * m + j] = Mc;
      P.col_s[(size_t)split * m + j] = Sc;
    }
    if (!elect_last(&P.counters[2 + strip], (unsigned)P.col_splits)) return;
    // parallel merge over splits: group g takes splits g, g+G, ...
    double Mg = kNegInf, Sg = 0.0;
    if (j < m) {
      // loads batched 4 at a time so their latencies overlap
      for (int q0 = g; q0 < P.col_splits; q0 += 4 * G) {
        double bm[4], bs[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int q = q0 + u * G;
          bm[u] = (q < P.col_splits) ? ldcg(P.col_m + (size_t)q * m + j) : kNegInf;
          bs[u] = (q < P.col_splits) ? ldcg(P.col_s + (size_t)q * m + j) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) lse2_merge(Mg, Sg, bm[u], bs[u], tab);
      }
    }
    __syncthreads();
    sm_mx[g][c] = Mg;
    sm_s[g][c] = Sg;
    __syncthreads();
    if (g == 0 && j < m) {
      Mc = sm_mx[0][c];
      Sc = sm_s[0][c];
      for (int q = 1; q < G; ++q) lse2_merge(Mc, Sc, sm_mx[q][c], sm_s[q][c], tab);
    }
  }
  const bool valid = (g == 0 && j < m);
  double db = 0.0;
  if (valid) {
    const double b_new = P.eta * P.logb[j] - (P.eta * kLn2) * (Mc + log2(Sc));
    P.beta[(t + 1) & 1][j] = b_new;
    P.betas[(t + 1) & 1][j] = b_new * s2;
    if (P.bsplit != nullptr && !split_of(b_new * s2, P.bsplit[j])) atomicOr(&st->split_bad_b, 1);
    db = b_new - P.beta[t & 1][j];
  }
  {
    // largest |betas change| of the strip (NaN orders above +inf)
    unsigned long long b = valid ? (unsigned long long)__double_as_longlong(fabs(db * s2)) : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long x = __shfl_xor_sync(0xffffffffu, b, o);
      b = x > b ? x : b;
    }
    if (lane == 0 && b != 0ull) atomicMax(&st->acc_b, b);
  }
  if (phase == 1) {
    double sn, smu, sm2;
    cta_stats(db, valid, red, sn, smu, sm2);
    if (threadIdx.x == 0) {
      P.col_part[(size_t)strip * 3] = sn;
      P.col_part[(size_t)strip * 3 + 1] = smu;
      P.col_part[(size_t)strip * 3 + 2] = sm2;
    }
  }

  if (!elect_last(&P.counters[1], (unsigned)P.col_strips)) return;

  // Last strip finisher: iteration bookkeeping (reference :551-591).
  const int tn = t + 1;
  if (threadIdx.x == 0) {
    st->drift_b = __longlong_as_double((long long)atomicExch(&st->acc_b, 0ull));
    st->split_bad_a = 0;  // every CTA of this pass has read it
  }
  if (phase == 1) {
    double bn = 0, bmu = 0, bm2 = 0;
    for (int q = threadIdx.x; q < P.col_strips; q += blockDim.x)
      chan_combine(bn, bmu, bm2, ldcg(P.col_part + (size_t)q * 3),
                   ldcg(P.col_part + (size_t)q * 3 + 1), ldcg(P.col_part + (size_t)q * 3 + 2));
    cta_chan(bn, bmu, bm2, shc);
    if (threadIdx.x == 0) {
      const double an = ldcg(&st->stat_a[0]), amu = ldcg(&st->stat_a[1]),
                   am2 = ldcg(&st->stat_a[2]);
      // K = c - d of the reference = (sum dbeta - sum dalpha) / (n + m)
      const double K = (bn * bmu - an * amu) / (double)(n + m);
      const double ea = amu + K, eb = bmu - K;
      const double diff = sqrt(am2 + an * ea * ea + bm2 + bn * eb * eb);
      st->last_err = diff;
      if (diff < st->tol * 10) st->phase = 2;
      if (!isfinite(diff)) {
        st->done = 1;
        st->nonfinite = 1;
      }
    }
  } else if (phase == 2 && threadIdx.x == 0) {
    st->check_pending = 1;
  }
  if (threadIdx.x == 0) {
    st->iter = tn;
    st->niter = tn;
    if (fast) st->fast_iters += 1;
    if (tn >= st->max_iter) st->done = 1;
  }
}

// The passes run as grid-stride loops over virtual CTAs: a launch with fewer
// CTAs than virtual blocks (the serving engine caps its batch launches) does
// the same work, in the same per-block order, leaving SM slots free for
// latency-bound kernels on other streams.
// LOOP = false: one virtual CTA per CTA (uncapped launches).
// flags & kPassStaged: long rows / column strips stream through per-warp
// shared-memory rings filled by bulk copies (dynamic shared memory:
// kRingDynBytes; launched with none otherwise, which leaves the SM's L1 to the
// cached dual vectors).  flags & kPassOnline: every pass takes the running
// maximum (no shifted sums).  flags >> kPassPrefetchShift: L2 bulk-prefetch
// distance of the register path, in chunks (0: none).
template <typename TM, bool LOOP>
__global__ void __launch_bounds__(kThreads, kBcdMinBlocks) bcd_row_kernel(const BcdProb* __restrict__ probs,
                                                            const int* __restrict__ cta_prob,
                                                            const int* __restrict__ cta_start,
                                                            int total, int flags) {
  extern __shared__ __align__(128) unsigned char ring_smem[];
  __shared__ uint64_t ring_bars[kWarps * kRingStages];
  WarpRing ring;
  rings_init(ring_smem, ring_bars, kWarps, ring);
  if (!LOOP) {
    row_block<TM>(probs, cta_prob, cta_start, (int)blockIdx.x, flags, ring);
    return;
  }
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    row_block<TM>(probs, cta_prob, cta_start, vb, flags, ring);
    __syncthreads();
  }
}

template <typename TM, bool LOOP>
__global__ void __launch_bounds__(kThreads, kBcdMinBlocks) bcd_col_kernel(const BcdProb* __restrict__ probs,
                                                            const int* __restrict__ cta_prob,
                                                            const int* __restrict__ cta_start,
                                                            int total, int flags) {
  extern __shared__ __align__(128) unsigned char ring_smem[];
  __shared__ uint64_t ring_bars[kWarps * kRingStages];
  WarpRing ring;
  rings_init(ring_smem, ring_bars, kWarps, ring);
  if (!LOOP) {
    col_block<TM>(probs, cta_prob, cta_start, (int)blockIdx.x, flags, ring);
    return;
  }
  for (int vb = blockIdx.x; vb < total; vb += gridDim.x) {
    col_block<TM>(probs, cta_prob, cta_start, vb, flags, ring);
    __syncthreads();
  }
}

// P = exp((alpha_i + beta_j - M_ij) / eta)
template <typename TM>
__global__ void plan_kernel(const TM* __restrict__ M, const double* __restrict__ alpha,
                            const double* __restrict__ beta, double* __restrict__ P,
                            double inv_eta, int n, int m) {
  const size_t total = (size_t)n * m;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / m);
    const int j = (int)(idx - (size_t)i * m);
    P[idx] = exp((alpha[i] + beta[j] - ld1(M + idx)) * inv_eta);
  }
}

namespace {
constexpr int kRingDynBytes = kWarps * kRingStages * kRingBytes;
std::atomic<int> g_staged{0};
std::atomic<int> g_l2pf{0};
std::atomic<int> g_online{0};
std::once_flag g_ring_attr_once;

// Opt the pass kernels into kRingDynBytes of dynamic shared memory (once per
// process; above the 48 KB default together with their static arrays).
void set_ring_attributes() {
  std::call_once(g_ring_attr_once, [] {
    cudaFuncSetAttribute(bcd_row_kernel<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingDynBytes);
    cudaFuncSetAttribute(bcd_row_kernel<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingDynBytes);
    cudaFuncSetAttribute(bcd_row_kernel<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingDynBytes);
    cudaFuncSetAttribute(bcd_row_kernel<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingDynBytes);
    cudaFuncSetAttribute(bcd_col_kernel<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingDynBytes);
    cudaFuncSetAttribute(bcd_col_kernel<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingDynBytes);
    cudaFuncSetAttribute(bcd_col_kernel<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingDynBytes);
    cudaFuncSetAttribute(bcd_col_kernel<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRingDynBytes);
  });
}
}  // namespace

void bcd_set_staging(bool on) { g_staged.store(on ? 1 : 0); }
void bcd_set_l2_prefetch(int chunks) { g_l2pf.store(std::clamp(chunks, 0, 64)); }
int bcd_l2_prefetch() { return g_l2pf.load(); }
void bcd_set_shifted_lse(bool on) { g_online.store(on ? 0 : 1); }

namespace {
int pass_flags(size_t& dyn_smem) {
  const int sg = g_staged.load();
  dyn_smem = sg ? (size_t)kRingDynBytes : 0;
  return (sg ? kPassStaged : 0) | (g_online.load() ? kPassOnline : 0) |
         (g_l2pf.load() << kPassPrefetchShift);
}
}  // namespace

void launch_bcd_row(bool f32, const BcdProb* d_probs, const int* d_cta_prob,
                    const int* d_cta_start, int total_ctas, cudaStream_t stream, int grid_cap) {
  set_ring_attributes();
  const bool loop = grid_cap > 0 && grid_cap < total_ctas;
  const int grid = loop ? grid_cap : total_ctas;
  size_t sm = 0;
  const int sg = pass_flags(sm);
  if (f32 && loop)
    { bcd_row_kernel<float, true><<<grid, kThreads, sm, stream>>>(d_probs, d_cta_prob, d_cta_start, total_ctas, sg); cg::count_launch(); }
  else if (f32)
    { bcd_row_kernel<float, false><<<grid, kThreads, sm, stream>>>(d_probs, d_cta_prob, d_cta_start, total_ctas, sg); cg::count_launch(); }
  else if (loop)
    { bcd_row_kernel<double, true><<<grid, kThreads, sm, stream>>>(d_probs, d_cta_prob, d_cta_start, total_ctas, sg); cg::count_launch(); }
  else
    { bcd_row_kernel<double, false><<<grid, kThreads, sm, stream>>>(d_probs, d_cta_prob, d_cta_start, total_ctas, sg); cg::count_launch(); }
}
void launch_bcd_col(bool f32, const BcdProb* d_probs, const int* d_cta_prob,
                    const int* d_cta_start, int total_ctas, cudaStream_t stream, int grid_cap) {
  set_ring_attributes();
  const bool loop = grid_cap > 0 && grid_cap < total_ctas;
  const int grid = loop ? grid_cap : total_ctas;
  size_t sm = 0;
  const int sg = pass_flags(sm);
  if (f32 && loop)
    { bcd_col_kernel<float, true><<<grid, kThreads, sm, stream>>>(d_probs, d_cta_prob, d_cta_start, total_ctas, sg); cg::count_launch(); }
  else if (f32)
    { bcd_col_kernel<float, false><<<grid, kThreads, sm, stream>>>(d_probs, d_cta_prob, d_cta_start, total_ctas, sg); cg::count_launch(); }
  else if (loop)
    { bcd_col_kernel<double, true><<<grid, kThreads, sm, stream>>>(d_probs, d_cta_prob, d_cta_start, total_ctas, sg); cg::count_launch(); }
  else
    { bcd_col_kernel<double, false><<<grid, kThreads, sm, stream>>>(d_probs, d_cta_prob, d_cta_start, total_ctas, sg); cg::count_launch(); }
}
template <typename TM>
void launch_plan(const TM* M, const double* alpha, const double* beta, double* P,
                 double inv_eta, int n, int m, cudaStream_t stream) {
  const size_t total = (size_t)n * m;
  const int blocks = (int)std::min<size_t>((total + kThreads - 1) / kThreads, 148 * 16);
  { plan_kernel<TM><<<std::max(blocks, 1), kThreads, 0, stream>>>(M, alpha, beta, P, inv_eta, n, m); cg::count_launch(); }
}
template void launch_plan<double>(const double*, const double*, const double*, double*, double,
                                  int, int, cudaStream_t);
template void launch_plan<float>(const float*, const double*, const double*, double*, double,
                                 int, int, cudaStream_t);

int sm_count_current() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return std::max(sms, 1);
}

void bcd_geometry(int n, int m, int elem_bytes, int sm_count, BcdProb& p) {
  const int vn = 16 / elem_bytes;
  // Row pass: prefer one warp per row; give short-n problems more warps per
  // row while each warp keeps at least one unrolled vector sweep of work.
  int R = kWarps;
  while (R > 1) {
    const int ctas = (n + R - 1) / R;
    const int wpr = kWarps / (R / 2);
    if (ctas >= 2 * sm_count) break;
    if (m < wpr * 32 * vn * kUnroll) break;
    R /= 2;
  }
  p.rows_per_cta = R;
  p.row_ctas = (n + R - 1) / R;
  // Column pass: 512-byte strips.
  const int W = 32 * vn;
  p.col_strips = (m + W - 1) / W;
  // as many row splits as fill one wave of resident CTAs (3 per SM) without
  // starting a partial second one, at least 128 rows per split
  int splits = (3 * sm_count) / p.col_strips;
  splits = std::max(1, std::min(splits, n / 128));
  p.col_splits = splits;
}

}  // namespace cg
