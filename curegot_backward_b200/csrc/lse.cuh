// Base-2 log-sum-exp building blocks shared by the Sinkhorn kernels: online
// (max, sum) accumulation over chunks of exponents, the pairwise merge of two
// partial (max, sum) pairs, and raw 16-byte vector loads of M.
#pragma once

#include "common.cuh"

namespace cg {

constexpr int kUnroll = 4;

// (max, sum) merge in base 2
__device__ __forceinline__ void lse2_merge(double& mx, double& s, double mx2, double s2,
                                           const double* tab) {
  if (s2 == 0.0) return;
  if (s == 0.0) {
    mx = mx2;
    s = s2;
    return;
  }
  if (mx2 > mx) {
    s = s * exp2_f64(mx - mx2, tab) + s2;
    mx = mx2;
  } else {
    s += s2 * exp2_f64(mx2 - mx, tab);
  }
}

// Shifted accumulation: with SHIFT the pair (mx, s) holds a fixed integer
// shift mx chosen before the pass (the previous iteration's LSE of the same
// row or column) and s += sum_q 2^(d_q - mx), with no running maximum.  The
// caller guarantees every exponent d_q - mx <= kShiftDrift (the LSE moved by
// at most the largest dual change of the other side since that LSE was
// taken), so no term overflows in FP32 or FP64.
constexpr double kShiftDrift = 40.0;

template <bool FAST, int K>
__device__ __forceinline__ void lse_shift_terms(const double (&d)[K], const bool* ok, double mx,
                                                double& s, const double* tab) {
  if (FAST) {
    float acc = 0.0f;
#pragma unroll
    for (int q = 0; q < K; ++q)
      if (ok == nullptr || ok[q]) acc += exp2_neg_mixed(d[q] - mx);
    s += static_cast<double>(acc);
  } else {
    const int k = static_cast<int>(mx);
    const double lo = mx - 1000.0;
    double acc = 0.0;
#pragma unroll
    for (int q = 0; q < K; ++q)
      if (ok == nullptr || ok[q]) acc += exp2_shift_f64(d[q], lo, k, tab);
    s += acc;
  }
}

// One term of the mixed-precision shifted sum from float-pair duals:
// 2^(v - k - s2 M) with v = hi + lo, s2 = s2h + s2l (FP32 pairs) and the
// integer shift k.  t = hi - k is exact (hi a multiple of 2^-9, |hi|, |k| <
// 2^14); fmaf(-s2h, M, t) is t - s2h M rounded once; the low parts add
// lo - s2l M.  The exponent is within 2^-18 of the FP64 value when it is
// at most 64 in magnitude (the terms that matter), the same order as the
// FP32 rounding the FP64-argument form applies.  No FP64 work and no
// conversions: one SFU operation per element.
__device__ __forceinline__ float split_term(float m, float hi, float lo, float k, float s2h,
                                            float s2l) {
  const float t = __fsub_rn(hi, k);
  const float u = fmaf(-s2h, m, t);
  const float c = fmaf(-s2l, m, lo);
  return ex2_approx(__fadd_rn(u, c));
}

// Accumulate K exponents (valid ones only) into the running (mx, s).
template <bool FAST, int K, bool SHIFT = false>
__device__ __forceinline__ void lse_chunk(const double (&d)[K], const bool (&ok)[K], double& mx,
                                          double& s, const double* tab) {
  if (SHIFT) {
    lse_shift_terms<FAST, K>(d, ok, mx, s, tab);
    return;
  }
  double cmax = kNegInf;
#pragma unroll
  for (int q = 0; q < K; ++q)
    if (ok[q]) cmax = fmax(cmax, d[q]);
  if (cmax > mx) {
    if (s != 0.0) s *= exp2_f64(mx - cmax, tab);
    mx = cmax;
  }
  if (FAST) {
    float acc = 0.0f;
#pragma unroll
    for (int q = 0; q < K; ++q)
      if (ok[q]) acc += exp2_neg_mixed(d[q] - mx);
    s += static_cast<double>(acc);
  } else {
#pragma unroll
    for (int q = 0; q < K; ++q)
      if (ok[q]) s += exp2_neg_f64(d[q] - mx, tab);
  }
}

// Same, for a chunk known to be fully in range (no predicates).
template <bool FAST, int K, bool SHIFT = false>
__device__ __forceinline__ void lse_chunk_full(const double (&d)[K], double& mx, double& s,
                                               const double* tab) {
  if (SHIFT) {
    lse_shift_terms<FAST, K>(d, nullptr, mx, s, tab);
    return;
  }
  double cmax = d[0];
#pragma unroll
  for (int q = 1; q < K; ++q) cmax = fmax(cmax, d[q]);
  if (cmax > mx) {
    if (s != 0.0) s *= exp2_f64(mx - cmax, tab);
    mx = cmax;
  }
  if (FAST) {
    float acc = 0.0f;
#pragma unroll
    for (int q = 0; q < K; ++q) acc += exp2_neg_mixed(d[q] - mx);
    s += static_cast<double>(acc);
  } else {
    double acc = 0.0;
#pragma unroll
    for (int q = 0; q < K; ++q) acc += exp2_neg_f64(d[q] - mx, tab);
    s += acc;
  }
}

// Raw 16-byte vector of M.  M is streamed once per pass, so its loads do not
// allocate in L1 (read-only path, L1::no_allocate): L1 stays with the dual
// vectors the passes re-read for every row.
template <typename TM>
struct Raw;
template <>
struct Raw<double> {
  using T = double2;
  __device__ __forceinline__ static T load(const double* p) {
#ifdef CG_M_L1_ALLOCATE
    return __ldg(reinterpret_cast<const double2*>(p));
#else
    T v;
    asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];"
                 : "=d"(v.x), "=d"(v.y)
                 : "l"(p));
    return v;
#endif
  }
  __device__ __forceinline__ static double get(const T& v, int k) { return k == 0 ? v.x : v.y; }
};
template <>
struct Raw<float> {
  using T = float4;
  __device__ __forceinline__ static T load(const float* p) {
#ifdef CG_M_L1_ALLOCATE
    return __ldg(reinterpret_cast<const float4*>(p));
#else
    T v;
    asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
                 : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
                 : "l"(p));
    return v;
#endif
  }
  __device__ __forceinline__ static double get(const T& v, int k) {
    return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
  }
};

}  // namespace cg
