// Shared device helpers for the sm_100a entropic-OT kernels.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>

#include "curegot_b200.h"

namespace cg {

constexpr int kThreads = 256;  // threads per CTA for the streaming passes
constexpr int kWarps = kThreads / 32;
constexpr double kNegInf = -INFINITY;

inline int status_from_cuda(cudaError_t e) {
  if (e == cudaSuccess) return CG_OK;
  if (e == cudaErrorMemoryAllocation) return CG_ERR_OOM;
  return CG_ERR_CUDA;
}

#define CG_TRY_CUDA(expr)                                   \
  do {                                                      \
    cudaError_t cg_e_ = (expr);                             \
    if (cg_e_ != cudaSuccess) {                             \
      cg::set_last_error(cudaGetErrorString(cg_e_), __FILE__, __LINE__); \
      return cg::status_from_cuda(cg_e_);                   \
    }                                                       \
  } while (0)

#define CG_TRY(expr)                   \
  do {                                 \
    int cg_s_ = (expr);                \
    if (cg_s_ != CG_OK) return cg_s_;  \
  } while (0)

void set_last_error(const char* msg, const char* file, int line);

// Number of SMs of the current device.
int sm_count_current();

// Kernel launches issued by this library (graph replays count their kernels).
void count_launch(long long k = 1);

// Stream-ordered allocation from the library's own memory pool on the current
// device (created on first use; it keeps freed memory mapped for reuse instead
// of returning it to the driver at every synchronization).  Free with
// cudaFreeAsync.
int pool_alloc_async(void** ptr, size_t bytes, cudaStream_t stream);
int library_pool(int device, cudaMemPool_t* out);

// Device-to-host reads of small solver state through a thread-local pinned
// buffer (a pageable destination would take the driver's staged-copy path,
// which serializes concurrent solver threads).  Both copies are queued on
// `st`, then the stream is synchronized once.  bytes1 + bytes2 <= 4096.
int read_device(void* host1, const void* dev1, size_t bytes1, cudaStream_t st,
                void* host2 = nullptr, const void* dev2 = nullptr, size_t bytes2 = 0);

// Warp reductions: the result is valid in lane 0 (shfl_down tree, a fixed
// association order, so results are bitwise reproducible).
__device__ __forceinline__ double warp_sum_down(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Online log-sum-exp state (max, scaled sum) merge.
__device__ __forceinline__ void lse_merge(double& mx, double& s, double mx2, double s2) {
  if (s2 == 0.0) return;
  if (s == 0.0) {
    mx = mx2;
    s = s2;
    return;
  }
  if (mx2 > mx) {
    s = s * exp(mx - mx2) + s2;
    mx = mx2;
  } else {
    s += s2 * exp(mx2 - mx);
  }
}

__device__ __forceinline__ void warp_lse_down(double& mx, double& s) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double m2 = __shfl_down_sync(0xffffffffu, mx, o);
    const double s2 = __shfl_down_sync(0xffffffffu, s, o);
    lse_merge(mx, s, m2, s2);
  }
}

// "Last CTA done" election: every CTA publishes its partial results, fences,
// then bumps a counter; the CTA that sees count == total-1 finalizes and
// resets the counter for the next launch.  No spinning is involved.
__device__ __forceinline__ bool elect_last(unsigned int* counter, unsigned int total) {
  __shared__ bool s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int prev = atomicAdd(counter, 1u);
    s_last = (prev == total - 1);
    if (s_last) *counter = 0u;
  }
  __syncthreads();
  if (s_last) __threadfence();
  return s_last;
}

// CTA-wide sum (kThreads threads); result valid in thread 0.
__device__ __forceinline__ double cta_sum(double v, double* red /* >= kWarps */) {
  v = warp_sum_down(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 0; w < nw; ++w) r += red[w];
  }
  return r;
}

// Vector loads of row-major cost matrices.
template <typename TM>
struct Vec;
template <>
struct Vec<double> {
  static constexpr int N = 2;
  __device__ __forceinline__ static void load(const double* p, double* out) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(p));
    out[0] = v.x;
    out[1] = v.y;
  }
};
template <>
struct Vec<float> {
  static constexpr int N = 4;
  __device__ __forceinline__ static void load(const float* p, double* out) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
    out[3] = v.w;
  }
};

template <typename TM>
__device__ __forceinline__ double ld1(const TM* p) {
  return static_cast<double>(__ldg(p));
}

// Load VN consecutive FP64 duals (16-byte aligned when VN >= 2).
template <int VN>
__device__ __forceinline__ void ld_duals(const double* p, double* out) {
#pragma unroll
  for (int k = 0; k < VN; k += 2) {
    const double2 v = *reinterpret_cast<const double2*>(p + k);
    out[k] = v.x;
    out[k + 1] = v.y;
  }
}

// L2-coherent load for data written by other CTAs of the same launch.
__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int ldcg(const int* p) { return __ldcg(p); }

// ---------------------------------------------------------------------------
// Exponentials in base 2.
//
// exp2_f64: table-driven method of P. T. P. Tang (ACM TOMS 15(2), 1989):
//   x = N/16 + f with N = round(16 x), |f| <= 1/32 (f exact in FP64),
//   2^f = exp(f ln2) by its Taylor series to degree 6 (coefficients
//   ln2^k / k!, truncation error < 4.5e-16), 2^(N/16) = 2^(N >> 4) * T[N & 15].
// All constants were computed from the mathematics (60-digit decimal) and
// rounded to double.  Valid for all x; returns 0 below -1020 and +inf at or
// above 1024; NaN propagates.
// ---------------------------------------------------------------------------
constexpr double kExpMagic = 6755399441055744.0;  // 1.5 * 2^52: round-to-integer
constexpr double kLog2e = 1.4426950408889634;
constexpr double kLn2 = 0.6931471805599453;

struct Exp2Table {
  double t[16];
};
__host__ __device__ constexpr Exp2Table make_exp2_table() {
  return Exp2Table{{1.0, 1.0442737824274138, 1.0905077326652577, 1.1387886347566916,
                    1.189207115002721, 1.241857812073484, 1.2968395546510096,
                    1.3542555469368927, 1.4142135623730951, 1.4768261459394993,
                    1.5422108254079407, 1.6104903319492543, 1.681792830507429,
                    1.7562521603732995, 1.8340080864093424, 1.9152065613971474}};
}

static __constant__ Exp2Table c_exp2_table = make_exp2_table();

// Loads the 16-entry table into shared memory (call from every thread, then sync).
__device__ __forceinline__ void load_exp2_table(double* sh) {
  if (threadIdx.x < 16) sh[threadIdx.x] = c_exp2_table.t[threadIdx.x];
}

__device__ __forceinline__ double exp2_f64(double x, const double* __restrict__ tab) {
  if (!(x >= -1020.0)) return (x != x) ? x : 0.0;
  if (x >= 1024.0) return INFINITY;
  const double t = fma(x, 16.0, kExpMagic);
  const int N = __double2loint(t);
  const double kf = t - kExpMagic;
  const double f = fma(kf, -0.0625, x);
  double p = fma(f, 0.0001540353039338161, 0.0013333558146428443);
  p = fma(f, p, 0.009618129107628477);
  p = fma(f, p, 0.05550410866482158);
  p = fma(f, p, 0.24022650695910072);
  p = fma(f, p, 0.6931471805599453);
  p = fma(f, p, 1.0);
  const double y = p * tab[N & 15];
  return __hiloint2double(__double2hiint(y) + ((N >> 4) << 20), __double2loint(y));
}

// Non-positive-argument variant used inside the LSE passes (x <= 0 by
// construction after the running-max shift): same method, no overflow branch.
__device__ __forceinline__ double exp2_neg_f64(double x, const double* __restrict__ tab) {
  x = fmax(x, -1020.0);
  const double t = fma(x, 16.0, kExpMagic);
  const int N = __double2loint(t);
  const double kf = t - kExpMagic;
  const double f = fma(kf, -0.0625, x);
  double p = fma(f, 0.0001540353039338161, 0.0013333558146428443);
  p = fma(f, p, 0.009618129107628477);
  p = fma(f, p, 0.05550410866482158);
  p = fma(f, p, 0.24022650695910072);
  p = fma(f, p, 0.6931471805599453);
  p = fma(f, p, 1.0);
  const double y = p * tab[N & 15];
  return __hiloint2double(__double2hiint(y) + ((N >> 4) << 20), __double2loint(y));
}

// Hardware 2^x on the SFU (ex2.approx.ftz.f32).
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Mixed-precision 2^x for x <= 0: the integer part is split off exactly in
// FP64 and only the fraction (|f| <= 1/2) goes through the FP32 SFU, so the
// relative error is that of ex2.approx on [-1/2, 1/2] regardless of |x|.
__device__ __forceinline__ float exp2_neg_mixed(double x) {
  x = fmax(x, -200.0);
  const double t = x + kExpMagic;
  const int N = __double2loint(t);
  const double kf = t - kExpMagic;
  const float f = static_cast<float>(x - kf);
  const float y = ex2_approx(f);
  const float sc = (N >= -126) ? __int_as_float((N + 127) << 23) : 0.0f;
  return y * sc;
}

// Chan et al. pairwise combine of (count, mean, M2) statistics.
__device__ __forceinline__ void chan_combine(double& nA, double& muA, double& m2A, double nB,
                                             double muB, double m2B) {
  if (nB == 0.0) return;
  if (nA == 0.0) {
    nA = nB;
    muA = muB;
    m2A = m2B;
    return;
  }
  const double n = nA + nB;
  const double d = muB - muA;
  muA = muA + d * (nB / n);
  m2A = m2A + m2B + d * d * (nA * nB / n);
  nA = n;
}

}  // namespace cg
