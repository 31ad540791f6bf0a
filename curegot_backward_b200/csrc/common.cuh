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
// `st`, then the stream is synchronized once.  At most 4096 bytes in all.
// Host wait for all work queued on `st`.  By default the calling thread
// blocks in cudaStreamSynchronize (the runtime spins while few contexts are
// active).  A thread that called host_wait_yield(true) -- the serving
// engine's batch and SPLR worker threads -- instead polls an event and
// yields its core between polls, so many solver threads can wait at once
// without occupying every host core.
int host_wait(cudaStream_t st);
void host_wait_yield(bool on);

struct ReadSpan {
  void* host;
  const void* dev;
  size_t bytes;
};
int read_device_spans(const ReadSpan* spans, int count, cudaStream_t st);
// Any size: through a thread-local pinned buffer that grows as needed (kept
// for the thread's lifetime), then host_wait on the stream.
int read_device_bulk(void* host, const void* dev, size_t bytes, cudaStream_t st);
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
// Vector and scalar loads of streamed matrices (M, T, G): read-only path,
// no L1 allocation (each element is read once per pass; L1 is left to the
// dual and index vectors that are re-read).
template <>
struct Vec<double> {
  static constexpr int N = 2;
  __device__ __forceinline__ static void load(const double* p, double* out) {
    asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(out[0]), "=d"(out[1]) : "l"(p));
  }
};
template <>
struct Vec<float> {
  static constexpr int N = 4;
  __device__ __forceinline__ static void load(const float* p, double* out) {
    float x, y, z, w;
    asm("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
        : "=f"(x), "=f"(y), "=f"(z), "=f"(w)
        : "l"(p));
    out[0] = x;
    out[1] = y;
    out[2] = z;
    out[3] = w;
  }
};

__device__ __forceinline__ double ld1(const double* p) {
  double v;
  asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld1(const float* p) {
  float v;
  asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return static_cast<double>(v);
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
//   x = N/T + f with N = round(T x), |f| <= 1/(2T) (f exact in FP64),
//   2^f = exp(f ln2) by its Taylor series, 2^(N/T) = 2^(N >> B) * tab[N & (T-1)].
// Valid for all x; returns 0 below -1020 and +inf at or above 1024; NaN
// propagates.
// ---------------------------------------------------------------------------
constexpr double kExpMagic = 6755399441055744.0;  // 1.5 * 2^52: round-to-integer
constexpr double kLog2e = 1.4426950408889634;
constexpr double kLn2 = 0.6931471805599453;

// Table size T = 2^B: x = N/T + f, |f| <= 1/(2T).  T = 256 with a degree-4
// polynomial (truncation < 3.8e-17 relative; default) takes one FMA less per
// element than T = 64 with degree 5 (< 3.4e-17), and two less than T = 16
// with degree 6 (< 4.5e-16); the table (2 KB of shared memory per CTA) and
// all coefficients were computed from the mathematics (70-digit decimal) and
// rounded to double.
#if defined(CG_EXP2_T16)
constexpr int kExp2Bits = 4;
#elif defined(CG_EXP2_T64)
constexpr int kExp2Bits = 6;
#else
constexpr int kExp2Bits = 8;
#endif
constexpr int kExp2TableSize = 1 << kExp2Bits;
constexpr double kExp2Scale = (double)kExp2TableSize;
constexpr double kExp2InvScale = 1.0 / kExp2Scale;

struct Exp2Table {
  double t[kExp2TableSize];
};
__host__ __device__ constexpr Exp2Table make_exp2_table() {
#if defined(CG_EXP2_T16)
  return Exp2Table{{1.0, 1.0442737824274138, 1.0905077326652577, 1.1387886347566916,
                    1.189207115002721, 1.241857812073484, 1.2968395546510096,
                    1.3542555469368927, 1.4142135623730951, 1.4768261459394993,
                    1.5422108254079407, 1.6104903319492543, 1.681792830507429,
                    1.7562521603732995, 1.8340080864093424, 1.9152065613971474}};
#elif defined(CG_EXP2_T64)
  return Exp2Table{{
      1.0, 1.0108892860517005, 1.0218971486541166, 1.0330248790212284,
      1.0442737824274138, 1.0556451783605572, 1.0671404006768237, 1.0787607977571199,
      1.0905077326652577, 1.102382583307841, 1.1143867425958924, 1.1265216186082418,
      1.1387886347566916, 1.1511892299529827, 1.1637248587775775, 1.1763969916502812,
      1.189207115002721, 1.202156731452703, 1.215247359980469, 1.22848053610687,
      1.241857812073484, 1.255380757024691, 1.2690509571917332, 1.2828700160787783,
      1.2968395546510096, 1.3109612115247644, 1.3252366431597413, 1.339667524053303,
      1.3542555469368927, 1.3690024229745905, 1.383909881963832, 1.3989796725383112,
      1.4142135623730951, 1.42961333839197, 1.4451808069770467, 1.460917794180647,
      1.4768261459394993, 1.4929077282912648, 1.5091644275934228, 1.5255981507445384,
      1.5422108254079407, 1.559004400237837, 1.5759808451078865, 1.593142151342267,
      1.6104903319492543, 1.6280274218573478, 1.645755478153965, 1.6636765803267364,
      1.681792830507429, 1.7001063537185235, 1.718619298122478, 1.7373338352737062,
      1.7562521603732995, 1.7753764925265212, 1.7947090750031072, 1.8142521755003989,
      1.8340080864093424, 1.8539791250833855, 1.8741676341103, 1.8945759815869656,
      1.9152065613971474, 1.9360617934922943, 1.9571441241754002, 1.978456026387951}};
#else
  return Exp2Table{{
      1.0, 1.0027112750502025, 1.0054299011128027, 1.0081558981184175,
      1.0108892860517005, 1.0136300849514894, 1.016378314910953, 1.019133996077738,
      1.0218971486541166, 1.0246677928971357, 1.0274459491187637, 1.030231637686041,
      1.0330248790212284, 1.0358256936019572, 1.0386341019613787, 1.041450124688316,
      1.0442737824274138, 1.0471050958792898, 1.0499440858006872, 1.0527907730046264,
      1.0556451783605572, 1.0585073227945128, 1.061377227289262, 1.0642549128844645,
      1.0671404006768237, 1.0700337118202419, 1.0729348675259756, 1.075843889062791,
      1.0787607977571199, 1.0816856149932152, 1.0846183622133092, 1.0875590609177697,
      1.0905077326652577, 1.0934643990728858, 1.0964290818163769, 1.099401802630222,
      1.102382583307841, 1.1053714457017412, 1.1083684117236787, 1.1113735033448175,
      1.1143867425958924, 1.1174081515673693, 1.1204377524096067, 1.12347556733302,
      1.1265216186082418, 1.129575928566288, 1.1326385195987192, 1.1357094141578055,
      1.1387886347566916, 1.1418762039695616, 1.1449721444318042, 1.148076478840179,
      1.1511892299529827, 1.154310420590216, 1.1574400736337511, 1.1605782120274988,
      1.1637248587775775, 1.1668800369524817, 1.1700437696832502, 1.1732160801636373,
      1.1763969916502812, 1.1795865274628758, 1.182784710984341, 1.1859915656609938,
      1.189207115002721, 1.1924313825831512, 1.1956643920398273, 1.1989061670743806,
      1.202156731452703, 1.2054161090051239, 1.2086843236265816, 1.2119613992768012,
      1.215247359980469, 1.2185422298274085, 1.2218460329727576, 1.2251587936371455,
      1.22848053610687, 1.2318112847340759, 1.2351510639369334, 1.2384998981998165,
      1.241857812073484, 1.245224830175258, 1.2486009771892048, 1.2519862778663162,
      1.255380757024691, 1.2587844395497165, 1.2621973503942507, 1.2656195145788063,
      1.2690509571917332, 1.2724917033894028, 1.275941778396392, 1.2794012075056693,
      1.2828700160787783, 1.2863482295460256, 1.2898358734066657, 1.2933329732290895,
      1.2968395546510096, 1.3003556433796506, 1.3038812651919358, 1.3074164459346773,
      1.3109612115247644, 1.3145155879493546, 1.318079601266064, 1.3216532776031575,
      1.3252366431597413, 1.3288297242059544, 1.3324325470831615, 1.3360451382041458,
      1.339667524053303, 1.3432997311868353, 1.3469417862329458, 1.3505937158920345,
      1.3542555469368927, 1.3579273062129011, 1.3616090206382248, 1.365300717204012,
      1.3690024229745905, 1.3727141650876684, 1.3764359707545302, 1.380167867260238,
      1.383909881963832, 1.387662042298529, 1.3914243757719262, 1.3951969099662003,
      1.3989796725383112, 1.4027726912202048, 1.4065759938190154, 1.4103896082172707,
      1.4142135623730951, 1.4180478843204152, 1.4218926021691656, 1.4257477441054942,
      1.42961333839197, 1.433489413367789, 1.4373759974489824, 1.4412731191286257,
      1.4451808069770467, 1.449099089642035, 1.4530279958490526, 1.4569675544014438,
      1.460917794180647, 1.4648787441464057, 1.4688504333369818, 1.4728328908693675,
      1.4768261459394993, 1.4808302278224719, 1.4848451658727524, 1.488870989524397,
      1.4929077282912648, 1.4969554117672355, 1.5010140696264256, 1.5050837316234065,
      1.5091644275934228, 1.5132561874526098, 1.5173590411982147, 1.5214730189088146,
      1.5255981507445384, 1.529734466947287, 1.533881997840956, 1.5380407738316568,
      1.5422108254079407, 1.5463921831410214, 1.550584877685, 1.5547889397770887,
      1.559004400237837, 1.5632312899713576, 1.567469639965553, 1.5717194812923414,
      1.5759808451078865, 1.5802537626528246, 1.5845382652524937, 1.588834384317164,
      1.593142151342267, 1.597461597908627, 1.6017927556826934, 1.606135656416771,
      1.6104903319492543, 1.6148568142048607, 1.6192351351948637, 1.6236253270173289,
      1.6280274218573478, 1.632441451987275, 1.6368674497669644, 1.6413054476440063,
      1.645755478153965, 1.6502175739206177, 1.6546917676561943, 1.6591780921616162,
      1.6636765803267364, 1.6681872651305825, 1.6727101796415966, 1.6772453570178785,
      1.681792830507429, 1.6863526334483934, 1.6909247992693053, 1.6955093614893326,
      1.7001063537185235, 1.7047158096580513, 1.709337763100463, 1.713972247929926,
      1.718619298122478, 1.723278947746274, 1.7279512309618377, 1.732636182022311,
      1.7373338352737062, 1.7420442251551564, 1.746767386199169, 1.7515033530318782,
      1.7562521603732995, 1.761013843037584, 1.7657884359332727, 1.7705759740635547,
      1.7753764925265212, 1.7801900265154245, 1.785016611318935, 1.789856282321401,
      1.7947090750031072, 1.7995750249405351, 1.804454167806624, 1.809346539371032,
      1.8142521755003989, 1.8191711121586085, 1.8241033854070534, 1.8290490314048973,
      1.8340080864093424, 1.8389805867758937, 1.843966568958626, 1.8489660695104508,
      1.8539791250833855, 1.8590057724288205, 1.864046048397789, 1.8690999899412386,
      1.8741676341103, 1.8792490180565602, 1.8843441790323345, 1.8894531543909392,
      1.8945759815869656, 1.8997126981765553, 1.9048633418176741, 1.9100279502703899,
      1.9152065613971474, 1.9203992131630474, 1.925605943636125, 1.930826790987627,
      1.9360617934922943, 1.9413109895286405, 1.9465744175792332, 1.9518521162309783,
      1.9571441241754002, 1.9624504802089273, 1.9677712232331759, 1.9731063922552343,
      1.978456026387951, 1.9838201648502194, 1.9891988469672663, 1.9945921121709402}};
#endif
}

static __constant__ Exp2Table c_exp2_table = make_exp2_table();

// Loads the table into shared memory (call from every thread, then sync).
__device__ __forceinline__ void load_exp2_table(double* sh) {
  for (int i = threadIdx.x; i < kExp2TableSize; i += blockDim.x) sh[i] = c_exp2_table.t[i];
}

// 2^f for |f| <= 1/(2T): Taylor series of exp(f ln2), coefficients ln2^k / k!.
__device__ __forceinline__ double exp2_poly(double f) {
#if defined(CG_EXP2_T16)
  double p = fma(f, 0.0001540353039338161, 0.0013333558146428443);
  p = fma(f, p, 0.009618129107628477);
  p = fma(f, p, 0.05550410866482158);
#elif defined(CG_EXP2_T64)
  double p = fma(f, 0.0013333558146428443, 0.009618129107628477);
  p = fma(f, p, 0.05550410866482158);
#else
  double p = fma(f, 0.009618129107628477, 0.05550410866482158);
#endif
  p = fma(f, p, 0.24022650695910072);
  p = fma(f, p, 0.6931471805599453);
  return fma(f, p, 1.0);
}

__device__ __forceinline__ double exp2_f64(double x, const double* __restrict__ tab) {
  if (!(x >= -1020.0)) return (x != x) ? x : 0.0;
  if (x >= 1024.0) return INFINITY;
  const double t = fma(x, kExp2Scale, kExpMagic);
  const int N = __double2loint(t);
  const double kf = t - kExpMagic;
  const double f = fma(kf, -kExp2InvScale, x);
  const double y = exp2_poly(f) * tab[N & (kExp2TableSize - 1)];
  return __hiloint2double(__double2hiint(y) + ((N >> kExp2Bits) << 20), __double2loint(y));
}

// exp2_f64 without branches: the same value for every x (bitwise), from the
// table method on x clamped to [-1020, 1024] and selects for the arguments
// outside [-1020, 1024) (0, +inf, NaN).  For loops over many elements, where
// the two early returns of exp2_f64 cost branch and reconvergence code.
__device__ __forceinline__ double exp2_f64_sel(double x, const double* __restrict__ tab) {
  const double xc = fmin(fmax(x, -1020.0), 1024.0);
  const double t = fma(xc, kExp2Scale, kExpMagic);
  const int N = __double2loint(t);
  const double kf = t - kExpMagic;
  const double f = fma(kf, -kExp2InvScale, xc);
  const double y = exp2_poly(f) * tab[N & (kExp2TableSize - 1)];
  double r = __hiloint2double(__double2hiint(y) + ((N >> kExp2Bits) << 20), __double2loint(y));
  r = (x >= 1024.0) ? INFINITY : r;
  return (x >= -1020.0) ? r : ((x != x) ? x : 0.0);
}

// exp2 for the plan pass, whose values only enter sums: the table method on x
// clamped to [-1020, 1024] and one select for NaN.  Equal to exp2_f64 for x in
// [-1020, 1024); +inf at or above 1024 (the clamped point 1024 assembles +inf
// exactly); below -1020 it gives 2^-1020 instead of 0, which no FP64 sum of
// the plan's magnitudes can see.
__device__ __forceinline__ double exp2_f64_clamped(double x, const double* __restrict__ tab) {
  const double xc = fmin(fmax(x, -1020.0), 1024.0);
  const double t = fma(xc, kExp2Scale, kExpMagic);
  const int N = __double2loint(t);
  const double kf = t - kExpMagic;
  const double f = fma(kf, -kExp2InvScale, xc);
  const double y = exp2_poly(f) * tab[N & (kExp2TableSize - 1)];
  const double r =
      __hiloint2double(__double2hiint(y) + ((N >> kExp2Bits) << 20), __double2loint(y));
  return (x != x) ? x : r;
}

// Non-positive-argument variant used inside the LSE passes (x <= 0 by
// construction after the running-max shift): same method, no overflow branch.
__device__ __forceinline__ double exp2_neg_f64(double x, const double* __restrict__ tab) {
  x = fmax(x, -1020.0);
  const double t = fma(x, kExp2Scale, kExpMagic);
  const int N = __double2loint(t);
  const double kf = t - kExpMagic;
  const double f = fma(kf, -kExp2InvScale, x);
  const double y = exp2_poly(f) * tab[N & (kExp2TableSize - 1)];
  return __hiloint2double(__double2hiint(y) + ((N >> kExp2Bits) << 20), __double2loint(y));
}

// 2^(x - k) for an integer k, inside the LSE passes that sum relative to a
// fixed shift k instead of a running maximum: the same table method applied
// to x itself, with k taken off the result's binary exponent (an integer add
// in place of an FP64 subtraction).  x is first raised to lo = k - 1000, so
// terms far below the shift come out near 2^-1000 instead of underflowing
// through the exponent field; the caller guarantees x - k <= 1000.
__device__ __forceinline__ double exp2_shift_f64(double x, double lo, int k,
                                                 const double* __restrict__ tab) {
  x = fmax(x, lo);
  const double t = fma(x, kExp2Scale, kExpMagic);
  const int N = __double2loint(t);
  const double kf = t - kExpMagic;
  const double f = fma(kf, -kExp2InvScale, x);
  const double y = exp2_poly(f) * tab[N & (kExp2TableSize - 1)];
  return __hiloint2double(__double2hiint(y) + (((N >> kExp2Bits) - k) << 20),
                          __double2loint(y));
}

// Hardware 2^x on the SFU (ex2.approx.ftz.f32).
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Mixed-precision 2^x for x <= 0 (the exponent after the running-max shift):
// one FP64 -> FP32 rounding of x, then ex2.approx.ftz.f32 on the whole value.
// The rounding adds at most |x| 2^-24 ln2 relative error to the term 2^x;
// weighted by the term's size (2^x |x| <= 0.53) that stays below ~2e-8 of
// the sum -- under the SFU's own ~2^-22.  Terms below 2^-126 flush to zero.
// (Splitting off the integer part in FP64 first cost four more FP64 adds and
// the integer scaling per element, for no accuracy that the LSE keeps.)
__device__ __forceinline__ float exp2_neg_mixed(double x) {
  return ex2_approx(static_cast<float>(x));
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
