// Sinkhorn BCD on a cost matrix recomputed from point clouds on the tensor
// cores, never stored:
//
//   M_ij = max(0, s * ((|x_i|^2 + |y_j|^2) - 2 x_i . y_j))      (FP32)
//
// with X (n x d) and Y (m x d) in BF16, x_i . y_j accumulated in FP32 by
// tcgen05.mma (kind::f16, BF16 operands, FP32 accumulator in tensor memory)
// and the squared norms summed in FP32 from the same BF16 values.  The
// log-sum-exp passes read M_ij straight out of TMEM (tcgen05.ld) into the
// same base-2 online (max, sum) accumulation as the Sinkhorn passes over a
// stored M, so a pass moves (n + m) d 2 bytes instead of n m sizeof(M).
//
// No reference counterpart: the reference always takes a materialised M
// (src/solvers.h:4-9).  The solver follows the reference's BCD updates
// (src/sinkhorn_bcd_kernel.cu:35-634): alpha_i = eta (log a_i - LSE_j((beta_j
// - M_ij)/eta)), then beta from alpha; its stopping rule is the row-marginal
// test ||T 1 - a||_2 < tol, evaluated for every iterate (the reference's
// iterate-difference pre-test is not used).  Mixed precision follows the
// Sinkhorn passes: SFU exponentials until the marginal estimate drops below
// tol / 2 (or stalls for 8 checks), then FP64 passes confirm convergence.
//
// Kernel structure (one launch per half-step, plus a merge launch):
//   * pts_lse_kernel: a CTA owns a tile of 128 "rows" (points of the side
//     being updated) and a contiguous range of column tiles (points of the
//     other side).  Per column tile: the 128 threads stage both BF16 tiles in
//     shared memory in the canonical no-swizzle K-major layout, one thread
//     issues d/16 MMAs (M = N = 128, K = 16) into a 128-column TMEM
//     accumulator and commits them to an mbarrier; after a bounded wait each
//     of the 8 warps loads 64 columns of its 32 rows (its TMEM lane quarter)
//     and folds the costs into per-thread running (max, sum) pairs; the two
//     halves of a row are merged at the end.  Partials per (row, column
//     range) go to global.
//   * pts_merge_kernel: one thread per row merges the partials in a fixed
//     order, writes the new dual (double-buffered by iteration parity) and,
//     on the row side, the marginal-test term of the previous iterate:
//       rowsum_i = a_i 2^(s2 (alpha_i^k - alpha_i^{k+1})).
//     The last CTA reduces the terms in a fixed order and updates the state.
// Both passes use the same operand roles (the updated side as MMA operand A)
// and the same K order, so row and column passes see identical M_ij.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <cmath>
#include <cstdint>

#include "common.cuh"
#include "curegot_b200.h"
#include "lse.cuh"
#include "workspace.cuh"

namespace cg {
namespace {

constexpr int kPtsTile = 128;     // rows per CTA tile (MMA M) = columns per tile (MMA N)
constexpr int kPtsThreads = 128;  // cost tiles: one thread per TMEM lane / tile row
constexpr int kPtsLseThreads = 256;  // LSE passes: two threads per row, 64 columns each
#ifndef CG_PTS_MINB
#define CG_PTS_MINB 4
#endif
constexpr int kPtsLseMinBlocks = CG_PTS_MINB;  // resident CTAs per SM (64 registers)
constexpr int kPtsMaxD = 64;      // padded feature dimension (multiple of 16)
constexpr int kPtsTmemCols = 128;
constexpr long kPtsSpinLimit = 1L << 24;  // mbarrier polls before giving up
// Poll limit of the first tensor-core completion wait of each tile
// (cg_points_set_wait_limit); the drain wait after a timeout keeps the full limit.
std::atomic<long> g_pts_first_wait{kPtsSpinLimit};
constexpr int kPtsChunk = 8;      // iterations per host check

// Operand tile in shared memory: kPtsTile rows x D BF16, canonical K-major
// layout without swizzle.  K slice s (16 elements, 32 bytes per row) starts
// at s * kSliceBytes; inside a slice the 16-byte chunk c of row r sits at
//   (r / 8) * 256 + c * 128 + (r % 8) * 16,
// i.e. 8 x 16-byte core matrices, leading (K) byte offset 128, stride (row
// group) byte offset 256.
constexpr int kSliceBytes = kPtsTile * 32;
constexpr int kTileBytesMax = kSliceBytes * (kPtsMaxD / 16);  // 16 KB
// Dynamic shared memory per CTA: A and B tiles, beta tile (FP64), norm tile
// (FP32), plus padding that keeps at most 4 CTAs per SM (4 x 128 TMEM
// columns = the whole tensor memory, so tcgen05.alloc never waits).
constexpr int kPtsSmem = 2 * kTileBytesMax + 2 * kPtsTile * 8 + kPtsTile * 4 + 1024;
constexpr int kPtsSmemLaunch = 50 * 1024;
static_assert(kPtsSmem <= kPtsSmemLaunch, "points smem");

struct PtsState {
  int k;           // half-step pairs completed (iterate index)
  int done;
  int niter;
  int max_iter;
  int fast;
  int stall;
  int fast_iters;
  int error;       // nonzero: an mbarrier wait gave up (device status)
  double tol;
  double best;
  double last_err;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with the given parity; false after `limit`
// polls (limit 0: give up without polling).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          long limit = kPtsSpinLimit) {
  for (long it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Shared memory matrix descriptor (tcgen05): start address, leading and
// stride byte offsets (16-byte units), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  return d;
}

// Instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), A and
// B both BF16 (bits 7-9 = 1, bits 10-12 = 1), both K-major, N >> 3 at bit
// 17, M >> 4 at bit 24.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) |
                            (static_cast<uint32_t>(kPtsTile >> 3) << 17) |
                            (static_cast<uint32_t>(kPtsTile >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n"
      " .reg .pred p;\n"
      " setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// 32 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

// Stage rows [r0, r0 + 128) of a padded point array (rows x D BF16, row
// stride D) into the canonical tile layout.  Rows past `rows` are zero.
__device__ __forceinline__ void stage_tile(const uint16_t* __restrict__ P, int rows, int D, int r0,
                                           char* __restrict__ tile) {
  const int cpr = D / 8;  // 16-byte chunks per row
  for (int e = threadIdx.x; e < kPtsTile * cpr; e += blockDim.x) {
    const int r = e / cpr, q = e - r * cpr;
    const int gr = r0 + r;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (gr < rows) v = __ldg(reinterpret_cast<const uint4*>(P + (size_t)gr * D) + q);
    const int s = q >> 1, c = q & 1;
    *reinterpret_cast<uint4*>(tile + s * kSliceBytes + (r >> 3) * 256 + c * 128 + (r & 7) * 16) = v;
  }
}

// Shared-memory tile setup common to both kernels: TMEM allocation (warp 0)
// and the MMA-completion mbarrier.
struct PtsShared {
  uint64_t bar;
  uint32_t tmem;
};

__device__ __forceinline__ void pts_setup(PtsShared& sh) {
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&sh.tmem)),
                 "r"(kPtsTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 0) {
    mbar_init(&sh.bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
}

__device__ __forceinline__ void pts_teardown(PtsShared& sh) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (threadIdx.x < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sh.tmem),
                 "r"(kPtsTmemCols)
                 : "memory");
}

// One column tile: stage B, MMA into TMEM, wait.  Returns false when the
// wait gave up (the accumulator is then not read).  first_wait bounds the
// completion wait; whatever it is, a wait that gave up is followed by one at
// the full limit, so the MMAs have drained before TMEM can be freed.
__device__ __forceinline__ bool pts_tile_mma(PtsShared& sh, const char* tA, char* tB, int D,
                                             uint32_t& phase, long first_wait) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0) {
    tc_fence_after();
    const uint32_t a0 = smem_u32(tA), b0 = smem_u32(tB);
    for (int s = 0; s < D / 16; ++s)
      mma_bf16(sh.tmem, umma_desc(a0 + s * kSliceBytes, 128, 256),
               umma_desc(b0 + s * kSliceBytes, 128, 256), s > 0 ? 1u : 0u);
    mma_commit(&sh.bar);
  }
  bool ok = mbar_wait(&sh.bar, phase, first_wait);
  ok = __syncthreads_and(ok) != 0;
  if (!ok) mbar_wait(&sh.bar, phase);  // bounded: let the MMAs drain before TMEM is freed
  phase ^= 1u;
  tc_fence_after();
  return ok;
}

// M_ij of one accumulator element (row norm nr, column norm nc).
__device__ __forceinline__ float pts_cost(float dot, float nr, float nc, float scale) {
  return fmaxf(0.0f, scale * fmaf(-2.0f, dot, nr + nc));
}

}  // namespace

// Cost tiles: M (rows x cols, FP32, row-major) from the padded points.
__global__ void __launch_bounds__(kPtsThreads) pts_cost_kernel(
    const uint16_t* __restrict__ P, const uint16_t* __restrict__ Q, const float* __restrict__ nP,
    const float* __restrict__ nQ, int rows, int cols, int D, float scale, float* __restrict__ M,
    int* __restrict__ error, long first_wait) {
  extern __shared__ __align__(1024) char smem[];
  __shared__ PtsShared sh;
  char* tA = smem;
  char* tB = smem + kTileBytesMax;
  pts_setup(sh);
  const int r0 = blockIdx.x * kPtsTile, c0 = blockIdx.y * kPtsTile;
  stage_tile(P, rows, D, r0, tA);
  stage_tile(Q, cols, D, c0, tB);
  uint32_t phase = 0;
  const bool ok = pts_tile_mma(sh, tA, tB, D, phase, first_wait);
  if (!ok) {
    if (threadIdx.x == 0) atomicExch(error, 1);
  } else {
    const int warp = threadIdx.x >> 5;
    const int r = r0 + threadIdx.x;
    const float nr = r < rows ? nP[r] : 0.0f;
#pragma unroll 1
    for (int cb = 0; cb < kPtsTile; cb += 32) {
      float v[32];
      tmem_ld32(sh.tmem + (static_cast<uint32_t>(warp * 32) << 16) + cb, v);
      if (r < rows) {
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          const int c = c0 + cb + q;
          if (c < cols) M[(size_t)r * cols + c] = pts_cost(v[q], nr, nQ[c], scale);
        }
      }
    }
  }
  pts_teardown(sh);
}

// Statistics of the unscaled cost c_ij = max(0, |x_i|^2 + |y_j|^2 - 2 x_i . y_j)
// (the FP32 values the cost tiles hold at scale 1), for the /max and /median
// normalisers: one pass per radix level over the recomputed tiles.  The keys
// are the FP32 bit patterns (c >= 0, sign cleared), which order like the
// values.  Level 0 also takes the maximum; level L histograms the digit
// (12, 12, 8 bits from the top) of the keys whose higher digits equal the
// prefix found so far (sel[0]).
constexpr int kStatBins = 4096;
struct StatSel {
  unsigned long long krem;  // rank (1-based) still to find inside the prefix
  unsigned int prefix;      // digits found so far
  unsigned int maxbits;     // maximum key (level 0)
};
__device__ __forceinline__ int stat_shift(int level) { return level == 0 ? 20 : (level == 1 ? 8 : 0); }
__device__ __forceinline__ int stat_width(int level) { return level == 2 ? 8 : 12; }

__global__ void __launch_bounds__(kPtsThreads) pts_stats_kernel(
    const uint16_t* __restrict__ P, const uint16_t* __restrict__ Q, const float* __restrict__ nP,
    const float* __restrict__ nQ, int rows, int cols, int D, int level,
    const StatSel* __restrict__ sel, unsigned long long* __restrict__ hist,
    unsigned int* __restrict__ maxbits, int* __restrict__ error, long first_wait) {
  extern __shared__ __align__(1024) char smem[];
  __shared__ PtsShared sh;
  __shared__ unsigned int shist[kStatBins];
  __shared__ unsigned int smax;
  char* tA = smem;
  char* tB = smem + kTileBytesMax;
  for (int b = threadIdx.x; b < kStatBins; b += blockDim.x) shist[b] = 0u;
  if (threadIdx.x == 0) smax = 0u;
  pts_setup(sh);  // ends with a block barrier
  const int r0 = blockIdx.x * kPtsTile, c0 = blockIdx.y * kPtsTile;
  stage_tile(P, rows, D, r0, tA);
  stage_tile(Q, cols, D, c0, tB);
  uint32_t phase = 0;
  const bool ok = pts_tile_mma(sh, tA, tB, D, phase, first_wait);
  const int sh_lo = stat_shift(level), width = stat_width(level);
  const unsigned int prefix = (level == 0) ? 0u : sel->prefix;
  const int sh_hi = sh_lo + width;
  if (!ok) {
    if (threadIdx.x == 0) atomicExch(error, 1);
  } else {
    const int warp = threadIdx.x >> 5;
    const int r = r0 + threadIdx.x;
    const float nr = r < rows ? nP[r] : 0.0f;
    const int lane = threadIdx.x & 31;
    unsigned int mymax = 0u;
#pragma unroll 1
    for (int cb = 0; cb < kPtsTile; cb += 32) {
      float v[32];
      tmem_ld32(sh.tmem + (static_cast<uint32_t>(warp * 32) << 16) + cb, v);
#pragma unroll 4
      for (int q = 0; q < 32; ++q) {
        const int c = c0 + cb + q;
        int bin = -1;
        if (r < rows && c < cols) {
          const unsigned int key = __float_as_uint(pts_cost(v[q], nr, nQ[c], 1.0f)) & 0x7FFFFFFFu;
          if (level == 0) mymax = max(mymax, key);
          if (level == 0 || (key >> sh_hi) == prefix)
            bin = (int)((key >> sh_lo) & ((1u << width) - 1u));
        }
        // warp-aggregated increment: one shared atomic per distinct bin
        const unsigned int act = __ballot_sync(0xffffffffu, bin >= 0);
        if (bin >= 0) {
          const unsigned int peers = __match_any_sync(act, bin);
          if ((__ffs(peers) - 1) == lane) atomicAdd(&shist[bin], (unsigned)__popc(peers));
        }
      }
    }
    if (level == 0) atomicMax(&smax, mymax);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < kStatBins; b += blockDim.x)
    if (shist[b]) atomicAdd(&hist[b], (unsigned long long)shist[b]);
  if (level == 0 && threadIdx.x == 0) atomicMax(maxbits, smax);
  pts_teardown(sh);
}

// One CTA of 1024 threads: the bin (ascending) holding the krem-th smallest
// key of this level; extends the prefix and clears the histogram.
__global__ void __launch_bounds__(1024) pts_stats_select_kernel(StatSel* sel,
                                                                 unsigned long long* hist,
                                                                 int level) {
  __shared__ unsigned long long part[1024];
  __shared__ int sh_b;
  __shared__ unsigned long long sh_below;
  const int t = threadIdx.x;
  const int nb = 1 << stat_width(level);
  unsigned long long c[4], mine = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int b = 4 * t + q;
    c[q] = (b < nb) ? hist[b] : 0ull;
    mine += c[q];
  }
  part[t] = mine;
  if (t == 0) sh_b = -1;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {  // inclusive prefix scan
    const unsigned long long v = (t >= off) ? part[t - off] : 0ull;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  const unsigned long long krem = sel->krem;
  const unsigned long long before = (t > 0) ? part[t - 1] : 0ull;
  if (before < krem && part[t] >= krem) {
    unsigned long long below = before;
    for (int q = 0; q < 4; ++q) {
      if (below + c[q] >= krem) {
        sh_b = 4 * t + q;
        sh_below = below;
        break;
      }
      below += c[q];
    }
  }
  __syncthreads();
  if (t == 0 && sh_b >= 0) {
    sel->krem = krem - sh_below;
    sel->prefix = (level == 0 ? 0u : (sel->prefix << stat_width(level))) | (unsigned int)sh_b;
  }
  __syncthreads();
  for (int b = t; b < kStatBins; b += blockDim.x) hist[b] = 0ull;
}

// Partial LSE over the column tiles [t0, t1) for the 128 rows of tile
// blockIdx.x: part[(split * rows_pad + r) * 2 + {0, 1}] = (max, sum) in base 2
// of xs_j - s2 M_rj, xs the other side's scaled duals.  The state's
// precision flag picks SFU or FP64 exponentials for the whole pass.
__global__ void __launch_bounds__(kPtsLseThreads, kPtsLseMinBlocks) pts_lse_kernel(
    const uint16_t* __restrict__ P, const uint16_t* __restrict__ Q, const float* __restrict__ nP,
    const float* __restrict__ nQ, int rows, int cols, int D, float scale,
    const double* __restrict__ xs_base, size_t xs_stride, int xs_parity, double s2,
    int tiles_per_split, double* __restrict__ part, int rows_pad, PtsState* __restrict__ st,
    long first_wait) {
  extern __shared__ __align__(1024) char smem[];
  __shared__ PtsShared sh;
  __shared__ double tab[kExp2TableSize];
  if (ldcg(&st->done)) return;
  const bool fast = ldcg(&st->fast) != 0;
  const int k = ldcg(&st->k);
  // row side: beta^k (parity k); column side: the alpha^{k+1} just written
  const double* __restrict__ xs = xs_base + (size_t)((k + xs_parity) & 1) * xs_stride;
  char* tA = smem;
  char* tB = smem + kTileBytesMax;
  double* sx = reinterpret_cast<double*>(smem + 2 * kTileBytesMax);
  float* sn = reinterpret_cast<float*>(smem + 2 * kTileBytesMax + 2 * kPtsTile * 8);
  load_exp2_table(tab);
  pts_setup(sh);

  const int r0 = blockIdx.x * kPtsTile;
  const int split = blockIdx.y;
  const int ntiles = (cols + kPtsTile - 1) / kPtsTile;
  const int t0 = split * tiles_per_split, t1 = min(ntiles, t0 + tiles_per_split);
  stage_tile(P, rows, D, r0, tA);
  // warp w reads TMEM lanes 32 (w % 4) .. + 31 (its lane quarter) and the
  // accumulator columns 64 (w / 4) .. + 63 of every tile
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quarter = warp & 3, half = warp >> 2;
  const int rl = quarter * 32 + lane;  // row within the tile
  const int r = r0 + rl;
  const float nr = r < rows ? nP[r] : 0.0f;
  double mx = kNegInf, s = 0.0;
  uint32_t phase = 0;
  bool ok = true;
  for (int t = t0; t < t1 && ok; ++t) {
    const int c0 = t * kPtsTile;
    __syncthreads();  // every thread is done with the previous tile's sx / sn
    stage_tile(Q, cols, D, c0, tB);
    for (int c = threadIdx.x; c < kPtsTile; c += blockDim.x) {
      const int gc = c0 + c;
      sx[c] = gc < cols ? xs[gc] : 0.0;
      sn[c] = gc < cols ? nQ[gc] : 0.0f;
    }
    ok = pts_tile_mma(sh, tA, tB, D, phase, first_wait);
    if (!ok) break;
#pragma unroll 1
    for (int cb = half * 64; cb < half * 64 + 64; cb += 32) {
      float v[32];
      tmem_ld32(sh.tmem + (static_cast<uint32_t>(quarter * 32) << 16) + cb, v);
#pragma unroll
      for (int q0 = 0; q0 < 32; q0 += 4) {
        double dd[4];
        bool in[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int c = cb + q0 + u;
          in[u] = c0 + c < cols;
          const float mc = pts_cost(v[q0 + u], nr, sn[c], scale);
          dd[u] = fma(-s2, static_cast<double>(mc), sx[c]);
        }
        if (fast)
          lse_chunk<true, 4>(dd, in, mx, s, tab);
        else
          lse_chunk<false, 4>(dd, in, mx, s, tab);
      }
    }
  }
  if (!ok && threadIdx.x == 0) atomicExch(&st->error, 1);
  // the two column halves of each row, merged in a fixed order
  double* hmx = sx;  // the tile buffers are free now
  double* hs = sx + kPtsTile;
  __syncthreads();
  if (half == 1) {
    hmx[rl] = mx;
    hs[rl] = s;
  }
  __syncthreads();
  if (half == 0 && r < rows) {
    lse2_merge(mx, s, hmx[rl], hs[rl], tab);
    double* o = part + ((size_t)split * rows_pad + r) * 2;
    o[0] = mx;
    o[1] = s;
  }
  pts_teardown(sh);
}

// Merge of the partials: new duals of the updated side (parity k+1), and on
// the row side the marginal test of iterate k.
__global__ void __launch_bounds__(256) pts_merge_kernel(
    const double* __restrict__ part, int rows, int rows_pad, int splits, double eta, double s2,
    const double* __restrict__ logw, const double* __restrict__ w, double* __restrict__ dual_base,
    double* __restrict__ duals_base, size_t stride, int row_side, unsigned int* counter,
    double* __restrict__ block_err, PtsState* __restrict__ st) {
  __shared__ double tab[kExp2TableSize];
  __shared__ double red[8];
  if (ldcg(&st->done)) return;
  load_exp2_table(tab);
  __syncthreads();
  const int k = ldcg(&st->k);
  const bool check = row_side && k >= 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e2 = 0.0;
  if (i < rows) {
    double M0 = kNegInf, S0 = 0.0;
    for (int q = 0; q < splits; ++q) {
      const double* o = part + ((size_t)q * rows_pad + i) * 2;
      lse2_merge(M0, S0, ldcg(o), ldcg(o + 1), tab);
    }
    const double v = eta * logw[i] - (eta * kLn2) * (M0 + log2(S0));
    const double vs = v * s2;
    dual_base[(size_t)((k + 1) & 1) * stride + i] = v;
    duals_base[(size_t)((k + 1) & 1) * stride + i] = vs;
    if (check) {
      const double wi = w[i];
      const double e = wi * exp2_f64(duals_base[(size_t)(k & 1) * stride + i] - vs, tab) - wi;
      e2 = e * e;
    }
  }
  if (!row_side) {
    // column side: the last CTA advances the iterate counter
    if (!elect_last(counter, gridDim.x)) return;
    if (threadIdx.x == 0) {
      const int kn = k + 1;
      st->k = kn;
      if (ldcg(&st->fast)) st->fast_iters += 1;
      if (kn >= st->max_iter) {
        st->done = 1;
        st->niter = kn;
      }
    }
    return;
  }
  const double bsum = cta_sum(e2, red);
  if (threadIdx.x == 0) block_err[blockIdx.x] = bsum;
  if (!elect_last(counter, gridDim.x)) return;
  if (!check) return;
  double v = 0.0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += blockDim.x) v += ldcg(block_err + q);
  const double tot = cta_sum(v, red);
  if (threadIdx.x == 0) {
    const double err = sqrt(tot);
    st->last_err = err;
    if (!ldcg(&st->fast)) {
      if (err < st->tol) {
        st->done = 1;
        st->niter = k;
      }
    } else if (err < 0.5 * st->tol) {
      st->fast = 0;
    } else if (err < 0.9 * st->best) {
      st->best = err;
      st->stall = 0;
    } else if (++st->stall >= 8) {
      st->fast = 0;
    }
  }
}

// Padded BF16 copy (rows x D, zero columns past d) and FP32 squared norms.
__global__ void pts_pad_kernel(const uint16_t* __restrict__ X, int rows, int d, int D,
                               uint16_t* __restrict__ Xp, float* __restrict__ nrm) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  float acc = 0.0f;
  for (int c = 0; c < D; ++c) {
    const uint16_t h = c < d ? X[(size_t)r * d + c] : uint16_t(0);
    Xp[(size_t)r * D + c] = h;
    const float f = __uint_as_float(static_cast<uint32_t>(h) << 16);
    acc = fmaf(f, f, acc);
  }
  nrm[r] = acc;
}

__global__ void pts_init_kernel(const double* __restrict__ a, const double* __restrict__ b, int n,
                                int m, double* loga, double* logb, double* al, double* als,
                                double* be, double* bes, PtsState* st, int max_iter, double tol,
                                int fast) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int i = tid; i < n; i += stride) {
    loga[i] = log(a[i]);
    al[i] = 0.0;
    als[i] = 0.0;
  }
  for (int j = tid; j < m; j += stride) {
    logb[j] = log(b[j]);
    be[j] = 0.0;
    bes[j] = 0.0;
  }
  if (tid == 0) {
    st->k = 0;
    st->done = max_iter <= 0 ? 1 : 0;
    st->niter = 0;
    st->max_iter = max_iter;
    st->fast = fast;
    st->stall = 0;
    st->fast_iters = 0;
    st->error = 0;
    st->tol = tol;
    st->best = INFINITY;
    st->last_err = INFINITY;
  }
}

__global__ void pts_out_kernel(const double* __restrict__ al_base, const double* __restrict__ be_base,
                               size_t sa, size_t sb, int n, int m, const PtsState* __restrict__ st,
                               double* __restrict__ dual) {
  const int k = st->niter;
  const double* al = al_base + (size_t)(k & 1) * sa;
  const double* be = be_base + (size_t)(k & 1) * sb;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  for (int i = tid; i < n; i += stride) dual[i] = al[i];
  for (int j = tid; j < m; j += stride) dual[n + j] = be[j];
}

namespace {

int check_points_args(int n, int m, int d, double scale) {
  if (n <= 0 || m <= 0 || d <= 0 || d > kPtsMaxD || !(scale > 0.0) || !std::isfinite(scale)) {
    set_last_error("points: need n, m > 0, 0 < d <= 64 and a positive finite cost scale",
                   __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  return CG_OK;
}

int pts_attrs() {
  static thread_local int done_dev = -1;
  int dev = 0;
  CG_TRY_CUDA(cudaGetDevice(&dev));
  if (done_dev == dev) return CG_OK;
  CG_TRY_CUDA(cudaFuncSetAttribute(pts_cost_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   kPtsSmemLaunch));
  CG_TRY_CUDA(cudaFuncSetAttribute(pts_lse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   kPtsSmemLaunch));
  CG_TRY_CUDA(cudaFuncSetAttribute(pts_stats_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   kPtsSmemLaunch));
  done_dev = dev;
  return CG_OK;
}

int pad_dim(int d) { return ((d + 15) / 16) * 16; }

struct PtsPoints {
  uint16_t* Xp;
  uint16_t* Yp;
  float* nX;
  float* nY;
};

}  // namespace
}  // namespace cg

using namespace cg;

extern "C" int cg_points_cost_bf16(const uint16_t* X, const uint16_t* Y, int n, int m, int d,
                                   double cost_scale, float* M, cudaStream_t stream) {
  CG_TRY(check_points_args(n, m, d, cost_scale));
  if (!X || !Y || !M) {
    set_last_error("points: null pointer", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  CG_TRY(pts_attrs());
  const int D = pad_dim(d);
  Workspace W(stream);
  const size_t oXp = W.reserve<uint16_t>((size_t)n * D), oYp = W.reserve<uint16_t>((size_t)m * D);
  const size_t onX = W.reserve<float>(n), onY = W.reserve<float>(m);
  const size_t oerr = W.reserve<int>(1);
  CG_TRY(W.allocate());
  uint16_t* Xp = W.at<uint16_t>(oXp);
  uint16_t* Yp = W.at<uint16_t>(oYp);
  float* nX = W.at<float>(onX);
  float* nY = W.at<float>(onY);
  int* err = W.at<int>(oerr);
  int rc = CG_OK;
  do {
    if ((rc = status_from_cuda(cudaMemsetAsync(err, 0, sizeof(int), stream))) != CG_OK) break;
    { pts_pad_kernel<<<(n + 255) / 256, 256, 0, stream>>>(X, n, d, D, Xp, nX); count_launch(); }
    { pts_pad_kernel<<<(m + 255) / 256, 256, 0, stream>>>(Y, m, d, D, Yp, nY); count_launch(); }
    dim3 grid((n + kPtsTile - 1) / kPtsTile, (m + kPtsTile - 1) / kPtsTile);
    { pts_cost_kernel<<<grid, kPtsThreads, kPtsSmemLaunch, stream>>>(
        Xp, Yp, nX, nY, n, m, D, static_cast<float>(cost_scale), M, err,
        g_pts_first_wait.load()); count_launch(); }
    if ((rc = status_from_cuda(cudaGetLastError())) != CG_OK) break;
    int herr = 0;
    if ((rc = read_device(&herr, err, sizeof(int), stream)) != CG_OK) break;
    if (herr) {
      set_last_error("points: tensor-core completion wait timed out", __FILE__, __LINE__);
      rc = CG_ERR_TIMEOUT;
    }
  } while (false);
  W.release();
  return rc;
}

extern "C" int cg_bcd_points_bf16(const uint16_t* X, const uint16_t* Y, int n, int m, int d,
                                  double cost_scale, const double* a, const double* b, double reg,
                                  int max_iter, double tol, int precision, int* niter_out,
                                  double* dual, int* fast_iters_out, cudaStream_t stream) {
  CG_TRY(check_points_args(n, m, d, cost_scale));
  if (!X || !Y || !a || !b || !dual || !(reg > 0.0) || max_iter < 0 ||
      (precision != CG_POINTS_FP64 && precision != CG_POINTS_MIXED)) {
    set_last_error("points: invalid argument", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  CG_TRY(pts_attrs());
  const int D = pad_dim(d);
  const int sms = sm_count_current();
  const int n_pad = ((n + kPtsTile - 1) / kPtsTile) * kPtsTile;
  const int m_pad = ((m + kPtsTile - 1) / kPtsTile) * kPtsTile;
  const int rt_n = n_pad / kPtsTile, rt_m = m_pad / kPtsTile;
  // column splits: about 4 CTAs per SM (one resident wave) per pass
  auto splits_for = [&](int row_tiles, int col_tiles, int& tiles_per_split) {
    int sp = std::max(1, std::min(col_tiles, (4 * sms + row_tiles - 1) / row_tiles));
    tiles_per_split = (col_tiles + sp - 1) / sp;
    return (col_tiles + tiles_per_split - 1) / tiles_per_split;
  };
  int tps_row = 1, tps_col = 1;
  const int sp_row = splits_for(rt_n, rt_m, tps_row);
  const int sp_col = splits_for(rt_m, rt_n, tps_col);
  const size_t part_elems = 2 * (size_t)std::max(sp_row * n_pad, sp_col * m_pad);
  const int mb_n = (n + 255) / 256, mb_m = (m + 255) / 256;

  Workspace W(stream);
  const size_t oXp = W.reserve<uint16_t>((size_t)n * D), oYp = W.reserve<uint16_t>((size_t)m * D);
  const size_t onX = W.reserve<float>(n), onY = W.reserve<float>(m);
  const size_t ologa = W.reserve<double>(n), ologb = W.reserve<double>(m);
  const size_t oal = W.reserve<double>(2 * (size_t)n), oals = W.reserve<double>(2 * (size_t)n);
  const size_t obe = W.reserve<double>(2 * (size_t)m), obes = W.reserve<double>(2 * (size_t)m);
  const size_t opart = W.reserve<double>(part_elems);
  const size_t oberr = W.reserve<double>(std::max(mb_n, 1));
  const size_t ocnt = W.reserve<unsigned int>(2);
  const size_t ost = W.reserve<PtsState>(1);
  CG_TRY(W.allocate());
  uint16_t* Xp = W.at<uint16_t>(oXp);
  uint16_t* Yp = W.at<uint16_t>(oYp);
  float* nX = W.at<float>(onX);
  float* nY = W.at<float>(onY);
  double* loga = W.at<double>(ologa);
  double* logb = W.at<double>(ologb);
  double* al = W.at<double>(oal);
  double* als = W.at<double>(oals);
  double* be = W.at<double>(obe);
  double* bes = W.at<double>(obes);
  double* part = W.at<double>(opart);
  double* berr = W.at<double>(oberr);
  unsigned int* cnt = W.at<unsigned int>(ocnt);
  PtsState* st = W.at<PtsState>(ost);

  const double s2 = kLog2e / reg;
  const float sc = static_cast<float>(cost_scale);
  const long first_wait = g_pts_first_wait.load();
  int rc = CG_OK;
  PtsState hs{};
  do {
    if ((rc = status_from_cuda(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned int), stream))) != CG_OK)
      break;
    { pts_pad_kernel<<<(n + 255) / 256, 256, 0, stream>>>(X, n, d, D, Xp, nX); count_launch(); }
    { pts_pad_kernel<<<(m + 255) / 256, 256, 0, stream>>>(Y, m, d, D, Yp, nY); count_launch(); }
    { pts_init_kernel<<<std::max(1, std::min((std::max(n, m) + 255) / 256, 256)), 256, 0, stream>>>(
        a, b, n, m, loga, logb, al, als, be, bes, st, max_iter, tol,
        precision == CG_POINTS_MIXED ? 1 : 0); count_launch(); }
    const dim3 grow(rt_n, sp_row), gcol(rt_m, sp_col);
    for (int it0 = 0; it0 < max_iter; it0 += kPtsChunk) {
      const int todo = std::min(kPtsChunk, max_iter - it0);
      for (int q = 0; q < todo; ++q) {
        // row side: alpha^{k+1} from beta^k
        { pts_lse_kernel<<<grow, kPtsLseThreads, kPtsSmemLaunch, stream>>>(
            Xp, Yp, nX, nY, n, m, D, sc, bes, (size_t)m, 0, s2, tps_row, part, n_pad, st,
            first_wait); count_launch(); }
        { pts_merge_kernel<<<mb_n, 256, 0, stream>>>(part, n, n_pad, sp_row, reg, s2, loga, a, al, als,
                                                    (size_t)n, 1, cnt, berr, st); count_launch(); }
        // column side: beta^{k+1} from alpha^{k+1}
        { pts_lse_kernel<<<gcol, kPtsLseThreads, kPtsSmemLaunch, stream>>>(
            Yp, Xp, nY, nX, m, n, D, sc, als, (size_t)n, 1, s2, tps_col, part, m_pad, st,
            first_wait); count_launch(); }
        { pts_merge_kernel<<<mb_m, 256, 0, stream>>>(part, m, m_pad, sp_col, reg, s2, logb, b, be, bes,
                                                    (size_t)m, 0, cnt + 1, berr, st); count_launch(); }
      }
      if ((rc = status_from_cuda(cudaGetLastError())) != CG_OK) break;
      if ((rc = read_device(&hs, st, sizeof(PtsState), stream)) != CG_OK) break;
      if (hs.error) break;
      if (hs.done) break;
    }
    if (rc != CG_OK) break;
    if (hs.error) {
      set_last_error("points: tensor-core completion wait timed out", __FILE__, __LINE__);
      rc = CG_ERR_TIMEOUT;
      break;
    }
    if (!hs.done && (rc = read_device(&hs, st, sizeof(PtsState), stream)) != CG_OK) break;
    { pts_out_kernel<<<std::max(1, std::min((n + m + 255) / 256, 256)), 256, 0, stream>>>(
        al, be, (size_t)n, (size_t)m, n, m, st, dual); count_launch(); }
    if ((rc = status_from_cuda(cudaGetLastError())) != CG_OK) break;
    if (niter_out) *niter_out = hs.niter;
    if (fast_iters_out) *fast_iters_out = hs.fast_iters;
  } while (false);
  W.release();
  return rc;
}

extern "C" int cg_points_set_wait_limit(long long polls) {
  cg::g_pts_first_wait.store(polls < 0 ? cg::kPtsSpinLimit : (long)polls);
  return CG_OK;
}

extern "C" int cg_points_cost_stats_bf16(const uint16_t* X, const uint16_t* Y, int n, int m,
                                         int d, double* max_out, double* median_out,
                                         cudaStream_t stream) {
  CG_TRY(check_points_args(n, m, d, 1.0));
  if (!X || !Y || !max_out || !median_out) {
    set_last_error("points: null pointer", __FILE__, __LINE__);
    return CG_ERR_INVALID_ARG;
  }
  CG_TRY(pts_attrs());
  const int D = pad_dim(d);
  Workspace W(stream);
  const size_t oXp = W.reserve<uint16_t>((size_t)n * D), oYp = W.reserve<uint16_t>((size_t)m * D);
  const size_t onX = W.reserve<float>(n), onY = W.reserve<float>(m);
  const size_t ohist = W.reserve<unsigned long long>(kStatBins);
  const size_t osel = W.reserve<StatSel>(1);
  const size_t omax = W.reserve<unsigned int>(1);
  const size_t oerr = W.reserve<int>(1);
  CG_TRY(W.allocate());
  uint16_t* Xp = W.at<uint16_t>(oXp);
  uint16_t* Yp = W.at<uint16_t>(oYp);
  float* nX = W.at<float>(onX);
  float* nY = W.at<float>(onY);
  unsigned long long* hist = W.at<unsigned long long>(ohist);
  StatSel* sel = W.at<StatSel>(osel);
  unsigned int* maxbits = W.at<unsigned int>(omax);
  int* err = W.at<int>(oerr);
  const long first_wait = g_pts_first_wait.load();
  int rc = CG_OK;
  do {
    // lower median: the ceil(N / 2)-th smallest of the N = n m values
    StatSel hs{};
    hs.krem = ((unsigned long long)n * (unsigned long long)m + 1ull) / 2ull;
    if ((rc = status_from_cuda(cudaMemcpyAsync(sel, &hs, sizeof(StatSel), cudaMemcpyHostToDevice,
                                               stream))) != CG_OK)
      break;
    if ((rc = status_from_cuda(cudaMemsetAsync(hist, 0, kStatBins * sizeof(unsigned long long),
                                               stream))) != CG_OK)
      break;
    if ((rc = status_from_cuda(cudaMemsetAsync(maxbits, 0, sizeof(unsigned int), stream))) != CG_OK)
      break;
    if ((rc = status_from_cuda(cudaMemsetAsync(err, 0, sizeof(int), stream))) != CG_OK) break;
    { pts_pad_kernel<<<(n + 255) / 256, 256, 0, stream>>>(X, n, d, D, Xp, nX); count_launch(); }
    { pts_pad_kernel<<<(m + 255) / 256, 256, 0, stream>>>(Y, m, d, D, Yp, nY); count_launch(); }
    dim3 grid((n + kPtsTile - 1) / kPtsTile, (m + kPtsTile - 1) / kPtsTile);
    for (int level = 0; level < 3; ++level) {
      { pts_stats_kernel<<<grid, kPtsThreads, kPtsSmemLaunch, stream>>>(
          Xp, Yp, nX, nY, n, m, D, level, sel, hist, maxbits, err, first_wait); count_launch(); }
      { pts_stats_select_kernel<<<1, 1024, 0, stream>>>(sel, hist, level); count_launch(); }
    }
    if ((rc = status_from_cuda(cudaGetLastError())) != CG_OK) break;
    struct {
      StatSel s;
      unsigned int mx;
      int err;
    } out{};
    const ReadSpan spans[3] = {{&out.s, sel, sizeof(StatSel)},
                               {&out.mx, maxbits, sizeof(unsigned int)},
                               {&out.err, err, sizeof(int)}};
    if ((rc = read_device_spans(spans, 3, stream)) != CG_OK) break;
    if (out.err) {
      set_last_error("points: tensor-core completion wait timed out", __FILE__, __LINE__);
      rc = CG_ERR_TIMEOUT;
      break;
    }
    float fmx, fmed;
    const unsigned int mb = out.mx, kb = out.s.prefix;
    std::memcpy(&fmx, &mb, sizeof(float));
    std::memcpy(&fmed, &kb, sizeof(float));
    *max_out = fmx;
    *median_out = fmed;
  } while (false);
  W.release();
  return rc;
}
