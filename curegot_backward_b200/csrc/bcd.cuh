// Batched Sinkhorn BCD: problem descriptors and pass launchers.
//
// One launch of a pass covers every problem of a batch: CTA b of the launch
// belongs to problem cta_prob[b] (or to problem 0 when cta_prob is null) and
// is its (b - cta_start[p])-th CTA.  The single-problem solver uses a batch
// of one; the serving engine packs many problems into the same launches.
#pragma once

#include "common.cuh"

namespace cg {

// Device-side BCD control state (one per problem).  The loop semantics are
// those of cuda_sinkhorn_bcd (reference src/sinkhorn_bcd_kernel.cu:532-592).
struct BcdState {
  int iter;           // iterations completed so far
  int phase;          // 0: no test (fixed sweeps); 1: iterate-difference test; 2: marginal test
  int check_pending;  // the marginal test of the current iterate is due
  int done;           // converged or max_iter reached
  int niter;          // reference niter
  int max_iter;
  int fast;           // mixed precision: 1 = SFU exp passes, 0 = FP64 exp passes
  int stall;          // mixed precision: checks without improvement
  double tol;
  double last_err;    // last test value (diff or marginal error)
  double best_est;    // mixed precision: best fast marginal estimate
  double stat_a[3];   // (count, mean, M2) of alpha^{t+1} - alpha^t
  int fast_iters;     // iterations run with SFU passes
  int nonfinite;      // a stop-test value was NaN / Inf (non-finite M, a, b or x0): done
  int error;          // a bounded device wait gave up (staging ring): done
  int pad_;
  // Largest dual change, in base-2 exponent units, of the latest row pass
  // (max_i |alphas^{t+1}_i - alphas^t_i|) and column pass; +inf until known.
  // The next pass of the other side sums relative to the previous LSE of its
  // row / column when this bound is below kShiftDrift.
  double drift_a;
  double drift_b;
  unsigned long long acc_a;  // running maxima (bit patterns of non-negative doubles)
  unsigned long long acc_b;
  // The float-pair copies of the latest scaled duals (BcdProb asplit /
  // bsplit) are out of range (|value| >= kSplitMax) or absent: set by the
  // pass that writes them, cleared by the last CTA of the pass that reads them.
  int split_bad_a;
  int split_bad_b;
};

// Float-pair duals for the mixed-precision shifted passes: v = hi + lo with hi
// a multiple of 2^-9 (exact in FP32 for |v| < kSplitMax) and lo the FP32
// rounding of the remainder.
constexpr double kSplitMax = 16384.0;

struct BcdProb {
  const void* M;        // row-major n x m (float or double, fixed per launch)
  int n, m;
  int rows_per_cta;     // row pass: rows per CTA (1, 2, 4 or 8)
  int row_ctas;         // row pass CTAs
  int col_splits;       // column pass: row splits per strip
  int col_strips;       // column pass: strips
  double eta;
  double s2;            // log2(e) / eta: scale into the base-2 exponent domain
  const double* a;      // [n]
  const double* loga;   // [n]
  const double* logb;   // [m]
  double* alpha[2];     // double-buffered duals (natural units)
  double* beta[2];
  double* alphas[2];    // the same duals times s2
  double* betas[2];
  double* col_m;        // [col_splits * m] partial LSE maxima (base 2)
  double* col_s;        // [col_splits * m] partial LSE sums
  double* row_part;     // [row_ctas * 4] marginal / stats partials
  double* col_part;     // [col_strips * 3] stats partials
  unsigned int* counters;  // [2 + col_strips], zero-initialised
  BcdState* st;
  // float-pair copies of the latest alphas / betas (FP32-M problems; null
  // otherwise): the SFU passes form exponents from them in FP32
  float2* asplit;       // [n]
  float2* bsplit;       // [m]
};

// total_ctas virtual CTAs; grid_cap > 0 limits the launched grid (the
// kernels loop over the virtual CTAs), 0 launches one CTA per virtual CTA.
void launch_bcd_row(bool f32, const BcdProb* d_probs, const int* d_cta_prob,
                    const int* d_cta_start, int total_ctas, cudaStream_t stream,
                    int grid_cap = 0);
void launch_bcd_col(bool f32, const BcdProb* d_probs, const int* d_cta_prob,
                    const int* d_cta_start, int total_ctas, cudaStream_t stream,
                    int grid_cap = 0);
template <typename TM>
void launch_plan(const TM* M, const double* alpha, const double* beta, double* P,
                 double inv_eta, int n, int m, cudaStream_t stream);

// Pass kernels stream long rows / column strips through shared-memory rings
// filled by bulk copies (process-wide; default off, measured slower on B200).  Off: every pass reads M
// with vector loads straight into registers.  Same results either way.
void bcd_set_staging(bool on);
// L2 bulk-prefetch distance (chunks ahead) of the register-path passes; 0 off.
void bcd_set_l2_prefetch(int chunks);
int bcd_l2_prefetch();  // the current distance (also used by the plan pass)

// Shifted LSE sums (default on): passes after the first sum relative to the
// previous LSE of their row / column when the drift bound allows; off, every
// pass keeps a running maximum.
void bcd_set_shifted_lse(bool on);

// Pass kernel flag word: bit 0 staging, bit 1 online maximum only, bits 8..
// the prefetch distance.
constexpr int kPassStaged = 1;
constexpr int kPassOnline = 2;
constexpr int kPassPrefetchShift = 8;

// Launch geometry for one problem.
void bcd_geometry(int n, int m, int elem_bytes, int sm_count, BcdProb& p);

// One problem of the cluster-resident solver (bcd_cluster.cu): a whole
// solve in one launch for cost matrices that fit one cluster's shared memory.
struct ClusterProb {
  const void* M;        // row-major n x m, float or double (fixed per launch)
  const double* a;
  const double* b;
  const double* x0;     // nullable [alpha; beta]
  double* dual;         // nullable output [alpha; beta] of iterate niter
  BcdState* st;         // output: niter, last_err, fast_iters, ...
  int n, m, max_iter;
  double eta, s2, tol;
};

// Cluster size (1..16) for an n x m problem when the cluster path is enabled
// and the problem fits, else 0.
template <typename TM>
int bcd_cluster_eligible(int n, int m);
int bcd_cluster_plan(int n, int m, int elem_bytes, int max_c);
bool bcd_cluster_enabled();
// Largest cluster size the current device runs this solver with (0: none).
int bcd_cluster_max(bool f32);
// Launch `nprob` problems (cluster size C each) on one stream.
template <typename TM>
int launch_bcd_cluster(const ClusterProb* d_probs, int nprob, int C, cudaStream_t st);


}  // namespace cg
