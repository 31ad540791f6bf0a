// Direction solve by leaf peeling + dense Schur complement on the 2-core.
//
// The SPLR sparsified Hessian A (H = n + m - 1) is a diagonal plus a
// bipartite graph between the alpha nodes (rows i < n) and the beta nodes
// (rows n + j).  At the default density the graph is close to a forest.
// Eliminating a node of degree <= 1 creates no fill (it only changes the
// pivot of its single neighbour), so the nodes outside the graph's 2-core
// are eliminated first, in rounds of independent leaves, as an LDL^T
// factorization with 1x1 pivots.  What remains (the 2-core, with updated
// diagonals) is factored like the dense Schur path: its larger side is
// eliminated exactly and the Schur complement of the smaller side is
// factored with cuSOLVER potrf in FP64.  The result is A^{-1} b to rounding,
// computed with a different elimination order than the reference's cuDSS
// call (src/linsolve.cu:159-268).
#pragma once

#include <cusolverDn.h>

#include <vector>

#include "sparsify.cuh"

namespace cg {

// Largest core Schur complement factored in shared memory inside one kernel.
constexpr int kPeelSmallCore = 160;
// Largest core whose triangular solves with the potrf factor run inside the
// single-CTA forward kernel (shared-memory right-hand sides) instead of potrs.
constexpr int kPeelTriMax = 2048;
// Largest core Schur complement assembled from host-planned contribution
// lists (one thread per entry); larger ones use the row-wise assembly.
constexpr int kPeelContribMax = 1024;

struct PeelFactor {
  int H = 0, n = 0, m = 0;
  int rounds = 0;       // peel rounds (the core is processed as one extra round)
  int npeel = 0;        // peeled nodes
  int kc = 0, ke = 0;   // core nodes on the Schur side / on the eliminated side
  long long nchild = 0, ns_adj = 0, ne_adj = 0;
  // host plan
  std::vector<int> h_ints;  // every int array below, packed in device order
  size_t off_order = 0, off_rptr = 0, off_hcnt = 0, off_diagq = 0, off_cpos = 0, off_child = 0,
         off_childq = 0, off_dqo = 0, off_ppar = 0, off_pparq = 0, off_snodes = 0, off_enodes = 0,
         off_sptr = 0, off_sadj = 0, off_sq = 0, off_eptr = 0, off_eadj = 0, off_eq = 0, off_ccp = 0,
         off_ce = 0, off_cq1 = 0, off_cq2 = 0;
  bool contrib = false;  // per-entry contribution lists of the core Schur complement
  // device
  void* block = nullptr;
  size_t block_bytes = 0;
  int* ints = nullptr;
  double* d = nullptr;      // [H] pivots (core nodes: updated diagonal)
  double* S = nullptr;      // [kc * kc] Schur complement / factor
  double* work = nullptr;   // potrf workspace
  int lwork = 0;
  int* info = nullptr;      // [3] potrf info, pivot check, potrs info
  double* y = nullptr;      // [2H] forward-substitution values
  double* rs = nullptr;     // [2 kc] reduced right-hand sides / Schur solution
  double* W = nullptr;      // [ne_adj] edge weights a_{e,t} / d_e of the core (E-list order)
  bool ready = false;
  bool stream_ordered = false;
  cudaStream_t alloc_stream = nullptr;
};

// Host plan of the current pattern of A (copies the pattern to the host and
// synchronizes the stream).  Sets rounds, kc, ke; ready stays false.
// no_peel = true: no elimination rounds, the core is the whole graph -- the
// contribution lists of the dense Schur complement (see peel_assemble_dense).
int peel_plan(PeelFactor& P, const SpHess& A, cudaStream_t st, bool no_peel = false);
// The host part of peel_plan, from the pattern already on the host (row
// pointers rp[H + 1] and column indices cl of A's lower CSR).  No CUDA calls:
// may run on any thread.
int peel_plan_host(PeelFactor& P, int n, int m, const std::vector<int>& rp,
                   const std::vector<int>& cl, bool no_peel = false);
// Device buffers + upload of the plan (plan_only: the integer plan alone).
int peel_upload(PeelFactor& P, cusolverDnHandle_t h, cudaStream_t st, bool plan_only = false);
// Dense Schur complement S (k x k, the dense direction-solve path) assembled
// from a no_peel plan, one thread per entry; same values and summation order
// as the row-wise assembly of schur.cu.
int peel_assemble_dense(const PeelFactor& P, const SpHess& A, double* S, int k, cudaStream_t st);
// Numeric factorization of A's current values (async; a non-positive pivot
// or a potrf failure lands in info[0] / info[1]).
int peel_factor(PeelFactor& P, const SpHess& A, cusolverDnHandle_t h, cudaStream_t st);
// Device-side status of the last factorization: copy of info[0..1] (async;
// non-zero = not positive definite).
int peel_info_async(const PeelFactor& P, int* host2, cudaStream_t st);
// Factorization followed by x = A^{-1} rhs (nrhs 0..2; 0 = factor only).  For
// small cores this is a single kernel launch.
int peel_factor_solve(PeelFactor& P, const SpHess& A, cusolverDnHandle_t h, const double* rhs,
                      double* x, int nrhs, cudaStream_t st);
// x = A^{-1} rhs for nrhs <= 2 column-major right-hand sides (leading dim H).
int peel_solve(PeelFactor& P, const SpHess& A, cusolverDnHandle_t h, const double* rhs,
               double* x, int nrhs, cudaStream_t st);
void peel_release(PeelFactor& P);

}  // namespace cg
