// Fused plan pass for the SPLR solver: T = exp((alpha + beta - M) / eta),
// row and column sums, dual objective, gradient, its norm and <g, d>.
#pragma once

#include "common.cuh"

namespace cg {

// Scalar results of one pass (device-resident; the host reads 32 bytes).
struct TResult {
  double f;       // reg * sum(T) - <gamma, (a, b)>
  double gnorm;   // ||g||_2, g = (r - a, c_{:m-1} - b_{:m-1})
  double dg;      // <g, direc> (trial mode)
  double tsum;    // sum(T)
  double gfull;   // full marginal error ||(r - a, c - b)||_2 (all m columns)
};

// Trial points evaluated by one multi-step pass (batched line search).
constexpr int kMaxTrialSteps = 2;

struct TPassArgs {
  const void* M;
  int n, m;
  double eta, s2;          // s2 = log2(e) / eta
  const double* ab;        // [n + m] = (a, b)
  // point: gamma directly, or gamma_prev + step * direc (trial mode)
  double* gamma;           // [n + m]; written in trial mode
  const double* gamma_prev;
  const double* direc;     // [n + m - 1]
  double step;
  int trial;
  // Multi-step trial mode (nsteps > 1): step k = steps[k] (steps[0] = step)
  // is evaluated as a separate trial point whose outputs and workspace sit at
  // slot k: gamma + k (n + m), rows + k n, cols + k m, grad + k (n + m - 1),
  // res + k, rowpart + k strips n, colpart + k splits m, scal + k (splits +
  // strips) kTScal.  Each slot gets exactly the values of a one-step pass.
  int nsteps;
  double steps[kMaxTrialSteps];
  // outputs
  double* rows;            // [n]
  double* cols;            // [m]
  double* grad;            // [n + m - 1]
  TResult* res;
  // workspace
  int strips, splits;      // tile grid: strips of 256 columns x row splits
  double* rowpart;         // [strips * n]
  double* colpart;         // [splits * m]
  double* scal;            // [(splits + strips) * kTScal]
  unsigned int* counters;  // [splits + strips + 1], zero-initialised
  int l2pf;                // L2 prefetch distance in row steps (set by launch_tpass)
};

constexpr int kTStrip = 256;  // columns per strip
constexpr int kTScal = 5;     // partial scalars per finisher CTA

void tpass_geometry(int n, int m, int sm_count, int& strips, int& splits);
size_t tpass_workspace_doubles(int n, int m, int strips, int splits);
int launch_tpass(bool f32, const TPassArgs& a, cudaStream_t stream);

}  // namespace cg
