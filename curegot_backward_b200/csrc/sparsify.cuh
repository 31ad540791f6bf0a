// Sparsified Hessian of the SPLR solver in CSR form.
#pragma once

#include "common.cuh"

namespace cg {

// Lower view of Hsl + shift*I (reference layout, sinkhorn_splr_kernel.cu:38-100):
// rows i < n hold only (i, i); row n+j holds the selected entries (n+j, i) of
// column j of T_t with i ascending, then its diagonal.  The same off-diagonal
// entries are also kept as per-row lists of T_sp (row i -> (j, value), j
// ascending) for the Schur-complement assembly.
struct SpHess {
  int n = 0, m = 0, H = 0;
  long long kcap = 0;   // capacity for off-diagonal entries
  long long K = 0;      // off-diagonal entries in the current pattern (host copy)
  double* val = nullptr;  // [kcap + H]
  int* col = nullptr;     // [kcap + H]
  int* rowptr = nullptr;  // [H + 1]
  int* ipt = nullptr;     // [n + 1] per-row list starts
  int* ij = nullptr;      // [kcap] column j
  double* iv = nullptr;   // [kcap] value T_ij
};

// Radix-select state (device).
struct SelState {
  unsigned long long prefix;  // digits fixed so far
  long long krem;             // entries still to select inside the prefix bucket
  int level;                  // digit level reached
  int done;
  unsigned long long tv;      // final predicate: key > tv || (key == tv && idx' >= ti)
  unsigned int ti;
  int pad;                    // 1: the selection exceeded the CSR capacity (nothing emitted)
};

struct SparsifyWork {
  unsigned int* hist = nullptr;  // [4096]
  SelState* sel = nullptr;
  int* colcnt = nullptr;         // [rowtiles * (m-1)]
  int* rowcnt = nullptr;         // [coltiles * n]
  int* coltot = nullptr;         // [m]
  int* rowtot = nullptr;         // [n]
  long long* kout = nullptr;     // [1] selected count
  int* scr_c = nullptr;          // [m] scan scratch
  int* scr_r = nullptr;          // [n] scan scratch
};

size_t sparsify_work_bytes(int n, int m);
void sparsify_work_carve(void* base, int n, int m, SparsifyWork& w);

// Full pattern update: exact top-Ks of T_t at gamma (ties: smaller flat Hsl
// index first), then CSR + per-row lists with values at gamma and the
// diagonal rows/cols + shift.  Asynchronous; K written to w.kout.
int sparsify_select_and_build(bool f32, const void* M, const double* gamma, const double* rows,
                              const double* cols, int n, int m, double s2, double shift,
                              long long Ks, SpHess& h, const SparsifyWork& w,
                              cudaStream_t stream);

// Fixed-pattern value refresh (reference recompute_nonzero_values_kernel).
int sparsify_refresh(bool f32, const void* M, const double* gamma, const double* rows,
                     const double* cols, int n, int m, double s2, double shift, const SpHess& h,
                     cudaStream_t stream);

}  // namespace cg
