// C-ABI shim around the reference's own GPU BCD solver (test infrastructure
// only).  build_ref.sh compiles this file together with the reference's
// src/sinkhorn_bcd_kernel.cu and src/utils.cu, read in place, into
// oracle/_ref/libref_bcd.so.  Nothing here is reference source: it only
// declares and forwards to cuda_sinkhorn_bcd (reference src/solvers.h:4-9).
void cuda_sinkhorn_bcd(const double* M, const double* a, const double* b, double* P,
                       double reg, int max_iter, double tol, int n, int m, int* niter,
                       const double* x0, double* dual, bool input_on_device,
                       bool output_on_device);

extern "C" int ref_sinkhorn_bcd_host(const double* M, const double* a, const double* b,
                                     double* P, double reg, int max_iter, double tol, int n,
                                     int m, int* niter, const double* x0, double* dual) {
  cuda_sinkhorn_bcd(M, a, b, P, reg, max_iter, tol, n, m, niter, x0, dual, false, false);
  return 0;
}

// Device-resident inputs and outputs (input_on_device = output_on_device =
// true): what a timing of the reference's own GPU path on data already in
// HBM calls.
extern "C" int ref_sinkhorn_bcd_device(const double* M, const double* a, const double* b,
                                       double* P, double reg, int max_iter, double tol, int n,
                                       int m, int* niter, const double* x0, double* dual) {
  cuda_sinkhorn_bcd(M, a, b, P, reg, max_iter, tol, n, m, niter, x0, dual, true, true);
  return 0;
}
