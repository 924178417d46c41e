// Host build of the device RRQR refinement (flam_b200/csrc/rrqr.cuh) so the
// tests can run it against the oracle on identical input.  Test harness only.
#include "../../flam_b200/csrc/rrqr.cuh"

extern "C" int flam_test_rrqr(double* R, int ld, int n, int k, int rows, int* jpvt, double tol, double Tmax,
                              long long rrqr_iter, double* aux, int* niter, int* capped) {
  return flam::rrqr_serial(R, 1, ld, n, k, rows, jpvt, tol, Tmax, (int64_t)rrqr_iter, aux, niter, capped);
}
