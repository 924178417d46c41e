// Per-factor terms of the log-determinant (rskelf/rskelf_logdet.m:11-33).
//
// For every factor of one level step a CTA reads the r diagonal entries of
// its LU (or Cholesky) block and, for LU, the row permutation p, and writes
//   out[2f]   = sum log|diag|          (x2 for the Cholesky factor L)
//   out[2f+1] = parity of (number of negative diagonal entries + inversions of p)
// The log of a negative real is log|d| + i*pi and log(detperm(p)) is 0 or
// i*pi, so the imaginary part of the total is pi times the parity of the sum
// of these counts; the host adds the per-factor terms in factor order.
#include "common.cuh"
#include "kernels.cuh"

namespace flam {

namespace {

constexpr int kLdThreads = 256;

__global__ void __launch_bounds__(kLdThreads) k_logdet(const FacDesc* __restrict__ fac, const double* __restrict__ fpool,
                                                       const int32_t* __restrict__ ppool, int chol,
                                                       double* __restrict__ out) {
  const FacDesc f = fac[blockIdx.x];
  const int r = f.r;
  const double* LU = fpool + f.LU_off;  // r x r, column-major
  double s = 0.0;
  long long cnt = 0;
  for (int i = threadIdx.x; i < r; i += kLdThreads) {
    const double d = LU[i + (int64_t)i * r];
    s += log(fabs(d));
    cnt += d < 0.0;
  }
  if (!chol) {
    // inversions of p: pairs i < j with p[i] > p[j]
    const int32_t* p = ppool + f.piv_off;
    for (int i = threadIdx.x; i < r; i += kLdThreads) {
      const int32_t pi = p[i];
      int c = 0;
      for (int j = i + 1; j < r; ++j) c += p[j] < pi;
      cnt += c;
    }
  }
  __shared__ double ss[kLdThreads / 32];
  __shared__ long long sc[kLdThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    ss[wid] = s;
    sc[wid] = cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    long long c = 0;
    for (int w = 0; w < kLdThreads / 32; ++w) {
      t += ss[w];
      c += sc[w];
    }
    out[2 * (int64_t)blockIdx.x] = chol ? 2.0 * t : t;
    out[2 * (int64_t)blockIdx.x + 1] = (double)(c & 1);
  }
}

}  // namespace

void launch_logdet(const FacDesc* fac, int nfac, const double* fpool, const int32_t* ppool, int chol, double* out,
                   cudaStream_t s) {
  if (nfac <= 0) return;
  k_logdet<<<nfac, kLdThreads, 0, s>>>(fac, fpool, ppool, chol, out);
}

}  // namespace flam
