// K8/K9: level-synchronous sweeps of rskelf_sv / rskelf_mv, plus the small
// data-movement kernels (id gathers, layout changes).
//
// A factorization step's factors touch disjoint rows (their sk and rd sets are
// slices of disjoint box point lists), so one launch applies a whole step: one
// CTA per (factor, tile of right-hand sides), one thread per right-hand side.
// The rows X(sk,:) and X(rd,:) of the tile are staged in shared memory
// (point-major X makes every row a contiguous, coalesced read), the factor
// matrices are read once per CTA from global memory as warp-broadcast loads.
//
// Reference sweeps (per factor, upward i = 1..n then downward i = n..1):
//   sv nn  up:  X(rd)-=T'X(sk); X(rd)=L\X(rd(p)); X(sk)-=E X(rd)      sv/rskelf_sv_nn.m:10-17
//          dn:  X(rd)-=G X(sk); X(rd)=U\X(rd);   X(sk)-=T X(rd)       sv/rskelf_sv_nn.m:21-28
//   sv nc  up:  X(rd)-=T'X(sk); X(rd)=U'\X(rd);  X(sk)-=G'X(rd)       sv/rskelf_sv_nc.m
//          dn:  X(rd)-=E'X(sk); X(rd(p))=L'\X(rd); X(sk)-=T X(rd)
//   sv p   up:  X(rd)-=T'X(sk); X(rd)=L\X(rd);   X(sk)-=E X(rd)       sv/rskelf_sv_p.m
//          dn:  X(rd)-=E'X(sk); X(rd)=L'\X(rd);  X(sk)-=T X(rd)
//   mv nn  up:  X(sk)+=T X(rd); X(rd)=U X(rd);   X(rd)+=G X(sk)       mv/rskelf_mv_nn.m
//          dn:  X(sk)+=E X(rd); X(rd(p))=L X(rd); X(rd)+=T'X(sk)
//   mv nc  up:  X(sk)+=T X(rd); X(rd)=L'X(rd(p)); X(rd)+=E'X(sk)      mv/rskelf_mv_nc.m
//          dn:  X(sk)+=G'X(rd); X(rd)=U'X(rd);   X(rd)+=T'X(sk)
//   mv p   up:  X(sk)+=T X(rd); X(rd)=L'X(rd);   X(rd)+=E'X(sk)       mv/rskelf_mv_p.m
//          dn:  X(sk)+=E X(rd); X(rd)=L X(rd);   X(rd)+=T'X(sk)
#include "common.cuh"
#include "kernels.cuh"

namespace flam {
namespace {

// ---- primitives on one right-hand side column held in shared memory with stride ts
// y(0:r) += sign * A' x(0:k), A k x r (ld k); y(i) pairs with column perm[i] of A
// when y is held in the permuted order X(rd(p)).
__device__ __forceinline__ void sub_At_x(double* y, const double* x, const double* A, int k, int r, int ts,
                                         double sign, const int32_t* perm = nullptr) {
  for (int i = 0; i < r; ++i) {
    const double* Ac = A + (int64_t)(perm ? perm[i] : i) * k;
    double s = 0.0;
    for (int b = 0; b < k; ++b) s += Ac[b] * x[b * ts];
    y[i * ts] += sign * s;
  }
}
// y(0:m) += sign * A x(0:q), A m x q (ld m); x(b) pairs with column perm[b] of A.
__device__ __forceinline__ void sub_A_x(double* y, const double* x, const double* A, int m, int q, int ts,
                                        double sign, const int32_t* perm = nullptr) {
  for (int i = 0; i < m; ++i) {
    double s = 0.0;
    for (int b = 0; b < q; ++b) s += A[i + (int64_t)(perm ? perm[b] : b) * m] * x[b * ts];
    y[i * ts] += sign * s;
  }
}
// triangular solves / products with the r x r factor M (ld r)
__device__ __forceinline__ void solve_lower(double* x, const double* M, int r, int ts, bool unit) {
  for (int i = 0; i < r; ++i) {
    double v = x[i * ts];
    for (int j = 0; j < i; ++j) v -= M[i + (int64_t)j * r] * x[j * ts];
    x[i * ts] = unit ? v : v / M[i + (int64_t)i * r];
  }
}
__device__ __forceinline__ void solve_upper(double* x, const double* M, int r, int ts) {
  for (int i = r - 1; i >= 0; --i) {
    double v = x[i * ts];
    for (int j = i + 1; j < r; ++j) v -= M[i + (int64_t)j * r] * x[j * ts];
    x[i * ts] = v / M[i + (int64_t)i * r];
  }
}
// x = U' \ x (U upper -> U' lower)
__device__ __forceinline__ void solve_upper_t(double* x, const double* M, int r, int ts) {
  for (int i = 0; i < r; ++i) {
    double v = x[i * ts];
    for (int j = 0; j < i; ++j) v -= M[j + (int64_t)i * r] * x[j * ts];
    x[i * ts] = v / M[i + (int64_t)i * r];
  }
}
// x = L' \ x (L lower -> L' upper)
__device__ __forceinline__ void solve_lower_t(double* x, const double* M, int r, int ts, bool unit) {
  for (int i = r - 1; i >= 0; --i) {
    double v = x[i * ts];
    for (int j = i + 1; j < r; ++j) v -= M[j + (int64_t)i * r] * x[j * ts];
    x[i * ts] = unit ? v : v / M[i + (int64_t)i * r];
  }
}
// x = U x
__device__ __forceinline__ void mul_upper(double* x, const double* M, int r, int ts) {
  for (int i = 0; i < r; ++i) {
    double s = 0.0;
    for (int j = i; j < r; ++j) s += M[i + (int64_t)j * r] * x[j * ts];
    x[i * ts] = s;
  }
}
// x = U' x
__device__ __forceinline__ void mul_upper_t(double* x, const double* M, int r, int ts) {
  for (int i = r - 1; i >= 0; --i) {
    double s = 0.0;
    for (int j = 0; j <= i; ++j) s += M[j + (int64_t)i * r] * x[j * ts];
    x[i * ts] = s;
  }
}
// x = L x
__device__ __forceinline__ void mul_lower(double* x, const double* M, int r, int ts, bool unit) {
  for (int i = r - 1; i >= 0; --i) {
    double s = unit ? x[i * ts] : M[i + (int64_t)i * r] * x[i * ts];
    for (int j = 0; j < i; ++j) s += M[i + (int64_t)j * r] * x[j * ts];
    x[i * ts] = s;
  }
}
// x = L' x
__device__ __forceinline__ void mul_lower_t(double* x, const double* M, int r, int ts, bool unit) {
  for (int i = 0; i < r; ++i) {
    double s = unit ? x[i * ts] : M[i + (int64_t)i * r] * x[i * ts];
    for (int j = i + 1; j < r; ++j) s += M[j + (int64_t)i * r] * x[j * ts];
    x[i * ts] = s;
  }
}

__global__ void k_sweep(SweepArgs a, double* gscr, int64_t slot) {
  extern __shared__ __align__(16) double smem[];
  const FacDesc f = a.fac[blockIdx.x];
  const int k = f.k, r = f.r;
  const int ts = blockDim.x;
  const int c = blockIdx.y * ts + threadIdx.x;
  const bool act = c < a.nrhs;
  double* xs = gscr ? gscr + ((int64_t)blockIdx.y * gridDim.x + blockIdx.x) * slot : smem;
  double* xr = xs + (int64_t)k * ts;
  double* ys = xs + threadIdx.x;  // this thread's column
  double* yr = xr + threadIdx.x;
  const int64_t* sk = a.ipool + f.sk_off;
  const int64_t* rd = sk + k;
  const double* T = a.fpool + f.T_off;
  const double* LU = a.fpool + f.LU_off;
  const double* E = a.fpool + f.E_off;
  const double* G = a.fpool + f.G_off;
  const int32_t* p = a.ppool + f.piv_off;
  const bool lu = a.symm != 'p';
  // gather with p for the steps that read X(rd(p))
  const bool gather_p = lu && ((a.op == 0 && a.trans == 0) || (a.op == 2 && a.trans == 1));
  const bool scatter_p = lu && ((a.op == 1 && a.trans == 1) || (a.op == 3 && a.trans == 0));
  if (act) {
    for (int b = 0; b < k; ++b) ys[b * ts] = a.X[sk[b] * a.ldx + c];
    for (int i = 0; i < r; ++i) yr[i * ts] = a.X[rd[gather_p ? p[i] : i] * a.ldx + c];
    const int tr = a.trans;
    switch (a.op) {
      case 0:  // sv upward
        sub_At_x(yr, ys, T, k, r, ts, -1.0, gather_p ? p : nullptr);
        if (!lu) {
          solve_lower(yr, LU, r, ts, false);
          sub_A_x(ys, yr, E, k, r, ts, -1.0);
        } else if (!tr) {
          solve_lower(yr, LU, r, ts, true);
          sub_A_x(ys, yr, E, k, r, ts, -1.0);
        } else {
          solve_upper_t(yr, LU, r, ts);
          sub_At_x(ys, yr, G, r, k, ts, -1.0);
        }
        break;
      case 1:  // sv downward
        if (!lu) {
          sub_At_x(yr, ys, E, k, r, ts, -1.0);
          solve_lower_t(yr, LU, r, ts, false);
        } else if (!tr) {
          sub_A_x(yr, ys, G, r, k, ts, -1.0);
          solve_upper(yr, LU, r, ts);
        } else {
          sub_At_x(yr, ys, E, k, r, ts, -1.0);
          solve_lower_t(yr, LU, r, ts, true);
        }
        sub_A_x(ys, yr, T, k, r, ts, -1.0, scatter_p ? p : nullptr);
        break;
      case 2:  // mv upward
        sub_A_x(ys, yr, T, k, r, ts, 1.0, gather_p ? p : nullptr);
        if (!lu) {
          mul_lower_t(yr, LU, r, ts, false);
          sub_At_x(yr, ys, E, k, r, ts, 1.0);
        } else if (!tr) {
          mul_upper(yr, LU, r, ts);
          sub_A_x(yr, ys, G, r, k, ts, 1.0);
        } else {
          mul_lower_t(yr, LU, r, ts, true);
          sub_At_x(yr, ys, E, k, r, ts, 1.0);
        }
        break;
      default:  // mv downward
        if (!lu) {
          sub_A_x(ys, yr, E, k, r, ts, 1.0);
          mul_lower(yr, LU, r, ts, false);
        } else if (!tr) {
          sub_A_x(ys, yr, E, k, r, ts, 1.0);
          mul_lower(yr, LU, r, ts, true);
        } else {
          sub_At_x(ys, yr, G, r, k, ts, 1.0);
          mul_upper_t(yr, LU, r, ts);
        }
        sub_At_x(yr, ys, T, k, r, ts, 1.0, scatter_p ? p : nullptr);
        break;
    }
    for (int b = 0; b < k; ++b) a.X[sk[b] * a.ldx + c] = ys[b * ts];
    for (int i = 0; i < r; ++i) a.X[rd[scatter_p ? p[i] : i] * a.ldx + c] = yr[i * ts];
  }
}

__global__ void k_gather_ids(const int64_t* src, int64_t* dst, const CopySeg* segs, int nseg) {
  const int s = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (s >= nseg) return;
  const CopySeg g = segs[s];
  for (int64_t i = threadIdx.x & 31; i < g.len; i += 32) dst[g.dst_off + i] = src[g.src_off + i];
}

__global__ void k_to_pm(const double* X, int64_t ld, int64_t N, int nrhs, double* W) {
  __shared__ double tile[32][33];
  const int64_t i0 = (int64_t)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  for (int q = threadIdx.y; q < 32; q += blockDim.y) {
    const int64_t i = i0 + threadIdx.x;
    const int c = c0 + q;
    tile[q][threadIdx.x] = (i < N && c < nrhs) ? X[i + (int64_t)c * ld] : 0.0;
  }
  __syncthreads();
  for (int q = threadIdx.y; q < 32; q += blockDim.y) {
    const int64_t i = i0 + q;
    const int c = c0 + threadIdx.x;
    if (i < N && c < nrhs) W[i * nrhs + c] = tile[threadIdx.x][q];
  }
}

__global__ void k_from_pm(const double* W, int64_t N, int nrhs, double* X, int64_t ld) {
  __shared__ double tile[32][33];
  const int64_t i0 = (int64_t)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  for (int q = threadIdx.y; q < 32; q += blockDim.y) {
    const int64_t i = i0 + q;
    const int c = c0 + threadIdx.x;
    tile[q][threadIdx.x] = (i < N && c < nrhs) ? W[i * nrhs + c] : 0.0;
  }
  __syncthreads();
  for (int q = threadIdx.y; q < 32; q += blockDim.y) {
    const int64_t i = i0 + threadIdx.x;
    const int c = c0 + q;
    if (i < N && c < nrhs) X[i + (int64_t)c * ld] = tile[threadIdx.x][q];
  }
}

}  // namespace

void launch_sweep(const SweepArgs& a, int nfac, int kmax, int rmax, cudaStream_t s) {
  if (nfac <= 0 || a.nrhs <= 0) return;
  int ts = a.nrhs >= 128 ? 128 : ((a.nrhs + 31) / 32) * 32;
  size_t need = sizeof(double) * (size_t)(kmax + rmax) * ts;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  dim3 g(nfac, (a.nrhs + ts - 1) / ts);
  if (need <= 160 * 1024) {
    k_sweep<<<g, ts, need, s>>>(a, nullptr, 0);
  } else {
    // rows of huge factors do not fit in shared memory: stage them in global scratch
    const int64_t slot = (int64_t)(kmax + rmax) * ts;
    double* scr = nullptr;
    cudaMallocAsync(&scr, sizeof(double) * slot * g.x * g.y, s);
    k_sweep<<<g, ts, 0, s>>>(a, scr, slot);
    cudaFreeAsync(scr, s);
  }
}

void launch_gather_ids(const int64_t* src, int64_t* dst, const CopySeg* segs, int nseg, cudaStream_t s) {
  if (nseg <= 0) return;
  k_gather_ids<<<(nseg + 7) / 8, 256, 0, s>>>(src, dst, segs, nseg);
}

void launch_to_pointmajor(const double* X, int64_t ld, int64_t N, int nrhs, double* W, cudaStream_t s) {
  if (N <= 0 || nrhs <= 0) return;
  dim3 g((unsigned)((N + 31) / 32), (nrhs + 31) / 32);
  k_to_pm<<<g, dim3(32, 8), 0, s>>>(X, ld, N, nrhs, W);
}

void launch_from_pointmajor(const double* W, int64_t N, int nrhs, double* X, int64_t ld, cudaStream_t s) {
  if (N <= 0 || nrhs <= 0) return;
  dim3 g((unsigned)((N + 31) / 32), (nrhs + 31) / 32);
  k_from_pm<<<g, dim3(32, 8), 0, s>>>(W, N, nrhs, X, ld);
}

}  // namespace flam
