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

// ---- CTA-cooperative primitives on a tile of kTs right-hand sides held in shared
// memory, row-major (X[row * kTs + col]); lane = column, warp w takes rows w, w+8, ...
// A matrix M is read through strides: M(i, j) = M[i * rs + j * cs], so the same
// routine applies a factor or its transpose.
constexpr int kTs = 32;
constexpr int kSw = 8;                 // warps per CTA
constexpr int kSweepThreads = 32 * kSw;

struct Mat {
  const double* p;
  int64_t rs, cs;
  const int32_t* rmap;  // optional row index map
  const int32_t* cmap;  // optional column index map
  __device__ __forceinline__ double at(int i, int j) const {
    const int ii = rmap ? rmap[i] : i, jj = cmap ? cmap[j] : j;
    return p[ii * rs + jj * cs];
  }
};

// The factor blocks are read through 32 x 32 tiles staged in shared memory (At,
// 32 x 33 doubles): every CTA thread loads a few entries with consecutive threads on
// consecutive addresses, and the products then read the tile as warp broadcasts.
constexpr int kAt = 33;   // row stride of the staged tile

// At[ii][bb] = A(i0 + ii, b0 + bb) for ii < mi, bb < qb, masked to a triangle in
// the (i, j) sense of A: tri 0 full, 1 lower (j <= i), 2 upper (j >= i); with unit the
// diagonal reads 1.
__device__ __forceinline__ void stage_tile(double* At, const Mat& A, int i0, int b0, int mi, int qb, int tri,
                                           bool unit) {
  const bool colmajor = A.rs == 1 && !A.rmap;
  for (int e = threadIdx.x; e < 32 * 32; e += kSweepThreads) {
    const int ii = colmajor ? (e & 31) : (e >> 5), bb = colmajor ? (e >> 5) : (e & 31);
    double v = 0.0;
    if (ii < mi && bb < qb) {
      const int i = i0 + ii, j = b0 + bb;
      const bool in = tri == 0 || (tri == 1 ? j <= i : j >= i);
      if (in) v = (unit && i == j) ? 1.0 : A.at(i, j);
    }
    At[ii * kAt + bb] = v;
  }
}

// Y(0:m, :) += sign * A(0:m, 0:q) X(0:q, :), A masked to a triangle by tri/unit as in
// stage_tile.  Warp w owns rows w, w+8, w+16, w+24 of each 32-row block.  Y and X must
// not overlap.  Called by every thread of the CTA.
__device__ void gemm_acc(double* Y, const double* X, Mat A, int m, int q, double sign, double* At, int tri = 0,
                         bool unit = false) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int i0 = 0; i0 < m; i0 += 32) {
    const int mi = min(32, m - i0);
    int bs = 0, be = q;
    if (tri == 1) be = min(q, i0 + 32);
    if (tri == 2) bs = i0;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (int b0 = bs; b0 < be; b0 += 32) {
      const int qb = min(32, q - b0);
      __syncthreads();
      stage_tile(At, A, i0, b0, mi, qb, tri, unit);
      __syncthreads();
      const double* a0 = At + w * kAt;
#pragma unroll 8
      for (int bb = 0; bb < qb; ++bb) {
        const double xb = X[(b0 + bb) * kTs + lane];
        s0 += a0[bb] * xb;
        s1 += a0[8 * kAt + bb] * xb;
        s2 += a0[16 * kAt + bb] * xb;
        s3 += a0[24 * kAt + bb] * xb;
      }
    }
    if (w < mi) Y[(i0 + w) * kTs + lane] += sign * s0;
    if (w + 8 < mi) Y[(i0 + w + 8) * kTs + lane] += sign * s1;
    if (w + 16 < mi) Y[(i0 + w + 16) * kTs + lane] += sign * s2;
    if (w + 24 < mi) Y[(i0 + w + 24) * kTs + lane] += sign * s3;
  }
}

__device__ __forceinline__ Mat shift(const Mat& M, int i0, int j0) {
  return Mat{M.p + i0 * M.rs + j0 * M.cs, M.rs, M.cs, nullptr, nullptr};
}

// X = M^-1 X for M (r x r) lower triangular in the (i, j) sense of M.at: 32-row blocks;
// a block first takes the contribution of the rows already solved (gemm_acc), then
// warp 0 solves the 32 x 32 diagonal block staged in shared memory.
__device__ void trsm_fwd(double* X, Mat M, int r, bool unit, double* At) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int i0 = 0; i0 < r; i0 += 32) {
    const int ib = min(32, r - i0);
    if (i0 > 0) gemm_acc(X + i0 * kTs, X, shift(M, i0, 0), ib, i0, -1.0, At);
    __syncthreads();
    stage_tile(At, M, i0, i0, ib, ib, 1, false);
    __syncthreads();
    if (w == 0)
      for (int ii = 0; ii < ib; ++ii) {
        double v = X[(i0 + ii) * kTs + lane];
        for (int jj = 0; jj < ii; ++jj) v -= At[ii * kAt + jj] * X[(i0 + jj) * kTs + lane];
        X[(i0 + ii) * kTs + lane] = unit ? v : v / At[ii * kAt + ii];
      }
    __syncthreads();
  }
}

// X = M^-1 X for M upper triangular (backward substitution), 32-row blocks from the end.
__device__ void trsm_bwd(double* X, Mat M, int r, bool unit, double* At) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int i1 = r; i1 > 0; i1 -= 32) {
    const int i0 = max(i1 - 32, 0), ib = i1 - i0;
    if (i1 < r) gemm_acc(X + i0 * kTs, X + i1 * kTs, shift(M, i0, i1), ib, r - i1, -1.0, At);
    __syncthreads();
    stage_tile(At, M, i0, i0, ib, ib, 2, false);
    __syncthreads();
    if (w == 0)
      for (int ii = ib - 1; ii >= 0; --ii) {
        double v = X[(i0 + ii) * kTs + lane];
        for (int jj = ii + 1; jj < ib; ++jj) v -= At[ii * kAt + jj] * X[(i0 + jj) * kTs + lane];
        X[(i0 + ii) * kTs + lane] = unit ? v : v / At[ii * kAt + ii];
      }
    __syncthreads();
  }
}

// X = M X for M triangular (lower: j <= i, upper: j >= i) through the scratch tile Y.
__device__ void trmm(double* X, double* Y, Mat M, int r, bool lower, bool unit, double* At) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int i = w; i < r; i += kSw) Y[i * kTs + lane] = 0.0;
  gemm_acc(Y, X, M, r, r, 1.0, At, lower ? 1 : 2, unit);
  __syncthreads();
  for (int i = w; i < r; i += kSw) X[i * kTs + lane] = Y[i * kTs + lane];
  __syncthreads();
}

__global__ void __launch_bounds__(kSweepThreads) k_sweep(SweepArgs a, double* gscr, int64_t slot) {
  extern __shared__ __align__(16) double smem[];
  __shared__ double At[32 * kAt];
  // consecutive CTAs take the right-hand-side tiles of one factor, so the factor's
  // blocks are read from DRAM once and then from L2
  const int ntile = (a.nrhs + kTs - 1) / kTs;
  const FacDesc f = a.fac[blockIdx.x / ntile];
  const int k = f.k, r = f.r;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c0 = (blockIdx.x % ntile) * kTs;
  const int c = c0 + lane;
  const bool act = c < a.nrhs;
  double* xs = gscr ? gscr + (int64_t)blockIdx.x * slot : smem;
  double* xr = xs + (int64_t)k * kTs;
  double* yt = xr + (int64_t)r * kTs;   // scratch tile for the triangular products
  const int64_t* sk = a.ipool + f.sk_off;
  const int64_t* rd = sk + k;
  const double* T = a.fpool + f.T_off;
  const double* LU = a.fpool + f.LU_off;
  const double* E = a.fpool + f.E_off;
  const double* G = a.fpool + f.G_off;
  const int32_t* p = a.ppool + f.piv_off;
  const bool lu = a.symm != 'p';
  const bool gather_p = lu && ((a.op == 0 && a.trans == 0) || (a.op == 2 && a.trans == 1));
  const bool scatter_p = lu && ((a.op == 1 && a.trans == 1) || (a.op == 3 && a.trans == 0));
  for (int b = w; b < k; b += kSw) xs[b * kTs + lane] = act ? a.X[sk[b] * a.ldx + c] : 0.0;
  for (int i = w; i < r; i += kSw) xr[i * kTs + lane] = act ? a.X[rd[gather_p ? p[i] : i] * a.ldx + c] : 0.0;
  __syncthreads();
  // factor views (column-major storage): A(i, j) = A[i + j * ld]; transposes swap strides
  const Mat Tn{T, 1, k, nullptr, nullptr}, Tt{T, k, 1, nullptr, nullptr};
  const Mat Ln{LU, 1, r, nullptr, nullptr}, Lt{LU, r, 1, nullptr, nullptr};
  const Mat En{E, 1, k, nullptr, nullptr}, Et{E, k, 1, nullptr, nullptr};
  const Mat Gn{G, 1, r, nullptr, nullptr}, Gt{G, r, 1, nullptr, nullptr};
  // T' X(sk) and T X(rd) with X(rd) held in the permuted order X(rd(p))
  const Mat Ttp{T, k, 1, gather_p || scatter_p ? p : nullptr, nullptr};
  const Mat Tnp{T, 1, k, nullptr, gather_p || scatter_p ? p : nullptr};
  const int tr = a.trans;
  switch (a.op) {
    case 0:  // sv upward
      gemm_acc(xr, xs, gather_p ? Ttp : Tt, r, k, -1.0, At);
      __syncthreads();
      if (!lu) {
        trsm_fwd(xr, Ln, r, false, At);
        gemm_acc(xs, xr, En, k, r, -1.0, At);
      } else if (!tr) {
        trsm_fwd(xr, Ln, r, true, At);
        gemm_acc(xs, xr, En, k, r, -1.0, At);
      } else {
        trsm_fwd(xr, Lt, r, false, At);      // U' \ x
        gemm_acc(xs, xr, Gt, k, r, -1.0, At);
      }
      break;
    case 1:  // sv downward
      if (!lu) {
        gemm_acc(xr, xs, Et, r, k, -1.0, At);
        __syncthreads();
        trsm_bwd(xr, Lt, r, false, At);      // L' \ x
      } else if (!tr) {
        gemm_acc(xr, xs, Gn, r, k, -1.0, At);
        __syncthreads();
        trsm_bwd(xr, Ln, r, false, At);      // U \ x
      } else {
        gemm_acc(xr, xs, Et, r, k, -1.0, At);
        __syncthreads();
        trsm_bwd(xr, Lt, r, true, At);       // L' \ x, unit
      }
      gemm_acc(xs, xr, scatter_p ? Tnp : Tn, k, r, -1.0, At);
      break;
    case 2:  // mv upward
      gemm_acc(xs, xr, gather_p ? Tnp : Tn, k, r, 1.0, At);
      __syncthreads();
      if (!lu) {
        trmm(xr, yt, Lt, r, false, false, At);   // L' x
        gemm_acc(xr, xs, Et, r, k, 1.0, At);
      } else if (!tr) {
        trmm(xr, yt, Ln, r, false, false, At);   // U x
        gemm_acc(xr, xs, Gn, r, k, 1.0, At);
      } else {
        trmm(xr, yt, Lt, r, false, true, At);    // L' x, unit
        gemm_acc(xr, xs, Et, r, k, 1.0, At);
      }
      break;
    default:  // mv downward
      if (!lu) {
        gemm_acc(xs, xr, En, k, r, 1.0, At);
        __syncthreads();
        trmm(xr, yt, Ln, r, true, false, At);    // L x
      } else if (!tr) {
        gemm_acc(xs, xr, En, k, r, 1.0, At);
        __syncthreads();
        trmm(xr, yt, Ln, r, true, true, At);     // L x, unit
      } else {
        gemm_acc(xs, xr, Gt, k, r, 1.0, At);
        __syncthreads();
        trmm(xr, yt, Lt, r, true, false, At);    // U' x
      }
      gemm_acc(xr, xs, scatter_p ? Ttp : Tt, r, k, 1.0, At);
      break;
  }
  __syncthreads();
  if (act) {
    for (int b = w; b < k; b += kSw) a.X[sk[b] * a.ldx + c] = xs[b * kTs + lane];
    for (int i = w; i < r; i += kSw) a.X[rd[scatter_p ? p[i] : i] * a.ldx + c] = xr[i * kTs + lane];
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

// Rows idx of the point-major work array <-> a column-major n x nrhs block Y
// (X(Si,:) of a partial factorization).  dir 0: gather into Y; 1: scatter back.
__global__ void k_rows_pm(double* W, int nrhs, const int64_t* idx, int64_t n, double* Y, int dir) {
  __shared__ double tile[32][33];
  const int64_t i0 = (int64_t)blockIdx.x * 32;
  const int c0 = blockIdx.y * 32;
  if (dir == 0) {
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
      const int64_t i = i0 + q;
      const int c = c0 + threadIdx.x;
      tile[q][threadIdx.x] = (i < n && c < nrhs) ? W[idx[i] * nrhs + c] : 0.0;
    }
    __syncthreads();
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
      const int64_t i = i0 + threadIdx.x;
      const int c = c0 + q;
      if (i < n && c < nrhs) Y[i + (int64_t)c * n] = tile[threadIdx.x][q];
    }
  } else {
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
      const int64_t i = i0 + threadIdx.x;
      const int c = c0 + q;
      tile[q][threadIdx.x] = (i < n && c < nrhs) ? Y[i + (int64_t)c * n] : 0.0;
    }
    __syncthreads();
    for (int q = threadIdx.y; q < 32; q += blockDim.y) {
      const int64_t i = i0 + q;
      const int c = c0 + threadIdx.x;
      if (i < n && c < nrhs) W[idx[i] * nrhs + c] = tile[threadIdx.x][q];
    }
  }
}

}  // namespace

void launch_rows_pm(double* W, int nrhs, const int64_t* idx, int64_t n, double* Y, int dir, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return;
  dim3 g((unsigned)((n + 31) / 32), (nrhs + 31) / 32);
  k_rows_pm<<<g, dim3(32, 8), 0, s>>>(W, nrhs, idx, n, Y, dir);
}

bool sweep_in_smem(int kmax, int rmax, int op) {
  return sizeof(double) * (size_t)((int64_t)(kmax + (op >= 2 ? 2 : 1) * rmax) * kTs) <= 200 * 1024;
}

void launch_sweep(const SweepArgs& a, int nfac, int kmax, int rmax, cudaStream_t s) {
  if (nfac <= 0 || a.nrhs <= 0) return;
  // X(sk), X(rd) and, for the multiplies, a scratch tile for the triangular
  // products (the solves work in place), kTs columns each
  const int64_t slot = (int64_t)(kmax + (a.op >= 2 ? 2 : 1) * rmax) * kTs;
  const size_t need = sizeof(double) * (size_t)slot;
  if (ensure_smem_attr(reinterpret_cast<const void*>(k_sweep), 200 * 1024) != cudaSuccess) return;
  const int64_t nblk = (int64_t)nfac * ((a.nrhs + kTs - 1) / kTs);
  const unsigned g = (unsigned)nblk;
  if (need <= 200 * 1024) {
    k_sweep<<<g, kSweepThreads, need, s>>>(a, nullptr, 0);
  } else {
    // rows of huge factors do not fit in shared memory: stage them in global scratch
    double* scr = nullptr;
    cudaMallocAsync(&scr, sizeof(double) * slot * nblk, s);
    k_sweep<<<g, kSweepThreads, 0, s>>>(a, scr, slot);
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
