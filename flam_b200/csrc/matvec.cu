// FP64 on-the-fly multiply by the registry matrix: Y = A X or Y = B - A X.
//
// This is the error oracle and the residual step of iterative refinement: the
// reference's tests form A*x from the matrix function (rskelf/test/ie_circle.m:
// 47-48,118-120; ie_sphere.m:100-116 uses ifmm at a tighter tolerance), which is
// O(N^2) work that nothing in the factorization can stand in for.  A is never
// stored: each CTA owns a tile of TM target rows x TN right-hand sides of one
// instance, streams that instance's sources in chunks of KC, evaluates the
// TM x KC block of A into shared memory (diagonal: dval; elsewhere
// scale * w_j * K(x_i, x_j)), and multiplies it with the KC x TN block of X on
// the FP64 tensor path (mma.sync m8n8k4 .f64; 8 warps, each a 32 x 32 tile of
// 4 x 4 fragments).  X chunks arrive by cp.async into a second buffer while the
// current chunk is multiplied.  Every CTA of a wave walks the sources in the same
// order, so a chunk of X is read from HBM about once per wave and from L2 by the
// other CTAs.
//
// Work per call: 2 N_i^2 nrhs flops (the dense product) plus N_i^2 kernel
// evaluations per instance, for every column tile (one tile up to 256 RHS).
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "matvec.cuh"

namespace flam {
namespace {

constexpr int kKC = 16;          // sources per chunk
constexpr int kLd = kKC + 4;     // shared row stride (doubles): 20 = 4 mod 16, no bank conflicts
constexpr int kThreadsMv = 256;  // 8 warps

__device__ __forceinline__ void mma_f64(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// WM x WN warps, each 32 x 32 outputs: TM = 32 WM target rows, TN = 32 WN columns.
template <int WM, int WN>
__global__ void __launch_bounds__(kThreadsMv) k_matvec(MatvecArgs a) {
  constexpr int TM = 32 * WM, TN = 32 * WN;
  extern __shared__ double smem[];
  double* As = smem;                        // 2 x TM x kLd
  double* Xs = As + 2 * TM * kLd;           // 2 x TN x kLd
  double* xt = Xs + 2 * TN * kLd;           // TM x d target coordinates
  const MatvecTile tile = a.tiles[blockIdx.x];
  const InstParams ip = a.P.ip[tile.inst];
  const int d = a.P.d;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp / WN, wn = warp % WN;
  const int col0 = blockIdx.y * TN;
  const int64_t src_beg = ip.pt_off, src_end = ip.pt_off + ip.N;
  for (int e = tid; e < TM * d; e += kThreadsMv) {
    const int m = e / d, c = e % d;
    xt[e] = m < tile.nrows ? a.P.x[(tile.row0 + m) * d + c] : 0.0;
  }
  __syncthreads();

  // A block of the chunk starting at source j0 into As[buf]: thread (k = tid % KC) owns
  // one source and evaluates rows m = tid / KC + 16 i.
  auto fill_a = [&](int buf, int64_t j0) {
    const int k = tid % kKC;
    const int64_t j = j0 + k;
    double* A = As + buf * TM * kLd;
    const bool live = j < src_end;
    double ys[kMaxDim] = {0.0, 0.0, 0.0}, ns[kMaxDim] = {0.0, 0.0, 0.0};
    double wj = 1.0;
    if (live) {
      for (int c = 0; c < d; ++c) ys[c] = a.P.x[j * d + c];
      if (ip.has_nrm)
        for (int c = 0; c < d; ++c) ns[c] = a.P.nrm[j * d + c];
      if (ip.has_w) wj = a.P.w[j];
    }
    const double sw = ip.scale * wj;
    for (int m = tid / kKC; m < TM; m += kThreadsMv / kKC) {
      double v = 0.0;
      if (live && m < tile.nrows) {
        const int64_t i = tile.row0 + m;
        v = (i == j) ? ip.dval : sw * keval(ip.kind, ip.param, d, xt + m * d, ys, ns);
      }
      A[m * kLd + k] = v;
    }
  };
  // X block of the chunk: column c of X holds KC consecutive sources (coalesced).
  auto fill_x = [&](int buf, int64_t j0) {
    double* X = Xs + buf * TN * kLd;
    for (int e = tid; e < TN * kKC; e += kThreadsMv) {
      const int k = e % kKC, c = e / kKC;
      const int64_t j = j0 + k;
      const int col = col0 + c;
      if (j < src_end && col < a.nrhs)
        cp_async8(X + c * kLd + k, a.X + j + (int64_t)col * a.ldx);
      else
        X[c * kLd + k] = 0.0;
    }
    cp_async_commit();
  };

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) acc[i][jj][0] = acc[i][jj][1] = 0.0;

  const int64_t nchunk = (ip.N + kKC - 1) / kKC;
  fill_x(0, src_beg);
  fill_a(0, src_beg);
  cp_async_wait_all();
  __syncthreads();
  for (int64_t ch = 0; ch < nchunk; ++ch) {
    const int buf = (int)(ch & 1);
    if (ch + 1 < nchunk) {
      fill_x(buf ^ 1, src_beg + (ch + 1) * kKC);
      fill_a(buf ^ 1, src_beg + (ch + 1) * kKC);
    }
    const double* A = As + buf * TM * kLd + (wm * 32 + g) * kLd + t;
    const double* X = Xs + buf * TN * kLd + (wn * 32 + g) * kLd + t;
#pragma unroll
    for (int kk = 0; kk < kKC; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = A[i * 8 * kLd + kk];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) bf[jj] = X[jj * 8 * kLd + kk];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) mma_f64(acc[i][jj], af[i], bf[jj]);
    }
    cp_async_wait_all();
    __syncthreads();
  }
  // epilogue: fragment (i, jj) element e is row 8 i + g, column 8 jj + 2 t + e of the warp tile
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = wm * 32 + i * 8 + g;
    if (m >= tile.nrows) continue;
    const int64_t row = tile.row0 + m;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = col0 + wn * 32 + jj * 8 + 2 * t + e;
        if (col >= a.nrhs) continue;
        const double v = acc[i][jj][e];
        a.Y[row + (int64_t)col * a.ldy] = a.B ? a.B[row + (int64_t)col * a.ldb] - v : v;
      }
  }
}

template <int WM, int WN>
size_t mv_smem(int d) {
  return sizeof(double) * (size_t)(2 * 32 * WM * kLd + 2 * 32 * WN * kLd + 32 * WM * d);
}

template <int WM, int WN>
void launch_wn(const MatvecArgs& a, int ntile, int ncol, cudaStream_t s) {
  const size_t sm = mv_smem<WM, WN>(a.P.d);
  if (ensure_smem_attr(reinterpret_cast<const void*>(k_matvec<WM, WN>), (int)sm) != cudaSuccess) return;
  k_matvec<WM, WN><<<dim3((unsigned)ntile, (unsigned)ncol), kThreadsMv, sm, s>>>(a);
}

// Sum of squares of each column of an N x nrhs block (leading dimension ld): one CTA per column.
__global__ void k_colsq(const double* Y, int64_t N, int64_t ld, double* out) {
  __shared__ double red[32];
  const double* col = Y + (int64_t)blockIdx.x * ld;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < N; i += blockDim.x) s += col[i] * col[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) out[blockIdx.x] = v;
  }
}

// X(:, c) += R(:, c) for c < nrhs.
__global__ void k_add_cols(double* X, int64_t ldx, const double* R, int64_t ldr, int64_t N, int nrhs) {
  const int64_t total = N * nrhs;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = e / N, i = e % N;
    X[i + c * ldx] += R[i + c * ldr];
  }
}

// out[c] = sum_i X(i, c) Y(i, c): one CTA per column.
__global__ void k_coldot(const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t N, double* out) {
  __shared__ double red[32];
  const double* x = X + (int64_t)blockIdx.x * ldx;
  const double* y = Y + (int64_t)blockIdx.x * ldy;
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < N; i += blockDim.x) s += x[i] * y[i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.0;
    v = warp_sum(v);
    if (threadIdx.x == 0) out[blockIdx.x] = v;
  }
}

// Y(:, c) = a[c] Y(:, c) + b[c] X(:, c) (a == null: 1).
__global__ void k_axpby_cols(double* Y, int64_t ldy, const double* X, int64_t ldx, const double* a, const double* b,
                             int64_t N, int nrhs) {
  const int64_t total = N * nrhs;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = e / N, i = e % N;
    const double ya = a ? a[c] * Y[i + c * ldy] : Y[i + c * ldy];
    Y[i + c * ldy] = ya + b[c] * X[i + c * ldx];
  }
}

}  // namespace

void launch_coldot(const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t N, int nrhs, double* out,
                   cudaStream_t s) {
  if (nrhs <= 0) return;
  k_coldot<<<nrhs, 256, 0, s>>>(X, ldx, Y, ldy, N, out);
}

void launch_axpby_cols(double* Y, int64_t ldy, const double* X, int64_t ldx, const double* a, const double* b, int64_t N,
                       int nrhs, cudaStream_t s) {
  if (N <= 0 || nrhs <= 0) return;
  const int64_t blocks = std::min<int64_t>((N * nrhs + 255) / 256, 148 * 16);
  k_axpby_cols<<<(unsigned)blocks, 256, 0, s>>>(Y, ldy, X, ldx, a, b, N, nrhs);
}

void launch_add_cols(double* X, int64_t ldx, const double* R, int64_t ldr, int64_t N, int nrhs, cudaStream_t s) {
  if (N <= 0 || nrhs <= 0) return;
  const int64_t blocks = std::min<int64_t>((N * nrhs + 255) / 256, 148 * 16);
  k_add_cols<<<(unsigned)blocks, 256, 0, s>>>(X, ldx, R, ldr, N, nrhs);
}

int matvec_tile_rows(int nrhs) {
  const int wn = nrhs <= 32 ? 1 : nrhs <= 64 ? 2 : nrhs <= 128 ? 4 : 8;
  return 32 * (8 / wn);
}

int matvec_tile_cols(int nrhs) { return 256 / (matvec_tile_rows(nrhs) / 32); }

void launch_matvec(const MatvecArgs& a, int ntile, cudaStream_t s) {
  if (ntile <= 0 || a.nrhs <= 0) return;
  const int tn = matvec_tile_cols(a.nrhs);
  const int ncol = (a.nrhs + tn - 1) / tn;
  switch (tn) {
    case 32: launch_wn<8, 1>(a, ntile, ncol, s); break;
    case 64: launch_wn<4, 2>(a, ntile, ncol, s); break;
    case 128: launch_wn<2, 4>(a, ntile, ncol, s); break;
    default: launch_wn<1, 8>(a, ntile, ncol, s); break;
  }
}

void launch_colsq(const double* Y, int64_t N, int64_t ld, int nrhs, double* out, cudaStream_t s) {
  if (nrhs <= 0) return;
  k_colsq<<<nrhs, 256, 0, s>>>(Y, N, ld, out);
}

}  // namespace flam
