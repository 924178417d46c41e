// CTA-level FP64 building blocks for the boxes whose work matrices live in
// global memory (L2-resident: a box's n x n block is at most a few MB).
//
// A strided view GV addresses element (i, j) at p[i * rs + j * cs]; a
// column-major matrix with leading dimension ld is {p, 1, ld} and its
// transpose {p, ld, 1}.  Every routine is called by all threads of the CTA
// (kTileThreads of them) and ends with __syncthreads().
#pragma once
#include <cstdint>

namespace flam {

constexpr int kTileThreads = 256;
constexpr int kTM = 64, kTN = 64, kTK = 16;   // C tile and k-chunk of cta_gemm
constexpr int kTLd = kTK + 4;                 // shared row stride (20 doubles: fragment loads in 2 wavefronts)
constexpr int kTileSmemDoubles = (kTM + kTN) * kTLd;

struct GV {
  const double* p;
  int64_t rs, cs;
  __device__ __forceinline__ double at(int64_t i, int64_t j) const { return p[i * rs + j * cs]; }
};

__device__ __forceinline__ void tile_dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// C(0:M, 0:N) += alpha * A(0:M, 0:K) * B(0:K, 0:N).  C is column-major-strided
// {c, crs, ccs}.  With lower != 0 only tiles that reach the lower triangle
// (i >= j) are computed (the Cholesky trailing update).  smem holds
// kTileSmemDoubles doubles.  The products run on the FP64 tensor path
// (mma.sync m8n8k4 .f64): the eight warps split a 64 x 64 tile into 32 x 16
// blocks (4 x 2 fragments each), over k-chunks of 16 staged in shared memory
// row by row (A by rows of C, B by columns of C, k contiguous), with the next
// chunk's global loads issued before the current chunk's products.
__device__ __forceinline__ void cta_gemm(double* C, int64_t crs, int64_t ccs, GV A, GV B, int M, int N, int K,
                                         double alpha, double* smem, int lower = 0) {
  if (M <= 0 || N <= 0 || K <= 0) return;
  double* As = smem;               // [kTM][kTLd]
  double* Bs = smem + kTM * kTLd;  // [kTN][kTLd]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3, wm = warp >> 2, wn = warp & 3;
  const bool a_col = A.rs == 1;   // consecutive rows are consecutive in memory
  const bool b_col = B.rs == 1;   // consecutive k are consecutive in memory
  const int tm = (M + kTM - 1) / kTM, tn = (N + kTN - 1) / kTN;
  for (int tile = 0; tile < tm * tn; ++tile) {
    const int i0 = (tile % tm) * kTM, j0 = (tile / tm) * kTN;
    if (lower && i0 + kTM <= j0) continue;
    double acc[4][2][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    double ra[4], rb[4];
    auto load = [&](int k0) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int e = tid + q * kTileThreads;
        const int ai = a_col ? (e & 63) : (e >> 4), al = a_col ? (e >> 6) : (e & 15);
        const int gi = i0 + ai, gl = k0 + al;
        ra[q] = (gi < M && gl < K) ? A.at(gi, gl) : 0.0;
        const int bl = b_col ? (e & 15) : (e >> 6), bj = b_col ? (e >> 4) : (e & 63);
        const int hl = k0 + bl, gj = j0 + bj;
        rb[q] = (hl < K && gj < N) ? B.at(hl, gj) : 0.0;
      }
    };
    auto stash = [&]() {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int e = tid + q * kTileThreads;
        const int ai = a_col ? (e & 63) : (e >> 4), al = a_col ? (e >> 6) : (e & 15);
        As[ai * kTLd + al] = ra[q];
        const int bl = b_col ? (e & 15) : (e >> 6), bj = b_col ? (e >> 4) : (e & 63);
        Bs[bj * kTLd + bl] = rb[q];
      }
    };
    load(0);
    for (int k0 = 0; k0 < K; k0 += kTK) {
      __syncthreads();
      stash();
      __syncthreads();
      if (k0 + kTK < K) load(k0 + kTK);
      const double* Aw = As + (wm * 32 + g) * kTLd + tq;
      const double* Bw = Bs + (wn * 16 + g) * kTLd + tq;
#pragma unroll
      for (int kk = 0; kk < kTK; kk += 4) {
        double af[4], bf[2];
#pragma unroll
        for (int a = 0; a < 4; ++a) af[a] = Aw[a * 8 * kTLd + kk];
#pragma unroll
        for (int b = 0; b < 2; ++b) bf[b] = Bw[b * 8 * kTLd + kk];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 2; ++b) tile_dmma(acc[a][b], af[a], bf[b]);
      }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int gi = i0 + wm * 32 + a * 8 + g;
      if (gi >= M) continue;
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int gj = j0 + wn * 16 + b * 8 + 2 * tq + e;
          if (gj < N) {
            double* c = C + gi * crs + gj * ccs;
            *c = fma(alpha, acc[a][b][e], *c);
          }
        }
    }
  }
  __syncthreads();
}

}  // namespace flam
