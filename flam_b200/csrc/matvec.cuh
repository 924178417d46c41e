// FP64 on-the-fly products with the registry matrix (matvec.cu).
#pragma once
#include "common.cuh"

namespace flam {

// TM target rows [row0, row0 + nrows) of instance inst (global point ids).
struct MatvecTile {
  int64_t row0;
  int32_t nrows;
  int32_t inst;
};

struct MatvecArgs {
  Problem P;
  const MatvecTile* tiles;
  const double* X;   // Ntot x nrhs, column-major, leading dimension ldx (global point order)
  int64_t ldx;
  const double* B;   // null: Y = A X; else Y = B - A X
  int64_t ldb;
  double* Y;
  int64_t ldy;
  int nrhs;
};

// Rows per tile (the host cuts every instance into tiles of this many rows).
int matvec_tile_rows(int nrhs);
int matvec_tile_cols(int nrhs);
void launch_matvec(const MatvecArgs& a, int ntile, cudaStream_t s);
// out[c] = sum_i Y(i, c)^2 for c < nrhs.
void launch_add_cols(double* X, int64_t ldx, const double* R, int64_t ldr, int64_t N, int nrhs, cudaStream_t s);
// out[c] = X(:, c) . Y(:, c) for c < nrhs.
void launch_coldot(const double* X, int64_t ldx, const double* Y, int64_t ldy, int64_t N, int nrhs, double* out,
                   cudaStream_t s);
// Y(:, c) = a[c] Y(:, c) + b[c] X(:, c), with a = null meaning 1 (a, b: device arrays).
void launch_axpby_cols(double* Y, int64_t ldy, const double* X, int64_t ldx, const double* a, const double* b, int64_t N,
                       int nrhs, cudaStream_t s);
void launch_colsq(const double* Y, int64_t N, int64_t ld, int nrhs, double* out, cudaStream_t s);

}  // namespace flam
