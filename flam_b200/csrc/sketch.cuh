// Randomized row sketch of the compression blocks on the tensor cores (sketch.cu).
#pragma once
#include "common.cuh"

namespace flam {

// Boxes up to this many points are sketched (two 128-column tiles of tensor memory);
// larger boxes take the exact compression.
constexpr int kSketchMaxN = 8192;
// Sketch rows at most: a box's full width plus the oversampling, so that a second sketch
// can always hold the rank.
constexpr int kSketchMaxW = kSketchMaxN + 64;
// One CTA sketches at most this many columns of K and rows of Y (tensor memory: 512 FP32
// columns of 128 lanes, i.e. tiles x padded rows <= 512).
constexpr int kSketchCtaCols = 256;
constexpr int kSketchCtaRows = 512;
// The FP64 sketch: one CTA forms at most this many rows of Y by columns of K.
constexpr int kSketchF64Rows = 64;
constexpr int kSketchF64Cols = 128;

// Columns of K (cstep) and rows of Y (jstep) one CTA of the sketch of an n-column box
// with w sketch rows takes.
inline void sketch_cta_tile(bool fp64, int n, int w, int* cstep, int* jstep) {
  if (fp64) {
    *cstep = kSketchF64Cols;
    *jstep = kSketchF64Rows;
    return;
  }
  const bool one = n <= kSketchCtaCols && w <= kSketchCtaCols;   // the whole box in one CTA
  *cstep = one ? n : 128;
  *jstep = one ? w : kSketchCtaRows;
}

// One box of a factorization step in the sketched form.
struct SketchTask {
  int64_t slf_off;   // ids in ipool (pull-up order)
  int64_t cand_off;  // neighbour candidates in cpool, already filtered (count in mfilt[out_idx])
  int64_t y_off;     // Y = Omega K (w x n, column-major, leading dimension w) in the sketch pool
  int64_t perm_off;  // the compression's local permutation of this box (permpool)
  int32_t n, w;
  int32_t inst, out_idx;
  int32_t box, flags;  // flags bit0: proxy rows (level > 2)
  // the part of Y this CTA forms: columns [col0, col0 + ncol) of K, rows [j0, j0 + nw) of Y
  // (ncol <= 256; nw <= 512 when ncol <= 128, else nw <= 256)
  int32_t col0, ncol, j0, nw;
  double ctr[kMaxDim];
  double l[kMaxDim];
};

struct SketchArgs {
  Problem P;
  const SketchTask* tasks;
  const int64_t* ipool;
  const int64_t* cpool;
  const int32_t* mfilt;   // filtered candidate count per out_idx
  double* ypool;
  int32_t* mrows;         // per out_idx: rows of K the sketch compressed
  int symm_n;
  uint32_t seed;
  int32_t* status;        // OR of StatusBits (ST_TIMEOUT)
  int fp64;               // 1: FP64 entries and products (k_sketch_f64), 0: TF32 tensor cores
};

size_t sketch_smem_bytes(int ncol, int nw);
void launch_sketch(const SketchArgs& a, int ntask, size_t smem, cudaStream_t s);
// Boxes idx[0, nidx) of tasks: restore the slf order the compression permuted (perm_off).
void launch_unpermute(const int32_t* idx, int nidx, const SketchTask* tasks, int64_t* ipool, const int32_t* permpool,
                      int nmax, cudaStream_t s);

}  // namespace flam
