// Device tree (forest) arrays and the launch wrappers of tree.cu.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace flam {

// Device view of the forest under construction.  Box ids are global over all
// instances; boxes of one depth are contiguous.
struct TreeDev {
  int d;
  const double* x;       // d x Ntot points
  int64_t* perm;         // position -> point id; a box's subtree is perm[seg_start, +seg_len)
  int32_t* pbox;         // position -> current leaf box
  double* ctr;           // box centres (nbox x d)
  double* lsz;           // box sizes (nbox x d)
  int32_t* prnt;
  int32_t* chfirst;      // first child (-1: leaf)
  int32_t* nch;
  int64_t* seg_start;
  int64_t* seg_len;
  int32_t* depth;        // 1 = root
  int32_t* inst;
  int32_t* keychild;     // 8 per box: child id of each key, or -1
  int64_t* nbor_ptr;     // CSR (nbox + 1)
  int32_t* nbor;
};

void tree_extent(const double* x, int d, const int64_t* inst_off_dev, int ninst, int nchunk, double* part,
                 cudaStream_t s);
void tree_level_flags(const TreeDev& t, int64_t ntot, int32_t b0, int32_t b1, int64_t occ, int can_split,
                      const int32_t* ldiv, int32_t* flags, int nl, cudaStream_t s);
void tree_level_count(const TreeDev& t, int64_t ntot, int32_t b0, int32_t b1, int64_t occ, int can_split,
                      const int32_t* scan, int nl, int32_t* nch_tmp, cudaStream_t s);
void tree_level_children(const TreeDev& t, int64_t ntot, int32_t b0, int32_t b1, const int32_t* scan, int nl,
                         const int32_t* base, const int32_t* ldiv, const double* lnew, cudaStream_t s);
void tree_level_scatter(const TreeDev& t, int64_t ntot, int32_t b0, int32_t b1, int64_t occ, int can_split,
                        const int32_t* ldiv, const int32_t* scan, int nl, int64_t* perm2, int32_t* pbox2,
                        cudaStream_t s);
void tree_neighbours(const TreeDev& t, int32_t b0, int32_t b1, int pass, int64_t* cnt_or_ptr, cudaStream_t s);
void tree_perm_offsets(const TreeDev& t, int32_t b0, int32_t b1, int64_t* off, cudaStream_t s);
void tree_perm_fill(const TreeDev& t, int32_t nbox, const int64_t* off, int64_t* P, cudaStream_t s);

}  // namespace flam
