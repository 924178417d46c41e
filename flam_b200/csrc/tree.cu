// Adaptive hyperoctree on the device (K1: subdivision, K2: neighbours), for a
// forest of independent instances.  Restates core/hypoct.m:51-171 and
// core/hypoct_perm.m:11-39; results are bit-exact with the reference:
// every floating-point step is the reference's (same operands, same order,
// no contraction into FMA), comparisons are exact, and the stable partition
// keeps each parent's point order inside every child (xi(idx == i), hypoct.m:109).
//
// Boxes of one depth are contiguous ids (like the reference's lvp), children
// of a box are consecutive ids in ascending key order (hypoct.m:94,106-115),
// and the points of a box's subtree are one contiguous segment of `perm`.
#include "common.cuh"
#include "tree.cuh"

namespace flam {
namespace {

// Root extent partials: one block per (instance, chunk).
__global__ void k_extent(const double* x, int d, const int64_t* inst_off, int nchunk, double* part) {
  const int inst = blockIdx.x, ch = blockIdx.y;
  const int64_t a = inst_off[inst], b = inst_off[inst + 1];
  const int64_t len = b - a;
  const int64_t per = (len + nchunk - 1) / nchunk;
  const int64_t s = a + per * ch, e = min(b, s + per);
  __shared__ double red[2 * kMaxDim][32];
  for (int k = 0; k < d; ++k) {
    double mn = INFINITY, mx = -INFINITY;
    for (int64_t i = s + threadIdx.x; i < e; i += blockDim.x) {
      double v = x[i * d + k];
      mn = fmin(mn, v);
      mx = fmax(mx, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
      mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
      red[2 * k][threadIdx.x >> 5] = mn;
      red[2 * k + 1][threadIdx.x >> 5] = mx;
    }
  }
  __syncthreads();
  if (threadIdx.x < 2 * d) {
    const int k = threadIdx.x >> 1, isMax = threadIdx.x & 1;
    double v = isMax ? -INFINITY : INFINITY;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
      v = isMax ? fmax(v, red[2 * k + 1][w]) : fmin(v, red[2 * k][w]);
    part[((int64_t)inst * nchunk + ch) * 2 * d + 2 * k + isMax] = v;
  }
}

// Per-position key flags for boxes of depth D that split (hypoct.m:90-93).
__global__ void k_flags(TreeDev t, int64_t ntot, int32_t b0, int32_t b1, int64_t occ, int can_split,
                        const int32_t* ldiv, int32_t* flags, int nl) {
  int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (pos > ntot) return;
  const int64_t stride = ntot + 1;
  int key = -1;
  if (pos < ntot && can_split) {
    int32_t b = t.pbox[pos];
    if (b >= b0 && b < b1 && t.seg_len[b] > occ) {
      const int dd = t.d;
      const int64_t pt = t.perm[pos];
      const int msk = ldiv[t.inst[b]];
      key = 0;
      for (int k = 0; k < dd; ++k)
        if (((msk >> k) & 1) && t.x[pt * dd + k] > t.ctr[(int64_t)b * dd + k]) key |= 1 << k;
    }
  }
  for (int c = 0; c < nl; ++c) flags[c * stride + pos] = (c == key) ? 1 : 0;
}

// Children of every splitting box (hypoct.m:94-115): count per key, number of children.
__global__ void k_count_children(TreeDev t, int64_t ntot, int32_t b0, int32_t b1, int64_t occ, int can_split,
                                 const int32_t* scan, int nl, int32_t* nch_tmp) {
  int32_t b = b0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= b1) return;
  int c = 0;
  if (can_split && t.seg_len[b] > occ) {
    const int64_t s = t.seg_start[b], e = s + t.seg_len[b], stride = ntot + 1;
    for (int k = 0; k < nl; ++k) c += (scan[k * stride + e] - scan[k * stride + s]) > 0;
  }
  nch_tmp[b - b0] = c;
}

__global__ void k_make_children(TreeDev t, int64_t ntot, int32_t b0, int32_t b1, const int32_t* scan, int nl,
                                const int32_t* base, const int32_t* ldiv, const double* lnew) {
  int32_t b = b0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= b1) return;
  const int32_t nc = base[b - b0 + 1] - base[b - b0];
  const int dd = t.d;
  if (nc == 0) {
    t.chfirst[b] = -1;
    t.nch[b] = 0;
    return;
  }
  const int32_t first = b1 + base[b - b0];
  t.chfirst[b] = first;
  t.nch[b] = nc;
  const int inst = t.inst[b];
  const int msk = ldiv[inst];
  const int64_t s = t.seg_start[b], e = s + t.seg_len[b], stride = ntot + 1;
  int64_t off = s;
  int32_t id = first;
  for (int k = 0; k < nl; ++k) {
    const int64_t cnt = scan[k * stride + e] - scan[k * stride + s];
    t.keychild[(int64_t)b * 8 + k] = cnt > 0 ? id : -1;
    if (cnt == 0) continue;
    for (int q = 0; q < dd; ++q) {
      // ctr + l.*ldiv.*(bitget(i,1:d) - 0.5)'  (hypoct.m:108); l.*ldiv is l or 0,
      // and the product with +-0.5 is exact, so the single rounded add matches.
      const double ll = ((msk >> q) & 1) ? lnew[inst * dd + q] : 0.0;
      const double h = __dmul_rn(ll, ((k >> q) & 1) ? 0.5 : -0.5);
      t.ctr[(int64_t)id * dd + q] = __dadd_rn(t.ctr[(int64_t)b * dd + q], h);
      t.lsz[(int64_t)id * dd + q] = lnew[inst * dd + q];
    }
    t.prnt[id] = b;
    t.seg_start[id] = off;
    t.seg_len[id] = cnt;
    t.depth[id] = t.depth[b] + 1;
    t.inst[id] = inst;
    t.chfirst[id] = -1;
    t.nch[id] = 0;
    off += cnt;
    ++id;
  }
}

// Stable partition of every splitting box's segment into its children.
__global__ void k_scatter(TreeDev t, int64_t ntot, int32_t b0, int32_t b1, int64_t occ, int can_split,
                          const int32_t* ldiv, const int32_t* flags_scan, int nl, int64_t* perm2, int32_t* pbox2) {
  int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= ntot) return;
  const int32_t b = t.pbox[pos];
  const int64_t pt = t.perm[pos];
  if (can_split && b >= b0 && b < b1 && t.seg_len[b] > occ) {
    const int dd = t.d;
    const int msk = ldiv[t.inst[b]];
    int key = 0;
    for (int k = 0; k < dd; ++k)
      if (((msk >> k) & 1) && t.x[pt * dd + k] > t.ctr[(int64_t)b * dd + k]) key |= 1 << k;
    const int32_t c = t.keychild[(int64_t)b * 8 + key];
    const int64_t stride = ntot + 1;
    const int64_t rank = flags_scan[key * stride + pos] - flags_scan[key * stride + t.seg_start[b]];
    const int64_t np = t.seg_start[c] + rank;
    perm2[np] = pt;
    pbox2[np] = c;
  } else {
    perm2[pos] = pt;
    pbox2[pos] = b;
  }
}

__device__ __forceinline__ bool coarse_adjacent(const TreeDev& t, int32_t i, int32_t j) {
  // dist = round((abs(ctr - jctr) - 0.5*(l + jl))./l); max(dist) <= 0   (hypoct.m:155-157)
  const int dd = t.d;
  double mx = -INFINITY;
  for (int q = 0; q < dd; ++q) {
    const double li = t.lsz[(int64_t)i * dd + q], lj = t.lsz[(int64_t)j * dd + q];
    const double a = fabs(__dsub_rn(t.ctr[(int64_t)i * dd + q], t.ctr[(int64_t)j * dd + q]));
    const double h = __dmul_rn(0.5, __dadd_rn(li, lj));
    const double v = round(__ddiv_rn(__dsub_rn(a, h), li));
    mx = fmax(mx, v);
  }
  return mx <= 0.0;
}

__device__ __forceinline__ bool child_adjacent(const TreeDev& t, int32_t i, int32_t c) {
  // dist = round(abs(ctr - ctr_c)./l); max(dist) <= 1   (hypoct.m:164-166)
  const int dd = t.d;
  double mx = -INFINITY;
  for (int q = 0; q < dd; ++q) {
    const double li = t.lsz[(int64_t)i * dd + q];
    const double a = fabs(__dsub_rn(t.ctr[(int64_t)i * dd + q], t.ctr[(int64_t)c * dd + q]));
    mx = fmax(mx, round(__ddiv_rn(a, li)));
  }
  return mx <= 1.0;
}

// Neighbours of the boxes of one depth (hypoct.m:141-170); pass 0 counts, pass 1 fills.
__global__ void k_neighbours(TreeDev t, int32_t b0, int32_t b1, int pass, int64_t* cnt_or_ptr) {
  int32_t i = b0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b1) return;
  const int32_t p = t.prnt[i];
  int64_t n = 0;
  int64_t w = pass ? cnt_or_ptr[i - b0] : 0;
  auto put = [&](int32_t j) {
    if (pass) t.nbor[w + n] = j;
    ++n;
  };
  // siblings, in child order (hypoct.m:148-149)
  for (int32_t c = t.chfirst[p]; c < t.chfirst[p] + t.nch[p]; ++c)
    if (c != i) put(c);
  const int64_t ps = t.nbor_ptr[p], pe = t.nbor_ptr[p + 1];
  // coarser leaf parent-neighbours (hypoct.m:152-160)
  for (int64_t q = ps; q < pe; ++q) {
    const int32_t j = t.nbor[q];
    if (t.nch[j] == 0 && coarse_adjacent(t, i, j)) put(j);
  }
  // children of parent-neighbours (hypoct.m:163-168)
  for (int64_t q = ps; q < pe; ++q) {
    const int32_t j = t.nbor[q];
    for (int32_t c = t.chfirst[j]; c < t.chfirst[j] + t.nch[j]; ++c)
      if (child_adjacent(t, i, c)) put(c);
  }
  if (!pass) cnt_or_ptr[i - b0] = n;
}

// hypoct_perm offsets, top-down: the stack pops the last child first (hypoct_perm.m:26-37).
__global__ void k_perm_offsets(TreeDev t, int32_t b0, int32_t b1, int64_t* off) {
  int32_t b = b0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= b1) return;
  if (t.nch[b] == 0) return;
  int64_t run = off[b];
  for (int32_t c = t.chfirst[b] + t.nch[b] - 1; c >= t.chfirst[b]; --c) {
    off[c] = run;
    run += t.seg_len[c];
  }
}

__global__ void k_perm_fill(TreeDev t, int32_t nbox, const int64_t* off, int64_t* P) {
  int32_t b = blockIdx.x;
  if (b >= nbox || t.nch[b] != 0) return;
  const int64_t s = t.seg_start[b], n = t.seg_len[b], o = off[b];
  for (int64_t q = threadIdx.x; q < n; q += blockDim.x) P[o + q] = t.perm[s + q];
}

}  // namespace

void tree_extent(const double* x, int d, const int64_t* inst_off_dev, int ninst, int nchunk, double* part,
                 cudaStream_t s) {
  dim3 g(ninst, nchunk);
  k_extent<<<g, 256, 0, s>>>(x, d, inst_off_dev, nchunk, part);
}

void tree_level_flags(const TreeDev& t, int64_t ntot, int32_t b0, int32_t b1, int64_t occ, int can_split,
                      const int32_t* ldiv, int32_t* flags, int nl, cudaStream_t s) {
  int64_t n = ntot + 1;
  k_flags<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(t, ntot, b0, b1, occ, can_split, ldiv, flags, nl);
}

void tree_level_count(const TreeDev& t, int64_t ntot, int32_t b0, int32_t b1, int64_t occ, int can_split,
                      const int32_t* scan, int nl, int32_t* nch_tmp, cudaStream_t s) {
  int32_t nb = b1 - b0;
  k_count_children<<<(nb + 127) / 128, 128, 0, s>>>(t, ntot, b0, b1, occ, can_split, scan, nl, nch_tmp);
}

void tree_level_children(const TreeDev& t, int64_t ntot, int32_t b0, int32_t b1, const int32_t* scan, int nl,
                         const int32_t* base, const int32_t* ldiv, const double* lnew, cudaStream_t s) {
  int32_t nb = b1 - b0;
  k_make_children<<<(nb + 127) / 128, 128, 0, s>>>(t, ntot, b0, b1, scan, nl, base, ldiv, lnew);
}

void tree_level_scatter(const TreeDev& t, int64_t ntot, int32_t b0, int32_t b1, int64_t occ, int can_split,
                        const int32_t* ldiv, const int32_t* scan, int nl, int64_t* perm2, int32_t* pbox2,
                        cudaStream_t s) {
  if (ntot <= 0) return;
  k_scatter<<<(unsigned)((ntot + 255) / 256), 256, 0, s>>>(t, ntot, b0, b1, occ, can_split, ldiv, scan, nl,
                                                            perm2, pbox2);
}

void tree_neighbours(const TreeDev& t, int32_t b0, int32_t b1, int pass, int64_t* cnt_or_ptr, cudaStream_t s) {
  int32_t nb = b1 - b0;
  if (nb <= 0) return;
  k_neighbours<<<(nb + 127) / 128, 128, 0, s>>>(t, b0, b1, pass, cnt_or_ptr);
}

void tree_perm_offsets(const TreeDev& t, int32_t b0, int32_t b1, int64_t* off, cudaStream_t s) {
  int32_t nb = b1 - b0;
  if (nb <= 0) return;
  k_perm_offsets<<<(nb + 127) / 128, 128, 0, s>>>(t, b0, b1, off);
}

void tree_perm_fill(const TreeDev& t, int32_t nbox, const int64_t* off, int64_t* P, cudaStream_t s) {
  if (nbox <= 0) return;
  k_perm_fill<<<nbox, 64, 0, s>>>(t, nbox, off, P);
}

}  // namespace flam
