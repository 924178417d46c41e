// K7: redundant-DOF elimination, one CTA per box of a factorization step.
//
// Reference (rskelf/rskelf.m:219-257), with [sk rd] the ID's split of slf:
//   K = A(slf,slf) + M                       M: children's blocks (rskelf.m:190-199)
//   K(rd,:) -= T' K(sk,:);  K(:,rd) -= K(:,sk) T
//   [L,U,p] = lu(K(rd,rd),'vector')          symm 'n'/'s'      (chol for 'p')
//   E = K(sk,rd)/U;  G = L\K(rd(p),sk)
//   M_new = M(sk,sk) - E*G                   (E*E' for 'p')
// The box's block lives in shared memory in [sk rd] order (global scratch for
// n > kSmemN); the children's M blocks are placed by the compress kernel's
// local permutation.  LU is right-looking with partial pivoting (the first
// maximum of |column|, as xGETF2), swapping whole rows so that the sk columns
// end up as K(rd(p),sk).
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"
#include "tile_f64.cuh"

namespace flam {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
// Dynamic shared memory of k_eliminate_big's LU panel: with its ~29 KB of static shared
// memory this stays inside the 227 KB a CTA may hold.
constexpr int kBigPanBytes = 192 * 1024;

struct AM {
  double v;
  int i;
};
__device__ __forceinline__ AM amax(AM a, AM b) {
  if (b.v > a.v || (b.v == a.v && b.i < a.i)) return b;
  return a;
}

// Child block of each position of slf: the compress kernel's local permutation
// maps a position to the concatenated children's skeleton order, and that order
// locates the entry inside the child's M block (rskelf.m:190-199).
__device__ __forceinline__ void locate_children(const ElimTask& t, const int32_t* perm, const ChildBlock* ch,
                                                int* pchild, int* ploc) {
  for (int q = threadIdx.x; q < t.n; q += kThreads) {
    const int o = perm[q];
    int c = -1, loc = 0;
    for (int b = 0; b < t.nch; ++b)
      if (o >= ch[b].coff && o < ch[b].coff + ch[b].kc) {
        c = b;
        loc = o - ch[b].coff;
      }
    pchild[q] = c;
    ploc[q] = loc;
  }
  __syncthreads();
}

// Entry (i, j) of the children's M blocks placed on the box (0 across children).
struct MVal {
  const double* m_in;
  const ChildBlock* ch;
  const int* pchild;
  const int* ploc;
  __device__ __forceinline__ double operator()(int i, int j) const {
    const int c = pchild[i];
    if (c < 0 || c != pchild[j]) return 0.0;
    const int kc = ch[c].kc;
    return m_in[ch[c].M_off + ploc[i] + (int64_t)ploc[j] * kc];
  }
};

__global__ void __launch_bounds__(kThreads) k_eliminate(ElimArgs a) {
  extern __shared__ __align__(16) double smem[];
  __shared__ __align__(16) double tsm[kTileSmemDoubles];
  __shared__ AM red[kWarps];
  __shared__ int s_piv;
  const ElimTask t = a.tasks[blockIdx.x];
  const Problem& P = a.P;
  const InstParams ip = P.ip[t.inst];
  const int n = t.n, k = t.k, r = n - k;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (n == 0) return;
  double* K = (t.scr_off >= 0) ? a.scratch + t.scr_off : smem;     // n x n, ld n
  int* pchild = reinterpret_cast<int*>(K + (int64_t)n * n);         // n: child block of each position
  int* ploc = pchild + n;                                           // n: index inside that block
  int* piv = ploc + n;                                              // r: LU row interchanges
  const int64_t* slf = a.ipool + t.slf_off;
  const int32_t* perm = a.permpool + t.perm_off;
  const ChildBlock* ch = a.children + t.ch_first;
  locate_children(t, perm, ch, pchild, ploc);
  const MVal mval{a.m_in, ch, pchild, ploc};

  // 2D loops use a fixed 32 x 8 thread tile: lane = row within a 32-row block
  // (consecutive column-major addresses), warp = column within an 8-column block;
  // no index is divided and every lane has work once a block has 32 rows.
  const int tr = lane, tcol = wid;
  if (r == 0) {  // no compression: the box keeps its whole modified block (rskelf.m:216)
    double* Mo = a.m_out + t.M_out;
    for (int j = tcol; j < n; j += kWarps)
      for (int i = tr; i < n; i += 32) Mo[i + (int64_t)j * n] = mval(i, j);
    return;
  }

  // K = A(slf,slf) + M in [sk rd] order
  for (int j = tcol; j < n; j += kWarps) {
    const int64_t sj = slf[j];
    for (int i = tr; i < n; i += 32) K[i + (int64_t)j * n] = aentry(P, ip, slf[i], sj) + mval(i, j);
  }
  __syncthreads();

  const double* T = a.tpool + t.T_off;  // k x r, ld k
  if (k > 0) {
    // K(rd,:) -= T' K(sk,:);  K(:,rd) -= K(:,sk) T   (T.' for 's': identical for real
    // data), as 64 x 64 tiles with T staged through shared memory
    const int64_t ldn = n;
    cta_gemm(K + k, 1, ldn, GV{T, k, 1}, GV{K, 1, ldn}, r, n, k, -1.0, tsm);
    cta_gemm(K + (int64_t)k * n, 1, ldn, GV{K, 1, ldn}, GV{T, 1, k}, n, r, k, -1.0, tsm);
  }

  double* Kr = K + k + (int64_t)k * n;  // r x r block, ld n
  if (a.symm == 'p') {
    // chol(K(rd,rd),'lower'), right-looking
    for (int j = 0; j < r; ++j) {
      const double dj = Kr[j + (int64_t)j * n];
      if (!(dj > 0.0)) {
        if (tid == 0) atomicOr(a.status, (int)ST_NOT_SPD);
        return;
      }
      const double lj = sqrt(dj);
      __syncthreads();
      for (int q = j + 1 + tid; q < r; q += kThreads) Kr[q + (int64_t)j * n] /= lj;
      if (tid == 0) Kr[j + (int64_t)j * n] = lj;
      __syncthreads();
      for (int c = j + 1 + tcol; c < r; c += kWarps) {
        const double lc = Kr[c + (int64_t)j * n];
        for (int q = c + tr; q < r; q += 32) Kr[q + (int64_t)c * n] -= Kr[q + (int64_t)j * n] * lc;
      }
      __syncthreads();
    }
    // E = K(sk,rd)/L'  : row a solves x L' = K(a, rd)
    for (int row = tid; row < k; row += kThreads) {
      for (int j = 0; j < r; ++j) {
        double v = K[row + (int64_t)(k + j) * n];
        for (int i = 0; i < j; ++i) v -= K[row + (int64_t)(k + i) * n] * Kr[j + (int64_t)i * n];
        K[row + (int64_t)(k + j) * n] = v / Kr[j + (int64_t)j * n];
      }
    }
    __syncthreads();
  } else {
    // [L,U,p] = lu(K(rd,rd),'vector')
    for (int j = 0; j < r; ++j) {
      AM am{-1.0, r};
      for (int q = j + tid; q < r; q += kThreads) am = amax(am, AM{fabs(Kr[q + (int64_t)j * n]), q});
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        AM b{__shfl_xor_sync(0xffffffffu, am.v, o), __shfl_xor_sync(0xffffffffu, am.i, o)};
        am = amax(am, b);
      }
      if (lane == 0) red[wid] = am;
      __syncthreads();
      if (tid == 0) {
        AM bm = red[0];
        for (int w = 1; w < kWarps; ++w) bm = amax(bm, red[w]);
        const int pv0 = (bm.i >= j && bm.i < r) ? bm.i : j;
        s_piv = pv0;
        piv[j] = pv0;
      }
      __syncthreads();
      const int pv = (s_piv >= j && s_piv < r) ? s_piv : j;   // NaN column: keep the row
      if (pv != j)
        for (int col = tid; col < n; col += kThreads) {
          const double tmp = K[k + j + (int64_t)col * n];
          K[k + j + (int64_t)col * n] = K[k + pv + (int64_t)col * n];
          K[k + pv + (int64_t)col * n] = tmp;
        }
      __syncthreads();
      const double dj = Kr[j + (int64_t)j * n];
      if (dj != 0.0) {
        for (int q = j + 1 + tid; q < r; q += kThreads) Kr[q + (int64_t)j * n] /= dj;
      } else if (tid == 0) {
        atomicOr(a.status, (int)ST_SINGULAR);
      }
      __syncthreads();
      for (int c = j + 1 + tcol; c < r; c += kWarps) {
        const double ujc = Kr[j + (int64_t)c * n];
        for (int q = j + 1 + tr; q < r; q += 32) Kr[q + (int64_t)c * n] -= Kr[q + (int64_t)j * n] * ujc;
      }
      __syncthreads();
    }
    // E = K(sk,rd)/U
    for (int row = tid; row < k; row += kThreads) {
      for (int j = 0; j < r; ++j) {
        double v = K[row + (int64_t)(k + j) * n];
        for (int i = 0; i < j; ++i) v -= K[row + (int64_t)(k + i) * n] * Kr[i + (int64_t)j * n];
        K[row + (int64_t)(k + j) * n] = v / Kr[j + (int64_t)j * n];
      }
    }
    // G = L\K(rd(p),sk): rows were swapped in place, L is unit lower
    for (int col = tid; col < k; col += kThreads) {
      for (int i = 0; i < r; ++i) {
        double v = K[k + i + (int64_t)col * n];
        for (int j = 0; j < i; ++j) v -= Kr[i + (int64_t)j * n] * K[k + j + (int64_t)col * n];
        K[k + i + (int64_t)col * n] = v;
      }
    }
    __syncthreads();
  }

  // M_new = M(sk,sk) - E*G   (E*E' for 'p')
  double* Mo = a.m_out + t.M_out;
  const bool chol = a.symm == 'p';
  for (int j = tcol; j < k; j += kWarps) {
    for (int i = tr; i < k; i += 32) {
      double s = 0.0;
      if (chol)
        for (int q = 0; q < r; ++q) s += K[i + (int64_t)(k + q) * n] * K[j + (int64_t)(k + q) * n];
      else
        for (int q = 0; q < r; ++q) s += K[i + (int64_t)(k + q) * n] * K[k + q + (int64_t)j * n];
      Mo[i + (int64_t)j * k] = mval(i, j) - s;
    }
  }

  // store the factor: T | LU (or L) | E | G
  double* F = a.fpool + t.fac_off;
  const int64_t kr = (int64_t)k * r, rr = (int64_t)r * r;
  for (int64_t e = tid; e < kr; e += kThreads) F[e] = T[e];
  for (int j = tcol; j < r; j += kWarps)
    for (int i = tr; i < r; i += 32) F[kr + i + (int64_t)j * r] = (chol && i < j) ? 0.0 : Kr[i + (int64_t)j * n];
  for (int j = tcol; j < r; j += kWarps)
    for (int i = tr; i < k; i += 32) F[kr + rr + i + (int64_t)j * k] = K[i + (int64_t)(k + j) * n];
  if (!chol) {
    for (int j = tcol; j < k; j += kWarps)
      for (int i = tr; i < r; i += 32) F[2 * kr + rr + i + (int64_t)j * r] = K[k + i + (int64_t)j * n];
    if (tid == 0) {  // p from the sequence of interchanges
      int32_t* pp = a.ppool + t.piv_off;
      for (int q = 0; q < r; ++q) pp[q] = q;
      for (int q = 0; q < r; ++q) {
        const int32_t x = pp[q];
        pp[q] = pp[piv[q]];
        pp[piv[q]] = x;
      }
    }
  }
}

// Boxes with n > kSmemN: the same elimination with the work matrix in global
// memory (L2-resident) and every O(n^3) part blocked over 32-column panels, so
// that the bulk of the flops are CTA-wide 64 x 64 tiles (cta_gemm) instead of
// rank-1 updates:
//   T updates              two GEMMs (inner dimension k)
//   LU / chol of K(rd,rd)  right-looking, unblocked 32-column panels (partial
//                          pivoting as xGETF2 inside the panel; the panel's row
//                          interchanges then applied to every other column),
//                          TRSM of the panel's U row block, GEMM trailing update
//   E, G                   blocked triangular solves: a 32 x 32 diagonal block
//                          staged in shared memory, GEMM update of the rest
//   Schur                  one GEMM (E G, or E E' for chol)
constexpr int kNb = 32;

__global__ void __launch_bounds__(kThreads) k_eliminate_big(ElimArgs a) {
  extern __shared__ __align__(16) double pan[];   // LU panel: a.pan_rows x kNb doubles
  __shared__ __align__(16) double tsm[kTileSmemDoubles];
  __shared__ double blk[kNb * (kNb + 1)];
  __shared__ AM red[kWarps];
  __shared__ int s_piv;
  const ElimTask t = a.tasks[blockIdx.x];
  const Problem& P = a.P;
  const InstParams ip = P.ip[t.inst];
  const int n = t.n, k = t.k, r = n - k;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (n == 0) return;
  double* K = a.scratch + t.scr_off;                                // n x n, ld n
  int* pchild = reinterpret_cast<int*>(K + (int64_t)n * n);
  int* ploc = pchild + n;
  int* piv = ploc + n;
  const int64_t* slf = a.ipool + t.slf_off;
  const int32_t* perm = a.permpool + t.perm_off;
  const ChildBlock* ch = a.children + t.ch_first;
  locate_children(t, perm, ch, pchild, ploc);
  const MVal mval{a.m_in, ch, pchild, ploc};
  const int tr = lane, tcol = wid;
  const int64_t ldn = n;
  if (r == 0) {
    double* Mo = a.m_out + t.M_out;
    for (int j = tcol; j < n; j += kWarps)
      for (int i = tr; i < n; i += 32) Mo[i + (int64_t)j * n] = mval(i, j);
    return;
  }
  for (int j = tcol; j < n; j += kWarps) {
    const int64_t sj = slf[j];
    for (int i = tr; i < n; i += 32) K[i + (int64_t)j * n] = aentry(P, ip, slf[i], sj) + mval(i, j);
  }
  __syncthreads();

  const double* T = a.tpool + t.T_off;  // k x r, ld k
  if (k > 0) {
    // K(rd,:) -= T' K(sk,:);  K(:,rd) -= K(:,sk) T
    cta_gemm(K + k, 1, ldn, GV{T, k, 1}, GV{K, 1, ldn}, r, n, k, -1.0, tsm);
    cta_gemm(K + (int64_t)k * n, 1, ldn, GV{K, 1, ldn}, GV{T, 1, k}, n, r, k, -1.0, tsm);
  }

  double* Kr = K + k + (int64_t)k * n;  // r x r block, ld n
  auto kr = [&](int i, int j) -> double& { return Kr[i + (int64_t)j * n]; };
  const bool chol = a.symm == 'p';
  for (int j0 = 0; j0 < r; j0 += kNb) {
    const int jb = min(kNb, r - j0), j1 = j0 + jb;
    if (chol) {
      for (int j = j0; j < j1; ++j) {
        const double dj = kr(j, j);
        if (!(dj > 0.0)) {
          if (tid == 0) atomicOr(a.status, (int)ST_NOT_SPD);
          return;
        }
        const double lj = sqrt(dj);
        __syncthreads();
        for (int q = j + 1 + tid; q < r; q += kThreads) kr(q, j) /= lj;
        if (tid == 0) kr(j, j) = lj;
        __syncthreads();
        for (int c = j + 1 + tcol; c < j1; c += kWarps) {
          const double lc = kr(c, j);
          for (int q = c + tr; q < r; q += 32) kr(q, c) -= kr(q, j) * lc;
        }
        __syncthreads();
      }
      // trailing lower part -= L21 L21'
      cta_gemm(&kr(j1, j1), 1, ldn, GV{&kr(j1, j0), 1, ldn}, GV{&kr(j1, j0), ldn, 1}, r - j1, r - j1, jb, -1.0,
               tsm, 1);
    } else {
      if (r <= a.pan_rows) {
        // the panel (rows j0.., jb columns) in shared memory: its pivot searches, swaps,
        // scalings and rank-1 updates read no L2
        const int pr = r - j0;
        auto pp = [&](int i, int c) -> double& { return pan[(i - j0) + c * pr]; };
        for (int e = tid; e < pr * jb; e += kThreads) pan[e] = kr(j0 + e % pr, j0 + e / pr);
        __syncthreads();
        for (int j = j0; j < j1; ++j) {
          const int jl = j - j0;
          AM am{-1.0, r};
          for (int q = j + tid; q < r; q += kThreads) am = amax(am, AM{fabs(pp(q, jl)), q});
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            AM b{__shfl_xor_sync(0xffffffffu, am.v, o), __shfl_xor_sync(0xffffffffu, am.i, o)};
            am = amax(am, b);
          }
          if (lane == 0) red[wid] = am;
          __syncthreads();
          if (tid == 0) {
            AM bm = red[0];
            for (int w = 1; w < kWarps; ++w) bm = amax(bm, red[w]);
            const int pv0 = (bm.i >= j && bm.i < r) ? bm.i : j;
            s_piv = pv0;
            piv[j] = pv0;
          }
          __syncthreads();
          const int pv = (s_piv >= j && s_piv < r) ? s_piv : j;
          if (pv != j && tid < jb) {
            const double x = pp(j, tid);
            pp(j, tid) = pp(pv, tid);
            pp(pv, tid) = x;
          }
          __syncthreads();
          const double dj = pp(j, jl);
          if (dj != 0.0) {
            for (int q = j + 1 + tid; q < r; q += kThreads) pp(q, jl) /= dj;
          } else if (tid == 0) {
            atomicOr(a.status, (int)ST_SINGULAR);
          }
          __syncthreads();
          for (int c = jl + 1 + tcol; c < jb; c += kWarps) {
            const double ujc = pp(j, c);
            for (int q = j + 1 + tr; q < r; q += 32) pp(q, c) -= pp(q, jl) * ujc;
          }
          __syncthreads();
        }
        for (int e = tid; e < pr * jb; e += kThreads) kr(j0 + e % pr, j0 + e / pr) = pan[e];
        __syncthreads();
      } else {
        for (int j = j0; j < j1; ++j) {
          AM am{-1.0, r};
          for (int q = j + tid; q < r; q += kThreads) am = amax(am, AM{fabs(kr(q, j)), q});
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            AM b{__shfl_xor_sync(0xffffffffu, am.v, o), __shfl_xor_sync(0xffffffffu, am.i, o)};
            am = amax(am, b);
          }
          if (lane == 0) red[wid] = am;
          __syncthreads();
          if (tid == 0) {
            AM bm = red[0];
            for (int w = 1; w < kWarps; ++w) bm = amax(bm, red[w]);
            const int pv0 = (bm.i >= j && bm.i < r) ? bm.i : j;
            s_piv = pv0;
            piv[j] = pv0;
          }
          __syncthreads();
          const int pv = (s_piv >= j && s_piv < r) ? s_piv : j;
          if (pv != j && tid < jb) {  // inside the panel; the other columns after it
            const double x = kr(j, j0 + tid);
            kr(j, j0 + tid) = kr(pv, j0 + tid);
            kr(pv, j0 + tid) = x;
          }
          __syncthreads();
          const double dj = kr(j, j);
          if (dj != 0.0) {
            for (int q = j + 1 + tid; q < r; q += kThreads) kr(q, j) /= dj;
          } else if (tid == 0) {
            atomicOr(a.status, (int)ST_SINGULAR);
          }
          __syncthreads();
          for (int c = j + 1 + tcol; c < j1; c += kWarps) {
            const double ujc = kr(j, c);
            for (int q = j + 1 + tr; q < r; q += 32) kr(q, c) -= kr(q, j) * ujc;
          }
          __syncthreads();
        }
      }
      // the panel's interchanges on every other column of K (whole rows of K(rd,:))
      for (int col = tid; col < n; col += kThreads) {
        if (col >= k + j0 && col < k + j1) continue;
        double* Kc = K + k + (int64_t)col * n;
        for (int j = j0; j < j1; ++j) {
          const int pv = piv[j];
          if (pv != j) {
            const double x = Kc[j];
            Kc[j] = Kc[pv];
            Kc[pv] = x;
          }
        }
      }
      // L11 (unit lower) to shared memory
      for (int e = tid; e < jb * jb; e += kThreads) {
        const int i = e % jb, c = e / jb;
        blk[i + c * (kNb + 1)] = kr(j0 + i, j0 + c);
      }
      __syncthreads();
      // U12 = L11 \ A12, one column per thread
      for (int c = j1 + tid; c < r; c += kThreads) {
        double x[kNb];
#pragma unroll
        for (int i = 0; i < kNb; ++i)
          if (i < jb) x[i] = kr(j0 + i, c);
#pragma unroll
        for (int i = 0; i < kNb; ++i) {
          if (i < jb) {
            double v = x[i];
#pragma unroll
            for (int l = 0; l < i; ++l) v -= blk[i + l * (kNb + 1)] * x[l];
            x[i] = v;
          }
        }
#pragma unroll
        for (int i = 0; i < kNb; ++i)
          if (i < jb) kr(j0 + i, c) = x[i];
      }
      __syncthreads();
      cta_gemm(&kr(j1, j1), 1, ldn, GV{&kr(j1, j0), 1, ldn}, GV{&kr(j0, j1), 1, ldn}, r - j1, r - j1, jb, -1.0, tsm);
    }
  }

  // E = K(sk,rd) / U  (U = L' for chol): row-parallel blocked solve
  if (k > 0) {
    double* C = K + (int64_t)k * n;   // K(sk, rd): k x r, ld n
    for (int j0 = 0; j0 < r; j0 += kNb) {
      const int jb = min(kNb, r - j0), j1 = j0 + jb;
      for (int e = tid; e < jb * jb; e += kThreads) {   // U(j0+i, j0+c)
        const int i = e % jb, c = e / jb;
        blk[i + c * (kNb + 1)] = chol ? kr(j0 + c, j0 + i) : kr(j0 + i, j0 + c);
      }
      __syncthreads();
      for (int row = tid; row < k; row += kThreads) {
        double x[kNb];
#pragma unroll
        for (int c = 0; c < kNb; ++c) {
          if (c < jb) {
            double v = C[row + (int64_t)(j0 + c) * n];
#pragma unroll
            for (int l = 0; l < c; ++l) v -= x[l] * blk[l + c * (kNb + 1)];
            x[c] = v / blk[c + c * (kNb + 1)];
          }
        }
#pragma unroll
        for (int c = 0; c < kNb; ++c)
          if (c < jb) C[row + (int64_t)(j0 + c) * n] = x[c];
      }
      __syncthreads();
      if (j1 < r) {
        const GV U12 = chol ? GV{&kr(j1, j0), ldn, 1} : GV{&kr(j0, j1), 1, ldn};
        cta_gemm(C + (int64_t)j1 * n, 1, ldn, GV{C + (int64_t)j0 * n, 1, ldn}, U12, k, r - j1, jb, -1.0, tsm);
      }
    }
    if (!chol) {
      // G = L \ K(rd(p), sk): column-parallel blocked solve, L unit lower
      double* Gc = K + k;               // K(rd, sk): r x k, ld n
      for (int j0 = 0; j0 < r; j0 += kNb) {
        const int jb = min(kNb, r - j0), j1 = j0 + jb;
        for (int e = tid; e < jb * jb; e += kThreads) {
          const int i = e % jb, c = e / jb;
          blk[i + c * (kNb + 1)] = kr(j0 + i, j0 + c);
        }
        __syncthreads();
        for (int col = tid; col < k; col += kThreads) {
          double x[kNb];
#pragma unroll
          for (int i = 0; i < kNb; ++i) {
            if (i < jb) {
              double v = Gc[j0 + i + (int64_t)col * n];
#pragma unroll
              for (int l = 0; l < i; ++l) v -= blk[i + l * (kNb + 1)] * x[l];
              x[i] = v;
            }
          }
#pragma unroll
          for (int i = 0; i < kNb; ++i)
            if (i < jb) Gc[j0 + i + (int64_t)col * n] = x[i];
        }
        __syncthreads();
        if (j1 < r)
          cta_gemm(Gc + j1, 1, ldn, GV{&kr(j1, j0), 1, ldn}, GV{Gc + j0, 1, ldn}, r - j1, k, jb, -1.0, tsm);
      }
    }
  }

  // M_new = M(sk,sk) - E G   (E E' for chol)
  double* Mo = a.m_out + t.M_out;
  for (int j = tcol; j < k; j += kWarps)
    for (int i = tr; i < k; i += 32) Mo[i + (int64_t)j * k] = mval(i, j);
  __syncthreads();
  if (k > 0) {
    const GV E{K + (int64_t)k * n, 1, ldn};
    const GV Bm = chol ? GV{K + (int64_t)k * n, ldn, 1} : GV{K + k, 1, ldn};
    cta_gemm(Mo, 1, k, E, Bm, k, k, r, -1.0, tsm);
  }

  // store the factor: T | LU (or L) | E | G
  double* F = a.fpool + t.fac_off;
  const int64_t kr_ = (int64_t)k * r, rr = (int64_t)r * r;
  for (int64_t e = tid; e < kr_; e += kThreads) F[e] = T[e];
  for (int j = tcol; j < r; j += kWarps)
    for (int i = tr; i < r; i += 32) F[kr_ + i + (int64_t)j * r] = (chol && i < j) ? 0.0 : kr(i, j);
  for (int j = tcol; j < r; j += kWarps)
    for (int i = tr; i < k; i += 32) F[kr_ + rr + i + (int64_t)j * k] = K[i + (int64_t)(k + j) * n];
  if (!chol) {
    for (int j = tcol; j < k; j += kWarps)
      for (int i = tr; i < r; i += 32) F[2 * kr_ + rr + i + (int64_t)j * r] = K[k + i + (int64_t)j * n];
    if (tid == 0) {
      int32_t* pp = a.ppool + t.piv_off;
      for (int q = 0; q < r; ++q) pp[q] = q;
      for (int q = 0; q < r; ++q) {
        const int32_t x = pp[q];
        pp[q] = pp[piv[q]];
        pp[piv[q]] = x;
      }
    }
  }
}

// ---------------------------------------------------------------- boxes eliminated by many CTAs
// A box whose redundant block is large (the few boxes near the root in 3D, the root of a
// 2D tree) is eliminated by a sequence of grid-wide launches instead of one CTA: the same
// algebra as k_eliminate_big (rskelf.m:219-257), with every O(n^3) part a batched FP64
// GEMM on the tensor path (mma.sync m8n8k4 .f64) over 64 x 64 tiles, and the LU panels
// (kHb columns, partial pivoting as xGETF2) factored by one CTA per box.  blockIdx.z is
// the box within the launch's task list; a box whose r is exhausted leaves at once.

// LU / solve panel width: the panel factorization streams its (r - j0) x kHb block
// through one SM once per column (~r^2 kHb bytes in all), the trailing updates stream
// the trailing matrix once per panel (~r^3 / kHb bytes, over the whole GPU); 32 balances
// the two for the redundant blocks of a few thousand rows this path takes.
constexpr int kHb = 32;
constexpr int kPanelThreads = 512;
constexpr int kGk = 16;         // GEMM k-chunk
constexpr int kGld = kGk + 4;   // shared row stride: 20 = 4 mod 16

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// Views of one box's work matrix (K: n x n, ld n, [sk rd] order) for each GEMM kind.
enum HbKind { HB_TROW = 0, HB_TCOL, HB_TRAIL, HB_TRAIL_CHOL, HB_EUPD, HB_GUPD, HB_SCHUR };

struct HbOp {
  double* C;
  int64_t crs, ccs;
  GV A, B;
  int M, N, K;
};

__device__ __forceinline__ HbOp hb_op(const ElimArgs& a, const ElimTask& t, int kind, int j0) {
  const int n = t.n, k = t.k, r = n - k;
  const int64_t ld = n;
  double* K = a.scratch + t.scr_off;
  double* Kr = K + k + (int64_t)k * n;
  const int jb = min(kHb, r - j0), j1 = j0 + jb;
  const double* T = a.tpool + t.T_off;
  HbOp o{};
  switch (kind) {
    case HB_TROW:   // K(rd,:) -= T' K(sk,:)
      o = HbOp{K + k, 1, ld, GV{T, k, 1}, GV{K, 1, ld}, r, n, k};
      break;
    case HB_TCOL:   // K(:,rd) -= K(:,sk) T
      o = HbOp{K + (int64_t)k * n, 1, ld, GV{K, 1, ld}, GV{T, 1, k}, n, r, k};
      break;
    case HB_TRAIL:  // A22 -= L21 U12
      o = HbOp{Kr + j1 + (int64_t)j1 * n, 1, ld, GV{Kr + j1 + (int64_t)j0 * n, 1, ld},
               GV{Kr + j0 + (int64_t)j1 * n, 1, ld}, r - j1, r - j1, jb};
      break;
    case HB_TRAIL_CHOL:   // A22 -= L21 L21'
      o = HbOp{Kr + j1 + (int64_t)j1 * n, 1, ld, GV{Kr + j1 + (int64_t)j0 * n, 1, ld},
               GV{Kr + j1 + (int64_t)j0 * n, ld, 1}, r - j1, r - j1, jb};
      break;
    case HB_EUPD: {   // E(:, j1:) -= E(:, j0:j1) U(j0:j1, j1:)
      double* E = K + (int64_t)k * n;
      const GV U12 = a.symm == 'p' ? GV{Kr + j1 + (int64_t)j0 * n, ld, 1} : GV{Kr + j0 + (int64_t)j1 * n, 1, ld};
      o = HbOp{E + (int64_t)j1 * n, 1, ld, GV{E + (int64_t)j0 * n, 1, ld}, U12, k, r - j1, jb};
      break;
    }
    case HB_GUPD: {   // G(j1:, :) -= L(j1:, j0:j1) G(j0:j1, :)
      double* G = K + k;
      o = HbOp{G + j1, 1, ld, GV{Kr + j1 + (int64_t)j0 * n, 1, ld}, GV{G + j0, 1, ld}, r - j1, k, jb};
      break;
    }
    default: {        // HB_SCHUR: M_new -= E G (E E' for 'p')
      const GV E{K + (int64_t)k * n, 1, ld};
      const GV Bm = a.symm == 'p' ? GV{K + (int64_t)k * n, ld, 1} : GV{K + k, 1, ld};
      o = HbOp{a.m_out + t.M_out, 1, k, E, Bm, k, k, r};
      break;
    }
  }
  return o;
}

// C tile (64 x 64) at (i0, c0) -= A B of the operation: 4 warps, each 32 x 32 outputs.
__device__ void hb_gemm_tile(const HbOp& o, int i0, int c0, double* As, double* Bs) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int wm = warp >> 1, wn = warp & 1;
  const bool a_col = o.A.rs == 1, b_col = o.B.rs == 1;
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  double ra[8], rb[8];
  auto load = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + 128 * q;
      const int m = a_col ? (e & 63) : (e >> 4), kk = a_col ? (e >> 6) : (e & 15);
      ra[q] = (i0 + m < o.M && k0 + kk < o.K) ? o.A.at(i0 + m, k0 + kk) : 0.0;
      const int nn = b_col ? (e >> 4) : (e & 63), kb = b_col ? (e & 15) : (e >> 6);
      rb[q] = (c0 + nn < o.N && k0 + kb < o.K) ? o.B.at(k0 + kb, c0 + nn) : 0.0;
    }
  };
  auto stash = [&]() {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + 128 * q;
      const int m = a_col ? (e & 63) : (e >> 4), kk = a_col ? (e >> 6) : (e & 15);
      As[m * kGld + kk] = ra[q];
      const int nn = b_col ? (e >> 4) : (e & 63), kb = b_col ? (e & 15) : (e >> 6);
      Bs[nn * kGld + kb] = rb[q];
    }
  };
  load(0);
  for (int k0 = 0; k0 < o.K; k0 += kGk) {
    __syncthreads();
    stash();
    __syncthreads();
    if (k0 + kGk < o.K) load(k0 + kGk);   // next chunk's loads in flight during the products
    const double* Aw = As + (wm * 32 + g) * kGld + tq;
    const double* Bw = Bs + (wn * 32 + g) * kGld + tq;
#pragma unroll
    for (int kk = 0; kk < kGk; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = Aw[i * 8 * kGld + kk];
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = Bw[j * 8 * kGld + kk];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j], af[i], bf[j]);
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int row = i0 + wm * 32 + i * 8 + g;
    if (row >= o.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = c0 + wn * 32 + j * 8 + 2 * tq + e;
        if (col < o.N) o.C[row * o.crs + col * o.ccs] -= acc[i][j][e];
      }
  }
}

__global__ void __launch_bounds__(128) k_hb_gemm(ElimArgs a, int kind, int j0) {
  __shared__ double As[kTM * kGld];
  __shared__ double Bs[kTN * kGld];
  const ElimTask t = a.tasks[blockIdx.z];
  const int r = t.n - t.k;
  if (r <= 0 || j0 >= r) return;
  if ((kind == HB_TROW || kind == HB_TCOL || kind == HB_EUPD || kind == HB_GUPD || kind == HB_SCHUR) && t.k == 0)
    return;
  const HbOp o = hb_op(a, t, kind, j0);
  const int i0 = blockIdx.x * kTM, c0 = blockIdx.y * kTN;
  if (i0 >= o.M || c0 >= o.N || o.K <= 0) return;
  hb_gemm_tile(o, i0, c0, As, Bs);
}

// One explicit product C -= A B over a grid of 64 x 64 tiles (the grid-wide sweep).
__global__ void __launch_bounds__(128) k_dgemm_op(HbOp o) {
  __shared__ double As[kTM * kGld];
  __shared__ double Bs[kTN * kGld];
  const int i0 = blockIdx.x * kTM, c0 = blockIdx.y * kTN;
  if (i0 >= o.M || c0 >= o.N || o.K <= 0) return;
  hb_gemm_tile(o, i0, c0, As, Bs);
}

// Rows j0..j0+jb of X (r x nrhs, column-major) solved against the diagonal block of the
// triangular view M (lower: forward, upper: backward; unit diagonal or not), one thread
// per right-hand side.
__global__ void __launch_bounds__(256) k_trsm_diag(GV M, double* X, int r, int nrhs, int j0, int jb, int lower,
                                                   int unit) {
  __shared__ double blk[kHb * (kHb + 1)];
  for (int e = threadIdx.x; e < jb * jb; e += blockDim.x) {
    const int i = e % jb, c = e / jb;
    blk[i + c * (kHb + 1)] = M.at(j0 + i, j0 + c);
  }
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= nrhs) return;
  double* x = X + j0 + (int64_t)col * r;
  double v[kHb];
#pragma unroll
  for (int i = 0; i < kHb; ++i) v[i] = i < jb ? x[i] : 0.0;
  if (lower) {
#pragma unroll
    for (int i = 0; i < kHb; ++i) {
      if (i < jb) {
        double s = v[i];
#pragma unroll
        for (int l = 0; l < i; ++l) s -= blk[i + l * (kHb + 1)] * v[l];
        v[i] = unit ? s : s / blk[i + i * (kHb + 1)];
      }
    }
  } else {
#pragma unroll
    for (int i = kHb - 1; i >= 0; --i) {
      if (i < jb) {
        double s = v[i];
#pragma unroll
        for (int l = i + 1; l < kHb; ++l)
          if (l < jb) s -= blk[i + l * (kHb + 1)] * v[l];
        v[i] = unit ? s : s / blk[i + i * (kHb + 1)];
      }
    }
  }
#pragma unroll
  for (int i = 0; i < kHb; ++i)
    if (i < jb) x[i] = v[i];
}

// Rows idx[perm ? perm[i] : i] of the point-major work array W (ld nrhs) <-> the dense
// r x nrhs block X; dir 0 gathers, 1 scatters.
__global__ void k_rows_gs(double* W, int nrhs, const int64_t* idx, const int32_t* perm, int r, double* X, int dir) {
  const int64_t total = (int64_t)r * nrhs;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(e % nrhs);
    const int i = (int)(e / nrhs);
    const int64_t pt = idx[perm ? perm[i] : i];
    if (dir == 0)
      X[i + (int64_t)c * r] = W[pt * nrhs + c];
    else
      W[pt * nrhs + c] = X[i + (int64_t)c * r];
  }
}

// Child lookup of every position (one CTA per box).
__global__ void __launch_bounds__(kThreads) k_hb_locate(ElimArgs a) {
  const ElimTask t = a.tasks[blockIdx.x];
  if (t.n == 0) return;
  double* K = a.scratch + t.scr_off;
  int* pchild = reinterpret_cast<int*>(K + (int64_t)t.n * t.n);
  locate_children(t, a.permpool + t.perm_off, a.children + t.ch_first, pchild, pchild + t.n);
}

// K = A(slf,slf) + M in [sk rd] order and M_new = M(sk,sk) (the Schur GEMM subtracts E G
// from it); a box with r = 0 passes its whole block on.  32 x 32 entries per CTA.
__global__ void __launch_bounds__(kThreads) k_hb_assemble(ElimArgs a) {
  const ElimTask t = a.tasks[blockIdx.z];
  const int n = t.n, k = t.k, r = n - k;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  if (i0 >= n || j0 >= n) return;
  const Problem& P = a.P;
  const InstParams ip = P.ip[t.inst];
  double* K = a.scratch + t.scr_off;
  const int* pchild = reinterpret_cast<const int*>(K + (int64_t)n * n);
  const MVal mval{a.m_in, a.children + t.ch_first, pchild, pchild + n};
  const int64_t* slf = a.ipool + t.slf_off;
  double* Mo = a.m_out + t.M_out;
  const int i = i0 + (threadIdx.x & 31);
  if (i >= n) return;
  const int64_t si = slf[i];
  for (int j = j0 + (threadIdx.x >> 5); j < min(n, j0 + 32); j += kThreads / 32) {
    const double mv = mval(i, j);
    if (r == 0) {
      Mo[i + (int64_t)j * n] = mv;
      continue;
    }
    K[i + (int64_t)j * n] = aentry(P, ip, si, slf[j]) + mv;
    if (i < k && j < k) Mo[i + (int64_t)j * k] = mv;
  }
}

// LU (or Cholesky) of the panel rows j0.., columns j0..j1 of K(rd,rd), one CTA per box.
__global__ void __launch_bounds__(kPanelThreads) k_hb_panel(ElimArgs a, int j0) {
  constexpr int kThreads = kPanelThreads, kWarps = kPanelThreads / 32;
  __shared__ AM red[kWarps];
  __shared__ int s_piv;
  const ElimTask t = a.tasks[blockIdx.x];
  const int n = t.n, k = t.k, r = n - k;
  if (r <= 0 || j0 >= r) return;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  double* K = a.scratch + t.scr_off;
  int* piv = reinterpret_cast<int*>(K + (int64_t)n * n) + 2 * n;
  double* Kr = K + k + (int64_t)k * n;
  auto kr = [&](int i, int j) -> double& { return Kr[i + (int64_t)j * n]; };
  const int jb = min(kHb, r - j0), j1 = j0 + jb;
  if (a.symm == 'p') {
    for (int j = j0; j < j1; ++j) {
      const double dj = kr(j, j);
      if (!(dj > 0.0)) {
        if (tid == 0) atomicOr(a.status, (int)ST_NOT_SPD);
        return;
      }
      const double lj = sqrt(dj);
      __syncthreads();
      for (int q = j + 1 + tid; q < r; q += kThreads) kr(q, j) /= lj;
      if (tid == 0) kr(j, j) = lj;
      __syncthreads();
      for (int q = j + 1 + tid; q < r; q += kThreads) {
        const double lq = kr(q, j);
        for (int c = j + 1; c < min(j1, q + 1); ++c) kr(q, c) -= lq * kr(c, j);
      }
      __syncthreads();
    }
    return;
  }
  for (int j = j0; j < j1; ++j) {
    AM am{-1.0, r};
    for (int q = j + tid; q < r; q += kThreads) am = amax(am, AM{fabs(kr(q, j)), q});
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      AM b{__shfl_xor_sync(0xffffffffu, am.v, o), __shfl_xor_sync(0xffffffffu, am.i, o)};
      am = amax(am, b);
    }
    if (lane == 0) red[wid] = am;
    __syncthreads();
    if (tid == 0) {
      AM bm = red[0];
      for (int w = 1; w < kWarps; ++w) bm = amax(bm, red[w]);
      const int pv0 = (bm.i >= j && bm.i < r) ? bm.i : j;
      s_piv = pv0;
      piv[j] = pv0;
    }
    __syncthreads();
    const int pv = s_piv;
    if (pv != j && tid < jb) {
      const double x = kr(j, j0 + tid);
      kr(j, j0 + tid) = kr(pv, j0 + tid);
      kr(pv, j0 + tid) = x;
    }
    __syncthreads();
    const double dj = kr(j, j);
    if (dj == 0.0 && tid == 0) atomicOr(a.status, (int)ST_SINGULAR);
    // scale column j and update the rest of the panel row by row
    for (int q = j + 1 + tid; q < r; q += kThreads) {
      const double lq = dj != 0.0 ? kr(q, j) / dj : kr(q, j);
      kr(q, j) = lq;
      for (int c = j + 1; c < j1; ++c) kr(q, c) -= lq * kr(j, c);
    }
    __syncthreads();
  }
}

// The same LU panel spread over P CTAs per box (one cooperative launch, so every CTA is
// resident): CTA `part` owns a contiguous block of the panel's rows.  Per column: local
// pivot search, box barrier, the first CTA swaps the two rows inside the panel and records
// the pivot, box barrier, every CTA scales and updates its rows.  The barriers are bounded
// (2 s): on expiry the kernel flags the timeout status and returns.
struct PanelSync {
  unsigned count, gen;
};
struct PanelSlot {
  double v;
  int i, pad;
};
constexpr int kCoopThreads = 256;

__device__ __forceinline__ uint64_t el_globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ bool box_barrier(PanelSync* ps, int P, int32_t* status) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    s_ok = 1;
    volatile unsigned* vgen = &ps->gen;
    const unsigned g = *vgen;
    __threadfence();
    if (atomicAdd(&ps->count, 1u) == (unsigned)P - 1) {
      ps->count = 0;
      __threadfence();
      atomicAdd(&ps->gen, 1u);
    } else {
      const uint64_t t0 = el_globaltimer();
      while (*vgen == g) {
        if (el_globaltimer() - t0 > 2000000000ull) {
          atomicOr(status, (int)ST_TIMEOUT);
          s_ok = 0;
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return s_ok != 0;
}

__global__ void __launch_bounds__(kCoopThreads) k_hb_panel_coop(ElimArgs a, int j0, int P, PanelSync* sync,
                                                                PanelSlot* slots) {
  constexpr int kW = kCoopThreads / 32;
  __shared__ AM red[kW];
  const int bx = blockIdx.x / P, part = blockIdx.x % P;
  const ElimTask t = a.tasks[bx];
  const int n = t.n, k = t.k, r = n - k;
  if (r <= 0 || j0 >= r) return;   // uniform over the box's CTAs
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  double* K = a.scratch + t.scr_off;
  int* piv = reinterpret_cast<int*>(K + (int64_t)n * n) + 2 * n;
  double* Kr = K + k + (int64_t)k * n;
  auto kr = [&](int i, int j) -> double& { return Kr[i + (int64_t)j * n]; };
  // other CTAs write the panel (the row swap, their rows): read it past L1
  auto ld = [&](int i, int j) { return __ldcg(&Kr[i + (int64_t)j * n]); };
  const int jb = min(kHb, r - j0), j1 = j0 + jb;
  const int rb = j0 + (int)((int64_t)(r - j0) * part / P), re = j0 + (int)((int64_t)(r - j0) * (part + 1) / P);
  PanelSync* ps = sync + bx;
  PanelSlot* sl = slots + (int64_t)bx * P;
  for (int j = j0; j < j1; ++j) {
    AM am{-1.0, r};
    for (int q = max(j, rb) + tid; q < re; q += kCoopThreads) am = amax(am, AM{fabs(ld(q, j)), q});
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      AM bb{__shfl_xor_sync(0xffffffffu, am.v, o), __shfl_xor_sync(0xffffffffu, am.i, o)};
      am = amax(am, bb);
    }
    if (lane == 0) red[wid] = am;
    __syncthreads();
    if (tid == 0) {
      AM bm = red[0];
      for (int w = 1; w < kW; ++w) bm = amax(bm, red[w]);
      sl[part] = PanelSlot{bm.v, bm.i, 0};
    }
    if (!box_barrier(ps, P, a.status)) return;
    AM bm{-1.0, r};
    for (int p = 0; p < P; ++p) {
      volatile PanelSlot* vp = sl + p;   // written by other CTAs before the barrier
      bm = amax(bm, AM{vp->v, vp->i});
    }
    const int pv = (bm.i >= j && bm.i < r) ? bm.i : j;
    if (part == 0) {
      if (pv != j && tid < jb) {
        const double x = ld(j, j0 + tid);
        kr(j, j0 + tid) = ld(pv, j0 + tid);
        kr(pv, j0 + tid) = x;
      }
      if (tid == 0) piv[j] = pv;
    }
    if (!box_barrier(ps, P, a.status)) return;
    const double dj = ld(j, j);
    if (dj == 0.0 && part == 0 && tid == 0) atomicOr(a.status, (int)ST_SINGULAR);
    for (int q = max(j + 1, rb) + tid; q < re; q += kCoopThreads) {
      const double lq = dj != 0.0 ? ld(q, j) / dj : ld(q, j);
      kr(q, j) = lq;
      for (int c = j + 1; c < j1; ++c) kr(q, c) = ld(q, c) - lq * ld(j, c);
    }
  }
}

// The panel's row interchanges on every column of K(rd,:) outside the panel.
__global__ void __launch_bounds__(kThreads) k_hb_swap(ElimArgs a, int j0) {
  const ElimTask t = a.tasks[blockIdx.z];
  const int n = t.n, k = t.k, r = n - k;
  if (r <= 0 || j0 >= r) return;
  const int col = blockIdx.x * kThreads + threadIdx.x;
  const int j1 = min(j0 + kHb, r);
  if (col >= n || (col >= k + j0 && col < k + j1)) return;
  double* K = a.scratch + t.scr_off;
  const int* piv = reinterpret_cast<const int*>(K + (int64_t)n * n) + 2 * n;
  double* Kc = K + k + (int64_t)col * n;
  for (int j = j0; j < j1; ++j) {
    const int pv = piv[j];
    if (pv != j) {
      const double x = Kc[j];
      Kc[j] = Kc[pv];
      Kc[pv] = x;
    }
  }
}

// Triangular solves with the panel's diagonal block, one thread per vector:
// op 0: U12 = L11 \ A12 (columns j1.. of K(rd,rd)); op 1: E(:, j0:j1) /= U11 (rows of
// K(sk,rd)); op 2: G(j0:j1, :) = L11 \ G(j0:j1, :) (columns of K(rd,sk)).
__global__ void __launch_bounds__(128) k_hb_trsm(ElimArgs a, int j0, int op) {
  __shared__ double blk[kHb * (kHb + 1)];
  const ElimTask t = a.tasks[blockIdx.z];
  const int n = t.n, k = t.k, r = n - k;
  if (r <= 0 || j0 >= r || (op > 0 && k == 0)) return;
  const int jb = min(kHb, r - j0), j1 = j0 + jb;
  const int nvec = op == 0 ? r - j1 : k;
  const int v0 = blockIdx.x * 128;
  if (v0 >= nvec) return;
  double* K = a.scratch + t.scr_off;
  double* Kr = K + k + (int64_t)k * n;
  const bool chol = a.symm == 'p';
  for (int e = threadIdx.x; e < jb * jb; e += 128) {   // blk(i, c) = U(i, c) or L(i, c) of the diagonal block
    const int i = e % jb, c = e / jb;
    blk[i + c * (kHb + 1)] = (op == 1 && chol) ? Kr[(j0 + c) + (int64_t)(j0 + i) * n] : Kr[(j0 + i) + (int64_t)(j0 + c) * n];
  }
  __syncthreads();
  const int v = v0 + threadIdx.x;
  if (v >= nvec) return;
  double x[kHb];
  if (op == 1) {   // row v of E: x U11 = e
    double* C = K + (int64_t)k * n;
#pragma unroll
    for (int c = 0; c < kHb; ++c) {
      if (c < jb) {
        double s = C[v + (int64_t)(j0 + c) * n];
#pragma unroll
        for (int l = 0; l < c; ++l) s -= x[l] * blk[l + c * (kHb + 1)];
        x[c] = s / blk[c + c * (kHb + 1)];
      }
    }
#pragma unroll
    for (int c = 0; c < kHb; ++c)
      if (c < jb) C[v + (int64_t)(j0 + c) * n] = x[c];
    return;
  }
  double* col = op == 0 ? Kr + j0 + (int64_t)(j1 + v) * n : K + k + j0 + (int64_t)v * n;
#pragma unroll
  for (int i = 0; i < kHb; ++i) {
    if (i < jb) {
      double s = col[i];
#pragma unroll
      for (int l = 0; l < i; ++l) s -= blk[i + l * (kHb + 1)] * x[l];
      x[i] = s;
    }
  }
#pragma unroll
  for (int i = 0; i < kHb; ++i)
    if (i < jb) col[i] = x[i];
}

// Store the factor [T | LU (L) | E | G] and the LU row permutation.
__global__ void __launch_bounds__(kThreads) k_hb_store(ElimArgs a) {
  const ElimTask t = a.tasks[blockIdx.z];
  const int n = t.n, k = t.k, r = n - k;
  if (r <= 0) return;
  const bool chol = a.symm == 'p';
  double* K = a.scratch + t.scr_off;
  const double* T = a.tpool + t.T_off;
  double* F = a.fpool + t.fac_off;
  const int64_t kr_ = (int64_t)k * r, rr = (int64_t)r * r;
  const int64_t total = 2 * kr_ + rr + (chol ? 0 : kr_);
  for (int64_t e = blockIdx.x * (int64_t)kThreads + threadIdx.x; e < total; e += (int64_t)gridDim.x * kThreads) {
    double v;
    if (e < kr_) {
      v = T[e];
    } else if (e < kr_ + rr) {
      const int64_t q = e - kr_;
      const int i = (int)(q % r), j = (int)(q / r);
      v = (chol && i < j) ? 0.0 : K[(k + i) + (int64_t)(k + j) * n];
    } else if (e < 2 * kr_ + rr) {
      const int64_t q = e - kr_ - rr;
      const int i = (int)(q % k), j = (int)(q / k);
      v = K[i + (int64_t)(k + j) * n];
    } else {
      const int64_t q = e - 2 * kr_ - rr;
      const int i = (int)(q % r), j = (int)(q / r);
      v = K[(k + i) + (int64_t)j * n];
    }
    F[e] = v;
  }
  if (!chol && blockIdx.x == 0 && threadIdx.x == 0) {
    const int* piv = reinterpret_cast<const int*>(K + (int64_t)n * n) + 2 * n;
    int32_t* pp = a.ppool + t.piv_off;
    for (int q = 0; q < r; ++q) pp[q] = q;
    for (int q = 0; q < r; ++q) {
      const int32_t x = pp[q];
      pp[q] = pp[piv[q]];
      pp[piv[q]] = x;
    }
  }
}

}  // namespace

void launch_eliminate_huge(const ElimArgs& a, int nbox, int nmax, int kmax, int rmax, cudaStream_t s) {
  if (nbox <= 0 || rmax <= 0) return;
  const unsigned z = (unsigned)nbox;
  auto tiles = [](int x) { return (unsigned)std::max(1, (x + 63) / 64); };
  auto gemm = [&](int kind, int j0, int M, int N) {
    k_hb_gemm<<<dim3(tiles(M), tiles(N), z), 128, 0, s>>>(a, kind, j0);
  };
  k_hb_locate<<<nbox, kThreads, 0, s>>>(a);
  k_hb_assemble<<<dim3((nmax + 31) / 32, (nmax + 31) / 32, z), kThreads, 0, s>>>(a);
  if (kmax > 0) {
    gemm(HB_TROW, 0, rmax, nmax);
    gemm(HB_TCOL, 0, nmax, rmax);
  }
  const bool chol = a.symm == 'p';
  // LU panels over several CTAs per box when the redundant blocks are tall (one CTA
  // streams an r x 32 panel through its SM 32 times); all CTAs resident: one cooperative
  // launch of at most one CTA per SM
  int P = 1;
  PanelSync* psync = nullptr;
  PanelSlot* pslot = nullptr;
  if (!chol && rmax >= 1024) {
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    P = std::max(1, std::min(64, nsm / nbox));
    if (P > 1 && (cudaMallocAsync(&psync, sizeof(PanelSync) * nbox, s) != cudaSuccess ||
                  cudaMallocAsync(&pslot, sizeof(PanelSlot) * nbox * P, s) != cudaSuccess)) {
      cudaGetLastError();
      P = 1;
    }
    if (P > 1) cudaMemsetAsync(psync, 0, sizeof(PanelSync) * nbox, s);
  }
  for (int j0 = 0; j0 < rmax; j0 += kHb) {
    const int rest = rmax - std::min(rmax, j0 + kHb);
    bool done = false;
    if (P > 1) {
      ElimArgs ac = a;
      int jj = j0, pp = P;
      void* args[] = {&ac, &jj, &pp, &psync, &pslot};
      if (cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_hb_panel_coop), dim3((unsigned)(nbox * P)),
                                      dim3(kCoopThreads), args, 0, s) == cudaSuccess)
        done = true;
      else
        cudaGetLastError();   // not resident together: the one-CTA panel
    }
    if (!done) k_hb_panel<<<nbox, kPanelThreads, 0, s>>>(a, j0);
    if (!chol) {
      k_hb_swap<<<dim3((nmax + kThreads - 1) / kThreads, 1, z), kThreads, 0, s>>>(a, j0);
      if (rest > 0) k_hb_trsm<<<dim3((rest + 127) / 128, 1, z), 128, 0, s>>>(a, j0, 0);
    }
    if (rest > 0) gemm(chol ? HB_TRAIL_CHOL : HB_TRAIL, j0, rest, rest);
  }
  if (kmax > 0) {
    for (int j0 = 0; j0 < rmax; j0 += kHb) {
      const int rest = rmax - std::min(rmax, j0 + kHb);
      k_hb_trsm<<<dim3((kmax + 127) / 128, 1, z), 128, 0, s>>>(a, j0, 1);
      if (rest > 0) gemm(HB_EUPD, j0, kmax, rest);
      if (!chol) {
        k_hb_trsm<<<dim3((kmax + 127) / 128, 1, z), 128, 0, s>>>(a, j0, 2);
        if (rest > 0) gemm(HB_GUPD, j0, rest, kmax);
      }
    }
    gemm(HB_SCHUR, 0, kmax, kmax);
  }
  if (psync) cudaFreeAsync(psync, s);
  if (pslot) cudaFreeAsync(pslot, s);
  const int64_t tot = 4 * (int64_t)std::max(kmax, 1) * rmax + (int64_t)rmax * rmax;
  k_hb_store<<<dim3((unsigned)std::min<int64_t>((tot + kThreads - 1) / kThreads, 4096), 1, z), kThreads, 0, s>>>(a);
}

int sweep_root_grid(double* W, int nrhs, const int64_t* rd, const int32_t* perm, const double* LU, int r, int op,
                    int trans, int symm, double* X, cudaStream_t s) {
  // k = 0: only the triangular factors act (rskelf_sv_*.m with empty sk)
  const bool lu = symm != 'p';
  const bool gather_p = lu && op == 0 && trans == 0;
  const bool scatter_p = lu && op == 1 && trans == 1;
  GV M;
  bool lower, unit;
  if (op == 0) {          // forward: L \ x ('n', or chol), U' \ x ('t')
    M = (lu && trans) ? GV{LU, (int64_t)r, 1} : GV{LU, 1, (int64_t)r};
    lower = true;
    unit = lu && !trans;
  } else {                // backward: U \ x ('n'), L' \ x (chol, or 't' unit)
    M = (lu && !trans) ? GV{LU, 1, (int64_t)r} : GV{LU, (int64_t)r, 1};
    lower = false;
    unit = lu && trans;
  }
  int launches = 0;
  const unsigned gblk = (unsigned)std::min<int64_t>(((int64_t)r * nrhs + 255) / 256, 148 * 8);
  k_rows_gs<<<gblk, 256, 0, s>>>(W, nrhs, rd, gather_p ? perm : nullptr, r, X, 0);
  ++launches;
  const unsigned cb = (unsigned)((nrhs + 255) / 256);
  auto tiles = [](int x) { return (unsigned)std::max(1, (x + 63) / 64); };
  if (lower) {
    for (int j0 = 0; j0 < r; j0 += kHb) {
      const int jb = std::min(kHb, r - j0), j1 = j0 + jb;
      k_trsm_diag<<<cb, 256, 0, s>>>(M, X, r, nrhs, j0, jb, 1, unit ? 1 : 0);
      ++launches;
      if (j1 < r) {
        HbOp o{X + j1, 1, (int64_t)r, GV{M.p + j1 * M.rs + j0 * M.cs, M.rs, M.cs}, GV{X + j0, 1, (int64_t)r},
               r - j1, nrhs, jb};
        k_dgemm_op<<<dim3(tiles(r - j1), tiles(nrhs)), 128, 0, s>>>(o);
        ++launches;
      }
    }
  } else {
    for (int j1 = r; j1 > 0;) {
      const int j0 = std::max(0, j1 - kHb), jb = j1 - j0;
      k_trsm_diag<<<cb, 256, 0, s>>>(M, X, r, nrhs, j0, jb, 0, unit ? 1 : 0);
      ++launches;
      if (j0 > 0) {
        HbOp o{X, 1, (int64_t)r, GV{M.p + j0 * M.cs, M.rs, M.cs}, GV{X + j0, 1, (int64_t)r}, j0, nrhs, jb};
        k_dgemm_op<<<dim3(tiles(j0), tiles(nrhs)), 128, 0, s>>>(o);
        ++launches;
      }
      j1 = j0;
    }
  }
  k_rows_gs<<<gblk, 256, 0, s>>>(W, nrhs, rd, scatter_p ? perm : nullptr, r, X, 1);
  return launches + 1;
}

int elim_huge_launches(int rmax, int kmax, bool chol) {
  const int np = (rmax + kHb - 1) / kHb;
  return 3 + (kmax > 0 ? 2 : 0) + np * (chol ? 2 : 4) + (kmax > 0 ? np * (chol ? 2 : 4) + 1 : 0);
}

size_t elim_smem_bytes(int n) {
  if (n > kSmemN) return sizeof(int) * 3 * (size_t)n + 64;
  return sizeof(double) * (size_t)n * n + sizeof(int) * 3 * (size_t)n + 64;
}

int64_t elim_scratch_doubles(int n) { return (int64_t)n * n + (3 * (int64_t)n) / 2 + 2; }

void launch_eliminate(const ElimArgs& a, int nsmall, int nbig, size_t smem, cudaStream_t s) {
  if (ensure_smem_attr(reinterpret_cast<const void*>(k_eliminate), 200 * 1024) != cudaSuccess ||
      ensure_smem_attr(reinterpret_cast<const void*>(k_eliminate_big), kBigPanBytes) != cudaSuccess)
    return;
  if (nsmall > 0) k_eliminate<<<nsmall, kThreads, smem, s>>>(a);
  if (nbig > 0) {
    ElimArgs b = a;
    b.tasks = a.tasks + nsmall;
    b.pan_rows = std::min(std::max(b.pan_rows, 0), elim_pan_rows_max());
    k_eliminate_big<<<nbig, kThreads, sizeof(double) * (size_t)b.pan_rows * kNb, s>>>(b);
  }
}

// Rows of the largest LU panel k_eliminate_big stages in shared memory (kBigPanBytes of kNb
// columns); the kernel holds all 65,536 registers of an SM, so the shared memory costs no
// occupancy.
int elim_pan_rows_max() { return kBigPanBytes / (int)(sizeof(double) * kNb); }

}  // namespace flam
