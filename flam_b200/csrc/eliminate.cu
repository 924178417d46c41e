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
#include "common.cuh"
#include "kernels.cuh"

namespace flam {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

struct AM {
  double v;
  int i;
};
__device__ __forceinline__ AM amax(AM a, AM b) {
  if (b.v > a.v || (b.v == a.v && b.i < a.i)) return b;
  return a;
}

__global__ void __launch_bounds__(kThreads) k_eliminate(ElimArgs a) {
  extern __shared__ __align__(16) double smem[];
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

  for (int q = tid; q < n; q += kThreads) {
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

  auto mval = [&](int i, int j) -> double {
    const int c = pchild[i];
    if (c < 0 || c != pchild[j]) return 0.0;
    const int kc = ch[c].kc;
    return a.m_in[ch[c].M_off + ploc[i] + (int64_t)ploc[j] * kc];
  };

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
    // K(rd,:) = K(rd,:) - T' K(sk,:)      (T.' for 's': identical for real data)
    for (int col = tcol; col < n; col += kWarps) {
      const double* Kc = K + (int64_t)col * n;
      for (int i = tr; i < r; i += 32) {
        const double* Ti = T + (int64_t)i * k;
        double s0 = 0.0, s1 = 0.0;
        int b = 0;
        for (; b + 1 < k; b += 2) {
          s0 += Ti[b] * Kc[b];
          s1 += Ti[b + 1] * Kc[b + 1];
        }
        if (b < k) s0 += Ti[b] * Kc[b];
        K[k + i + (int64_t)col * n] -= s0 + s1;
      }
    }
    __syncthreads();
    // K(:,rd) = K(:,rd) - K(:,sk) T
    for (int j = tcol; j < r; j += kWarps) {
      const double* Tj = T + (int64_t)j * k;
      for (int row = tr; row < n; row += 32) {
        double s0 = 0.0, s1 = 0.0;
        int b = 0;
        for (; b + 1 < k; b += 2) {
          s0 += K[row + (int64_t)b * n] * Tj[b];
          s1 += K[row + (int64_t)(b + 1) * n] * Tj[b + 1];
        }
        if (b < k) s0 += K[row + (int64_t)b * n] * Tj[b];
        K[row + (int64_t)(k + j) * n] -= s0 + s1;
      }
    }
    __syncthreads();
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

}  // namespace

size_t elim_smem_bytes(int n) {
  if (n > kSmemN) return sizeof(int) * 3 * (size_t)n + 64;
  return sizeof(double) * (size_t)n * n + sizeof(int) * 3 * (size_t)n + 64;
}

int64_t elim_scratch_doubles(int n) { return (int64_t)n * n + (3 * (int64_t)n) / 2 + 2; }

void launch_eliminate(const ElimArgs& a, int ntask, size_t smem, cudaStream_t s) {
  if (ntask <= 0) return;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_eliminate, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  k_eliminate<<<ntask, kThreads, smem, s>>>(a);
}

}  // namespace flam
