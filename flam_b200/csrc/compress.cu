// K4+K5+K6: fused proxy filter, block assembly and interpolative decomposition,
// one CTA per box of a factorization step.
//
// Reference path (rskelf/rskelf.m:201-213, core/id.m:59-240):
//   nbr  = nbr(inside proxy surface)                 pxyfun's filter
//   K    = [A(nbr,slf); A(slf,nbr)'; Kpxy]            m x n
//   [~,R,p] = qr(K,0)                                xGEQP3 (column pivoting)
//   k    = nnz(|diag R| > tol |R11|), T = R11\R12
//   RRQR swaps until max|T| <= Tmax
//
// Device design: K is never written to memory.  Its rows are generated 32 at
// a time (one per lane) straight from the point coordinates and folded into an
// n x n triangular factor R0 with Householder reflections (TSQR), so the only
// per-box state is R0 (shared memory for n <= kSmemN).  The column-pivoted QR
// then runs on R0: K = Q0 R0 with orthogonal Q0, so every column norm the
// pivot rule reads -- and therefore every pivot, the rank and T -- is that of
// the reference's QR of K, up to rounding.  The pivoted QR follows LAPACK's
// xLAQP2 (first maximum of the partial column norms, norm downdating with the
// sqrt(eps) recomputation threshold) for min(m, n) steps.
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"
#include "rrqr.cuh"

namespace flam {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

struct ArgMax {
  double v;
  int i;
};

__device__ __forceinline__ ArgMax better(ArgMax a, ArgMax b) {
  // larger value wins; ties go to the lower index (IDAMAX returns the first maximum)
  if (b.v > a.v || (b.v == a.v && b.i < a.i)) return b;
  return a;
}

__device__ ArgMax block_argmax(ArgMax a, ArgMax* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ArgMax b;
    b.v = __shfl_xor_sync(0xffffffffu, a.v, o);
    b.i = __shfl_xor_sync(0xffffffffu, a.i, o);
    a = better(a, b);
  }
  if (lane == 0) red[wid] = a;
  __syncthreads();
  ArgMax r = red[0];
  for (int w = 1; w < kWarps; ++w) r = better(r, red[w]);
  __syncthreads();
  return r;
}

__device__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double r = 0.0;
  for (int w = 0; w < kWarps; ++w) r += red[w];
  __syncthreads();
  return r;
}

// Value of row `rho` (0-based) of K at column c, for the row descriptor a lane holds.
struct RowDesc {
  int type;        // 0: A(nbr,slf)  1: A(slf,nbr)'  2: proxy  3: zero
  int64_t q;       // neighbour point id (types 0, 1)
  double y[kMaxDim];  // proxy point (type 2)
  double wmul;     // proxy multiplier for types 2 (wbar for the second half, 0 = use w_slf)
};

__device__ __forceinline__ double row_entry(const Problem& P, const InstParams& ip, const RowDesc& rd,
                                            int64_t sc) {
  const int d = P.d;
  switch (rd.type) {
    case 0:
      return aentry(P, ip, rd.q, sc);
    case 1:
      return aentry(P, ip, sc, rd.q);
    case 2: {
      double v = ip.pscale * keval(ip.pkernel, ip.pparam, d, rd.y, P.x + sc * d, nullptr);
      if (rd.wmul != 0.0) return v * rd.wmul;
      return ip.has_w ? v * P.w[sc] : v;
    }
    default:
      return 0.0;
  }
}

__global__ void __launch_bounds__(kThreads) k_compress(CompressArgs a) {
  extern __shared__ __align__(16) double smem[];
  __shared__ ArgMax red_am[kWarps];
  __shared__ double red_d[kWarps];
  __shared__ int s_cnt[kWarps];
  __shared__ double s_tau;
  __shared__ double s_tau2[2];
  __shared__ int s_m1, s_k, s_ktol, s_niter, s_cap, s_conv;

  const CompressTask t = a.tasks[blockIdx.x];
  const Problem& P = a.P;
  const InstParams ip = P.ip[t.inst];
  const int n = t.n;
  const int d = P.d;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  CompressOut* out = a.out + t.out_idx;
  int64_t* slf = a.ipool + t.slf_off;
  int64_t* cand = a.cpool + t.cand_off;
  if (n == 0) {
    if (tid == 0) *out = CompressOut{0, 0, 0, 0};
    return;
  }

  // ---- work arrays: shared memory for small boxes, global scratch otherwise
  double* base = (t.scr_off >= 0) ? a.scratch + t.scr_off : smem;
  double* R = base;                                 // n x n, ld n
  double* Pn = R + (int64_t)n * n;                  // 32 x n panel, column-major ld 32
  double* vn1 = Pn + (int64_t)32 * n;
  double* vn2 = vn1 + n;
  int* jpvt = reinterpret_cast<int*>(vn2 + n);      // n ints (n/2+1 doubles)

  // ---- (1) neighbour filter (pxyfun's nbr selection), stable compaction in place
  if (tid == 0) s_m1 = 0;
  __syncthreads();
  int m1 = t.ncand;
  if (t.flags & 2) {
    int total = 0;
    for (int c0 = 0; c0 < t.ncand; c0 += kThreads) {
      const int ci = c0 + tid;
      int64_t q = -1;
      bool keep = false;
      if (ci < t.ncand) {
        q = cand[ci];
        const double* xq = P.x + q * d;
        if (ip.pkind == P_ANNULUS) {
          double mx = 0.0;
          for (int k = 0; k < d; ++k) mx = fmax(mx, __ddiv_rn(fabs(__dsub_rn(xq[k], t.ctr[k])), t.l[k]));
          keep = mx < 1.5;
        } else {
          double s = 0.0;
          for (int k = 0; k < d; ++k) {
            const double z = __ddiv_rn(__dsub_rn(xq[k], t.ctr[k]), t.l[k]);
            s = __dadd_rn(s, __dmul_rn(z, z));
          }
          keep = s < 2.25;
        }
      }
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      if (lane == 0) s_cnt[wid] = __popc(bal);
      __syncthreads();
      int pre = total;
      for (int w = 0; w < wid; ++w) pre += s_cnt[w];
      int tot = 0;
      for (int w = 0; w < kWarps; ++w) tot += s_cnt[w];
      if (keep) cand[pre + __popc(bal & ((1u << lane) - 1u))] = q;
      total += tot;
      __syncthreads();
    }
    m1 = total;
  }
  const int nrep = a.symm_n ? 2 : 1;
  const int npr = (t.flags & 1) ? (ip.two_sided ? 2 * P.npxy : P.npxy) : 0;
  const int m = a.Aexp ? t.ncand : nrep * m1 + npr;
  const int mn = min(m, n);

  // ---- (2) TSQR: fold row panels of K into R0 (n x n upper triangular)
  for (int64_t e = tid; e < (int64_t)n * n; e += kThreads) R[e] = 0.0;
  __syncthreads();
  for (int p0 = 0; p0 < m; p0 += 32) {
    RowDesc rd;
    const int rho = p0 + lane;
    rd.type = 3;
    rd.q = -1;
    rd.wmul = 0.0;
    if (a.Aexp) {
      // explicit matrix: rows read below
    } else if (rho < m1) {
      rd.type = 0;
      rd.q = cand[rho];
    } else if (a.symm_n && rho < 2 * m1) {
      rd.type = 1;
      rd.q = cand[rho - m1];
    } else if (rho < m) {
      int pr = rho - nrep * m1;
      rd.type = 2;
      if (ip.two_sided && pr >= P.npxy) {
        pr -= P.npxy;
        rd.wmul = ip.wbar;
      }
      for (int k = 0; k < d; ++k) {
        const double pk = P.pxy_pts[pr * d + k];
        rd.y[k] = P.pxy_shift ? pk + P.pxy_shift[pr * d + k] * t.l[k] + t.ctr[k] : pk * t.l[k] + t.ctr[k];
      }
    }
    if (a.Aexp) {
      for (int c = wid; c < n; c += kWarps) Pn[(int64_t)c * 32 + lane] = rho < m ? a.Aexp[rho + c * a.lda] : 0.0;
    } else {
      for (int c = wid; c < n; c += kWarps) Pn[(int64_t)c * 32 + lane] = row_entry(P, ip, rd, slf[c]);
    }
    __syncthreads();
    for (int j = 0; j < n; ++j) {
      if (wid == 0) {
        const double pj = Pn[(int64_t)j * 32 + lane];
        const double sig = warp_sum(pj * pj);
        double tau = 0.0;
        if (sig != 0.0) {
          const double al = R[j + (int64_t)j * n];
          const double be = -copysign(sqrt(al * al + sig), al);
          tau = (be - al) / be;
          Pn[(int64_t)j * 32 + lane] = pj / (al - be);
          if (lane == 0) R[j + (int64_t)j * n] = be;
        }
        if (lane == 0) s_tau2[j & 1] = tau;
      }
      __syncthreads();
      // double-buffered: a warp still reading step j's tau cannot see step j+1's
      const double tau = s_tau2[j & 1];
      if (tau != 0.0) {
        const double vl = Pn[(int64_t)j * 32 + lane];
        for (int c = j + 1 + wid; c < n; c += kWarps) {
          const double pc = Pn[(int64_t)c * 32 + lane];
          const double w = R[j + (int64_t)c * n] + warp_sum(vl * pc);
          const double tw = tau * w;
          Pn[(int64_t)c * 32 + lane] = pc - tw * vl;
          if (lane == 0) R[j + (int64_t)c * n] -= tw;
        }
        __syncthreads();
      }
    }
  }

  // ---- (3) column-pivoted QR of R0 (xLAQP2 semantics) for min(m, n) steps
  for (int c = wid; c < n; c += kWarps) {
    double s = 0.0;
    for (int row = lane; row < n; row += 32) s += R[row + (int64_t)c * n] * R[row + (int64_t)c * n];
    s = sqrt(warp_sum(s));
    if (lane == 0) {
      vn1[c] = s;
      vn2[c] = s;
    }
  }
  for (int c = tid; c < n; c += kThreads) jpvt[c] = c;
  __syncthreads();
  const double tol3z = 1.0536712127723509e-08;  // sqrt(2^-53), LAPACK's dlamch('Epsilon')
  for (int i = 0; i < mn; ++i) {
    ArgMax am{-1.0, n};
    for (int c = i + tid; c < n; c += kThreads) am = better(am, ArgMax{vn1[c], c});
    am = block_argmax(am, red_am);
    // a NaN partial norm (non-finite input) leaves the sentinel index: stay in range
    const int pvt = (am.i >= i && am.i < n) ? am.i : i;
    if (pvt != i) {
      for (int row = tid; row < n; row += kThreads) {
        const double tmp = R[row + (int64_t)pvt * n];
        R[row + (int64_t)pvt * n] = R[row + (int64_t)i * n];
        R[row + (int64_t)i * n] = tmp;
      }
      if (tid == 0) {
        const int tj = jpvt[pvt];
        jpvt[pvt] = jpvt[i];
        jpvt[i] = tj;
        vn1[pvt] = vn1[i];
        vn2[pvt] = vn2[i];
      }
    }
    __syncthreads();
    if (wid == 0) {  // DLARFG on R[i:m, i]
      double s = 0.0;
      if (i + 1 < m)
        for (int row = i + 1 + lane; row < n; row += 32) s += R[row + (int64_t)i * n] * R[row + (int64_t)i * n];
      s = warp_sum(s);
      double tau = 0.0;
      if (s != 0.0) {
        const double xn = sqrt(s);
        const double al = R[i + (int64_t)i * n];
        const double be = -copysign(hypot(al, xn), al);
        tau = (be - al) / be;
        const double sc = 1.0 / (al - be);
        for (int row = i + 1 + lane; row < n; row += 32) R[row + (int64_t)i * n] *= sc;
        __syncwarp();
        if (lane == 0) R[i + (int64_t)i * n] = be;
      }
      if (lane == 0) s_tau = tau;
    }
    __syncthreads();
    const double tau = s_tau;
    if (tau != 0.0) {
      for (int c = i + 1 + wid; c < n; c += kWarps) {
        double s = 0.0;
        for (int row = i + 1 + lane; row < n; row += 32) s += R[row + (int64_t)i * n] * R[row + (int64_t)c * n];
        const double w = R[i + (int64_t)c * n] + warp_sum(s);
        const double tw = tau * w;
        for (int row = i + 1 + lane; row < n; row += 32) R[row + (int64_t)c * n] -= tw * R[row + (int64_t)i * n];
        if (lane == 0) R[i + (int64_t)c * n] -= tw;
      }
    }
    __syncthreads();
    for (int c = i + 1 + tid; c < n; c += kThreads) {  // partial norm downdate
      if (vn1[c] != 0.0) {
        double temp = fabs(R[i + (int64_t)c * n]) / vn1[c];
        temp = 1.0 - temp * temp;
        temp = fmax(temp, 0.0);
        const double q = vn1[c] / vn2[c];
        const double temp2 = temp * q * q;
        if (temp2 <= tol3z) {
          if (i + 1 < m) {
            double s = 0.0;
            for (int row = i + 1; row < n; ++row) s += R[row + (int64_t)c * n] * R[row + (int64_t)c * n];
            vn1[c] = sqrt(s);
            vn2[c] = vn1[c];
          } else {
            vn1[c] = 0.0;
            vn2[c] = 0.0;
          }
        } else {
          vn1[c] *= sqrt(temp);
        }
      }
    }
    __syncthreads();
  }

  // The reflectors are stored below the diagonal (as xGEQP3 does); the RRQR
  // update reads R as the reference's upper-trapezoidal matrix, so clear them.
  for (int64_t e = tid; e < (int64_t)n * n; e += kThreads) {
    const int row = (int)(e % n), col = (int)(e / n);
    if (row > col) R[e] = 0.0;
  }
  __syncthreads();

  // ---- (4) rank by precision and by the rank cap (id.m:106-113)
  if (tid == 0) {
    const double tol = a.rel_tol * fabs(R[0]);
    int kt = 0;
    if (m > 0)
      for (int i = 0; i < mn; ++i) kt += fabs(R[i + (int64_t)i * n]) > tol;
    int kmax = a.kmax;
    if (kmax == 0 || kmax > n) kmax = n;
    s_ktol = kt;
    s_k = min(kt, kmax);
    s_niter = 0;
    s_cap = 0;
    s_conv = 1;
  }
  __syncthreads();
  int k = s_k;
  const int ktol = s_ktol;

  // ---- (5) T = R11 \ R12 (id.m:114), one column per thread
  if (k > 0 && k < n && m > 0) {
    for (int c = k + tid; c < n; c += kThreads) {
      for (int i = k - 1; i >= 0; --i) {
        double v = R[i + (int64_t)c * n];
        for (int j = i + 1; j < k; ++j) v -= R[i + (int64_t)j * n] * R[j + (int64_t)c * n];
        R[i + (int64_t)c * n] = v / R[i + (int64_t)i * n];
      }
    }
  }
  __syncthreads();

  // ---- (6) RRQR refinement (id.m:117-236)
  if (m > 0 && !isinf(a.Tmax) && a.rrqr_iter != 0 && k > 0 && k < n) {
    bool need = ktol > k;
    if (!need) {
      double mx = 0.0;
      for (int64_t e = tid; e < (int64_t)k * (n - k); e += kThreads) {
        const int i = (int)(e % k), c = k + (int)(e / k);
        const double v = R[i + (int64_t)c * n];
        mx = fmax(mx, v * v);
      }
      for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (lane == 0) red_d[wid] = mx;
      __syncthreads();
      double bm = 0.0;
      for (int w = 0; w < kWarps; ++w) bm = fmax(bm, red_d[w]);
      need = bm > a.Tmax * a.Tmax;
      __syncthreads();
    }
    if (need) {
      if (tid == 0) {
        int niter = 0, capped = 0;
        const double tol = a.rel_tol * fabs(R[0]);
        // aux scratch: the panel region is free after the TSQR (32 n doubles)
        const int kk = rrqr_serial(R, 1, n, n, k, ktol, jpvt, tol, a.Tmax, a.rrqr_iter, Pn, &niter, &capped);
        s_k = kk;
        s_niter = niter;
        s_cap = capped;
      }
      __syncthreads();
      k = s_k;
    }
  }

  // ---- (7) outputs: [sk rd] order of slf, local permutation, T
  const int r = n - k;
  int* perm_out = a.permpool + t.perm_off;
  const bool keep_order = (r == 0) || (m == 0);   // rskelf.m:216 (no factor) / id.m:64-68 (empty block)
  int64_t* tmp_ids = reinterpret_cast<int64_t*>(Pn);  // panel region reused (n int64 <= 32 n doubles)
  for (int c = tid; c < n; c += kThreads) tmp_ids[c] = slf[c];
  __syncthreads();
  for (int c = tid; c < n; c += kThreads) {
    const int src = keep_order ? c : jpvt[c];
    perm_out[c] = src;
    slf[c] = tmp_ids[src];
  }
  if (r > 0 && k > 0) {
    double* T = a.tpool + t.T_off;
    for (int64_t e = tid; e < (int64_t)k * r; e += kThreads) {
      const int i = (int)(e % k), j = (int)(e / k);
      T[e] = R[i + (int64_t)(k + j) * n];
    }
  }
  if (tid == 0) *out = CompressOut{k, m, s_niter, s_cap ? (int)ST_RRQR_CAP : 0};
}

}  // namespace

size_t compress_smem_bytes(int n) {
  if (n > kSmemN) return 0;
  return sizeof(double) * ((size_t)n * n + 32 * (size_t)n + 2 * (size_t)n + (size_t)n / 2 + 1);
}

int64_t compress_scratch_doubles(int n) {
  return (int64_t)n * n + 32 * (int64_t)n + 2 * (int64_t)n + n / 2 + 1;
}

void launch_compress(const CompressArgs& a, int ntask, size_t smem, cudaStream_t s) {
  if (ntask <= 0) return;
  if (ensure_smem_attr(reinterpret_cast<const void*>(k_compress), 200 * 1024) != cudaSuccess) return;
  k_compress<<<ntask, kThreads, smem, s>>>(a);
}

}  // namespace flam
