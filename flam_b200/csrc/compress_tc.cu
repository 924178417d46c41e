// K4+K5+K6, thread-per-column form: fused proxy filter, block assembly and
// interpolative decomposition, one CTA per box, one thread per column of the
// box's block K = [A(nbr,slf); A(slf,nbr)'; Kpxy] (rskelf/rskelf.m:201-213,
// core/id.m:59-240).
//
// TSQR.  Rows of K are generated B at a time; thread c keeps its column's B
// panel entries in registers and R (n x n, upper triangular, row-major) lives
// in shared memory (global scratch for large n).  Reflector j annihilates the
// panel's column j into R(j,j); the thread owning column j+1 applies
// reflector j to its column and immediately forms reflector j+1, so each
// reflector costs one barrier and every other thread's work is a register
// dot product and update with the reflector broadcast from shared memory.
//
// Pivoted QR of R0 (xLAQP2 rule: first maximum of the partial column norms,
// sqrt(eps) downdating threshold, min(m, n) steps), then rank, T = R11\R12 and
// the RRQR refinement (rrqr.cuh) exactly as the per-column kernel in
// compress.cu, whose results this kernel reproduces up to rounding.
#include <algorithm>
#include <cmath>
#include <cstdlib>

#include "common.cuh"
#include "kernels.cuh"
#include "rrqr.cuh"

namespace flam {
namespace {

struct AMx {
  double v;
  int i;
};

__device__ __forceinline__ AMx amx_better(AMx a, AMx b) {
  if (b.v > a.v || (b.v == a.v && b.i < a.i)) return b;  // first maximum, like IDAMAX
  return a;
}

template <int B>
struct Stage {
  double y[B][kMaxDim];  // proxy point of a proxy row
  double wmul[B];        // proxy multiplier (0: use the column's weight)
  int64_t q[B];          // neighbour point of an A(nbr,slf) / A(slf,nbr)' row
  int type[B];           // 0 A(nbr,slf), 1 A(slf,nbr)', 2 proxy, 3 zero
};

// Sum over the G consecutive lanes that share a column (G divides 32).
template <int G>
__device__ __forceinline__ double group_sum(double v, unsigned gmask) {
#pragma unroll
  for (int o = 1; o < G; o <<= 1) v += __shfl_xor_sync(gmask, v, o);
  return v;
}

// Reflector j of the current panel, formed by the G threads that own column j
// (thread g holds panel rows g*B .. g*B+B-1): annihilates the panel's column j
// into R(j,j) (DLARFG conventions).
template <int B, int G, int VS>
__device__ __forceinline__ void reflect_col(double (&p)[B], double al, double* R, int ld, int j, int g,
                                            unsigned gmask, double* vb, double* tau_out) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;   // four chains: this sum is on the critical path
#pragma unroll
  for (int i = 0; i < B; i += 4) {
    s0 += p[i] * p[i];
    s1 += p[i + 1] * p[i + 1];
    s2 += p[i + 2] * p[i + 2];
    s3 += p[i + 3] * p[i + 3];
  }
  const double sig = group_sum<G>((s0 + s1) + (s2 + s3), gmask);
  double tau = 0.0;
  if (sig != 0.0) {
    const double be = -copysign(sqrt(al * al + sig), al);
    tau = (be - al) / be;
    const double scal = 1.0 / (al - be);
#pragma unroll
    for (int i = 0; i < B; ++i) vb[g * VS + i] = p[i] * scal;
    __syncwarp(gmask);
    if (g == 0) R[(int64_t)j * ld + j] = be;
  }
  if (g == 0) *tau_out = tau;
}

// pxyfun's neighbour selection (the reference test drivers' filters): stable
// compaction of the box's candidate list in place; returns the kept count.
__device__ __forceinline__ int filter_candidates(const CompressTask& t, const Problem& P, const InstParams& ip,
                                                 int64_t* cand, int* s_cnt) {
  const int NT = blockDim.x, nw = NT >> 5, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int d = P.d;
  int total = 0;
  for (int c0 = 0; c0 < t.ncand; c0 += NT) {
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
    int pre = total, tot = 0;
    for (int w = 0; w < nw; ++w) {
      if (w < wid) pre += s_cnt[w];
      tot += s_cnt[w];
    }
    if (keep) cand[pre + __popc(bal & ((1u << lane) - 1u))] = q;
    total += tot;
    __syncthreads();
  }
  return total;
}

__global__ void __launch_bounds__(256) k_filter(CompressArgs a) {
  __shared__ int s_cnt[8];
  const CompressTask t = a.tasks[blockIdx.x];
  const InstParams ip = a.P.ip[t.inst];
  const int m1 = (t.flags & 2) ? filter_candidates(t, a.P, ip, a.cpool + t.cand_off, s_cnt) : t.ncand;
  if (threadIdx.x == 0) a.mfilt[t.out_idx] = m1;
}

template <int B, int G>
__global__ void __launch_bounds__(B == 64 ? 256 : (B == 32 ? 512 : 1024)) k_compress_tc(CompressArgs a) {
  constexpr int PH = B * G;  // panel height
  // loads in flight per thread in the pivoted QR's column passes (64 measured slower in
  // the 64-row shape: it spills at 255 registers)
  constexpr int LD = 32;
  extern __shared__ __align__(16) double smem[];
  __shared__ Stage<PH> st;
  // reflector of the row folding; lane g of a column reads its B entries at g * VS, so
  // the G lanes of a column start on different banks
  constexpr int VS = G == 1 ? B : B + 1;
  __shared__ double vbuf[2][G * VS];
  __shared__ double tau2[2];
  __shared__ AMx red_am[2][32];
  __shared__ double vcol[B == 16 ? 1024 : (B == 64 ? 256 : 512)];   // reflector of the pivoted QR step
  __shared__ double red_d[64];
  __shared__ int s_cnt[32];
  __shared__ int s_k, s_ktol, s_niter, s_cap, s_need;

  const CompressTask t = a.tasks[blockIdx.x];
  const Problem& P = a.P;
  const InstParams ip = P.ip[t.inst];
  const int n = t.n, d = P.d;
  const int NT = blockDim.x, nw = NT >> 5;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int c = tid;  // the column this thread owns (if c < n)
  CompressOut* out = a.out + t.out_idx;
  int64_t* slf = a.ipool + t.slf_off;
  int64_t* cand = a.cpool + t.cand_off;
  if (n == 0) {
    if (tid == 0) *out = CompressOut{0, 0, 0, 0};
    return;
  }
  const int ld = n | 1;  // odd row stride: column accesses of R hit distinct banks
  double* R = (t.scr_off >= 0) ? a.scratch + t.scr_off : smem;   // n x ld, row-major
  double* vn1 = R + (int64_t)n * ld;
  double* vn2 = vn1 + n;
  double* aux = vn2 + n;                                         // 6n (RRQR), reused for ids
  int* jpvt = reinterpret_cast<int*>(aux + 6 * (int64_t)n);

  // ---- (1) neighbour filter (pxyfun's nbr selection), stable compaction in place;
  // the row-split parts read the count the filter launch left
  const int mode = t.mode;
  const int m1 = mode != 0 ? a.mfilt[t.out_idx] : ((t.flags & 2) ? filter_candidates(t, P, ip, cand, s_cnt) : t.ncand);
  const int nrep = a.symm_n ? 2 : 1;
  const int npr = (t.flags & 1) ? (ip.two_sided ? 2 * P.npxy : P.npxy) : 0;
  // explicit rows: flam_id's matrix, or this box's row sketch
  const double* Ax = a.Aexp ? a.Aexp : (t.ax_rows > 0 ? a.ypool + t.ax_off : nullptr);
  const int64_t lda = a.Aexp ? a.lda : t.ax_rows;
  const int m = a.Aexp ? t.ncand : (Ax ? t.ax_rows : nrep * m1 + npr);
  const int mn = min(m, n);

  // ---- (2) TSQR: fold PH-row panels of K into R0; G threads per column.  A part of
  // the row-split form folds rows [rbeg, rend) of K; a merge folds the rows of the
  // upper triangular R at rsrc_off into the R already in place.
  int rbeg = 0, rend = m;
  const double* Rsrc = nullptr;
  if (mode == 1) {
    rbeg = (int)((int64_t)t.part * m / t.nparts);
    rend = (int)((int64_t)(t.part + 1) * m / t.nparts);
  } else if (mode >= 2) {
    Rsrc = a.scratch + t.rsrc_off;
    rend = n;
  }
  if (mode < 2)
    for (int64_t e = tid; e < (int64_t)n * ld; e += NT) R[e] = 0.0;
  const int col = tid / G, g = tid % G;
  const unsigned gmask = (G == 1) ? (1u << lane) : (((1u << G) - 1u) << (lane & ~(G - 1)));
  const int64_t sc = col < n ? slf[col] : 0;
  __syncthreads();
  // A row sketch with no more rows than columns is not folded: its pivoted QR runs on Y
  // itself (Y and the R of Y = Q R have the same column norms, hence the same pivots
  // and the same T up to rounding), rows m..n-1 of R staying zero.
  const bool direct = Ax && !a.Aexp && mode == 0 && m <= n;
  const int nrow = direct ? m : n;   // rows of R the pivoted QR touches
  if (direct) {
    for (int64_t e = tid; e < (int64_t)m * n; e += NT) {
      const int r = (int)(e % m), cc = (int)(e / m);
      R[(int64_t)r * ld + cc] = Ax[r + (int64_t)cc * lda];
    }
    __syncthreads();
  }
  double p[B];
  for (int p0 = rbeg; p0 < (direct ? rbeg : rend); p0 += PH) {
    if (!Ax && !Rsrc && tid < PH) {
      const int rho = p0 + tid < rend ? p0 + tid : m;   // rows past the part are zero
      int ty = 3;
      int64_t q = -1;
      double wm = 0.0;
      if (rho < m1) {
        ty = 0;
        q = cand[rho];
      } else if (a.symm_n && rho < 2 * m1) {
        ty = 1;
        q = cand[rho - m1];
      } else if (rho < m) {
        int pr = rho - nrep * m1;
        ty = 2;
        if (ip.two_sided && pr >= P.npxy) {
          pr -= P.npxy;
          wm = ip.wbar;
        }
        for (int k = 0; k < d; ++k) {
          const double pk = P.pxy_pts[pr * d + k];
          st.y[tid][k] = P.pxy_shift ? pk + P.pxy_shift[pr * d + k] * t.l[k] + t.ctr[k] : pk * t.l[k] + t.ctr[k];
        }
      }
      st.type[tid] = ty;
      st.q[tid] = q;
      st.wmul[tid] = wm;
    }
    __syncthreads();
    if (col < n) {
      const int r0 = p0 + g * B;
      if (Rsrc) {
#pragma unroll
        for (int i = 0; i < B; ++i) p[i] = (r0 + i < rend) ? Rsrc[(int64_t)(r0 + i) * ld + col] : 0.0;
      } else if (Ax) {
#pragma unroll
        for (int i = 0; i < B; ++i) p[i] = (r0 + i < m) ? Ax[(r0 + i) + (int64_t)col * lda] : 0.0;
      } else {
#pragma unroll
        for (int i = 0; i < B; ++i) {
          const int s = g * B + i;
          p[i] = block_entry(P, ip, st.type[s], st.q[s], st.y[s], st.wmul[s], sc);
        }
      }
    }
    // first reflector of this panel, formed by its owners.  Thread col is the only
    // writer of column col of R, so it reads R(j+1, col) one reflector ahead
    // (the load overlaps step j and its barrier).  Rows p0.. of a triangular R are
    // zero left of column p0: those reflectors are the identity and are skipped.
    const int js = Rsrc ? p0 : 0;
    double rcur = col < n ? R[(int64_t)js * ld + col] : 0.0;   // R(js, col)
    if (col == js) reflect_col<B, G, VS>(p, rcur, R, ld, js, g, gmask, vbuf[js & 1], &tau2[js & 1]);
    __syncthreads();
    for (int j = js; j < n; ++j) {
      const int b = j & 1;
      const double rnext = (col > j && col < n && j + 1 < n) ? R[(int64_t)(j + 1) * ld + col] : 0.0;
      const double tau = tau2[b];
      if (tau != 0.0 && col > j && col < n) {
        const double* v = vbuf[b] + g * VS;
        double w0 = 0.0, w1 = 0.0, w2 = 0.0, w3 = 0.0;
#pragma unroll
        for (int i = 0; i < B; i += 4) {
          w0 += v[i] * p[i];
          w1 += v[i + 1] * p[i + 1];
          w2 += v[i + 2] * p[i + 2];
          w3 += v[i + 3] * p[i + 3];
        }
        const double tw = tau * (rcur + group_sum<G>((w0 + w1) + (w2 + w3), gmask));
        if (g == 0) R[(int64_t)j * ld + col] = rcur - tw;
#pragma unroll
        for (int i = 0; i < B; ++i) p[i] -= tw * v[i];
      }
      if (col == j + 1 && col < n)
        reflect_col<B, G, VS>(p, rnext, R, ld, j + 1, g, gmask, vbuf[b ^ 1], &tau2[b ^ 1]);
      rcur = rnext;
      __syncthreads();
    }
  }

  if (mode == 1 || mode == 2) return;   // this part's R stays in place for the next merge

  // ---- (3) column-pivoted QR of R0 (xLAQP2) for min(m, n) steps
  if (c < n) {
    double s = 0.0;
    for (int r = 0; r < nrow; ++r) s += R[(int64_t)r * ld + c] * R[(int64_t)r * ld + c];
    vn1[c] = vn2[c] = sqrt(s);
    jpvt[c] = c;
  }
  __syncthreads();
  const double tol3z = 1.0536712127723509e-08;  // sqrt(2^-53), LAPACK's dlamch('Epsilon')
  // In tolerance mode the rank is the number of |R(i,i)| > tol |R(0,0)| (id.m:106-113);
  // the pivoted diagonal does not increase, so the loop stops at the first entry at or
  // below the tolerance: the skeleton set, R11 and R12 are final by then.  (Only the
  // order of the redundant columns -- later pivots -- is left as it stands.)
  const bool stop_early = a.kmax == 0 && !a.Aexp;
  double r00 = 0.0;
  int mn_eff = mn;
  for (int i = 0; i < mn; ++i) {
    AMx am{-1.0, n};
    if (c >= i && c < n) am = AMx{vn1[c], c};
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      AMx o2{__shfl_xor_sync(0xffffffffu, am.v, o), __shfl_xor_sync(0xffffffffu, am.i, o)};
      am = amx_better(am, o2);
    }
    AMx* ra = red_am[i & 1];   // alternating buffers: no barrier needed before the next step's writes
    if (lane == 0) ra[wid] = am;
    __syncthreads();
    AMx bm = ra[0];
    for (int w = 1; w < nw; ++w) bm = amx_better(bm, ra[w]);
    const int pvt = (bm.i >= i && bm.i < n) ? bm.i : i;   // NaN norms keep the column
    // swap columns i and pvt, and gather column i's rows below the diagonal (the
    // reflector) into shared memory with its sum of squares, one row per thread
    double s = 0.0;
    for (int r = tid; r < nrow; r += NT) {
      double v = R[(int64_t)r * ld + pvt];
      if (pvt != i) {
        R[(int64_t)r * ld + pvt] = R[(int64_t)r * ld + i];
        R[(int64_t)r * ld + i] = v;
      }
      if (r > i && i + 1 < m) {
        vcol[r] = v;
        s += v * v;
      }
    }
    if (tid == 0 && pvt != i) {
      const int tj = jpvt[pvt];
      jpvt[pvt] = jpvt[i];
      jpvt[i] = tj;
      vn1[pvt] = vn1[i];
      vn2[pvt] = vn2[i];
    }
    s = warp_sum(s);
    double* rd_ = red_d + (i & 1) * 32;   // alternating halves
    if (lane == 0) rd_[wid] = s;
    __syncthreads();
    s = 0.0;
    for (int w = 0; w < nw; ++w) s += rd_[w];
    // DLARFG on column i, rows i..m-1, computed by every thread alike
    double tau = 0.0, be = 0.0;
    const double al = R[(int64_t)i * ld + i];
    const double dii = s != 0.0 ? -copysign(hypot(al, sqrt(s)), al) : al;   // R(i,i) after this step
    if (i == 0) r00 = fabs(dii);
    if (stop_early && i > 0 && !(fabs(dii) > a.rel_tol * r00)) {
      mn_eff = i;      // uniform: every thread computed the same dii
      break;
    }
    if (s != 0.0) {
      be = dii;
      tau = (be - al) / be;
      const double scal = 1.0 / (al - be);
      for (int r = i + 1 + tid; r < nrow; r += NT) {
        const double v = vcol[r] * scal;
        vcol[r] = v;
        R[(int64_t)r * ld + i] = v;
      }
    }
    __syncthreads();   // every thread has read R(i,i); the reflector is complete
    if (tid == 0 && s != 0.0) R[(int64_t)i * ld + i] = be;
    if (c > i && c < n) {
      if (tau != 0.0) {
        // column c from R (L2 for large n) LD rows at a time -- LD loads in flight per
        // thread hide the L2 latency of the long columns -- the reflector from shared memory
        double* Rc = R + c;
        double w0 = Rc[(int64_t)i * ld], w1 = 0.0, w2 = 0.0, w3 = 0.0;
        int r = i + 1;
        for (; r + LD - 1 < nrow; r += LD) {
          double b[LD];
#pragma unroll
          for (int u = 0; u < LD; ++u) b[u] = Rc[(int64_t)(r + u) * ld];
#pragma unroll
          for (int u = 0; u < LD; u += 4) {
            w0 += vcol[r + u] * b[u];
            w1 += vcol[r + u + 1] * b[u + 1];
            w2 += vcol[r + u + 2] * b[u + 2];
            w3 += vcol[r + u + 3] * b[u + 3];
          }
        }
        for (; r + 7 < nrow; r += 8) {
          double b[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) b[u] = Rc[(int64_t)(r + u) * ld];
          w0 += vcol[r] * b[0] + vcol[r + 4] * b[4];
          w1 += vcol[r + 1] * b[1] + vcol[r + 5] * b[5];
          w2 += vcol[r + 2] * b[2] + vcol[r + 6] * b[6];
          w3 += vcol[r + 3] * b[3] + vcol[r + 7] * b[7];
        }
        for (; r < nrow; ++r) w0 += vcol[r] * Rc[(int64_t)r * ld];
        const double tw = tau * ((w0 + w1) + (w2 + w3));
        Rc[(int64_t)i * ld] -= tw;
        int rr = i + 1;
        for (; rr + LD - 1 < nrow; rr += LD) {
          double b[LD];
#pragma unroll
          for (int u = 0; u < LD; ++u) b[u] = Rc[(int64_t)(rr + u) * ld];
#pragma unroll
          for (int u = 0; u < LD; ++u) Rc[(int64_t)(rr + u) * ld] = b[u] - tw * vcol[rr + u];
        }
        for (; rr + 7 < nrow; rr += 8) {
          double b[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) b[u] = Rc[(int64_t)(rr + u) * ld];
#pragma unroll
          for (int u = 0; u < 8; ++u) Rc[(int64_t)(rr + u) * ld] = b[u] - tw * vcol[rr + u];
        }
        for (; rr < nrow; ++rr) Rc[(int64_t)rr * ld] -= tw * vcol[rr];
      }
      if (vn1[c] != 0.0) {  // partial norm downdate (xLAQP2)
        double temp = fabs(R[(int64_t)i * ld + c]) / vn1[c];
        temp = fmax(1.0 - temp * temp, 0.0);
        const double q = vn1[c] / vn2[c];
        if (temp * q * q <= tol3z) {
          if (i + 1 < m) {
            double s = 0.0;
            for (int rr = i + 1; rr < nrow; ++rr) s += R[(int64_t)rr * ld + c] * R[(int64_t)rr * ld + c];
            vn1[c] = vn2[c] = sqrt(s);
          } else {
            vn1[c] = vn2[c] = 0.0;
          }
        } else {
          vn1[c] *= sqrt(temp);
        }
      }
    }
    // the next step's pivot reduction starts with a barrier-separated exchange
  }
  __syncthreads();
  // clear the reflectors below the diagonal (the RRQR update reads R as upper trapezoidal)
  if (c < n)
    for (int r = c + 1; r < nrow; ++r) R[(int64_t)r * ld + c] = 0.0;

  // ---- (4) rank (id.m:106-113)
  if (tid == 0) {
    const double tol = a.rel_tol * fabs(R[0]);
    int kt = 0;
    if (m > 0)
      for (int i = 0; i < mn_eff; ++i) kt += fabs(R[(int64_t)i * ld + i]) > tol;
    int kmax = a.kmax;
    if (kmax == 0 || kmax > n) kmax = n;
    s_ktol = kt;
    s_k = min(kt, kmax);
    s_niter = 0;
    s_cap = 0;
  }
  __syncthreads();
  int k = s_k;
  const int ktol = s_ktol;

  // ---- (5) T = R11 \ R12 (id.m:114), one column per thread
  if (k > 0 && k < n && m > 0 && c >= k && c < n) {
    for (int i = k - 1; i >= 0; --i) {
      double v = R[(int64_t)i * ld + c];
      for (int j = i + 1; j < k; ++j) v -= R[(int64_t)i * ld + j] * R[(int64_t)j * ld + c];
      R[(int64_t)i * ld + c] = v / R[(int64_t)i * ld + i];
    }
  }
  __syncthreads();

  // ---- (6) RRQR refinement (id.m:117-236), only when some |T| > Tmax (or R22 is present);
  // not for a sketch whose rank fills it (the posterior check discards that ID)
  const bool sketch_full = t.ax_rows > 0 && k > t.ax_rows - t.ax_guard;
  if (m > 0 && !isinf(a.Tmax) && a.rrqr_iter != 0 && k > 0 && k < n && !sketch_full) {
    double mx = 0.0;
    if (c >= k && c < n)
      for (int i = 0; i < k; ++i) mx = fmax(mx, R[(int64_t)i * ld + c] * R[(int64_t)i * ld + c]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red_d[wid] = mx;
    __syncthreads();
    if (tid == 0) {
      double bm = 0.0;
      for (int w = 0; w < nw; ++w) bm = fmax(bm, red_d[w]);
      s_need = (ktol > k || bm > a.Tmax * a.Tmax) ? 1 : 0;
    }
    __syncthreads();
    if (s_need) {
      // the norms RRQR starts from, in parallel: r2(i) = |row i of inv(R11)|^2 by forward
      // substitution on thread i (the row kept in column i of R's empty strict lower
      // triangle), c2(j) = |column j of R22|^2 (id.m:120-121)
      for (int i = tid; i < k; i += NT) {
        const double yi = 1.0 / R[(int64_t)i * ld + i];
        double s2 = yi * yi;
        for (int j = i + 1; j < k; ++j) {
          double sj = yi * R[(int64_t)i * ld + j];
          for (int l = i + 1; l < j; ++l) sj += R[(int64_t)l * ld + i] * R[(int64_t)l * ld + j];
          const double yj = -sj / R[(int64_t)j * ld + j];
          R[(int64_t)j * ld + i] = yj;
          s2 += yj * yj;
        }
        aux[i] = s2;
      }
      for (int j = tid; j < n - k; j += NT) {
        double s2 = 0.0;
        for (int row = k; row < ktol; ++row) s2 += R[(int64_t)row * ld + k + j] * R[(int64_t)row * ld + k + j];
        aux[n + j] = s2;
      }
      __syncthreads();
      for (int i = tid; i < k; i += NT)
        for (int j = i + 1; j < k; ++j) R[(int64_t)j * ld + i] = 0.0;
      __syncthreads();
      if (tid == 0) {
        int niter = 0, capped = 0;
        const double tol = a.rel_tol * fabs(R[0]);
        const int kk = rrqr_serial(R, ld, 1, n, k, ktol, jpvt, tol, a.Tmax, a.rrqr_iter, aux, &niter, &capped, true);
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
  int64_t* tmp_ids = reinterpret_cast<int64_t*>(aux);
  for (int q = tid; q < n; q += NT) tmp_ids[q] = slf[q];
  __syncthreads();
  for (int q = tid; q < n; q += NT) {
    const int src = keep_order ? q : jpvt[q];
    perm_out[q] = src;
    slf[q] = tmp_ids[src];
  }
  if (r > 0 && k > 0 && c >= k && c < n) {
    double* T = a.tpool + t.T_off;
    for (int i = 0; i < k; ++i) T[i + (int64_t)(c - k) * k] = R[(int64_t)i * ld + c];
  }
  if (tid == 0) {
    int st = s_cap ? (int)ST_RRQR_CAP : 0;
    // sketched ID check: a rank within ax_guard of the sketch's rows may have been cut by the sketch
    if (t.ax_rows > 0 && k > t.ax_rows - t.ax_guard) st |= ST_ID_CHECK;
    *out = CompressOut{k, m, s_niter, st};
  }
}

template <int B, int G>
void launch_b(const CompressArgs& a, int ntask, int nt, size_t smem, cudaStream_t s) {
  if (ensure_smem_attr(reinterpret_cast<const void*>(k_compress_tc<B, G>), 200 * 1024) != cudaSuccess) return;
  k_compress_tc<B, G><<<ntask, nt, smem, s>>>(a);
}

}  // namespace

int64_t compress_tc_doubles(int n) { return (int64_t)n * (n | 1) + 8 * (int64_t)n + n / 2 + 2; }

size_t compress_tc_smem_bytes(int n) { return sizeof(double) * (size_t)compress_tc_doubles(n); }

// Panel rows per thread (measured on the star-curve workload, N = 262144): 64 for
// 128 < n <= 256 (one thread per column: 256 threads, so a 64-row column panel fits
// in registers); 32 for smaller boxes (several threads per column, more CTAs per SM
// on the levels with thousands of boxes) and up to n = 512; 16 beyond.
int compress_tc_rows(int n) { return (n > 128 && n <= 256) ? 64 : (n <= 512 ? 32 : 16); }

// Threads per column: with 64 rows per thread 1; with 32 rows 4 for n <= 64, 2 for
// n <= 256, else 1 (512 threads at most); with 16 rows (n > 512) 1.
int compress_tc_group(int n) {
  if (compress_tc_rows(n) == 64) return 1;
  return n <= 64 ? 4 : (n <= 256 ? 2 : 1);
}

int compress_tc_threads(int n) {
  int cols = 32;
  while (cols < n) cols <<= 1;
  const int nt = cols * compress_tc_group(n);
  return std::max(nt, compress_tc_rows(n) * compress_tc_group(n));   // at least one thread per panel row
}

void launch_filter(const CompressArgs& a, int ntask, cudaStream_t s) {
  if (ntask > 0) k_filter<<<ntask, 256, 0, s>>>(a);
}

void launch_compress_tc(const CompressArgs& a, int ntask, int nt, int b, int g, size_t smem, cudaStream_t s) {
  if (ntask <= 0) return;
  if (b == 16)
    launch_b<16, 1>(a, ntask, nt, smem, s);
  else if (b == 64)
    launch_b<64, 1>(a, ntask, nt, smem, s);   // 64-row panels are used with one thread per column
  else if (g == 4)
    launch_b<32, 4>(a, ntask, nt, smem, s);
  else if (g == 2)
    launch_b<32, 2>(a, ntask, nt, smem, s);
  else
    launch_b<32, 1>(a, ntask, nt, smem, s);
}

}  // namespace flam
