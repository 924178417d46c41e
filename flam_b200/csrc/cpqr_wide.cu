// ID of a short, wide explicit matrix: the row sketch Y (w x n, w <= 2048 rows) of a box
// with more points than the thread-per-column compression takes (n > 1024).
//
// Same decisions as the other compression kernels (core/id.m:102-114 on Y): column-
// pivoted Householder QR with LAPACK xLAQP2's rule (first maximum of the partial column
// norms, sqrt(eps) recomputation threshold), stopping at the first |R(i,i)| <=
// tol |R(0,0)| in tolerance mode, the rank, T = R11 \ R12 and, when some |T| > Tmax, the
// RRQR refinement of id.m:116-236 (rrqr.cuh).  One CTA per box; Y is updated in place
// in global memory (L2-resident), a warp per column for the reflector products (lanes
// over rows: coalesced), the reflector in shared memory.  T is solved a column per
// thread in 32-row blocks (the block's unknowns in registers).
#include <algorithm>
#include <cmath>

#include "common.cuh"
#include "kernels.cuh"
#include "rrqr.cuh"
#include "sketch.cuh"

namespace flam {
namespace {

constexpr int kWThreads = 512;
constexpr int kWWarps = kWThreads / 32;
constexpr int kWMaxRows = 2048;          // single-CTA form (its reflector lives in shared memory)
constexpr int kGwMaxRows = kSketchMaxW;   // grid form (reflector in dynamic shared memory)

struct WAm {
  double v;
  int i;
};
__device__ __forceinline__ WAm wbetter(WAm a, WAm b) {
  if (b.v > a.v || (b.v == a.v && b.i < a.i)) return b;
  return a;
}

// T = R11 \ R12 in place for the columns c = k + c0 + tid (one per thread, c0 over
// blockDim-wide groups), R11 (k x k, upper) and R12 in Y (ld w).  Back substitution by
// 32-row blocks from the bottom; the block's diagonal part and, 64 rows at a time, the
// part above it are staged in shared memory (coalesced loads, broadcast reads), so a
// thread streams only its own column.  Called by every thread of the CTA.
__device__ void tsolve_block_columns(double* Y, int w, int k, int n, int cfirst, int cstep, double* sd, double* su) {
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int cg = cfirst; cg < n - k; cg += cstep) {
    const int c = k + cg + tid;
    const bool live = c < n;
    double* yc = Y + (int64_t)(live ? c : k) * w;
    for (int i1 = k; i1 > 0;) {
      const int i0 = i1 > 32 ? i1 - 32 : 0, bs = i1 - i0;
      __syncthreads();
      for (int e = tid; e < 32 * 32; e += nt) {   // sd[j * 33 + l] = R(i0 + j, i0 + l)
        const int j = e % 32, l = e / 32;
        sd[j * 33 + l] = (j < bs && l < bs) ? Y[(i0 + j) + (int64_t)(i0 + l) * w] : 0.0;
      }
      __syncthreads();
      double x[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) x[j] = (live && j < bs) ? yc[i0 + j] : 0.0;
#pragma unroll
      for (int j = 31; j >= 0; --j) {
        if (j < bs) {
          double v = x[j];
#pragma unroll
          for (int l = j + 1; l < 32; ++l)
            if (l < bs) v -= sd[j * 33 + l] * x[l];
          x[j] = v / sd[j * 33 + j];
        }
      }
      if (live) {
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (j < bs) yc[i0 + j] = x[j];
      }
      for (int r0 = 0; r0 < i0; r0 += 64) {
        const int rn = min(64, i0 - r0);
        __syncthreads();
        for (int e = tid; e < 64 * 32; e += nt) {   // su[rr * 33 + j] = R(r0 + rr, i0 + j)
          const int rr = e % 64, j = e / 64;
          su[rr * 33 + j] = (rr < rn && j < bs) ? Y[(r0 + rr) + (int64_t)(i0 + j) * w] : 0.0;
        }
        __syncthreads();
        if (live) {
          for (int rr = 0; rr < rn; ++rr) {
            double v = yc[r0 + rr];
#pragma unroll
            for (int j = 0; j < 32; ++j) v -= su[rr * 33 + j] * x[j];
            yc[r0 + rr] = v;
          }
        }
      }
      i1 = i0;
    }
  }
}

__global__ void __launch_bounds__(kWThreads) k_cpqr_wide(CompressArgs a) {
  __shared__ double vbuf[kWMaxRows];
  __shared__ double tsd[32 * 33], tsu[64 * 33];
  __shared__ double red[kWWarps];
  __shared__ WAm ram[kWWarps];
  __shared__ int s_k, s_ktol, s_niter, s_cap, s_need, s_pvt, s_stop;
  __shared__ double s_tau, s_r00;
  const CompressTask t = a.tasks[blockIdx.x];
  const int n = t.n, w = t.ax_rows;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  CompressOut* out = a.out + t.out_idx;
  double* Y = const_cast<double*>(a.ypool) + t.ax_off;   // w x n, ld w
  auto y = [&](int r, int c) -> double& { return Y[r + (int64_t)c * w]; };
  double* sc = a.scratch + t.scr_off;
  double* vn1 = sc;
  double* vn2 = vn1 + n;
  double* aux = vn2 + n;                                  // 6n: RRQR norms and work
  int* jpvt = reinterpret_cast<int*>(aux + 6 * (int64_t)n);
  int64_t* slf = a.ipool + t.slf_off;
  if (n == 0 || w > kWMaxRows) {
    if (tid == 0) *out = CompressOut{0, 0, 0, n == 0 ? 0 : (int)ST_ID_CHECK};
    return;
  }
  const int mn = min(w, n);
  // column norms
  for (int c = wid; c < n; c += kWWarps) {
    double s = 0.0;
    for (int r = lane; r < w; r += 32) s += y(r, c) * y(r, c);
    s = warp_sum(s);
    if (lane == 0) {
      vn1[c] = vn2[c] = sqrt(s);
      jpvt[c] = c;
    }
  }
  if (tid == 0) s_stop = mn;
  __syncthreads();
  const double tol3z = 1.0536712127723509e-08;   // sqrt(2^-53)
  const bool stop_early = a.kmax == 0;
  for (int i = 0; i < mn; ++i) {
    // pivot: the first maximum of the partial norms over columns i..n-1
    WAm am{-1.0, n};
    for (int c = i + tid; c < n; c += kWThreads) am = wbetter(am, WAm{vn1[c], c});
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      WAm b{__shfl_xor_sync(0xffffffffu, am.v, o), __shfl_xor_sync(0xffffffffu, am.i, o)};
      am = wbetter(am, b);
    }
    if (lane == 0) ram[wid] = am;
    __syncthreads();
    if (tid == 0) {
      WAm bm = ram[0];
      for (int q = 1; q < kWWarps; ++q) bm = wbetter(bm, ram[q]);
      s_pvt = (bm.i >= i && bm.i < n) ? bm.i : i;
    }
    __syncthreads();
    const int pvt = s_pvt;
    // swap columns i and pvt; gather the reflector's rows into shared memory
    double s = 0.0;
    for (int r = tid; r < w; r += kWThreads) {
      const double v = y(r, pvt);
      if (pvt != i) {
        y(r, pvt) = y(r, i);
        y(r, i) = v;
      }
      vbuf[r] = v;
      if (r > i) s += v * v;
    }
    if (tid == 0 && pvt != i) {
      const int tj = jpvt[pvt];
      jpvt[pvt] = jpvt[i];
      jpvt[i] = tj;
      vn1[pvt] = vn1[i];
      vn2[pvt] = vn2[i];
    }
    s = warp_sum(s);
    if (lane == 0) red[wid] = s;
    __syncthreads();
    if (tid == 0) {
      double ss = 0.0;
      for (int q = 0; q < kWWarps; ++q) ss += red[q];
      const double al = vbuf[i];
      const double dii = ss != 0.0 ? -copysign(hypot(al, sqrt(ss)), al) : al;
      if (i == 0) s_r00 = fabs(dii);
      if (stop_early && i > 0 && !(fabs(dii) > a.rel_tol * s_r00)) {
        s_stop = i;
        s_tau = -1.0;
      } else {
        double tau = 0.0;
        if (ss != 0.0) {
          tau = (dii - al) / dii;
          const double scal = 1.0 / (al - dii);
          for (int r = i + 1; r < w; ++r) vbuf[r] *= scal;
          y(i, i) = dii;
          for (int r = i + 1; r < w; ++r) y(r, i) = vbuf[r];
        }
        s_tau = tau;
      }
    }
    __syncthreads();
    const double tau = s_tau;
    if (tau < 0.0) break;   // rank reached (uniform)
    // apply the reflector to columns i+1..n-1 (a warp per column) and downdate the norms
    for (int c = i + 1 + wid; c < n; c += kWWarps) {
      if (tau != 0.0) {
        double d = lane == 0 ? y(i, c) : 0.0;
        for (int r = i + 1 + lane; r < w; r += 32) d += vbuf[r] * y(r, c);
        d = tau * warp_sum(d);
        if (lane == 0) y(i, c) -= d;
        for (int r = i + 1 + lane; r < w; r += 32) y(r, c) -= d * vbuf[r];
      }
      __syncwarp();
      double nv = vn1[c];
      if (nv != 0.0) {
        double temp = fabs(y(i, c)) / nv;
        temp = fmax(1.0 - temp * temp, 0.0);
        const double q = nv / vn2[c];
        if (temp * q * q <= tol3z) {
          double s2 = 0.0;
          for (int r = i + 1 + lane; r < w; r += 32) s2 += y(r, c) * y(r, c);
          s2 = warp_sum(s2);
          if (lane == 0) vn1[c] = vn2[c] = (i + 1 < w) ? sqrt(s2) : 0.0;
        } else if (lane == 0) {
          vn1[c] = nv * sqrt(temp);
        }
      }
    }
    __syncthreads();
  }
  // rank (id.m:106-113)
  if (tid == 0) {
    const int mn_eff = s_stop;
    const double tol = a.rel_tol * fabs(y(0, 0));
    int kt = 0;
    for (int i = 0; i < mn_eff; ++i) kt += fabs(y(i, i)) > tol;
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
  // clear the reflectors below the diagonal of the first ktol rows (R is upper trapezoidal)
  for (int c = wid; c < min(ktol, n); c += kWWarps)
    for (int r = c + 1 + lane; r < ktol; r += 32) y(r, c) = 0.0;
  __syncthreads();
  // a rank that fills the sketch fails the posterior check: that ID is discarded, so it
  // gets neither T nor the RRQR refinement
  const bool sketch_full = k > w - t.ax_guard;
  // T = R11 \ R12 (shared-memory staged blocks)
  if (k > 0 && k < n && !sketch_full) tsolve_block_columns(Y, w, k, n, 0, kWThreads, tsd, tsu);
  __syncthreads();
  // RRQR refinement (id.m:117-236), on thread 0, when some |T| > Tmax or rows were cut
  if (!isinf(a.Tmax) && a.rrqr_iter != 0 && k > 0 && k < n && !sketch_full) {
    double mx = 0.0;
    for (int c = k + tid; c < n; c += kWThreads)
      for (int i = 0; i < k; ++i) mx = fmax(mx, y(i, c) * y(i, c));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 16));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 8));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 4));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    if (lane == 0) red[wid] = mx;
    __syncthreads();
    if (tid == 0) {
      double bm = 0.0;
      for (int q = 0; q < kWWarps; ++q) bm = fmax(bm, red[q]);
      s_need = (ktol > k || bm > a.Tmax * a.Tmax) ? 1 : 0;
      if (s_need) {
        int niter = 0, capped = 0;
        const double tol = a.rel_tol * fabs(y(0, 0));
        s_k = rrqr_serial(Y, 1, w, n, k, ktol, jpvt, tol, a.Tmax, a.rrqr_iter, aux, &niter, &capped);
        s_niter = niter;
        s_cap = capped;
      }
    }
    __syncthreads();
    k = s_k;
  }
  // outputs: [sk rd] order of slf, local permutation, T
  const int r = n - k;
  int* perm_out = a.permpool + t.perm_off;
  int64_t* tmp_ids = reinterpret_cast<int64_t*>(aux);
  for (int q = tid; q < n; q += kWThreads) tmp_ids[q] = slf[q];
  __syncthreads();
  const bool keep_order = r == 0;
  for (int q = tid; q < n; q += kWThreads) {
    const int src = keep_order ? q : jpvt[q];
    perm_out[q] = src;
    slf[q] = tmp_ids[src];
  }
  if (r > 0 && k > 0) {
    double* T = a.tpool + t.T_off;
    for (int c = k + wid; c < n; c += kWWarps)
      for (int i = lane; i < k; i += 32) T[i + (int64_t)(c - k) * k] = y(i, c);
  }
  if (tid == 0) {
    int st = s_cap ? (int)ST_RRQR_CAP : 0;
    if (k > w - t.ax_guard) st |= ST_ID_CHECK;
    *out = CompressOut{k, w, s_niter, st};
  }
}

// ---------------------------------------------------------------- grid form
// The same factorization with every pivot step split over the GPU: for few wide boxes
// (the 8 boxes below a 3D root) one CTA per box leaves most SMs idle.  Step i is two
// launches over all boxes of the step: k_gw_pivot (one CTA per box: pivot, column swap,
// reflector) and k_gw_apply (16 columns per CTA: reflector products and norm downdates);
// then k_gw_rank, k_gw_tsolve (a thread per column of T) and k_gw_out (RRQR, outputs).
// Per-box state (the step at which the rank was reached, tau, |R(0,0)|, k) lives in a
// small device array.

struct GwState {
  int stop;      // steps done (the rank in tolerance mode, else min(w, n))
  int k, ktol;
  int niter, cap;
  int pad;
  double tau, r00;
};

__global__ void __launch_bounds__(kWThreads) k_gw_norms(CompressArgs a, GwState* gs) {
  const CompressTask t = a.tasks[blockIdx.y];
  const int n = t.n, w = t.ax_rows, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const double* Y = a.ypool + t.ax_off;
  double* vn1 = a.scratch + t.scr_off;
  double* vn2 = vn1 + n;
  int* jpvt = reinterpret_cast<int*>(vn2 + 7 * (int64_t)n);
  const int c = blockIdx.x * kWWarps + wid;
  if (c < n) {
    double s = 0.0;
    for (int r = lane; r < w; r += 32) s += Y[r + (int64_t)c * w] * Y[r + (int64_t)c * w];
    s = warp_sum(s);
    if (lane == 0) {
      vn1[c] = vn2[c] = sqrt(s);
      jpvt[c] = c;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    GwState z{};
    z.stop = (n == 0 || w > kGwMaxRows) ? 0 : min(w, n);
    z.r00 = 0.0;
    gs[blockIdx.y] = z;
  }
}

__global__ void __launch_bounds__(kWThreads) k_gw_pivot(CompressArgs a, GwState* gs, int i) {
  __shared__ double red[kWWarps];
  __shared__ WAm ram[kWWarps];
  __shared__ int s_pvt;
  const int b = blockIdx.x;
  if (i >= gs[b].stop) return;
  const CompressTask t = a.tasks[b];
  const int n = t.n, w = t.ax_rows;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  double* Y = const_cast<double*>(a.ypool) + t.ax_off;
  auto y = [&](int r, int c) -> double& { return Y[r + (int64_t)c * w]; };
  double* vn1 = a.scratch + t.scr_off;
  double* vn2 = vn1 + n;
  int* jpvt = reinterpret_cast<int*>(vn2 + 7 * (int64_t)n);
  WAm am{-1.0, n};
  for (int c = i + tid; c < n; c += kWThreads) am = wbetter(am, WAm{vn1[c], c});
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    WAm bb{__shfl_xor_sync(0xffffffffu, am.v, o), __shfl_xor_sync(0xffffffffu, am.i, o)};
    am = wbetter(am, bb);
  }
  if (lane == 0) ram[wid] = am;
  __syncthreads();
  if (tid == 0) {
    WAm bm = ram[0];
    for (int q = 1; q < kWWarps; ++q) bm = wbetter(bm, ram[q]);
    s_pvt = (bm.i >= i && bm.i < n) ? bm.i : i;
  }
  __syncthreads();
  const int pvt = s_pvt;
  double s = 0.0;
  for (int r = tid; r < w; r += kWThreads) {
    const double v = y(r, pvt);
    if (pvt != i) {
      y(r, pvt) = y(r, i);
      y(r, i) = v;
    }
    if (r > i) s += v * v;
  }
  if (tid == 0 && pvt != i) {
    const int tj = jpvt[pvt];
    jpvt[pvt] = jpvt[i];
    jpvt[i] = tj;
    vn1[pvt] = vn1[i];
    vn2[pvt] = vn2[i];
  }
  s = warp_sum(s);
  if (lane == 0) red[wid] = s;
  __syncthreads();
  double ss = 0.0;
  for (int q = 0; q < kWWarps; ++q) ss += red[q];
  const double al = y(i, i);
  const double dii = ss != 0.0 ? -copysign(hypot(al, sqrt(ss)), al) : al;
  const double r00 = i == 0 ? fabs(dii) : gs[b].r00;
  if (a.kmax == 0 && i > 0 && !(fabs(dii) > a.rel_tol * r00)) {   // rank reached (tolerance mode)
    __syncthreads();
    if (tid == 0) gs[b].stop = i;
    return;
  }
  double tau = 0.0;
  if (ss != 0.0) {
    tau = (dii - al) / dii;
    const double scal = 1.0 / (al - dii);
    for (int r = i + 1 + tid; r < w; r += kWThreads) y(r, i) *= scal;
  }
  __syncthreads();   // every thread has read y(i, i)
  if (tid == 0) {
    if (ss != 0.0) y(i, i) = dii;
    gs[b].tau = tau;
    if (i == 0) gs[b].r00 = r00;
  }
}

__global__ void __launch_bounds__(kWThreads) k_gw_apply(CompressArgs a, GwState* gs, int i) {
  extern __shared__ double v[];   // rows of the reflector (w doubles)
  const int b = blockIdx.y;
  if (i >= gs[b].stop) return;
  const CompressTask t = a.tasks[b];
  const int n = t.n, w = t.ax_rows;
  const int c0 = i + 1 + blockIdx.x * kWWarps;
  if (c0 >= n) return;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  double* Y = const_cast<double*>(a.ypool) + t.ax_off;
  auto y = [&](int r, int c) -> double& { return Y[r + (int64_t)c * w]; };
  double* vn1 = a.scratch + t.scr_off;
  double* vn2 = vn1 + n;
  const double tau = gs[b].tau;
  for (int r = i + 1 + tid; r < w; r += kWThreads) v[r] = y(r, i);
  __syncthreads();
  const double tol3z = 1.0536712127723509e-08;
  const int c = c0 + wid;
  if (c >= n) return;
  double* yc = Y + (int64_t)c * w;
  // each lane streams rows lane, lane + 32, ... of its warp's column; four rows are in
  // flight per lane (independent partial sums), so a warp keeps 1 KB of loads outstanding
  // instead of one 256-byte row at a time
  const int r0 = i + 1 + lane;
  if (tau != 0.0) {
    double d0 = lane == 0 ? yc[i] : 0.0, d1 = 0.0, d2 = 0.0, d3 = 0.0;
    int r = r0;
    for (; r + 96 < w; r += 128) {
      const double a0 = yc[r], a1 = yc[r + 32], a2 = yc[r + 64], a3 = yc[r + 96];
      d0 += v[r] * a0;
      d1 += v[r + 32] * a1;
      d2 += v[r + 64] * a2;
      d3 += v[r + 96] * a3;
    }
    for (; r < w; r += 32) d0 += v[r] * yc[r];
    const double d = tau * warp_sum((d0 + d1) + (d2 + d3));
    if (lane == 0) yc[i] -= d;
    r = r0;
    for (; r + 96 < w; r += 128) {
      const double a0 = yc[r], a1 = yc[r + 32], a2 = yc[r + 64], a3 = yc[r + 96];
      yc[r] = a0 - d * v[r];
      yc[r + 32] = a1 - d * v[r + 32];
      yc[r + 64] = a2 - d * v[r + 64];
      yc[r + 96] = a3 - d * v[r + 96];
    }
    for (; r < w; r += 32) yc[r] -= d * v[r];
  }
  __syncwarp();
  const double nv = vn1[c];
  if (nv != 0.0) {
    double temp = fabs(yc[i]) / nv;
    temp = fmax(1.0 - temp * temp, 0.0);
    const double q = nv / vn2[c];
    if (temp * q * q <= tol3z) {
      double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
      int r = r0;
      for (; r + 96 < w; r += 128) {
        const double a0 = yc[r], a1 = yc[r + 32], a2 = yc[r + 64], a3 = yc[r + 96];
        s0 += a0 * a0;
        s1 += a1 * a1;
        s2 += a2 * a2;
        s3 += a3 * a3;
      }
      for (; r < w; r += 32) s0 += yc[r] * yc[r];
      s2 = warp_sum((s0 + s1) + (s2 + s3));
      if (lane == 0) vn1[c] = vn2[c] = (i + 1 < w) ? sqrt(s2) : 0.0;
    } else if (lane == 0) {
      vn1[c] = nv * sqrt(temp);
    }
  }
}

__global__ void __launch_bounds__(kWThreads) k_gw_rank(CompressArgs a, GwState* gs) {
  const int b = blockIdx.x;
  const CompressTask t = a.tasks[b];
  const int n = t.n, w = t.ax_rows;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double* Y = const_cast<double*>(a.ypool) + t.ax_off;
  __shared__ int s_ktol;
  if (threadIdx.x == 0) {
    const int mn_eff = gs[b].stop;
    const double tol = a.rel_tol * fabs(Y[0]);
    int kt = 0;
    for (int i = 0; i < mn_eff; ++i) kt += fabs(Y[i + (int64_t)i * w]) > tol;
    int kmax = a.kmax;
    if (kmax == 0 || kmax > n) kmax = n;
    gs[b].ktol = kt;
    gs[b].k = (n == 0 || w > kGwMaxRows) ? 0 : min(kt, kmax);
    s_ktol = kt;
  }
  __syncthreads();
  const int ktol = s_ktol;
  for (int c = wid; c < min(ktol, n); c += kWWarps)
    for (int r = c + 1 + lane; r < ktol; r += 32) Y[r + (int64_t)c * w] = 0.0;
}

// T = R11 \ R12 for 64 columns of R12 per CTA (8 warps), with every global access
// coalesced: lanes run over rows.  Back substitution by 32-row blocks from the bottom:
// a warp solves a column's diagonal block with the block's rows in its lanes (x_j
// broadcast by shuffle), the solved x go to shared memory, then the rows above are
// updated 64 at a time, R's 64 x 32 slab held in registers (two rows a lane) and x read
// by broadcast.
constexpr int kTsCols = 64;
__global__ void __launch_bounds__(256) k_gw_tsolve(CompressArgs a, GwState* gs) {
  __shared__ double sd[32 * 33];            // sd[j * 33 + l] = R(i0 + j, i0 + l)
  __shared__ double su[32 * 64];            // su[j * 64 + rr] = R(r0 + rr, i0 + j)
  __shared__ double xs[kTsCols * 33];       // xs[cl * 33 + j] = x_j of local column cl
  const int b = blockIdx.y;
  const CompressTask t = a.tasks[b];
  const int n = t.n, w = t.ax_rows, k = gs[b].k;
  const int cbase = k + (int)blockIdx.x * kTsCols;
  // uniform over the CTA; a rank that fills the sketch fails the posterior check (no T)
  if (k <= 0 || k >= n || cbase >= n || k > w - t.ax_guard) return;
  const int ncol = min(kTsCols, n - cbase);
  double* Y = const_cast<double*>(a.ypool) + t.ax_off;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int i1 = k; i1 > 0;) {
    const int i0 = i1 > 32 ? i1 - 32 : 0, bs = i1 - i0;
    __syncthreads();
    for (int e = tid; e < 32 * 32; e += 256) {
      const int j = e & 31, l = e >> 5;
      sd[j * 33 + l] = (j < bs && l < bs) ? Y[(i0 + j) + (int64_t)(i0 + l) * w] : 0.0;
    }
    __syncthreads();
    for (int cl = wid; cl < ncol; cl += 8) {
      double* yc = Y + (int64_t)(cbase + cl) * w;
      double bv = lane < bs ? yc[i0 + lane] : 0.0;
      for (int j = bs - 1; j >= 0; --j) {
        const double xj = __shfl_sync(0xffffffffu, bv, j) / sd[j * 33 + j];
        if (lane == j) bv = xj;
        if (lane < j) bv -= sd[lane * 33 + j] * xj;
      }
      if (lane < bs) yc[i0 + lane] = bv;
      xs[cl * 33 + lane] = lane < bs ? bv : 0.0;
    }
    for (int r0 = 0; r0 < i0; r0 += 64) {
      const int rn = min(64, i0 - r0);
      __syncthreads();   // xs written; the previous slab's readers are done
      for (int e = tid; e < 64 * 32; e += 256) {
        const int rr = e & 63, j = e >> 6;
        su[j * 64 + rr] = (rr < rn && j < bs) ? Y[(r0 + rr) + (int64_t)(i0 + j) * w] : 0.0;
      }
      __syncthreads();
      double ra[32], rb[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        ra[j] = su[j * 64 + lane];
        rb[j] = su[j * 64 + lane + 32];
      }
      for (int cl = wid; cl < ncol; cl += 8) {
        double* yc = Y + (int64_t)(cbase + cl) * w + r0;
        double u0 = lane < rn ? yc[lane] : 0.0;
        double u1 = lane + 32 < rn ? yc[lane + 32] : 0.0;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const double xj = xs[cl * 33 + j];   // zero beyond bs: su is zero there
          u0 -= ra[j] * xj;
          u1 -= rb[j] * xj;
        }
        if (lane < rn) yc[lane] = u0;
        if (lane + 32 < rn) yc[lane + 32] = u1;
      }
    }
    i1 = i0;
  }
}

__global__ void __launch_bounds__(kWThreads) k_gw_out(CompressArgs a, GwState* gs) {
  __shared__ double red[kWWarps];
  __shared__ int s_k;
  const int b = blockIdx.x;
  const CompressTask t = a.tasks[b];
  const int n = t.n, w = t.ax_rows;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  CompressOut* out = a.out + t.out_idx;
  if (n == 0 || w > kGwMaxRows) {
    if (tid == 0) *out = CompressOut{0, 0, 0, n == 0 ? 0 : (int)ST_ID_CHECK};
    return;
  }
  double* Y = const_cast<double*>(a.ypool) + t.ax_off;
  auto y = [&](int r, int c) -> double& { return Y[r + (int64_t)c * w]; };
  double* vn1 = a.scratch + t.scr_off;
  double* aux = vn1 + 2 * (int64_t)n;
  int* jpvt = reinterpret_cast<int*>(aux + 6 * (int64_t)n);
  int64_t* slf = a.ipool + t.slf_off;
  int k = gs[b].k;
  const int ktol = gs[b].ktol;
  if (tid == 0) s_k = k;
  if (!isinf(a.Tmax) && a.rrqr_iter != 0 && k > 0 && k < n && k <= w - t.ax_guard) {
    double mx = 0.0;
    for (int c = k + tid; c < n; c += kWThreads)
      for (int i = 0; i < k; ++i) mx = fmax(mx, y(i, c) * y(i, c));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red[wid] = mx;
    __syncthreads();
    if (tid == 0) {
      double bm = 0.0;
      for (int q = 0; q < kWWarps; ++q) bm = fmax(bm, red[q]);
      if (ktol > k || bm > a.Tmax * a.Tmax) {
        int niter = 0, capped = 0;
        const double tol = a.rel_tol * fabs(y(0, 0));
        s_k = rrqr_serial(Y, 1, w, n, k, ktol, jpvt, tol, a.Tmax, a.rrqr_iter, aux, &niter, &capped);
        gs[b].niter = niter;
        gs[b].cap = capped;
      }
    }
  }
  __syncthreads();
  k = s_k;
  const int r = n - k;
  int* perm_out = a.permpool + t.perm_off;
  int64_t* tmp_ids = reinterpret_cast<int64_t*>(aux);
  for (int q = tid; q < n; q += kWThreads) tmp_ids[q] = slf[q];
  __syncthreads();
  for (int q = tid; q < n; q += kWThreads) {
    const int src = r == 0 ? q : jpvt[q];
    perm_out[q] = src;
    slf[q] = tmp_ids[src];
  }
  if (r > 0 && k > 0) {
    double* T = a.tpool + t.T_off;
    for (int c = k + wid; c < n; c += kWWarps)
      for (int i = lane; i < k; i += 32) T[i + (int64_t)(c - k) * k] = y(i, c);
  }
  if (tid == 0) {
    int st = gs[b].cap ? (int)ST_RRQR_CAP : 0;
    if (k > w - t.ax_guard) st |= ST_ID_CHECK;
    *out = CompressOut{k, w, gs[b].niter, st};
  }
}

}  // namespace

int64_t cpqr_wide_scratch_doubles(int n) { return 8 * (int64_t)n + n / 2 + 2; }

void launch_cpqr_wide(const CompressArgs& a, int ntask, cudaStream_t s) {
  if (ntask <= 0) return;
  k_cpqr_wide<<<ntask, kWThreads, 0, s>>>(a);
}

size_t cpqr_grid_state_bytes(int ntask) { return sizeof(GwState) * (size_t)std::max(ntask, 1); }

int cpqr_wide_max_rows() { return kWMaxRows; }

void launch_cpqr_grid(const CompressArgs& a, int ntask, int nmax, int wmax, int steps, void* state, cudaStream_t s) {
  if (ntask <= 0) return;
  GwState* gs = static_cast<GwState*>(state);
  const unsigned cb = (unsigned)((nmax + kWWarps - 1) / kWWarps), z = (unsigned)ntask;
  const int vbytes = (int)sizeof(double) * std::max(1, std::min(wmax, kGwMaxRows));
  if (ensure_smem_attr(reinterpret_cast<const void*>(k_gw_apply), vbytes) != cudaSuccess) return;
  k_gw_norms<<<dim3(cb, z), kWThreads, 0, s>>>(a, gs);
  for (int i = 0; i < steps; ++i) {
    k_gw_pivot<<<z, kWThreads, 0, s>>>(a, gs, i);
    k_gw_apply<<<dim3(cb, z), kWThreads, vbytes, s>>>(a, gs, i);
  }
  k_gw_rank<<<z, kWThreads, 0, s>>>(a, gs);
  k_gw_tsolve<<<dim3((unsigned)((nmax + kTsCols - 1) / kTsCols), z), 256, 0, s>>>(a, gs);
  k_gw_out<<<z, kWThreads, 0, s>>>(a, gs);
}

}  // namespace flam
