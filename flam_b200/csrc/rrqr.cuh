// Sequential RRQR refinement of the interpolative decomposition
// (core/id.m:117-236), shared by the device kernel (one thread per box; the
// loop runs only when max|T| > Tmax, which is rare) and a host build used to
// check it against the oracle on identical input.
#pragma once
#include <cmath>
#include <cstdint>

#ifndef FLAM_HD
#ifdef __CUDACC__
#define FLAM_HD __host__ __device__
#else
#define FLAM_HD
#endif
#endif

namespace flam {

constexpr int kRrqrCapH = 4096;

// Givens rotation zeroing b in (a; b): returns c, s with [c s; -s c] (a; b) = (r; 0).
FLAM_HD inline void rot(double a, double b, double& c, double& s) {
  if (b == 0.0) {
    c = 1.0;
    s = 0.0;
    return;
  }
  const double r = hypot(a, b);
  c = a / r;
  s = b / r;
}

FLAM_HD inline void apply_rows(double* R, int64_t rs, int64_t cs, int r0, int c0, int c1, double c, double s) {
  for (int col = c0; col < c1; ++col) {
    const double a = R[r0 * rs + col * cs], b = R[(r0 + 1) * rs + col * cs];
    R[r0 * rs + col * cs] = c * a + s * b;
    R[(r0 + 1) * rs + col * cs] = -s * a + c * b;
  }
}

// Swap columns i and k-1 of R11 (k x k) and re-triangularise (id.m:134,217).
FLAM_HD inline void swap_retri(double* R, int64_t rs, int64_t cs, int i, int k) {
  for (int row = 0; row < k; ++row) {
    double t = R[(int64_t)(row) * rs + (int64_t)i * cs];
    R[(int64_t)(row) * rs + (int64_t)i * cs] = R[(int64_t)(row) * rs + (int64_t)(k - 1) * cs];
    R[(int64_t)(row) * rs + (int64_t)(k - 1) * cs] = t;
  }
  double c, s;
  for (int row = k - 1; row > i; --row) {  // clear the spike in column i bottom-up
    rot(R[(int64_t)(row - 1) * rs + (int64_t)i * cs], R[(int64_t)(row) * rs + (int64_t)i * cs], c, s);
    apply_rows(R, rs, cs, row - 1, i, k, c, s);
    R[(int64_t)(row) * rs + (int64_t)i * cs] = 0.0;
  }
  for (int col = i + 1; col < k - 1; ++col) {  // clear the subdiagonal left behind
    rot(R[(int64_t)(col) * rs + (int64_t)col * cs], R[(int64_t)(col + 1) * rs + (int64_t)col * cs], c, s);
    apply_rows(R, rs, cs, col, col, k, c, s);
    R[(int64_t)(col + 1) * rs + (int64_t)col * cs] = 0.0;
  }
}

// x = R[0:k,0:k] \ b (upper triangular), sequential.
FLAM_HD inline void trisolve(const double* R, int64_t rs, int64_t cs, int k, const double* b, int64_t bs,
                             double* x) {
  for (int i = k - 1; i >= 0; --i) {
    double v = b[i * bs];
    for (int j = i + 1; j < k; ++j) v -= R[(int64_t)(i) * rs + (int64_t)j * cs] * x[j];
    x[i] = v / R[(int64_t)(i) * rs + (int64_t)i * cs];
  }
}

// Sequential RRQR refinement of id.m:117-236 on thread 0.  R holds `rows` rows
// (R11 | T) over n columns; returns the final rank, updates jpvt, niter.  With
// norms_ready the caller has already put the squared row norms of inv(R11) in
// aux[0:k] and the squared column norms of R22 in aux[n:2n-k] (id.m:120-121).
FLAM_HD inline int rrqr_serial(double* R, int64_t rs, int64_t cs, int n, int k, int rows, int* jpvt, double tol, double Tmax,
                           int64_t rrqr_iter, double* aux, int* niter_out, int* capped, bool norms_ready = false) {
  double* r2 = aux;            // k
  double* c2 = aux + n;        // n - k (+1)
  double* u = aux + 2 * n;     // k
  double* tv = aux + 3 * n;    // scratch
  const double f2 = Tmax * Tmax;
  int niter = 0;
  // c2 = column norms^2 of R22, r2 = row norms^2 of inv(R11)
  if (!norms_ready) {
    for (int j = 0; j < n - k; ++j) {
      double s = 0.0;
      for (int row = k; row < rows; ++row) s += R[(int64_t)(row) * rs + (int64_t)(k + j) * cs] * R[(int64_t)(row) * rs + (int64_t)(k + j) * cs];
      c2[j] = s;
    }
    for (int i = 0; i < k; ++i) r2[i] = 0.0;
    for (int j = 0; j < k; ++j) {
      for (int i = 0; i < k; ++i) u[i] = (i == j) ? 1.0 : 0.0;
      trisolve(R, rs, cs, k, u, 1, tv);
      for (int i = 0; i < k; ++i) r2[i] += tv[i] * tv[i];
    }
  }
  bool conv = false;
  while ((rrqr_iter < 0 || niter < rrqr_iter) && niter < kRrqrCapH) {
    double t2 = -1.0;
    int bi = 0, bj = 0;
    for (int j = 0; j < n - k; ++j)
      for (int i = 0; i < k; ++i) {
        const double tij = R[(int64_t)(i) * rs + (int64_t)(k + j) * cs];
        const double v = fabs(tij * tij + r2[i] * c2[j]);
        if (v > t2) {
          t2 = v;
          bi = i;
          bj = j;
        }
      }
    if (t2 <= f2) {
      conv = true;
      break;
    }
    ++niter;
    if (bi < k - 1) {  // swap i-th and k-th columns (id.m:132-138)
      int t = jpvt[bi];
      jpvt[bi] = jpvt[k - 1];
      jpvt[k - 1] = t;
      swap_retri(R, rs, cs, bi, k);
      for (int col = k; col < n; ++col) {
        double a = R[(int64_t)(bi) * rs + (int64_t)col * cs];
        R[(int64_t)(bi) * rs + (int64_t)col * cs] = R[(int64_t)(k - 1) * rs + (int64_t)col * cs];
        R[(int64_t)(k - 1) * rs + (int64_t)col * cs] = a;
      }
      double a = r2[bi];
      r2[bi] = r2[k - 1];
      r2[k - 1] = a;
    }
    if (bj > 0) {  // swap (k+1)-th and (k+j)-th columns (id.m:141-145)
      int t = jpvt[k];
      jpvt[k] = jpvt[k + bj];
      jpvt[k + bj] = t;
      for (int row = 0; row < rows; ++row) {
        double a = R[(int64_t)(row) * rs + (int64_t)k * cs];
        R[(int64_t)(row) * rs + (int64_t)k * cs] = R[(int64_t)(row) * rs + (int64_t)(k + bj) * cs];
        R[(int64_t)(row) * rs + (int64_t)(k + bj) * cs] = a;
      }
      double a = c2[0];
      c2[0] = c2[bj];
      c2[bj] = a;
    }
    // downdate inverse row norms (id.m:148-149)
    if (k > 1) {
      trisolve(R, rs, cs, k - 1, R + (int64_t)(k - 1) * cs, rs, tv);
      const double rkk = R[(int64_t)(k - 1) * rs + (int64_t)(k - 1) * cs];
      for (int i = 0; i < k - 1; ++i) r2[i] -= fabs(tv[i] / rkk) * fabs(tv[i] / rkk);
    }
    r2[k - 1] = 0.0;
    if (rows == k) {  // id.m:164-167
      for (int i = 0; i < k; ++i) u[i] = R[(int64_t)(i) * rs + (int64_t)k * cs];
      for (int i = 0; i < k; ++i) {
        double s = 0.0;
        for (int j = i; j < k; ++j) s += R[(int64_t)(i) * rs + (int64_t)j * cs] * u[j];
        tv[i] = s;
      }
      for (int i = 0; i < k; ++i) R[(int64_t)(i) * rs + (int64_t)k * cs] = tv[i];
      for (int i = 0; i < k - 1; ++i) R[(int64_t)(i) * rs + (int64_t)(k - 1) * cs] = 0.0;
      R[(int64_t)(k - 1) * rs + (int64_t)(k - 1) * cs] = 1.0;
    } else {  // id.m:168-198 (fixed-rank truncation leaves an R22 block)
      const int h = rows - k;   // length of the Householder vector
      double* v = tv;           // rows k..rows-1
      double nv = 0.0;
      for (int q = 0; q < h; ++q) v[q] = R[(int64_t)(k + q) * rs + (int64_t)k * cs];
      const double rkk1 = R[(int64_t)(k) * rs + (int64_t)k * cs];
      v[0] += sqrt(c2[0]) * (rkk1 < 0.0 ? -1.0 : 1.0);
      for (int q = 0; q < h; ++q) nv += v[q] * v[q];
      nv = sqrt(nv);
      for (int q = 0; q < h; ++q) v[q] /= nv;
      for (int col = k + 1; col < n; ++col) {
        double s = 0.0;
        for (int q = 0; q < h; ++q) s += v[q] * R[(int64_t)(k + q) * rs + (int64_t)col * cs];
        for (int q = 0; q < h; ++q) R[(int64_t)(k + q) * rs + (int64_t)col * cs] -= 2.0 * v[q] * s;
      }
      for (int q = 1; q < h; ++q) R[(int64_t)(k + q) * rs + (int64_t)k * cs] = 0.0;
      R[(int64_t)(k) * rs + (int64_t)k * cs] = sqrt(c2[0]);
      // restore entries of T to "R space"
      for (int i = 0; i < k; ++i) {
        double s = 0.0;
        for (int j = i; j < k; ++j) s += R[(int64_t)(i) * rs + (int64_t)j * cs] * R[(int64_t)(j) * rs + (int64_t)k * cs];
        u[i] = s;
      }
      for (int i = 0; i < k; ++i) R[(int64_t)(i) * rs + (int64_t)k * cs] = u[i];
      const double rkk = R[(int64_t)(k - 1) * rs + (int64_t)(k - 1) * cs];
      for (int col = k + 1; col < n; ++col) R[(int64_t)(k - 1) * rs + (int64_t)col * cs] *= rkk;
      // r = R(1:k,k) and s = R(k,k+2:end) are kept in aux tail
      double* rv = aux + 4 * n;       // k
      double* sv = aux + 5 * n;       // n - k - 1
      for (int i = 0; i < k; ++i) rv[i] = R[(int64_t)(i) * rs + (int64_t)(k - 1) * cs];
      for (int col = k + 1; col < n; ++col) sv[col - k - 1] = R[(int64_t)(k - 1) * rs + (int64_t)col * cs];
      for (int col = k; col < n; ++col) c2[col - k] -= R[(int64_t)(k) * rs + (int64_t)col * cs] * R[(int64_t)(k) * rs + (int64_t)col * cs];
      {  // MATLAB givens(R(k,k+1), R(k+1,k+1)) applied to rows k, k+1 over columns k..end
        const double a = R[(int64_t)(k - 1) * rs + (int64_t)k * cs], b = R[(int64_t)(k) * rs + (int64_t)k * cs];
        double c, s;
        if (a == 0.0) {
          c = 0.0;
          s = 1.0;
        } else {
          const double nr = hypot(a, b);
          c = fabs(a) / nr;
          s = (a < 0.0 ? -1.0 : 1.0) * (b / nr);
        }
        apply_rows(R, rs, cs, k - 1, k - 1, n, c, s);
      }
      for (int col = k; col < n; ++col) c2[col - k] += R[(int64_t)(k) * rs + (int64_t)col * cs] * R[(int64_t)(k) * rs + (int64_t)col * cs];
      c2[0] = R[(int64_t)(k) * rs + (int64_t)(k - 1) * cs] * R[(int64_t)(k) * rs + (int64_t)(k - 1) * cs];
      const double tmp = R[(int64_t)(k - 1) * rs + (int64_t)(k - 1) * cs];
      R[(int64_t)(k - 1) * rs + (int64_t)(k - 1) * cs] = rv[k - 1];
      trisolve(R, rs, cs, k, R + (int64_t)k * cs, rs, u);
      R[(int64_t)(k - 1) * rs + (int64_t)(k - 1) * cs] = tmp;
      trisolve(R, rs, cs, k - 1, rv, 1, tv);  // v = R(1:k-1,1:k-1)\r(1:k-1)
      R[(int64_t)(k - 1) * rs + (int64_t)(k - 1) * cs] /= rv[k - 1];
      const double rk = R[(int64_t)(k - 1) * rs + (int64_t)(k - 1) * cs];
      for (int i = 0; i < k - 1; ++i) R[(int64_t)(i) * rs + (int64_t)(k - 1) * cs] = tv[i] * (1.0 - rk);
      for (int col = k + 1; col < n; ++col) {
        const double ds = sv[col - k - 1] - R[(int64_t)(k - 1) * rs + (int64_t)col * cs];
        for (int i = 0; i < k - 1; ++i) R[(int64_t)(i) * rs + (int64_t)col * cs] += tv[i] / rv[k - 1] * ds;
        R[(int64_t)(k - 1) * rs + (int64_t)col * cs] /= rv[k - 1];
      }
    }
    // swap k-th and (k+1)-th columns; update inverse row norms (id.m:201-204)
    {
      int t = jpvt[k - 1];
      jpvt[k - 1] = jpvt[k];
      jpvt[k] = t;
      for (int row = 0; row < rows; ++row) {
        double a = R[(int64_t)(row) * rs + (int64_t)(k - 1) * cs];
        R[(int64_t)(row) * rs + (int64_t)(k - 1) * cs] = R[(int64_t)(row) * rs + (int64_t)k * cs];
        R[(int64_t)(row) * rs + (int64_t)k * cs] = a;
      }
    }
    if (k > 1) {
      trisolve(R, rs, cs, k - 1, R + (int64_t)(k - 1) * cs, rs, tv);
      const double rkk = R[(int64_t)(k - 1) * rs + (int64_t)(k - 1) * cs];
      for (int i = 0; i < k - 1; ++i) r2[i] += fabs(tv[i] / rkk) * fabs(tv[i] / rkk);
    }
    {
      const double rkk = R[(int64_t)(k - 1) * rs + (int64_t)(k - 1) * cs];
      r2[k - 1] = 1.0 / (rkk * rkk);
    }
    // Sherman-Morrison (id.m:207-208)
    u[k - 1] -= 1.0;
    for (int col = k; col < n; ++col) {
      const double a = R[(int64_t)(k - 1) * rs + (int64_t)col * cs] / (1.0 + u[k - 1]);
      for (int i = 0; i < k; ++i) R[(int64_t)(i) * rs + (int64_t)col * cs] -= u[i] * a;
    }
    // rank reduction (id.m:211-229)
    double rmin = HUGE_VAL;
    int imin = 0;
    for (int i = 0; i < k; ++i) {
      const double v = 1.0 / sqrt(r2[i]);
      if (v < rmin) {
        rmin = v;
        imin = i;
      }
    }
    if (rmin > tol) continue;
    if (imin < k - 1) {
      int t = jpvt[imin];
      jpvt[imin] = jpvt[k - 1];
      jpvt[k - 1] = t;
      swap_retri(R, rs, cs, imin, k);
      for (int col = k; col < n; ++col) {
        double a = R[(int64_t)(imin) * rs + (int64_t)col * cs];
        R[(int64_t)(imin) * rs + (int64_t)col * cs] = R[(int64_t)(k - 1) * rs + (int64_t)col * cs];
        R[(int64_t)(k - 1) * rs + (int64_t)col * cs] = a;
      }
      double a = r2[imin];
      r2[imin] = r2[k - 1];
      r2[k - 1] = a;
    }
    for (int j = 0; j <= n - k; ++j) c2[j] = 0.0;
    if (k > 1) {
      trisolve(R, rs, cs, k - 1, R + (int64_t)(k - 1) * cs, rs, tv);
      const double rkk = R[(int64_t)(k - 1) * rs + (int64_t)(k - 1) * cs];
      for (int i = 0; i < k - 1; ++i) r2[i] -= fabs(tv[i] / rkk) * fabs(tv[i] / rkk);
    }
    k -= 1;
    trisolve(R, rs, cs, k, R + (int64_t)k * cs, rs, tv);  // r = R(1:k,1:k)\R(1:k,k+1)
    for (int i = 0; i < k; ++i) R[(int64_t)(i) * rs + (int64_t)k * cs] = tv[i];
    for (int col = k + 1; col < n; ++col)
      for (int i = 0; i < k; ++i) R[(int64_t)(i) * rs + (int64_t)col * cs] += tv[i] * R[(int64_t)(k) * rs + (int64_t)col * cs];
    rows = k;
    if (k == 0) break;
  }
  *niter_out = niter;
  // id.m:232-235 warns whenever the loop ends unconverged, i.e. at rrqr_iter swaps
  // (or at the device's hard cap when rrqr_iter is Inf)
  *capped = (!conv && k > 0 && (niter >= kRrqrCapH || (rrqr_iter >= 0 && niter >= rrqr_iter))) ? 1 : 0;
  return k;
}

}  // namespace flam
