// Diagonal of the factored matrix or of its inverse by unfolding the
// factorization top-down (rskelf/rskelf_diag.m:95-177), one CTA per box.
//
// The reference unfolds into one global sparse matrix restricted to the entries
// later levels need.  Those entries are, for every box, the block of its
// skeletons -- and a box's skeletons all lie in its parent's point set.  So here
// every box keeps the whole unfolded block X over its own points, [rd sk] order:
// the box takes X(sk,sk) from its parent's block (the previous step top-down),
// undoes its own elimination and sparsification (dinv: the inverse operators), and
// writes X for its children.  Boxes that kept all their points pass the parent's
// block on unchanged.  diag(X) over the box's points is written each step; the
// deepest box containing a point writes last, which is the reference's final
// spdiags(M, 0).
#include "common.cuh"
#include "kernels.cuh"
#include "tile_f64.cuh"

namespace flam {
namespace {

__global__ void __launch_bounds__(kTileThreads) k_unfold(UnfoldArgs a) {
  __shared__ __align__(16) double tsm[kTileSmemDoubles];
  const UnfoldTask t = a.tasks[blockIdx.x];
  const int n = t.n, k = t.k, r = n - k;
  const int tid = threadIdx.x;
  constexpr int NT = kTileThreads;
  const int64_t* sk = a.ipool + t.ids_off;   // [sk | rd] global ids
  const int64_t* rd = sk + k;
  double* X = a.xcur + t.xout;               // n x n, ld n, local order [rd | sk]
  const int64_t ld = n;

  // X = [I 0; 0 X_parent(sk, sk)]
  for (int64_t e = tid; e < (int64_t)n * n; e += NT) {
    const int i = (int)(e % n), j = (int)(e / n);
    double v = 0.0;
    if (i < r || j < r) {
      v = (i == j) ? 1.0 : 0.0;
    } else {
      const int64_t pa = sk[i - r], pb = sk[j - r];
      const int64_t off = a.xoff[pa];
      if (off >= 0 && off == a.xoff[pb]) v = a.xprev[off + a.xpos[pa] + (int64_t)a.xpos[pb] * a.xld[pa]];
    }
    X[e] = v;
  }
  __syncthreads();
  // the children of this box read its block next step
  for (int q = tid; q < n; q += NT) {
    const int64_t pt = q < r ? rd[q] : sk[q - r];
    a.xoff[pt] = t.xout;
    a.xpos[pt] = q;
    a.xld[pt] = n;
  }

  if (r > 0) {
    const double* T = a.fpool + t.fac_off;   // k x r
    const double* LU = T + (int64_t)k * r;   // r x r
    const double* E = LU + (int64_t)r * r;   // k x r
    const double* G = E + (int64_t)k * r;    // r x k ('n', 's')
    const int32_t* p = a.ppool + t.piv_off;
    const bool chol = a.symm == 'p';
    const GV Xc_rd{X, 1, ld}, Xc_sk{X + (int64_t)r * ld, 1, ld};   // X(:,rd), X(:,sk)
    const GV Xr_rd{X, 1, ld}, Xr_sk{X + r, 1, ld};                  // X(rd,:), X(sk,:)
    const GV Gv = chol ? GV{E, k, 1} : GV{G, 1, r};                  // G = E' for chol
    auto Lf = [&](int i, int j) { return LU[i + (int64_t)j * r]; };  // L (strictly lower part for LU)
    auto Uf = [&](int i, int j) { return chol ? LU[j + (int64_t)i * r] : LU[i + (int64_t)j * r]; };
    double* tmp = a.tmp + t.tmp_off;          // n x r
    if (a.dinv) {
      // X(:,rd) = (X(:,rd) - X(:,sk) E) / L
      cta_gemm(X, 1, ld, Xc_sk, GV{E, 1, k}, n, r, k, -1.0, tsm);
      for (int i = tid; i < n; i += NT)
        for (int j = r - 1; j >= 0; --j) {
          double v = X[i + (int64_t)j * ld];
          for (int l = j + 1; l < r; ++l) v -= X[i + (int64_t)l * ld] * Lf(l, j);
          X[i + (int64_t)j * ld] = chol ? v / Lf(j, j) : v;
        }
      __syncthreads();
      // X(rd,:) = U \ (X(rd,:) - G X(sk,:))
      cta_gemm(X, 1, ld, Gv, Xr_sk, r, n, k, -1.0, tsm);
      for (int c = tid; c < n; c += NT)
        for (int j = r - 1; j >= 0; --j) {
          double v = X[j + (int64_t)c * ld];
          for (int l = j + 1; l < r; ++l) v -= Uf(j, l) * X[l + (int64_t)c * ld];
          X[j + (int64_t)c * ld] = v / Uf(j, j);
        }
      __syncthreads();
      if (!chol) {   // X(:,rd(p)) = X(:,rd)
        for (int64_t e = tid; e < (int64_t)n * r; e += NT) tmp[e] = X[e];
        __syncthreads();
        for (int64_t e = tid; e < (int64_t)n * r; e += NT) {
          const int i = (int)(e % n), j = (int)(e / n);
          X[i + (int64_t)p[j] * ld] = tmp[e];
        }
        __syncthreads();
      }
      // X(:,sk) -= X(:,rd) T';  X(sk,:) -= T X(rd,:)
      cta_gemm(X + (int64_t)r * ld, 1, ld, Xc_rd, GV{T, k, 1}, n, k, r, -1.0, tsm);
      cta_gemm(X + r, 1, ld, GV{T, 1, k}, Xr_rd, k, n, r, -1.0, tsm);
    } else {
      // X(:,sk) += X(:,rd) G;  X(sk,:) += E X(rd,:)
      cta_gemm(X + (int64_t)r * ld, 1, ld, Xc_rd, Gv, n, k, r, 1.0, tsm);
      cta_gemm(X + r, 1, ld, GV{E, 1, k}, Xr_rd, k, n, r, 1.0, tsm);
      // X(:,rd) = X(:,rd) U
      for (int i = tid; i < n; i += NT)
        for (int j = r - 1; j >= 0; --j) {
          double v = 0.0;
          for (int l = 0; l <= j; ++l) v += X[i + (int64_t)l * ld] * Uf(l, j);
          X[i + (int64_t)j * ld] = v;
        }
      __syncthreads();
      // X(rd,:) = L X(rd,:)
      for (int c = tid; c < n; c += NT)
        for (int j = r - 1; j >= 0; --j) {
          double v = chol ? Lf(j, j) * X[j + (int64_t)c * ld] : X[j + (int64_t)c * ld];
          for (int l = 0; l < j; ++l) v += Lf(j, l) * X[l + (int64_t)c * ld];
          X[j + (int64_t)c * ld] = v;
        }
      __syncthreads();
      if (!chol) {   // X(rd(p),:) = X(rd,:)
        for (int64_t e = tid; e < (int64_t)r * n; e += NT) {
          const int j = (int)(e % r), c = (int)(e / r);
          tmp[e] = X[j + (int64_t)c * ld];
        }
        __syncthreads();
        for (int64_t e = tid; e < (int64_t)r * n; e += NT) {
          const int j = (int)(e % r), c = (int)(e / r);
          X[p[j] + (int64_t)c * ld] = tmp[e];
        }
        __syncthreads();
      }
      // X(:,rd) += X(:,sk) T;  X(rd,:) += T' X(sk,:)
      cta_gemm(X, 1, ld, Xc_sk, GV{T, 1, k}, n, r, k, 1.0, tsm);
      cta_gemm(X, 1, ld, GV{T, k, 1}, Xr_sk, r, n, k, 1.0, tsm);
    }
  }
  __syncthreads();
  for (int q = tid; q < n; q += NT) {
    const int64_t pt = q < r ? rd[q] : sk[q - r];
    a.D[pt] = X[q + (int64_t)q * ld];
  }
}

}  // namespace

void launch_unfold(const UnfoldArgs& a, int ntask, cudaStream_t s) {
  if (ntask > 0) k_unfold<<<ntask, kTileThreads, 0, s>>>(a);
}

}  // namespace flam
