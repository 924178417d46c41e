// Internal declarations shared by the device kernels and the host driver.
//
// Layout in HBM (all instances of a batched handle share every pool):
//   x        d x Ntot FP64, point-major (MATLAB's column-major d x N)
//   ipool    int64 point ids: [ tree permutation (Ntot) | per-step slf lists ]
//            a box's current point list ("xi" in rskelf.m) is a slice of it
//   fpool    FP64 factors, per factor [T (k x r) | LU (r x r) | E (k x r) | G (r x k)]
//   ppool    int32 LU row permutations, r per factor
// Every matrix is column-major.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace flam {

constexpr int kMaxDim = 3;
constexpr int kWarp = 32;
// Boxes with more points than this keep their work matrices in global
// scratch instead of shared memory.
constexpr int kSmemN = 128;
// Hard cap on RRQR swaps per box (the reference loops until convergence;
// each swap grows |det R11| by more than Tmax, so the cap is never met on
// well-posed input -- it only bounds the device loop).
constexpr int kRrqrCap = 4096;

enum KernelKind { K_LAPLACE2D = 0, K_LAPLACE2D_DL = 1, K_LAPLACE3D = 2, K_GAUSSIAN = 3, K_MATERN32 = 4 };
enum ProxyKind { P_NONE = 0, P_RING = 1, P_SPHERE = 2, P_ANNULUS = 3 };

// Per-instance matrix and proxy parameters.
struct InstParams {
  int64_t pt_off;   // first global point id of the instance
  int64_t N;
  int kind;         // KernelKind
  int has_w;        // column weights present
  double scale, dval, param, wbar;
  int pkind;        // ProxyKind
  int pkernel;      // kernel of the proxy block
  double pscale, pparam;
  int two_sided;
  int has_nrm;
};

// Device view of the problem.
struct Problem {
  int d;
  const double* x;        // d x Ntot
  const double* w;        // Ntot or null
  const double* nrm;      // d x Ntot or null
  const InstParams* ip;   // per instance
  const double* pxy_pts;  // d x npxy reference proxy points
  const double* pxy_shift;// d x npxy (annulus) or null
  int npxy;               // reference proxy points (rows of one proxy block)
};

// One box of a factorization step (compress kernel).
struct CompressTask {
  int64_t slf_off;   // slf list in ipool (int64 ids); reordered in place to [sk rd]
  int64_t cand_off;  // neighbour candidates in cpool
  int64_t T_off;     // T slot (k x r, ld k) in tpool
  int64_t perm_off;  // local permutation (n int32) in perm pool
  int64_t scr_off;   // global scratch (doubles) for n > kSmemN, else -1
  int32_t n;         // |slf|
  int32_t ncand;
  int32_t box;
  int32_t inst;
  int32_t flags;     // bit0: compress with proxy (lvl > 2); bit1: filter candidates
  int32_t out_idx;   // slot of this box in the CompressOut array
  double ctr[kMaxDim];
  double l[kMaxDim];
  // Row-split form for boxes of the few-box levels: the rows of K are divided into
  // nparts parts whose R factors are merged pairwise.  mode 0: the whole ID in one
  // CTA; 1: R of rows [part*m/nparts, (part+1)*m/nparts) into this task's R area;
  // 2: fold the triangular R at rsrc_off into this task's R (merge); 3: as 2, then
  // the rest of the ID.  Modes 1-3 read the filtered candidate count from mfilt.
  int32_t mode;
  int32_t part, nparts;
  int32_t depth;     // tree level of the box (box features of the rank predictor)
  int64_t rsrc_off;
  // Sketched form: with ax_rows > 0 the rows of the block are the explicit ax_rows x n
  // matrix (column-major, leading dimension ax_rows) at ax_off of the sketch pool -- the
  // box's row sketch Y = Omega K -- instead of rows generated from the points, and the
  // result is flagged ST_ID_CHECK when the rank exceeds ax_rows - ax_guard.
  int64_t ax_off;
  int32_t ax_rows;
  int32_t ax_guard;
};

// Per-box results of the compress kernel.
struct CompressOut {
  int32_t k;         // skeleton count
  int32_t m;         // rows of the compressed block
  int32_t niter;     // RRQR swaps
  int32_t status;    // bit0: RRQR hit its cap
};

// Children block of the modified diagonal block M (rskelf.m:190-199).
struct ChildBlock {
  int32_t coff;      // offset of the child's points inside the parent's slf
  int32_t kc;        // child's |xi|
  int64_t M_off;     // child's M (kc x kc) in the M pool read this step
};

// One box of the elimination kernel.
struct ElimTask {
  int64_t slf_off;   // [sk rd] global ids in ipool
  int64_t T_off;     // T slot from compress
  int64_t perm_off;  // local permutation from compress
  int64_t M_out;     // M_new (k x k, or n x n when r == 0) in the M pool written this step
  int64_t fac_off;   // factor block in fpool (-1 when r == 0)
  int64_t piv_off;   // LU permutation in ppool
  int64_t scr_off;   // global scratch (n x n doubles) for n > kSmemN, else -1
  int32_t n, k;
  int32_t inst;
  int32_t ch_first;  // first ChildBlock
  int32_t nch;
  int32_t pad;
};

// A stored factor, read by the sweeps (rskelf.m:249-257).
struct FacDesc {
  int64_t sk_off;    // ipool offset of sk (k ids) followed by rd (r ids)
  int64_t T_off, LU_off, E_off, G_off;  // fpool offsets
  int64_t piv_off;   // ppool offset
  int32_t k, r;
};

// Record the message flam_last_error() returns on this thread (defined with the C ABI).
void set_last_error(const char* msg);

// Raise `func`'s dynamic shared-memory limit to `bytes` on the current device.
// Function attributes are per device, so this runs once per (kernel, device),
// under a lock; a failure is not remembered (the next launch tries again) and
// leaves the CUDA error pending for the caller's cudaGetLastError().
// Returns the result of cudaFuncSetAttribute (cudaSuccess once done).
cudaError_t ensure_smem_attr(const void* func, int bytes);

// Factorization status word bits (device -> host).
// ST_ID_CHECK: a sketched ID used (nearly) all of its sketch rows, so the sketch may
// have cut the numerical rank; ST_TIMEOUT: a bounded device wait gave up.
enum StatusBits { ST_NOT_SPD = 1, ST_SINGULAR = 2, ST_RRQR_CAP = 4, ST_ID_CHECK = 8, ST_TIMEOUT = 16 };

// ---------------------------------------------------------------- device helpers
#ifdef __CUDACC__

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Kernel value K(xt, xs) for target xt and source xs (source normal ns).
__device__ __forceinline__ double keval(int kind, double param, int d, const double* xt, const double* xs,
                                        const double* ns) {
  double dx0 = xt[0] - xs[0];
  double dx1 = d > 1 ? xt[1] - xs[1] : 0.0;
  double dx2 = d > 2 ? xt[2] - xs[2] : 0.0;
  double r2 = dx0 * dx0 + dx1 * dx1 + dx2 * dx2;
  switch (kind) {
    case K_LAPLACE2D:
      return -0.07957747154594767 * log(r2);   // -log(r)/(2 pi) = -log(r^2)/(4 pi)
    case K_LAPLACE2D_DL: {
      double rdotn = dx0 * ns[0] + dx1 * ns[1];
      return 0.15915494309189535 * rdotn / r2;  // 1/(2 pi)
    }
    case K_LAPLACE3D:
      return 0.07957747154594767 * rsqrt(r2);  // 1/(4 pi r)
    case K_GAUSSIAN: {
      double dr2 = param * param * r2;
      return exp(-0.5 * dr2);
    }
    default: {  // K_MATERN32
      double dr = 1.7320508075688772 * param * sqrt(r2);
      return (1.0 + dr) * exp(-dr);
    }
  }
}

// A(i, j) of instance ip for global point ids i, j.
__device__ __forceinline__ double aentry(const Problem& P, const InstParams& ip, int64_t i, int64_t j) {
  if (i == j) return ip.dval;
  const int d = P.d;
  double v = ip.scale * keval(ip.kind, ip.param, d, P.x + i * d, P.x + j * d,
                              ip.has_nrm ? P.nrm + j * d : nullptr);
  if (ip.has_w) v *= P.w[j];
  return v;
}

// Row `type` of a box's compression block K at column point sc (rskelf.m:201-212):
// 0 A(q, sc) for a neighbour q, 1 A(sc, q)' (the transposed block of symm 'n'),
// 2 the proxy row at point y (multiplier wmul, or the column's weight when 0), 3 zero.
__device__ __forceinline__ double block_entry(const Problem& P, const InstParams& ip, int type, int64_t q,
                                              const double* y, double wmul, int64_t sc) {
  switch (type) {
    case 0:
      return aentry(P, ip, q, sc);
    case 1:
      return aentry(P, ip, sc, q);
    case 2: {
      const double v = ip.pscale * keval(ip.pkernel, ip.pparam, P.d, y, P.x + sc * P.d, nullptr);
      if (wmul != 0.0) return v * wmul;
      return ip.has_w ? v * P.w[sc] : v;
    }
    default:
      return 0.0;
  }
}

#endif  // __CUDACC__

}  // namespace flam
