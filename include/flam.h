/*
 * flam.h -- C ABI of the B200 (sm_100a) recursive skeletonization factorization.
 *
 * This is the drop-in boundary for the reference's MATLAB/Octave entry points
 *
 *   F = rskelf(A, x, occ, rank_or_tol, pxyfun, opts)   rskelf/rskelf.m:109
 *   Y = rskelf_sv(F, X, trans)                          rskelf/rskelf_sv.m:13
 *   Y = rskelf_mv(F, X, trans)                          rskelf/rskelf_mv.m:13
 *   T = hypoct(x, occ, lvlmax, ext)                     core/hypoct.m:51
 *   P = hypoct_perm(T)                                  core/hypoct_perm.m:11
 *
 * A MEX/oct gateway (or ctypes, cgo, JNI ...) binds these symbols.  The
 * reference's function handles A(I,J) and pxyfun(x,slf,nbr,l,ctr) are
 * replaced by registry descriptors (flam_kernel, flam_proxy): the matrix is
 * evaluated on the device, there is no callback into the host and no CPU
 * fallback.
 *
 * Conventions
 *   - Arrays are column-major like MATLAB: x is d x N (point-major), X is
 *     N x nrhs with leading dimension ldx.
 *   - Pointers may be host or device memory; the library detects which.
 *   - Index arrays returned by the export calls are 0-based; a MATLAB
 *     gateway adds 1.
 *   - Every call returns a flam_status; flam_last_error() gives the message,
 *     prefixed with the reference's error identifier ("FLAM:id:...").
 *   - A handle is bound to the device that was current when it was created
 *     and to the stream given in flam_opts (0: the legacy default stream).
 *     Calls on one handle must not run concurrently from several threads.
 */
#ifndef FLAM_B200_H
#define FLAM_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define FLAM_API __attribute__((visibility("default")))
#else
#define FLAM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  FLAM_OK = 0,
  FLAM_ERR_ARG = 1,          /* invalid argument (FLAM:chksymm, FLAM:hypoct, FLAM:id ...) */
  FLAM_ERR_NOT_SPD = 2,      /* chol of a redundant block failed (symm = 'p') */
  FLAM_ERR_CUDA = 3,         /* a CUDA runtime call failed */
  FLAM_ERR_NOMEM = 4,        /* device allocation failed */
  FLAM_ERR_UNSUPPORTED = 5,  /* option not available on the device path */
  FLAM_ERR_TIMEOUT = 6,      /* a bounded device wait gave up (the sketch kernel's mbarrier) */
  FLAM_WARN_RRQR_MAXITER = 100, /* FLAM:id:maxIterCount (factor is still valid) */
  FLAM_WARN_SINGULAR = 101,     /* an LU pivot of a redundant block was exactly zero */
  FLAM_WARN_IR_NOT_CONVERGED = 102, /* refinement stopped above ir_tol (X is the last iterate) */
  FLAM_WARN_LDL_AS_LU = 103         /* symm 'h' factored with LU, FLAM:rskelf:octaveLDL (rskelf.m:124-127) */
} flam_status;

/* Kernel registry: the matrix entry is A(i,j) = scale * w_j * K(x_i, x_j) for
 * i != j and A(i,i) = dval.  Kernels follow the reference's test drivers. */
typedef enum {
  FLAM_KERNEL_LAPLACE2D = 0,     /* -log(r)/(2 pi)             rskelf/test/ie_circle.m:85-95   */
  FLAM_KERNEL_LAPLACE2D_DL = 1,  /* (r . n_j)/(2 pi r^2)       rskelf/test/ie_circle.m:91-94   */
  FLAM_KERNEL_LAPLACE3D = 2,     /* 1/(4 pi r)                 rskelf/test/ie_cube1.m:115-121  */
  FLAM_KERNEL_GAUSSIAN = 3,      /* exp(-(param r)^2/2)        rskelf/test/cov_circle1.m:130   */
  FLAM_KERNEL_MATERN32 = 4       /* (1+sqrt3 param r)e^{-sqrt3 param r} rskelf/test/cov_circle2.m:129 */
} flam_kernel_kind;

typedef struct {
  int kind;               /* flam_kernel_kind */
  double scale;           /* multiplies every off-diagonal entry */
  double dval;            /* diagonal value A(i,i) */
  double param;           /* inverse length scale for GAUSSIAN / MATERN32 */
  const double* weights;  /* N column weights, or NULL (all ones) */
  const double* normals;  /* d x N source normals (LAPLACE2D_DL), or NULL */
} flam_kernel;

/* Proxy registry (replaces pxyfun): far field of a box of size l, centre c. */
typedef enum {
  FLAM_PROXY_NONE = 0,    /* no pxyfun: naive global compression (rskelf.m:204) */
  FLAM_PROXY_RING = 1,    /* p points 1.5(cos t, sin t).*l + c, ellipse filter   ie_circle.m:35,106-115 */
  FLAM_PROXY_SPHERE = 2,  /* p Fibonacci points radius 1.5 .*l + c, ellipsoid filter  ie_cube1.m:131-140 */
  FLAM_PROXY_ANNULUS = 3  /* base*t + 1.5 base.*l + c, t in [0, 3/param], box filter  cov_circle1.m:34-40,146-152 */
} flam_proxy_kind;

typedef struct {
  int kind;          /* flam_proxy_kind */
  int p;             /* number of reference points (directions for ANNULUS) */
  int p_rad;         /* ANNULUS: radii per direction */
  int kernel_kind;   /* kernel evaluated between proxy and box points */
  double scale;      /* multiplies the proxy block */
  double param;      /* kernel parameter for the proxy kernel */
  int two_sided;     /* 1: rows [K diag(w_slf); wbar K] for weighted unsymmetric matrices */
} flam_proxy;

typedef struct {
  int lvlmax;            /* maximum tree depth; <= 0 means Inf           (rskelf.m:114) */
  const double* ext;     /* d x 2 root extent or NULL                     (rskelf.m:115) */
  double Tmax;           /* ID entry bound, >= 1; INFINITY disables RRQR  (rskelf.m:116) */
  int64_t rrqr_iter;     /* max RRQR iterations; < 0 means Inf            (rskelf.m:117) */
  char symm;             /* 'n', 's', 'h' or 'p'                          (rskelf.m:118) */
  int stop;              /* stop after this many levels; < 0 means Inf    (rskelf.m:119) */
  int verb;              /* 1: print the per-level table                  (rskelf.m:120) */
  void* stream;          /* cudaStream_t the handle runs on (NULL: default stream) */
  int profile;           /* 1: time every launch with CUDA events (see flam_profile) */
  /* Sketched (mixed-precision) compression -- not in the reference.  0: the reference's
   * ID of the full block K (id.m).  1: the ID of a row sketch Y = Omega K (Omega w x m,
   * +-1 entries) formed in FP32 on the tensor cores (K split into two TF32 parts),
   * with the FP64 pivoted QR, rank and R11 \ R12 on Y; boxes of more than 8192 points
   * use the exact ID.  A box whose rank comes within sketch_guard of w is redone with a
   * second sketch at full width, or exactly when that fills too (the posterior check).  Meant for loose tolerances (>= ~1e-7: the sketch carries
   * ~21 bits) followed by flam_rskelf_ir_sv.  2: the same sketched ID with K's entries and
   * the products in FP64 (FP64 tensor path), for tight tolerances without refinement.
   * Other values: FLAM_ERR_ARG (FLAM:rskelf:invalidSketch). */
  int sketch;
  int sketch_p;          /* sketch rows beyond the rank estimate (default 8; w >= 8) */
  int sketch_guard;      /* posterior check margin in rows (default 2) */
  unsigned sketch_seed;  /* seed of Omega */
  const void* predictor; /* flam_predictor* giving each box's rank estimate, or NULL:
                            w = n + sketch_p (never below the rank) */
  int rank_log;          /* 1: keep every box's features and rank (flam_rank_log) */
} flam_opts;

typedef struct flam_factor flam_factor;

/* Fill opts with the reference defaults (rskelf.m:112-120). */
FLAM_API void flam_opts_default(flam_opts* opts);

/* F = rskelf(A, x, occ, rank_or_tol, pxyfun, opts)   rskelf/rskelf.m:109-309 */
FLAM_API flam_status flam_rskelf(const double* x, int d, int64_t N, const flam_kernel* A, double occ,
                        double rank_or_tol, const flam_proxy* pxy, const flam_opts* opts,
                        flam_factor** F);

/* T = hypoct(x, occ, lvlmax, ext) alone: a handle holding only the tree
 * (read it with flam_tree_export / flam_tree_perm).  lvlmax <= 0 means Inf,
 * ext is d x 2 or NULL.   core/hypoct.m:51-171 */
FLAM_API flam_status flam_hypoct(const double* x, int d, int64_t N, double occ, int lvlmax, const double* ext,
                                 void* stream, flam_factor** T);

/* [sk, rd, T] = id(A, rank_or_tol, Tmax, rrqr_iter) on the device for an
 * explicit m x n matrix (leading dimension lda, host or device memory).
 * Outputs (host): *k, perm (n entries: sk = perm[0:k], rd = perm[k:n]),
 * T (k x (n-k), leading dimension k) and *niter.  core/id.m:44-248 */
FLAM_API flam_status flam_id(const double* A, int64_t m, int64_t n, int64_t lda, double rank_or_tol, double Tmax,
                             int64_t rrqr_iter, int64_t* k, int64_t* perm, double* T, int64_t* niter);

/* Column limit of flam_id_noalloc. */
#define FLAM_ID_NOALLOC_NMAX 128

/* The device's RRQR loop stops after this many swaps when rrqr_iter is Inf. */
#define FLAM_RRQR_HARD_CAP 4096

/* flam_id without device allocation -- no counterpart in the reference.
 * For callers that cannot allocate device memory (a MEX/oct gateway running
 * inside a MATLAB or Octave session whose GPU memory manager owns the device
 * heap, a thread that must not enter cudaMalloc/cudaFree): the caller passes
 * DEVICE pointers on the current device for the m x n matrix A (leading
 * dimension lda) and for every output -- *k, perm (n entries, sk = perm[0:k],
 * rd = perm[k:n]), T (room for n*n/4 + 1 doubles; written k x (n-k), leading
 * dimension k) and *niter (may be NULL) -- and the work runs asynchronously on
 * `stream` (NULL: legacy default stream).  Because the call does not wait for
 * the GPU it cannot return flam_id's FLAM_WARN_RRQR_MAXITER: the RRQR loop
 * stopped unconverged at its limit exactly when *niter equals rrqr_iter (or
 * FLAM_RRQR_HARD_CAP when rrqr_iter < 0).  n = 0 writes *k = *niter = 0.
 * Scratch is a 64 KiB array compiled into the library, resident on every GPU
 * that loads it until the process exits; n is limited to
 * FLAM_ID_NOALLOC_NMAX (larger n returns FLAM_ERR_ARG).  The first call on a
 * device looks up that array's address with the device current; make that
 * first call before any stream capture.  All calls share the array: calls that
 * overlap on one GPU race and must be serialised by the caller.
 * Same algorithm and results as flam_id. */
FLAM_API flam_status flam_id_noalloc(const double* A, int64_t m, int64_t n, int64_t lda, double rank_or_tol,
                                     double Tmax, int64_t rrqr_iter, int64_t* k, int64_t* perm, double* T,
                                     int64_t* niter, void* stream);

/* Many independent problems in one pipeline: instance i has N[i] points at
 * x + d * (N[0] + ... + N[i-1]) and matrix A[i].  Every step of the
 * factorization runs all instances' boxes of the matching level in one launch.
 * Semantically identical to ninst calls of flam_rskelf. */
FLAM_API flam_status flam_rskelf_batched(int ninst, const double* x, int d, const int64_t* N,
                                const flam_kernel* A, double occ, double rank_or_tol,
                                const flam_proxy* pxy, const flam_opts* opts, flam_factor** F);

/* Y = rskelf_sv(F, X, trans), in place on X (N x nrhs, leading dim ldx).
 * rskelf/rskelf_sv.m:13-36.  For a batched handle N is the total over instances. */
FLAM_API flam_status flam_rskelf_sv(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans);

/* Y = rskelf_mv(F, X, trans), in place.  rskelf/rskelf_mv.m:13-36. */
FLAM_API flam_status flam_rskelf_mv(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans);

/* Y = rskelf_cholmv(F, X, trans): Y = C X ('n') or C' X ('t'/'c') for F = C C', in place.
 * One half of the 'p' multiply: the downward half for 'n', the upward half otherwise.
 * rskelf/rskelf_cholmv.m:15-50.  F must have symm 'p' (FLAM:rskelf_cholmv:invalidSymm). */
FLAM_API flam_status flam_rskelf_cholmv(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans);

/* Y = rskelf_cholsv(F, X, trans): Y = C \ X ('n') or C' \ X, in place.  The upward half of
 * the 'p' solve for 'n', the downward half otherwise.  rskelf/rskelf_cholsv.m:15-50. */
FLAM_API flam_status flam_rskelf_cholsv(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans);

/* ld = rskelf_logdet(F): log det of the factored matrix, one complex number per instance
 * (re[i] + 1i*im[i], im in [0, 2 pi)).  rskelf/rskelf_logdet.m:11-33: 2 sum log diag(L)
 * for 'p'; sum log diag(U) + log detperm(p) for 'n'/'s'.  Either pointer may be NULL. */
FLAM_API flam_status flam_rskelf_logdet(const flam_factor* F, double* re, double* im);

/* D = rskelf_diag(F, dinv) / rskelf_spdiag(F, dinv): the diagonal of the factored
 * matrix (dinv = 0) or of its inverse (dinv = 1), N values (all instances, host or device
 * memory).  rskelf/rskelf_diag.m:35-185 (unfolding of the factorization top-down) and
 * rskelf/rskelf_spdiag.m:19-85 compute the same D; this library unfolds box by box on the
 * device.  symm 'n', 's', 'p'; a complete factorization made by flam_rskelf*
 * (FLAM:rskelf_diag:partial for opts.stop, FLAM:rskelf_diag:noTree for imported factors). */
FLAM_API flam_status flam_rskelf_diag(const flam_factor* F, int dinv, double* D);

/* The remaining skeleton system of a partial factorization (opts.stop), per instance:
 * [Si, S] = rskelf_partial_info(F) -- rskelf/rskelf_partial_info.m:12-20, assembled as in
 * rskelf/rskelf.m:278-308.  The skeleton block left to the caller is A(Si,Si) + S.
 * flam_partial_sizes gives Sn = numel(Si) and nnz(S); flam_partial_export fills Si (Sn,
 * 0-based, ascending, instance-local) and S in compressed-column form (colptr: Sn+1, rowind
 * and val: nnz; rows ascending in each column, exact zeros dropped like MATLAB's sparse).
 * A complete factorization has Sn = 0.  Any output pointer may be NULL. */
FLAM_API flam_status flam_partial_sizes(const flam_factor* F, int inst, int64_t* Sn, int64_t* nnz);
FLAM_API flam_status flam_partial_export(const flam_factor* F, int inst, int64_t* Si, int64_t* colptr,
                                         int64_t* rowind, double* val);

/* Device handle from a factorization given on the host in the reference's F layout
 * (rskelf.m:157-159,249-257): N, symm and factors(1..nfac) in application order, sk and rd
 * 0-based.  Factorizations produced elsewhere in rskelf format are applied this way: the
 * hifie2/hifie3 factorizations, whose hifie_sv/mv/cholsv/cholmv/logdet are rskelf_sv/...
 * on that F (hifie/hifie_sv.m:21), or a factorization saved from a MATLAB session.
 * Factor j (k_j = |sk|, r_j = |rd|) occupies, one factor after another: sk (k_j), rd (r_j),
 * T (k_j x r_j), L (r_j x r_j), U (r_j x r_j; NULL for 'p'), p (r_j; NULL for 'p'),
 * E (k_j x r_j), G (r_j x k_j, the reference's field F; NULL for 'p'), column-major.
 * Consecutive factors with disjoint index sets are applied in one launch; a factor that
 * touches an index of the current group starts the next, so the factors act in the
 * reference's loop order.  symm 'n', 's' or 'p'; the handle runs on `stream`.
 * Errors: FLAM:gpu:invalidFactor (an index outside [0, N), repeated inside a factor, a
 * permutation entry outside [0, r), a missing array). */
FLAM_API flam_status flam_factor_import(int64_t N, char symm, int64_t nfac, const int64_t* k, const int64_t* r,
                                        const int64_t* sk, const int64_t* rd, const double* T, const double* L,
                                        const double* U, const int64_t* p, const double* E, const double* G,
                                        void* stream, flam_factor** F);

/* Callback applying the remaining skeleton system: Y (n x nrhs, column-major, leading
 * dimension n, DEVICE memory) holds X(Si,:) of every instance in instance order; the
 * callback overwrites it with svfun(Y, trans) / mvfun(Y, trans) and returns 0, or returns
 * nonzero to abort.  Y is valid in stream order on `stream` (the handle's stream); work the
 * callback enqueues elsewhere must complete before it returns.  trans is 'n' or 'c'. */
typedef int (*flam_skel_fn)(double* Y, int64_t n, int64_t nrhs, char trans, void* stream, void* ctx);

/* Y = rskelf_partial_sv(F, X, svfun, trans), in place: upward sweep, fn on X(Si,:),
 * downward sweep.  rskelf/rskelf_partial_sv.m:23-62 ('t' is handled as 'c': real data). */
FLAM_API flam_status flam_rskelf_partial_sv(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans,
                                            flam_skel_fn fn, void* ctx);

/* Y = rskelf_partial_mv(F, X, mvfun, trans), in place.  rskelf/rskelf_partial_mv.m:23-62. */
FLAM_API flam_status flam_rskelf_partial_mv(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans,
                                            flam_skel_fn fn, void* ctx);

/* Y = A X, or Y = B - A X when B is not NULL: the handle's registry matrix (block
 * diagonal over the instances of a batched handle) applied in FP64, evaluated on the
 * fly -- the O(N^2) product the reference's tests form from A(I,J) to measure errors
 * (rskelf/test/ie_circle.m:47-48, ie_ellipse.m:51-80).  X, B, Y are N x nrhs with
 * leading dimensions ldx, ldb, ldy, host or device memory; Y may not alias X.
 * Errors: FLAM:gpu:noMatrix for imported factors (no matrix). */
FLAM_API flam_status flam_matvec(const flam_factor* F, const double* X, int64_t ldx, int64_t nrhs, const double* B,
                                 int64_t ldb, double* Y, int64_t ldy);

/* X = A \ B by iterative refinement on the factorization F of A: X = F \ B
 * (rskelf_sv), then X += F \ (B - A X) with the FP64 residual of flam_matvec
 * until max_j ||B_j - A X_j|| / ||B_j|| <= ir_tol or max_iter refinement steps.
 * For symm 'p' (A and F positive definite) the steps are conjugate gradients
 * preconditioned by F, which also converge when A's conditioning spreads the
 * spectrum of F \ A beyond what stationary refinement contracts.
 * F may be a loose (larger rank_or_tol) factorization; the returned error is the
 * FP64 relative residual per column (relres, nrhs entries, may be NULL), and
 * *iters the refinement steps taken.  FLAM_WARN_IR_NOT_CONVERGED when the
 * tolerance was not met.  No counterpart in the reference (its users pass
 * rskelf_sv as a preconditioner to an iterative solver, ie_square1.m:102). */
FLAM_API flam_status flam_rskelf_ir_sv(const flam_factor* F, const double* B, int64_t ldb, double* X, int64_t ldx,
                                       int64_t nrhs, double ir_tol, int max_iter, int* iters, double* relres);

/* Learned rank predictor -- no counterpart in the reference.  A BF16 MLP
 * 16 -> 128 -> 128 -> 1 (ReLU, sigmoid output) that maps 16 features of a box (point
 * count, neighbour count, -log10 tol, aspect, depth, point spread and offset moments,
 * proxy use, dimension, kernel) to its ID rank as a fraction of its point count; with
 * opts.sketch and opts.predictor the sketch of a box has w = ceil(pred * n) + sketch_p
 * rows, and the posterior check sends a box whose rank fills its sketch back to the
 * exact ID (core/id.m, the judge of the prediction).  Training and inference run on the
 * GPU with the library's own kernels (tensor-core BF16 products, FP32 accumulation,
 * FP32 master weights, Adam).  Parameters: FP32, layout W1 (128 x 16, row-major) | b1 |
 * W2 (128 x 128) | b2 | W3 (128) | b3.  The object lives on the device that was current
 * at creation; its calls run on the legacy default stream. */
#define FLAM_PREDICTOR_NFEAT 16
#define FLAM_PREDICTOR_NPARAM 18817
typedef struct flam_predictor flam_predictor;
FLAM_API flam_status flam_predictor_create(uint64_t seed, flam_predictor** P);
FLAM_API void flam_predictor_free(flam_predictor* P);
FLAM_API flam_status flam_predictor_get(const flam_predictor* P, float* w);
FLAM_API flam_status flam_predictor_set(flam_predictor* P, const float* w);
/* Adam on mean (pred - y)^2 over nsamp samples (X: nsamp x 16 row-major, y: nsamp; host
 * or device memory), `epochs` passes in shuffled minibatches of `batch`; *loss (may be
 * NULL) gets the last epoch's mean loss. */
FLAM_API flam_status flam_predictor_train(flam_predictor* P, const float* X, const float* y, int64_t nsamp, int epochs,
                                          int batch, float lr, uint64_t seed, float* loss);
FLAM_API flam_status flam_predictor_eval(const flam_predictor* P, const float* X, int64_t nsamp, float* yhat);
/* One forward and backward pass: *loss = mean (pred - y)^2 and grad (NPARAM floats) its
 * gradient, for checking the training kernels. */
FLAM_API flam_status flam_predictor_grad(const flam_predictor* P, const float* X, const float* y, int64_t nsamp,
                                         float* loss, float* grad);
/* The features (count x 16) and rank fractions k/n (count) of every compressed box of a
 * factorization made with opts.rank_log; call with X = y = NULL for *count. */
FLAM_API flam_status flam_rank_log(const flam_factor* F, int64_t* count, float* X, float* y);

/* Launch shapes of the factorization, per device and problem class -- not in the
 * reference.  A step with few boxes splits each box of more than split_min_n points over
 * up to split_max CTAs (row-split compression with pairwise merges) so that the step
 * fills about split_ctas CTAs; work matrices of up to tc_smem_max bytes stay in shared
 * memory.  flam_autotune measures candidate settings on a given problem (coordinate
 * search, device time of the factorization) and records the fastest for its class
 * (dimension, kernel, log2 N) on the current device; every later factorization of that
 * class on that device uses it.  flam_tune_get / flam_tune_set read and write the
 * table (to save a tuning and load it in another process). */
typedef struct {
  int split_ctas;   /* CTAs a few-box step aims at (default 148, the SM count) */
  int split_max;    /* row-split parts per box at most (default 8) */
  int split_min_n;  /* boxes above this many points are split (default 32) */
  int tc_smem_max;  /* bytes of work matrix kept in shared memory (default 40960) */
} flam_tune;
FLAM_API flam_status flam_autotune(const double* x, int d, int64_t N, const flam_kernel* A, double occ,
                                   double rank_or_tol, const flam_proxy* pxy, const flam_opts* opts, int reps,
                                   flam_tune* best);
FLAM_API flam_status flam_tune_get(int d, int kernel_kind, int64_t N, flam_tune* t);
FLAM_API flam_status flam_tune_set(int d, int kernel_kind, int64_t N, const flam_tune* t);

/* Sizes of a handle. */
typedef struct {
  int64_t N;          /* total points */
  int ninst;          /* instances */
  int d;
  char symm;
  int64_t nbox;       /* tree boxes (all instances) */
  int nlvl_max;       /* deepest tree */
  int64_t nfactor;    /* stored box factors */
  int nstep;          /* factorization steps (levels processed, deepest instance) */
  int64_t bytes;      /* device bytes held by the factor (pools) */
  int64_t nrem;       /* points left uneliminated (partial factorization) */
  double t_tree, t_factor;  /* seconds on the device (CUDA events) */
} flam_info;

FLAM_API flam_status flam_factor_info(const flam_factor* F, flam_info* info);

/* Tree of instance `inst`, the reference's T = hypoct(...) struct flattened:
 * nlvl, lvp (nlvl+1), l (d x nlvl), and per box ctr (d), prnt, children,
 * neighbours and points as CSR arrays.  Call once with all array pointers NULL
 * to get the sizes in *nbox, *nchld_tot, *nnbor_tot, *npts_tot, then again
 * with host arrays of those sizes.   core/hypoct.m:15-37 */
FLAM_API flam_status flam_tree_export(const flam_factor* F, int inst, int* nlvl, int64_t* nbox,
                             int64_t* nchld_tot, int64_t* nnbor_tot, int64_t* npts_tot,
                             int64_t* lvp, double* l, double* ctr, int64_t* prnt,
                             int64_t* chld_ptr, int64_t* chld, int64_t* nbor_ptr, int64_t* nbor,
                             int64_t* xi_ptr, int64_t* xi);

/* P = hypoct_perm(T) for instance `inst` (N[inst] entries, 0-based). core/hypoct_perm.m:11-39 */
FLAM_API flam_status flam_tree_perm(const flam_factor* F, int inst, int64_t* P);

/* Factor list of instance `inst`: F.lvp (nstep+1 entries) and, per factor,
 * k = |sk|, r = |rd|.  Arrays may be NULL to query *nfac / *nlvp. */
FLAM_API flam_status flam_factor_sizes(const flam_factor* F, int inst, int64_t* nfac, int* nlvp,
                              int64_t* lvp, int64_t* k, int64_t* r);

/* Factor j of instance `inst` (rskelf.m:249-257): sk (k), rd (r), T (k x r),
 * L (r x r), U (r x r), p (r), E (k x r), G (r x k).  Any pointer may be NULL.
 * symm 'p': U, p, G untouched.  symm 'h': U holds the block-diagonal D, p and G untouched. */
FLAM_API flam_status flam_factor_export(const flam_factor* F, int inst, int64_t j, int64_t* sk, int64_t* rd,
                               double* T, double* L, double* U, int64_t* p, double* E, double* G);

/* Per-level table of opts.verb (rskelf.m:267-272) for instance `inst`:
 * rows of (lvl, nblk, nrem1, nrem2); returns the row count in *nrows. */
FLAM_API flam_status flam_level_stats(const flam_factor* F, int inst, int* nrows, int64_t* rows);

FLAM_API void flam_factor_free(flam_factor* F);

/* The library keeps the work buffers of factorizations and sweeps per
 * (device, stream) and reuses them (they only grow), so steady-state calls
 * allocate no device memory.  This returns that memory to the device pool;
 * call it with no library work in flight (it synchronises those streams). */
FLAM_API void flam_workspace_release(void);

/* Launch accounting of a handle (factorization and every sv/mv call since the
 * last reset): device time per kernel family from CUDA events on the handle's
 * stream, and the algorithmic work those launches did (flops of the
 * reference's dense operations on each box, bytes of factor and X traffic). */
typedef struct {
  int64_t launches;                       /* all kernels this library launched */
  int64_t n_compress, n_elim, n_sweep;    /* launches of each hot kernel */
  double t_compress, t_elim, t_sweep;     /* seconds (0 unless profiling is on) */
  double flop_compress, flop_elim, flop_sweep;
  double byte_sweep;
  int64_t n_sketch;        /* boxes whose ID came from a row sketch (opts.sketch) */
  int64_t n_sketch_redo;   /* of those, boxes the posterior check sent to the exact ID */
  int64_t sketch_rows;     /* sum over the sketched boxes of their sketch rows w */
  int64_t sketch_rows_k;   /* sum over the same boxes of rows(K), the rows the exact ID folds */
  int64_t id_rows;         /* rows every ID of the factorization folded (w if sketched, else rows(K)) */
  int64_t graph_replays;   /* applies run as a replayed CUDA graph of their sweep launches */
  /* executed work of the sketched form (t_compress and flop_compress count the reference's
   * operations on the full blocks K, which the sketch replaces) */
  double t_sketch;         /* seconds in the row-sketch launches (part of t_compress) */
  double flop_sketch;      /* their products: 2 w rows(K) n per sketch (x2 for the TF32 hi/lo split) */
  double flop_id;          /* pivoted QR + R11 \ R12 as run: on the w sketch rows, else on K */
} flam_prof;

FLAM_API flam_status flam_profile(const flam_factor* F, flam_prof* out, int reset);

/* Message of the last failed call on this thread ("FLAM:<fn>:<id>: text"). */
FLAM_API const char* flam_last_error(void);

/* Library version string. */
FLAM_API const char* flam_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FLAM_B200_H */
