// Launch interfaces of the factorization and sweep kernels.
#pragma once
#include "common.cuh"

namespace flam {

struct CompressArgs {
  Problem P;
  const CompressTask* tasks;
  int64_t* ipool;      // slf lists (reordered to [sk rd])
  int64_t* cpool;      // neighbour candidates (filtered in place)
  double* tpool;       // T slots
  int32_t* permpool;   // local permutations
  double* scratch;     // work matrices of boxes with n > kSmemN
  CompressOut* out;
  double rel_tol;      // rem(rank_or_tol, 1)
  int kmax;            // floor(rank_or_tol)
  int symm_n;          // 1: compress [A(nbr,slf); A(slf,nbr)'; Kpxy] (symm 'n')
  double Tmax;
  int64_t rrqr_iter;   // < 0: unlimited
  const double* Aexp;  // explicit m x n matrix (flam_id); rows are generated from points when null
  int64_t lda;
  int32_t* mfilt;      // per box (out_idx): candidates kept by the neighbour filter (row-split form)
  const double* ypool; // row sketches of the sketched boxes (CompressTask::ax_off)
};

size_t compress_smem_bytes(int n);
int64_t compress_scratch_doubles(int n);
void launch_compress(const CompressArgs& a, int ntask, size_t smem, cudaStream_t s);

// Thread-per-column compress (compress_tc.cu) for n <= kTcMaxN: nt threads per box
// (compress_tc_threads(n)), work arrays of compress_tc_doubles(n) in shared memory
// when they fit kTcSmemMax, else in the task's global scratch.
constexpr int kTcMaxN = 1024;
// Work arrays above the tuned tc_smem_max bytes (flam_tune) go to global scratch (L2):
// by default only the small boxes (n <~ 64) keep R in shared memory, larger ones read it
// from L2 with a one-step prefetch, which leaves room for more CTAs per SM.
int64_t compress_tc_doubles(int n);
size_t compress_tc_smem_bytes(int n);
int compress_tc_threads(int n);
int compress_tc_group(int n);
int compress_tc_rows(int n);
void launch_compress_tc(const CompressArgs& a, int ntask, int nt, int b, int g, size_t smem, cudaStream_t s);
// ID of the explicit row sketch of boxes with n > kTcMaxN (ax_rows <= 1024 rows), one CTA
// per box; scratch: cpqr_wide_scratch_doubles(n) at the task's scr_off.
int64_t cpqr_wide_scratch_doubles(int n);
void launch_cpqr_wide(const CompressArgs& a, int ntask, cudaStream_t s);
// The same with every pivot step spread over the GPU (fewer wide boxes than SMs): 2 launches per step
// for `steps` steps (>= min(rows, n) of every task), per-task state of
// cpqr_grid_state_bytes(ntask) bytes in device memory.
size_t cpqr_grid_state_bytes(int ntask);
// wmax: the most sketch rows of a task (at most kSketchMaxW).
void launch_cpqr_grid(const CompressArgs& a, int ntask, int nmax, int wmax, int steps, void* state, cudaStream_t s);
// Sketch rows the single-CTA form (launch_cpqr_wide) takes at most.
int cpqr_wide_max_rows();
// Neighbour filter alone (row-split form): tasks[0, ntask) compact their candidates
// and write the kept count to a.mfilt[out_idx].
void launch_filter(const CompressArgs& a, int ntask, cudaStream_t s);

struct ElimArgs {
  Problem P;
  const ElimTask* tasks;
  const ChildBlock* children;
  const int64_t* ipool;
  const double* tpool;
  const int32_t* permpool;
  const double* m_in;   // children's M blocks
  double* m_out;        // this step's M blocks
  double* fpool;        // factors
  int32_t* ppool;       // LU permutations
  double* scratch;      // work matrices of boxes with n > kSmemN
  int32_t* status;      // OR of StatusBits
  int symm;             // 'n', 's', 'p', 'h'
  int pan_rows;         // big boxes: rows of the LU panel staged in shared memory (0: none)
};

size_t elim_smem_bytes(int n);
int elim_pan_rows_max();
int64_t elim_scratch_doubles(int n);
// tasks[0, nsmall): n <= kSmemN (shared-memory kernel); tasks[nsmall, nsmall + nbig): the rest.
void launch_eliminate(const ElimArgs& a, int nsmall, int nbig, size_t smem, cudaStream_t s);
// Boxes a.tasks[0, nbox) (work matrices in global scratch) eliminated by grid-wide launches:
// batched FP64 tensor-path GEMMs and one CTA per box for each LU panel.  nmax, kmax, rmax:
// the largest n, k and r among them.
void launch_eliminate_huge(const ElimArgs& a, int nbox, int nmax, int kmax, int rmax, cudaStream_t s);
int elim_huge_launches(int rmax, int kmax, bool chol);
// The solve sweep (op 0 upward, 1 downward; rskelf_sv_*.m) of a factor with no skeletons
// (k = 0: the root) and a large redundant block, spread over the GPU: its rows of the
// point-major work array W gathered into the dense r x nrhs block X (device scratch),
// blocked triangular solves with the factor's LU (or L) block -- diagonal blocks one
// thread per right-hand side, off-diagonal updates as FP64 tensor-path GEMMs -- and
// scattered back.  Returns the number of launches.
int sweep_root_grid(double* W, int nrhs, const int64_t* rd, const int32_t* perm, const double* LU, int r, int op,
                    int trans, int symm, double* X, cudaStream_t s);
// Factors with no skeletons and at least this many redundant rows take sweep_root_grid.
constexpr int kRootGridR = 1024;
// Redundant blocks from this size up take the grid-wide elimination.
constexpr int kHugeR = 320;

// Segmented copies of int64 ids: dst[dst_off + i] = src[src_off + i], i < len.
struct CopySeg {
  int64_t src_off, dst_off, len;
};
void launch_gather_ids(const int64_t* src, int64_t* dst, const CopySeg* segs, int nseg, cudaStream_t s);

// Sweeps over the factors of one step (rskelf_sv_*.m / rskelf_mv_*.m).
// op: 0 sv upward, 1 sv downward, 2 mv upward, 3 mv downward; trans 0 = 'n', 1 = 'c'/'t'.
struct SweepArgs {
  const FacDesc* fac;
  const int64_t* ipool;
  const double* fpool;
  const int32_t* ppool;
  double* X;            // point-major: X[pt * ldx + c]
  int64_t ldx;
  int nrhs;
  int op;
  int trans;
  int symm;
};
void launch_sweep(const SweepArgs& a, int nfac, int kmax, int rmax, cudaStream_t s);
// Whether a step's sweep keeps its tiles in shared memory (otherwise it allocates scratch).
bool sweep_in_smem(int kmax, int rmax, int op);

// Layout changes for the user's column-major X (N x nrhs, ld) <-> point-major work array.
void launch_to_pointmajor(const double* X, int64_t ld, int64_t N, int nrhs, double* W, cudaStream_t s);
void launch_from_pointmajor(const double* W, int64_t N, int nrhs, double* X, int64_t ld, cudaStream_t s);
// Rows idx (n of them) of the point-major W <-> column-major n x nrhs Y; dir 0 gathers, 1 scatters.
void launch_rows_pm(double* W, int nrhs, const int64_t* idx, int64_t n, double* Y, int dir, cudaStream_t s);

// Top-down unfolding for rskelf_diag (diag.cu): one task per box of a step.
struct UnfoldTask {
  int64_t ids_off;   // ipool offset of the box's [sk | rd] ids
  int64_t fac_off;   // fpool offset of its factor [T | LU | E | G] (unused when r == 0)
  int64_t piv_off;   // ppool offset of its LU permutation
  int64_t xout;      // this box's n x n block in the current step's pool
  int64_t tmp_off;   // n x r doubles of work space
  int32_t n, k;
};
struct UnfoldArgs {
  const UnfoldTask* tasks;
  const int64_t* ipool;
  const double* fpool;
  const int32_t* ppool;
  const double* xprev;  // blocks of the step above
  double* xcur;         // blocks of this step
  int64_t* xoff;        // per point: its block's offset (-1: none yet)
  int32_t* xpos;        // per point: its row in that block
  int32_t* xld;         // per point: that block's order
  double* tmp;
  double* D;            // per point: the diagonal
  int dinv;
  int symm;
};
void launch_unfold(const UnfoldArgs& a, int ntask, cudaStream_t s);

// Per-factor log-determinant terms of one step: out[2f] = sum log|diag| (x2 if chol),
// out[2f+1] = parity of (negative diagonal entries + inversions of p).
void launch_logdet(const FacDesc* fac, int nfac, const double* fpool, const int32_t* ppool, int chol, double* out,
                   cudaStream_t s);

}  // namespace flam
