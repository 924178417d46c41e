// Host driver and C ABI (include/flam.h).
//
// The host plans, the device computes.  After the device builds the forest
// (tree.cu), its arrays are copied to the host once; every factorization step
// is then planned on the host from the skeleton counts the previous step
// returned (one small device-to-host copy per step), and executed as four
// launches: id gathers (slf lists and neighbour candidates), the fused
// compress kernel, and the elimination kernel.
//
// Reference loop being replaced: rskelf/rskelf.m:168-263.  Steps run the
// boxes of every instance whose level is (its depth - step), leaves first.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/flam.h"
#include "common.cuh"
#include "kernels.cuh"
#include "matvec.cuh"
#include "predictor.cuh"
#include "scan.cuh"
#include "sketch.cuh"
#include "tree.cuh"

namespace flam {
namespace {

thread_local std::string g_err;

struct FlamError : std::runtime_error {
  flam_status code;
  FlamError(flam_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void fail(flam_status c, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  throw FlamError(c, buf);
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      fail(e_ == cudaErrorMemoryAllocation ? FLAM_ERR_NOMEM : FLAM_ERR_CUDA, "FLAM:gpu:cuda: %s (%s:%d)", \
           cudaGetErrorString(e_), __FILE__, __LINE__);                                   \
  } while (0)

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// Growable device array on one stream.
template <class T>
struct DBuf {
  T* p = nullptr;
  int64_t n = 0, cap = 0;
  void reserve(int64_t c, cudaStream_t s) {
    if (c <= cap) return;
    int64_t nc = std::max<int64_t>(c, 2 * cap);
    nc = std::max<int64_t>(nc, 16);
    T* q = nullptr;
    CK(cudaMallocAsync(reinterpret_cast<void**>(&q), sizeof(T) * nc, s));
    if (n > 0) CK(cudaMemcpyAsync(q, p, sizeof(T) * n, cudaMemcpyDeviceToDevice, s));
    if (p) CK(cudaFreeAsync(p, s));
    p = q;
    cap = nc;
  }
  void resize(int64_t c, cudaStream_t s) {
    reserve(c, s);
    n = c;
  }
  void upload(const std::vector<T>& v, cudaStream_t s) {
    n = 0;
    resize((int64_t)v.size(), s);
    if (!v.empty()) CK(cudaMemcpyAsync(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
  }
  void release(cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = cap = 0;
  }
  // size c without keeping the old contents (work buffers)
  void ensure(int64_t c, cudaStream_t s) {
    if (c > cap) {
      if (p) CK(cudaFreeAsync(p, s));
      p = nullptr;
      cap = 0;
      n = 0;
      reserve(c, s);
    }
    n = c;
  }
  int64_t bytes() const { return cap * (int64_t)sizeof(T); }
};

template <class T>
std::vector<T> download(const T* p, int64_t n, cudaStream_t s) {
  std::vector<T> v((size_t)n);
  if (n > 0) CK(cudaMemcpyAsync(v.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return v;
}

// FP64 work of an ID as run on `rows` x n rows (the TSQR fold when rows > n, then k
// pivoted Householder steps on the n x n R and R11 \ R12).
double id_flops(double rows, double n, double k) {
  double f = 0.0;
  if (rows > n) f += 2 * rows * n * n - 2.0 / 3.0 * n * n * n;
  const double a = std::min(rows, n);
  k = std::min(k, a);
  f += 4 * a * n * k - 2 * (a + n) * k * k + 4.0 / 3.0 * k * k * k;
  return f + k * k * (n - k);
}

struct HostFac {
  int inst, step;
  int64_t sk_off;
  int32_t k, r;
  int64_t fac_off, piv_off;
};

// A box of a factorization step, for the top-down unfolding of rskelf_diag: its
// [sk rd] ids at ipool[slf_off, slf_off + n), k skeletons, and its factor (index
// into hfac) or -1 when the box kept all its points (r = 0).
struct BoxRec {
  int64_t slf_off;
  int32_t n, k;
  int64_t fac;
};

// An M block left when an instance stops: rows/columns ipool[idx_off, idx_off + n),
// values (column-major n x n) at val_off of the host copy.
struct KeptBlock {
  int inst;
  int64_t idx_off, n, val_off;
};

struct StepDev {
  DBuf<FacDesc> fac;
  int nfac = 0, kmax = 0, rmax = 0;
  double flop_per_rhs = 0;   // sum over factors of 4kr + r^2 (one direction, one right-hand side)
  double fac_bytes = 0;      // sum of 8 (2kr + r^2): factor data one direction reads
  double x_rows = 0;         // sum of k + r
  // Factors with no skeletons and r >= kRootGridR (the root of a problem that stops
  // with a large block): the solve sweeps run them grid-wide (sweep_root_grid) and the
  // per-box sweep kernel takes the rest, listed in sfac with maxima skmax / srmax.
  std::vector<FacDesc> roots;
  DBuf<FacDesc> sfac;
  int nsfac = 0, skmax = 0, srmax = 0;

  // Fill from the step's factor list (in hfac order: the log-determinant indexes by it).
  void set(const std::vector<FacDesc>& fd, cudaStream_t s) {
    fac.upload(fd, s);
    nfac = (int)fd.size();
    std::vector<FacDesc> rest;
    for (const FacDesc& f : fd) {
      const double k = f.k, r = f.r;
      kmax = std::max(kmax, f.k);
      rmax = std::max(rmax, f.r);
      flop_per_rhs += 4 * k * r + r * r;
      fac_bytes += 8 * (2 * k * r + r * r);
      x_rows += k + r;
      if (f.k == 0 && f.r >= kRootGridR) {
        roots.push_back(f);
      } else {
        rest.push_back(f);
        skmax = std::max(skmax, f.k);
        srmax = std::max(srmax, f.r);
      }
    }
    if (!roots.empty()) sfac.upload(rest, s);
    nsfac = (int)rest.size();
  }
  int root_rmax() const {
    int m = 0;
    for (const FacDesc& f : roots) m = std::max(m, f.r);
    return m;
  }
};

struct LevelStat {
  int64_t lvl, nblk, nrem1, nrem2;
};

// Work buffers of the factorization steps and the sweeps, kept per (device,
// stream) for the life of the process and only ever grown: after the first
// call no step allocates device memory (a fresh pool allocation of the
// multi-hundred-MB sweep buffer can cost the driver hundreds of ms).  Calls on
// one stream run in order, so they can share it; flam_workspace_release()
// returns the memory.
struct Workspace {
  // final sizes of the last factorizations on this stream: a new factorization
  // reserves its factor pools at these sizes once instead of growing them step by
  // step (each growth is an allocation plus a copy; large stream-ordered
  // allocations can cost the driver hundreds of ms when the pool is fragmented)
  int64_t hint_ipool = 0, hint_fpool = 0, hint_ppool = 0;
  DBuf<int64_t> cpool;
  DBuf<double> tpool, scratch, mpool[2], W, tmp;
  DBuf<int32_t> permpool, status, mfilt;
  DBuf<CompressTask> ctask;
  DBuf<ElimTask> etask;
  DBuf<ChildBlock> chb;
  DBuf<CopySeg> segs, csegs;
  DBuf<CompressOut> cout;
  // FP64 products with the registry matrix and iterative refinement (matvec.cu)
  DBuf<MatvecTile> mvt;
  // sketched compression: row sketches, their tasks, rows of K per box, boxes redone exactly
  DBuf<double> ypool;
  DBuf<SketchTask> sktask;
  DBuf<CompressTask> skfilt, redo_task, wtask, rsk_task;
  DBuf<int32_t> mrows, redo_idx;
  DBuf<CompressTask> ftask;
  DBuf<unsigned char> gwstate;
  DBuf<float> feat, fyhat;
  DBuf<double> irB, irX, irR, irW, colsq;
  cudaStream_t copy = nullptr;   // host<->device copies overlapped with the sweeps
  cudaStream_t cap = nullptr;    // stream the sweep graphs are captured on
  // side streams for the independent launches of one step (the kernel shapes of a
  // compress segment, the two elimination kernels): forked from the step's stream
  // by one event and joined back by one event each
  static constexpr int kSide = 6;
  cudaStream_t side[kSide] = {};
  cudaEvent_t fork = nullptr, join[kSide] = {};
  // The elimination of a step runs on its own two streams (boxes with n <= 128 and
  // larger ones) while the host plans the next step and its compress runs: the
  // T / permutation / scratch pools alternate between two sets by step parity, and
  // edone[parity][stream] marks the end of that step's elimination kernels.
  DBuf<double> tpool_b, scratch_b;
  DBuf<int32_t> permpool_b;
  cudaStream_t es[2] = {};
  cudaEvent_t ecomp = nullptr, eprep = nullptr, edone[2][2] = {};
  void ensure_side() {
    if (fork) return;
    CK(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    for (int i = 0; i < kSide; ++i) {
      CK(cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming));
    }
    CK(cudaEventCreateWithFlags(&ecomp, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&eprep, cudaEventDisableTiming));
    for (int i = 0; i < 2; ++i) {
      CK(cudaStreamCreateWithFlags(&es[i], cudaStreamNonBlocking));
      for (int j = 0; j < 2; ++j) CK(cudaEventCreateWithFlags(&edone[i][j], cudaEventDisableTiming));
    }
  }
  // s waits for the elimination kernels of the steps with parity par
  void wait_elim(cudaStream_t s, int par) {
    CK(cudaStreamWaitEvent(s, edone[par][0], 0));
    CK(cudaStreamWaitEvent(s, edone[par][1], 0));
  }
  // side streams 0..nuse-1 wait for the work issued on s so far
  void fork_to(cudaStream_t s, int nuse) {
    CK(cudaEventRecord(fork, s));
    for (int i = 0; i < nuse; ++i) CK(cudaStreamWaitEvent(side[i], fork, 0));
  }
  // s waits for the work issued on side streams 0..nuse-1
  void join_to(cudaStream_t s, int nuse) {
    for (int i = 0; i < nuse; ++i) {
      CK(cudaEventRecord(join[i], side[i]));
      CK(cudaStreamWaitEvent(s, join[i], 0));
    }
  }
  void release(cudaStream_t s) {
    if (cap) {
      cudaStreamDestroy(cap);
      cap = nullptr;
    }
    if (copy) {
      cudaStreamSynchronize(copy);
      cudaStreamDestroy(copy);
      copy = nullptr;
    }
    if (fork) {
      for (int i = 0; i < kSide; ++i) {
        cudaStreamSynchronize(side[i]);
        cudaStreamDestroy(side[i]);
        cudaEventDestroy(join[i]);
        side[i] = nullptr;
        join[i] = nullptr;
      }
      cudaEventDestroy(fork);
      fork = nullptr;
      for (int i = 0; i < 2; ++i) {
        cudaStreamSynchronize(es[i]);
        cudaStreamDestroy(es[i]);
        es[i] = nullptr;
        for (int j = 0; j < 2; ++j) {
          cudaEventDestroy(edone[i][j]);
          edone[i][j] = nullptr;
        }
      }
      cudaEventDestroy(ecomp);
      cudaEventDestroy(eprep);
      ecomp = eprep = nullptr;
    }
    tpool_b.release(s);
    scratch_b.release(s);
    permpool_b.release(s);
    for (auto* b : {&tpool, &scratch, &mpool[0], &mpool[1], &W, &tmp, &irB, &irX, &irR, &irW, &colsq}) b->release(s);
    mvt.release(s);
    ypool.release(s);
    sktask.release(s);
    skfilt.release(s);
    redo_task.release(s);
    wtask.release(s);
    mrows.release(s);
    redo_idx.release(s);
    ftask.release(s);
    gwstate.release(s);
    feat.release(s);
    fyhat.release(s);
    cpool.release(s);
    permpool.release(s);
    status.release(s);
    mfilt.release(s);
    ctask.release(s);
    etask.release(s);
    chb.release(s);
    segs.release(s);
    csegs.release(s);
    cout.release(s);
  }
};

// ---------------------------------------------------------------- launch-shape tuning
// Table of tuned launch shapes per (device, dimension, kernel kind, log2 N).
struct TuneKey {
  int dev, d, kind, lg;
  bool operator<(const TuneKey& o) const {
    return std::tie(dev, d, kind, lg) < std::tie(o.dev, o.d, o.kind, o.lg);
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, flam_tune> g_tune;

flam_tune tune_default() { return flam_tune{148, 8, 32, 40 * 1024}; }

TuneKey tune_key(int dev, int d, int kind, int64_t N) {
  int lg = 0;
  while ((int64_t(1) << (lg + 1)) <= std::max<int64_t>(N, 1)) ++lg;
  return TuneKey{dev, d, kind, lg};
}

flam_tune tune_lookup(const TuneKey& k) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(k);
  return it == g_tune.end() ? tune_default() : it->second;
}

void tune_check(const flam_tune& t) {
  if (t.split_ctas < 1 || t.split_max < 1 || t.split_min_n < 1 || t.tc_smem_max < 0 || t.tc_smem_max > 200 * 1024)
    fail(FLAM_ERR_ARG, "FLAM:tune:invalidArg: split_ctas, split_max, split_min_n >= 1, 0 <= tc_smem_max <= 204800");
}

std::mutex g_ws_mu;
std::map<std::pair<int, cudaStream_t>, std::unique_ptr<Workspace>> g_ws;

Workspace& workspace(int dev, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(g_ws_mu);
  auto& w = g_ws[{dev, s}];
  if (!w) w.reset(new Workspace());
  return *w;
}

}  // namespace
}  // namespace flam

using namespace flam;

struct flam_factor {
  int dev = 0;
  cudaStream_t s = nullptr;
  int d = 0, ninst = 0;
  int64_t Ntot = 0;
  char symm = 'n';
  std::vector<int64_t> inst_off;
  std::vector<InstParams> iph;
  // device inputs
  DBuf<double> x, w, nrm, pxy_pts, pxy_shift;
  DBuf<InstParams> ip;
  int npxy = 0;
  bool has_w = false, has_nrm = false;
  // tree (host mirror)
  int64_t nbox = 0;
  std::vector<int64_t> lvb;  // global depth pointers
  std::vector<int32_t> prnt, chfirst, nch, depth, binst;
  std::vector<int64_t> seg_start, seg_len, nbor_ptr;
  std::vector<int32_t> nbor;
  std::vector<double> ctr, lsz;
  std::vector<int> nlvl;     // per instance
  DBuf<int64_t> hperm;       // hypoct_perm, global positions
  // factor
  DBuf<int64_t> ipool;
  DBuf<double> fpool;
  DBuf<int32_t> ppool;
  std::vector<StepDev> steps;
  int root_rmax = 0;   // largest r of a grid-swept root factor (its r x nrhs scratch follows W)
  std::vector<HostFac> hfac;
  std::vector<std::vector<int64_t>> inst_fac;     // per instance: indices into hfac
  std::vector<std::vector<int64_t>> inst_lvp;     // per instance F.lvp
  std::vector<std::vector<LevelStat>> stats;
  std::vector<std::vector<BoxRec>> step_boxes;    // per step, every box (rskelf_diag)
  std::vector<int64_t> rem;  // remaining points per instance
  // partial factorization (rskelf.m:278-308): per instance the remaining skeletons Si
  // (instance-local, ascending) and S in compressed-column form
  std::vector<std::vector<int64_t>> Si, Scp, Sri;
  std::vector<std::vector<double>> Sv;
  DBuf<int64_t> Si_dev;      // global ids of every instance's Si, instance order
  int64_t Sn_tot = 0;
  double t_tree = 0, t_factor = 0;
  int64_t warn = 0;
  std::vector<float> rlog_X, rlog_y;   // opts.rank_log: features and k/n of every compressed box
  bool profile = false;
  mutable flam_prof prof{};
  // CUDA graphs of the sweep launches of an apply, by (X, ld, nrhs, trans, solve, halves,
  // work array): the second apply with the same key captures, later ones replay
  struct GraphKey {
    const void* X;
    int64_t ld, nrhs;
    int t, solve, halves;
    const void* W;
    bool operator<(const GraphKey& o) const {
      return std::tie(X, ld, nrhs, t, solve, halves, W) < std::tie(o.X, o.ld, o.nrhs, o.t, o.solve, o.halves, o.W);
    }
  };
  struct GraphRec {
    cudaGraphExec_t exec;
    flam_prof delta;   // the accounting of one apply's launches
  };
  mutable std::map<GraphKey, GraphRec> graphs;
  mutable std::map<GraphKey, int> graph_seen;
  mutable cudaEvent_t pend[2] = {nullptr, nullptr};   // sweep timing not yet read
  mutable bool has_pend = false;
  void resolve_pending() const {
    if (!has_pend) return;
    float ms = 0;
    if (cudaEventSynchronize(pend[1]) == cudaSuccess && cudaEventElapsedTime(&ms, pend[0], pend[1]) == cudaSuccess)
      prof.t_sweep += ms * 1e-3;
    cudaEventDestroy(pend[0]);
    cudaEventDestroy(pend[1]);
    has_pend = false;
  }

  ~flam_factor() {
    resolve_pending();
    for (auto& g : graphs) cudaGraphExecDestroy(g.second.exec);
    const bool any = x.p || ipool.p || fpool.p || ppool.p || hperm.p || ip.p || !steps.empty();
    if (!any) return;   // nothing on the device (e.g. a handle that failed before its uploads)
    cudaStream_t st = s;
    x.release(st);
    w.release(st);
    nrm.release(st);
    pxy_pts.release(st);
    pxy_shift.release(st);
    ip.release(st);
    hperm.release(st);
    ipool.release(st);
    fpool.release(st);
    ppool.release(st);
    Si_dev.release(st);
    for (auto& q : steps) q.fac.release(st);
    cudaStreamSynchronize(st);
  }
};

struct flam_predictor {
  int dev = 0;
  DBuf<float> w, m, v, grad, scal, X, y, yhat;
  int step = 0;
  ~flam_predictor() {
    for (auto* b : {&w, &m, &v, &grad, &scal, &X, &y, &yhat}) b->release(nullptr);
    cudaStreamSynchronize(nullptr);
  }
};

namespace flam {
namespace {

// --------------------------------------------------------------- registry setup
void proxy_points(const flam_proxy& px, int d, std::vector<double>& pts, std::vector<double>& shift) {
  const double pi = 3.14159265358979323846;
  pts.clear();
  shift.clear();
  auto fib = [&](int p, double rad, std::vector<double>& out) {
    out.resize((size_t)p * 3);
    for (int i = 0; i < p; ++i) {
      double z = 1.0 - (2.0 * i + 1.0) / p;
      double rr = std::sqrt(std::max(0.0, 1.0 - z * z));
      double phi = i * pi * (3.0 - std::sqrt(5.0));
      out[i * 3 + 0] = rad * rr * std::cos(phi);
      out[i * 3 + 1] = rad * rr * std::sin(phi);
      out[i * 3 + 2] = rad * z;
    }
  };
  if (px.kind == FLAM_PROXY_RING) {
    pts.resize((size_t)px.p * 2);
    for (int j = 0; j < px.p; ++j) {
      double t = (j + 1) * 2 * pi / px.p;
      pts[j * 2] = 1.5 * std::cos(t);
      pts[j * 2 + 1] = 1.5 * std::sin(t);
    }
  } else if (px.kind == FLAM_PROXY_SPHERE) {
    fib(px.p, 1.5, pts);
  } else if (px.kind == FLAM_PROXY_ANNULUS) {
    std::vector<double> base;
    if (d == 2) {
      base.resize((size_t)px.p * 2);
      for (int j = 0; j < px.p; ++j) {
        double t = (j + 1) * 2 * pi / px.p;
        base[j * 2] = std::cos(t);
        base[j * 2 + 1] = std::sin(t);
      }
    } else {
      fib(px.p, 1.0, base);
    }
    for (int j = 0; j < px.p; ++j) {
      double mx = 0;
      for (int q = 0; q < d; ++q) mx = std::max(mx, std::fabs(base[j * d + q]));
      for (int q = 0; q < d; ++q) base[j * d + q] /= mx;
    }
    const int nr = px.p_rad;
    const double R = 3.0 / px.param;
    pts.resize((size_t)px.p * nr * d);
    shift.resize((size_t)px.p * nr * d);
    for (int jr = 0; jr < nr; ++jr) {
      double rad = nr > 1 ? (jr == nr - 1 ? R : jr * (R / (nr - 1))) : 0.0;
      for (int j = 0; j < px.p; ++j)
        for (int q = 0; q < d; ++q) {
          pts[((size_t)jr * px.p + j) * d + q] = base[j * d + q] * rad;
          shift[((size_t)jr * px.p + j) * d + q] = 1.5 * base[j * d + q];
        }
    }
  }
}

// Stream-ordered allocations come from the device's default pool; keep freed
// memory in the pool instead of returning it to the driver at every
// synchronisation, so the per-level work buffers are recycled, not remapped.
// (Process-local runtime state; nothing about the GPU itself changes.)
void keep_pool_memory(int dev) {
  static bool done[64] = {};
  if (dev < 0 || dev >= 64 || done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  done[dev] = true;
}

char chksymm(char c) {
  c = (char)std::tolower((unsigned char)c);
  if (c != 'n' && c != 's' && c != 'h' && c != 'p')
    fail(FLAM_ERR_ARG, "FLAM:chksymm:invalidSymm: Symmetry parameter must be one of 'N', 'S', 'H', or 'P'.");
  return c;
}

char chktrans(char c) {
  c = (char)std::tolower((unsigned char)c);
  if (c != 'n' && c != 't' && c != 'c')
    fail(FLAM_ERR_ARG, "FLAM:chktrans:invalidTrans: Transpose parameter must be one of 'N', 'T', or 'C'.");
  return c;
}

// --------------------------------------------------------------- tree build (K1, K2)
void build_tree(flam_factor& F, double occ, const flam_opts& o) {
  cudaStream_t s = F.s;
  const int d = F.d, ninst = F.ninst;
  const int64_t ntot = F.Ntot;
  const int nl = 1 << d;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, s));

  DBuf<int64_t> inst_off_d;
  inst_off_d.upload(F.inst_off, s);

  // root extents (hypoct.m:65-69)
  std::vector<double> ext((size_t)ninst * 2 * d);
  if (o.ext) {
    for (int i = 0; i < ninst; ++i)
      for (int q = 0; q < d; ++q) {
        ext[((size_t)i * d + q) * 2] = o.ext[q];
        ext[((size_t)i * d + q) * 2 + 1] = o.ext[d + q];
      }
  } else {
    const int nchunk = ninst == 1 ? 64 : 1;
    DBuf<double> part;
    part.resize((int64_t)ninst * nchunk * 2 * d, s);
    tree_extent(F.x.p, d, inst_off_d.p, ninst, nchunk, part.p, s);
    F.prof.launches += 1;
    auto ph = download(part.p, part.n, s);
    for (int i = 0; i < ninst; ++i)
      for (int q = 0; q < d; ++q) {
        double mn = INFINITY, mx = -INFINITY;
        for (int c = 0; c < nchunk; ++c) {
          mn = std::min(mn, ph[(((size_t)i * nchunk + c) * 2 * d) + 2 * q]);
          mx = std::max(mx, ph[(((size_t)i * nchunk + c) * 2 * d) + 2 * q + 1]);
        }
        ext[((size_t)i * d + q) * 2] = mn;
        ext[((size_t)i * d + q) * 2 + 1] = mx;
      }
    part.release(s);
  }

  // device tree arrays
  DBuf<int64_t> perm, perm2, seg_start, seg_len, nbor_ptr;
  DBuf<int32_t> pbox, pbox2, prnt, chfirst, nch, depth, binst, keychild, nbor;
  DBuf<double> ctr, lsz;
  auto reserve_boxes = [&](int64_t c) {
    ctr.reserve(c * d, s);
    lsz.reserve(c * d, s);
    prnt.reserve(c, s);
    chfirst.reserve(c, s);
    nch.reserve(c, s);
    seg_start.reserve(c, s);
    seg_len.reserve(c, s);
    depth.reserve(c, s);
    binst.reserve(c, s);
    keychild.reserve(c * 8, s);
    nbor_ptr.reserve(c + 1, s);
    ctr.n = lsz.n = c * d;
    prnt.n = chfirst.n = nch.n = seg_start.n = seg_len.n = depth.n = binst.n = c;
    keychild.n = c * 8;
    nbor_ptr.n = c + 1;
  };
  {
    std::vector<int64_t> pv(ntot);
    std::vector<int32_t> pb(ntot);
    for (int i = 0; i < ninst; ++i)
      for (int64_t q = F.inst_off[i]; q < F.inst_off[i + 1]; ++q) {
        pv[q] = q;
        pb[q] = i;
      }
    perm.upload(pv, s);
    pbox.upload(pb, s);
    perm2.resize(ntot, s);
    pbox2.resize(ntot, s);
  }
  std::vector<double> lcur((size_t)ninst * d);
  {
    reserve_boxes(std::max<int64_t>(ninst * 4, 64));
    std::vector<double> c0((size_t)ninst * d), l0((size_t)ninst * d);
    std::vector<int32_t> z(ninst, 0), one(ninst, 1), mneg(ninst, -1), ids(ninst);
    std::vector<int64_t> ss(ninst), sl(ninst);
    for (int i = 0; i < ninst; ++i) {
      for (int q = 0; q < d; ++q) {
        const double a = ext[((size_t)i * d + q) * 2], b = ext[((size_t)i * d + q) * 2 + 1];
        l0[i * d + q] = b - a;
        c0[i * d + q] = 0.5 * (a + b);
      }
      ss[i] = F.inst_off[i];
      sl[i] = F.inst_off[i + 1] - F.inst_off[i];
      ids[i] = i;
    }
    lcur = l0;
    CK(cudaMemcpyAsync(ctr.p, c0.data(), sizeof(double) * c0.size(), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(lsz.p, l0.data(), sizeof(double) * l0.size(), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(prnt.p, mneg.data(), sizeof(int32_t) * ninst, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(chfirst.p, mneg.data(), sizeof(int32_t) * ninst, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(nch.p, z.data(), sizeof(int32_t) * ninst, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(depth.p, one.data(), sizeof(int32_t) * ninst, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(binst.p, ids.data(), sizeof(int32_t) * ninst, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(seg_start.p, ss.data(), sizeof(int64_t) * ninst, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(seg_len.p, sl.data(), sizeof(int64_t) * ninst, cudaMemcpyHostToDevice, s));
  }
  auto tdev = [&]() {
    TreeDev t;
    t.d = d;
    t.x = F.x.p;
    t.perm = perm.p;
    t.pbox = pbox.p;
    t.ctr = ctr.p;
    t.lsz = lsz.p;
    t.prnt = prnt.p;
    t.chfirst = chfirst.p;
    t.nch = nch.p;
    t.seg_start = seg_start.p;
    t.seg_len = seg_len.p;
    t.depth = depth.p;
    t.inst = binst.p;
    t.keychild = keychild.p;
    t.nbor_ptr = nbor_ptr.p;
    t.nbor = nbor.p;
    return t;
  };

  const int64_t lvlmax = o.lvlmax <= 0 ? INT64_MAX : o.lvlmax;
  const int64_t iocc = (int64_t)std::floor(occ);  // xn > occ  <=>  xn > floor(occ) for integer xn
  std::vector<int64_t> lvb = {0, ninst};
  DBuf<int32_t> flags, scr32, nchtmp, ldiv_d;
  DBuf<double> lnew_d;
  std::vector<int32_t> ldiv(ninst);
  std::vector<double> lnew((size_t)ninst * d);
  int D = 1;
  while (true) {
    if (D >= lvlmax) break;                                        // hypoct.m:77
    if (D > 200) fail(FLAM_ERR_ARG, "FLAM:hypoct:depth: tree deeper than 200 levels (duplicate points?)");
    const int32_t b0 = (int32_t)lvb[D - 1], b1 = (int32_t)lvb[D];
    for (int i = 0; i < ninst; ++i) {                              // hypoct.m:81-82
      double mx = -INFINITY;
      for (int q = 0; q < d; ++q) mx = std::max(mx, lcur[i * d + q]);
      const double thr = mx / std::sqrt(2.0);
      int m = 0;
      for (int q = 0; q < d; ++q) {
        const bool dv = lcur[i * d + q] >= thr;
        m |= dv ? (1 << q) : 0;
        lnew[i * d + q] = dv ? 0.5 * lcur[i * d + q] : lcur[i * d + q];
      }
      ldiv[i] = m;
    }
    ldiv_d.upload(ldiv, s);
    lnew_d.upload(lnew, s);
    TreeDev t = tdev();
    const int64_t L = (int64_t)nl * (ntot + 1);
    flags.resize(L + 1, s);
    scr32.resize(scan_scratch_elems(std::max<int64_t>(L, b1 - b0)) + 1, s);
    F.prof.launches += 9;  // flags, 2 scans of 3 kernels, count, children/scatter below
    tree_level_flags(t, ntot, b0, b1, iocc, 1, ldiv_d.p, flags.p, nl, s);
    exclusive_scan<int32_t>(flags.p, flags.p, L, scr32.p, s);
    nchtmp.resize(b1 - b0 + 1, s);
    tree_level_count(t, ntot, b0, b1, iocc, 1, flags.p, nl, nchtmp.p, s);
    exclusive_scan<int32_t>(nchtmp.p, nchtmp.p, b1 - b0, scr32.p, s);
    int32_t added = 0;
    CK(cudaMemcpyAsync(&added, nchtmp.p + (b1 - b0), sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (added <= 0) break;                                         // hypoct.m:121
    reserve_boxes((int64_t)b1 + added);
    t = tdev();
    tree_level_children(t, ntot, b0, b1, flags.p, nl, nchtmp.p, ldiv_d.p, lnew_d.p, s);
    tree_level_scatter(t, ntot, b0, b1, iocc, 1, ldiv_d.p, flags.p, nl, perm2.p, pbox2.p, s);
    std::swap(perm.p, perm2.p);
    std::swap(pbox.p, pbox2.p);
    lvb.push_back((int64_t)b1 + added);
    ++D;
    lcur = lnew;
  }
  const int64_t nbox = lvb.back();
  const int maxdepth = (int)lvb.size() - 1;
  // leaves get chfirst = -1 / nch = 0 from their creation; boxes of the last level too.

  // neighbours (hypoct.m:141-170), depth by depth
  {
    std::vector<int64_t> z(ninst + 1, 0);
    CK(cudaMemcpyAsync(nbor_ptr.p, z.data(), sizeof(int64_t) * (ninst + 1), cudaMemcpyHostToDevice, s));
    DBuf<int64_t> cnt, scr64;
    int64_t total = 0;
    nbor.reserve(std::max<int64_t>(nbox * 8, 64), s);
    for (int Dd = 2; Dd <= maxdepth; ++Dd) {
      const int32_t b0 = (int32_t)lvb[Dd - 1], b1 = (int32_t)lvb[Dd];
      const int32_t nb = b1 - b0;
      cnt.resize(nb + 1, s);
      scr64.resize(scan_scratch_elems(nb) + 1, s);
      TreeDev t = tdev();
      F.prof.launches += 5;
      tree_neighbours(t, b0, b1, 0, cnt.p, s);
      exclusive_scan<int64_t>(cnt.p, cnt.p, nb, scr64.p, s);
      auto h = download(cnt.p, (int64_t)nb + 1, s);
      for (auto& v : h) v += total;
      CK(cudaMemcpyAsync(nbor_ptr.p + b0, h.data(), sizeof(int64_t) * (nb + 1), cudaMemcpyHostToDevice, s));
      total = h[nb];
      nbor.reserve(total, s);
      nbor.n = total;
      t = tdev();
      tree_neighbours(t, b0, b1, 1, nbor_ptr.p + b0, s);
    }
    cnt.release(s);
    scr64.release(s);
  }

  // hypoct_perm (hypoct_perm.m:11-39)
  {
    DBuf<int64_t> off;
    off.resize(nbox, s);
    CK(cudaMemcpyAsync(off.p, F.inst_off.data(), sizeof(int64_t) * ninst, cudaMemcpyHostToDevice, s));
    TreeDev t = tdev();
    for (int Dd = 1; Dd < maxdepth; ++Dd) tree_perm_offsets(t, (int32_t)lvb[Dd - 1], (int32_t)lvb[Dd], off.p, s);
    F.hperm.resize(ntot, s);
    tree_perm_fill(t, (int32_t)nbox, off.p, F.hperm.p, s);
    F.prof.launches += maxdepth;
    off.release(s);
  }
  CK(cudaEventRecord(e1, s));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  F.t_tree = ms * 1e-3;
  CK(cudaEventDestroy(e0));
  CK(cudaEventDestroy(e1));

  // host mirror
  F.nbox = nbox;
  F.lvb = lvb;
  F.prnt = download(prnt.p, nbox, s);
  F.chfirst = download(chfirst.p, nbox, s);
  F.nch = download(nch.p, nbox, s);
  F.depth = download(depth.p, nbox, s);
  F.binst = download(binst.p, nbox, s);
  F.seg_start = download(seg_start.p, nbox, s);
  F.seg_len = download(seg_len.p, nbox, s);
  F.nbor_ptr = download(nbor_ptr.p, nbox + 1, s);
  F.nbor = download(nbor.p, F.nbor_ptr[nbox], s);
  F.ctr = download(ctr.p, nbox * d, s);
  F.lsz = download(lsz.p, nbox * d, s);
  F.nlvl.assign(ninst, 1);
  for (int64_t b = 0; b < nbox; ++b) F.nlvl[F.binst[b]] = std::max(F.nlvl[F.binst[b]], (int)F.depth[b]);
  // the point ids in tree order become the start of the id pool
  F.ipool.resize(ntot, s);
  CK(cudaMemcpyAsync(F.ipool.p, perm.p, sizeof(int64_t) * ntot, cudaMemcpyDeviceToDevice, s));
  for (auto* b : {&perm, &perm2, &seg_start, &seg_len, &nbor_ptr}) b->release(s);
  for (auto* b : {&pbox, &pbox2, &prnt, &chfirst, &nch, &depth, &binst, &keychild, &nbor, &flags, &scr32,
                  &nchtmp, &ldiv_d})
    b->release(s);
  ctr.release(s);
  lsz.release(s);
  lnew_d.release(s);
  inst_off_d.release(s);
  CK(cudaStreamSynchronize(s));
}

// --------------------------------------------------------------- factorization (K3-K7)
// Remaining skeletons and their sparse system after a partial factorization
// (rskelf.m:278-308): Si = the points of each instance that no factor eliminated,
// S = the kept M blocks scattered to Si positions, in compressed-column form with
// rows ascending (what MATLAB's sparse(I,J,V,Sn,Sn) holds; exact zeros dropped).
void assemble_partial(flam_factor& F, const std::vector<KeptBlock>& kept, const std::vector<double>& val) {
  const int ninst = F.ninst;
  F.Si.assign(ninst, {});
  F.Scp.assign(ninst, {0});
  F.Sri.assign(ninst, {});
  F.Sv.assign(ninst, {});
  F.Sn_tot = 0;
  int64_t nrem = 0;
  for (auto v : F.rem) nrem += v;
  if (nrem == 0) return;
  const cudaStream_t s = F.s;
  auto ids = download(F.ipool.p, F.ipool.n, s);
  std::vector<uint8_t> gone((size_t)F.Ntot, 0);
  for (const HostFac& h : F.hfac)
    for (int64_t j = h.sk_off + h.k; j < h.sk_off + h.k + h.r; ++j) gone[ids[j]] = 1;
  std::vector<int64_t> pos((size_t)F.Ntot, -1), glob;
  for (int i = 0; i < ninst; ++i) {
    for (int64_t g = F.inst_off[i]; g < F.inst_off[i + 1]; ++g)
      if (!gone[g]) {
        pos[g] = (int64_t)F.Si[i].size();
        F.Si[i].push_back(g - F.inst_off[i]);
        glob.push_back(g);
      }
    if ((int64_t)F.Si[i].size() != F.rem[i])
      fail(FLAM_ERR_CUDA, "FLAM:gpu:internal: remaining point count disagrees with the factors");
  }
  F.Sn_tot = (int64_t)glob.size();
  F.Si_dev.upload(glob, s);
  // columns: each remaining point lies in at most one kept block
  std::vector<std::vector<int64_t>> cnt(ninst);
  for (int i = 0; i < ninst; ++i) cnt[i].assign(F.Si[i].size() + 1, 0);
  struct Col { int64_t blk, a; };
  std::vector<std::vector<Col>> owner(ninst);
  for (int i = 0; i < ninst; ++i) owner[i].assign(F.Si[i].size(), Col{-1, -1});
  std::vector<std::vector<int64_t>> order(kept.size());
  for (size_t q = 0; q < kept.size(); ++q) {
    const KeptBlock& kb = kept[q];
    std::vector<int64_t> ps(kb.n);
    for (int64_t a = 0; a < kb.n; ++a) {
      ps[a] = pos[ids[kb.idx_off + a]];
      if (ps[a] < 0) fail(FLAM_ERR_CUDA, "FLAM:gpu:internal: a kept skeleton was eliminated");
      owner[kb.inst][ps[a]] = Col{(int64_t)q, a};
    }
    auto& ord = order[q];
    ord.resize(kb.n);
    for (int64_t a = 0; a < kb.n; ++a) ord[a] = a;
    std::sort(ord.begin(), ord.end(), [&](int64_t x, int64_t y) { return ps[x] < ps[y]; });
  }
  for (int i = 0; i < ninst; ++i) {
    const int64_t Sn = (int64_t)F.Si[i].size();
    auto& cp = F.Scp[i];
    auto& ri = F.Sri[i];
    auto& v = F.Sv[i];
    cp.assign(Sn + 1, 0);
    for (int64_t c = 0; c < Sn; ++c) {
      const Col o = owner[i][c];
      if (o.blk >= 0) {
        const KeptBlock& kb = kept[o.blk];
        const double* M = val.data() + kb.val_off + o.a * kb.n;   // column a of the block
        for (int64_t e : order[o.blk]) {
          if (M[e] == 0.0) continue;
          ri.push_back(pos[ids[kb.idx_off + e]]);
          v.push_back(M[e]);
        }
      }
      cp[c + 1] = (int64_t)ri.size();
    }
  }
}

// Device view of a handle's matrix and proxy.
Problem problem_of(const flam_factor& F) {
  Problem P;
  P.d = F.d;
  P.x = F.x.p;
  P.w = F.has_w ? F.w.p : nullptr;
  P.nrm = F.has_nrm ? F.nrm.p : nullptr;
  P.ip = F.ip.p;
  P.pxy_pts = F.pxy_pts.p;
  P.pxy_shift = F.pxy_shift.n ? F.pxy_shift.p : nullptr;
  P.npxy = F.npxy;
  return P;
}

void factorize(flam_factor& F, double rank_or_tol, const flam_opts& o) {
  cudaStream_t s = F.s;
  const int ninst = F.ninst;
  const int64_t nbox = F.nbox;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, s));

  // boxes of each (instance, depth), ascending id
  std::vector<std::vector<std::vector<int32_t>>> byl(ninst);
  for (int i = 0; i < ninst; ++i) byl[i].resize(F.nlvl[i] + 1);
  for (int64_t b = 0; b < nbox; ++b) byl[F.binst[b]][F.depth[b]].push_back((int32_t)b);
  // nonempty (leaf) boxes per level for the verbose table (rskelf.m:146-152)
  std::vector<std::vector<int64_t>> pblk(ninst);
  for (int i = 0; i < ninst; ++i) {
    pblk[i].assign(F.nlvl[i] + 2, 0);
    for (int L = 1; L <= F.nlvl[i]; ++L) {
      int64_t c = 0;
      for (int32_t b : byl[i][L]) c += F.nch[b] == 0;
      pblk[i][L + 1] = pblk[i][L] + c;
    }
  }

  // global compression (no proxy function): the leaf boxes of each instance
  bool any_global = false;
  for (int i = 0; i < ninst; ++i) any_global |= F.iph[i].pkind == P_NONE;
  std::vector<std::vector<int32_t>> leaves(any_global ? ninst : 0);
  if (any_global)
    for (int64_t b = 0; b < nbox; ++b)
      if (F.nch[b] == 0 && F.iph[F.binst[b]].pkind == P_NONE) leaves[F.binst[b]].push_back((int32_t)b);

  std::vector<int64_t> xoff(nbox), xlen(nbox), Moff(nbox, -1);
  for (int64_t b = 0; b < nbox; ++b) {
    const bool leaf = F.nch[b] == 0;
    xoff[b] = leaf ? F.seg_start[b] : 0;
    xlen[b] = leaf ? F.seg_len[b] : 0;
  }
  F.rem.resize(ninst);
  for (int i = 0; i < ninst; ++i) F.rem[i] = F.inst_off[i + 1] - F.inst_off[i];
  F.inst_fac.assign(ninst, {});
  F.inst_lvp.assign(ninst, {0});
  F.stats.assign(ninst, {});

  const double rel_tol = std::fmod(rank_or_tol, 1.0);
  const int kmax = (int)std::min<double>(std::floor(rank_or_tol), 2e9);
  const int maxsteps = *std::max_element(F.nlvl.begin(), F.nlvl.end());
  const int64_t stop = o.stop < 0 ? INT64_MAX : o.stop;

  Workspace& ws = workspace(F.dev, s);
  ws.ensure_side();
  auto& cpool = ws.cpool;
  auto& mpool = ws.mpool;
  auto& status = ws.status;
  auto& ctask = ws.ctask;
  auto& etask = ws.etask;
  auto& chb = ws.chb;
  auto& segs = ws.segs;
  auto& csegs = ws.csegs;
  auto& cout = ws.cout;
  status.ensure(1, s);
  CK(cudaMemsetAsync(status.p, 0, sizeof(int32_t), s));
  if (ws.hint_ipool > F.ipool.cap) F.ipool.reserve(ws.hint_ipool, s);
  if (ws.hint_fpool > F.fpool.cap) F.fpool.reserve(ws.hint_fpool, s);
  if (ws.hint_ppool > F.ppool.cap) F.ppool.reserve(ws.hint_ppool, s);
  const Problem P = problem_of(F);
  int cur = 0;  // M pool written this step
  int64_t fpool_top = 0, ppool_top = 0;
  const bool prof = F.profile;
  const bool prof_print = std::getenv("FLAM_PROFILE") != nullptr;
  // FLAM_PROFILE=2: also one event pair per compress launch, printed with its shape
  const bool prof_launch = prof_print && std::getenv("FLAM_PROFILE")[0] == '2';
  struct LaunchRec {
    int key, t0, t1;
    cudaEvent_t e0, e1;
  };
  std::vector<LaunchRec> lrec;
  // FLAM_PROFILE=2: event pairs around the phases of the sketched compression on stream s
  // (key -1 filter + sketch, -2 ID of the wide sketches, -3 second sketch, -4 ID of the wide
  // second sketches, -5 ID of the narrow second sketches, -6 exact redo)
  auto ph_begin = [&](int key, cudaStream_t st) {
    if (!(prof && prof_launch)) return;
    LaunchRec lr{key, 0, 0, nullptr, nullptr};
    CK(cudaEventCreate(&lr.e0));
    CK(cudaEventCreate(&lr.e1));
    CK(cudaEventRecord(lr.e0, st));
    lrec.push_back(lr);
  };
  auto ph_end = [&](cudaStream_t st) {
    if (prof && prof_launch) CK(cudaEventRecord(lrec.back().e1, st));
  };
  // profiling: event pairs around the sketch launches, resolved with the step events
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> sk_ev;
  auto sk_begin = [&](cudaStream_t st) {
    if (!prof) return;
    sk_ev.emplace_back();
    CK(cudaEventCreate(&sk_ev.back().first));
    CK(cudaEventCreate(&sk_ev.back().second));
    CK(cudaEventRecord(sk_ev.back().first, st));
  };
  auto sk_end = [&](cudaStream_t st) {
    if (prof) CK(cudaEventRecord(sk_ev.back().second, st));
  };
  // per-step CUDA events around the compress and elimination launches; resolved
  // after the last step so that profiling adds no synchronisation
  std::vector<cudaEvent_t> step_ev;
  cudaEvent_t* pe = nullptr;
  // M blocks still unfactored when an instance stops: (instance, ipool offset, n, offset in kept_val)
  std::vector<KeptBlock> kept;
  std::vector<double> kept_val;
  const int64_t nrun = std::min<int64_t>(stop, maxsteps);
  const flam_tune tune = tune_lookup(tune_key(F.dev, F.d, F.iph[0].kind, F.Ntot));

  for (int step = 0; step < maxsteps && step < stop; ++step) {
    // this step's T / permutation / scratch set was last read by the elimination two
    // steps back
    const int par = step & 1;
    auto& tpool = par ? ws.tpool_b : ws.tpool;
    auto& scratch = par ? ws.scratch_b : ws.scratch;
    auto& permpool = par ? ws.permpool_b : ws.permpool;
    ws.wait_elim(s, par);
    // ---- boxes of this step: level nlvl_i - step of each instance
    std::vector<int32_t> boxes;
    std::vector<int> binst_step;
    for (int i = 0; i < ninst; ++i) {
      const int L = F.nlvl[i] - step;
      if (L < 1) continue;
      for (int32_t b : byl[i][L]) boxes.push_back(b);
    }
    if (boxes.empty()) break;
    const int nb = (int)boxes.size();
    std::vector<int64_t> rem1 = F.rem;
    // ---- slf lists: own points (leaf) or children's current xi (rskelf.m:179-181)
    std::vector<int64_t> slf_off(nb), nslf(nb);
    std::vector<CopySeg> sg;
    std::vector<ChildBlock> ch;
    std::vector<int32_t> ch_first(nb), nchv(nb);
    int64_t top = F.ipool.n;
    std::vector<int64_t> pos_in_step(nbox, -1);
    for (int q = 0; q < nb; ++q) {
      const int32_t b = boxes[q];
      pos_in_step[b] = q;
      slf_off[q] = top;
      int64_t n = 0;
      if (F.nch[b] == 0) {
        sg.push_back(CopySeg{xoff[b], top + n, xlen[b]});
        n += xlen[b];
      }
      ch_first[q] = (int32_t)ch.size();
      for (int32_t c = F.chfirst[b]; c >= 0 && c < F.chfirst[b] + F.nch[b]; ++c) {
        ch.push_back(ChildBlock{(int32_t)n, (int32_t)xlen[c], Moff[c]});
        if (xlen[c] > 0) sg.push_back(CopySeg{xoff[c], top + n, xlen[c]});
        n += xlen[c];
      }
      nchv[q] = (int32_t)ch.size() - ch_first[q];
      nslf[q] = n;
      top += n;
    }
    if (top > F.ipool.cap) ws.wait_elim(s, par ^ 1);   // growth frees the pool the last elimination reads
    F.ipool.reserve(top, s);
    F.ipool.n = top;
    // ---- neighbour candidates: current xi of every neighbour (rskelf.m:186).  Without a
    // proxy function a box below level 2 is compressed against every remaining point of
    // its instance instead (rskelf.m:204, nbr = setdiff(find(rem), slf)): the other boxes
    // of this level after the pull-up, and the leaves of coarser levels (not yet reached).
    std::vector<CopySeg> cs;
    std::vector<int64_t> cand_off(nb), ncand(nb);
    std::vector<std::vector<int>> inst_q;   // global compression: this step's boxes per instance
    if (any_global) {
      inst_q.resize(ninst);
      for (int q = 0; q < nb; ++q) inst_q[F.binst[boxes[q]]].push_back(q);
    }
    int64_t ctop = 0;
    for (int q = 0; q < nb; ++q) {
      const int32_t b = boxes[q];
      cand_off[q] = ctop;
      int64_t n = 0;
      const int ib = F.binst[b];
      if (F.iph[ib].pkind == P_NONE && F.depth[b] > 2) {
        for (int q2 : inst_q[ib])
          if (q2 != q && nslf[q2] > 0) {
            cs.push_back(CopySeg{slf_off[q2], ctop + n, nslf[q2]});
            n += nslf[q2];
          }
        for (int32_t j : leaves[ib])
          if (F.depth[j] < F.depth[b] && xlen[j] > 0) {
            cs.push_back(CopySeg{xoff[j], ctop + n, xlen[j]});
            n += xlen[j];
          }
        if (n > INT32_MAX / 2)
          fail(FLAM_ERR_ARG, "FLAM:gpu:globalTooLarge: global compression of a box against %lld points exceeds "
                             "the device limit", (long long)n);
        ncand[q] = n;
        ctop += n;
        continue;
      }
      for (int64_t e = F.nbor_ptr[b]; e < F.nbor_ptr[b + 1]; ++e) {
        const int32_t j = F.nbor[e];
        int64_t so, sl;
        if (pos_in_step[j] >= 0) {  // same level: its list after the pull-up (level-synchronous)
          so = slf_off[pos_in_step[j]];
          sl = nslf[pos_in_step[j]];
        } else {                    // coarser leaf: its original points
          so = xoff[j];
          sl = xlen[j];
        }
        if (sl > 0) cs.push_back(CopySeg{so, ctop + n, sl});
        n += sl;
      }
      ncand[q] = n;
      ctop += n;
    }
    cpool.ensure(std::max<int64_t>(ctop, 1), s);
    // ---- tasks
    std::vector<CompressTask> ct(nb);
    std::vector<int64_t> elim_scr(nb, -1);
    // Row-split form on the levels with few boxes: each large box's rows go to
    // nparts CTAs whose R factors are then merged pairwise, so that the step
    // occupies more of the GPU's 148 SMs.
    const int split_ctas = tune.split_ctas;     // CTAs a split step aims at
    const int split_max = tune.split_max;       // parts per box at most
    const int split_min_n = tune.split_min_n;   // boxes above this size are split
    // sketched compression (opts.sketch): boxes of at most kSketchMaxN points whose block
    // has more rows than the sketch take Y = Omega K (w rows) and an ID of Y
    // box features (rank predictor, rank log): from the slf lists, gathered here already
    const flam_predictor* pred = o.sketch ? static_cast<const flam_predictor*>(o.predictor) : nullptr;
    std::vector<int> pred_k;   // per box: the rank predictor's estimate (empty: no predictor)
    std::vector<CompressTask> ftv;
    if (pred || o.rank_log) {
      ftv.resize(nb);
      for (int q = 0; q < nb; ++q) {
        const int32_t b = boxes[q];
        const int i = F.binst[b];
        CompressTask& u = ftv[q];
        u.slf_off = slf_off[q];
        u.n = (int32_t)nslf[q];
        u.ncand = (int32_t)ncand[q];
        u.inst = i;
        u.box = b;
        u.depth = F.depth[b];
        u.flags = (F.depth[b] > 2 && F.iph[i].pkind != P_NONE) ? 1 : 0;
        for (int c = 0; c < kMaxDim; ++c) {
          u.ctr[c] = c < F.d ? F.ctr[(size_t)b * F.d + c] : 0.0;
          u.l[c] = c < F.d ? F.lsz[(size_t)b * F.d + c] : 0.0;
        }
      }
      segs.upload(sg, s);
      launch_gather_ids(F.ipool.p, F.ipool.p, segs.p, (int)sg.size(), s);
      ws.ftask.upload(ftv, s);
      ws.feat.ensure((int64_t)nb * kPredFeatures, s);
      launch_box_features(ws.ftask.p, nb, F.ipool.p, P, rel_tol > 0 ? (float)-std::log10(rel_tol) : 16.f, ws.feat.p,
                          s);
      F.prof.launches += 2;
      if (pred) {
        if (pred->dev != F.dev) fail(FLAM_ERR_ARG, "FLAM:gpu:predictorDevice: the predictor lives on another device");
        ws.fyhat.ensure(nb, s);
        launch_mlp(ws.feat.p, nullptr, nb, pred->w.p, ws.fyhat.p, nullptr, nullptr, 0.f, 0, s);
        F.prof.launches += 1;
        CK(cudaGetLastError());
        auto yh = download(ws.fyhat.p, nb, s);
        pred_k.resize(nb);
        // 25% above the prediction: a low estimate costs a second sketch, a high one only rows
        for (int q = 0; q < nb; ++q) pred_k[q] = (int)std::ceil(1.25 * (double)yh[q] * (double)nslf[q]);
      }
    }
    std::vector<int> skw(nb, 0);
    std::vector<int64_t> yoff(nb, -1);
    int64_t ytop = 0;
    if (o.sketch) {
      const int sp = o.sketch_p;
      for (int q = 0; q < nb; ++q) {
        const int n = (int)nslf[q];
        if (n == 0 || n > kSketchMaxN) continue;
        const int32_t b = boxes[q];
        const int i = F.binst[b];
        const bool use_proxy = F.depth[b] > 2 && F.iph[i].pkind != P_NONE;
        const int64_t mcap = (F.symm == 'n' ? 2 : 1) * ncand[q] +
                             (use_proxy ? (F.iph[i].two_sided ? 2 : 1) * (int64_t)F.npxy : 0);
        const int kest = pred_k.empty() ? n : std::min(n, pred_k[q]);
        const int w = std::min(std::max(kest + sp, 8), kSketchMaxW);
        if (mcap <= w) continue;   // the block is no taller than its sketch: exact ID
        skw[q] = w;
        yoff[q] = ytop;
        ytop += (int64_t)w * n;
      }
    }
    int nparts = 1;
    while (nparts * 2 <= split_max && nparts * 2 * nb <= split_ctas) nparts *= 2;
    std::vector<char> split(nb, 0);
    std::vector<int> npq(nb, 1);   // parts of each split box
    int64_t ttop = 0, ptop = 0, stop_s = 0;
    int nmax_small = 0;
    for (int q = 0; q < nb; ++q) {
      const int32_t b = boxes[q];
      const int i = F.binst[b];
      CompressTask& t = ct[q];
      t.slf_off = slf_off[q];
      t.cand_off = cand_off[q];
      t.n = (int32_t)nslf[q];
      t.ncand = (int32_t)ncand[q];
      t.box = b;
      t.inst = i;
      const bool use_proxy = F.depth[b] > 2 && F.iph[i].pkind != P_NONE;   // rskelf.m:203
      t.flags = use_proxy ? 3 : 0;
      for (int c = 0; c < kMaxDim; ++c) {
        t.ctr[c] = c < F.d ? F.ctr[(size_t)b * F.d + c] : 0.0;
        t.l[c] = c < F.d ? F.lsz[(size_t)b * F.d + c] : 0.0;
      }
      t.T_off = ttop;
      ttop += (nslf[q] * nslf[q]) / 4 + 1;
      t.perm_off = ptop;
      ptop += nslf[q];
      t.out_idx = q;
      t.depth = F.depth[b];
      // work matrices: shared memory when they fit, else a per-box slot of global scratch
      // shared by the compress and elimination kernels of this step
      const int n = (int)nslf[q];
      const bool tc = n <= kTcMaxN;
      const int64_t mcap = (F.symm == 'n' ? 2 : 1) * ncand[q] +
                           (use_proxy ? (F.iph[i].two_sided ? 2 : 1) * (int64_t)F.npxy : 0);
      // as many parts (up to nparts) as leave each part at least one row panel
      if (nparts > 1 && tc && n > split_min_n && skw[q] == 0) {
        const int64_t ph = (int64_t)compress_tc_rows(n) * compress_tc_group(n);
        int np = nparts;
        while (np > 1 && mcap < np * ph) np /= 2;
        npq[q] = np;
      }
      split[q] = npq[q] > 1;
      const bool c_glob = split[q] || (tc ? compress_tc_smem_bytes(n) > (size_t)tune.tc_smem_max : n > kSmemN);
      const bool e_glob = n > kSmemN;
      t.scr_off = -1;
      elim_scr[q] = -1;
      if (c_glob || e_glob) {
        const int64_t cslot = split[q] ? npq[q] * compress_tc_doubles(n)
                                       : (tc ? compress_tc_doubles(n) : compress_scratch_doubles(n));
        const int64_t slot = std::max(cslot, elim_scratch_doubles(n));
        if (c_glob) t.scr_off = stop_s;
        if (e_glob) elim_scr[q] = stop_s;
        stop_s += slot;
      }
      if (!tc && !c_glob) nmax_small = std::max<int>(nmax_small, n);
    }
    tpool.ensure(std::max<int64_t>(ttop, 1), s);
    permpool.ensure(std::max<int64_t>(ptop, 1), s);
    scratch.ensure(std::max<int64_t>(stop_s, 1), s);
    segs.upload(sg, s);
    launch_gather_ids(F.ipool.p, F.ipool.p, segs.p, (int)sg.size(), s);
    csegs.upload(cs, s);
    launch_gather_ids(F.ipool.p, cpool.p, csegs.p, (int)cs.size(), s);
    // group the boxes by kernel shape: thread-per-column blocks of 32..1024 threads,
    // and the per-column kernel for n > kTcMaxN
    auto kkey_n = [](int n) {
      return n <= kTcMaxN ? compress_tc_threads(n) * 1000 + compress_tc_rows(n) * 10 + compress_tc_group(n) : 0;
    };
    auto kkey = [&](int q) { return kkey_n((int)nslf[q]); };
    std::vector<int> ord;
    for (int q = 0; q < nb; ++q)
      if (!split[q]) ord.push_back(q);
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return kkey(x) < kkey(y); });
    // task segments: [whole boxes | filter of split boxes | parts | merge level 0 | level 1 ...]
    std::vector<CompressTask> cts;
    cts.reserve(nb * 3);
    // ID of the sketches of boxes wider than a thread per column: few boxes spread every
    // pivot step over the GPU, many take one CTA each
    auto launch_wide = [&](const CompressArgs& cw, const std::vector<CompressTask>& tasks) {
      const int nt = (int)tasks.size();
      int nmx = 0, wmx = 0, steps = 0;
      for (const CompressTask& u : tasks) {
        nmx = std::max(nmx, u.n);
        wmx = std::max(wmx, u.ax_rows);
        steps = std::max(steps, std::min(u.n, u.ax_rows));
      }
      if (nt < 148 || wmx > cpqr_wide_max_rows()) {
        ws.gwstate.ensure((int64_t)cpqr_grid_state_bytes(nt), s);
        launch_cpqr_grid(cw, nt, nmx, wmx, steps, ws.gwstate.p, s);
        F.prof.launches += 5 + 2 * steps;
      } else {
        launch_cpqr_wide(cw, nt, s);
        F.prof.launches += 1;
      }
    };
    // sketched boxes: their filter and sketch tasks, and the ID of Y in place of K's rows
    std::vector<SketchTask> skt;
    std::vector<CompressTask> skf, wts;
    std::vector<int> sk_of(nb, -1);
    const int sk_guard = std::max(0, o.sketch_guard);
    for (int q : ord) {
      if (skw[q] == 0) {
        cts.push_back(ct[q]);
        continue;
      }
      const CompressTask& c0 = ct[q];
      SketchTask u{};
      u.slf_off = c0.slf_off;
      u.cand_off = c0.cand_off;
      u.y_off = yoff[q];
      u.perm_off = c0.perm_off;
      u.n = c0.n;
      u.w = skw[q];
      u.inst = c0.inst;
      u.out_idx = c0.out_idx;
      u.box = c0.box;
      u.flags = c0.flags & 1;
      for (int c = 0; c < kMaxDim; ++c) {
        u.ctr[c] = c0.ctr[c];
        u.l[c] = c0.l[c];
      }
      sk_of[q] = (int)skt.size();
      int cstep, jstep;   // the box's CTAs: column and sketch-row extents
      sketch_cta_tile(o.sketch == 2, u.n, u.w, &cstep, &jstep);
      for (int c0i = 0; c0i < u.n; c0i += cstep)
        for (int j0i = 0; j0i < u.w; j0i += jstep) {
          SketchTask v2 = u;
          v2.col0 = c0i;
          v2.ncol = std::min(cstep, u.n - c0i);
          v2.j0 = j0i;
          v2.nw = std::min(jstep, u.w - j0i);
          skt.push_back(v2);
        }
      skf.push_back(c0);
      CompressTask v = c0;
      v.flags = 0;
      v.ncand = skw[q];
      v.ax_off = yoff[q];
      v.ax_rows = skw[q];
      v.ax_guard = sk_guard;
      if (v.n > kTcMaxN)
        wts.push_back(v);   // wider than a thread per column: the wide pivoted QR
      else
        cts.push_back(v);
    }
    std::vector<int> seg{(int)cts.size()};
    std::vector<int> sord;
    for (int q = 0; q < nb; ++q)
      if (split[q]) sord.push_back(q);
    std::stable_sort(sord.begin(), sord.end(), [&](int x, int y) { return kkey(x) < kkey(y); });
    if (!sord.empty()) {
      for (int q : sord) cts.push_back(ct[q]);
      seg.push_back((int)cts.size());
      for (int q : sord)
        for (int pt = 0; pt < npq[q]; ++pt) {
          CompressTask u = ct[q];
          u.mode = 1;
          u.part = pt;
          u.nparts = npq[q];
          u.scr_off = ct[q].scr_off + pt * compress_tc_doubles(u.n);
          cts.push_back(u);
        }
      seg.push_back((int)cts.size());
      for (int h = 1; h < nparts; h *= 2) {   // merge level h: boxes with more than h parts
        for (int q : sord)
          for (int pt = 0; pt + h < npq[q]; pt += 2 * h) {
            CompressTask u = ct[q];
            u.mode = 2 * h == npq[q] ? 3 : 2;
            u.scr_off = ct[q].scr_off + pt * compress_tc_doubles(u.n);
            u.rsrc_off = ct[q].scr_off + (pt + h) * compress_tc_doubles(u.n);
            cts.push_back(u);
          }
        seg.push_back((int)cts.size());
      }
    }
    ctask.upload(cts, s);
    cout.ensure(nb, s);
    ws.mfilt.ensure(nb, s);
    CompressArgs ca{};
    ca.P = P;
    ca.tasks = ctask.p;
    ca.ipool = F.ipool.p;
    ca.cpool = cpool.p;
    ca.tpool = tpool.p;
    ca.permpool = permpool.p;
    ca.scratch = scratch.p;
    ca.out = cout.p;
    ca.rel_tol = rel_tol;
    ca.kmax = kmax;
    ca.symm_n = F.symm == 'n' ? 1 : 0;
    ca.Tmax = o.Tmax;
    ca.rrqr_iter = o.rrqr_iter;
    ca.Aexp = nullptr;
    ca.lda = 0;
    ca.mfilt = ws.mfilt.p;
    if (ytop > 0) ws.ypool.ensure(ytop, s);
    ca.ypool = ws.ypool.p;
    F.prof.launches += 2 + 1;  // two id gathers, compress
    F.prof.n_compress += 1;
    if (prof) {
      const size_t base = step_ev.size();
      step_ev.resize(base + 4);
      for (size_t e = base; e < base + 4; ++e) CK(cudaEventCreate(&step_ev[e]));
      pe = step_ev.data() + base;
      CK(cudaEventRecord(pe[0], s));
    }
    // one launch per kernel shape within a segment of the task array; the shapes
    // (independent boxes) run concurrently on side streams, so that the few-box steps
    // near the root, where every launch holds a few SMs, overlap their launches
    auto launch_segment = [&](int t0, int t1) {
      std::vector<std::pair<int, int>> groups;
      for (int b0 = t0; b0 < t1;) {
        const int key = kkey_n(cts[b0].n);
        int b1 = b0;
        while (b1 < t1 && kkey_n(cts[b1].n) == key) ++b1;
        groups.emplace_back(b0, b1);
        b0 = b1;
      }
      const int nuse = std::min<int>((int)groups.size(), Workspace::kSide);
      if (nuse > 1) ws.fork_to(s, nuse);
      for (size_t gi = 0; gi < groups.size(); ++gi) {
        const int b0 = groups[gi].first, b1 = groups[gi].second;
        const cudaStream_t gs = nuse > 1 ? ws.side[gi % Workspace::kSide] : s;
        const int key = kkey_n(cts[b0].n);
        size_t sm = 16;
        for (int u = b0; u < b1; ++u)
          if (key > 0 && cts[u].scr_off < 0) sm = std::max(sm, compress_tc_smem_bytes(cts[u].n));
        CompressArgs cb = ca;
        cb.tasks = ctask.p + b0;
        if (prof && prof_launch) {
          LaunchRec lr{key, b0, b1, nullptr, nullptr};
          CK(cudaEventCreate(&lr.e0));
          CK(cudaEventCreate(&lr.e1));
          CK(cudaEventRecord(lr.e0, gs));
          lrec.push_back(lr);
        }
        if (key == 0)
          launch_compress(cb, b1 - b0, compress_smem_bytes(nmax_small), gs);
        else
          launch_compress_tc(cb, b1 - b0, key / 1000, (key / 10) % 100, key % 10, sm, gs);
        if (prof && prof_launch) CK(cudaEventRecord(lrec.back().e1, gs));
        F.prof.launches += 1;
      }
      if (nuse > 1) ws.join_to(s, nuse);
    };
    if (!skt.empty()) {   // neighbour filter and row sketch of the sketched boxes, before their IDs
      ph_begin(-1, s);
      ws.mrows.ensure(nb, s);
      ws.sktask.upload(skt, s);
      ws.skfilt.upload(skf, s);
      CompressArgs cf = ca;
      cf.tasks = ws.skfilt.p;
      launch_filter(cf, (int)skf.size(), s);
      SketchArgs sa{};
      sa.P = P;
      sa.tasks = ws.sktask.p;
      sa.ipool = F.ipool.p;
      sa.cpool = cpool.p;
      sa.mfilt = ws.mfilt.p;
      sa.ypool = ws.ypool.p;
      sa.mrows = ws.mrows.p;
      sa.symm_n = F.symm == 'n' ? 1 : 0;
      sa.seed = o.sketch_seed;
      sa.status = status.p;
      sa.fp64 = o.sketch == 2;
      size_t smx = 0;
      for (const SketchTask& u : skt) smx = std::max(smx, sketch_smem_bytes(u.ncol, u.nw));
      sk_begin(s);
      launch_sketch(sa, (int)skt.size(), smx, s);
      sk_end(s);
      ph_end(s);
      F.prof.launches += 2;
      if (!wts.empty()) {
        ph_begin(-2, s);
        ws.wtask.upload(wts, s);
        CompressArgs cw = ca;
        cw.tasks = ws.wtask.p;
        launch_wide(cw, wts);
        ph_end(s);
      }
      F.prof.n_sketch += (int64_t)skf.size();
    }
    launch_segment(0, seg[0]);
    if (seg.size() > 1) {
      CompressArgs cf = ca;
      cf.tasks = ctask.p + seg[0];
      launch_filter(cf, seg[1] - seg[0], s);
      F.prof.launches += 1;
      for (size_t g = 1; g + 1 < seg.size(); ++g) launch_segment(seg[g], seg[g + 1]);
    }
    F.prof.launches -= 1;
    CK(cudaGetLastError());
    if (prof) CK(cudaEventRecord(pe[1], s));
    auto co = download(cout.p, nb, s);
    std::vector<char> redone(nb, 0);
    if (!skt.empty()) {
      // posterior check of the sketched IDs: a box whose rank came within sketch_guard of
      // its sketch rows is redone with the exact ID of K (from the pull-up order, with the
      // candidates the filter kept)
      std::vector<int> redo;
      for (int q = 0; q < nb; ++q)
        if (skw[q] > 0 && (co[q].status & ST_ID_CHECK)) redo.push_back(q);
      auto mr = download(ws.mrows.p, nb, s);
      for (int q = 0; q < nb; ++q)
        if (skw[q] > 0) {
          co[q].m = mr[q];   // rows of K, for the work accounting
          F.prof.sketch_rows += skw[q];
          F.prof.sketch_rows_k += mr[q];
          F.prof.flop_sketch += (o.sketch == 2 ? 2.0 : 4.0) * skw[q] * (double)mr[q] * (double)nslf[q];
        }
      if (!redo.empty()) {
        auto mf = download(ws.mfilt.p, nb, s);
        // every redone box back to its pull-up order (the first pass permuted its slf)
        {
          std::vector<int32_t> ridx;
          int nmx = 0;
          for (int q : redo) {
            ridx.push_back(sk_of[q]);
            nmx = std::max(nmx, (int)nslf[q]);
          }
          ws.redo_idx.upload(ridx, s);
          launch_unpermute(ws.redo_idx.p, (int)ridx.size(), ws.sktask.p, F.ipool.p, permpool.p, nmx, s);
          F.prof.launches += 1;
        }
        // a second sketch at full width n + p (the rank cannot fill it); a box whose first
        // sketch already had that width, or whose second sketch fills too, takes the exact ID
        std::vector<int> exact;
        std::vector<int> resk;
        const int spf = std::max(o.sketch_p, 8);
        for (int q : redo) {
          const int wf = std::min((int)nslf[q] + spf, kSketchMaxW);
          if (wf > skw[q])
            resk.push_back(q);
          else
            exact.push_back(q);
        }
        if (!resk.empty()) {
          std::vector<SketchTask> skt2;
          std::vector<CompressTask> wts2, nts2;   // IDs of the second sketches: wide, thread-per-column
          std::vector<int> first2;
          int64_t y2 = 0;
          for (int q : resk) {
            const int wf = std::min((int)nslf[q] + spf, kSketchMaxW);
            SketchTask u = skt[sk_of[q]];
            u.w = wf;
            u.y_off = y2;
            first2.push_back((int)skt2.size());
            int cstep, jstep;
            sketch_cta_tile(o.sketch == 2, u.n, wf, &cstep, &jstep);
            for (int c0i = 0; c0i < u.n; c0i += cstep)
              for (int j0i = 0; j0i < wf; j0i += jstep) {
                SketchTask v2 = u;
                v2.col0 = c0i;
                v2.ncol = std::min(cstep, u.n - c0i);
                v2.j0 = j0i;
                v2.nw = std::min(jstep, wf - j0i);
                skt2.push_back(v2);
              }
            CompressTask v = ct[q];
            v.flags = 0;
            v.ncand = wf;
            v.ax_off = y2;
            v.ax_rows = wf;
            v.ax_guard = sk_guard;
            (v.n > kTcMaxN ? wts2 : nts2).push_back(v);
            F.prof.id_rows += skw[q];   // the first sketch's rows
            F.prof.flop_id += id_flops(skw[q], nslf[q], co[q].k);
            F.prof.flop_sketch += (o.sketch == 2 ? 2.0 : 4.0) * wf * (double)mr[q] * (double)nslf[q];
            skw[q] = wf;
            y2 += (int64_t)wf * nslf[q];
          }
          ws.ypool.ensure(y2, s);   // the first pass's sketches are consumed
          ws.sktask.upload(skt2, s);
          SketchArgs sa{};
          sa.P = P;
          sa.tasks = ws.sktask.p;
          sa.ipool = F.ipool.p;
          sa.cpool = cpool.p;
          sa.mfilt = ws.mfilt.p;
          sa.ypool = ws.ypool.p;
          sa.mrows = ws.mrows.p;
          sa.symm_n = F.symm == 'n' ? 1 : 0;
          sa.seed = o.sketch_seed ^ 0x9E3779B9u;
          sa.status = status.p;
          sa.fp64 = o.sketch == 2;
          size_t smx = 0;
          for (const SketchTask& u : skt2) smx = std::max(smx, sketch_smem_bytes(u.ncol, u.nw));
          ph_begin(-3, s);
          sk_begin(s);
          launch_sketch(sa, (int)skt2.size(), smx, s);
          sk_end(s);
          ph_end(s);
          F.prof.launches += 1;
          if (!wts2.empty()) {
            ph_begin(-4, s);
            ws.wtask.upload(wts2, s);
            CompressArgs cw = ca;
            cw.tasks = ws.wtask.p;
            cw.ypool = ws.ypool.p;
            launch_wide(cw, wts2);
            ph_end(s);
          }
          if (!nts2.empty()) {   // grouped by kernel shape, as the first pass
            ph_begin(-5, s);
            std::stable_sort(nts2.begin(), nts2.end(), [&](const CompressTask& x, const CompressTask& y) {
              return kkey_n(x.n) < kkey_n(y.n);
            });
            ws.rsk_task.upload(nts2, s);
            for (size_t b0 = 0; b0 < nts2.size();) {
              const int key = kkey_n(nts2[b0].n);
              size_t b1 = b0;
              size_t sm = 16;
              while (b1 < nts2.size() && kkey_n(nts2[b1].n) == key) {
                if (nts2[b1].scr_off < 0) sm = std::max(sm, compress_tc_smem_bytes(nts2[b1].n));
                ++b1;
              }
              CompressArgs cr = ca;
              cr.tasks = ws.rsk_task.p + b0;
              cr.ypool = ws.ypool.p;
              launch_compress_tc(cr, (int)(b1 - b0), key / 1000, (key / 10) % 100, key % 10, sm, s);
              F.prof.launches += 1;
              b0 = b1;
            }
            ph_end(s);
          }
          CK(cudaGetLastError());
          auto co3 = download(cout.p, nb, s);
          std::vector<int32_t> ridx2;
          int nmx2 = 0;
          for (size_t e = 0; e < resk.size(); ++e) {
            const int q = resk[e];
            if (co3[q].status & ST_ID_CHECK) {   // filled even at full width: exact ID
              exact.push_back(q);
              ridx2.push_back(first2[e]);
              nmx2 = std::max(nmx2, (int)nslf[q]);
            } else {
              co[q] = co3[q];
            }
          }
          if (!ridx2.empty()) {
            ws.redo_idx.upload(ridx2, s);
            launch_unpermute(ws.redo_idx.p, (int)ridx2.size(), ws.sktask.p, F.ipool.p, permpool.p, nmx2, s);
            F.prof.launches += 1;
          }
        }
        std::vector<CompressTask> rt;
        for (int q : exact) {
          CompressTask v = ct[q];
          v.flags &= ~2;          // candidates already filtered
          v.ncand = mf[q];
          rt.push_back(v);
        }
        std::stable_sort(rt.begin(), rt.end(),
                         [&](const CompressTask& x, const CompressTask& y) { return kkey_n(x.n) < kkey_n(y.n); });
        ws.redo_task.upload(rt, s);
        if (!rt.empty()) ph_begin(-6, s);
        for (size_t b0 = 0; b0 < rt.size();) {
          const int key = kkey_n(rt[b0].n);
          size_t b1 = b0;
          size_t sm = 16;
          while (b1 < rt.size() && kkey_n(rt[b1].n) == key) {
            if (rt[b1].scr_off < 0) sm = std::max(sm, compress_tc_smem_bytes(rt[b1].n));
            ++b1;
          }
          CompressArgs cr = ca;
          cr.tasks = ws.redo_task.p + b0;
          if (key == 0)   // n > kTcMaxN: the per-column kernel
            launch_compress(cr, (int)(b1 - b0), 0, s);
          else
            launch_compress_tc(cr, (int)(b1 - b0), key / 1000, (key / 10) % 100, key % 10, sm, s);
          F.prof.launches += 1;
          b0 = b1;
        }
        if (!rt.empty()) ph_end(s);
        CK(cudaGetLastError());
        F.prof.n_sketch_redo += (int64_t)redo.size();
        auto co2 = download(cout.p, nb, s);
        for (int q : exact) {
          co[q] = co2[q];
          redone[q] = 1;   // folded its sketch, then K
        }
      }
    }

    for (int q = 0; q < nb; ++q) {   // a redone box folded its sketch and then K
      F.prof.id_rows += skw[q] > 0 ? skw[q] + (redone[q] ? co[q].m : 0) : co[q].m;
      if (nslf[q] > 0)
        F.prof.flop_id += id_flops(skw[q] > 0 && !redone[q] ? skw[q] : co[q].m, nslf[q], co[q].k) +
                          (redone[q] ? id_flops(skw[q], nslf[q], co[q].k) : 0.0);
    }
    if (o.rank_log) {   // features and k/n of every box that was compressed (n > 0)
      auto fv = download(ws.feat.p, (int64_t)nb * kPredFeatures, s);
      for (int q = 0; q < nb; ++q) {
        if (nslf[q] == 0) continue;
        F.rlog_X.insert(F.rlog_X.end(), fv.begin() + (size_t)q * kPredFeatures,
                        fv.begin() + (size_t)(q + 1) * kPredFeatures);
        F.rlog_y.push_back((float)co[q].k / (float)nslf[q]);
      }
    }
    // ---- elimination plan
    std::vector<ElimTask> et(nb);
    std::vector<FacDesc> fd;
    std::vector<BoxRec> brec;
    int64_t mtop = 0;
    int nmax_e = 0;
    const bool chol = F.symm == 'p';
    for (int q = 0; q < nb; ++q) {
      const int32_t b = boxes[q];
      const int n = (int)nslf[q], k = co[q].k, r = n - k;
      if (co[q].status & ST_RRQR_CAP) F.warn |= 1;
      ElimTask& t = et[q];
      t.slf_off = slf_off[q];
      t.T_off = ct[q].T_off;
      t.perm_off = ct[q].perm_off;
      t.n = n;
      t.k = k;
      t.inst = F.binst[b];
      t.ch_first = ch_first[q];
      t.nch = nchv[q];
      t.scr_off = elim_scr[q];
      if (n <= kSmemN) nmax_e = std::max(nmax_e, n);
      t.M_out = mtop;
      mtop += r > 0 ? (int64_t)k * k : (int64_t)n * n;
      if (r > 0) {
        const int64_t kr = (int64_t)k * r, rr = (int64_t)r * r;
        t.fac_off = fpool_top;
        t.piv_off = ppool_top;
        FacDesc f;
        f.sk_off = slf_off[q];
        f.T_off = fpool_top;
        f.LU_off = fpool_top + kr;
        f.E_off = fpool_top + kr + rr;
        f.G_off = fpool_top + 2 * kr + rr;
        f.piv_off = ppool_top;
        f.k = k;
        f.r = r;
        fd.push_back(f);
        HostFac h{t.inst, step, slf_off[q], k, r, fpool_top, ppool_top};
        brec.push_back(BoxRec{slf_off[q], n, k, (int64_t)F.hfac.size()});
        F.inst_fac[t.inst].push_back((int64_t)F.hfac.size());
        F.hfac.push_back(h);
        fpool_top += 2 * kr + rr + (chol ? 0 : kr);
        ppool_top += chol ? 0 : r;
        F.rem[t.inst] -= r;
      } else {
        t.fac_off = -1;
        t.piv_off = -1;
        if (n > 0) brec.push_back(BoxRec{slf_off[q], n, k, -1});
      }
    }
    F.step_boxes.push_back(std::move(brec));
    // the elimination's pools grow, and its tasks upload, on its first stream, after
    // this step's compress and the previous step's elimination
    const cudaStream_t es0 = ws.es[0], es1 = ws.es[1];
    CK(cudaEventRecord(ws.ecomp, s));
    CK(cudaStreamWaitEvent(es0, ws.ecomp, 0));
    CK(cudaStreamWaitEvent(es0, ws.edone[par ^ 1][1], 0));
    F.fpool.reserve(std::max<int64_t>(fpool_top, 1), es0);
    F.fpool.n = fpool_top;
    F.ppool.reserve(std::max<int64_t>(ppool_top, 1), es0);
    F.ppool.n = ppool_top;
    mpool[cur].ensure(std::max<int64_t>(mtop, 1), es0);
    // boxes whose work matrix is in global memory go to the blocked kernel: upload them last
    // [n <= kSmemN: shared-memory kernel | larger: one CTA per box | r >= kHugeR: grid-wide]
    auto huge = [](const ElimTask& e) { return e.n > kSmemN && e.n - e.k >= kHugeR; };
    std::vector<ElimTask> ets;
    ets.reserve(nb);
    for (const ElimTask& e : et)
      if (e.n <= kSmemN) ets.push_back(e);
    const int nsmall_e = (int)ets.size();
    for (const ElimTask& e : et)
      if (e.n > kSmemN && !huge(e)) ets.push_back(e);
    const int nbig_e = (int)ets.size() - nsmall_e;
    int hn = 0, hk = 0, hr = 0;
    for (const ElimTask& e : et)
      if (huge(e)) {
        ets.push_back(e);
        hn = std::max(hn, e.n);
        hk = std::max(hk, e.k);
        hr = std::max(hr, e.n - e.k);
      }
    const int nhuge_e = (int)ets.size() - nsmall_e - nbig_e;
    etask.upload(ets, es0);
    chb.upload(ch, es0);
    ElimArgs ea{};
    ea.P = P;
    ea.tasks = etask.p;
    ea.children = chb.p;
    ea.ipool = F.ipool.p;
    ea.tpool = tpool.p;
    ea.permpool = permpool.p;
    ea.m_in = mpool[cur ^ 1].p;
    ea.m_out = mpool[cur].p;
    ea.fpool = F.fpool.p;
    ea.ppool = F.ppool.p;
    ea.scratch = scratch.p;
    ea.status = status.p;
    ea.symm = F.symm;
    F.prof.launches += 1;
    F.prof.n_elim += 1;
    for (int q = 0; q < nb; ++q) {  // algorithmic work of this step (reference operations per box)
      const double n = (double)nslf[q], m = (double)co[q].m, k = co[q].k, r = n - k;
      if (m > 0 && n > 0) {
        const double a = std::max(m, n), b = std::min(m, n);
        F.prof.flop_compress += 2 * a * b * b - 2.0 / 3.0 * b * b * b + k * k * r;  // xGEQP3 + R11\R12
      }
      if (r > 0) {
        const double fac = chol ? r * r * r / 3 + k * r * r : 2.0 / 3.0 * r * r * r + 2 * k * r * r;
        F.prof.flop_elim += 4 * k * r * n + fac + 2 * k * k * r;
      }
    }
    if (prof) CK(cudaEventRecord(pe[2], es0));
    CK(cudaEventRecord(ws.eprep, es0));
    if (nsmall_e > 0) launch_eliminate(ea, nsmall_e, 0, elim_smem_bytes(nmax_e), es0);
    if (nb - nsmall_e > 0) {   // the two kernels' boxes are independent
      CK(cudaStreamWaitEvent(es1, ws.eprep, 0));
      ElimArgs eb = ea;
      eb.tasks = etask.p + nsmall_e;
      int rbig = 0;   // the largest redundant block among the big boxes: its LU panel height
      for (int q = nsmall_e; q < nsmall_e + nbig_e; ++q) rbig = std::max(rbig, ets[q].n - ets[q].k);
      eb.pan_rows = rbig <= elim_pan_rows_max() ? rbig : 0;
      if (nbig_e > 0) launch_eliminate(eb, 0, nbig_e, 0, es1);
      if (nhuge_e > 0) {
        ElimArgs eh = ea;
        eh.tasks = etask.p + nsmall_e + nbig_e;
        launch_eliminate_huge(eh, nhuge_e, hn, hk, hr, es1);
        F.prof.launches += elim_huge_launches(hr, hk, F.symm == 'p') - 1;
      }
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(ws.edone[par][0], es0));
    CK(cudaEventRecord(ws.edone[par][1], es1));
    if (prof) {
      CK(cudaStreamWaitEvent(es0, ws.edone[par][1], 0));
      CK(cudaEventRecord(pe[3], es0));
    }
    if (prof && prof_print) {
      CK(cudaEventSynchronize(pe[3]));
      float tc = 0, tel = 0;
      CK(cudaEventElapsedTime(&tc, pe[0], pe[1]));
      CK(cudaEventElapsedTime(&tel, pe[2], pe[3]));
      int64_t nmx = 0, cmx = 0, mmx = 0, kmx2 = 0, nit = 0, nbig = 0;
      for (int q = 0; q < nb; ++q) {
        nmx = std::max<int64_t>(nmx, nslf[q]);
        cmx = std::max<int64_t>(cmx, ncand[q]);
        mmx = std::max<int64_t>(mmx, co[q].m);
        kmx2 = std::max<int64_t>(kmx2, co[q].k);
        nit += co[q].niter;
        nbig += nslf[q] > kSmemN;
      }
      int wmx = 0, nsk = 0;
      for (int q = 0; q < nb; ++q) {
        wmx = std::max(wmx, skw[q]);
        nsk += skw[q] > 0;
      }
      fprintf(stderr, "[flam] step %2d boxes %6d nmax %5lld big %4lld candmax %6lld mmax %6lld kmax %4lld rrqr %5lld"
              "  compress %8.3f ms  elim %8.3f ms  sketched %d wmax %d\n", step, nb, (long long)nmx, (long long)nbig,
              (long long)cmx, (long long)mmx, (long long)kmx2, (long long)nit, tc, tel, nsk, wmx);
      // per launch: tasks, sum of n, reflector steps of the row folding (panels x n)
      for (LaunchRec& lr : lrec) {
        float tl = 0;
        CK(cudaEventElapsedTime(&tl, lr.e0, lr.e1));
        const int ph = lr.key > 0 ? ((lr.key / 10) % 100) * (lr.key % 10) : 1;
        int64_t sn = 0, nsteps = 0, nmx3 = 0, mode_mask = 0;
        for (int u = lr.t0; u < lr.t1; ++u) {
          const CompressTask& c = cts[u];
          const int64_t mq = co[c.out_idx].m;
          const int64_t rows = c.mode == 0 ? mq : (c.mode == 1 ? (mq * (c.part + 1)) / c.nparts - (mq * c.part) / c.nparts : c.n);
          sn += c.n;
          nmx3 = std::max<int64_t>(nmx3, c.n);
          nsteps += (rows + ph - 1) / ph * c.n;
          mode_mask |= 1 << c.mode;
        }
        fprintf(stderr, "[flam]   launch key %7d modes %lld tasks %6d sum_n %8lld nmax %5lld steps %10lld  %8.3f ms\n",
                lr.key, (long long)mode_mask, lr.t1 - lr.t0, (long long)sn, (long long)nmx3, (long long)nsteps, tl);
        CK(cudaEventDestroy(lr.e0));
        CK(cudaEventDestroy(lr.e1));
      }
      lrec.clear();
    }
    StepDev sd;
    sd.set(fd, s);
    F.root_rmax = std::max(F.root_rmax, sd.root_rmax());
    F.steps.push_back(std::move(sd));
    // ---- host state for the next step (rskelf.m:245-261)
    for (int q = 0; q < nb; ++q) {
      const int32_t b = boxes[q];
      const int n = (int)nslf[q], k = co[q].k;
      xoff[b] = slf_off[q];
      xlen[b] = (n - k > 0) ? k : n;
      Moff[b] = et[q].M_out;
    }
    // the boxes of an instance's last processed level keep their M blocks: the
    // remaining skeleton system of a partial factorization (rskelf.m:280-308)
    {
      const bool last = step + 1 == nrun;
      std::vector<double> mh;
      if (last) ws.wait_elim(s, par);
      if (last && mtop > 0) mh = download(mpool[cur].p, mtop, s);
      for (int q = 0; q < nb; ++q) {
        const int32_t b = boxes[q];
        const int i = F.binst[b];
        if (!(last || F.nlvl[i] - step == 1) || xlen[b] == 0) continue;
        const int64_t nn = xlen[b] * xlen[b];
        kept.push_back(KeptBlock{i, xoff[b], xlen[b], (int64_t)kept_val.size()});
        kept_val.resize(kept_val.size() + nn);
        if (last) {
          std::copy(mh.begin() + Moff[b], mh.begin() + Moff[b] + nn, kept_val.end() - nn);
        } else {
          ws.wait_elim(s, par);
          auto v = download(mpool[cur].p + Moff[b], nn, s);
          std::copy(v.begin(), v.end(), kept_val.end() - nn);
        }
      }
    }
    // per instance: F.lvp and the verbose table row
    std::vector<int> seen(ninst, 0);
    for (int q = 0; q < nb; ++q) seen[F.binst[boxes[q]]] = 1;
    for (int i = 0; i < ninst; ++i) {
      if (!seen[i]) continue;
      F.inst_lvp[i].push_back((int64_t)F.inst_fac[i].size());
      const int L = F.nlvl[i] - step;
      const int64_t nblk = pblk[i][L] + (int64_t)byl[i][L].size();
      F.stats[i].push_back(LevelStat{L, nblk, rem1[i], F.rem[i]});
    }
    cur ^= 1;
  }
  ws.wait_elim(s, 0);
  ws.wait_elim(s, 1);
  // make sure the pools reflect their sizes
  int32_t st = 0;
  CK(cudaMemcpyAsync(&st, status.p, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  CK(cudaEventRecord(e1, s));
  CK(cudaEventSynchronize(e1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  F.t_factor = ms * 1e-3;
  CK(cudaEventDestroy(e0));
  CK(cudaEventDestroy(e1));
  float gap_elim = 0, gap_next = 0;   // stream time between a step's kernels (host planning)
  for (size_t e = 0; e + 3 < step_ev.size(); e += 4) {
    float tc = 0, tel = 0, g = 0;
    CK(cudaEventElapsedTime(&tc, step_ev[e], step_ev[e + 1]));
    CK(cudaEventElapsedTime(&tel, step_ev[e + 2], step_ev[e + 3]));
    F.prof.t_compress += tc * 1e-3;
    F.prof.t_elim += tel * 1e-3;
    CK(cudaEventElapsedTime(&g, step_ev[e + 1], step_ev[e + 2]));
    gap_elim += g;
    if (e + 4 < step_ev.size()) {
      CK(cudaEventElapsedTime(&g, step_ev[e + 3], step_ev[e + 4]));
      gap_next += g;
    }
  }
  if (prof_print && !step_ev.empty())
    fprintf(stderr, "[flam] gaps: compress->elim %.3f ms  elim->next compress %.3f ms\n", gap_elim, gap_next);
  for (auto& e : step_ev) CK(cudaEventDestroy(e));
  for (auto& e : sk_ev) {
    float t = 0;
    CK(cudaEventElapsedTime(&t, e.first, e.second));
    F.prof.t_sketch += t * 1e-3;
    CK(cudaEventDestroy(e.first));
    CK(cudaEventDestroy(e.second));
  }
  CK(cudaStreamSynchronize(s));
  if (st & ST_NOT_SPD)
    fail(FLAM_ERR_NOT_SPD, "FLAM:rskelf:notPosDef: a redundant block is not positive definite (chol failed)");
  if (st & ST_TIMEOUT)
    fail(FLAM_ERR_TIMEOUT, "FLAM:gpu:timeout: a tensor-core sketch did not complete within its wait limit");
  if (st & ST_SINGULAR) F.warn |= 2;
  ws.hint_ipool = std::max(ws.hint_ipool, F.ipool.n);
  ws.hint_fpool = std::max(ws.hint_fpool, F.fpool.n);
  ws.hint_ppool = std::max(ws.hint_ppool, F.ppool.n);
  assemble_partial(F, kept, kept_val);
}

void print_table(const flam_factor& F) {
  if (F.stats.empty()) return;
  printf("%s\n", std::string(69, '-').c_str());
  printf("%3s | %6s | %19s | %19s | %10s\n", "lvl", "nblk", "start/end npts", "start/end npts/blk", "time (s)");
  printf("%s\n", std::string(69, '-').c_str());
  printf("%3s | %63.2e\n", "t", F.t_tree);
  for (const auto& r : F.stats[0])
    printf("%3lld | %6lld | %8lld | %8lld | %8.2f | %8.2f | %10s\n", (long long)r.lvl, (long long)r.nblk,
           (long long)r.nrem1, (long long)r.nrem2, (double)r.nrem1 / r.nblk, (double)r.nrem2 / r.nblk, "-");
  printf("%s\n", std::string(69, '-').c_str());
  fflush(stdout);
}

flam_status create(int ninst, const double* x, int d, const int64_t* N, const flam_kernel* A, double occ,
                   double rank_or_tol, const flam_proxy* pxy, const flam_opts* opts_in, flam_factor** out) {
  if (!out) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: output handle pointer is NULL");
  *out = nullptr;
  flam_opts o;
  flam_opts_default(&o);
  if (opts_in) o = *opts_in;
  if (ninst < 1) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: need at least one instance");
  if (d < 1 || d > kMaxDim) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidDim: dimension must be 1, 2 or 3");
  if (!x || !A || !N) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: x, N and A must not be NULL");
  if (!(occ >= 0)) fail(FLAM_ERR_ARG, "FLAM:hypoct:invalidOcc: Leaf occupancy must be nonnegative.");
  if (!(rank_or_tol >= 0)) fail(FLAM_ERR_ARG, "FLAM:id:invalidRankOrTol: Rank or tolerance must be nonnegative.");
  if (!(o.Tmax >= 1)) fail(FLAM_ERR_ARG, "FLAM:id:invalidTmax: Interpolation matrix entry bound must be >= 1.");
  char symm = chksymm(o.symm);
  if (o.sketch < 0 || o.sketch > 2)
    fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidSketch: opts.sketch must be 0 (exact ID), 1 (TF32 sketch) or 2 (FP64 sketch)");
  // symm 'h' (LDL of the redundant blocks, rskelf.m:229): there is no LDL on the device, so
  // the factorization takes LU ('n') and warns, as the reference does under Octave
  // (rskelf.m:124-127, FLAM:rskelf:octaveLDL)
  const bool ldl_as_lu = symm == 'h';
  if (ldl_as_lu) symm = 'n';
  flam_proxy px{};
  px.kind = FLAM_PROXY_NONE;
  if (pxy) px = *pxy;
  if (px.kind < 0 || px.kind > 3) fail(FLAM_ERR_ARG, "FLAM:gpu:unsupportedProxy: unknown proxy kind %d", px.kind);
  // px.kind == FLAM_PROXY_NONE: global compression (rskelf.m:204), nothing more to check
  if (px.kind != FLAM_PROXY_NONE) {
    if (px.kind == FLAM_PROXY_RING && d != 2) fail(FLAM_ERR_ARG, "FLAM:gpu:invalidProxy: ring proxy needs d = 2");
    if (px.kind == FLAM_PROXY_SPHERE && d != 3) fail(FLAM_ERR_ARG, "FLAM:gpu:invalidProxy: sphere proxy needs d = 3");
    if (px.p < 1) fail(FLAM_ERR_ARG, "FLAM:gpu:invalidProxy: proxy needs p >= 1 points");
    if (px.kind == FLAM_PROXY_ANNULUS && (px.p_rad < 1 || !(px.param > 0)))
      fail(FLAM_ERR_ARG, "FLAM:gpu:invalidProxy: annulus proxy needs p_rad >= 1 and param > 0");
    if (px.kernel_kind < 0 || px.kernel_kind > 4 || px.kernel_kind == FLAM_KERNEL_LAPLACE2D_DL)
      fail(FLAM_ERR_ARG, "FLAM:gpu:invalidProxy: proxy kernel must be a single-layer registry kernel");
  }
  bool any_w = false, any_n = false;
  for (int i = 0; i < ninst; ++i) {
    if (N[i] < 1) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: every instance needs N >= 1");
    if (A[i].kind < 0 || A[i].kind > 4) fail(FLAM_ERR_ARG, "FLAM:gpu:unsupportedKernel: unknown kernel %d", A[i].kind);
    if (A[i].kind == FLAM_KERNEL_LAPLACE2D_DL && (!A[i].normals || d != 2))
      fail(FLAM_ERR_ARG, "FLAM:gpu:invalidKernel: the 2D double layer needs d = 2 and normals");
    any_w |= A[i].weights != nullptr;
    any_n |= A[i].normals != nullptr;
  }
  if (any_w)
    for (int i = 0; i < ninst; ++i)
      if (!A[i].weights) fail(FLAM_ERR_ARG, "FLAM:gpu:invalidKernel: weights must be given for all instances or none");

  std::unique_ptr<flam_factor> F(new flam_factor());
  CK(cudaGetDevice(&F->dev));
  keep_pool_memory(F->dev);
  F->s = (cudaStream_t)o.stream;
  F->profile = o.profile != 0 || std::getenv("FLAM_PROFILE") != nullptr;
  F->d = d;
  F->ninst = ninst;
  F->symm = symm;
  F->inst_off.assign(ninst + 1, 0);
  for (int i = 0; i < ninst; ++i) F->inst_off[i + 1] = F->inst_off[i] + N[i];
  F->Ntot = F->inst_off[ninst];
  cudaStream_t s = F->s;
  const int64_t ntot = F->Ntot;
  // inputs to the device
  F->x.resize(ntot * d, s);
  CK(cudaMemcpyAsync(F->x.p, x, sizeof(double) * ntot * d, cudaMemcpyDefault, s));
  if (any_w) {
    F->has_w = true;
    F->w.resize(ntot, s);
    for (int i = 0; i < ninst; ++i)
      CK(cudaMemcpyAsync(F->w.p + F->inst_off[i], A[i].weights, sizeof(double) * N[i], cudaMemcpyDefault, s));
  }
  if (any_n) {
    F->has_nrm = true;
    F->nrm.resize(ntot * d, s);
    CK(cudaMemsetAsync(F->nrm.p, 0, sizeof(double) * ntot * d, s));
    for (int i = 0; i < ninst; ++i)
      if (A[i].normals)
        CK(cudaMemcpyAsync(F->nrm.p + F->inst_off[i] * d, A[i].normals, sizeof(double) * N[i] * d,
                           cudaMemcpyDefault, s));
  }
  F->iph.resize(ninst);
  for (int i = 0; i < ninst; ++i) {
    InstParams& p = F->iph[i];
    p.pt_off = F->inst_off[i];
    p.N = N[i];
    p.kind = A[i].kind;
    p.has_w = A[i].weights ? 1 : 0;
    p.has_nrm = A[i].normals ? 1 : 0;
    p.scale = A[i].scale;
    p.dval = A[i].dval;
    p.param = A[i].param;
    p.wbar = 1.0;
    if (A[i].weights) {
      // mean column weight, summed on the host from the caller's array (host or device)
      std::vector<double> wv(N[i]);
      CK(cudaMemcpyAsync(wv.data(), A[i].weights, sizeof(double) * N[i], cudaMemcpyDefault, s));
      CK(cudaStreamSynchronize(s));
      double acc = 0;
      for (double v : wv) acc += v;
      p.wbar = acc / N[i];
    }
    p.pkind = px.kind;
    p.pkernel = px.kernel_kind;
    p.pscale = px.scale;
    p.pparam = px.param;
    p.two_sided = px.two_sided && A[i].weights ? 1 : 0;
  }
  F->ip.upload(F->iph, s);
  std::vector<double> pts, shift;
  proxy_points(px, d, pts, shift);
  F->npxy = (int)(pts.size() / d);
  F->pxy_pts.upload(pts, s);
  if (!shift.empty()) F->pxy_shift.upload(shift, s);

  const bool pp = std::getenv("FLAM_PROFILE") != nullptr;
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto t0 = now();
  CK(cudaStreamSynchronize(s));
  auto t1 = now();
  build_tree(*F, occ, o);
  auto t2 = now();
  factorize(*F, rank_or_tol, o);
  auto t3 = now();
  if (pp)
    fprintf(stderr, "[flam] create: upload %.3f ms  tree %.3f ms (device %.3f)  factorize %.3f ms (device %.3f)\n",
            std::chrono::duration<double, std::milli>(t1 - t0).count(),
            std::chrono::duration<double, std::milli>(t2 - t1).count(), F->t_tree * 1e3,
            std::chrono::duration<double, std::milli>(t3 - t2).count(), F->t_factor * 1e3);
  if (o.verb) print_table(*F);
  *out = F.release();
  if ((*out)->warn & 1) {
    g_err = "FLAM:id:maxIterCount: Maximum number of RRQR iterations reached.";
    return FLAM_WARN_RRQR_MAXITER;
  }
  if ((*out)->warn & 2) {
    g_err = "FLAM:rskelf:singular: an LU pivot of a redundant block was exactly zero";
    return FLAM_WARN_SINGULAR;
  }
  if (ldl_as_lu) {
    g_err = "FLAM:rskelf:octaveLDL: No LDL decomposition on the device; using LU.";
    return FLAM_WARN_LDL_AS_LU;
  }
  return FLAM_OK;
}

// Which halves of the sweeps an apply runs.
enum : int { kUp = 1, kDown = 2, kBoth = 3 };

// Doubles of the point-major work array of an apply: N x nrhs, then the r x nrhs block
// of the largest grid-swept root factor.
int64_t sweep_w_size(const flam_factor* F, int64_t nrhs) { return (F->Ntot + F->root_rmax) * nrhs; }

// The sweep of one step in direction a.op (launches only): the per-box kernel over the
// step's factors, except that a solve sweeps the large root factors grid-wide with the
// scratch block rscr.
void sweep_step(const flam_factor* F, const StepDev& sd, SweepArgs& a, double* rscr, cudaStream_t s) {
  if (sd.nfac == 0) return;
  const bool grid = !sd.roots.empty() && a.op <= 1;
  if (grid) {
    a.fac = sd.sfac.p;
    launch_sweep(a, sd.nsfac, sd.skmax, sd.srmax, s);
    F->prof.launches += sd.nsfac > 0;
    for (const FacDesc& f : sd.roots) {
      const int64_t* rd = F->ipool.p + f.sk_off;
      F->prof.launches += sweep_root_grid(a.X, a.nrhs, rd, F->ppool.p + f.piv_off, F->fpool.p + f.LU_off, f.r, a.op,
                                          a.trans, a.symm, rscr, s);
    }
  } else {
    a.fac = sd.fac.p;
    launch_sweep(a, sd.nfac, sd.kmax, sd.rmax, s);
    F->prof.launches += 1;
  }
  F->prof.n_sweep += 1;
  F->prof.flop_sweep += sd.flop_per_rhs * (double)a.nrhs;
  F->prof.byte_sweep += sd.fac_bytes + 16.0 * sd.x_rows * (double)a.nrhs;
}

// The sweeps on a column-major device block Xd (N x nrhs, leading dimension ld), with the
// point-major work array Wp (N x nrhs) -- launches only, on stream s.
void sweeps_on_device(const flam_factor* F, double* Xd, int64_t ld, int64_t nrhs, double* Wp, int t, bool solve,
                      int halves, cudaStream_t s) {
  const int64_t N = F->Ntot;
  launch_to_pointmajor(Xd, ld, N, (int)nrhs, Wp, s);
  SweepArgs a{};
  a.ipool = F->ipool.p;
  a.fpool = F->fpool.p;
  a.ppool = F->ppool.p;
  a.X = Wp;
  a.ldx = nrhs;
  a.nrhs = (int)nrhs;
  a.trans = t;
  a.symm = F->symm;
  const int ns = (int)F->steps.size();
  double* rscr = Wp + N * nrhs;
  auto sweep = [&](int q) { sweep_step(F, F->steps[q], a, rscr, s); };
  F->prof.launches += 2;
  if (halves & kUp) {
    a.op = solve ? 0 : 2;
    for (int q = 0; q < ns; ++q) sweep(q);
  }
  if (halves & kDown) {
    a.op = solve ? 1 : 3;
    for (int q = ns - 1; q >= 0; --q) sweep(q);
  }
  launch_from_pointmajor(Wp, N, (int)nrhs, Xd, ld, s);
}

// The sweeps of an apply as a CUDA graph.  Once a factorization exists its apply is a
// fixed launch sequence (layout change, one sweep launch per step and direction, layout
// change), so the second apply on the same device buffers and shape captures it (on a
// workspace stream, so that the caller's stream may be the legacy default stream) and
// every later one replays it with one launch.  Returns false when the caller should run
// the launches itself (first sighting, or a step whose sweep allocates scratch).
bool apply_graph(const flam_factor* F, double* Xd, int64_t ld, int64_t nrhs, double* Wp, int t, bool solve,
                 int halves, cudaStream_t s) {
  const flam_factor::GraphKey key{Xd, ld, nrhs, t, solve ? 1 : 0, halves, Wp};
  auto it = F->graphs.find(key);
  if (it == F->graphs.end()) {
    if (F->graph_seen[key]++ == 0) return false;
    for (const StepDev& sd : F->steps) {
      const bool grid = !sd.roots.empty() && solve;
      if (!sweep_in_smem(grid ? sd.skmax : sd.kmax, grid ? sd.srmax : sd.rmax, solve ? 0 : 2)) return false;
    }
    Workspace& ws = workspace(F->dev, s);
    if (!ws.cap) CK(cudaStreamCreateWithFlags(&ws.cap, cudaStreamNonBlocking));
    const flam_prof before = F->prof;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(ws.cap, cudaStreamCaptureModeThreadLocal));
    sweeps_on_device(F, Xd, ld, nrhs, Wp, t, solve, halves, ws.cap);
    CK(cudaStreamEndCapture(ws.cap, &g));
    cudaGraphExec_t ex = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    CK(ei);
    flam_factor::GraphRec rec{ex, {}};
    rec.delta.launches = F->prof.launches - before.launches;
    rec.delta.n_sweep = F->prof.n_sweep - before.n_sweep;
    rec.delta.flop_sweep = F->prof.flop_sweep - before.flop_sweep;
    rec.delta.byte_sweep = F->prof.byte_sweep - before.byte_sweep;
    F->prof = before;
    it = F->graphs.emplace(key, rec).first;
  }
  CK(cudaGraphLaunch(it->second.exec, s));
  F->prof.launches += it->second.delta.launches;
  F->prof.n_sweep += it->second.delta.n_sweep;
  F->prof.flop_sweep += it->second.delta.flop_sweep;
  F->prof.byte_sweep += it->second.delta.byte_sweep;
  F->prof.graph_replays += 1;
  return true;
}

// Apply with X in host memory: the right-hand sides go in two column halves whose
// host->device copy, sweeps and device->host copy overlap (the copies run on the
// workspace's copy stream, ordered by events).  Pinned X gives the overlap; pageable X
// is still correct.
flam_status apply_host_pipelined(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, int t, bool solve,
                                 int halves) {
  const cudaStream_t s = F->s;
  const int64_t N = F->Ntot;
  Workspace& ws = workspace(F->dev, s);
  if (!ws.copy) CK(cudaStreamCreateWithFlags(&ws.copy, cudaStreamNonBlocking));
  const cudaStream_t cs = ws.copy;
  ws.tmp.ensure(N * nrhs, s);
  ws.W.ensure(sweep_w_size(F, nrhs), s);
  constexpr int kChunks = 2;
  cudaEvent_t ev[2 * kChunks + 2];
  for (auto& e : ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  F->resolve_pending();
  CK(cudaEventRecord(ev[0], s));     // the buffers are free once earlier work on s is done
  CK(cudaStreamWaitEvent(cs, ev[0], 0));
  int64_t c0[kChunks + 1];
  for (int c = 0; c <= kChunks; ++c) c0[c] = nrhs * c / kChunks;
  for (int c = 0; c < kChunks; ++c) {
    const int64_t w = c0[c + 1] - c0[c];
    CK(cudaMemcpy2DAsync(ws.tmp.p + N * c0[c], sizeof(double) * N, X + ldx * c0[c], sizeof(double) * ldx,
                         sizeof(double) * N, w, cudaMemcpyHostToDevice, cs));
    CK(cudaEventRecord(ev[1 + c], cs));
  }
  for (int c = 0; c < kChunks; ++c) {
    const int64_t w = c0[c + 1] - c0[c];
    CK(cudaStreamWaitEvent(s, ev[1 + c], 0));
    sweeps_on_device(F, ws.tmp.p + N * c0[c], N, w, ws.W.p + N * c0[c], t, solve, halves, s);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ev[1 + kChunks + c], s));
    CK(cudaStreamWaitEvent(cs, ev[1 + kChunks + c], 0));
    CK(cudaMemcpy2DAsync(X + ldx * c0[c], sizeof(double) * ldx, ws.tmp.p + N * c0[c], sizeof(double) * N,
                         sizeof(double) * N, w, cudaMemcpyDeviceToHost, cs));
  }
  CK(cudaEventRecord(ev[2 * kChunks + 1], cs));
  CK(cudaStreamWaitEvent(s, ev[2 * kChunks + 1], 0));   // later work on s follows the copies
  CK(cudaEventSynchronize(ev[2 * kChunks + 1]));
  for (auto& e : ev) CK(cudaEventDestroy(e));
  return FLAM_OK;
}

// The sweeps of rskelf_sv / rskelf_mv (solve = true / false) on X, in place.
// halves selects the upward and/or downward half; with a skeleton function fn
// (partial factorization) X(Si,:) is passed to fn between the halves
// (rskelf_partial_sv.m:33-62).  sweep_trans overrides trans for the sweeps
// (the Cholesky halves always run the 'n' variant: rskelf_cholsv.m:32-50).
flam_status apply(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans, bool solve,
                  int halves = kBoth, flam_skel_fn fn = nullptr, void* ctx = nullptr, char sweep_trans = 0) {
  if (!F) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: NULL factor");
  trans = chktrans(trans);
  if (nrhs < 0 || ldx < F->Ntot) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: bad X dimensions");
  if (nrhs == 0 || F->Ntot == 0) return FLAM_OK;
  if (!X) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: X is NULL");
  cudaStream_t s = F->s;
  const bool pp = std::getenv("FLAM_PROFILE") != nullptr;
  cudaEvent_t pev[6] = {};
  if (pp)
    for (auto& e : pev) CK(cudaEventCreate(&e));
  auto mark = [&](int i) {
    if (pp) CK(cudaEventRecord(pev[i], s));
  };
  auto hstart = std::chrono::steady_clock::now();
  mark(0);
  const char tc = trans == 'n' ? 'n' : 'c';   // real data: 't' == 'c' (rskelf_sv.m:22)
  const int t = (sweep_trans ? sweep_trans : tc) == 'n' ? 0 : 1;
  const int64_t N = F->Ntot;
  const bool dev = is_device_ptr(X);
  if (!dev && !fn && !pp && nrhs >= 64) return apply_host_pipelined(F, X, ldx, nrhs, t, solve, halves);
  double* Xd = X;
  int64_t ld = ldx;
  Workspace& ws = workspace(F->dev, s);
  // with a skeleton function the work arrays are private to this call: the
  // function may itself apply another factorization on the same stream
  const bool own = fn && F->Sn_tot > 0;
  DBuf<double> own_tmp, own_W, own_Y;
  struct Release {
    DBuf<double>* b[3];
    cudaStream_t s;
    ~Release() {
      for (auto* q : b) q->release(s);
    }
  } release_own{{&own_tmp, &own_W, &own_Y}, s};
  auto& tmp = own ? own_tmp : ws.tmp;
  auto& W = own ? own_W : ws.W;
  if (dev && !fn && !pp && !F->profile) {
    F->resolve_pending();
    W.ensure(sweep_w_size(F, nrhs), s);
    if (apply_graph(F, Xd, ld, nrhs, W.p, t, solve, halves, s)) return FLAM_OK;
  }
  if (!dev) {
    tmp.ensure(N * nrhs, s);
    CK(cudaMemcpy2DAsync(tmp.p, sizeof(double) * N, X, sizeof(double) * ldx, sizeof(double) * N, nrhs,
                         cudaMemcpyHostToDevice, s));
    Xd = tmp.p;
    ld = N;
  }
  W.ensure(sweep_w_size(F, nrhs), s);
  mark(1);
  launch_to_pointmajor(Xd, ld, N, (int)nrhs, W.p, s);
  mark(2);
  SweepArgs a{};
  a.ipool = F->ipool.p;
  a.fpool = F->fpool.p;
  a.ppool = F->ppool.p;
  a.X = W.p;
  a.ldx = nrhs;
  a.nrhs = (int)nrhs;
  a.trans = t;
  a.symm = F->symm;
  const int ns = (int)F->steps.size();
  // profiling: one event pair around the sweep launches (back to back on the
  // stream), read when the profile is next asked for -- no synchronisation here
  F->resolve_pending();
  if (F->profile) {
    CK(cudaEventCreate(&F->pend[0]));
    CK(cudaEventCreate(&F->pend[1]));
    CK(cudaEventRecord(F->pend[0], s));
  }
  // FLAM_PROFILE: one event pair per sweep launch, printed with the step's shape
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> sev;
  std::vector<int> sstep;
  double* rscr = W.p + N * nrhs;
  auto sweep = [&](int q) {
    const StepDev& sd = F->steps[q];
    if (sd.nfac == 0) return;
    if (pp) {
      sev.emplace_back();
      CK(cudaEventCreate(&sev.back().first));
      CK(cudaEventCreate(&sev.back().second));
      CK(cudaEventRecord(sev.back().first, s));
      sstep.push_back(q);
    }
    sweep_step(F, sd, a, rscr, s);
    if (pp) CK(cudaEventRecord(sev.back().second, s));
  };
  F->prof.launches += 2;  // layout changes
  if (halves & kUp) {
    a.op = solve ? 0 : 2;
    for (int q = 0; q < ns; ++q) sweep(q);
  }
  if (fn && F->Sn_tot > 0) {
    // X(Si,:) = fn(X(Si,:), trans) on a column-major copy
    const int64_t Sn = F->Sn_tot;
    auto& Y = own_Y;
    Y.ensure(Sn * nrhs, s);
    launch_rows_pm(W.p, (int)nrhs, F->Si_dev.p, Sn, Y.p, 0, s);
    CK(cudaGetLastError());
    const int rc = fn(Y.p, Sn, nrhs, tc, (void*)s, ctx);
    if (rc != 0 && F->profile) {
      cudaEventDestroy(F->pend[0]);
      cudaEventDestroy(F->pend[1]);
    }
    if (rc != 0)
      fail(FLAM_ERR_ARG, "%s:callback: the skeleton function returned %d",
           solve ? "FLAM:rskelf_partial_sv" : "FLAM:rskelf_partial_mv", rc);
    launch_rows_pm(W.p, (int)nrhs, F->Si_dev.p, Sn, Y.p, 1, s);
    F->prof.launches += 2;
  }
  if (halves & kDown) {
    a.op = solve ? 1 : 3;
    for (int q = ns - 1; q >= 0; --q) sweep(q);
  }
  if (F->profile) {
    CK(cudaEventRecord(F->pend[1], s));
    F->has_pend = true;
  }
  CK(cudaGetLastError());
  mark(3);
  launch_from_pointmajor(W.p, N, (int)nrhs, Xd, ld, s);
  mark(4);
  if (!dev)
    CK(cudaMemcpy2DAsync(X, sizeof(double) * ldx, tmp.p, sizeof(double) * N, sizeof(double) * N, nrhs,
                         cudaMemcpyDeviceToHost, s));
  mark(5);
  if (!dev) CK(cudaStreamSynchronize(s));
  if (pp) {
    auto henq = std::chrono::steady_clock::now();
    CK(cudaEventSynchronize(pev[5]));
    auto hend = std::chrono::steady_clock::now();
    float a[5];
    for (int i = 0; i < 5; ++i) CK(cudaEventElapsedTime(&a[i], pev[i], pev[i + 1]));
    fprintf(stderr, "[flam] apply: alloc %.3f  to_pm %.3f  sweeps %.3f  from_pm %.3f  free %.3f ms  (host enqueue %.3f, wait %.3f ms)\n",
            a[0], a[1], a[2], a[3], a[4], std::chrono::duration<double, std::milli>(henq - hstart).count(),
            std::chrono::duration<double, std::milli>(hend - henq).count());
    for (auto& e : pev) CK(cudaEventDestroy(e));
    for (size_t e = 0; e < sev.size(); ++e) {
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, sev[e].first, sev[e].second));
      const StepDev& sd = F->steps[sstep[e]];
      fprintf(stderr, "[flam] sweep step %2d nfac %6d kmax %4d rmax %4d  %8.3f ms\n", sstep[e], sd.nfac, sd.kmax,
              sd.rmax, ms);
      CK(cudaEventDestroy(sev[e].first));
      CK(cudaEventDestroy(sev[e].second));
    }
  }
  return FLAM_OK;
}

// ---------------------------------------------------------------- FP64 products (K10)
// Yd = A Xd, or Yd = Bd - A Xd, on device blocks (column-major), launches only.
void matvec_device(const flam_factor* F, const double* Xd, int64_t ldx, int64_t nrhs, const double* Bd, int64_t ldb,
                   double* Yd, int64_t ldy, cudaStream_t s) {
  Workspace& ws = workspace(F->dev, s);
  const int tm = matvec_tile_rows((int)nrhs);
  std::vector<MatvecTile> tiles;
  for (int i = 0; i < F->ninst; ++i)
    for (int64_t r = F->inst_off[i]; r < F->inst_off[i + 1]; r += tm)
      tiles.push_back(MatvecTile{r, (int32_t)std::min<int64_t>(tm, F->inst_off[i + 1] - r), i});
  ws.mvt.upload(tiles, s);
  MatvecArgs a{};
  a.P = problem_of(*F);
  a.tiles = ws.mvt.p;
  a.X = Xd;
  a.ldx = ldx;
  a.B = Bd;
  a.ldb = ldb;
  a.Y = Yd;
  a.ldy = ldy;
  a.nrhs = (int)nrhs;
  launch_matvec(a, (int)tiles.size(), s);
  F->prof.launches += 1;
}

void check_matrix(const flam_factor* F) {
  if (!F) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: NULL factor");
  if (!F->x.p || !F->ip.p)
    fail(FLAM_ERR_ARG, "FLAM:gpu:noMatrix: the handle holds no registry matrix (imported factors)");
}

// A block on the device: the caller's pointer if it is device memory, else a copy in buf.
const double* device_block(const double* X, int64_t ldx, int64_t N, int64_t nrhs, DBuf<double>& buf, int64_t* ld,
                           cudaStream_t s) {
  if (is_device_ptr(X)) {
    *ld = ldx;
    return X;
  }
  buf.ensure(N * nrhs, s);
  CK(cudaMemcpy2DAsync(buf.p, sizeof(double) * N, X, sizeof(double) * ldx, sizeof(double) * N, nrhs,
                       cudaMemcpyHostToDevice, s));
  *ld = N;
  return buf.p;
}

flam_status matvec(const flam_factor* F, const double* X, int64_t ldx, int64_t nrhs, const double* B, int64_t ldb,
                   double* Y, int64_t ldy) {
  check_matrix(F);
  const int64_t N = F->Ntot;
  if (nrhs < 0 || ldx < N || ldy < N || (B && ldb < N)) fail(FLAM_ERR_ARG, "FLAM:matvec:invalidArg: bad dimensions");
  if (nrhs == 0) return FLAM_OK;
  if (!X || !Y) fail(FLAM_ERR_ARG, "FLAM:matvec:invalidArg: X and Y must not be NULL");
  const cudaStream_t s = F->s;
  Workspace& ws = workspace(F->dev, s);
  int64_t lx = 0, lb = 0;
  const double* Xd = device_block(X, ldx, N, nrhs, ws.irX, &lx, s);
  const double* Bd = B ? device_block(B, ldb, N, nrhs, ws.irB, &lb, s) : nullptr;
  const bool ydev = is_device_ptr(Y);
  double* Yd = Y;
  int64_t ly = ldy;
  if (!ydev) {
    ws.irR.ensure(N * nrhs, s);
    Yd = ws.irR.p;
    ly = N;
  }
  matvec_device(F, Xd, lx, nrhs, Bd, lb, Yd, ly, s);
  CK(cudaGetLastError());
  if (!ydev) {
    CK(cudaMemcpy2DAsync(Y, sizeof(double) * ldy, Yd, sizeof(double) * N, sizeof(double) * N, nrhs,
                         cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  }
  return FLAM_OK;
}

// X = A \ B by iterative refinement on the handle's factorization: X = F \ B, then while
// max_j ||B_j - A X_j|| / ||B_j|| > tol: X += F \ (B - A X), with the FP64 residual of
// matvec_device.  The factorization may be loose (a larger rank_or_tol) or mixed precision;
// the residual, and so the reported error, is FP64.
flam_status ir_solve(const flam_factor* F, const double* B, int64_t ldb, double* X, int64_t ldx, int64_t nrhs,
                     double tol, int maxit, int* iters, double* relres) {
  check_matrix(F);
  const int64_t N = F->Ntot;
  if (nrhs < 0 || ldx < N || ldb < N) fail(FLAM_ERR_ARG, "FLAM:rskelf_ir_sv:invalidArg: bad dimensions");
  if (!(tol >= 0) || maxit < 0) fail(FLAM_ERR_ARG, "FLAM:rskelf_ir_sv:invalidArg: need ir_tol >= 0, max_iter >= 0");
  if (F->Sn_tot > 0) fail(FLAM_ERR_ARG, "FLAM:rskelf_ir_sv:partial: needs a complete factorization");
  if (F->symm == 'h') fail(FLAM_ERR_UNSUPPORTED, "FLAM:gpu:unsupportedSymm: symm 'h'");
  if (iters) *iters = 0;
  if (nrhs == 0) return FLAM_OK;
  if (!B || !X) fail(FLAM_ERR_ARG, "FLAM:rskelf_ir_sv:invalidArg: B and X must not be NULL");
  const cudaStream_t s = F->s;
  Workspace& ws = workspace(F->dev, s);
  F->resolve_pending();
  int64_t lb = 0;
  const double* Bd = device_block(B, ldb, N, nrhs, ws.irB, &lb, s);
  const bool xdev = is_device_ptr(X);
  double* Xd = X;
  int64_t lx = ldx;
  if (!xdev) {
    ws.irX.ensure(N * nrhs, s);
    Xd = ws.irX.p;
    lx = N;
  }
  ws.irR.ensure(N * nrhs, s);
  ws.W.ensure(sweep_w_size(F, nrhs), s);
  ws.colsq.ensure(6 * nrhs, s);   // column norms and the conjugate-gradient coefficients
  double* R = ws.irR.p;
  // X = F \ B
  CK(cudaMemcpy2DAsync(Xd, sizeof(double) * lx, Bd, sizeof(double) * lb, sizeof(double) * N, nrhs,
                       cudaMemcpyDeviceToDevice, s));
  sweeps_on_device(F, Xd, lx, nrhs, ws.W.p, 0, true, kBoth, s);
  launch_colsq(Bd, N, lb, (int)nrhs, ws.colsq.p + nrhs, s);
  std::vector<double> bn;
  double worst = 0;
  int it = 0;
  if (F->symm == 'p') {
    // A and F symmetric positive definite: conjugate gradients preconditioned by F (one
    // FP64 product and one solve per step, like stationary refinement, but a spectrum of
    // F^-1 A spread by an ill-conditioned A still converges); column-wise coefficients
    ws.irW.ensure(2 * N * nrhs, s);
    double* P = ws.irW.p;        // search directions
    double* Q = P + N * nrhs;    // A P, then the preconditioned residual Z
    double* dv = ws.colsq.p;     // [ r.r | b.b | p.q | r.z | alpha | beta ]
    auto cs = download(dv + nrhs, nrhs, s);   // |B|^2 (launched above)
    matvec_device(F, Xd, lx, nrhs, Bd, lb, R, N, s);                 // R = B - A X0
    CK(cudaMemcpy2DAsync(P, sizeof(double) * N, R, sizeof(double) * N, sizeof(double) * N, nrhs,
                         cudaMemcpyDeviceToDevice, s));
    sweeps_on_device(F, P, N, nrhs, ws.W.p, 0, true, kBoth, s);       // P = Z0 = F \ R0
    launch_coldot(R, N, P, N, N, (int)nrhs, dv + 3 * nrhs, s);        // rho = r.z
    auto rho = download(dv + 3 * nrhs, nrhs, s);
    std::vector<double> al(nrhs), be(nrhs);
    for (;;) {
      launch_colsq(R, N, N, (int)nrhs, dv, s);
      CK(cudaGetLastError());
      auto rr = download(dv, nrhs, s);
      worst = 0;
      for (int64_t c = 0; c < nrhs; ++c) {
        const double v = cs[c] > 0 ? std::sqrt(rr[c] / cs[c]) : std::sqrt(rr[c]);
        if (relres) relres[c] = v;
        worst = std::max(worst, v);
      }
      if (!(worst > tol) || it >= maxit) break;
      matvec_device(F, P, N, nrhs, nullptr, 0, Q, N, s);             // Q = A P
      launch_coldot(P, N, Q, N, N, (int)nrhs, dv + 2 * nrhs, s);
      auto pq = download(dv + 2 * nrhs, nrhs, s);
      for (int64_t c = 0; c < nrhs; ++c) al[c] = (pq[c] != 0.0 && rho[c] != 0.0) ? rho[c] / pq[c] : 0.0;
      CK(cudaMemcpyAsync(dv + 4 * nrhs, al.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, s));
      launch_axpby_cols(Xd, lx, P, N, nullptr, dv + 4 * nrhs, N, (int)nrhs, s);   // X += alpha P
      for (int64_t c = 0; c < nrhs; ++c) al[c] = -al[c];
      CK(cudaMemcpyAsync(dv + 4 * nrhs, al.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, s));
      launch_axpby_cols(R, N, Q, N, nullptr, dv + 4 * nrhs, N, (int)nrhs, s);     // R -= alpha Q
      CK(cudaMemcpy2DAsync(Q, sizeof(double) * N, R, sizeof(double) * N, sizeof(double) * N, nrhs,
                           cudaMemcpyDeviceToDevice, s));
      sweeps_on_device(F, Q, N, nrhs, ws.W.p, 0, true, kBoth, s);    // Z = F \ R
      launch_coldot(R, N, Q, N, N, (int)nrhs, dv + 3 * nrhs, s);
      auto rn = download(dv + 3 * nrhs, nrhs, s);
      std::vector<double> one(nrhs, 1.0);
      for (int64_t c = 0; c < nrhs; ++c) be[c] = rho[c] != 0.0 ? rn[c] / rho[c] : 0.0;
      rho = rn;
      CK(cudaMemcpyAsync(dv + 5 * nrhs, be.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(dv + 4 * nrhs, one.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, s));
      launch_axpby_cols(P, N, Q, N, dv + 5 * nrhs, dv + 4 * nrhs, N, (int)nrhs, s);  // P = Z + beta P
      F->prof.launches += 6;
      ++it;
    }
    // the reported error is the true FP64 residual, not the recurrence
    matvec_device(F, Xd, lx, nrhs, Bd, lb, R, N, s);
    launch_colsq(R, N, N, (int)nrhs, dv, s);
    auto rr = download(dv, nrhs, s);
    worst = 0;
    for (int64_t c = 0; c < nrhs; ++c) {
      const double v = cs[c] > 0 ? std::sqrt(rr[c] / cs[c]) : std::sqrt(rr[c]);
      if (relres) relres[c] = v;
      worst = std::max(worst, v);
    }
  }
  for (; F->symm != 'p';) {
    matvec_device(F, Xd, lx, nrhs, Bd, lb, R, N, s);   // R = B - A X
    launch_colsq(R, N, N, (int)nrhs, ws.colsq.p, s);
    CK(cudaGetLastError());
    auto cs = download(ws.colsq.p, 2 * nrhs, s);
    worst = 0;
    for (int64_t c = 0; c < nrhs; ++c) {
      const double rr = cs[nrhs + c] > 0 ? std::sqrt(cs[c] / cs[nrhs + c]) : std::sqrt(cs[c]);
      if (relres) relres[c] = rr;
      worst = std::max(worst, rr);
    }
    if (!(worst > tol) || it >= maxit) break;
    sweeps_on_device(F, R, N, nrhs, ws.W.p, 0, true, kBoth, s);   // R = F \ R
    launch_add_cols(Xd, lx, R, N, N, (int)nrhs, s);                 // X += R
    F->prof.launches += 1;
    ++it;
  }
  if (iters) *iters = it;
  if (!xdev) {
    CK(cudaMemcpy2DAsync(X, sizeof(double) * ldx, Xd, sizeof(double) * lx, sizeof(double) * N, nrhs,
                         cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  }
  if (!std::isfinite(worst) || worst > tol) {
    char buf[160];
    snprintf(buf, sizeof buf, "FLAM:rskelf_ir_sv:notConverged: relative residual %.3e after %d refinement steps",
             worst, it);
    g_err = buf;
    return FLAM_WARN_IR_NOT_CONVERGED;
  }
  return FLAM_OK;
}

template <class Fn>
flam_status guard(Fn&& fn) {
  try {
    return fn();
  } catch (const FlamError& e) {
    g_err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_err = std::string("FLAM:gpu:internal: ") + e.what();
    return FLAM_ERR_CUDA;
  }
}

}  // namespace

void set_last_error(const char* msg) { g_err = msg; }

cudaError_t ensure_smem_attr(const void* func, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> done;   // (kernel, device) -> bytes set
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  auto it = done.find({func, dev});
  if (it != done.end() && it->second >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done[{func, dev}] = bytes;
  return e;
}

}  // namespace flam

extern "C" {

void flam_opts_default(flam_opts* o) {
  if (!o) return;
  o->lvlmax = 0;
  o->ext = nullptr;
  o->Tmax = 2.0;
  o->rrqr_iter = -1;
  o->symm = 'n';
  o->stop = -1;
  o->verb = 0;
  o->stream = nullptr;
  o->profile = 0;
  o->sketch = 0;
  o->sketch_p = 8;
  o->sketch_guard = 2;
  o->sketch_seed = 0x5eed1234u;
  o->predictor = nullptr;
  o->rank_log = 0;
}

flam_status flam_rskelf(const double* x, int d, int64_t N, const flam_kernel* A, double occ, double rank_or_tol,
                        const flam_proxy* pxy, const flam_opts* opts, flam_factor** F) {
  return guard([&] { return create(1, x, d, &N, A, occ, rank_or_tol, pxy, opts, F); });
}

flam_status flam_hypoct(const double* x, int d, int64_t N, double occ, int lvlmax, const double* ext, void* stream,
                        flam_factor** T) {
  return guard([&] {
    if (!T) fail(FLAM_ERR_ARG, "FLAM:hypoct:invalidArg: output handle pointer is NULL");
    *T = nullptr;
    if (!x || N < 1 || d < 1 || d > kMaxDim) fail(FLAM_ERR_ARG, "FLAM:hypoct:invalidArg: bad points");
    if (!(occ >= 0)) fail(FLAM_ERR_ARG, "FLAM:hypoct:invalidOcc: Leaf occupancy must be nonnegative.");
    std::unique_ptr<flam_factor> F(new flam_factor());
    CK(cudaGetDevice(&F->dev));
    F->s = (cudaStream_t)stream;
    F->d = d;
    F->ninst = 1;
    F->inst_off = {0, N};
    F->Ntot = N;
    F->x.resize(N * d, F->s);
    CK(cudaMemcpyAsync(F->x.p, x, sizeof(double) * N * d, cudaMemcpyDefault, F->s));
    flam_opts o;
    flam_opts_default(&o);
    o.lvlmax = lvlmax;
    o.ext = ext;
    build_tree(*F, occ, o);
    F->rem.assign(1, N);
    F->inst_fac.assign(1, {});
    F->inst_lvp.assign(1, {0});
    F->stats.assign(1, {});
    *T = F.release();
    return FLAM_OK;
  });
}

flam_status flam_id(const double* A, int64_t m, int64_t n, int64_t lda, double rank_or_tol, double Tmax,
                    int64_t rrqr_iter, int64_t* k, int64_t* perm, double* T, int64_t* niter) {
  return guard([&] {
    if (!(rank_or_tol >= 0)) fail(FLAM_ERR_ARG, "FLAM:id:invalidRankOrTol: Rank or tolerance must be nonnegative.");
    if (!(Tmax >= 1)) fail(FLAM_ERR_ARG, "FLAM:id:invalidTmax: Interpolation matrix entry bound must be >= 1.");
    if (m < 0 || n < 0 || (m > 0 && lda < m)) fail(FLAM_ERR_ARG, "FLAM:id:invalidArg: bad matrix dimensions");
    if (n > 4096 || m > (int64_t)1 << 30) fail(FLAM_ERR_ARG, "FLAM:id:invalidArg: matrix too large for flam_id");
    if (!k || !perm) fail(FLAM_ERR_ARG, "FLAM:id:invalidArg: NULL output");
    cudaStream_t s = nullptr;
    if (n == 0) {
      *k = 0;
      if (niter) *niter = 0;
      return FLAM_OK;
    }
    DBuf<double> Ad, tp, scr, dummy;
    DBuf<int64_t> ids, cp;
    DBuf<int32_t> pp;
    DBuf<CompressTask> tk;
    DBuf<CompressOut> co;
    DBuf<InstParams> ipd;
    Ad.resize(std::max<int64_t>(m * n, 1), s);
    if (m > 0) CK(cudaMemcpy2DAsync(Ad.p, sizeof(double) * m, A, sizeof(double) * lda, sizeof(double) * m, n,
                                    cudaMemcpyDefault, s));
    std::vector<int64_t> iv(n);
    for (int64_t q = 0; q < n; ++q) iv[q] = q;
    ids.upload(iv, s);
    cp.resize(1, s);
    tp.resize(n * n / 4 + 1, s);
    pp.resize(n, s);
    CompressTask t{};
    t.slf_off = 0;
    t.cand_off = 0;
    t.T_off = 0;
    t.perm_off = 0;
    t.n = (int32_t)n;
    t.ncand = (int32_t)m;
    t.flags = 0;
    if (n > kSmemN) {
      scr.resize(compress_scratch_doubles((int)n), s);
      t.scr_off = 0;
    } else {
      scr.resize(1, s);
      t.scr_off = -1;
    }
    tk.upload(std::vector<CompressTask>{t}, s);
    co.resize(1, s);
    InstParams ip{};
    ipd.upload(std::vector<InstParams>{ip}, s);
    dummy.resize(4, s);
    CompressArgs ca{};
    ca.P.d = 1;
    ca.P.x = dummy.p;
    ca.P.ip = ipd.p;
    ca.P.pxy_pts = dummy.p;
    ca.tasks = tk.p;
    ca.ipool = ids.p;
    ca.cpool = cp.p;
    ca.tpool = tp.p;
    ca.permpool = pp.p;
    ca.scratch = scr.p;
    ca.out = co.p;
    ca.rel_tol = std::fmod(rank_or_tol, 1.0);
    ca.kmax = (int)std::min<double>(std::floor(rank_or_tol), 2e9);
    ca.symm_n = 0;
    ca.Tmax = Tmax;
    ca.rrqr_iter = rrqr_iter;
    ca.Aexp = Ad.p;
    ca.lda = m;
    launch_compress(ca, 1, compress_smem_bytes((int)n), s);
    CK(cudaGetLastError());
    auto o = download(co.p, 1, s);
    auto pv = download(pp.p, n, s);
    *k = o[0].k;
    for (int64_t q = 0; q < n; ++q) perm[q] = pv[q];
    if (niter) *niter = o[0].niter;
    if (T && o[0].k > 0 && o[0].k < n) {
      auto tv = download(tp.p, (int64_t)o[0].k * (n - o[0].k), s);
      std::copy(tv.begin(), tv.end(), T);
    }
    for (auto* b : {&Ad, &tp, &scr, &dummy}) b->release(s);
    ids.release(s);
    cp.release(s);
    pp.release(s);
    tk.release(s);
    co.release(s);
    ipd.release(s);
    CK(cudaStreamSynchronize(s));
    if (o[0].status & ST_RRQR_CAP) {
      g_err = "FLAM:id:maxIterCount: Maximum number of RRQR iterations reached.";
      return FLAM_WARN_RRQR_MAXITER;
    }
    return FLAM_OK;
  });
}

flam_status flam_rskelf_batched(int ninst, const double* x, int d, const int64_t* N, const flam_kernel* A,
                                double occ, double rank_or_tol, const flam_proxy* pxy, const flam_opts* opts,
                                flam_factor** F) {
  return guard([&] { return create(ninst, x, d, N, A, occ, rank_or_tol, pxy, opts, F); });
}

flam_status flam_matvec(const flam_factor* F, const double* X, int64_t ldx, int64_t nrhs, const double* B, int64_t ldb,
                        double* Y, int64_t ldy) {
  return guard([&] { return matvec(F, X, ldx, nrhs, B, ldb, Y, ldy); });
}

flam_status flam_rskelf_ir_sv(const flam_factor* F, const double* B, int64_t ldb, double* X, int64_t ldx, int64_t nrhs,
                              double ir_tol, int max_iter, int* iters, double* relres) {
  return guard([&] { return ir_solve(F, B, ldb, X, ldx, nrhs, ir_tol, max_iter, iters, relres); });
}

// ---------------------------------------------------------------- rank predictor
flam_status flam_predictor_create(uint64_t seed, flam_predictor** P) {
  return guard([&] {
    if (!P) fail(FLAM_ERR_ARG, "FLAM:predictor:invalidArg: NULL output");
    *P = nullptr;
    std::unique_ptr<flam_predictor> p(new flam_predictor());
    CK(cudaGetDevice(&p->dev));
    // He initialisation (Box-Muller on a splitmix64 stream), zero biases
    std::vector<float> w(FLAM_PREDICTOR_NPARAM, 0.f);
    uint64_t st = seed + 0x9E3779B97F4A7C15ull;
    auto next = [&]() {
      uint64_t z = (st += 0x9E3779B97F4A7C15ull);
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      return ((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
    };
    auto gauss = [&]() {
      const double u1 = std::max(next(), 1e-300), u2 = next();
      return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    };
    const int nin = FLAM_PREDICTOR_NFEAT, nh = 128;
    for (int e = 0; e < nh * nin; ++e) w[e] = (float)(gauss() * std::sqrt(2.0 / nin));
    const int w2 = nh * nin + nh;
    for (int e = 0; e < nh * nh; ++e) w[w2 + e] = (float)(gauss() * std::sqrt(2.0 / nh));
    const int w3 = w2 + nh * nh + nh;
    for (int e = 0; e < nh; ++e) w[w3 + e] = (float)(gauss() * std::sqrt(1.0 / nh));
    p->w.upload(w, nullptr);
    std::vector<float> z(FLAM_PREDICTOR_NPARAM, 0.f);
    p->m.upload(z, nullptr);
    p->v.upload(z, nullptr);
    p->grad.upload(z, nullptr);
    p->scal.ensure(4, nullptr);
    CK(cudaStreamSynchronize(nullptr));
    *P = p.release();
    return FLAM_OK;
  });
}

void flam_predictor_free(flam_predictor* P) { delete P; }

flam_status flam_predictor_get(const flam_predictor* P, float* w) {
  return guard([&] {
    if (!P || !w) fail(FLAM_ERR_ARG, "FLAM:predictor:invalidArg: NULL argument");
    CK(cudaMemcpy(w, P->w.p, sizeof(float) * FLAM_PREDICTOR_NPARAM, cudaMemcpyDefault));
    return FLAM_OK;
  });
}

flam_status flam_predictor_set(flam_predictor* P, const float* w) {
  return guard([&] {
    if (!P || !w) fail(FLAM_ERR_ARG, "FLAM:predictor:invalidArg: NULL argument");
    CK(cudaMemcpy(P->w.p, w, sizeof(float) * FLAM_PREDICTOR_NPARAM, cudaMemcpyDefault));
    CK(cudaMemset(P->m.p, 0, sizeof(float) * FLAM_PREDICTOR_NPARAM));
    CK(cudaMemset(P->v.p, 0, sizeof(float) * FLAM_PREDICTOR_NPARAM));
    P->step = 0;
    return FLAM_OK;
  });
}

namespace {
void pred_inputs(flam_predictor* P, const float* X, const float* y, int64_t nsamp) {
  if (nsamp < 0) fail(FLAM_ERR_ARG, "FLAM:predictor:invalidArg: nsamp < 0");
  if (nsamp == 0) return;
  if (!X) fail(FLAM_ERR_ARG, "FLAM:predictor:invalidArg: X is NULL");
  P->X.ensure(nsamp * FLAM_PREDICTOR_NFEAT, nullptr);
  CK(cudaMemcpy(P->X.p, X, sizeof(float) * nsamp * FLAM_PREDICTOR_NFEAT, cudaMemcpyDefault));
  if (y) {
    P->y.ensure(nsamp, nullptr);
    CK(cudaMemcpy(P->y.p, y, sizeof(float) * nsamp, cudaMemcpyDefault));
  }
}
}  // namespace

flam_status flam_predictor_train(flam_predictor* P, const float* X, const float* y, int64_t nsamp, int epochs,
                                 int batch, float lr, uint64_t seed, float* loss) {
  return guard([&] {
    if (!P || !y) fail(FLAM_ERR_ARG, "FLAM:predictor:invalidArg: NULL argument");
    if (epochs < 0 || batch < 1 || !(lr > 0)) fail(FLAM_ERR_ARG, "FLAM:predictor:invalidArg: epochs, batch or lr");
    if (nsamp == 0) return FLAM_OK;
    // shuffled copies per epoch (the samples are small: 68 bytes each)
    std::vector<float> hx((size_t)nsamp * FLAM_PREDICTOR_NFEAT), hy((size_t)nsamp);
    CK(cudaMemcpy(hx.data(), X, sizeof(float) * hx.size(), cudaMemcpyDefault));
    CK(cudaMemcpy(hy.data(), y, sizeof(float) * hy.size(), cudaMemcpyDefault));
    std::vector<int64_t> idx((size_t)nsamp);
    uint64_t st = seed * 0x2545F4914F6CDD1Dull + 1;
    auto rnd = [&]() {
      st ^= st >> 12;
      st ^= st << 25;
      st ^= st >> 27;
      return st * 0x2545F4914F6CDD1Dull;
    };
    std::vector<float> sx(hx.size()), sy(hy.size());
    double last = 0;
    for (int ep = 0; ep < epochs; ++ep) {
      for (int64_t i = 0; i < nsamp; ++i) idx[i] = i;
      for (int64_t i = nsamp - 1; i > 0; --i) std::swap(idx[i], idx[rnd() % (uint64_t)(i + 1)]);
      for (int64_t i = 0; i < nsamp; ++i) {
        std::memcpy(&sx[(size_t)i * FLAM_PREDICTOR_NFEAT], &hx[(size_t)idx[i] * FLAM_PREDICTOR_NFEAT],
                    sizeof(float) * FLAM_PREDICTOR_NFEAT);
        sy[i] = hy[idx[i]];
      }
      pred_inputs(P, sx.data(), sy.data(), nsamp);
      CK(cudaMemset(P->scal.p, 0, sizeof(float)));
      for (int64_t b0 = 0; b0 < nsamp; b0 += batch) {
        const int64_t nbat = std::min<int64_t>(batch, nsamp - b0);
        launch_mlp(P->X.p + b0 * FLAM_PREDICTOR_NFEAT, P->y.p + b0, nbat, P->w.p, nullptr, P->grad.p, P->scal.p,
                   1.f / (float)nbat, 1, nullptr);
        launch_adam(P->w.p, P->m.p, P->v.p, P->grad.p, lr, ++P->step, nullptr);
      }
      CK(cudaGetLastError());
      float sse = 0;
      CK(cudaMemcpy(&sse, P->scal.p, sizeof(float), cudaMemcpyDeviceToHost));
      last = sse / (double)nsamp;
    }
    if (loss) *loss = (float)last;
    return FLAM_OK;
  });
}

flam_status flam_predictor_eval(const flam_predictor* P, const float* X, int64_t nsamp, float* yhat) {
  return guard([&] {
    if (!P || !yhat) fail(FLAM_ERR_ARG, "FLAM:predictor:invalidArg: NULL argument");
    auto* Q = const_cast<flam_predictor*>(P);
    pred_inputs(Q, X, nullptr, nsamp);
    if (nsamp == 0) return FLAM_OK;
    Q->yhat.ensure(nsamp, nullptr);
    launch_mlp(Q->X.p, nullptr, nsamp, Q->w.p, Q->yhat.p, nullptr, nullptr, 0.f, 0, nullptr);
    CK(cudaGetLastError());
    CK(cudaMemcpy(yhat, Q->yhat.p, sizeof(float) * nsamp, cudaMemcpyDefault));
    return FLAM_OK;
  });
}

flam_status flam_predictor_grad(const flam_predictor* P, const float* X, const float* y, int64_t nsamp, float* loss,
                                float* grad) {
  return guard([&] {
    if (!P || !y || !grad || nsamp < 1) fail(FLAM_ERR_ARG, "FLAM:predictor:invalidArg: NULL argument or no samples");
    auto* Q = const_cast<flam_predictor*>(P);
    pred_inputs(Q, X, y, nsamp);
    DBuf<float> g;
    g.ensure(FLAM_PREDICTOR_NPARAM + 1, nullptr);
    CK(cudaMemset(g.p, 0, sizeof(float) * (FLAM_PREDICTOR_NPARAM + 1)));
    launch_mlp(Q->X.p, Q->y.p, nsamp, Q->w.p, nullptr, g.p, g.p + FLAM_PREDICTOR_NPARAM, 1.f / (float)nsamp, 1,
               nullptr);
    CK(cudaGetLastError());
    std::vector<float> h(FLAM_PREDICTOR_NPARAM + 1);
    CK(cudaMemcpy(h.data(), g.p, sizeof(float) * h.size(), cudaMemcpyDeviceToHost));
    g.release(nullptr);
    std::copy(h.begin(), h.begin() + FLAM_PREDICTOR_NPARAM, grad);
    if (loss) *loss = h[FLAM_PREDICTOR_NPARAM] / (float)nsamp;
    return FLAM_OK;
  });
}

flam_status flam_rank_log(const flam_factor* F, int64_t* count, float* X, float* y) {
  return guard([&] {
    if (!F || !count) fail(FLAM_ERR_ARG, "FLAM:rank_log:invalidArg: NULL argument");
    *count = (int64_t)F->rlog_y.size();
    if (X) std::copy(F->rlog_X.begin(), F->rlog_X.end(), X);
    if (y) std::copy(F->rlog_y.begin(), F->rlog_y.end(), y);
    return FLAM_OK;
  });
}

flam_status flam_tune_get(int d, int kernel_kind, int64_t N, flam_tune* t) {
  return guard([&] {
    if (!t) fail(FLAM_ERR_ARG, "FLAM:tune:invalidArg: NULL output");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    *t = tune_lookup(tune_key(dev, d, kernel_kind, N));
    return FLAM_OK;
  });
}

flam_status flam_tune_set(int d, int kernel_kind, int64_t N, const flam_tune* t) {
  return guard([&] {
    if (!t) fail(FLAM_ERR_ARG, "FLAM:tune:invalidArg: NULL argument");
    tune_check(*t);
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[tune_key(dev, d, kernel_kind, N)] = *t;
    return FLAM_OK;
  });
}

flam_status flam_autotune(const double* x, int d, int64_t N, const flam_kernel* A, double occ, double rank_or_tol,
                          const flam_proxy* pxy, const flam_opts* opts, int reps, flam_tune* best) {
  return guard([&] {
    if (!A || !best) fail(FLAM_ERR_ARG, "FLAM:tune:invalidArg: NULL argument");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    const TuneKey key = tune_key(dev, d, A->kind, N);
    reps = std::max(1, reps);
    flam_opts o;
    flam_opts_default(&o);
    if (opts) o = *opts;
    o.verb = 0;
    o.profile = 0;
    // device time of the factorization with setting t (the fastest of reps runs)
    auto measure = [&](const flam_tune& t) {
      {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[key] = t;
      }
      double tb = 1e300;
      for (int r = 0; r < reps; ++r) {
        flam_factor* F = nullptr;
        const flam_status st = create(1, x, d, &N, A, occ, rank_or_tol, pxy, &o, &F);
        if (st != FLAM_OK && st < 100) fail(st, "%s", g_err.c_str());
        tb = std::min(tb, F->t_tree + F->t_factor);
        flam_factor_free(F);
      }
      return tb;
    };
    flam_tune cur = tune_lookup(key);
    double tbest = measure(cur);
    const std::vector<int> c_ctas{74, 148, 296}, c_max{2, 4, 8, 16}, c_min{16, 32, 64, 128},
        c_smem{0, 40 * 1024, 96 * 1024, 200 * 1024};
    auto sweep = [&](int flam_tune::*field, const std::vector<int>& vals) {
      for (int v : vals) {
        if (cur.*field == v) continue;
        flam_tune t = cur;
        t.*field = v;
        const double tm = measure(t);
        if (tm < tbest) {
          tbest = tm;
          cur = t;
        }
      }
    };
    sweep(&flam_tune::split_ctas, c_ctas);
    sweep(&flam_tune::split_max, c_max);
    sweep(&flam_tune::split_min_n, c_min);
    sweep(&flam_tune::tc_smem_max, c_smem);
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      g_tune[key] = cur;
    }
    *best = cur;
    return FLAM_OK;
  });
}

flam_status flam_rskelf_sv(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans) {
  return guard([&] { return apply(F, X, ldx, nrhs, trans, true); });
}

flam_status flam_rskelf_mv(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans) {
  return guard([&] { return apply(F, X, ldx, nrhs, trans, false); });
}

flam_status flam_rskelf_cholmv(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans) {
  return guard([&] {
    if (F && F->symm != 'p') fail(FLAM_ERR_ARG, "FLAM:rskelf_cholmv:invalidSymm: Symmetry parameter must be 'P'.");
    const char t = F ? chktrans(trans) : 'n';
    return apply(F, X, ldx, nrhs, trans, false, t == 'n' ? kDown : kUp, nullptr, nullptr, 'n');
  });
}

flam_status flam_rskelf_cholsv(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans) {
  return guard([&] {
    if (F && F->symm != 'p') fail(FLAM_ERR_ARG, "FLAM:rskelf_cholsv:invalidSymm: Symmetry parameter must be 'P'.");
    const char t = F ? chktrans(trans) : 'n';
    return apply(F, X, ldx, nrhs, trans, true, t == 'n' ? kUp : kDown, nullptr, nullptr, 'n');
  });
}

flam_status flam_rskelf_partial_sv(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans,
                                   flam_skel_fn fn, void* ctx) {
  return guard([&] {
    if (!fn) fail(FLAM_ERR_ARG, "FLAM:rskelf_partial_sv:invalidArg: svfun is NULL");
    return apply(F, X, ldx, nrhs, trans, true, kBoth, fn, ctx);
  });
}

flam_status flam_rskelf_partial_mv(const flam_factor* F, double* X, int64_t ldx, int64_t nrhs, char trans,
                                   flam_skel_fn fn, void* ctx) {
  return guard([&] {
    if (!fn) fail(FLAM_ERR_ARG, "FLAM:rskelf_partial_mv:invalidArg: mvfun is NULL");
    return apply(F, X, ldx, nrhs, trans, false, kBoth, fn, ctx);
  });
}

flam_status flam_rskelf_logdet(const flam_factor* F, double* re, double* im) {
  return guard([&] {
    if (!F) fail(FLAM_ERR_ARG, "FLAM:rskelf_logdet:invalidArg: NULL factor");
    if (F->symm == 'h') fail(FLAM_ERR_UNSUPPORTED, "FLAM:gpu:unsupportedSymm: symm 'h' is not built on the device");
    const cudaStream_t s = F->s;
    const int64_t nf = (int64_t)F->hfac.size();
    std::vector<double> sr(F->ninst, 0.0);
    std::vector<int64_t> par(F->ninst, 0);
    if (nf > 0) {
      DBuf<double> out;
      out.resize(2 * nf, s);
      int64_t base = 0;
      for (const StepDev& sd : F->steps) {
        launch_logdet(sd.fac.p, sd.nfac, F->fpool.p, F->ppool.p, F->symm == 'p', out.p + 2 * base, s);
        F->prof.launches += sd.nfac > 0;
        base += sd.nfac;
      }
      CK(cudaGetLastError());
      auto h = download(out.p, 2 * nf, s);
      out.release(s);
      // per instance, in factor order (rskelf_logdet.m:18-29)
      for (int i = 0; i < F->ninst; ++i)
        for (int64_t f : F->inst_fac[i]) {
          sr[i] += h[2 * f];
          par[i] += (int64_t)h[2 * f + 1];
        }
    }
    const double pi = 3.14159265358979323846;
    for (int i = 0; i < F->ninst; ++i) {
      if (re) re[i] = sr[i];
      if (im) im[i] = (par[i] & 1) ? pi : 0.0;   // mod(imag, 2*pi) of a multiple of pi
    }
    return FLAM_OK;
  });
}

flam_status flam_rskelf_diag(const flam_factor* F, int dinv, double* D) {
  return guard([&] {
    if (!F || !D) fail(FLAM_ERR_ARG, "FLAM:rskelf_diag:invalidArg: NULL argument");
    if (F->symm == 'h') fail(FLAM_ERR_UNSUPPORTED, "FLAM:gpu:unsupportedSymm: symm 'h' is not built on the device");
    if (F->step_boxes.size() != F->steps.size())
      fail(FLAM_ERR_UNSUPPORTED, "FLAM:rskelf_diag:noTree: the handle has no box structure (imported factors)");
    int64_t nrem = 0;
    for (auto v : F->rem) nrem += v;
    if (nrem > 0) fail(FLAM_ERR_ARG, "FLAM:rskelf_diag:partial: the factorization is partial (opts.stop)");
    const cudaStream_t s = F->s;
    const int64_t N = F->Ntot;
    if (N == 0) return FLAM_OK;
    const bool dev = is_device_ptr(D);
    DBuf<double> xp[2], tmp, Dd;
    DBuf<int64_t> xoff;
    DBuf<int32_t> xpos, xld;
    DBuf<UnfoldTask> tk;
    xoff.resize(N, s);
    xpos.resize(N, s);
    xld.resize(N, s);
    CK(cudaMemsetAsync(xoff.p, 0xff, sizeof(int64_t) * N, s));   // -1: no block yet
    double* Dp = D;
    if (!dev) {
      Dd.resize(N, s);
      Dp = Dd.p;
    }
    CK(cudaMemsetAsync(Dp, 0, sizeof(double) * N, s));
    int cur = 0;
    for (int q = (int)F->steps.size() - 1; q >= 0; --q) {   // top-down
      const auto& br = F->step_boxes[q];
      std::vector<UnfoldTask> ts;
      int64_t xtop = 0, ttop = 0;
      for (const BoxRec& b : br) {
        UnfoldTask u{};
        u.ids_off = b.slf_off;
        u.n = b.n;
        u.k = b.n;
        u.fac_off = 0;
        u.piv_off = 0;
        if (b.fac >= 0) {
          const HostFac& h = F->hfac[b.fac];
          u.k = h.k;
          u.fac_off = h.fac_off;
          u.piv_off = h.piv_off;
        }
        u.xout = xtop;
        u.tmp_off = ttop;
        xtop += (int64_t)b.n * b.n;
        ttop += (int64_t)b.n * (b.n - u.k);
        ts.push_back(u);
      }
      if (ts.empty()) continue;
      xp[cur].ensure(std::max<int64_t>(xtop, 1), s);
      tmp.ensure(std::max<int64_t>(ttop, 1), s);
      tk.upload(ts, s);
      UnfoldArgs a{};
      a.tasks = tk.p;
      a.ipool = F->ipool.p;
      a.fpool = F->fpool.p;
      a.ppool = F->ppool.p;
      a.xprev = xp[cur ^ 1].p ? xp[cur ^ 1].p : xp[cur].p;
      a.xcur = xp[cur].p;
      a.xoff = xoff.p;
      a.xpos = xpos.p;
      a.xld = xld.p;
      a.tmp = tmp.p;
      a.D = Dp;
      a.dinv = dinv ? 1 : 0;
      a.symm = F->symm;
      launch_unfold(a, (int)ts.size(), s);
      CK(cudaGetLastError());
      F->prof.launches += 1;
      cur ^= 1;
    }
    if (!dev) CK(cudaMemcpyAsync(D, Dp, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
    for (auto* b : {&xp[0], &xp[1], &tmp, &Dd}) b->release(s);
    xoff.release(s);
    xpos.release(s);
    xld.release(s);
    tk.release(s);
    CK(cudaStreamSynchronize(s));
    return FLAM_OK;
  });
}

flam_status flam_partial_sizes(const flam_factor* F, int inst, int64_t* Sn, int64_t* nnz) {
  return guard([&] {
    if (!F || inst < 0 || inst >= F->ninst) fail(FLAM_ERR_ARG, "FLAM:rskelf_partial_info:invalidArg: bad instance");
    const bool have = (int)F->Si.size() == F->ninst;
    if (Sn) *Sn = have ? (int64_t)F->Si[inst].size() : 0;
    if (nnz) *nnz = have ? (int64_t)F->Sri[inst].size() : 0;
    return FLAM_OK;
  });
}

flam_status flam_partial_export(const flam_factor* F, int inst, int64_t* Si, int64_t* colptr, int64_t* rowind,
                                double* val) {
  return guard([&] {
    if (!F || inst < 0 || inst >= F->ninst) fail(FLAM_ERR_ARG, "FLAM:rskelf_partial_info:invalidArg: bad instance");
    if ((int)F->Si.size() != F->ninst) {
      if (colptr) colptr[0] = 0;
      return FLAM_OK;
    }
    if (Si) std::copy(F->Si[inst].begin(), F->Si[inst].end(), Si);
    if (colptr) std::copy(F->Scp[inst].begin(), F->Scp[inst].end(), colptr);
    if (rowind) std::copy(F->Sri[inst].begin(), F->Sri[inst].end(), rowind);
    if (val) std::copy(F->Sv[inst].begin(), F->Sv[inst].end(), val);
    return FLAM_OK;
  });
}

flam_status flam_factor_info(const flam_factor* F, flam_info* info) {
  return guard([&] {
    if (!F || !info) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: NULL argument");
    info->N = F->Ntot;
    info->ninst = F->ninst;
    info->d = F->d;
    info->symm = F->symm;
    info->nbox = F->nbox;
    info->nlvl_max = F->nlvl.empty() ? 0 : *std::max_element(F->nlvl.begin(), F->nlvl.end());
    info->nfactor = (int64_t)F->hfac.size();
    info->nstep = (int)F->steps.size();
    int64_t b = F->ipool.bytes() + F->fpool.bytes() + F->ppool.bytes() + F->x.bytes() + F->hperm.bytes();
    for (auto& q : F->steps) b += q.fac.bytes();
    info->bytes = b;
    int64_t r = 0;
    for (auto v : F->rem) r += v;
    info->nrem = r;
    info->t_tree = F->t_tree;
    info->t_factor = F->t_factor;
    return FLAM_OK;
  });
}

flam_status flam_tree_export(const flam_factor* F, int inst, int* nlvl, int64_t* nbox_o, int64_t* nchld_tot,
                             int64_t* nnbor_tot, int64_t* npts_tot, int64_t* lvp, double* l, double* ctr,
                             int64_t* prnt, int64_t* chld_ptr, int64_t* chld, int64_t* nbor_ptr, int64_t* nbor,
                             int64_t* xi_ptr, int64_t* xi) {
  return guard([&] {
    if (!F || inst < 0 || inst >= F->ninst) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: bad instance");
    const int d = F->d;
    std::vector<int64_t> loc(F->nbox, -1), boxes;
    for (int64_t b = 0; b < F->nbox; ++b)
      if (F->binst[b] == inst) {
        loc[b] = (int64_t)boxes.size();
        boxes.push_back(b);
      }
    const int64_t nb = (int64_t)boxes.size();
    int64_t nc = 0, nn = 0, np = 0;
    for (int64_t b : boxes) {
      nc += F->nch[b];
      nn += F->nbor_ptr[b + 1] - F->nbor_ptr[b];
      np += F->nch[b] == 0 ? F->seg_len[b] : 0;
    }
    if (nlvl) *nlvl = F->nlvl[inst];
    if (nbox_o) *nbox_o = nb;
    if (nchld_tot) *nchld_tot = nc;
    if (nnbor_tot) *nnbor_tot = nn;
    if (npts_tot) *npts_tot = np;
    const int L = F->nlvl[inst];
    if (lvp) {
      lvp[0] = 0;
      for (int q = 1; q <= L; ++q) {
        int64_t c = 0;
        for (int64_t b : boxes) c += F->depth[b] <= q;
        lvp[q] = c;
      }
    }
    if (l)
      for (int q = 1; q <= L; ++q)
        for (int64_t b : boxes)
          if (F->depth[b] == q) {
            for (int c = 0; c < d; ++c) l[(q - 1) * d + c] = F->lsz[b * d + c];
            break;
          }
    std::vector<int64_t> ptsv;
    if (xi) {
      std::vector<int64_t> all = download(F->ipool.p, F->Ntot, F->s);
      ptsv.swap(all);
    }
    int64_t oc = 0, on = 0, op = 0;
    for (int64_t q = 0; q < nb; ++q) {
      const int64_t b = boxes[q];
      if (ctr)
        for (int c = 0; c < d; ++c) ctr[q * d + c] = F->ctr[b * d + c];
      if (prnt) prnt[q] = F->prnt[b] < 0 ? -1 : loc[F->prnt[b]];
      if (chld_ptr) chld_ptr[q] = oc;
      for (int32_t c = 0; c < F->nch[b]; ++c) {
        if (chld) chld[oc] = loc[F->chfirst[b] + c];
        ++oc;
      }
      if (nbor_ptr) nbor_ptr[q] = on;
      for (int64_t e = F->nbor_ptr[b]; e < F->nbor_ptr[b + 1]; ++e) {
        if (nbor) nbor[on] = loc[F->nbor[e]];
        ++on;
      }
      if (xi_ptr) xi_ptr[q] = op;
      if (F->nch[b] == 0) {
        for (int64_t e = 0; e < F->seg_len[b]; ++e) {
          if (xi) xi[op] = ptsv[F->seg_start[b] + e] - F->inst_off[inst];
          ++op;
        }
      }
    }
    if (chld_ptr) chld_ptr[nb] = oc;
    if (nbor_ptr) nbor_ptr[nb] = on;
    if (xi_ptr) xi_ptr[nb] = op;
    return FLAM_OK;
  });
}

flam_status flam_tree_perm(const flam_factor* F, int inst, int64_t* P) {
  return guard([&] {
    if (!F || inst < 0 || inst >= F->ninst || !P) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: bad argument");
    const int64_t a = F->inst_off[inst], n = F->inst_off[inst + 1] - a;
    auto v = download(F->hperm.p + a, n, F->s);
    for (int64_t q = 0; q < n; ++q) P[q] = v[q] - a;
    return FLAM_OK;
  });
}

flam_status flam_factor_sizes(const flam_factor* F, int inst, int64_t* nfac, int* nlvp, int64_t* lvp, int64_t* k,
                              int64_t* r) {
  return guard([&] {
    if (!F || inst < 0 || inst >= F->ninst) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: bad instance");
    const auto& fl = F->inst_fac[inst];
    if (nfac) *nfac = (int64_t)fl.size();
    if (nlvp) *nlvp = (int)F->inst_lvp[inst].size();
    if (lvp)
      for (size_t q = 0; q < F->inst_lvp[inst].size(); ++q) lvp[q] = F->inst_lvp[inst][q];
    for (size_t q = 0; q < fl.size(); ++q) {
      if (k) k[q] = F->hfac[fl[q]].k;
      if (r) r[q] = F->hfac[fl[q]].r;
    }
    return FLAM_OK;
  });
}

flam_status flam_factor_export(const flam_factor* F, int inst, int64_t j, int64_t* sk, int64_t* rd, double* T,
                               double* L, double* U, int64_t* p, double* E, double* G) {
  return guard([&] {
    if (!F || inst < 0 || inst >= F->ninst) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: bad instance");
    const auto& fl = F->inst_fac[inst];
    if (j < 0 || j >= (int64_t)fl.size()) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: factor index out of range");
    const HostFac& h = F->hfac[fl[j]];
    const int64_t k = h.k, r = h.r, kr = k * r, rr = r * r;
    const bool chol = F->symm == 'p';
    auto ids = download(F->ipool.p + h.sk_off, k + r, F->s);
    const int64_t a = F->inst_off[inst];
    if (sk)
      for (int64_t q = 0; q < k; ++q) sk[q] = ids[q] - a;
    if (rd)
      for (int64_t q = 0; q < r; ++q) rd[q] = ids[k + q] - a;
    auto fv = download(F->fpool.p + h.fac_off, 2 * kr + rr + (chol ? 0 : kr), F->s);
    if (T) std::copy(fv.begin(), fv.begin() + kr, T);
    const double* LU = fv.data() + kr;
    for (int64_t c = 0; c < r; ++c)
      for (int64_t q = 0; q < r; ++q) {
        const double v = LU[q + c * r];
        if (chol) {
          if (L) L[q + c * r] = q >= c ? v : 0.0;
        } else {
          if (L) L[q + c * r] = q > c ? v : (q == c ? 1.0 : 0.0);
          if (U) U[q + c * r] = q <= c ? v : 0.0;
        }
      }
    if (E) std::copy(fv.begin() + kr + rr, fv.begin() + 2 * kr + rr, E);
    if (!chol) {
      if (G) std::copy(fv.begin() + 2 * kr + rr, fv.begin() + 3 * kr + rr, G);
      if (p) {
        auto pv = download(F->ppool.p + h.piv_off, r, F->s);
        for (int64_t q = 0; q < r; ++q) p[q] = pv[q];
      }
    }
    return FLAM_OK;
  });
}

flam_status flam_factor_import(int64_t N, char symm, int64_t nfac, const int64_t* k, const int64_t* r,
                               const int64_t* sk, const int64_t* rd, const double* T, const double* L,
                               const double* U, const int64_t* p, const double* E, const double* G, void* stream,
                               flam_factor** F) {
  return guard([&] {
    if (!F) fail(FLAM_ERR_ARG, "FLAM:gpu:invalidFactor: output handle pointer is NULL");
    *F = nullptr;
    symm = chksymm(symm);
    if (symm == 'h') fail(FLAM_ERR_UNSUPPORTED, "FLAM:gpu:unsupportedSymm: symm 'h' is not built on the device");
    const bool chol = symm == 'p';
    if (N < 0 || nfac < 0) fail(FLAM_ERR_ARG, "FLAM:gpu:invalidFactor: negative size");
    if (nfac > 0 && (!k || !r || !sk || !rd || !T || !L || !E || (!chol && (!U || !p || !G))))
      fail(FLAM_ERR_ARG, "FLAM:gpu:invalidFactor: a factor array is NULL");
    // host images of the pools; groups of consecutive factors with disjoint index sets
    std::vector<int64_t> ids;
    std::vector<double> fp;
    std::vector<int32_t> pp;
    std::vector<std::vector<FacDesc>> groups(1);
    std::vector<HostFac> hf;
    std::vector<int64_t> gstamp((size_t)N, -1), fstamp((size_t)N, -1);
    int64_t g = 0, ko = 0, ro = 0, kro = 0, rro = 0, ntot_r = 0;
    for (int64_t j = 0; j < nfac; ++j) {
      const int64_t kj = k[j], rj = r[j];
      if (kj < 0 || rj < 0 || kj > N || rj > N) fail(FLAM_ERR_ARG, "FLAM:gpu:invalidFactor: bad factor size");
      bool clash = false;
      for (int64_t q = 0; q < kj + rj; ++q) {
        const int64_t v = q < kj ? sk[ko + q] : rd[ro + q - kj];
        if (v < 0 || v >= N) fail(FLAM_ERR_ARG, "FLAM:gpu:invalidFactor: factor %lld: index outside [0, N)", (long long)j);
        if (fstamp[v] == j) fail(FLAM_ERR_ARG, "FLAM:gpu:invalidFactor: factor %lld: repeated index", (long long)j);
        fstamp[v] = j;
        clash |= gstamp[v] == g;
      }
      if (rj > 0) {
        if (clash) {
          groups.emplace_back();
          ++g;
        }
        for (int64_t q = 0; q < kj + rj; ++q) gstamp[q < kj ? sk[ko + q] : rd[ro + q - kj]] = g;
        const int64_t kr = kj * rj, rr = rj * rj;
        FacDesc f{};
        f.sk_off = (int64_t)ids.size();
        for (int64_t q = 0; q < kj; ++q) ids.push_back(sk[ko + q]);
        for (int64_t q = 0; q < rj; ++q) ids.push_back(rd[ro + q]);
        const int64_t off = (int64_t)fp.size();
        f.T_off = off;
        f.LU_off = off + kr;
        f.E_off = off + kr + rr;
        f.G_off = off + 2 * kr + rr;
        fp.insert(fp.end(), T + kro, T + kro + kr);
        for (int64_t c = 0; c < rj; ++c)       // [L\U] (unit L implicit) or the Cholesky factor
          for (int64_t q = 0; q < rj; ++q)
            fp.push_back(chol ? (q >= c ? L[rro + q + c * rj] : 0.0)
                              : (q > c ? L[rro + q + c * rj] : U[rro + q + c * rj]));
        fp.insert(fp.end(), E + kro, E + kro + kr);
        f.piv_off = (int64_t)pp.size();
        if (!chol) {
          fp.insert(fp.end(), G + kro, G + kro + kr);
          for (int64_t q = 0; q < rj; ++q) {
            if (p[ro + q] < 0 || p[ro + q] >= rj)
              fail(FLAM_ERR_ARG, "FLAM:gpu:invalidFactor: factor %lld: permutation entry outside [0, r)",
                   (long long)j);
            pp.push_back((int32_t)p[ro + q]);
          }
        }
        f.k = (int32_t)kj;
        f.r = (int32_t)rj;
        groups[g].push_back(f);
        hf.push_back(HostFac{0, (int)g, f.sk_off, f.k, f.r, off, f.piv_off});
        ntot_r += rj;
      }
      ko += kj;
      ro += rj;
      kro += kj * rj;
      rro += rj * rj;
    }
    std::unique_ptr<flam_factor> H(new flam_factor());
    CK(cudaGetDevice(&H->dev));
    H->s = (cudaStream_t)stream;
    H->d = 0;
    H->ninst = 1;
    H->inst_off = {0, N};
    H->Ntot = N;
    H->symm = symm;
    H->ipool.upload(ids, H->s);
    H->fpool.upload(fp, H->s);
    H->ppool.upload(pp, H->s);
    H->hfac = hf;
    H->inst_fac.assign(1, {});
    H->inst_lvp.assign(1, {0});
    for (size_t q = 0; q < hf.size(); ++q) H->inst_fac[0].push_back((int64_t)q);
    for (auto& grp : groups) {
      if (grp.empty()) continue;
      StepDev sd;
      sd.set(grp, H->s);
      H->root_rmax = std::max(H->root_rmax, sd.root_rmax());
      H->steps.push_back(std::move(sd));
      H->inst_lvp[0].push_back(H->inst_lvp[0].back() + (int64_t)grp.size());
    }
    H->rem.assign(1, N - ntot_r);
    H->stats.assign(1, {});
    H->nlvl.assign(1, 0);
    CK(cudaStreamSynchronize(H->s));
    *F = H.release();
    return FLAM_OK;
  });
}

flam_status flam_level_stats(const flam_factor* F, int inst, int* nrows, int64_t* rows) {
  return guard([&] {
    if (!F || inst < 0 || inst >= F->ninst) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: bad instance");
    const auto& st = F->stats[inst];
    if (nrows) *nrows = (int)st.size();
    if (rows)
      for (size_t q = 0; q < st.size(); ++q) {
        rows[q * 4 + 0] = st[q].lvl;
        rows[q * 4 + 1] = st[q].nblk;
        rows[q * 4 + 2] = st[q].nrem1;
        rows[q * 4 + 3] = st[q].nrem2;
      }
    return FLAM_OK;
  });
}

void flam_factor_free(flam_factor* F) { delete F; }

void flam_workspace_release(void) {
  std::lock_guard<std::mutex> lk(g_ws_mu);
  int cur = 0;
  cudaGetDevice(&cur);
  for (auto& kv : g_ws) {
    cudaSetDevice(kv.first.first);
    cudaStreamSynchronize(kv.first.second);
    kv.second->release(kv.first.second);
    cudaStreamSynchronize(kv.first.second);
  }
  g_ws.clear();
  cudaSetDevice(cur);
}

flam_status flam_profile(const flam_factor* F, flam_prof* out, int reset) {
  return guard([&] {
    if (!F) fail(FLAM_ERR_ARG, "FLAM:rskelf:invalidArg: NULL factor");
    F->resolve_pending();
    if (out) *out = F->prof;
    if (reset) F->prof = flam_prof{};
    return FLAM_OK;
  });
}

const char* flam_last_error(void) { return g_err.c_str(); }

const char* flam_version(void) { return "flam_b200 0.1 (sm_100a)"; }

}  // extern "C"
