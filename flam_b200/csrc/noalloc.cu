// flam_id_noalloc: the interpolative decomposition of flam_id for callers that
// cannot allocate device memory.
//
// Who needs it: code that runs with a fixed device-memory budget it does not
// own -- e.g. a MEX/oct gateway inside a MATLAB or Octave session whose GPU
// memory manager owns the device heap, or a host thread that must not enter
// the CUDA allocator (cudaMalloc/cudaFree can synchronise the device and can
// fail under someone else's memory pressure).  Such a caller hands in device
// buffers for the matrix and the outputs; every other byte the compress kernel
// needs lives in the file-scope array below.
//
// The array holds kNoAllocBytes on every GPU that loads this library, until
// the process exits.  All calls share it and it keeps the last call's
// contents, so calls whose kernels overlap on the GPU (different streams,
// different host threads, same device) race on it: serialise them.  Each call
// rewrites every part it reads before reading it.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>

#include "../../include/flam.h"
#include "common.cuh"
#include "kernels.cuh"

namespace flam {
namespace {

constexpr int kNoAllocN = FLAM_ID_NOALLOC_NMAX;             // largest n (shared-memory path only)
constexpr size_t kNoAllocBytes = 64 * 1024;

// Layout inside the array (byte offsets, 256-byte aligned sections).
constexpr size_t kOffTask = 0;                                       // CompressTask
constexpr size_t kOffOut = 256;                                      // CompressOut
constexpr size_t kOffInst = 512;                                     // InstParams
constexpr size_t kOffDummy = 768;                                    // 4 doubles (unused point data)
constexpr size_t kOffCand = 1024;                                    // 1 int64 (unused candidate list)
constexpr size_t kOffIds = 1280;                                     // n int64 column ids
constexpr size_t kOffPerm = kOffIds + 8 * kNoAllocN;                 // n int32 permutation
constexpr size_t kOffT = (kOffPerm + 4 * kNoAllocN + 255) / 256 * 256;  // n*n/4+1 doubles
constexpr size_t kEnd = kOffT + 8 * ((size_t)kNoAllocN * kNoAllocN / 4 + 1);
static_assert(kEnd <= kNoAllocBytes, "no-alloc scratch layout exceeds the array");
static_assert(sizeof(CompressTask) <= kOffOut - kOffTask && sizeof(CompressOut) <= kOffInst - kOffOut &&
                  sizeof(InstParams) <= kOffDummy - kOffInst,
              "no-alloc scratch sections too small for their records");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Host-side copy of the array's device address, per device (set up on first use).
std::mutex g_mu;
unsigned char* g_addr[64] = {};

__global__ void k_noalloc_setup(unsigned char* base, CompressTask t, InstParams ip) {
  if (threadIdx.x == 0) {
    *reinterpret_cast<CompressTask*>(base + kOffTask) = t;
    *reinterpret_cast<CompressOut*>(base + kOffOut) = CompressOut{0, 0, 0, 0};
    *reinterpret_cast<InstParams*>(base + kOffInst) = ip;
    double* dm = reinterpret_cast<double*>(base + kOffDummy);
    for (int q = 0; q < 4; ++q) dm[q] = 0.0;
    *reinterpret_cast<int64_t*>(base + kOffCand) = 0;
  }
  int64_t* ids = reinterpret_cast<int64_t*>(base + kOffIds);
  for (int q = threadIdx.x; q < t.n; q += blockDim.x) ids[q] = q;
}

__global__ void k_noalloc_finish(const unsigned char* base, int n, int64_t* k_out, int64_t* perm_out, double* T_out,
                                 int64_t* niter_out) {
  const CompressOut o = *reinterpret_cast<const CompressOut*>(base + kOffOut);
  const int32_t* perm = reinterpret_cast<const int32_t*>(base + kOffPerm);
  const double* T = reinterpret_cast<const double*>(base + kOffT);
  const int k = o.k, r = n - k;
  if (threadIdx.x == 0) {
    *k_out = k;
    if (niter_out) *niter_out = o.niter;
  }
  for (int q = threadIdx.x; q < n; q += blockDim.x) perm_out[q] = perm[q];
  if (k > 0 && r > 0)
    for (int e = threadIdx.x; e < k * r; e += blockDim.x) T_out[e] = T[e];
}

// Device (or managed) memory that kernels launched on device `dev` may read: a
// buffer owned by another GPU is rejected rather than read through a peer mapping.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (at.type == cudaMemoryTypeManaged) return true;
  return at.type == cudaMemoryTypeDevice && at.device == dev;
}

flam_status fail_na(flam_status c, const char* msg) {
  set_last_error(msg);
  return c;
}

}  // namespace
}  // namespace flam

using namespace flam;

extern "C" flam_status flam_id_noalloc(const double* A, int64_t m, int64_t n, int64_t lda, double rank_or_tol,
                                       double Tmax, int64_t rrqr_iter, int64_t* k, int64_t* perm, double* T,
                                       int64_t* niter, void* stream) {
  if (!(rank_or_tol >= 0))
    return fail_na(FLAM_ERR_ARG, "FLAM:id:invalidRankOrTol: Rank or tolerance must be nonnegative.");
  if (!(Tmax >= 1)) return fail_na(FLAM_ERR_ARG, "FLAM:id:invalidTmax: Interpolation matrix entry bound must be >= 1.");
  if (n < 0 || n > kNoAllocN)
    return fail_na(FLAM_ERR_ARG, "FLAM:id:tooLarge: flam_id_noalloc takes 0 <= n <= FLAM_ID_NOALLOC_NMAX (128) "
                                 "columns; use flam_id for larger matrices");
  if (m < 0 || m > ((int64_t)1 << 30) || (m > 0 && lda < m))
    return fail_na(FLAM_ERR_ARG, "FLAM:id:invalidArg: need 0 <= m <= 2^30 and lda >= m");
  if (!k || (n > 0 && (!perm || !T || (m > 0 && !A))))
    return fail_na(FLAM_ERR_ARG, "FLAM:id:invalidArg: NULL pointer");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return fail_na(FLAM_ERR_CUDA, "FLAM:gpu:cuda: cudaGetDevice failed");
  if (!on_device(k, dev) || (niter && !on_device(niter, dev)) ||
      (n > 0 && (!on_device(perm, dev) || !on_device(T, dev) || (m > 0 && !on_device(A, dev)))))
    return fail_na(FLAM_ERR_ARG, "FLAM:id:invalidArg: flam_id_noalloc needs device pointers on the current device "
                                 "for A and every output");
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) {   // no columns: k = 0, nothing to permute (as flam_id)
    if (cudaMemsetAsync(k, 0, sizeof(int64_t), s) != cudaSuccess ||
        (niter && cudaMemsetAsync(niter, 0, sizeof(int64_t), s) != cudaSuccess)) {
      cudaGetLastError();
      return fail_na(FLAM_ERR_CUDA, "FLAM:gpu:cuda: cudaMemsetAsync failed in flam_id_noalloc");
    }
    return FLAM_OK;
  }
  unsigned char* base = nullptr;
  {
    // First call on this device (with it current): look up the array's device
    // address.  In host code the symbol names a host-side stand-in, never the
    // device memory itself.
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return fail_na(FLAM_ERR_CUDA, "FLAM:gpu:cuda: cudaGetSymbolAddress of the no-alloc scratch failed");
      }
      g_addr[dev] = static_cast<unsigned char*>(p);
    }
    base = g_addr[dev];
  }
  CompressTask t{};
  t.slf_off = 0;
  t.cand_off = 0;
  t.T_off = 0;
  t.perm_off = 0;
  t.scr_off = -1;
  t.n = (int32_t)n;
  t.ncand = (int32_t)m;
  t.flags = 0;
  InstParams ip{};
  k_noalloc_setup<<<1, 128, 0, s>>>(base, t, ip);
  CompressArgs ca{};
  ca.P.d = 1;
  ca.P.x = reinterpret_cast<const double*>(base + kOffDummy);
  ca.P.ip = reinterpret_cast<const InstParams*>(base + kOffInst);
  ca.P.pxy_pts = reinterpret_cast<const double*>(base + kOffDummy);
  ca.tasks = reinterpret_cast<const CompressTask*>(base + kOffTask);
  ca.ipool = reinterpret_cast<int64_t*>(base + kOffIds);
  ca.cpool = reinterpret_cast<int64_t*>(base + kOffCand);
  ca.tpool = reinterpret_cast<double*>(base + kOffT);
  ca.permpool = reinterpret_cast<int32_t*>(base + kOffPerm);
  ca.scratch = reinterpret_cast<double*>(base + kOffDummy);
  ca.out = reinterpret_cast<CompressOut*>(base + kOffOut);
  ca.rel_tol = std::fmod(rank_or_tol, 1.0);
  ca.kmax = (int)std::min<double>(std::floor(rank_or_tol), 2e9);
  ca.symm_n = 0;
  ca.Tmax = Tmax;
  ca.rrqr_iter = rrqr_iter;
  ca.Aexp = A;
  ca.lda = m > 0 ? lda : 1;
  launch_compress(ca, 1, compress_smem_bytes((int)n), s);
  k_noalloc_finish<<<1, 256, 0, s>>>(base, (int)n, k, perm, T, niter);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_na(FLAM_ERR_CUDA, "FLAM:gpu:cuda: launch failed in flam_id_noalloc");
  return FLAM_OK;
}
