// Randomized row sketch of a box's compression block on the tensor cores:
// Y = Omega K (w x n) for K = [A(nbr,slf); A(slf,nbr)'; Kpxy] (m x n,
// rskelf/rskelf.m:201-212) and a Rademacher Omega (w x m, entries +-1).
//
// The ID of K (core/id.m:102-114) only needs K's column geometry: the pivoted
// QR of Y = Omega K picks skeletons whose interpolation error is within a small
// factor of K's (randomized ID), so the FP64 column-pivoted QR that follows
// folds w ~ k + p rows instead of m.  This kernel is the mixed-precision part:
//   * K is generated in FP32 straight from the points (coordinate differences
//     in FP64, then FP32 kernel evaluation), never written to memory;
//   * K = K_hi + K_lo with K_hi = tf32(K) (round to nearest), so the two
//     products Omega K_hi + Omega K_lo carry ~21 bits of every entry; Omega is
//     exactly representable, so no third product is needed;
//   * the products run as tcgen05.mma kind::tf32 (M = 128 columns of K per
//     tile, N = w padded to 16, 8 rows of K per instruction), accumulated in
//     FP32 in tensor memory, one elected thread issuing, completion signalled
//     through an mbarrier;
//   * the epilogue reads the accumulator with tcgen05.ld and writes Y in FP64
//     for the FP64 pivoted QR, rank decision and R11 \ R12.
// One CTA per box (n <= kSketchMaxN, w <= 256).  Operands live in shared memory
// in the canonical no-swizzle K-major layout: 8 x 16-byte core matrices, core
// matrices of one 16-byte K slice stacked along M (stride 128 B), K slices
// LBO bytes apart.  Every wait on the mbarrier is bounded; on expiry the kernel
// flags FLAM's timeout status, frees its tensor memory and returns.
#include <cstdint>

#include "common.cuh"
#include "sketch.cuh"

namespace flam {
namespace {

constexpr int kKc = 32;               // rows of K per chunk (4 MMA instructions of K = 8)
constexpr int kSkThreads = 256;
constexpr uint64_t kWaitNs = 2000000000ull;   // 2 s bound on any wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t fmix32(uint32_t h) {
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

// Rademacher entry Omega(j, r) of box `box`: +1 or -1.
__device__ __forceinline__ float omega(uint32_t seed, int box, int r, int j) {
  uint32_t h = fmix32(seed ^ (uint32_t)box * 0x9E3779B1u ^ (uint32_t)r * 0x85EBCA77u);
  h = fmix32(h ^ (uint32_t)j * 0xC2B2AE3Du);
  return (h & 1u) ? -1.0f : 1.0f;
}

__device__ __forceinline__ float tf32_rna(float v) {
  uint32_t u;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(v));
  return __uint_as_float(u);
}

// FP32 kernel value for the coordinate difference (dx, dy, dz) (computed in FP64 by the caller).
__device__ __forceinline__ float keval_f32(int kind, float param, float dx, float dy, float dz, float n0, float n1) {
  const float r2 = dx * dx + dy * dy + dz * dz;
  switch (kind) {
    case K_LAPLACE2D:
      return -0.0795774715f * __logf(r2);
    case K_LAPLACE2D_DL:
      return 0.159154943f * (dx * n0 + dy * n1) / r2;
    case K_LAPLACE3D:
      return 0.0795774715f * rsqrtf(r2);
    case K_GAUSSIAN:
      return __expf(-0.5f * param * param * r2);
    default: {
      const float dr = 1.7320508f * param * sqrtf(r2);
      return (1.0f + dr) * __expf(-dr);
    }
  }
}

// Shared-memory matrix descriptor: no swizzle, K-major, LBO between 16-byte K slices,
// SBO between 8-row groups, version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// Bounded wait for phase `parity` of the mbarrier; false on expiry.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
  const uint64_t t0 = globaltimer();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (globaltimer() - t0 > kWaitNs) return false;
  }
}

struct RowDescF {
  int type;          // 0 A(nbr,slf), 1 A(slf,nbr)', 2 proxy, 3 zero
  int64_t q;
  double y[kMaxDim];
  double wmul;
};

__global__ void __launch_bounds__(kSkThreads) k_sketch(SketchArgs a) {
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  __shared__ RowDescF rows[kKc];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int s_fail;

  const SketchTask t = a.tasks[blockIdx.x];
  const Problem& P = a.P;
  const InstParams ip = P.ip[t.inst];
  const int n = t.ncol, w = t.nw, d = P.d;        // this CTA's columns of K and rows of Y
  const int MT = (n + 127) / 128;                  // M tiles of 128 columns of K
  const int NP = (w + 15) / 16 * 16;               // N padded
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // operand tiles: A_hi, A_lo (MT x 128 x 32 fp32 each), B (NP x 32 fp32)
  uint8_t* base = reinterpret_cast<uint8_t*>(((uintptr_t)sm_raw + 1023) & ~(uintptr_t)1023);
  float* Ahi = reinterpret_cast<float*>(base);
  float* Alo = Ahi + MT * 128 * kKc;
  float* Bm = Alo + MT * 128 * kKc;
  uint32_t ncols = 32;
  while ((int)ncols < MT * NP) ncols <<= 1;

  const int m1 = a.mfilt[t.out_idx];
  const int nrep = a.symm_n ? 2 : 1;
  const int npr = (t.flags & 1) ? (ip.two_sided ? 2 * P.npxy : P.npxy) : 0;
  const int m = nrep * m1 + npr;
  if (tid == 0) {
    a.mrows[t.out_idx] = m;
    s_fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t barp = smem_u32(&bar);

  // this thread's column of K (fixed over the chunks) and its row quads
  const int cpass = MT * 128;
  const int c = tid % cpass;
  const int rq0 = tid / cpass, rqs = kSkThreads / cpass;
  const int64_t sc = c < n ? a.ipool[t.slf_off + t.col0 + c] : -1;
  double xc[kMaxDim] = {0.0, 0.0, 0.0};
  float nc[2] = {0.f, 0.f};
  double wc = 1.0;
  if (sc >= 0) {
    for (int k = 0; k < d; ++k) xc[k] = P.x[sc * d + k];
    if (ip.has_nrm) {
      nc[0] = (float)P.nrm[sc * d];
      nc[1] = (float)P.nrm[sc * d + 1];
    }
    if (ip.has_w) wc = P.w[sc];
  }
  const int64_t* cand = a.cpool + t.cand_off;
  // instruction descriptor: FP32 accumulate, TF32 A and B, both K-major, M = 128; N = 256 for
  // the first 256 rows of Y, the rest in a second product
  const int N0 = NP > 256 ? 256 : NP, N1 = NP - N0;
  const uint32_t idesc0 = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N0 >> 3) << 17) | ((128u >> 4) << 24);
  const uint32_t idesc1 = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N1 >> 3) << 17) | ((128u >> 4) << 24);
  const uint32_t lboA = 16 * 128, lboB = (uint32_t)(NP / 8) * 128;
  uint32_t phase = 0;
  bool issued = false;

  for (int r0 = 0; r0 < m; r0 += kKc) {
    if (issued) {   // the previous chunk's products have read the operand tiles
      if (!bar_wait(barp, phase)) s_fail = 1;
      phase ^= 1;
    }
    __syncthreads();
    if (s_fail) break;
    if (tid < kKc) {
      const int rho = r0 + tid;
      RowDescF rd;
      rd.type = 3;
      rd.q = -1;
      rd.wmul = 0.0;
      rd.y[0] = rd.y[1] = rd.y[2] = 0.0;
      if (rho < m1) {
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
      rows[tid] = rd;
    }
    __syncthreads();
    // A = K^T: column c of K is row c of the operand; 4 consecutive rows of K per 16-byte store
    const int mt = c >> 7, cr = c & 127;
    for (int rq = rq0; rq < kKc / 4; rq += rqs) {
      float hi[4], lo[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const RowDescF& rd = rows[rq * 4 + i];
        float e = 0.f;
        if (sc >= 0 && rd.type != 3) {
          if (rd.type == 2) {
            const double* y = rd.y;
            const float kv = keval_f32(ip.pkernel, (float)ip.pparam, (float)(y[0] - xc[0]),
                                       d > 1 ? (float)(y[1] - xc[1]) : 0.f, d > 2 ? (float)(y[2] - xc[2]) : 0.f,
                                       0.f, 0.f);
            e = (float)ip.pscale * kv * (float)(rd.wmul != 0.0 ? rd.wmul : (ip.has_w ? wc : 1.0));
          } else {
            const int64_t q = rd.q;
            const double* xq = P.x + q * d;
            if (q == sc) {
              e = (float)ip.dval;
            } else if (rd.type == 0) {   // A(q, sc): target q, source sc
              const float kv = keval_f32(ip.kind, (float)ip.param, (float)(xq[0] - xc[0]),
                                         d > 1 ? (float)(xq[1] - xc[1]) : 0.f, d > 2 ? (float)(xq[2] - xc[2]) : 0.f,
                                         nc[0], nc[1]);
              e = (float)(ip.scale * wc) * kv;
            } else {                     // A(sc, q): target sc, source q
              float n0 = 0.f, n1 = 0.f;
              if (ip.has_nrm) {
                n0 = (float)P.nrm[q * d];
                n1 = (float)P.nrm[q * d + 1];
              }
              const float kv = keval_f32(ip.kind, (float)ip.param, (float)(xc[0] - xq[0]),
                                         d > 1 ? (float)(xc[1] - xq[1]) : 0.f, d > 2 ? (float)(xc[2] - xq[2]) : 0.f,
                                         n0, n1);
              e = (float)(ip.scale * (ip.has_w ? P.w[q] : 1.0)) * kv;
            }
          }
        }

        hi[i] = tf32_rna(e);
        lo[i] = e - hi[i];
      }
      const int off = mt * 128 * kKc + (rq * 16 + (cr >> 3)) * 32 + (cr & 7) * 4;
      *reinterpret_cast<float4*>(Ahi + off) = make_float4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<float4*>(Alo + off) = make_float4(lo[0], lo[1], lo[2], lo[3]);

    }
    // B = Omega^T (NP x 32): row j of the operand is sketch row j
    for (int it = tid; it < NP * (kKc / 4); it += kSkThreads) {
      const int j = it % NP, rq = it / NP;
      float o[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int rho = r0 + rq * 4 + i;
        o[i] = (j < w && rho < m) ? omega(a.seed, t.box, rho, t.j0 + j) : 0.f;
      }
      const int off = (rq * (NP / 8) + (j >> 3)) * 32 + (j & 7) * 4;
      *reinterpret_cast<float4*>(Bm + off) = make_float4(o[0], o[1], o[2], o[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int tm = 0; tm < MT; ++tm) {
        const uint32_t ahi = smem_u32(Ahi + tm * 128 * kKc), alo = smem_u32(Alo + tm * 128 * kKc);
        const uint32_t bb = smem_u32(Bm);
        for (int s = 0; s < kKc / 8; ++s) {
          // K slices 2s, 2s+1 (8 rows of K) of every operand
          const uint64_t ah = smem_desc(ahi + (uint32_t)(2 * s) * lboA, lboA, 128);
          const uint64_t al = smem_desc(alo + (uint32_t)(2 * s) * lboA, lboA, 128);
          const uint32_t acc = (r0 > 0 || s > 0) ? 1u : 0u;
          const uint64_t bd0 = smem_desc(bb + (uint32_t)(2 * s) * lboB, lboB, 128);
          mma_tf32(tmem + (uint32_t)(tm * NP), ah, bd0, idesc0, acc);
          mma_tf32(tmem + (uint32_t)(tm * NP), al, bd0, idesc0, 1u);
          if (N1 > 0) {   // rows 256.. of the B operand: 32 core matrices further on
            const uint64_t bd1 = smem_desc(bb + (uint32_t)(2 * s) * lboB + 32 * 128, lboB, 128);
            mma_tf32(tmem + (uint32_t)(tm * NP + 256), ah, bd1, idesc1, acc);
            mma_tf32(tmem + (uint32_t)(tm * NP + 256), al, bd1, idesc1, 1u);
          }
        }
      }
      mma_commit(barp);
    }
    issued = true;
    __syncwarp();
  }
  if (issued && !s_fail) {
    if (!bar_wait(barp, phase)) s_fail = 1;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  double* Y = a.ypool + t.y_off;
  if (s_fail) {
    if (tid == 0) atomicOr(a.status, (int)ST_TIMEOUT);
    if (issued && warp == 0 && lane == 0) bar_wait(barp, phase);   // let the products in flight drain (bounded)
  } else if (!issued) {
    for (int e = tid; e < w * n; e += kSkThreads) Y[(t.j0 + e % w) + (int64_t)(t.col0 + e / w) * t.w] = 0.0;
  } else {
    // warp: lanes 32 (warp % 4) .. +31 of the accumulator (columns of K), one half of its columns
    const int lq = warp & 3, half = warp >> 2;
    const int j0 = half * (NP / 2), j1 = j0 + NP / 2;
    for (int tm = 0; tm < MT; ++tm) {
      const int cc = tm * 128 + lq * 32 + lane;
      for (int jb = j0; jb < j1; jb += 8) {
        uint32_t r[8];
        const uint32_t addr = tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)(tm * NP + jb);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
            : "r"(addr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (cc < n)
#pragma unroll
          for (int q = 0; q < 8; ++q)
            if (jb + q < w) Y[(t.j0 + jb + q) + (int64_t)(t.col0 + cc) * t.w] = (double)__uint_as_float(r[q]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// FP64 form of the sketch (opts.sketch = 2): the same Y = Omega K, with K's entries
// evaluated in FP64 exactly as the exact compression generates them (block_entry) and the
// products on the FP64 tensor path (mma.sync m8n8k4 .f64), accumulated in FP64.  The
// sketch then carries full precision, so the randomized ID meets tight tolerances directly
// (no refinement needed).  One CTA forms a tile of at most kSketchF64Rows rows of Y by
// kSketchF64Cols columns of K; chunks of kFk rows of K are staged through shared memory
// (K transposed, Omega row-major; stride kFld = 20 doubles keeps the fragment loads at two
// wavefronts), eight warps each own a 32 x 32 block of the tile.
constexpr int kFk = 16;
constexpr int kFld = kFk + 4;

__device__ __forceinline__ void dmma_f64(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(kSkThreads) k_sketch_f64(SketchArgs a) {
  __shared__ double Ks[kSketchF64Cols * kFld];
  __shared__ double Os[kSketchF64Rows * kFld];
  __shared__ RowDescF rows[kFk];
  const SketchTask t = a.tasks[blockIdx.x];
  const Problem& P = a.P;
  const InstParams ip = P.ip[t.inst];
  const int n = t.ncol, w = t.nw, d = P.d;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int wj = warp >> 2, wc = warp & 3;
  const int m1 = a.mfilt[t.out_idx];
  const int nrep = a.symm_n ? 2 : 1;
  const int npr = (t.flags & 1) ? (ip.two_sided ? 2 * P.npxy : P.npxy) : 0;
  const int m = nrep * m1 + npr;
  if (tid == 0) a.mrows[t.out_idx] = m;
  const int64_t* cand = a.cpool + t.cand_off;
  // entries (rho, columns cg * cpt .. + cpt - 1) of each chunk for this thread: a tile of
  // at most half the columns spreads them over every thread (cpt = 4), not half of them
  constexpr int kCpt = kSketchF64Cols / (kSkThreads / kFk);
  const int cpt = n <= kSketchF64Cols / 2 ? kCpt / 2 : kCpt;
  const int rho_t = tid & (kFk - 1), cg = tid / kFk;
  int64_t scol[kCpt];
#pragma unroll
  for (int i = 0; i < kCpt; ++i) {
    const int c = cg * cpt + i;
    scol[i] = (i < cpt && c < n) ? a.ipool[t.slf_off + t.col0 + c] : -1;
  }
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  for (int r0 = 0; r0 < m; r0 += kFk) {
    if (tid < kFk) {
      const int rho = r0 + tid;
      RowDescF rd;
      rd.type = 3;
      rd.q = -1;
      rd.wmul = 0.0;
      rd.y[0] = rd.y[1] = rd.y[2] = 0.0;
      if (rho < m1) {
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
      rows[tid] = rd;
    }
    __syncthreads();   // rows ready; the previous chunk's products are done with Ks / Os
    {
      const RowDescF& rd = rows[rho_t];
#pragma unroll
      for (int i = 0; i < kCpt; ++i) {
        if (i < cpt)
          Ks[(cg * cpt + i) * kFld + rho_t] =
              scol[i] >= 0 && rd.type != 3 ? block_entry(P, ip, rd.type, rd.q, rd.y, rd.wmul, scol[i]) : 0.0;
      }
    }
    for (int e = tid; e < kSketchF64Rows * kFk; e += kSkThreads) {
      const int j = e / kFk, rr = e % kFk, rho = r0 + rr;
      Os[j * kFld + rr] = (j < w && rho < m) ? (double)omega(a.seed, t.box, rho, t.j0 + j) : 0.0;
    }
    __syncthreads();
    // warps whose 32 x 32 block lies beyond the tile's rows or columns have no products
    // (with cpt = 4, Ks holds only columns below 64)
    if (wj * 32 < w && wc * 32 < n) {
      const double* Aw = Os + (wj * 32 + g) * kFld + tq;
      const double* Bw = Ks + (wc * 32 + g) * kFld + tq;
#pragma unroll
      for (int kk = 0; kk < kFk; kk += 4) {
        double af[4], bf[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) af[i] = Aw[i * 8 * kFld + kk];
#pragma unroll
        for (int j = 0; j < 4; ++j) bf[j] = Bw[j * 8 * kFld + kk];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma_f64(acc[i][j], af[i], bf[j]);
      }
    }
    __syncthreads();
  }
  double* Y = a.ypool + t.y_off;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int j = wj * 32 + i * 8 + g;
    if (j >= w) continue;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int c = wc * 32 + jj * 8 + 2 * tq + e;
        if (c < n) Y[(t.j0 + j) + (int64_t)(t.col0 + c) * t.w] = acc[i][jj][e];
      }
  }
}

// Restore the pull-up order of the slf lists of boxes whose sketch was rejected, so the
// exact compression that redoes them starts from the order the elimination expects.
__global__ void k_unpermute(const int32_t* idx, const SketchTask* tasks, int64_t* ipool, const int32_t* permpool) {
  extern __shared__ int64_t ids[];
  const SketchTask t = tasks[idx[blockIdx.x]];
  int64_t* slf = ipool + t.slf_off;
  const int32_t* perm = permpool + t.perm_off;
  for (int q = threadIdx.x; q < t.n; q += blockDim.x) ids[q] = slf[q];
  __syncthreads();
  for (int q = threadIdx.x; q < t.n; q += blockDim.x) slf[perm[q]] = ids[q];
}

}  // namespace

size_t sketch_smem_bytes(int ncol, int nw) {
  const int MT = (ncol + 127) / 128, NP = (nw + 15) / 16 * 16;
  return 1024 + sizeof(float) * (size_t)(2 * MT * 128 * kKc + NP * kKc);
}

void launch_sketch(const SketchArgs& a, int ntask, size_t smem, cudaStream_t s) {
  if (ntask <= 0) return;
  if (a.fp64) {
    k_sketch_f64<<<ntask, kSkThreads, 0, s>>>(a);
    return;
  }
  if (ensure_smem_attr(reinterpret_cast<const void*>(k_sketch), (int)smem) != cudaSuccess) return;
  k_sketch<<<ntask, kSkThreads, smem, s>>>(a);
}

void launch_unpermute(const int32_t* idx, int nidx, const SketchTask* tasks, int64_t* ipool, const int32_t* permpool,
                      int nmax, cudaStream_t s) {
  if (nidx <= 0) return;
  k_unpermute<<<nidx, 256, sizeof(int64_t) * (size_t)nmax, s>>>(idx, tasks, ipool, permpool);
}

}  // namespace flam
