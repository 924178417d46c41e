// Learned sketch width: a BF16 MLP 16 -> 128 -> 128 -> 1 that predicts a box's ID rank
// as a fraction of its point count, so the sketched compression forms one sketch of
// w = k_pred + p rows per box instead of growing the rank adaptively.  The adaptive
// FP64 ID (core/id.m:106-113) stays the judge: the posterior check of the sketched ID
// sends a box whose rank fills its sketch back to it.
//
// Network: z1 = W1 x + b1, h1 = relu(z1), z2 = W2 h1 + b2, h2 = relu(z2),
// yhat = sigmoid(W3 h2 + b3); loss = mean (yhat - y)^2.  Weights are kept in FP32
// (master copy, Adam moments) and used as BF16; activations are BF16 between the
// layers; every product accumulates in FP32 on the tensor cores (mma.sync m16n8k16
// .bf16 -- the shapes, 64-sample tiles by 128, are far below one tcgen05 tile).
// One CTA (4 warps) owns 64 samples: the forward pass, the loss and the backward pass
// of the tile run in shared memory; weight gradients are summed over the CTAs with
// FP32 atomics, then one Adam step updates the master weights and their BF16 copies.
//
// Features of a box (k_box_features), 16 per box, scale-free:
//   0 log2(1 + n)/10          1 log2(1 + neighbour candidates)/12   2 -log10(tol)/12
//   3-5 l_c / max(l)          6 depth/20                            7-9 std(x_c - ctr_c)/l_c
//   10-12 mean(x_c - ctr_c)/l_c   13 proxy rows present   14 d/3    15 kernel kind/4
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_bf16.h>

#include "../../include/flam.h"
#include "common.cuh"
#include "predictor.cuh"

namespace flam {
namespace {

constexpr int kIn = kPredFeatures, kH = 128;
constexpr int kTile = 64;          // samples per CTA
constexpr int kPThreads = 128;     // 4 warps
// parameter layout (floats): W1 [kH x kIn] | b1 [kH] | W2 [kH x kH] | b2 [kH] | W3 [kH] | b3 [1]
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kIn, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH,
              kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH, kNParam = kOffB3 + 1;
static_assert(kNParam == FLAM_PREDICTOR_NPARAM, "parameter count");

// shared-memory row strides (bf16 elements): +8 keeps the fragment loads off one bank
constexpr int kLdX = kIn + 8, kLdH = kH + 8;

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Warp product over a 16 x 16 A fragment at (row r0, col k0) of a row-major bf16 matrix
// (stride lda) and an 8-wide B fragment whose column j holds row j of Bt (row-major,
// stride ldb), i.e. B = Bt^T.  acc += A(r0:r0+16, k0:k0+16) Bt(n0:n0+8, k0:k0+16)^T.
__device__ __forceinline__ void frag_mma(float (&acc)[4], const __nv_bfloat16* A, int lda, int r0,
                                         const __nv_bfloat16* Bt, int ldb, int n0, int k0) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  uint32_t a[4], b[2];
  const __nv_bfloat16* a0 = A + (r0 + g) * lda + k0 + 2 * t;
  const __nv_bfloat16* a1 = A + (r0 + g + 8) * lda + k0 + 2 * t;
  a[0] = pack2(a0[0], a0[1]);
  a[1] = pack2(a1[0], a1[1]);
  a[2] = pack2(a0[8], a0[9]);
  a[3] = pack2(a1[8], a1[9]);
  const __nv_bfloat16* b0 = Bt + (n0 + g) * ldb + k0 + 2 * t;
  b[0] = pack2(b0[0], b0[1]);
  b[1] = pack2(b0[8], b0[9]);
  mma_bf16(acc, a, b);
}

struct TileSmem {
  __nv_bfloat16 x[kTile * kLdX];      // inputs
  __nv_bfloat16 w1[kH * kLdX];        // W1 (row j: the weights of hidden unit j)
  __nv_bfloat16 w2[kH * kLdH];        // W2
  __nv_bfloat16 w2t[kH * kLdH];       // W2^T (backward)
  __nv_bfloat16 h1[kTile * kLdH];     // relu(z1), later dZ1
  __nv_bfloat16 h2[kTile * kLdH];     // relu(z2)
  __nv_bfloat16 dz2[kTile * kLdH];    // dL/dz2
  __nv_bfloat16 dz2t[kH * (kTile + 8)];   // dZ2^T (weight gradient of layer 2)
  __nv_bfloat16 h1t[kH * (kTile + 8)];    // H1^T
  __nv_bfloat16 dz1t[kH * (kTile + 8)];   // dZ1^T
  __nv_bfloat16 xt[kIn * (kTile + 8)];    // X^T
  float b1[kH], b2[kH], w3[kH];
  float dz3[kTile];
  float yhat[kTile];
  float red[kPThreads / 32];
};

// Forward (and with train, backward) of one 64-sample tile.  grad: FP32 gradient sums;
// loss: sum of squared errors of the tile (atomic).
__global__ void __launch_bounds__(kPThreads) k_mlp(const float* __restrict__ X, const float* __restrict__ y,
                                                   int64_t nsamp, const float* __restrict__ wt, float* yhat_out,
                                                   float* grad, float* loss, float inv_batch, int train) {
  extern __shared__ __align__(16) unsigned char smraw[];
  TileSmem& S = *reinterpret_cast<TileSmem*>(smraw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int64_t s0 = (int64_t)blockIdx.x * kTile;
  const int ns = (int)(nsamp - s0 < kTile ? nsamp - s0 : kTile);
  for (int e = tid; e < kH * kIn; e += kPThreads) S.w1[(e / kIn) * kLdX + e % kIn] = __float2bfloat16(wt[kOffW1 + e]);
  for (int e = tid; e < kH * kH; e += kPThreads) {
    const int i = e / kH, j = e % kH;
    const __nv_bfloat16 v = __float2bfloat16(wt[kOffW2 + e]);
    S.w2[i * kLdH + j] = v;
    S.w2t[j * kLdH + i] = v;
  }
  for (int e = tid; e < kH; e += kPThreads) {
    S.b1[e] = wt[kOffB1 + e];
    S.b2[e] = wt[kOffB2 + e];
    S.w3[e] = wt[kOffW3 + e];
  }
  for (int e = tid; e < kTile * kIn; e += kPThreads) {
    const int s = e / kIn, f = e % kIn;
    const __nv_bfloat16 v = __float2bfloat16(s < ns ? X[(s0 + s) * kIn + f] : 0.f);
    S.x[s * kLdX + f] = v;
    S.xt[f * (kTile + 8) + s] = v;
  }
  __syncthreads();
  // layer 1: warp w owns samples 16w..16w+15, all 128 units (16 n-fragments of 8)
  {
    const int r0 = warp * 16;
    for (int nf = 0; nf < kH / 8; ++nf) {
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      frag_mma(acc, S.x, kLdX, r0, S.w1, kLdX, nf * 8, 0);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = r0 + g + (q >> 1) * 8, col = nf * 8 + 2 * t + (q & 1);
        const float z = acc[q] + S.b1[col];
        S.h1[row * kLdH + col] = __float2bfloat16(z > 0.f ? z : 0.f);
      }
    }
  }
  __syncthreads();
  // layer 2
  {
    const int r0 = warp * 16;
    for (int nf = 0; nf < kH / 8; ++nf) {
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      for (int k0 = 0; k0 < kH; k0 += 16) frag_mma(acc, S.h1, kLdH, r0, S.w2, kLdH, nf * 8, k0);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = r0 + g + (q >> 1) * 8, col = nf * 8 + 2 * t + (q & 1);
        const float z = acc[q] + S.b2[col];
        S.h2[row * kLdH + col] = __float2bfloat16(z > 0.f ? z : 0.f);
      }
    }
  }
  __syncthreads();
  // output unit: one warp per 16 samples, lanes over the 128 inputs
  {
    const float b3 = wt[kOffB3];
    for (int s = warp * 16; s < warp * 16 + 16; ++s) {
      float v = 0.f;
      for (int j = lane; j < kH; j += 32) v += __bfloat162float(S.h2[s * kLdH + j]) * S.w3[j];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) {
        const float yh = 1.f / (1.f + __expf(-(v + b3)));
        S.yhat[s] = yh;
        if (s < ns && yhat_out) yhat_out[s0 + s] = yh;
        float d = 0.f;
        if (train && s < ns) {
          const float e = yh - y[s0 + s];
          atomicAdd(loss, e * e);
          d = 2.f * e * inv_batch * yh * (1.f - yh);
        }
        S.dz3[s] = d;
      }
    }
  }
  if (!train) return;
  __syncthreads();
  // output layer gradients and dZ2 = (dz3 w3^T) .* [z2 > 0]
  for (int j = tid; j < kH; j += kPThreads) {
    float gw = 0.f;
    for (int s = 0; s < kTile; ++s) gw += S.dz3[s] * __bfloat162float(S.h2[s * kLdH + j]);
    atomicAdd(grad + kOffW3 + j, gw);
  }
  if (tid == 0) {
    float gb = 0.f;
    for (int s = 0; s < kTile; ++s) gb += S.dz3[s];
    atomicAdd(grad + kOffB3, gb);
  }
  for (int e = tid; e < kTile * kH; e += kPThreads) {
    const int s = e / kH, j = e % kH;
    const float h = __bfloat162float(S.h2[s * kLdH + j]);
    const __nv_bfloat16 v = __float2bfloat16(h > 0.f ? S.dz3[s] * S.w3[j] : 0.f);
    S.dz2[s * kLdH + j] = v;
    S.dz2t[j * (kTile + 8) + s] = v;
    S.h1t[j * (kTile + 8) + s] = S.h1[s * kLdH + j];
  }
  __syncthreads();
  // dW2 += dZ2^T H1 (128 x 128, k = samples): warp w owns rows 32w..32w+31; db2
  for (int mf = 0; mf < 2; ++mf) {
    const int r0 = warp * 32 + mf * 16;
    for (int nf = 0; nf < kH / 8; ++nf) {
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      for (int k0 = 0; k0 < kTile; k0 += 16) frag_mma(acc, S.dz2t, kTile + 8, r0, S.h1t, kTile + 8, nf * 8, k0);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = r0 + g + (q >> 1) * 8, col = nf * 8 + 2 * t + (q & 1);
        atomicAdd(grad + kOffW2 + row * kH + col, acc[q]);
      }
    }
  }
  for (int j = tid; j < kH; j += kPThreads) {
    float gb = 0.f;
    for (int s = 0; s < kTile; ++s) gb += __bfloat162float(S.dz2[s * kLdH + j]);
    atomicAdd(grad + kOffB2 + j, gb);
  }
  // dZ1 = (dZ2 W2) .* [z1 > 0]  (W2 as B^T: row j of W2^T)
  __syncthreads();
  {
    const int r0 = warp * 16;
    for (int nf = 0; nf < kH / 8; ++nf) {
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      for (int k0 = 0; k0 < kH; k0 += 16) frag_mma(acc, S.dz2, kLdH, r0, S.w2t, kLdH, nf * 8, k0);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = r0 + g + (q >> 1) * 8, col = nf * 8 + 2 * t + (q & 1);
        const float h = __bfloat162float(S.h1[row * kLdH + col]);
        S.dz1t[col * (kTile + 8) + row] = __float2bfloat16(h > 0.f ? acc[q] : 0.f);
      }
    }
  }
  __syncthreads();
  // dW1 += dZ1^T X (128 x 16, k = samples); db1
  for (int mf = 0; mf < 2; ++mf) {
    const int r0 = warp * 32 + mf * 16;
    for (int nf = 0; nf < kIn / 8; ++nf) {
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      for (int k0 = 0; k0 < kTile; k0 += 16) frag_mma(acc, S.dz1t, kTile + 8, r0, S.xt, kTile + 8, nf * 8, k0);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int row = r0 + g + (q >> 1) * 8, col = nf * 8 + 2 * t + (q & 1);
        atomicAdd(grad + kOffW1 + row * kIn + col, acc[q]);
      }
    }
  }
  for (int j = tid; j < kH; j += kPThreads) {
    float gb = 0.f;
    for (int s = 0; s < kTile; ++s) gb += __bfloat162float(S.dz1t[j * (kTile + 8) + s]);
    atomicAdd(grad + kOffB1 + j, gb);
  }
}

// Adam step on the master weights; clears the gradient sums.
__global__ void k_adam(float* w, float* m, float* v, float* grad, float lr, float b1t, float b2t) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kNParam) return;
  const float g = grad[i];
  grad[i] = 0.f;
  const float mi = 0.9f * m[i] + 0.1f * g, vi = 0.999f * v[i] + 0.001f * g * g;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / (1.f - b1t)) / (sqrtf(vi / (1.f - b2t)) + 1e-8f);
}

// Features of each box of a step (one warp per box).
__global__ void k_box_features(const CompressTask* tasks, int ntask, const int64_t* ipool, Problem P, float neg_log_tol,
                               float* out) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= ntask) return;
  const CompressTask t = tasks[w];
  const InstParams ip = P.ip[t.inst];
  const int d = P.d, n = t.n;
  double s1[kMaxDim] = {0, 0, 0}, s2[kMaxDim] = {0, 0, 0};
  for (int q = lane; q < n; q += 32) {
    const int64_t id = ipool[t.slf_off + q];
    for (int c = 0; c < d; ++c) {
      const double z = (P.x[id * d + c] - t.ctr[c]) / (t.l[c] > 0 ? t.l[c] : 1.0);
      s1[c] += z;
      s2[c] += z * z;
    }
  }
  for (int c = 0; c < kMaxDim; ++c) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s1[c] += __shfl_xor_sync(0xffffffffu, s1[c], o);
      s2[c] += __shfl_xor_sync(0xffffffffu, s2[c], o);
    }
  }
  if (lane != 0) return;
  float* f = out + (int64_t)w * kIn;
  double lmax = 0;
  for (int c = 0; c < d; ++c) lmax = fmax(lmax, t.l[c]);
  f[0] = log2f(1.f + n) / 10.f;
  f[1] = log2f(1.f + t.ncand) / 12.f;
  f[2] = neg_log_tol / 12.f;
  for (int c = 0; c < 3; ++c) {
    const bool in = c < d && n > 0;
    const double mu = in ? s1[c] / n : 0.0;
    f[3 + c] = (c < d && lmax > 0) ? (float)(t.l[c] / lmax) : 0.f;
    f[7 + c] = in ? (float)sqrt(fmax(s2[c] / n - mu * mu, 0.0)) : 0.f;
    f[10 + c] = (float)mu;
  }
  f[6] = t.depth / 20.f;
  f[13] = (t.flags & 1) ? 1.f : 0.f;
  f[14] = d / 3.f;
  f[15] = ip.kind / 4.f;
}

}  // namespace

void launch_box_features(const CompressTask* tasks, int ntask, const int64_t* ipool, const Problem& P, float neg_log_tol,
                         float* out, cudaStream_t s) {
  if (ntask <= 0) return;
  k_box_features<<<(ntask * 32 + 255) / 256, 256, 0, s>>>(tasks, ntask, ipool, P, neg_log_tol, out);
}

size_t mlp_smem_bytes() { return sizeof(TileSmem); }

void launch_mlp(const float* X, const float* y, int64_t nsamp, const float* w, float* yhat, float* grad, float* loss,
                float inv_batch, int train, cudaStream_t s) {
  if (nsamp <= 0) return;
  const size_t sm = sizeof(TileSmem);
  if (ensure_smem_attr(reinterpret_cast<const void*>(k_mlp), (int)sm) != cudaSuccess) return;
  k_mlp<<<(unsigned)((nsamp + kTile - 1) / kTile), kPThreads, sm, s>>>(X, y, nsamp, w, yhat, grad, loss, inv_batch,
                                                                       train);
}

void launch_adam(float* w, float* m, float* v, float* grad, float lr, int step, cudaStream_t s) {
  const float b1t = powf(0.9f, (float)step), b2t = powf(0.999f, (float)step);
  k_adam<<<(kNParam + 255) / 256, 256, 0, s>>>(w, m, v, grad, lr, b1t, b2t);
}

}  // namespace flam
