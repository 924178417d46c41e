// Device-wide exclusive scan (see scan.cuh).
#include "scan.cuh"

namespace flam {
namespace {

template <typename T>
__device__ T block_excl_scan(T v, T* total) {
  __shared__ T wsum[kScanThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  T inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) wsum[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    T w = lane < kScanThreads / 32 ? wsum[lane] : T(0);
    T wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < kScanThreads / 32) wsum[lane] = wi - w;
    if (lane == kScanThreads / 32 - 1) *total = wi;
  }
  __syncthreads();
  T r = wsum[wid] + inc - v;
  __syncthreads();
  return r;
}

template <typename T>
__global__ void k_block_reduce(const T* in, int64_t n, T* sums) {
  __shared__ T tot;
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  T s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j)
    if (base + j < n) s += in[base + j];
  block_excl_scan<T>(s, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template <typename T>
__global__ void k_scan_sums(T* sums, int64_t nb) {
  __shared__ T tot;
  T carry = 0;
  for (int64_t c = 0; c < nb; c += kScanTile) {
    int64_t base = c + (int64_t)threadIdx.x * kScanItems;
    T v[kScanItems];
    T s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
      v[j] = base + j < nb ? sums[base + j] : T(0);
      s += v[j];
    }
    T pre = block_excl_scan<T>(s, &tot) + carry;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
      if (base + j < nb) sums[base + j] = pre;
      pre += v[j];
    }
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[nb] = carry;
}

template <typename T>
__global__ void k_block_scan(const T* in, T* out, int64_t n, const T* sums, int64_t nb) {
  __shared__ T tot;
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  T v[kScanItems];
  T s = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    v[j] = base + j < n ? in[base + j] : T(0);
    s += v[j];
  }
  T pre = block_excl_scan<T>(s, &tot) + sums[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    if (base + j < n) out[base + j] = pre;
    pre += v[j];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = sums[nb];
}

}  // namespace

template <typename T>
void exclusive_scan(const T* in, T* out, int64_t n, T* scratch, cudaStream_t s) {
  int64_t nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 0) {
    cudaMemsetAsync(out, 0, sizeof(T), s);
    return;
  }
  k_block_reduce<T><<<(unsigned)nb, kScanThreads, 0, s>>>(in, n, scratch);
  k_scan_sums<T><<<1, kScanThreads, 0, s>>>(scratch, nb);
  k_block_scan<T><<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, scratch, nb);
}

template void exclusive_scan<int32_t>(const int32_t*, int32_t*, int64_t, int32_t*, cudaStream_t);
template void exclusive_scan<int64_t>(const int64_t*, int64_t*, int64_t, int64_t*, cudaStream_t);

}  // namespace flam
