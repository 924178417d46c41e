// Device-wide exclusive prefix sum (three phases: block reduce, scan of the
// block sums, block scan + offset).  Used for every CSR build on the device.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace flam {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// Scratch (in elements of T) needed by exclusive_scan for n items.
inline int64_t scan_scratch_elems(int64_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

// out[i] = sum(in[0..i-1]) for i in [0, n]; out has n+1 entries (out[n] = total).
// `in` and `out` may alias.  `scratch` holds scan_scratch_elems(n) elements.
template <typename T>
void exclusive_scan(const T* in, T* out, int64_t n, T* scratch, cudaStream_t s);

}  // namespace flam
