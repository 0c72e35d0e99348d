// Device-wide exclusive scan (reduce-then-scan, three launches, no waits).
#pragma once
#include "common.cuh"

namespace ygx {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

inline int64_t scan_tiles(int64_t n) { return (n + kScanTile - 1) / kScanTile; }
inline size_t scan_scratch_elems(int64_t n) { return (size_t)scan_tiles(n) + 1; }

// out[i] = sum_{k<i} in[i] for i in [0, n]; out[n] is the total (so `out`
// must hold n + 1 elements).  `tmp` holds scan_scratch_elems(n) int64s.
// `in` may be int32 or int64 (InT); the result is int64.
template <typename InT>
int exclusive_scan(const InT* in, int64_t n, int64_t* out, int64_t* tmp, cudaStream_t st);

}  // namespace ygx
