// Stable LSD radix sort of (uint64 key, uint32 value) pairs: one
// "onesweep" kernel per 8-bit digit with decoupled look-back.
#pragma once
#include "common.cuh"

namespace ygx {

constexpr int kSortRadixBits = 8;
constexpr int kSortRadix = 1 << kSortRadixBits;
constexpr int kSortThreads = 256;
static_assert(kSortThreads == kSortRadix, "onesweep: thread t owns digit t");

// Tile shapes of the onesweep kernel (knob YGX_TUNE_SORT_TILE): keys per
// thread and CTAs resident per SM.  Shape 0 is the default.  The look-back
// scratch is sized for the smallest tile, so every shape fits the same
// workspace.
struct SortTileShape {
  int items;          // keys per thread; tile = 256 * items keys
  int blocks_per_sm;  // launch bound: CTAs resident per SM
};
constexpr int kSortTileShapes = 4;
constexpr SortTileShape kSortShape[kSortTileShapes] = {{16, 3}, {12, 4}, {20, 2}, {24, 2}};
constexpr int kSortTileMin = kSortThreads * 12;  // 3072 keys: the smallest tile

inline int sort_passes(int begin_bit, int end_bit) {
  return (end_bit - begin_bit + kSortRadixBits - 1) / kSortRadixBits;
}
inline int64_t sort_tiles(int64_t n, int tile) { return (n + tile - 1) / tile; }

// Scratch needed by onesweep_sort for n keys (per-pass histograms, digit
// offsets, look-back words, tile counters, ping-pong key/value buffers).
size_t onesweep_scratch_bytes(int64_t n, int max_passes = 8);

struct SortScratch {
  uint32_t* hist;       // [passes][256] digit counts
  uint32_t* offsets;    // [passes][256] exclusive digit offsets
  uint32_t* rank_mode;  // [passes] ranking method of each pass (k_hist_scan)
  uint32_t* lookback;   // [passes][tiles][256]
  uint32_t* counters;   // [passes] tile tickets
  uint64_t* keys_tmp;   // [n]
  uint32_t* vals_tmp;   // [n]
};
SortScratch carve_sort_scratch(Arena& a, int64_t n, int max_passes = 8);

// Zeroes the histogram, look-back words and tile counters (one memset).
cudaError_t sort_scratch_reset(const SortScratch& s, int64_t n, int passes, cudaStream_t st);

// Sorts keys_in[0..n) by bits [begin_bit, end_bit), carrying values
// (vals_in == nullptr means value = input position).  Results land in
// keys_out / vals_out; keys_in may alias keys_out.  If hist_ready, the
// per-pass histograms in scratch.hist were filled by the caller (e.g. fused
// into the Morton encode) and only the offsets scan runs.
int onesweep_sort(const uint64_t* keys_in, const uint32_t* vals_in, int64_t n, int begin_bit,
                  int end_bit, uint64_t* keys_out, uint32_t* vals_out, const SortScratch& s,
                  bool hist_ready, uint32_t* status, cudaStream_t st);

// Per-block digit-histogram accumulation helper for fused producers: adds
// the digits of `key` for `passes` passes starting at begin_bit into a
// shared [passes][256] histogram.
__device__ __forceinline__ void hist_add_key(uint32_t* s_hist, uint64_t key, int begin_bit,
                                             int passes) {
  for (int p = 0; p < passes; ++p) {
    uint32_t d = (uint32_t)(key >> (begin_bit + p * kSortRadixBits)) & (kSortRadix - 1);
    atomicAdd(&s_hist[p * kSortRadix + d], 1u);
  }
}

}  // namespace ygx
