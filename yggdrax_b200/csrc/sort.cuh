// Stable LSD radix sort of (uint64 key, uint32 value) pairs: one
// "onesweep" kernel per digit with decoupled look-back -- 8-bit digits
// (sort.cu), or 11-bit digits where the tuning knob asks for them and they
// cut passes (sort_wide.cu).
#pragma once
#include "common.cuh"

namespace ygx {

// Look-back word of one (tile, digit): a 30-bit count and two flag bits --
// the tile's own count (aggregate) or the count of every tile up to and
// including it (inclusive).  Zero means nothing published yet.
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1;

__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_volatile_u32(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

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

// Wide digits (knob YGX_TUNE_SORT_BITS = 11): 2048 bins, thread t of the
// 256 owns digits [8t, 8t + 8).  A 63-bit key takes 6 passes instead of 8.
// A sort runs wide only where that cuts passes (sort_uses_wide).
constexpr int kWideBits = 11;
constexpr int kWideRadix = 1 << kWideBits;
constexpr int kWideDigitsPerThread = kWideRadix / kSortThreads;
constexpr int kWideItems = 16;                           // keys per thread
constexpr int kWideTile = kSortThreads * kWideItems;     // 4096 keys
constexpr int kWideMaxPasses = (64 + kWideBits - 1) / kWideBits;
static_assert(kWideDigitsPerThread == 8, "wide pass: two uint4 of digit words per thread");

inline int sort_passes_wide(int begin_bit, int end_bit) {
  return (end_bit - begin_bit + kWideBits - 1) / kWideBits;
}
// True when the current digit-width knob asks for wide digits and they take
// fewer passes over [begin_bit, end_bit) than 8-bit ones.
bool sort_uses_wide(int begin_bit, int end_bit);

// Scratch needed by onesweep_sort for n keys (per-pass histograms, digit
// offsets, look-back words, tile counters, ping-pong key/value buffers, and
// for max_passes >= 2 the wide pass's histograms and two look-back buffers).
size_t onesweep_scratch_bytes(int64_t n, int max_passes = 8);

struct SortScratch {
  uint32_t* hist;       // [passes][256] digit counts
  uint32_t* offsets;    // [passes][256] exclusive digit offsets
  uint32_t* rank_mode;  // [passes] ranking method of each pass (k_hist_scan)
  uint32_t* lookback;   // [passes][tiles][256]
  uint32_t* counters;   // [passes] tile tickets
  uint64_t* keys_tmp;   // [n]
  uint32_t* vals_tmp;   // [n]
  // wide pass (nullptr when not carved): wcounters, whist and wlook[0] are
  // contiguous so one memset clears them; pass p reads wlook[p & 1] and
  // clears its own tile's words of wlook[(p + 1) & 1] for pass p + 1.
  uint32_t* wcounters;  // [kWideMaxPasses] tile tickets
  uint32_t* whist;      // [kWideMaxPasses][2048]
  uint32_t* wlook[2];   // [wtiles][2048] each
  uint32_t* woffsets;   // [kWideMaxPasses][2048]
  int64_t wtiles;
};
SortScratch carve_sort_scratch(Arena& a, int64_t n, int max_passes = 8);

// The wide-digit sort (sort_wide.cu); same contract as onesweep_sort, which
// calls it.  Computes its own digit histograms.
int onesweep_sort_wide(const uint64_t* keys_in, const uint32_t* vals_in, int64_t n, int begin_bit,
                       int end_bit, uint64_t* keys_out, uint32_t* vals_out, const SortScratch& s,
                       uint32_t* status, cudaStream_t st);

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
