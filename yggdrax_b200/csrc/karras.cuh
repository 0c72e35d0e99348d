// Karras (2012) radix-tree construction over sorted leaf codes, shared by
// the single-tree and the batched (forest) builds.
// _tree_impl.py:1115-1270.
#pragma once
#include "common.cuh"

namespace ygx {

__device__ __forceinline__ int64_t kdelta(const uint64_t* __restrict__ c, int64_t L, int64_t i,
                                          int64_t j, uint64_t ci) {
  if (j < 0 || j >= L) return -1;
  uint64_t cj = c[j];
  if (ci == cj) return 64 + clz64((uint64_t)i ^ (uint64_t)j);
  return clz64(ci ^ cj);
}
__device__ __forceinline__ int64_t lcp_codes(uint64_t a, uint64_t b) {
  return a == b ? 64 : clz64(a ^ b);
}

// Internal node i of a Karras topology over L leaf codes: direction, span,
// range, split, children.  Outputs are written through the given bases (all
// indexed by the local i / local node id); children and parent claims hold
// local node ids (leaf j = L - 1 + j); left32 / right32 get node_base + the
// local child id.
__device__ __forceinline__ void karras_node(const uint64_t* __restrict__ codes,
                                            const void* starts, const void* ends, int64_t L,
                                            int64_t i, int index_bits, void* left, void* right,
                                            uint8_t* __restrict__ lil, uint8_t* __restrict__ ril,
                                            void* ranges, int32_t* __restrict__ left32,
                                            int32_t* __restrict__ right32,
                                            int32_t* __restrict__ parent_claim,
                                            int64_t node_base) {
  const int64_t ni = L - 1;
    const uint64_t ci = codes[i];
    int64_t dp = kdelta(codes, L, i, i + 1, ci);
    int64_t dm = kdelta(codes, L, i, i - 1, ci);
    int64_t d = (dp - dm) > 0 ? 1 : ((dp - dm) < 0 ? -1 : 0);
    if (i == 0 || d == 0) d = 1;
    const int64_t dmin = kdelta(codes, L, i, i - d, ci);
    int64_t span = 0;
    for (int k = 30; k >= 0; --k) {
      int64_t step = (int64_t)1 << k;
      int64_t cand = i + (span + step) * d;
      if (cand >= 0 && cand < L && kdelta(codes, L, i, cand, ci) > dmin) span += step;
    }
    const int64_t end = i + span * d;
    const int64_t first = i < end ? i : end, last = i < end ? end : i;
    store_idx(ranges, index_bits, 2 * i, load_idx(starts, index_bits, first));
    store_idx(ranges, index_bits, 2 * i + 1, load_idx(ends, index_bits, last) - 1);
    const uint64_t fc = codes[first];
    const int64_t cp = lcp_codes(fc, codes[last]);
    int64_t split = first;
    for (int k = 30; k >= 0; --k) {
      int64_t mid = split + ((int64_t)1 << k);
      if (mid < last && lcp_codes(fc, codes[mid]) > cp) split = mid;
    }
    const bool ll = split == first, rl = split + 1 == last;
    const int64_t lc = ll ? ni + first : split;
    const int64_t rc = rl ? ni + last : split + 1;
    lil[i] = ll;
    ril[i] = rl;
    store_idx(left, index_bits, i, lc);
    store_idx(right, index_bits, i, rc);
    left32[i] = (int32_t)(node_base + lc);
    right32[i] = (int32_t)(node_base + rc);
    // Serial-scatter semantics of parent.at[left].set / .at[right].set:
    // any right claim beats every left claim, larger index wins within a side.
    atomicMax(&parent_claim[lc], (int32_t)i);
    atomicMax(&parent_claim[rc], (int32_t)(i + ni));
}

}  // namespace ygx
