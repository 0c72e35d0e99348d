// Onesweep stable LSD radix sort (Adinets & Merrill 2022 style) for
// sm_100a.  Each pass is one kernel: a CTA takes the next tile ticket,
// counts its 4096 keys' digits, publishes the counts, resolves its global
// digit offsets by decoupled look-back over the preceding tiles (bounded
// spin), ranks its keys stably with a ballot multisplit, then scatters
// through shared memory so global writes are contiguous within each digit
// run.
#include "sort.cuh"

namespace ygx {

namespace {

__global__ void k_histogram(const uint64_t* __restrict__ keys, int64_t n, int begin_bit,
                            int passes, uint32_t* __restrict__ hist) {
  __shared__ uint32_t s_hist[8 * kSortRadix];
  for (int i = threadIdx.x; i < passes * kSortRadix; i += blockDim.x) s_hist[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    hist_add_key(s_hist, keys[i], begin_bit, passes);
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kSortRadix; i += blockDim.x)
    if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
}

// One CTA per pass: exclusive scan of 256 digit counts, and the pass's
// ranking method (rank_mode[p]): policy 0 = ballots, 1 = peer tables,
// 2 = peer tables unless one digit holds more than skew_q8 / 256 of the keys
// (many lanes of a warp then share a digit and the peer-table atomics
// serialise on it).
__global__ void k_hist_scan(const uint32_t* __restrict__ hist, uint32_t* __restrict__ offsets,
                            uint32_t* __restrict__ rank_mode, int policy, int skew_q8) {
  __shared__ uint32_t s[kSortRadix];
  __shared__ uint32_t s_max;
  const int p = blockIdx.x, t = threadIdx.x;
  uint32_t v = hist[p * kSortRadix + t];
  if (t == 0) s_max = 0;
  __syncthreads();
  atomicMax(&s_max, v);
  s[t] = v;
  __syncthreads();
  for (int off = 1; off < kSortRadix; off <<= 1) {
    uint32_t add = t >= off ? s[t - off] : 0;
    __syncthreads();
    s[t] += add;
    __syncthreads();
  }
  offsets[p * kSortRadix + t] = s[t] - v;
  if (t == kSortRadix - 1) {
    const uint64_t tot = s[t];
    rank_mode[p] = policy == 2 ? ((uint64_t)s_max * 256u <= tot * (uint64_t)skew_q8 ? 1u : 0u)
                               : (uint32_t)policy;
  }
}

constexpr int kPeerWords = (kSortThreads / 32) * 2 * kSortRadix;  // peer tables, in keys[]

template <int kItems>
struct __align__(16) OnesweepSmem {
  static constexpr int kTile = kSortThreads * kItems;
  uint32_t warp_hist[kSortThreads / 32][kSortRadix];
  uint32_t tile_start[kSortRadix];
  uint32_t glob[kSortRadix];
  uint32_t warp_tot[kSortThreads / 32];
  uint32_t ticket;
  alignas(16) uint64_t keys[kTile];  // 16-byte aligned: zeroed with uint4 stores
  uint32_t vals[kTile];
};
static_assert(kPeerWords * sizeof(uint32_t) <= kSortTileMin * sizeof(uint64_t),
              "peer tables fit in the key staging area of the smallest tile");

template <bool kIotaValues, int kItems, int kBlocksPerSM>
__global__ void __launch_bounds__(kSortThreads, kBlocksPerSM)
    k_onesweep(const uint64_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
               int64_t n, int shift, const uint32_t* __restrict__ digit_offsets,
               uint32_t* __restrict__ lookback, uint32_t* __restrict__ ticket_counter,
               uint64_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
               const uint32_t* __restrict__ rank_mode, uint32_t* __restrict__ status,
               uint32_t spin_limit) {
  using Smem = OnesweepSmem<kItems>;
  static_assert(offsetof(Smem, keys) % 16 == 0, "key staging area is 16-byte aligned");
  constexpr int kSortItems = kItems;
  constexpr int kSortTile = Smem::kTile;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const bool peer_tables = *rank_mode != 0;  // uniform over the grid

  for (int i = tid; i < (kSortThreads / 32) * kSortRadix; i += kSortThreads)
    (&sm.warp_hist[0][0])[i] = 0;
  if (peer_tables) {  // two zeroed 256-word tables per warp, in the (idle) key staging area
    uint4* z = reinterpret_cast<uint4*>(sm.keys);
    for (int i = tid; i < kPeerWords / 4; i += kSortThreads) z[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  __shared__ uint32_t s_cnt[kSortRadix];
  if (tid < kSortRadix) s_cnt[tid] = 0;
  if (tid == 0) sm.ticket = atomicAdd(ticket_counter, 1u);
  __syncthreads();
  const uint32_t tile = sm.ticket;
  // n < 2^30 (checked on the host): 32-bit positions throughout
  const uint32_t n32 = (uint32_t)n;
  const uint32_t base = tile * (uint32_t)kSortTile;
  const uint32_t wbase = base + (uint32_t)warp * (kSortItems * 32);
  // The digit of a key: one funnel shift of its two 32-bit halves (or the
  // high half alone for shift >= 32).
  const bool high = shift >= 32;
  const uint32_t sh = (uint32_t)shift & 31u;
  auto digit_of = [&](uint64_t k) -> uint32_t {
    const uint32_t lo = (uint32_t)k, hi = (uint32_t)(k >> 32);
    return (high ? hi >> sh : __funnelshift_r(lo, hi, sh)) & (kSortRadix - 1);
  };

  uint64_t keys[kSortItems];
  uint32_t vals[kSortItems];
  uint16_t rank[kSortItems];
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    const uint32_t idx = wbase + i * 32 + lane;
    keys[i] = idx < n32 ? keys_in[idx] : ~0ull;
  }
  // Early counts: the tile's digit histogram first, so its aggregate is
  // published and its look-back resolved before the (longer) ranking --
  // successors then find an inclusive prefix sooner.
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) atomicAdd(&s_cnt[digit_of(keys[i])], 1u);
  __syncthreads();
  const int d = tid;
  uint32_t total = s_cnt[d];
  uint32_t* my_lb = lookback + (size_t)tile * kSortRadix;
  if (tile == 0) st_volatile_u32(&my_lb[d], kFlagInc | total);
  else st_volatile_u32(&my_lb[d], kFlagAgg | total);
  // Decoupled look-back for digit d, kLookback predecessors per step: their
  // words are read together (independent loads) and resolved in order; only
  // a predecessor that has published nothing yet is waited for (bounded).
  uint32_t excl = 0;
  if (tile > 0) {
    constexpr int kLookback = 8;
    int64_t j = (int64_t)tile - 1;
    bool done = false, timed_out = false;
    while (!done && !timed_out) {
      uint32_t v[kLookback];
#pragma unroll
      for (int k = 0; k < kLookback; ++k)
        v[k] = j - k >= 0 ? ld_volatile_u32(lookback + (size_t)(j - k) * kSortRadix + d)
                          : kFlagInc;  // before tile 0: inclusive zero
#pragma unroll
      for (int k = 0; k < kLookback; ++k) {
        if (done || timed_out) continue;
        uint32_t w = v[k];
        if ((w & ~kCountMask) == 0) {
          const uint32_t* p = lookback + (size_t)(j - k) * kSortRadix + d;
          uint32_t spins = 0;
          while ((w & ~kCountMask) == 0 && spins < spin_limit) {
            __nanosleep(32);
            w = ld_volatile_u32(p);
            ++spins;
          }
          if ((w & ~kCountMask) == 0) {
            timed_out = true;
            continue;
          }
        }
        excl += w & kCountMask;
        if ((w & ~kCountMask) == kFlagInc) done = true;
      }
      j -= kLookback;
    }
    if (timed_out) raise_flag(status, kFlagTimeout);
    st_volatile_u32(&my_lb[d], kFlagInc | ((excl + total) & kCountMask));
  }
  const uint32_t glob_d = digit_offsets[d] + excl;
  // The look-back can leave the warp's lanes diverged (each waited on its
  // own digit); the ranking needs them converged so that the leader lanes'
  // atomics of successive items apply in item order.
  __syncwarp();
  // Stable warp multisplit, kRankGroup items at a time: the peer mask of
  // every item (lanes holding the same digit) from one ballot per digit bit
  // (match-any measured slower here), then one shared-memory atomic per
  // distinct digit (issued back to back; atomics of one warp on one counter
  // apply in program order, so earlier items get lower ranks), then the
  // shuffles.
  const unsigned lt_mask = (1u << lane) - 1u;
  constexpr int kRankGroup = 4;
  if (peer_tables) {
    // Peer-table multisplit: every lane ORs its lane bit into its digit's
    // word of a per-warp table, reads back the word (its peer mask) and the
    // warp's running count of that digit; the highest peer advances the
    // count and clears the word.  Two tables alternate so a clear never
    // races the next item's ORs.  Earlier items, then lower lanes, rank first.
    uint32_t* tb0 = reinterpret_cast<uint32_t*>(sm.keys) + warp * (2 * kSortRadix);
    uint32_t* wh = sm.warp_hist[warp];
#pragma unroll
    for (int i = 0; i < kSortItems; ++i) {
      uint32_t* tb = tb0 + (i & 1) * kSortRadix;
      const uint32_t dg = digit_of(keys[i]);
      atomicOr(&tb[dg], 1u << lane);
      __syncwarp();
      const unsigned pm = tb[dg];
      const uint32_t before = wh[dg];
      __syncwarp();
      rank[i] = (uint16_t)(before + __popc(pm & lt_mask));
      if ((pm >> lane) == 1u) {
        wh[dg] = before + __popc(pm);
        tb[dg] = 0u;
      }
    }
  } else {
#pragma unroll
  for (int g = 0; g < kSortItems; g += kRankGroup) {
    unsigned peers[kRankGroup];
    uint32_t dg[kRankGroup], old[kRankGroup];
#pragma unroll
    for (int u = 0; u < kRankGroup; ++u) {
      dg[u] = digit_of(keys[g + u]);
      unsigned pm = 0xffffffffu;
#pragma unroll
      for (int b = 0; b < kSortRadixBits; ++b) {
        const unsigned bb = __ballot_sync(0xffffffffu, (dg[u] >> b) & 1u);
        pm &= ((dg[u] >> b) & 1u) ? bb : ~bb;
      }
      peers[u] = pm;
    }
#pragma unroll
    for (int u = 0; u < kRankGroup; ++u) {
      old[u] = 0;
      if (lane == __ffs(peers[u]) - 1)
        old[u] = atomicAdd(&sm.warp_hist[warp][dg[u]], (uint32_t)__popc(peers[u]));
    }
#pragma unroll
    for (int u = 0; u < kRankGroup; ++u) {
      const uint32_t o = __shfl_sync(0xffffffffu, old[u], __ffs(peers[u]) - 1);
      rank[g + u] = (uint16_t)(o + __popc(peers[u] & lt_mask));
    }
  }
  }
  // values travel with the keys; loading them here overlaps the look-back
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    const uint32_t idx = wbase + i * 32 + lane;
    vals[i] = kIotaValues ? idx : (idx < n32 ? vals_in[idx] : 0u);
  }
  __syncthreads();

  // Thread t owns digit t: warp-exclusive prefixes and the tile total.
  total = 0;
#pragma unroll
  for (int w = 0; w < kSortThreads / 32; ++w) {
    uint32_t c = sm.warp_hist[w][d];
    sm.warp_hist[w][d] = total;
    total += c;
  }

  // Block exclusive scan of the digit totals -> tile-local digit starts.
  uint32_t incl = total;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += v;
  }
  if (lane == 31) sm.warp_tot[warp] = incl;
  __syncthreads();
  uint32_t wpre = 0;
  for (int w = 0; w < warp; ++w) wpre += sm.warp_tot[w];
  sm.tile_start[d] = wpre + incl - total;
  // global position of tile slot k holding digit dd = glob[dd] + k
  sm.glob[d] = glob_d - (wpre + incl - total);

  __syncthreads();

  // Scatter into shared memory in tile-sorted order.
#pragma unroll
  for (int i = 0; i < kSortItems; ++i) {
    const uint32_t dd = digit_of(keys[i]);
    uint32_t pos = sm.tile_start[dd] + sm.warp_hist[warp][dd] + rank[i];
    sm.keys[pos] = keys[i];
    sm.vals[pos] = vals[i];
  }
  __syncthreads();
  const int nvalid = n32 - base < (uint32_t)kSortTile ? (int)(n32 - base) : kSortTile;
#pragma unroll 4
  for (int k = tid; k < nvalid; k += kSortThreads) {
    const uint64_t key = sm.keys[k];
    const uint32_t g = sm.glob[digit_of(key)] + (uint32_t)k;
    if (g < n32) {
      keys_out[g] = key;
      vals_out[g] = sm.vals[k];
    } else {
      raise_flag(status, kFlagBadInput);  // inconsistent histogram: never write out of range
    }
  }
}

// Arguments of one onesweep pass.
struct OnesweepPass {
  const uint64_t* keys_in;
  const uint32_t* vals_in;  // nullptr: values are the input positions
  int64_t n;
  int shift;
  const uint32_t* offsets;
  uint32_t* lookback;
  uint32_t* counter;
  uint64_t* keys_out;
  uint32_t* vals_out;
  const uint32_t* rank_mode;
  uint32_t* status;
  uint32_t spin_limit;
};

template <int kItems, int kBlocksPerSM>
cudaError_t launch_onesweep(const OnesweepPass& a, unsigned tiles, cudaStream_t st) {
  const size_t smem = sizeof(OnesweepSmem<kItems>);
  static std::atomic<uint64_t> attr_iota{0}, attr_vals{0};
  if (ensure_smem_limit(k_onesweep<true, kItems, kBlocksPerSM>, (int)smem, attr_iota) !=
          cudaSuccess ||
      ensure_smem_limit(k_onesweep<false, kItems, kBlocksPerSM>, (int)smem, attr_vals) !=
          cudaSuccess)
    return cudaErrorInvalidValue;
  if (a.vals_in == nullptr)
    k_onesweep<true, kItems, kBlocksPerSM><<<tiles, kSortThreads, smem, st>>>(
        a.keys_in, nullptr, a.n, a.shift, a.offsets, a.lookback, a.counter, a.keys_out,
        a.vals_out, a.rank_mode, a.status, a.spin_limit);
  else
    k_onesweep<false, kItems, kBlocksPerSM><<<tiles, kSortThreads, smem, st>>>(
        a.keys_in, a.vals_in, a.n, a.shift, a.offsets, a.lookback, a.counter, a.keys_out,
        a.vals_out, a.rank_mode, a.status, a.spin_limit);
  note_launch();
  return cudaGetLastError();
}

}  // namespace

size_t onesweep_scratch_bytes(int64_t n, int max_passes) {
  Arena a{nullptr, 0, 0};
  carve_sort_scratch(a, n, max_passes);
  return a.used + 256;
}

SortScratch carve_sort_scratch(Arena& a, int64_t n, int max_passes) {
  SortScratch s;
  const int64_t tiles = sort_tiles(n, kSortTileMin) > 0 ? sort_tiles(n, kSortTileMin) : 1;
  // hist, lookback and counters are contiguous so one memset clears them.
  s.hist = a.take<uint32_t>((size_t)max_passes * kSortRadix);
  s.lookback = a.take<uint32_t>((size_t)max_passes * tiles * kSortRadix);
  s.counters = a.take<uint32_t>(64);
  s.offsets = a.take<uint32_t>((size_t)max_passes * kSortRadix);
  s.rank_mode = a.take<uint32_t>(64);
  s.keys_tmp = a.take<uint64_t>((size_t)(n > 0 ? n : 1));
  s.vals_tmp = a.take<uint32_t>((size_t)(n > 0 ? n : 1));
  s.wcounters = s.whist = s.woffsets = nullptr;
  s.wlook[0] = s.wlook[1] = nullptr;
  s.wtiles = 0;
  if (max_passes >= 2) {  // a range of 9..11 bits already takes one wide pass instead of two
    s.wtiles = sort_tiles(n, kWideTile) > 0 ? sort_tiles(n, kWideTile) : 1;
    s.wcounters = a.take<uint32_t>(64);
    s.whist = a.take<uint32_t>((size_t)kWideMaxPasses * kWideRadix);
    s.wlook[0] = a.take<uint32_t>((size_t)s.wtiles * kWideRadix);
    s.wlook[1] = a.take<uint32_t>((size_t)s.wtiles * kWideRadix);
    s.woffsets = a.take<uint32_t>((size_t)kWideMaxPasses * kWideRadix);
  }
  return s;
}

bool sort_uses_wide(int begin_bit, int end_bit) {
  return g_tune.sort_bits == kWideBits &&
         sort_passes_wide(begin_bit, end_bit) < sort_passes(begin_bit, end_bit);
}

cudaError_t sort_scratch_reset(const SortScratch& s, int64_t n, int passes, cudaStream_t st) {
  (void)passes;
  size_t bytes = (size_t)((char*)(s.counters + 64) - (char*)s.hist);
  return cudaMemsetAsync(s.hist, 0, bytes, st);
}

int onesweep_sort(const uint64_t* keys_in, const uint32_t* vals_in, int64_t n, int begin_bit,
                  int end_bit, uint64_t* keys_out, uint32_t* vals_out, const SortScratch& s,
                  bool hist_ready, uint32_t* status, cudaStream_t st) {
  if (n <= 0) return YGX_OK;
  if (n >= (int64_t)kCountMask) return YGX_ERR_ARG;
  if (begin_bit < 0 || end_bit > 64 || end_bit <= begin_bit) return YGX_ERR_ARG;
  if (vals_in != nullptr && (const void*)vals_in == (const void*)vals_out) return YGX_ERR_ARG;
  if (s.wlook[0] != nullptr && sort_uses_wide(begin_bit, end_bit))
    return onesweep_sort_wide(keys_in, vals_in, n, begin_bit, end_bit, keys_out, vals_out, s,
                              status, st);
  const int passes = sort_passes(begin_bit, end_bit);
  if (passes > 8) return YGX_ERR_ARG;
  if (!hist_ready) {
    if (sort_scratch_reset(s, n, passes, st) != cudaSuccess) return YGX_ERR_CUDA;
    k_histogram<<<grid_for(n, 256, kNumSMs * 4), 256, 0, st>>>(keys_in, n, begin_bit, passes,
                                                               s.hist);
    YGX_CHECK_LAUNCH();
  }
  k_hist_scan<<<passes, kSortRadix, 0, st>>>(s.hist, s.offsets, s.rank_mode,
                                             g_tune.sort_rank_policy, g_tune.sort_skew_q8);
  YGX_CHECK_LAUNCH();

  const uint64_t* src_k = keys_in;
  const uint32_t* src_v = vals_in;
  const int shape = g_tune.sort_tile;
  const int64_t tiles = sort_tiles(n, kSortThreads * kSortShape[shape].items);
  for (int p = 0; p < passes; ++p) {
    bool to_out = ((passes - 1 - p) % 2) == 0;
    uint64_t* dk = to_out ? keys_out : s.keys_tmp;
    uint32_t* dv = to_out ? vals_out : s.vals_tmp;
    if (p == 0 && (const void*)src_k == (const void*)dk) {
      // Input aliases this pass's destination: stage it in the other buffer.
      uint64_t* stage = to_out ? s.keys_tmp : keys_out;
      if (cudaMemcpyAsync(stage, src_k, sizeof(uint64_t) * n, cudaMemcpyDeviceToDevice, st) !=
          cudaSuccess)
        return YGX_ERR_CUDA;
      src_k = stage;
    }
    OnesweepPass a;
    a.keys_in = src_k;
    a.vals_in = (p == 0 && src_v == nullptr) ? nullptr : src_v;
    a.n = n;
    a.shift = begin_bit + p * kSortRadixBits;
    a.offsets = s.offsets + p * kSortRadix;
    a.lookback = s.lookback + (size_t)p * tiles * kSortRadix;
    a.counter = s.counters + p;
    a.keys_out = dk;
    a.vals_out = dv;
    a.rank_mode = s.rank_mode + p;
    a.status = status;
    a.spin_limit = (uint32_t)g_tune.spin_limit;
    cudaError_t e;
    switch (shape) {
      case 1: e = launch_onesweep<12, 4>(a, (unsigned)tiles, st); break;
      case 2: e = launch_onesweep<20, 2>(a, (unsigned)tiles, st); break;
      case 3: e = launch_onesweep<24, 2>(a, (unsigned)tiles, st); break;
      default: e = launch_onesweep<16, 3>(a, (unsigned)tiles, st); break;
    }
    if (e != cudaSuccess) return YGX_ERR_CUDA;
    src_k = dk;
    src_v = dv;
  }
  return YGX_OK;
}

}  // namespace ygx

extern "C" {

size_t ygx_sort_pairs_workspace_size(int64_t n) {
  return 256 + ygx::onesweep_scratch_bytes(n);
}

int ygx_sort_pairs(const uint64_t* keys_in, const uint32_t* values_in, int64_t n, int begin_bit,
                   int end_bit, uint64_t* keys_out, uint32_t* values_out, void* ws,
                   size_t ws_bytes, cudaStream_t stream) {
  if (n < 0 || (n > 0 && (!keys_in || !keys_out || !values_out || !ws))) return YGX_ERR_ARG;
  if (ws_bytes < ygx_sort_pairs_workspace_size(n)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  uint32_t* status = a.take<uint32_t>(64);
  ygx::SortScratch s = ygx::carve_sort_scratch(a, n);
  return ygx::onesweep_sort(keys_in, values_in, n, begin_bit, end_bit, keys_out, values_out, s,
                            false, status, stream);
}

}  // extern "C"
