// Onesweep pass with 11-bit digits (2048 bins) for sm_100a: the decoupled
// look-back scheme of the 8-bit pass (sort.cu) with six passes over a 63-bit
// key instead of eight (knob YGX_TUNE_SORT_BITS).  Differences that the
// wider digit needs:
//   * thread t owns the eight consecutive digits [8t, 8t + 8): its look-back
//     words move as two 16-byte accesses, and the tile's digit scan is a
//     thread-local scan of eight counts plus a block scan of 256 sums;
//   * the per-warp digit counters are 16-bit halves of shared words, two
//     adjacent digits of one warp per word (a warp ranks at most 32 x 16 =
//     512 keys), so a CTA needs 88 KB of shared memory and two fit on an
//     SM;
//   * the look-back words of a pass are 8 KB per tile, so instead of one
//     zeroed region per pass there are two buffers: pass p reads buffer p & 1
//     and clears its own tile's words of the other buffer for pass p + 1;
//   * the last pass's digit is masked to the bits below end_bit.
// Ranking is the ballot multisplit of the 8-bit pass with up to 11 ballots.
#include "sort.cuh"

namespace ygx {

namespace {

__device__ __forceinline__ uint4 ld_relaxed_v4(const uint32_t* p) {
  uint4 v;
  asm volatile("ld.relaxed.gpu.global.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p)
               : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_v4(uint32_t* p, uint4 v) {
  asm volatile("st.relaxed.gpu.global.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(v.x),
               "r"(v.y), "r"(v.z), "r"(v.w)
               : "memory");
}

constexpr int kWideHistThreads = 1024;

// Digit histograms of every wide pass (shared [passes][2048], then added to
// the global counts).
__global__ void __launch_bounds__(kWideHistThreads)
    k_wide_histogram(const uint64_t* __restrict__ keys, int64_t n, int begin_bit, int end_bit,
                     int passes, uint32_t* __restrict__ hist) {
  extern __shared__ uint32_t s_whist[];
  for (int i = threadIdx.x; i < passes * kWideRadix; i += blockDim.x) s_whist[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    for (int p = 0; p < passes; ++p) {
      const int shift = begin_bit + p * kWideBits;
      const int nb = end_bit - shift < kWideBits ? end_bit - shift : kWideBits;
      atomicAdd(&s_whist[p * kWideRadix + (uint32_t)((k >> shift) & ((1ull << nb) - 1))], 1u);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kWideRadix; i += blockDim.x)
    if (s_whist[i]) atomicAdd(&hist[i], s_whist[i]);
}

// One CTA per pass: exclusive scan of the 2048 digit counts.
__global__ void __launch_bounds__(kSortThreads)
    k_wide_scan(const uint32_t* __restrict__ hist, uint32_t* __restrict__ offsets) {
  __shared__ uint32_t s_warp[kSortThreads / 32];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const uint4* h = reinterpret_cast<const uint4*>(hist + (size_t)blockIdx.x * kWideRadix + 8 * t);
  const uint4 a = h[0], b = h[1];
  const uint32_t c[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  uint32_t ex[8], run = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    ex[k] = run;
    run += c[k];
  }
  uint32_t incl = run;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += v;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  uint32_t base = incl - run;
  for (int w = 0; w < warp; ++w) base += s_warp[w];
  uint4* o = reinterpret_cast<uint4*>(offsets + (size_t)blockIdx.x * kWideRadix + 8 * t);
  o[0] = make_uint4(base + ex[0], base + ex[1], base + ex[2], base + ex[3]);
  o[1] = make_uint4(base + ex[4], base + ex[5], base + ex[6], base + ex[7]);
}

template <int kItems>
struct __align__(16) WideSmem {
  static constexpr int kTile = kSortThreads * kItems;
  uint32_t warp_cnt[kSortThreads / 32][kWideRadix / 2];  // digit d: word d / 2, half d % 2
  uint32_t glob[kWideRadix];  // the tile's digit counts, then each digit's global base
  uint32_t warp_tot[kSortThreads / 32];
  uint32_t ticket;
  alignas(16) uint64_t keys[kTile];
  uint32_t vals[kTile];
};

template <bool kIotaValues, int kItems>
__global__ void __launch_bounds__(kSortThreads, 2)
    k_onesweep_wide(const uint64_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
                    int64_t n, int shift, int nbits, const uint32_t* __restrict__ digit_offsets,
                    uint32_t* __restrict__ lookback, uint32_t* __restrict__ lookback_next,
                    uint32_t* __restrict__ ticket_counter, uint64_t* __restrict__ keys_out,
                    uint32_t* __restrict__ vals_out, uint32_t* __restrict__ status,
                    uint32_t spin_limit) {
  using Smem = WideSmem<kItems>;
  constexpr int kTile = Smem::kTile;
  static_assert(kTile < 65536, "tile offsets fit the 16-bit counter halves");
  static_assert(offsetof(Smem, glob) == sizeof(uint32_t) * (kSortThreads / 32) * (kWideRadix / 2),
                "counters and digit words are one zeroed block");
  static_assert(offsetof(Smem, keys) % 16 == 0, "key staging area is 16-byte aligned");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  {
    constexpr int kZero = ((kSortThreads / 32) * (kWideRadix / 2) + kWideRadix) / 4;
    uint4* z = reinterpret_cast<uint4*>(&sm.warp_cnt[0][0]);
    for (int i = tid; i < kZero; i += kSortThreads) z[i] = make_uint4(0u, 0u, 0u, 0u);
  }
  if (tid == 0) sm.ticket = atomicAdd(ticket_counter, 1u);
  __syncthreads();
  const uint32_t tile = sm.ticket;
  const int d0 = kWideDigitsPerThread * tid;
  if (lookback_next != nullptr) {  // this tile's words of the next pass start at zero
    uint4* nx = reinterpret_cast<uint4*>(lookback_next + (size_t)tile * kWideRadix + d0);
    nx[0] = make_uint4(0u, 0u, 0u, 0u);
    nx[1] = make_uint4(0u, 0u, 0u, 0u);
  }
  // n < 2^30 (checked on the host): 32-bit positions throughout
  const uint32_t n32 = (uint32_t)n;
  const uint32_t base = tile * (uint32_t)kTile;
  const uint32_t wbase = base + (uint32_t)warp * (kItems * 32);
  const bool high = shift >= 32;
  const uint32_t sh = (uint32_t)shift & 31u;
  const uint32_t dmask = (1u << nbits) - 1u;
  auto digit_of = [&](uint64_t k) -> uint32_t {
    const uint32_t lo = (uint32_t)k, hi = (uint32_t)(k >> 32);
    return (high ? hi >> sh : __funnelshift_r(lo, hi, sh)) & dmask;
  };

  uint64_t keys[kItems];
  uint32_t vals[kItems];
  uint16_t rank[kItems];
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const uint32_t idx = wbase + i * 32 + lane;
    keys[i] = idx < n32 ? keys_in[idx] : ~0ull;  // padding: the top digit, ranked last
  }
  // The tile's digit counts first, so its aggregate is published and its
  // look-back resolved before the ranking.
#pragma unroll
  for (int i = 0; i < kItems; ++i) atomicAdd(&sm.glob[digit_of(keys[i])], 1u);
  __syncthreads();
  uint32_t tot[8];
  {
    const uint4 a = *reinterpret_cast<const uint4*>(&sm.glob[d0]);
    const uint4 b = *reinterpret_cast<const uint4*>(&sm.glob[d0 + 4]);
    tot[0] = a.x, tot[1] = a.y, tot[2] = a.z, tot[3] = a.w;
    tot[4] = b.x, tot[5] = b.y, tot[6] = b.z, tot[7] = b.w;
  }
  uint32_t* my_lb = lookback + (size_t)tile * kWideRadix + d0;
  {
    const uint32_t f = tile == 0 ? kFlagInc : kFlagAgg;
    st_relaxed_v4(my_lb, make_uint4(f | tot[0], f | tot[1], f | tot[2], f | tot[3]));
    st_relaxed_v4(my_lb + 4, make_uint4(f | tot[4], f | tot[5], f | tot[6], f | tot[7]));
  }
  // Tile-local start of each digit: exclusive scan of the 2048 counts.
  uint32_t ts[8];
  {
    uint32_t run = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      ts[k] = run;
      run += tot[k];
    }
    uint32_t incl = run;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
      if (lane >= off) incl += v;
    }
    if (lane == 31) sm.warp_tot[warp] = incl;
    __syncthreads();
    uint32_t tb = incl - run;
    for (int w = 0; w < warp; ++w) tb += sm.warp_tot[w];
#pragma unroll
    for (int k = 0; k < 8; ++k) ts[k] += tb;
  }
  // Decoupled look-back for the eight digits together, two predecessors per
  // step (four independent 16-byte loads); a word with nothing published is
  // waited for (bounded), a tile before tile 0 reads as an inclusive zero.
  uint32_t excl[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
  if (tile > 0) {
    uint32_t pend = 0xffu;
    bool timed_out = false;
    int64_t j = (int64_t)tile - 1;
    while (pend != 0u && !timed_out) {
      uint32_t w[2][8];
#pragma unroll
      for (int s = 0; s < 2; ++s) {
        if (j - s >= 0) {
          const uint32_t* q = lookback + (size_t)(j - s) * kWideRadix + d0;
          const uint4 a = ld_relaxed_v4(q), b = ld_relaxed_v4(q + 4);
          w[s][0] = a.x, w[s][1] = a.y, w[s][2] = a.z, w[s][3] = a.w;
          w[s][4] = b.x, w[s][5] = b.y, w[s][6] = b.z, w[s][7] = b.w;
        } else {
#pragma unroll
          for (int k = 0; k < 8; ++k) w[s][k] = kFlagInc;
        }
      }
#pragma unroll
      for (int s = 0; s < 2; ++s) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          if (((pend >> k) & 1u) == 0u || timed_out) continue;
          uint32_t v = w[s][k];
          if ((v & ~kCountMask) == 0u) {  // j - s >= 0 here: padding words carry a flag
            const uint32_t* q = lookback + (size_t)(j - s) * kWideRadix + d0 + k;
            uint32_t spins = 0;
            while ((v & ~kCountMask) == 0u && spins < spin_limit) {
              __nanosleep(32);
              v = ld_volatile_u32(q);
              ++spins;
            }
            if ((v & ~kCountMask) == 0u) {
              timed_out = true;
              continue;
            }
          }
          excl[k] += v & kCountMask;
          if ((v & ~kCountMask) == kFlagInc) pend &= ~(1u << k);
        }
      }
      j -= 2;
    }
    if (timed_out) raise_flag(status, kFlagTimeout);
    st_relaxed_v4(my_lb, make_uint4(kFlagInc | ((excl[0] + tot[0]) & kCountMask),
                                    kFlagInc | ((excl[1] + tot[1]) & kCountMask),
                                    kFlagInc | ((excl[2] + tot[2]) & kCountMask),
                                    kFlagInc | ((excl[3] + tot[3]) & kCountMask)));
    st_relaxed_v4(my_lb + 4, make_uint4(kFlagInc | ((excl[4] + tot[4]) & kCountMask),
                                        kFlagInc | ((excl[5] + tot[5]) & kCountMask),
                                        kFlagInc | ((excl[6] + tot[6]) & kCountMask),
                                        kFlagInc | ((excl[7] + tot[7]) & kCountMask)));
  }
  // Global position of tile slot s holding digit dd = glob[dd] + s.  Each
  // thread reads and writes only its own eight digits' words here.
  {
    const uint4* go = reinterpret_cast<const uint4*>(digit_offsets + d0);
    const uint4 a = __ldg(go), b = __ldg(go + 1);
    uint4* g = reinterpret_cast<uint4*>(&sm.glob[d0]);
    g[0] = make_uint4(a.x + excl[0] - ts[0], a.y + excl[1] - ts[1], a.z + excl[2] - ts[2],
                      a.w + excl[3] - ts[3]);
    g[1] = make_uint4(b.x + excl[4] - ts[4], b.y + excl[5] - ts[5], b.z + excl[6] - ts[6],
                      b.w + excl[7] - ts[7]);
  }
  // The look-back left the warp's lanes diverged (each waited on its own
  // words); the ranking below needs them converged, so that the leader
  // lanes' atomics of successive items apply in item order.  Without this
  // the order of two leaders' atomics on one word was not kept and equal
  // digits of one tile came out swapped.
  __syncwarp();
  // Stable warp multisplit, four items at a time: the peer mask of every
  // item from one ballot per digit bit, one shared atomic per distinct digit
  // on the digit's 16-bit half of this warp's counter word (atomics of one
  // converged warp on one word apply in program order), then the shuffles.
  {
    const unsigned lt_mask = (1u << lane) - 1u;
    uint32_t* wc = sm.warp_cnt[warp];
    constexpr int kRankGroup = 4;
    static_assert(kItems % kRankGroup == 0, "whole rank groups");
#pragma unroll
    for (int g = 0; g < kItems; g += kRankGroup) {
      unsigned peers[kRankGroup];
      uint32_t dg[kRankGroup], old[kRankGroup];
#pragma unroll
      for (int u = 0; u < kRankGroup; ++u) {
        dg[u] = digit_of(keys[g + u]);
        unsigned pm = 0xffffffffu;
#pragma unroll
        for (int b = 0; b < kWideBits; ++b) {
          if (b < nbits) {  // nbits is the same for the whole grid
            const unsigned bb = __ballot_sync(0xffffffffu, (dg[u] >> b) & 1u);
            pm &= ((dg[u] >> b) & 1u) ? bb : ~bb;
          }
        }
        peers[u] = pm;
      }
#pragma unroll
      for (int u = 0; u < kRankGroup; ++u) {
        old[u] = 0;
        if (lane == __ffs(peers[u]) - 1) {
          const uint32_t hs = (dg[u] & 1u) * 16u;
          old[u] = (atomicAdd(&wc[dg[u] >> 1], (uint32_t)__popc(peers[u]) << hs) >> hs) & 0xffffu;
        }
      }
#pragma unroll
      for (int u = 0; u < kRankGroup; ++u) {
        const uint32_t o = __shfl_sync(0xffffffffu, old[u], __ffs(peers[u]) - 1);
        rank[g + u] = (uint16_t)(o + __popc(peers[u] & lt_mask));
      }
    }
  }
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const uint32_t idx = wbase + i * 32 + lane;
    vals[i] = kIotaValues ? idx : (idx < n32 ? vals_in[idx] : 0u);
  }
  __syncthreads();
  // Each warp's start within each digit's tile run: tile start plus the
  // counts of the lower warps, written back into the counter halves.  The
  // thread's eight digits are four words (one uint4) of each warp's row.
  {
    uint32_t run[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) run[k] = ts[k];
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) {
      uint4* cp = reinterpret_cast<uint4*>(&sm.warp_cnt[w][d0 / 2]);
      const uint4 a = *cp;
      const uint32_t c[4] = {a.x, a.y, a.z, a.w};
      uint32_t nw[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint32_t lo = c[q] & 0xffffu, hi = c[q] >> 16;  // digits d0 + 2q, d0 + 2q + 1
        nw[q] = run[2 * q] | (run[2 * q + 1] << 16);
        run[2 * q] += lo;
        run[2 * q + 1] += hi;
      }
      *cp = make_uint4(nw[0], nw[1], nw[2], nw[3]);
    }
  }
  __syncthreads();
  {
    const uint32_t* wc = sm.warp_cnt[warp];
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      const uint32_t dd = digit_of(keys[i]);
      const uint32_t pos = ((wc[dd >> 1] >> ((dd & 1u) * 16u)) & 0xffffu) + rank[i];
      if (pos < (uint32_t)kTile) {
        sm.keys[pos] = keys[i];
        sm.vals[pos] = vals[i];
      } else {
        raise_flag(status, kFlagBadInput);  // inconsistent counts: stay inside the tile
      }
    }
  }
  __syncthreads();
  const int nvalid = n32 - base < (uint32_t)kTile ? (int)(n32 - base) : kTile;
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

template <bool kIota>
cudaError_t launch_wide(const uint64_t* keys_in, const uint32_t* vals_in, int64_t n, int shift,
                        int nbits, const uint32_t* offsets, uint32_t* lookback,
                        uint32_t* lookback_next, uint32_t* counter, uint64_t* keys_out,
                        uint32_t* vals_out, uint32_t* status, unsigned tiles, cudaStream_t st) {
  const size_t smem = sizeof(WideSmem<kWideItems>);
  static std::atomic<uint64_t> attr{0};
  if (ensure_smem_limit(k_onesweep_wide<kIota, kWideItems>, (int)smem, attr) != cudaSuccess)
    return cudaErrorInvalidValue;
  k_onesweep_wide<kIota, kWideItems><<<tiles, kSortThreads, smem, st>>>(
      keys_in, vals_in, n, shift, nbits, offsets, lookback, lookback_next, counter, keys_out,
      vals_out, status, (uint32_t)g_tune.spin_limit);
  note_launch();
  return cudaGetLastError();
}

}  // namespace

int onesweep_sort_wide(const uint64_t* keys_in, const uint32_t* vals_in, int64_t n, int begin_bit,
                       int end_bit, uint64_t* keys_out, uint32_t* vals_out, const SortScratch& s,
                       uint32_t* status, cudaStream_t st) {
  // onesweep_sort checked n, the bit range and the value aliasing
  const int passes = sort_passes_wide(begin_bit, end_bit);
  const int64_t tiles = sort_tiles(n, kWideTile);
  if (passes < 1 || passes > kWideMaxPasses || s.wlook[0] == nullptr || tiles > s.wtiles)
    return YGX_ERR_ARG;
  // tickets, histograms and the first look-back buffer: one memset
  const size_t bytes =
      (size_t)((const char*)(s.wlook[0] + (size_t)tiles * kWideRadix) - (const char*)s.wcounters);
  if (cudaMemsetAsync(s.wcounters, 0, bytes, st) != cudaSuccess) return YGX_ERR_CUDA;
  {
    const size_t hsm = (size_t)passes * kWideRadix * sizeof(uint32_t);
    static std::atomic<uint64_t> attr{0};  // set once per device, for the most passes
    if (ensure_smem_limit(k_wide_histogram, kWideMaxPasses * kWideRadix * (int)sizeof(uint32_t),
                          attr) != cudaSuccess)
      return YGX_ERR_CUDA;
    k_wide_histogram<<<grid_for(n, kWideHistThreads, kNumSMs * 2), kWideHistThreads, hsm, st>>>(
        keys_in, n, begin_bit, end_bit, passes, s.whist);
    YGX_CHECK_LAUNCH();
  }
  k_wide_scan<<<passes, kSortThreads, 0, st>>>(s.whist, s.woffsets);
  YGX_CHECK_LAUNCH();

  const uint64_t* src_k = keys_in;
  const uint32_t* src_v = vals_in;
  for (int p = 0; p < passes; ++p) {
    const bool to_out = ((passes - 1 - p) % 2) == 0;
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
    const int shift = begin_bit + p * kWideBits;
    const int nbits = end_bit - shift < kWideBits ? end_bit - shift : kWideBits;
    uint32_t* next = p + 1 < passes ? s.wlook[(p + 1) & 1] : nullptr;
    const uint32_t* vin = (p == 0 && src_v == nullptr) ? nullptr : src_v;
    cudaError_t e =
        vin == nullptr
            ? launch_wide<true>(src_k, nullptr, n, shift, nbits, s.woffsets + p * kWideRadix,
                                s.wlook[p & 1], next, s.wcounters + p, dk, dv, status,
                                (unsigned)tiles, st)
            : launch_wide<false>(src_k, vin, n, shift, nbits, s.woffsets + p * kWideRadix,
                                 s.wlook[p & 1], next, s.wcounters + p, dk, dv, status,
                                 (unsigned)tiles, st);
    if (e != cudaSuccess) return YGX_ERR_CUDA;
    src_k = dk;
    src_v = dv;
  }
  return YGX_OK;
}

}  // namespace ygx
