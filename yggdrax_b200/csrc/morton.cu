// Bounding box + 63-bit Morton encode + stable sort (L0 of the pipeline).
//
// Replaces infer_bounds (bounds.py:11-33), morton_encode_impl
// (morton.py:43-77) and the stable argsort of the codes
// (_tree_impl.py:401, tree.py:403).
//
// k_bbox_encode (one cooperative launch) reduces the per-axis min / max, pads
// the bounds in its last-arriving CTA, and encodes every point with them,
// building the per-pass digit histograms of the following radix sort so the
// sort never re-reads the keys for them; each thread keeps its first chunks
// in registers across the wait and re-reads the rest in L2-friendly order.
// k_bbox + k_encode are the two-launch form (used for caller-supplied bounds
// and where a cooperative launch is unavailable).
#include "morton.cuh"
#include "sort.cuh"

namespace ygx {
namespace {

constexpr int kBBoxThreads = 256;
constexpr int kBBoxBlocks = kNumSMs * 4;
constexpr int kFusedMaxBlocks = kNumSMs * 8;  // the fused kernel's grid at most

struct Box {
  float mn[3], mx[3];
  unsigned nan;
  __device__ void init() {
    for (int a = 0; a < 3; ++a) { mn[a] = __int_as_float(0x7f800000); mx[a] = -__int_as_float(0x7f800000); }
    nan = 0;
  }
  __device__ __forceinline__ void add(int a, float v) {
    if (v != v) nan |= 1u << a;
    mn[a] = fminf(mn[a], v);
    mx[a] = fmaxf(mx[a], v);
  }
  __device__ void merge(const Box& o) {
    for (int a = 0; a < 3; ++a) { mn[a] = fminf(mn[a], o.mn[a]); mx[a] = fmaxf(mx[a], o.mx[a]); }
    nan |= o.nan;
  }
  __device__ void warp_reduce() {
    for (int off = 16; off > 0; off >>= 1) {
      for (int a = 0; a < 3; ++a) {
        mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
        mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
      }
      nan |= __shfl_xor_sync(0xffffffffu, nan, off);
    }
  }
};

// Four particles = twelve floats = three 16-byte words.
__device__ __forceinline__ void load_chunk(const float* __restrict__ pos, int64_t c, bool vec,
                                           float f[12]) {
  if (vec) {
    const float4* p4 = reinterpret_cast<const float4*>(pos) + 3 * c;
    float4 a = __ldg(p4), b = __ldg(p4 + 1), d = __ldg(p4 + 2);
    f[0] = a.x; f[1] = a.y; f[2] = a.z; f[3] = a.w;
    f[4] = b.x; f[5] = b.y; f[6] = b.z; f[7] = b.w;
    f[8] = d.x; f[9] = d.y; f[10] = d.z; f[11] = d.w;
  } else {
#pragma unroll
    for (int k = 0; k < 12; ++k) f[k] = __ldg(pos + 12 * c + k);
  }
}

__global__ void __launch_bounds__(kBBoxThreads)
    k_bbox(const float* __restrict__ pos, int64_t n, float* __restrict__ partials,
           unsigned* __restrict__ arrivals, float* __restrict__ bounds_out) {
  __shared__ Box s_box[kBBoxThreads / 32];
  __shared__ bool s_last;
  Box b;
  b.init();
  const bool vec = (reinterpret_cast<uintptr_t>(pos) & 15) == 0;
  const int64_t chunks = n / 4;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < chunks;
       c += (int64_t)gridDim.x * blockDim.x) {
    float f[12];
    load_chunk(pos, c, vec, f);
#pragma unroll
    for (int k = 0; k < 12; ++k) b.add(k % 3, f[k]);
  }
  if (blockIdx.x == 0)
    for (int64_t i = chunks * 4 + threadIdx.x; i < n; i += blockDim.x)
      for (int a = 0; a < 3; ++a) b.add(a, pos[3 * i + a]);
  b.warp_reduce();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_box[warp] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    Box t = s_box[0];
    for (int w = 1; w < kBBoxThreads / 32; ++w) t.merge(s_box[w]);
    float* out = partials + 8 * blockIdx.x;
    for (int a = 0; a < 3; ++a) { out[a] = t.mn[a]; out[3 + a] = t.mx[a]; }
    out[6] = __uint_as_float(t.nan);
    __threadfence();
    unsigned ticket = atomicAdd(arrivals, 1u);
    s_last = ticket == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  // Last CTA to arrive: reduce the per-CTA partials.
  __threadfence();
  Box t;
  t.init();
  for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
    const volatile float* p = partials + 8 * k;
    Box o;
    for (int a = 0; a < 3; ++a) { o.mn[a] = p[a]; o.mx[a] = p[3 + a]; }
    o.nan = __float_as_uint(p[6]);
    t.merge(o);
  }
  t.warp_reduce();
  if (lane == 0) s_box[warp] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    Box r = s_box[0];
    for (int w = 1; w < kBBoxThreads / 32; ++w) r.merge(s_box[w]);
    const float qnan = __int_as_float(0x7fc00000);
    for (int a = 0; a < 3; ++a) {
      float lo = (r.nan >> a) & 1 ? qnan : r.mn[a];
      float hi = (r.nan >> a) & 1 ? qnan : r.mx[a];
      // bounds.py:29-33: span * 0.05 (fp32), floor 1e-6, min - pad, max + pad
      float span = __fsub_rn(hi, lo);
      float pad = fmax_nan(__fmul_rn(span, 0.05f), 1e-6f);
      bounds_out[a] = __fsub_rn(lo, pad);
      bounds_out[3 + a] = __fadd_rn(hi, pad);
    }
    *arrivals = 0;  // ready for the next call
  }
}

constexpr int kEncodeThreads = 256;

__global__ void __launch_bounds__(kEncodeThreads)
    k_encode(const float* __restrict__ pos, int64_t n, const float* __restrict__ bounds,
             uint64_t* __restrict__ codes, uint32_t* __restrict__ hist, int hist_passes) {
  __shared__ uint32_t s_hist[8 * kSortRadix];
  for (int i = threadIdx.x; i < hist_passes * kSortRadix; i += blockDim.x) s_hist[i] = 0;
  __syncthreads();
  float mn[3], span[3];
  for (int a = 0; a < 3; ++a) {
    mn[a] = bounds[a];
    span[a] = __fsub_rn(bounds[3 + a], bounds[a]);
  }
  const bool vec = (reinterpret_cast<uintptr_t>(pos) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(codes) & 15) == 0;
  const int64_t chunks = (n + 3) / 4;
  const int64_t full = n / 4;
  const int lane = threadIdx.x & 31;
  // Every lane of a warp runs the same number of iterations so the
  // warp-aggregated histogram updates below see a full warp.
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t start = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31);
  for (int64_t cw = start; cw < chunks; cw += stride) {
    const int64_t c = cw + lane;
    uint64_t code[4];
    int valid = 0;
    if (c < full) {
      float f[12];
      load_chunk(pos, c, vec, f);
#pragma unroll
      for (int k = 0; k < 4; ++k) code[k] = encode_one(f[3 * k], f[3 * k + 1], f[3 * k + 2], mn, span);
      valid = 4;
      if (vec) {
        ulonglong2* o = reinterpret_cast<ulonglong2*>(codes + 4 * c);
        o[0] = make_ulonglong2(code[0], code[1]);
        o[1] = make_ulonglong2(code[2], code[3]);
      } else {
        for (int k = 0; k < 4; ++k) codes[4 * c + k] = code[k];
      }
    } else if (c < chunks) {
      for (int64_t i = 4 * c; i < n; ++i, ++valid) {
        code[valid] = encode_one(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], mn, span);
        codes[i] = code[valid];
      }
    }
    if (hist_passes > 0) {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        for (int p = 0; p < hist_passes; ++p) {
          uint32_t d = k < valid ? (uint32_t)(code[k] >> (p * kSortRadixBits)) & (kSortRadix - 1)
                                 : 0xFFFFu;
          // One atomic for the warp when all its digits agree (the high
          // digits of clustered inputs), else one per lane: cheaper than a
          // match-any, which runs on a slow pipe here.
          const unsigned vm = __ballot_sync(0xffffffffu, d != 0xFFFFu);
          const uint32_t dl = __shfl_sync(0xffffffffu, d, vm ? __ffs(vm) - 1 : 0);
          if (__all_sync(0xffffffffu, d == dl || d == 0xFFFFu)) {
            if (lane == 0 && vm) atomicAdd(&s_hist[p * kSortRadix + dl], (uint32_t)__popc(vm));
          } else if (d != 0xFFFFu) {
            atomicAdd(&s_hist[p * kSortRadix + d], 1u);
          }
        }
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < hist_passes * kSortRadix; i += blockDim.x)
    if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
}

// Digit histograms of the following sort for the (up to) four codes of one
// lane; every lane of the warp calls it together.
__device__ __forceinline__ void hist_codes(uint32_t* s_hist, const uint64_t* code, int valid,
                                           int passes, int lane) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    for (int p = 0; p < passes; ++p) {
      const uint32_t d = k < valid ? (uint32_t)(code[k] >> (p * kSortRadixBits)) & (kSortRadix - 1)
                                   : 0xFFFFu;
      const unsigned vm = __ballot_sync(0xffffffffu, d != 0xFFFFu);
      const uint32_t dl = __shfl_sync(0xffffffffu, d, vm ? __ffs(vm) - 1 : 0);
      if (__all_sync(0xffffffffu, d == dl || d == 0xFFFFu)) {
        if (lane == 0 && vm) atomicAdd(&s_hist[p * kSortRadix + dl], (uint32_t)__popc(vm));
      } else if (d != 0xFFFFu) {
        atomicAdd(&s_hist[p * kSortRadix + d], 1u);
      }
    }
  }
}

// Loads chunk c (four particles) into f; returns the number of particles in it.
__device__ __forceinline__ int load_any_chunk(const float* __restrict__ pos, int64_t n, int64_t c,
                                              bool vec, float f[12]) {
  if (4 * c + 4 <= n) {
    load_chunk(pos, c, vec, f);
    return 4;
  }
  int v = 0;
  for (int k = 0; k < 4; ++k) {
    const int64_t i = 4 * c + k;
    if (i < n) {
      f[3 * k] = pos[3 * i];
      f[3 * k + 1] = pos[3 * i + 1];
      f[3 * k + 2] = pos[3 * i + 2];
      ++v;
    } else {
      f[3 * k] = f[3 * k + 1] = f[3 * k + 2] = 0.0f;
    }
  }
  return v;
}

// Fused infer_bounds + morton_encode_impl + sort histograms, one cooperative
// launch (every CTA resident).  Phase 1 reduces the per-axis min / max; each
// thread walks its chunks from the last to the first and keeps its first two
// in registers.  The last CTA to arrive pads the bounds (bounds.py:29-33) and
// publishes them; the others wait for that flag (bounded spin; on give-up the
// status word gets YGX_FLAG_TIMEOUT and the CTA stops).  Phase 2 encodes the
// two kept chunks without reading them again, then the rest first to last --
// the order in which phase 1 read them last, so the re-reads are mostly
// served from L2.
__global__ void __launch_bounds__(kEncodeThreads, 3)
    k_bbox_encode(const float* __restrict__ pos, int64_t n, float* __restrict__ partials,
                  unsigned* __restrict__ arrivals, float* __restrict__ bounds_out,
                  uint64_t* __restrict__ codes, uint32_t* __restrict__ hist, int passes,
                  uint32_t spin_limit, uint32_t* __restrict__ status) {
  __shared__ uint32_t s_hist[8 * kSortRadix];
  __shared__ Box s_box[kEncodeThreads / 32];
  __shared__ int s_last, s_ok;
  for (int i = threadIdx.x; i < passes * kSortRadix; i += blockDim.x) s_hist[i] = 0;
  const bool vec = (reinterpret_cast<uintptr_t>(pos) & 15) == 0 &&
                   (reinterpret_cast<uintptr_t>(codes) & 15) == 0;
  const int64_t chunks = (n + 3) / 4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // the same iteration count for every lane of a warp (histogram ballots)
  const int64_t gw = g - lane;
  const int64_t K = gw < chunks ? (chunks - gw + stride - 1) / stride : 0;
  Box b;
  b.init();
  float keep0[12], keep1[12];
  int v0 = 0, v1 = 0;
  for (int64_t k = K - 1; k >= 0; --k) {
    const int64_t c = g + k * stride;
    float f[12];
    int v = 0;
    if (c < chunks) {
      v = load_any_chunk(pos, n, c, vec, f);
#pragma unroll
      for (int j = 0; j < 12; ++j)
        if (j / 3 < v) b.add(j % 3, f[j]);
    } else {
#pragma unroll
      for (int j = 0; j < 12; ++j) f[j] = 0.0f;
    }
    if (k == 0) {
#pragma unroll
      for (int j = 0; j < 12; ++j) keep0[j] = f[j];
      v0 = v;
    } else if (k == 1) {
#pragma unroll
      for (int j = 0; j < 12; ++j) keep1[j] = f[j];
      v1 = v;
    }
  }
  b.warp_reduce();
  if (lane == 0) s_box[warp] = b;
  __syncthreads();
  if (threadIdx.x == 0) {
    Box t = s_box[0];
    for (int w = 1; w < kEncodeThreads / 32; ++w) t.merge(s_box[w]);
    float* out = partials + 8 * blockIdx.x;
    for (int a = 0; a < 3; ++a) { out[a] = t.mn[a]; out[3 + a] = t.mx[a]; }
    out[6] = __uint_as_float(t.nan);
    __threadfence();
    s_last = atomicAdd(&arrivals[0], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    Box t;
    t.init();
    for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
      const volatile float* q = partials + 8 * k;
      Box o;
      for (int a = 0; a < 3; ++a) { o.mn[a] = q[a]; o.mx[a] = q[3 + a]; }
      o.nan = __float_as_uint(q[6]);
      t.merge(o);
    }
    t.warp_reduce();
    if (lane == 0) s_box[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
      Box r = s_box[0];
      for (int w = 1; w < kEncodeThreads / 32; ++w) r.merge(s_box[w]);
      const float qnan = __int_as_float(0x7fc00000);
      for (int a = 0; a < 3; ++a) {
        const float lo = (r.nan >> a) & 1 ? qnan : r.mn[a];
        const float hi = (r.nan >> a) & 1 ? qnan : r.mx[a];
        const float span = __fsub_rn(hi, lo);
        const float pad = fmax_nan(__fmul_rn(span, 0.05f), 1e-6f);
        bounds_out[a] = __fsub_rn(lo, pad);
        bounds_out[3 + a] = __fadd_rn(hi, pad);
      }
      __threadfence();
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(arrivals + 1), "r"(1u) : "memory");
    }
  }
  if (threadIdx.x == 0) {
    unsigned ready = 0, spins = 0;
    while (true) {
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(ready) : "l"(arrivals + 1) : "memory");
      if (ready || spins >= spin_limit) break;
      __nanosleep(64);
      ++spins;
    }
    s_ok = ready != 0;
    if (!ready) raise_flag(status, kFlagTimeout);
  }
  __syncthreads();
  if (!s_ok) return;
  float mn[3], span[3];
  for (int a = 0; a < 3; ++a) {
    mn[a] = bounds_out[a];
    span[a] = __fsub_rn(bounds_out[3 + a], bounds_out[a]);
  }
  for (int64_t k = 0; k < K; ++k) {
    const int64_t c = g + k * stride;
    float f[12];
    int v;
    if (k == 0) {
#pragma unroll
      for (int j = 0; j < 12; ++j) f[j] = keep0[j];
      v = v0;
    } else if (k == 1) {
#pragma unroll
      for (int j = 0; j < 12; ++j) f[j] = keep1[j];
      v = v1;
    } else {
      v = c < chunks ? load_any_chunk(pos, n, c, vec, f) : 0;
    }
    uint64_t code[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) code[q] = encode_one(f[3 * q], f[3 * q + 1], f[3 * q + 2], mn, span);
    if (v == 4 && vec) {
      ulonglong2* o = reinterpret_cast<ulonglong2*>(codes + 4 * c);
      o[0] = make_ulonglong2(code[0], code[1]);
      o[1] = make_ulonglong2(code[2], code[3]);
    } else {
      for (int q = 0; q < v; ++q) codes[4 * c + q] = code[q];
    }
    if (passes > 0) hist_codes(s_hist, code, v, passes, lane);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kSortRadix; i += blockDim.x)
    if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
}

// ---- batched sets (segments [off[s], off[s+1]) of one position array) ---------

// Bounds of every set: one CTA per set, the same reduction and padding as
// k_bbox (bounds.py:29-33), and the set id of every point.
__global__ void __launch_bounds__(kBBoxThreads)
    k_seg_bbox(const float* __restrict__ pos, const int64_t* __restrict__ off, int64_t S,
               float* __restrict__ bounds_out, int32_t* __restrict__ seg_of) {
  __shared__ Box s_box[kBBoxThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t sg = blockIdx.x; sg < S; sg += gridDim.x) {
    const int64_t b = off[sg], e = off[sg + 1];
    Box bx;
    bx.init();
    for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) {
      for (int a = 0; a < 3; ++a) bx.add(a, pos[3 * i + a]);
      seg_of[i] = (int32_t)sg;
    }
    bx.warp_reduce();
    if (lane == 0) s_box[warp] = bx;
    __syncthreads();
    if (threadIdx.x == 0) {
      Box r = s_box[0];
      for (int w = 1; w < kBBoxThreads / 32; ++w) r.merge(s_box[w]);
      const float qnan = __int_as_float(0x7fc00000);
      for (int a = 0; a < 3; ++a) {
        float lo = (r.nan >> a) & 1 ? qnan : r.mn[a];
        float hi = (r.nan >> a) & 1 ? qnan : r.mx[a];
        float span = __fsub_rn(hi, lo);
        float pad = fmax_nan(__fmul_rn(span, 0.05f), 1e-6f);
        bounds_out[6 * sg + a] = __fsub_rn(lo, pad);
        bounds_out[6 * sg + 3 + a] = __fadd_rn(hi, pad);
      }
    }
    __syncthreads();
  }
}

// Codes of every point with its set's bounds, plus the digit histograms of
// the 8 code passes of the sort.
__global__ void __launch_bounds__(kEncodeThreads)
    k_seg_encode(const float* __restrict__ pos, int64_t n, const int32_t* __restrict__ seg_of,
                 const float* __restrict__ bounds, uint64_t* __restrict__ codes,
                 uint32_t* __restrict__ hist) {
  __shared__ uint32_t s_hist[8 * kSortRadix];
  for (int i = threadIdx.x; i < 8 * kSortRadix; i += blockDim.x) s_hist[i] = 0;
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float* bd = bounds + 6 * seg_of[i];
    float mn[3], span[3];
    for (int a = 0; a < 3; ++a) {
      mn[a] = bd[a];
      span[a] = __fsub_rn(bd[3 + a], bd[a]);
    }
    const uint64_t c = encode_one(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], mn, span);
    codes[i] = c;
    for (int p = 0; p < 8; ++p)
      atomicAdd(&s_hist[p * kSortRadix + ((uint32_t)(c >> (p * kSortRadixBits)) & (kSortRadix - 1))],
                1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 8 * kSortRadix; i += blockDim.x)
    if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
}

__global__ void k_u64_to_i32(const uint64_t* __restrict__ in, int64_t n, int32_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int32_t)in[i];
}

// Sort keys of the second (stable, by set) sort: the set of each point in
// the code order.
__global__ void k_seg_keys(const uint32_t* __restrict__ perm, const int32_t* __restrict__ seg_of,
                           int64_t n, uint64_t* __restrict__ keys) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    keys[i] = (uint64_t)(uint32_t)seg_of[perm[i]];
}

__global__ void k_gather_codes(const uint64_t* __restrict__ codes, const uint32_t* __restrict__ perm,
                               int64_t n, uint64_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = codes[perm[i]];
}

}  // namespace

// Grid of the fused kernel: every CTA must be resident at once (cooperative
// launch), at most kFusedMaxBlocks; 0 when the device cannot say.
static int fused_grid() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
  static std::atomic<int> cache[64];
  int g = cache[dev].load(std::memory_order_relaxed);
  if (g != 0) return g > 0 ? g : 0;
  int per_sm = 0, sms = 0, coop = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bbox_encode, kEncodeThreads, 0) !=
          cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess) {
    (void)cudaGetLastError();
    g = -1;
  } else {
    g = coop ? per_sm * sms : -1;
    if (g > kFusedMaxBlocks) g = kFusedMaxBlocks;
    if (g <= 0) g = -1;
  }
  cache[dev].store(g, std::memory_order_relaxed);
  return g > 0 ? g : 0;
}

struct EncodeSortLayout {
  uint32_t* status;
  float* partials;
  unsigned* arrivals;
  SortScratch sort;
};

static EncodeSortLayout carve_encode_sort(Arena& a, int64_t n) {
  EncodeSortLayout l;
  l.status = a.take<uint32_t>(64);
  l.partials = a.take<float>(8 * kFusedMaxBlocks);
  l.arrivals = a.take<unsigned>(64);
  l.sort = carve_sort_scratch(a, n);
  return l;
}

struct BatchEncodeLayout {
  uint32_t* status;
  int32_t* seg_of;
  uint64_t* codes;
  uint32_t* perm_code;
  uint64_t* seg_keys;
  uint64_t* seg_sorted;
  SortScratch sort;
};

static BatchEncodeLayout carve_batch_encode(Arena& a, int64_t n) {
  BatchEncodeLayout l;
  const int64_t m = n > 0 ? n : 1;
  l.status = a.take<uint32_t>(64);
  l.seg_of = a.take<int32_t>(m);
  l.codes = a.take<uint64_t>(m);
  l.perm_code = a.take<uint32_t>(m);
  l.seg_keys = a.take<uint64_t>(m);
  l.seg_sorted = a.take<uint64_t>(m);
  l.sort = carve_sort_scratch(a, n);
  return l;
}

}  // namespace ygx

extern "C" {

size_t ygx_batch_encode_sort_workspace_size(int64_t n) {
  ygx::Arena a{nullptr, 0, 0};
  ygx::carve_batch_encode(a, n);
  return a.used + 256;
}

// Batched bounds + Morton codes + stable order of S point sets stored back to
// back (set s = positions[offsets[s] .. offsets[s+1]), offsets on the
// device): per set what infer_bounds / morton_encode_impl / the stable
// argsort of _tree_impl.py:401 give for that set alone.  bounds_out (S x 6:
// min xyz, max xyz), codes_sorted (n) in (set, code, original index) order,
// order_out (n) the global input index of each sorted point, seg_sorted_out
// (n, int32, may be null) its set.
int ygx_batch_encode_sort(const float* positions, int64_t n, const int64_t* offsets, int64_t S,
                          float* bounds_out, uint64_t* codes_sorted, uint32_t* order_out,
                          int32_t* seg_sorted_out, void* ws, size_t ws_bytes,
                          cudaStream_t stream) {
  if (n < 1 || S < 1 || S > (int64_t)1 << 16 || n >= (int64_t)UINT32_MAX || !positions ||
      !offsets || !bounds_out || !codes_sorted || !order_out || !ws)
    return YGX_ERR_ARG;
  if (ws_bytes < ygx_batch_encode_sort_workspace_size(n)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::BatchEncodeLayout l = ygx::carve_batch_encode(a, n);
  if (cudaMemsetAsync(l.status, 0, 64 * sizeof(uint32_t), stream) != cudaSuccess ||
      ygx::sort_scratch_reset(l.sort, n, 8, stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  ygx::k_seg_bbox<<<(unsigned)(S < 65535 ? S : 65535), ygx::kBBoxThreads, 0, stream>>>(
      positions, offsets, S, bounds_out, l.seg_of);
  YGX_CHECK_LAUNCH();
  ygx::k_seg_encode<<<ygx::grid_for(n, ygx::kEncodeThreads), ygx::kEncodeThreads, 0, stream>>>(
      positions, n, l.seg_of, bounds_out, l.codes, l.sort.hist);
  YGX_CHECK_LAUNCH();
  // stable by code (63 bits), then stable by set (16 bits): (set, code, index)
  int rc = ygx::onesweep_sort(l.codes, nullptr, n, 0, 63, codes_sorted, l.perm_code, l.sort, true,
                              l.status, stream);
  if (rc) return rc;
  ygx::k_seg_keys<<<ygx::grid_for(n, 256), 256, 0, stream>>>(l.perm_code, l.seg_of, n,
                                                             l.seg_keys);
  YGX_CHECK_LAUNCH();
  rc = ygx::onesweep_sort(l.seg_keys, l.perm_code, n, 0, 16, l.seg_sorted, order_out, l.sort,
                          false, l.status, stream);
  if (rc) return rc;
  ygx::k_gather_codes<<<ygx::grid_for(n, 256), 256, 0, stream>>>(l.codes, order_out, n,
                                                                 codes_sorted);
  YGX_CHECK_LAUNCH();
  if (seg_sorted_out) {
    ygx::k_u64_to_i32<<<ygx::grid_for(n, 256), 256, 0, stream>>>(l.seg_sorted, n, seg_sorted_out);
    YGX_CHECK_LAUNCH();
  }
  return YGX_OK;
}

size_t ygx_encode_sort_workspace_size(int64_t n) {
  ygx::Arena a{nullptr, 0, 0};
  ygx::carve_encode_sort(a, n);
  return a.used + 256;
}

int ygx_workspace_init(void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (!ws || ws_bytes < 512) return YGX_ERR_ARG;
  return cudaMemsetAsync(ws, 0, 512, stream) == cudaSuccess ? YGX_OK : YGX_ERR_CUDA;
}

int ygx_status_read(const void* ws, uint32_t* host_flags, cudaStream_t stream) {
  if (!ws || !host_flags) return YGX_ERR_ARG;
  if (cudaMemcpyAsync(host_flags, ws, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream) !=
      cudaSuccess)
    return YGX_ERR_CUDA;
  if (cudaStreamSynchronize(stream) != cudaSuccess) return YGX_ERR_CUDA;
  return YGX_OK;
}

int ygx_bounds(const float* positions, int64_t n, float* bounds_out, void* ws, size_t ws_bytes,
               cudaStream_t stream) {
  if (n < 1 || !positions || !bounds_out || !ws) return YGX_ERR_ARG;
  if (ws_bytes < ygx_encode_sort_workspace_size(0)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::EncodeSortLayout l = ygx::carve_encode_sort(a, 0);
  if (cudaMemsetAsync(l.arrivals, 0, sizeof(unsigned), stream) != cudaSuccess) return YGX_ERR_CUDA;
  int grid = ygx::grid_for((n + 3) / 4, ygx::kBBoxThreads, ygx::kBBoxBlocks);
  ygx::k_bbox<<<grid, ygx::kBBoxThreads, 0, stream>>>(positions, n, l.partials, l.arrivals,
                                                      bounds_out);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

int ygx_morton_encode(const float* positions, int64_t n, const float* bounds, uint64_t* codes,
                      cudaStream_t stream) {
  if (n < 0 || (n > 0 && (!positions || !bounds || !codes))) return YGX_ERR_ARG;
  if (n == 0) return YGX_OK;
  int grid = ygx::grid_for((n + 3) / 4, ygx::kEncodeThreads, ygx::kNumSMs * 8);
  ygx::k_encode<<<grid, ygx::kEncodeThreads, 0, stream>>>(positions, n, bounds, codes, nullptr, 0);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

int ygx_encode_sort(const float* positions, int64_t n, const float* bounds_in, float* bounds_out,
                    uint64_t* codes_sorted, uint32_t* order, void* ws, size_t ws_bytes,
                    cudaStream_t stream) {
  if (n < 1 || !positions || !bounds_out || !codes_sorted || !order || !ws) return YGX_ERR_ARG;
  if (ws_bytes < ygx_encode_sort_workspace_size(n)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::EncodeSortLayout l = ygx::carve_encode_sort(a, n);
  if (bounds_in) {
    if (cudaMemcpyAsync(bounds_out, bounds_in, 6 * sizeof(float), cudaMemcpyDeviceToDevice,
                        stream) != cudaSuccess)
      return YGX_ERR_CUDA;
  }
  // the 8-bit sort's digit histograms come out of the encode; the 11-bit
  // sort counts its own
  const int passes = ygx::sort_uses_wide(0, 63) ? 0 : ygx::sort_passes(0, 63);
  if (ygx::sort_scratch_reset(l.sort, n, passes, stream) != cudaSuccess) return YGX_ERR_CUDA;
  bool fused = false;
  if (!bounds_in) {
    // one cooperative launch: bounds, codes and histograms (see k_bbox_encode)
    int grid = ygx::fused_grid();
    if (grid > 0) {
      const int64_t want = ((n + 3) / 4 + ygx::kEncodeThreads - 1) / ygx::kEncodeThreads;
      if (want < grid) grid = want > 0 ? (int)want : 1;
      if (cudaMemsetAsync(l.arrivals, 0, 2 * sizeof(unsigned), stream) != cudaSuccess)
        return YGX_ERR_CUDA;
      const float* p_ = positions;
      int64_t n_ = n;
      float* part_ = l.partials;
      unsigned* arr_ = l.arrivals;
      float* bo_ = bounds_out;
      uint64_t* co_ = codes_sorted;
      uint32_t* hi_ = l.sort.hist;
      int pa_ = passes;
      uint32_t sl_ = (uint32_t)ygx::g_tune.spin_limit;
      uint32_t* st_ = l.status;
      void* args[] = {&p_, &n_, &part_, &arr_, &bo_, &co_, &hi_, &pa_, &sl_, &st_};
      const cudaError_t e = cudaLaunchCooperativeKernel((const void*)ygx::k_bbox_encode,
                                                        dim3((unsigned)grid),
                                                        dim3(ygx::kEncodeThreads), args, 0, stream);
      ygx::note_launch();
      if (e == cudaSuccess) fused = true;
      else (void)cudaGetLastError();  // not launchable here: the two-kernel path below
    }
    if (!fused) {
      if (cudaMemsetAsync(l.arrivals, 0, sizeof(unsigned), stream) != cudaSuccess)
        return YGX_ERR_CUDA;
      int g2 = ygx::grid_for((n + 3) / 4, ygx::kBBoxThreads, ygx::kBBoxBlocks);
      ygx::k_bbox<<<g2, ygx::kBBoxThreads, 0, stream>>>(positions, n, l.partials, l.arrivals,
                                                        bounds_out);
      YGX_CHECK_LAUNCH();
    }
  }
  if (!fused) {
    int grid = ygx::grid_for((n + 3) / 4, ygx::kEncodeThreads, ygx::kNumSMs * 8);
    ygx::k_encode<<<grid, ygx::kEncodeThreads, 0, stream>>>(positions, n, bounds_out,
                                                            codes_sorted, l.sort.hist, passes);
    YGX_CHECK_LAUNCH();
  }
  return ygx::onesweep_sort(codes_sorted, nullptr, n, 0, 63, codes_sorted, order, l.sort, true,
                            l.status, stream);
}

}  // extern "C"
