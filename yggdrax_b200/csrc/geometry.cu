// Per-node geometry (L2): replaces compute_tree_geometry
// (_geometry_impl.py:176-338).
//
// Leaves: masked min/max of their particle range (one warp per leaf, the
// range is contiguous in Morton order) or the Morton cell box.  Internal
// nodes: a bottom-up refit in which each finished node increments an arrival
// counter on its parent and the second arrival merges the two children and
// climbs on -- nothing ever waits.  min/max are exact, so this equals the
// reference's level-serial pass on every well-formed topology.  For the
// malformed topologies that tied leaf codes can produce (children whose
// parent entry names another node), a single-CTA level-serial pass
// reproduces the reference's order of evaluation, including the zeros that
// internal nodes start from.
#include "common.cuh"

namespace ygx {
namespace {

__device__ __forceinline__ void finalize_node(int64_t k, const float lo[3], const float hi[3],
                                              float* __restrict__ center,
                                              float* __restrict__ half,
                                              float* __restrict__ radius,
                                              float* __restrict__ max_extent) {
  float h[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    center[3 * k + a] = __fmul_rn(0.5f, __fadd_rn(lo[a], hi[a]));
    h[a] = fmax_nan(__fmul_rn(0.5f, __fsub_rn(hi[a], lo[a])), 1e-6f);
    half[3 * k + a] = h[a];
  }
  float s = __fmul_rn(h[0], h[0]);
  s = __fadd_rn(s, __fmul_rn(h[1], h[1]));
  s = __fadd_rn(s, __fmul_rn(h[2], h[2]));
  radius[k] = __fsqrt_rn(s);
  max_extent[k] = fmax_nan(fmax_nan(h[0], h[1]), h[2]);
}

__device__ __forceinline__ void ld_box(const float* __restrict__ mn, const float* __restrict__ mx,
                                       int64_t k, float lo[3], float hi[3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = __ldcg(mn + 3 * k + a);
    hi[a] = __ldcg(mx + 3 * k + a);
  }
}

// Arrival on a parent: release this thread's box writes, acquire the
// sibling's (one acq_rel atomic instead of a fence on either side).
__device__ __forceinline__ int arrive_acq_rel(int32_t* p) {
  int old;
  asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(old) : "l"(p) : "memory");
  return old;
}

__device__ void climb(int64_t node, const int32_t* __restrict__ parent32,
                      const int32_t* __restrict__ left32, const int32_t* __restrict__ right32,
                      float* __restrict__ mn, float* __restrict__ mx, int32_t* __restrict__ arrive,
                      float* __restrict__ center, float* __restrict__ half,
                      float* __restrict__ radius, float* __restrict__ max_extent) {
  int64_t p = parent32[node];
  while (p >= 0) {
    if (arrive_acq_rel(&arrive[p]) == 0) return;  // sibling not finished yet
    const int64_t l = left32[p], r = right32[p];
    float llo[3], lhi[3], rlo[3], rhi[3], lo[3], hi[3];
    ld_box(mn, mx, l, llo, lhi);
    ld_box(mn, mx, r, rlo, rhi);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      lo[a] = fmin_nan(llo[a], rlo[a]);
      hi[a] = fmax_nan(lhi[a], rhi[a]);
      __stcg(mn + 3 * p + a, lo[a]);
      __stcg(mx + 3 * p + a, hi[a]);
    }
    finalize_node(p, lo, hi, center, half, radius, max_extent);
    p = parent32[p];
  }
}

// Leaf boxes from particle ranges.  A warp reduces 32 leaves one after the
// other (coalesced particle loads, shuffle reductions); lane j keeps leaf j's
// box, and then all 32 lanes climb at once.
__global__ void k_leaf_ranges_refit(const void* ranges, int64_t ni, int64_t L, int index_bits,
                                    const float* __restrict__ pos, int64_t cap, bool empty_inf,
                                    const int32_t* __restrict__ parent32,
                                    const int32_t* __restrict__ left32,
                                    const int32_t* __restrict__ right32, float* __restrict__ mn,
                                    float* __restrict__ mx, int32_t* __restrict__ arrive,
                                    const uint32_t* __restrict__ tree_flags, float* center,
                                    float* half, float* radius, float* max_extent) {
  const bool climb_ok = !(*tree_flags & kFlagMalformed);
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const float big = empty_inf ? __int_as_float(0x7f800000) : 3.402823466e38f;
  const float qnan = __int_as_float(0x7fc00000);
  for (int64_t base = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32;
       base < L; base += warps * 32) {
    float my_lo[3] = {0.f, 0.f, 0.f}, my_hi[3] = {0.f, 0.f, 0.f};
    const int nl = L - base < 32 ? (int)(L - base) : 32;
    for (int jj = 0; jj < nl; ++jj) {
      const int64_t node = ni + base + jj;
      const int64_t s = load_idx(ranges, index_bits, 2 * node);
      int64_t c = load_idx(ranges, index_bits, 2 * node + 1) - s + 1;
      if (cap >= 0 && c > cap) c = cap;
      float lo[3] = {big, big, big}, hi[3] = {-big, -big, -big};
      unsigned nan = 0;
      for (int64_t k = lane; k < c; k += 32) {
        const float* p = pos + 3 * (s + k);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          float v = __ldg(p + a);
          if (v != v) nan |= 1u << a;
          lo[a] = fminf(lo[a], v);
          hi[a] = fmaxf(hi[a], v);
        }
      }
      for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          lo[a] = fminf(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], off));
          hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], off));
        }
        nan |= __shfl_xor_sync(0xffffffffu, nan, off);
      }
      if (lane == jj) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          my_lo[a] = (nan >> a) & 1 ? qnan : lo[a];
          my_hi[a] = (nan >> a) & 1 ? qnan : hi[a];
        }
      }
    }
    if (lane < nl) {
      const int64_t node = ni + base + lane;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        __stcg(mn + 3 * node + a, my_lo[a]);
        __stcg(mx + 3 * node + a, my_hi[a]);
      }
      finalize_node(node, my_lo, my_hi, center, half, radius, max_extent);
      if (climb_ok) climb(node, parent32, left32, right32, mn, mx, arrive, center, half, radius,
                          max_extent);
    }
  }
}

// Leaf boxes from Morton cells (_geometry_impl.py:133-172).
__global__ void k_leaf_morton_refit(const uint64_t* __restrict__ leaf_codes, const void* leaf_depths,
                                    int64_t ni, int64_t L, int index_bits,
                                    const float* __restrict__ bounds,
                                    const int32_t* __restrict__ parent32,
                                    const int32_t* __restrict__ left32,
                                    const int32_t* __restrict__ right32, float* __restrict__ mn,
                                    float* __restrict__ mx, int32_t* __restrict__ arrive,
                                    const uint32_t* __restrict__ tree_flags, float* center,
                                    float* half, float* radius, float* max_extent) {
  const bool climb_ok = !(*tree_flags & kFlagMalformed);
  float bmin[3], dom[3];
  for (int a = 0; a < 3; ++a) {
    bmin[a] = bounds[a];
    dom[a] = __fsub_rn(bounds[3 + a], bounds[a]);
  }
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < L;
       j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t node = ni + j;
    int64_t dc = load_idx(leaf_depths, index_bits, j);
    dc = dc < 0 ? 0 : (dc > 21 ? 21 : dc);
    const uint64_t sh = (uint64_t)(21 - dc);
    const uint64_t code = leaf_codes[j];
    const uint64_t q[3] = {compact3(code) >> sh, compact3(code >> 1) >> sh, compact3(code >> 2) >> sh};
    const float cnt = (float)(1ull << dc);
    float lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      float cell = __fdiv_rn(dom[a], cnt);
      lo[a] = __fadd_rn(bmin[a], __fmul_rn(cell, (float)q[a]));
      hi[a] = __fadd_rn(lo[a], cell);
      __stcg(mn + 3 * node + a, lo[a]);
      __stcg(mx + 3 * node + a, hi[a]);
    }
    finalize_node(node, lo, hi, center, half, radius, max_extent);
    if (climb_ok) climb(node, parent32, left32, right32, mn, mx, arrive, center, half, radius,
                        max_extent);
  }
}

// Reference-order fallback for malformed topologies: one CTA, levels from
// the deepest internal level up, synchronous within a level.
__global__ void __launch_bounds__(1024)
    k_serial_refit(int64_t total, int64_t ni, const int32_t* __restrict__ level32,
                   const int32_t* __restrict__ left32, const int32_t* __restrict__ right32,
                   float* __restrict__ mn, float* __restrict__ mx, float* __restrict__ tmp,
                   const uint32_t* __restrict__ tree_flags, float* center, float* half,
                   float* radius, float* max_extent) {
  if (!(*tree_flags & kFlagMalformed)) return;
  __shared__ int s_max;
  if (threadIdx.x == 0) s_max = 0;
  __syncthreads();
  int mxl = 0;
  for (int64_t k = threadIdx.x; k < total; k += blockDim.x) mxl = max(mxl, level32[k]);
  atomicMax(&s_max, mxl);
  for (int64_t k = threadIdx.x; k < ni; k += blockDim.x)
    for (int a = 0; a < 3; ++a) { mn[3 * k + a] = 0.0f; mx[3 * k + a] = 0.0f; }
  __syncthreads();
  const int maxd = s_max;
  for (int level = maxd - 1; level >= 0; --level) {
    for (int64_t i = threadIdx.x; i < ni; i += blockDim.x) {
      if (level32[i] != level) continue;
      const int64_t l = left32[i], r = right32[i];
      for (int a = 0; a < 3; ++a) {
        tmp[6 * i + a] = fmin_nan(mn[3 * l + a], mn[3 * r + a]);
        tmp[6 * i + 3 + a] = fmax_nan(mx[3 * l + a], mx[3 * r + a]);
      }
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < ni; i += blockDim.x) {
      if (level32[i] != level) continue;
      for (int a = 0; a < 3; ++a) { mn[3 * i + a] = tmp[6 * i + a]; mx[3 * i + a] = tmp[6 * i + 3 + a]; }
    }
    __syncthreads();
  }
  for (int64_t k = threadIdx.x; k < ni; k += blockDim.x) {
    float lo[3], hi[3];
    for (int a = 0; a < 3; ++a) { lo[a] = mn[3 * k + a]; hi[a] = mx[3 * k + a]; }
    finalize_node(k, lo, hi, center, half, radius, max_extent);
  }
}

// ---- batched sets (a forest: set s at nodes NO_s = 2 leaf_off[s] - s) ------

// k_leaf_ranges_refit over the leaves of all sets: a warp reduces 32 leaves
// (global leaf positions) one after the other, then every lane climbs its
// set's tree.  Particle ranges are local to the set (offset off[s]).
__global__ void k_seg_leaf_refit(const void* ranges, const int64_t* __restrict__ leaf_off,
                                 const int32_t* __restrict__ leaf_seg,
                                 const int64_t* __restrict__ off, int64_t Ltot, int index_bits,
                                 const float* __restrict__ pos, int64_t cap, bool empty_inf,
                                 const int32_t* __restrict__ parent32,
                                 const int32_t* __restrict__ left32,
                                 const int32_t* __restrict__ right32, float* __restrict__ mn,
                                 float* __restrict__ mx, int32_t* __restrict__ arrive,
                                 const uint32_t* __restrict__ seg_flags, float* center,
                                 float* half, float* radius, float* max_extent) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const float big = empty_inf ? __int_as_float(0x7f800000) : 3.402823466e38f;
  const float qnan = __int_as_float(0x7fc00000);
  for (int64_t base = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32;
       base < Ltot; base += warps * 32) {
    float my_lo[3] = {0.f, 0.f, 0.f}, my_hi[3] = {0.f, 0.f, 0.f};
    int64_t my_node = -1;
    int32_t my_seg = 0;
    const int nl = Ltot - base < 32 ? (int)(Ltot - base) : 32;
    for (int jj = 0; jj < nl; ++jj) {
      const int64_t g = base + jj;
      const int32_t sg = leaf_seg[g];
      const int64_t a = leaf_off[sg], Ls = leaf_off[sg + 1] - a;
      const int64_t node = 2 * a - sg + Ls - 1 + (g - a);
      const int64_t s0 = load_idx(ranges, index_bits, 2 * node);
      int64_t c = load_idx(ranges, index_bits, 2 * node + 1) - s0 + 1;
      if (cap >= 0 && c > cap) c = cap;
      const int64_t pb = off[sg] + s0;
      float lo[3] = {big, big, big}, hi[3] = {-big, -big, -big};
      unsigned nan = 0;
      for (int64_t k = lane; k < c; k += 32) {
        const float* p = pos + 3 * (pb + k);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          float v = __ldg(p + q);
          if (v != v) nan |= 1u << q;
          lo[q] = fminf(lo[q], v);
          hi[q] = fmaxf(hi[q], v);
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          lo[q] = fminf(lo[q], __shfl_xor_sync(0xffffffffu, lo[q], o));
          hi[q] = fmaxf(hi[q], __shfl_xor_sync(0xffffffffu, hi[q], o));
        }
        nan |= __shfl_xor_sync(0xffffffffu, nan, o);
      }
      if (lane == jj) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          my_lo[q] = (nan >> q) & 1 ? qnan : lo[q];
          my_hi[q] = (nan >> q) & 1 ? qnan : hi[q];
        }
        my_node = node;
        my_seg = sg;
      }
    }
    if (lane < nl) {
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        __stcg(mn + 3 * my_node + q, my_lo[q]);
        __stcg(mx + 3 * my_node + q, my_hi[q]);
      }
      finalize_node(my_node, my_lo, my_hi, center, half, radius, max_extent);
      if (!(seg_flags[my_seg] & kFlagMalformed))
        climb(my_node, parent32, left32, right32, mn, mx, arrive, center, half, radius,
              max_extent);
    }
  }
}

// k_serial_refit per malformed set: one CTA per set (others return).
__global__ void __launch_bounds__(1024)
    k_seg_serial_refit(const int64_t* __restrict__ leaf_off, int64_t S,
                       const int32_t* __restrict__ level32, const int32_t* __restrict__ left32,
                       const int32_t* __restrict__ right32, float* __restrict__ mn,
                       float* __restrict__ mx, float* __restrict__ tmp,
                       const uint32_t* __restrict__ seg_flags, float* center, float* half,
                       float* radius, float* max_extent) {
  __shared__ int s_max;
  for (int64_t sg = blockIdx.x; sg < S; sg += gridDim.x) {
    if (!(seg_flags[sg] & kFlagMalformed)) continue;
    const int64_t a = leaf_off[sg], Ls = leaf_off[sg + 1] - a, NO = 2 * a - sg;
    const int64_t ni = Ls - 1, total = 2 * Ls - 1;
    if (threadIdx.x == 0) s_max = 0;
    __syncthreads();
    int mxl = 0;
    for (int64_t k = threadIdx.x; k < total; k += blockDim.x) mxl = max(mxl, level32[NO + k]);
    atomicMax(&s_max, mxl);
    for (int64_t k = threadIdx.x; k < ni; k += blockDim.x)
      for (int q = 0; q < 3; ++q) { mn[3 * (NO + k) + q] = 0.0f; mx[3 * (NO + k) + q] = 0.0f; }
    __syncthreads();
    const int maxd = s_max;
    for (int level = maxd - 1; level >= 0; --level) {
      for (int64_t i = NO + threadIdx.x; i < NO + ni; i += blockDim.x) {
        if (level32[i] != level) continue;
        const int64_t l = left32[i], r = right32[i];
        for (int q = 0; q < 3; ++q) {
          tmp[6 * i + q] = fmin_nan(mn[3 * l + q], mn[3 * r + q]);
          tmp[6 * i + 3 + q] = fmax_nan(mx[3 * l + q], mx[3 * r + q]);
        }
      }
      __syncthreads();
      for (int64_t i = NO + threadIdx.x; i < NO + ni; i += blockDim.x) {
        if (level32[i] != level) continue;
        for (int q = 0; q < 3; ++q) {
          mn[3 * i + q] = tmp[6 * i + q];
          mx[3 * i + q] = tmp[6 * i + 3 + q];
        }
      }
      __syncthreads();
    }
    for (int64_t k = NO + threadIdx.x; k < NO + ni; k += blockDim.x) {
      float lo[3], hi[3];
      for (int q = 0; q < 3; ++q) { lo[q] = mn[3 * k + q]; hi[q] = mx[3 * k + q]; }
      finalize_node(k, lo, hi, center, half, radius, max_extent);
    }
    __syncthreads();
  }
}

}  // namespace

struct GeoScratch {
  uint32_t* status;
  float* mn;
  float* mx;
  float* tmp;
  int32_t* arrive;
};

static GeoScratch carve_geo(Arena& a, int64_t total) {
  GeoScratch s;
  s.status = a.take<uint32_t>(64);
  s.mn = a.take<float>(3 * total);
  s.mx = a.take<float>(3 * total);
  s.tmp = a.take<float>(6 * total);
  s.arrive = a.take<int32_t>(total);
  return s;
}

}  // namespace ygx

extern "C" {

size_t ygx_geometry_workspace_size(int64_t total) {
  ygx::Arena a{nullptr, 0, 0};
  ygx::carve_geo(a, total);
  return a.used + 256;
}

// use_morton: leaf boxes from (leaf_codes, leaf_depths, bounds) cells; else
// from particle ranges of positions_sorted, at most max_leaf_size particles
// per leaf (max_leaf_size < 0: no cap).  parent32/left32/right32 are the
// int32 topology copies of ygx_build_topology (left/right = -1 on leaves);
// level32 the node levels; tree_flags the device flags word it wrote.
int ygx_tree_geometry(const void* node_ranges, int64_t total, int index_bits,
                      const int32_t* parent32, const int32_t* left32, const int32_t* right32,
                      const int32_t* level32, const uint32_t* tree_flags,
                      const float* positions_sorted, int64_t n, int use_morton,
                      const float* bounds, const uint64_t* leaf_codes, const void* leaf_depths,
                      int64_t max_leaf_size, float* center, float* half_extent, float* radius,
                      float* max_extent, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (total < 1 || (index_bits != 32 && index_bits != 64)) return YGX_ERR_ARG;
  if (ws_bytes < ygx_geometry_workspace_size(total)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::GeoScratch s = ygx::carve_geo(a, total);
  const int64_t ni = (total - 1) / 2, L = total - ni;
  if (cudaMemsetAsync(s.arrive, 0, sizeof(int32_t) * total, stream) != cudaSuccess) return YGX_ERR_CUDA;
  if (use_morton) {
    ygx::k_leaf_morton_refit<<<ygx::grid_for(L, 128), 128, 0, stream>>>(
        leaf_codes, leaf_depths, ni, L, index_bits, bounds, parent32, left32, right32, s.mn, s.mx,
        s.arrive, tree_flags, center, half_extent, radius, max_extent);
  } else {
    const int warps = ygx::g_tune.refit_warps;
    ygx::k_leaf_ranges_refit<<<ygx::grid_for((L + 31) / 32, warps, ygx::kNumSMs * 16), warps * 32, 0,
                               stream>>>(
        node_ranges, ni, L, index_bits, positions_sorted, max_leaf_size, max_leaf_size == 0,
        parent32, left32, right32, s.mn, s.mx, s.arrive, tree_flags, center, half_extent, radius,
        max_extent);
  }
  YGX_CHECK_LAUNCH();
  if (ni > 0) {
    ygx::k_serial_refit<<<1, 1024, 0, stream>>>(total, ni, level32, left32, right32, s.mn, s.mx,
                                                s.tmp, tree_flags, center, half_extent, radius,
                                                max_extent);
    YGX_CHECK_LAUNCH();
  }
  return YGX_OK;
}

// Geometry of every tree of a batched forest (ygx_batch_build_topology):
// leaf boxes from the sets' particle ranges in positions_sorted (set s at
// offsets[s]), at most max_leaf_size particles per leaf; total = 2
// total_leaves - S nodes.
int ygx_batch_tree_geometry(const void* node_ranges, int64_t total, int64_t S,
                            const int64_t* leaf_off, const int32_t* leaf_seg,
                            int64_t total_leaves, const int64_t* offsets, int index_bits,
                            const int32_t* parent32, const int32_t* left32,
                            const int32_t* right32, const int32_t* level32,
                            const uint32_t* seg_flags, const float* positions_sorted,
                            int64_t max_leaf_size, float* center, float* half_extent,
                            float* radius, float* max_extent, void* ws, size_t ws_bytes,
                            cudaStream_t stream) {
  if (total < 1 || S < 1 || total != 2 * total_leaves - S || (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  if (ws_bytes < ygx_geometry_workspace_size(total)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::GeoScratch s = ygx::carve_geo(a, total);
  if (cudaMemsetAsync(s.arrive, 0, sizeof(int32_t) * total, stream) != cudaSuccess) return YGX_ERR_CUDA;
  const int warps = ygx::g_tune.refit_warps;
  ygx::k_seg_leaf_refit<<<ygx::grid_for((total_leaves + 31) / 32, warps, ygx::kNumSMs * 16),
                          warps * 32, 0, stream>>>(
      node_ranges, leaf_off, leaf_seg, offsets, total_leaves, index_bits, positions_sorted,
      max_leaf_size, max_leaf_size == 0, parent32, left32, right32, s.mn, s.mx, s.arrive,
      seg_flags, center, half_extent, radius, max_extent);
  YGX_CHECK_LAUNCH();
  ygx::k_seg_serial_refit<<<(unsigned)(S < 1024 ? S : 1024), 1024, 0, stream>>>(
      leaf_off, S, level32, left32, right32, s.mn, s.mx, s.tmp, seg_flags, center, half_extent,
      radius, max_extent);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

}  // extern "C"
