// Tree build kernels (L1): reorder, leaf partitions (adaptive, fixed depth,
// local aspect refinement), Karras LBVH topology and node levels.
#include "scan.cuh"
#include "karras.cuh"
#include "sort.cuh"

namespace ygx {
namespace {

// ---------------------------------------------------------------------------
// _tree_impl.py:900-926 and :1047-1050: positions/masses gathered into Morton
// order, particle_indices in the index dtype, inverse permutation scatter.
// Each thread takes kReorderItems particles of a 256 x kReorderItems chunk
// (coalesced index loads and sorted-order stores) and issues all of their
// random gathers before any store, so several gathers are in flight per
// thread instead of one dependent chain per particle.
constexpr int kReorderItems = 4;
constexpr int kReorderThreads = 256;

__global__ void __launch_bounds__(kReorderThreads)
    k_reorder(const float* __restrict__ pos, const float* __restrict__ mass,
              const uint32_t* __restrict__ order, int64_t n, int index_bits,
              float* __restrict__ pos_sorted, float* __restrict__ mass_sorted,
              void* __restrict__ particle_indices, void* __restrict__ inverse) {
  constexpr int64_t kChunk = (int64_t)kReorderThreads * kReorderItems;
  for (int64_t k0 = (int64_t)blockIdx.x * kChunk + threadIdx.x; k0 < n;
       k0 += (int64_t)gridDim.x * kChunk) {
    uint32_t v[kReorderItems];
    float x[kReorderItems], y[kReorderItems], z[kReorderItems], m[kReorderItems];
#pragma unroll
    for (int u = 0; u < kReorderItems; ++u) {
      const int64_t k = k0 + (int64_t)u * kReorderThreads;
      v[u] = k < n ? order[k] : 0u;
    }
#pragma unroll
    for (int u = 0; u < kReorderItems; ++u) {
      const int64_t k = k0 + (int64_t)u * kReorderThreads;
      if (k < n && pos_sorted) {
        x[u] = __ldg(pos + 3 * (int64_t)v[u]);
        y[u] = __ldg(pos + 3 * (int64_t)v[u] + 1);
        z[u] = __ldg(pos + 3 * (int64_t)v[u] + 2);
      }
      if (k < n && mass_sorted) m[u] = __ldg(mass + v[u]);
    }
#pragma unroll
    for (int u = 0; u < kReorderItems; ++u) {
      const int64_t k = k0 + (int64_t)u * kReorderThreads;
      if (k >= n) continue;
      if (pos_sorted) {
        pos_sorted[3 * k] = x[u];
        pos_sorted[3 * k + 1] = y[u];
        pos_sorted[3 * k + 2] = z[u];
      }
      if (mass_sorted) mass_sorted[k] = m[u];
      if (particle_indices) store_idx(particle_indices, index_bits, k, v[u]);
      if (inverse) store_idx(inverse, index_bits, v[u], k);
    }
  }
}

// The same reorder from particles packed as (x, y, z, mass) float4 records:
// one aligned 16-byte gather (a single sector) per particle instead of a
// 12-byte position that may straddle two sectors plus a 4-byte mass in a
// third.  k_pack_particles writes the records in one coalesced pass.
__global__ void k_pack_particles(const float* __restrict__ pos, const float* __restrict__ mass,
                                 int64_t n, float4* __restrict__ packed) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    packed[k] = make_float4(pos[3 * k], pos[3 * k + 1], pos[3 * k + 2], mass[k]);
}

__global__ void __launch_bounds__(kReorderThreads)
    k_reorder_packed(const float4* __restrict__ packed, const uint32_t* __restrict__ order,
                     int64_t n, int index_bits, float* __restrict__ pos_sorted,
                     float* __restrict__ mass_sorted, void* __restrict__ particle_indices,
                     void* __restrict__ inverse) {
  constexpr int64_t kChunk = (int64_t)kReorderThreads * kReorderItems;
  for (int64_t k0 = (int64_t)blockIdx.x * kChunk + threadIdx.x; k0 < n;
       k0 += (int64_t)gridDim.x * kChunk) {
    uint32_t v[kReorderItems];
    float4 p[kReorderItems];
#pragma unroll
    for (int u = 0; u < kReorderItems; ++u) {
      const int64_t k = k0 + (int64_t)u * kReorderThreads;
      v[u] = k < n ? order[k] : 0u;
    }
#pragma unroll
    for (int u = 0; u < kReorderItems; ++u) {
      const int64_t k = k0 + (int64_t)u * kReorderThreads;
      if (k < n) p[u] = __ldg(packed + v[u]);
    }
#pragma unroll
    for (int u = 0; u < kReorderItems; ++u) {
      const int64_t k = k0 + (int64_t)u * kReorderThreads;
      if (k >= n) continue;
      if (pos_sorted) {
        pos_sorted[3 * k] = p[u].x;
        pos_sorted[3 * k + 1] = p[u].y;
        pos_sorted[3 * k + 2] = p[u].z;
      }
      if (mass_sorted) mass_sorted[k] = p[u].w;
      if (particle_indices) store_idx(particle_indices, index_bits, k, v[u]);
      if (inverse) store_idx(inverse, index_bits, v[u], k);
    }
  }
}

// _tree_impl.py:405-406: fixed-size chunks of the sorted order.
__global__ void k_leaves_adaptive(const uint64_t* __restrict__ codes, int64_t n, int64_t leaf_size,
                                  int64_t L, int index_bits, void* starts, void* ends,
                                  uint64_t* __restrict__ leaf_codes, void* depths) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < L;
       j += (int64_t)gridDim.x * blockDim.x) {
    int64_t s = j * leaf_size;
    int64_t e = s + leaf_size < n ? s + leaf_size : n;
    store_idx(starts, index_bits, j, s);
    store_idx(ends, index_bits, j, e);
    leaf_codes[j] = codes[s];
    if (depths) store_idx(depths, index_bits, j, -1);
  }
}

__device__ __forceinline__ int64_t lower_bound_u64(const uint64_t* a, int64_t n, uint64_t q) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] < q) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// _tree_impl.py:1373-1401: dense 8^d buckets over the sorted codes.  Because
// the codes are sorted, bucket b starts at lower_bound(b << shift); counts
// and the exclusive scan of the reference follow from the bucket bounds.
__global__ void k_leaves_fixed(const uint64_t* __restrict__ codes, int64_t n, int depth,
                               int64_t L, int index_bits, void* starts, void* ends,
                               uint64_t* __restrict__ leaf_codes, void* depths) {
  const int shift = 63 - 3 * depth > 0 ? 63 - 3 * depth : 0;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < L;
       b += (int64_t)gridDim.x * blockDim.x) {
    uint64_t lo = (uint64_t)b << shift;
    int64_t s = lower_bound_u64(codes, n, lo);
    int64_t e = b + 1 < L ? lower_bound_u64(codes, n, (uint64_t)(b + 1) << shift) : n;
    store_idx(starts, index_bits, b, s);
    store_idx(ends, index_bits, b, e);
    leaf_codes[b] = lo;
    store_idx(depths, index_bits, b, depth);
  }
}

// ---------------------------------------------------------------------------
// _tree_impl.py:96-227 (_refine_leaf_partitions_by_aspect), one warp per
// input bucket.  The reference walks a FIFO queue and finally orders leaves
// by (start, code); within a bucket the emitted leaves tile its particle
// range in increasing sub-octant order, so a depth-first walk that visits
// sub-octants in increasing order emits them already in (start, code) order,
// and buckets are emitted in bucket order.  The float64 aspect test, the
// fp32 comparison of the 1e-12 floor and the 64 - 3*depth entry shift follow
// the reference exactly.
struct RefineItem {
  int64_t s, e;
  uint64_t code;
  int32_t depth;
  int32_t final_leaf;  // child with <= min_leaf particles: emitted as is
};

constexpr int kRefineStack = 64;

template <bool kEmit>
__global__ void k_refine(const float* __restrict__ pos_sorted, const uint64_t* __restrict__ codes,
                         const void* starts, const void* ends, const uint64_t* __restrict__ bcodes,
                         const void* bdepths, int64_t L, int current_depth,
                         int max_refine_levels, double aspect_threshold, int min_leaf,
                         int index_bits, int64_t* __restrict__ counts,
                         const int64_t* __restrict__ offsets, void* o_starts, void* o_ends,
                         uint64_t* __restrict__ o_codes, void* o_depths,
                         uint32_t* __restrict__ status) {
  __shared__ RefineItem s_stack[8][kRefineStack];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  RefineItem* stack = s_stack[wib];
  for (int64_t b = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib; b < L; b += warps) {
    int64_t emitted = 0;
    const int64_t out_base = kEmit ? offsets[b] : 0;
    if (lane == 0) {
      stack[0].s = load_idx(starts, index_bits, b);
      stack[0].e = load_idx(ends, index_bits, b);
      stack[0].code = bcodes[b];
      stack[0].depth = (int32_t)load_idx(bdepths, index_bits, b);
      stack[0].final_leaf = 0;
    }
    int sp = 1;
    __syncwarp();
    while (sp > 0) {
      const RefineItem it = stack[sp - 1];
      __syncwarp();
      --sp;
      bool keep = it.final_leaf != 0 || it.e <= it.s;
      int64_t cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      int64_t child_shift = -1;
      if (!keep) {
        float mn[3], mx[3];
        unsigned nan = 0;
        for (int a = 0; a < 3; ++a) { mn[a] = __int_as_float(0x7f800000); mx[a] = -__int_as_float(0x7f800000); }
        for (int64_t p = it.s + lane; p < it.e; p += 32)
          for (int a = 0; a < 3; ++a) {
            float v = pos_sorted[3 * p + a];
            if (v != v) nan |= 1u << a;
            mn[a] = fminf(mn[a], v);
            mx[a] = fmaxf(mx[a], v);
          }
        for (int off = 16; off > 0; off >>= 1) {
          for (int a = 0; a < 3; ++a) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], off));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], off));
          }
          nan |= __shfl_xor_sync(0xffffffffu, nan, off);
        }
        const float qnan = __int_as_float(0x7fc00000);
        float ext[3];
        for (int a = 0; a < 3; ++a) ext[a] = ((nan >> a) & 1) ? qnan : __fsub_rn(mx[a], mn[a]);
        const float emin = fmin_nan(fmin_nan(ext[0], ext[1]), ext[2]);
        const float emax = fmax_nan(fmax_nan(ext[0], ext[1]), ext[2]);
        // max(emin, 1e-12) in Python compares in fp32 and keeps emin unless
        // the floor is strictly larger; the ratio is taken in float64.
        const double min_axis = (1e-12f > emin) ? 1e-12 : (double)emin;
        const double aspect = (min_axis > 0.0) ? (double)emax / min_axis
                                               : __longlong_as_double(0x7ff0000000000000ll);
        const bool exceeded = (it.depth - current_depth) >= max_refine_levels;
        int64_t entry_shift = 64 - (int64_t)it.depth * 3;
        if (entry_shift < 0) entry_shift = 0;
        child_shift = entry_shift - 3;
        if (aspect <= aspect_threshold || exceeded || child_shift < 0) {
          keep = true;
        } else {
          for (int64_t p = it.s + lane; p < it.e; p += 32) cnt[(codes[p] >> child_shift) & 7ull]++;
          int nz = 0;
          for (int k = 0; k < 8; ++k) {
            int64_t c = cnt[k];
            for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
            cnt[k] = c;
            nz += c != 0;
          }
          if (nz <= 1) keep = true;
        }
      }
      if (keep) {
        if (kEmit && lane == 0) {
          const int64_t o = out_base + emitted;
          store_idx(o_starts, index_bits, o, it.s);
          store_idx(o_ends, index_bits, o, it.e);
          o_codes[o] = it.code;
          store_idx(o_depths, index_bits, o, it.depth);
        }
        ++emitted;
        continue;
      }
      // The children tile [s, e) in increasing sub order.  Push them in
      // reverse so the lowest pops first; a refined child is expanded
      // completely before its next sibling pops (depth-first pre-order).
      int64_t child_off[8];
      int64_t off = it.s;
      for (int sub = 0; sub < 8; ++sub) { child_off[sub] = off; off += cnt[sub]; }
      for (int sub = 7; sub >= 0; --sub) {
        if (cnt[sub] == 0) continue;
        if (sp >= kRefineStack) {
          if (lane == 0) raise_flag(status, kFlagQueueOverflow);
          continue;
        }
        if (lane == 0) {
          RefineItem c;
          c.s = child_off[sub];
          c.e = child_off[sub] + cnt[sub];
          c.code = it.code | ((uint64_t)sub << child_shift);
          c.depth = it.depth + 1;
          c.final_leaf = cnt[sub] <= min_leaf ? 1 : 0;
          stack[sp] = c;
        }
        ++sp;
      }
      __syncwarp();
    }
    if (!kEmit && lane == 0) counts[b] = emitted;
    __syncwarp();
  }
}

__global__ void k_karras(const uint64_t* __restrict__ codes, const void* starts, const void* ends,
                         int64_t L, int index_bits, void* left, void* right,
                         uint8_t* __restrict__ lil, uint8_t* __restrict__ ril, void* ranges,
                         int32_t* __restrict__ left32, int32_t* __restrict__ right32,
                         int32_t* __restrict__ parent_claim) {
  const int64_t ni = L - 1;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ni;
       i += (int64_t)gridDim.x * blockDim.x)
    karras_node(codes, starts, ends, L, i, index_bits, left, right, lil, ril, ranges, left32,
                right32, parent_claim, 0);
}

__global__ void k_leaf_ranges(const void* starts, const void* ends, int64_t L, int index_bits,
                              void* ranges, int32_t* __restrict__ left32,
                              int32_t* __restrict__ right32) {
  const int64_t ni = L - 1;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < L;
       j += (int64_t)gridDim.x * blockDim.x) {
    store_idx(ranges, index_bits, 2 * (ni + j), load_idx(starts, index_bits, j));
    store_idx(ranges, index_bits, 2 * (ni + j) + 1, load_idx(ends, index_bits, j) - 1);
    left32[ni + j] = -1;
    right32[ni + j] = -1;
  }
}

// Decode the claims into parent, and flag any internal node whose children
// do not name it back (a malformed topology from tied codes).
__global__ void k_parent_decode(const int32_t* __restrict__ claim, int64_t total, int64_t ni,
                                int index_bits, void* parent, int32_t* __restrict__ parent32) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    int32_t c = claim[k];
    int64_t p = c < 0 ? -1 : (c >= ni ? c - ni : c);
    store_idx(parent, index_bits, k, p);
    parent32[k] = (int32_t)p;
  }
}

__global__ void k_check_wellformed(const int32_t* __restrict__ parent32,
                                   const int32_t* __restrict__ left32,
                                   const int32_t* __restrict__ right32, int64_t total, int64_t ni,
                                   uint32_t* __restrict__ tree_flags) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    bool bad = (k == 0) ? parent32[0] != -1 : parent32[k] < 0;
    if (k < ni) bad = bad || parent32[left32[k]] != (int32_t)k || parent32[right32[k]] != (int32_t)k;
    if (bad) atomicOr(tree_flags, kFlagMalformed);
  }
}

// _tree_impl.py:1272-1299: depth by synchronous pointer doubling.  Rounds
// after the state stops changing are no-ops, so a round that sees the
// previous round unchanged returns at once; `stop` records how many rounds
// actually ran so the final state can be read from the right buffer.
__global__ void k_depth_init(const int32_t* __restrict__ parent32, int64_t total,
                             int32_t* __restrict__ sc, int32_t* __restrict__ d) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    int32_t p = parent32[k];
    sc[k] = p < 0 ? (int32_t)k : p;
    d[k] = p < 0 ? 0 : 1;
  }
}

__global__ void k_depth_round(const int32_t* __restrict__ sc_in, const int32_t* __restrict__ d_in,
                              int32_t* __restrict__ sc_out, int32_t* __restrict__ d_out,
                              int64_t total, int round, uint32_t* __restrict__ changed,
                              uint32_t* __restrict__ stop) {
  if (round > 0 && ((volatile uint32_t*)changed)[round - 1] == 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicMin(stop, (uint32_t)round);
    return;
  }
  bool any = false;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    int32_t s = sc_in[k];
    int32_t nd = d_in[k] + d_in[s];
    int32_t ns = sc_in[s];
    sc_out[k] = ns;
    d_out[k] = nd;
    any |= (ns != s) || (nd != d_in[k]);
  }
  if (__syncthreads_or(any) && threadIdx.x == 0) atomicOr(&changed[round], 1u);
}

// Final node levels (from whichever buffer holds the last state), the level
// histogram over 64 bins and the 16-bit sort keys for nodes_by_level.
__global__ void k_depth_finish(const int32_t* __restrict__ sc0, const int32_t* __restrict__ d0,
                               const int32_t* __restrict__ sc1, const int32_t* __restrict__ d1,
                               int64_t total, const uint32_t* __restrict__ stop, uint32_t rounds,
                               int index_bits,
                               void* node_level, int32_t* __restrict__ level32,
                               uint64_t* __restrict__ level_keys, uint32_t* __restrict__ level_hist,
                               int32_t* __restrict__ max_level, uint32_t* __restrict__ tree_flags) {
  const uint32_t r = *stop < rounds ? *stop : rounds;
  const int32_t* sc = (r & 1) ? sc1 : sc0;
  const int32_t* d = (r & 1) ? d1 : d0;
  __shared__ uint32_t s_hist[64];
  if (threadIdx.x < 64) s_hist[threadIdx.x] = 0;
  __syncthreads();
  int32_t mx = 0;
  bool detached = false;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    int32_t lv = d[k];
    store_idx(node_level, index_bits, k, lv);
    level32[k] = lv;
    level_keys[k] = (uint64_t)(uint32_t)lv;
    if (lv >= 0 && lv < 64) atomicAdd(&s_hist[lv], 1u);
    mx = lv > mx ? lv : mx;
    detached |= sc[k] != 0;
  }
  __syncthreads();
  if (threadIdx.x < 64 && s_hist[threadIdx.x]) atomicAdd(&level_hist[threadIdx.x], s_hist[threadIdx.x]);
  atomicMax(max_level, mx);
  if (detached) atomicOr(tree_flags, kFlagMalformed);
}

__global__ void k_level_tables(const uint32_t* __restrict__ level_hist,
                               const int32_t* __restrict__ max_level, int index_bits,
                               void* level_offsets, void* num_levels) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int64_t acc = 0;
    store_idx(level_offsets, index_bits, 0, 0);
    for (int l = 0; l < 64; ++l) {
      acc += level_hist[l];
      store_idx(level_offsets, index_bits, l + 1, acc);
    }
    int64_t nl = (int64_t)(*max_level) + 1;
    nl = nl < 1 ? 1 : (nl > 64 ? 64 : nl);
    store_idx(num_levels, index_bits, 0, nl);
  }
}

__global__ void k_u32_to_index(const uint32_t* __restrict__ in, int64_t n, int index_bits,
                               void* out, int32_t* __restrict__ out32) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    store_idx(out, index_bits, k, in[k]);
    if (out32) out32[k] = (int32_t)in[k];
  }
}

// ---- batched sets: a forest of per-set trees --------------------------------
// Set s has L_s leaves at global leaf positions [leaf_off[s], leaf_off[s+1])
// and its 2 L_s - 1 nodes at global node ids [NO_s, NO_s + 2 L_s - 1) with
// NO_s = 2 leaf_off[s] - s, in the reference's per-tree layout (internal
// nodes first).  Per-set output arrays hold local values (what build_tree
// gives for that set alone); the int32 copies hold global node ids.

__device__ __forceinline__ int64_t seg_search(const int64_t* __restrict__ off, int64_t S,
                                              int64_t g) {
  int64_t lo = 0, hi = S;  // last s with off[s] <= g
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (off[mid] <= g) lo = mid; else hi = mid;
  }
  return lo;
}

// Per-set reorder: positions / masses gathered into the sets' sorted order,
// particle_indices and the inverse permutation local to each set.
__global__ void k_seg_reorder(const float* __restrict__ pos, const float* __restrict__ mass,
                              const uint32_t* __restrict__ order,
                              const int32_t* __restrict__ seg_sorted,
                              const int64_t* __restrict__ off, int64_t n, int index_bits,
                              float* __restrict__ pos_sorted, float* __restrict__ mass_sorted,
                              void* particle_indices, void* inverse) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t v = order[k];
    const int64_t base = off[seg_sorted[k]];
    pos_sorted[3 * k] = __ldg(pos + 3 * (int64_t)v);
    pos_sorted[3 * k + 1] = __ldg(pos + 3 * (int64_t)v + 1);
    pos_sorted[3 * k + 2] = __ldg(pos + 3 * (int64_t)v + 2);
    if (mass_sorted) mass_sorted[k] = __ldg(mass + v);
    if (particle_indices) store_idx(particle_indices, index_bits, k, (int64_t)v - base);
    if (inverse) store_idx(inverse, index_bits, v, k - base);
  }
}

__global__ void k_seg_leaf_counts(const int64_t* __restrict__ off, int64_t S, int64_t leaf,
                                  int32_t* __restrict__ cnt) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < S;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = off[s + 1] - off[s];
    cnt[s] = (int32_t)((n + leaf - 1) / leaf);
  }
}

// _tree_impl.py:405-406 per set: fixed-size chunks of the set's sorted order.
__global__ void k_seg_leaves(const uint64_t* __restrict__ codes, const int64_t* __restrict__ off,
                             const int64_t* __restrict__ leaf_off, int64_t S, int64_t Ltot,
                             int64_t leaf, int index_bits, void* starts, void* ends,
                             uint64_t* __restrict__ leaf_codes, void* depths,
                             int32_t* __restrict__ leaf_seg) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < Ltot;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int64_t sg = seg_search(leaf_off, S, g);
    const int64_t j = g - leaf_off[sg], n = off[sg + 1] - off[sg];
    const int64_t b = j * leaf, e = b + leaf < n ? b + leaf : n;
    store_idx(starts, index_bits, g, b);
    store_idx(ends, index_bits, g, e);
    leaf_codes[g] = codes[off[sg] + b];
    if (depths) store_idx(depths, index_bits, g, -1);
    leaf_seg[g] = (int32_t)sg;
  }
}

__device__ __forceinline__ void* idx_ptr(void* base, int index_bits, int64_t k) {
  return (char*)base + k * (index_bits == 32 ? 4 : 8);
}
__device__ __forceinline__ const void* idx_ptr(const void* base, int index_bits, int64_t k) {
  return (const char*)base + k * (index_bits == 32 ? 4 : 8);
}

// One thread per global leaf position: the internal node of that position
// (if any) through karras_node on the set's slice, the leaf node's range,
// and the set id of both nodes.
__global__ void k_seg_karras(const uint64_t* __restrict__ codes, const void* starts,
                             const void* ends, const int64_t* __restrict__ leaf_off,
                             const int32_t* __restrict__ leaf_seg, int64_t Ltot, int index_bits,
                             void* left, void* right, uint8_t* __restrict__ lil,
                             uint8_t* __restrict__ ril, void* ranges,
                             int32_t* __restrict__ left32, int32_t* __restrict__ right32,
                             int32_t* __restrict__ parent_claim,
                             int32_t* __restrict__ node_seg, int32_t* __restrict__ leafpos32,
                             int32_t* __restrict__ node_base, int32_t* __restrict__ leaf_base) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < Ltot;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int32_t sg = leaf_seg[g];
    const int64_t a = leaf_off[sg], Ls = leaf_off[sg + 1] - a, j = g - a;
    const int64_t NO = 2 * a - sg, IO = a - sg;
    if (j < Ls - 1) {
      karras_node(codes + a, idx_ptr(starts, index_bits, a), idx_ptr(ends, index_bits, a), Ls, j,
                  index_bits, idx_ptr(left, index_bits, IO), idx_ptr(right, index_bits, IO),
                  lil + IO, ril + IO, idx_ptr(ranges, index_bits, 2 * NO), left32 + NO,
                  right32 + NO, parent_claim + NO, NO);
      node_seg[NO + j] = sg;
      leafpos32[NO + j] = -1;
      node_base[NO + j] = (int32_t)NO;
    }
    const int64_t node = NO + Ls - 1 + j;
    leafpos32[node] = (int32_t)g;  // near rows: the sets' leaves back to back
    node_base[node] = (int32_t)NO;
    leaf_base[g] = (int32_t)NO;
    store_idx(ranges, index_bits, 2 * node, load_idx(starts, index_bits, g));
    store_idx(ranges, index_bits, 2 * node + 1, load_idx(ends, index_bits, g) - 1);
    left32[node] = -1;
    right32[node] = -1;
    node_seg[node] = sg;
  }
}

__global__ void k_seg_parent_decode(const int32_t* __restrict__ claim,
                                    const int32_t* __restrict__ node_seg,
                                    const int64_t* __restrict__ leaf_off, int64_t total,
                                    int index_bits, void* parent, int32_t* __restrict__ parent32) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t sg = node_seg[k];
    const int64_t a = leaf_off[sg], Ls = leaf_off[sg + 1] - a, NO = 2 * a - sg, ni = Ls - 1;
    const int32_t c = claim[k];
    const int64_t p = c < 0 ? -1 : (c >= ni ? c - ni : c);
    store_idx(parent, index_bits, k, p);
    parent32[k] = p < 0 ? -1 : (int32_t)(NO + p);
  }
}

__global__ void k_seg_check_wellformed(const int32_t* __restrict__ parent32,
                                       const int32_t* __restrict__ left32,
                                       const int32_t* __restrict__ right32,
                                       const int32_t* __restrict__ node_seg,
                                       const int64_t* __restrict__ leaf_off, int64_t total,
                                       uint32_t* __restrict__ seg_flags,
                                       uint32_t* __restrict__ tree_flags) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t sg = node_seg[k];
    const int64_t a = leaf_off[sg], Ls = leaf_off[sg + 1] - a, NO = 2 * a - sg;
    const int64_t x = k - NO;
    bool bad = x == 0 ? parent32[k] != -1 : parent32[k] < 0;
    if (x < Ls - 1)
      bad = bad || parent32[left32[k]] != (int32_t)k || parent32[right32[k]] != (int32_t)k;
    if (bad) {
      atomicOr(&seg_flags[sg], kFlagMalformed);
      atomicOr(tree_flags, kFlagMalformed);
    }
  }
}

// Levels of the forest (pointer doubling ran over all sets at once), the
// per-set level histograms and maxima, and (set, level) sort keys.  A node
// whose root is not its set's node 0 marks its set malformed.
__global__ void k_seg_depth_finish(const int32_t* __restrict__ sc0, const int32_t* __restrict__ d0,
                                   const int32_t* __restrict__ sc1, const int32_t* __restrict__ d1,
                                   int64_t total, const uint32_t* __restrict__ stop,
                                   uint32_t rounds, const int32_t* __restrict__ node_seg,
                                   const int64_t* __restrict__ leaf_off, int index_bits,
                                   void* node_level, int32_t* __restrict__ level32,
                                   uint64_t* __restrict__ level_keys,
                                   uint32_t* __restrict__ seg_hist,
                                   int32_t* __restrict__ seg_max, uint32_t* __restrict__ seg_flags,
                                   uint32_t* __restrict__ tree_flags) {
  const uint32_t r = *stop < rounds ? *stop : rounds;
  const int32_t* sc = (r & 1) ? sc1 : sc0;
  const int32_t* d = (r & 1) ? d1 : d0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t sg = node_seg[k];
    const int64_t NO = 2 * leaf_off[sg] - sg;
    const int32_t lv = d[k];
    store_idx(node_level, index_bits, k, lv);
    level32[k] = lv;
    const uint32_t klv = lv < 0 ? 0u : (lv > 0xFFFF ? 0xFFFFu : (uint32_t)lv);
    level_keys[k] = ((uint64_t)(uint32_t)sg << 16) | klv;
    if (lv >= 0 && lv < 64) atomicAdd(&seg_hist[(int64_t)sg * 64 + lv], 1u);
    atomicMax(&seg_max[sg], lv);
    if (sc[k] != (int32_t)NO) {
      atomicOr(&seg_flags[sg], kFlagMalformed);
      atomicOr(tree_flags, kFlagMalformed);
    }
  }
}

__global__ void k_seg_level_tables(const uint32_t* __restrict__ seg_hist,
                                   const int32_t* __restrict__ seg_max,
                                   const int64_t* __restrict__ leaf_off, int64_t S,
                                   int index_bits, void* level_offsets, void* num_levels) {
  for (int64_t sg = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; sg < S;
       sg += (int64_t)gridDim.x * blockDim.x) {
    // a one-leaf tree has the reference's literal table (_tree_impl.py:1052-1110)
    const bool single = leaf_off[sg + 1] - leaf_off[sg] == 1;
    int64_t acc = 0;
    store_idx(level_offsets, index_bits, sg * 65, 0);
    for (int l = 0; l < 64; ++l) {
      acc += seg_hist[sg * 64 + l];
      store_idx(level_offsets, index_bits, sg * 65 + l + 1, single ? (l == 0 ? 1 : 0) : acc);
    }
    int64_t nl = (int64_t)seg_max[sg] + 1;
    nl = nl < 1 ? 1 : (nl > 64 ? 64 : nl);
    store_idx(num_levels, index_bits, sg, nl);
  }
}

// nodes_by_level per set: local ids in the index dtype, global ids in nbl32.
__global__ void k_seg_nbl(const uint32_t* __restrict__ ids, const int32_t* __restrict__ node_seg,
                          const int64_t* __restrict__ leaf_off, int64_t total, int index_bits,
                          void* nbl, int32_t* __restrict__ nbl32) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t id = ids[k];
    const int32_t sg = node_seg[id];
    store_idx(nbl, index_bits, k, (int64_t)id - (2 * leaf_off[sg] - sg));
    nbl32[k] = (int32_t)id;
  }
}

}  // namespace

// Scratch layout of ygx_build_topology.
struct TopoScratch {
  uint32_t* status;
  uint32_t* tree_flags;
  int32_t* parent_claim;
  int32_t* sc[2];
  int32_t* d[2];
  uint32_t* changed;
  uint32_t* stop;
  uint32_t* level_hist;
  int32_t* max_level;
  uint64_t* level_keys;
  uint64_t* level_keys_sorted;
  uint32_t* nbl_u32;
  SortScratch sort;
};

static TopoScratch carve_topo(Arena& a, int64_t L) {
  const int64_t total = L > 0 ? 2 * L - 1 : 1;
  TopoScratch s;
  s.status = a.take<uint32_t>(64);
  s.tree_flags = a.take<uint32_t>(64);
  s.changed = a.take<uint32_t>(128);
  s.stop = a.take<uint32_t>(64);
  s.level_hist = a.take<uint32_t>(64);
  s.max_level = a.take<int32_t>(64);
  s.parent_claim = a.take<int32_t>(total);
  for (int b = 0; b < 2; ++b) { s.sc[b] = a.take<int32_t>(total); s.d[b] = a.take<int32_t>(total); }
  s.level_keys = a.take<uint64_t>(total);
  s.level_keys_sorted = a.take<uint64_t>(total);
  s.nbl_u32 = a.take<uint32_t>(total);
  s.sort = carve_sort_scratch(a, total, 2);
  return s;
}

}  // namespace ygx

extern "C" {

int ygx_pack_particles(const float* positions, const float* masses, int64_t n, void* packed,
                       cudaStream_t stream) {
  if (n < 1 || !positions || !masses || !packed ||
      (reinterpret_cast<uintptr_t>(packed) & 15u) != 0)
    return YGX_ERR_ARG;
  ygx::k_pack_particles<<<ygx::grid_for(n, 256), 256, 0, stream>>>(
      positions, masses, n, reinterpret_cast<float4*>(packed));
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

int ygx_reorder_packed(const void* packed, const uint32_t* order, int64_t n, int index_bits,
                       float* positions_sorted, float* masses_sorted, void* particle_indices,
                       void* inverse, cudaStream_t stream) {
  if (n < 1 || !order || !packed || (reinterpret_cast<uintptr_t>(packed) & 15u) != 0 ||
      (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  ygx::k_reorder_packed<<<ygx::grid_for((n + ygx::kReorderItems - 1) / ygx::kReorderItems,
                                         ygx::kReorderThreads),
                          ygx::kReorderThreads, 0, stream>>>(
      reinterpret_cast<const float4*>(packed), order, n, index_bits, positions_sorted,
      masses_sorted, particle_indices, inverse);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

int ygx_reorder(const float* positions, const float* masses, const uint32_t* order, int64_t n,
                int index_bits, float* positions_sorted, float* masses_sorted,
                void* particle_indices, void* inverse, cudaStream_t stream) {
  if (n < 1 || !order || (index_bits != 32 && index_bits != 64)) return YGX_ERR_ARG;
  ygx::k_reorder<<<ygx::grid_for((n + ygx::kReorderItems - 1) / ygx::kReorderItems,
                                  ygx::kReorderThreads),
                   ygx::kReorderThreads, 0, stream>>>(
      positions, masses, order, n, index_bits, positions_sorted, masses_sorted, particle_indices,
      inverse);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

int ygx_leaves_adaptive(const uint64_t* codes_sorted, int64_t n, int64_t leaf_size, int index_bits,
                        void* leaf_starts, void* leaf_ends, uint64_t* leaf_codes,
                        void* leaf_depths, cudaStream_t stream) {
  if (n < 1 || leaf_size < 1) return YGX_ERR_ARG;
  const int64_t L = (n + leaf_size - 1) / leaf_size;
  ygx::k_leaves_adaptive<<<ygx::grid_for(L, 256), 256, 0, stream>>>(
      codes_sorted, n, leaf_size, L, index_bits, leaf_starts, leaf_ends, leaf_codes, leaf_depths);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

int ygx_leaves_fixed(const uint64_t* codes_sorted, int64_t n, int depth, int index_bits,
                     void* leaf_starts, void* leaf_ends, uint64_t* leaf_codes, void* leaf_depths,
                     cudaStream_t stream) {
  if (n < 1 || depth < 1 || depth > 10) return YGX_ERR_ARG;
  const int64_t L = (int64_t)1 << (3 * depth);
  ygx::k_leaves_fixed<<<ygx::grid_for(L, 256), 256, 0, stream>>>(
      codes_sorted, n, depth, L, index_bits, leaf_starts, leaf_ends, leaf_codes, leaf_depths);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

size_t ygx_refine_workspace_size(int64_t num_buckets) {
  ygx::Arena a{nullptr, 0, 0};
  a.take<uint32_t>(64);
  a.take<int64_t>(num_buckets + 1);
  a.take<int64_t>(num_buckets + 1);
  a.take<int64_t>(ygx::scan_scratch_elems(num_buckets));
  return a.used + 256;
}

// Pass 1: per-bucket output counts and their exclusive scan; the total
// number of refined leaves is left at device address *total_out.
int ygx_refine_count(const float* positions_sorted, const uint64_t* codes_sorted,
                     const void* starts, const void* ends, const uint64_t* codes,
                     const void* depths, int64_t L, int current_depth, int max_refine_levels,
                     double aspect_threshold, int min_leaf_particles, int index_bits,
                     int64_t* total_out, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (L < 1 || ws_bytes < ygx_refine_workspace_size(L)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  uint32_t* status = a.take<uint32_t>(64);
  int64_t* counts = a.take<int64_t>(L + 1);
  int64_t* offsets = a.take<int64_t>(L + 1);
  int64_t* tmp = a.take<int64_t>(ygx::scan_scratch_elems(L));
  const int warps_per_block = 8;
  int grid = ygx::grid_for(L, warps_per_block, ygx::kNumSMs * 16);
  ygx::k_refine<false><<<grid, 32 * warps_per_block, 0, stream>>>(
      positions_sorted, codes_sorted, starts, ends, codes, depths, L, current_depth,
      max_refine_levels, aspect_threshold, min_leaf_particles, index_bits, counts, nullptr,
      nullptr, nullptr, nullptr, nullptr, status);
  YGX_CHECK_LAUNCH();
  int rc = ygx::exclusive_scan<int64_t>(counts, L, offsets, tmp, stream);
  if (rc) return rc;
  if (cudaMemcpyAsync(total_out, offsets + L, sizeof(int64_t), cudaMemcpyDeviceToDevice,
                      stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  return YGX_OK;
}

// Pass 2: emit the refined leaves (same arguments as pass 1, same workspace).
int ygx_refine_emit(const float* positions_sorted, const uint64_t* codes_sorted,
                    const void* starts, const void* ends, const uint64_t* codes,
                    const void* depths, int64_t L, int current_depth, int max_refine_levels,
                    double aspect_threshold, int min_leaf_particles, int index_bits,
                    void* out_starts, void* out_ends, uint64_t* out_codes, void* out_depths,
                    void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (L < 1 || ws_bytes < ygx_refine_workspace_size(L)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  uint32_t* status = a.take<uint32_t>(64);
  a.take<int64_t>(L + 1);
  int64_t* offsets = a.take<int64_t>(L + 1);
  const int warps_per_block = 8;
  int grid = ygx::grid_for(L, warps_per_block, ygx::kNumSMs * 16);
  ygx::k_refine<true><<<grid, 32 * warps_per_block, 0, stream>>>(
      positions_sorted, codes_sorted, starts, ends, codes, depths, L, current_depth,
      max_refine_levels, aspect_threshold, min_leaf_particles, index_bits, nullptr, offsets,
      out_starts, out_ends, out_codes, out_depths, status);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

size_t ygx_topology_workspace_size(int64_t num_leaves) {
  ygx::Arena a{nullptr, 0, 0};
  ygx::carve_topo(a, num_leaves);
  return a.used + 256;
}

// Karras topology + levels for L >= 2 leaves (total = 2L - 1 nodes).
// Outputs in the index dtype: parent (total), left/right (L-1), node_ranges
// (total x 2), node_level (total), level_offsets (65), nodes_by_level
// (total), num_levels (1); bool flags (L-1); int32 traversal copies
// parent32/left32/right32/level32 (total, -1 children for leaves) and
// nbl32 (total).  tree_flags_out (device, 1 word) receives kFlagMalformed
// when the parent array and the child arrays disagree.
int ygx_build_topology(const uint64_t* leaf_codes, const void* leaf_starts, const void* leaf_ends,
                       int64_t L, int index_bits, void* parent, void* left, void* right,
                       uint8_t* left_is_leaf, uint8_t* right_is_leaf, void* node_ranges,
                       void* node_level, void* level_offsets, void* nodes_by_level,
                       void* num_levels, int32_t* parent32, int32_t* left32, int32_t* right32,
                       int32_t* level32, int32_t* nbl32, uint32_t* tree_flags_out, void* ws,
                       size_t ws_bytes, cudaStream_t stream) {
  if (L < 2 || (index_bits != 32 && index_bits != 64)) return YGX_ERR_ARG;
  if ((2 * L - 1) >= (int64_t)INT32_MAX / 2) return YGX_ERR_ARG;
  if (ws_bytes < ygx_topology_workspace_size(L)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::TopoScratch s = ygx::carve_topo(a, L);
  const int64_t total = 2 * L - 1, ni = L - 1;
  // flags, changed, stop, hist, max_level are contiguous: one memset.
  if (cudaMemsetAsync(s.tree_flags, 0, (char*)(s.max_level + 64) - (char*)s.tree_flags, stream) !=
      cudaSuccess)
    return YGX_ERR_CUDA;
  if (cudaMemsetAsync(s.stop, 0xFF, 64 * sizeof(uint32_t), stream) != cudaSuccess) return YGX_ERR_CUDA;
  if (cudaMemsetAsync(s.parent_claim, 0xFF, total * sizeof(int32_t), stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  ygx::k_karras<<<ygx::grid_for(L, 256), 256, 0, stream>>>(
      leaf_codes, leaf_starts, leaf_ends, L, index_bits, left, right, left_is_leaf, right_is_leaf,
      node_ranges, left32, right32, s.parent_claim);
  YGX_CHECK_LAUNCH();
  ygx::k_leaf_ranges<<<ygx::grid_for(L, 256), 256, 0, stream>>>(leaf_starts, leaf_ends, L,
                                                                index_bits, node_ranges, left32,
                                                                right32);
  YGX_CHECK_LAUNCH();
  ygx::k_parent_decode<<<ygx::grid_for(total, 256), 256, 0, stream>>>(s.parent_claim, total, ni,
                                                                      index_bits, parent, parent32);
  YGX_CHECK_LAUNCH();
  ygx::k_check_wellformed<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      parent32, left32, right32, total, ni, s.tree_flags);
  YGX_CHECK_LAUNCH();
  // Levels by pointer doubling: bit_length(total) + 1 rounds.
  int bl = 0;
  while (((int64_t)1 << bl) <= total) ++bl;
  const int rounds = bl + 1 > 1 ? bl + 1 : 1;
  ygx::k_depth_init<<<ygx::grid_for(total, 256), 256, 0, stream>>>(parent32, total, s.sc[0], s.d[0]);
  YGX_CHECK_LAUNCH();
  for (int r = 0; r < rounds; ++r) {
    ygx::k_depth_round<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
        s.sc[r & 1], s.d[r & 1], s.sc[(r + 1) & 1], s.d[(r + 1) & 1], total, r, s.changed, s.stop);
    YGX_CHECK_LAUNCH();
  }
  ygx::k_depth_finish<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      s.sc[0], s.d[0], s.sc[1], s.d[1], total, s.stop, (uint32_t)rounds, index_bits, node_level,
      level32, s.level_keys, s.level_hist, s.max_level, s.tree_flags);
  YGX_CHECK_LAUNCH();
  ygx::k_level_tables<<<1, 32, 0, stream>>>(s.level_hist, s.max_level, index_bits, level_offsets,
                                            num_levels);
  YGX_CHECK_LAUNCH();
  // nodes_by_level: stable argsort of node_level (levels < 2^16).
  int rc = ygx::onesweep_sort(s.level_keys, nullptr, total, 0, 16, s.level_keys_sorted, s.nbl_u32,
                              s.sort, false, s.status, stream);
  if (rc) return rc;
  ygx::k_u32_to_index<<<ygx::grid_for(total, 256), 256, 0, stream>>>(s.nbl_u32, total, index_bits,
                                                                     nodes_by_level, nbl32);
  YGX_CHECK_LAUNCH();
  if (tree_flags_out &&
      cudaMemcpyAsync(tree_flags_out, s.tree_flags, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                      stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  return YGX_OK;
}


// ---- batched sets -------------------------------------------------------------

// Leaf offsets of S sets (leaf_off: S + 1 int64, device): ceil(n_s /
// leaf_size) adaptive leaves per set.  *total_leaves_out (host) = their sum.
// Synchronizes the stream.
int ygx_batch_leaf_offsets(const int64_t* offsets, int64_t S, int64_t leaf_size,
                           int64_t* leaf_off, int64_t* total_leaves_out, void* ws,
                           size_t ws_bytes, cudaStream_t stream) {
  if (S < 1 || leaf_size < 1 || !offsets || !leaf_off || !total_leaves_out) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  int32_t* cnt = a.take<int32_t>(S);
  int64_t* tmp = a.take<int64_t>(ygx::scan_scratch_elems(S));
  if (a.used > ws_bytes) return YGX_ERR_ARG;
  ygx::k_seg_leaf_counts<<<ygx::grid_for(S, 256), 256, 0, stream>>>(offsets, S, leaf_size, cnt);
  YGX_CHECK_LAUNCH();
  int rc = ygx::exclusive_scan<int32_t>(cnt, S, leaf_off, tmp, stream);
  if (rc) return rc;
  if (cudaMemcpyAsync(total_leaves_out, leaf_off + S, sizeof(int64_t), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  return YGX_OK;
}

size_t ygx_batch_leaf_offsets_workspace_size(int64_t S) {
  ygx::Arena a{nullptr, 0, 0};
  a.take<int32_t>(S > 0 ? S : 1);
  a.take<int64_t>(ygx::scan_scratch_elems(S > 0 ? S : 1));
  return a.used + 256;
}

// Positions / masses in the sets' sorted order (ygx_batch_encode_sort's
// order and seg_sorted), particle_indices and inverse local to each set.
int ygx_batch_reorder(const float* positions, const float* masses, const uint32_t* order,
                      const int32_t* seg_sorted, const int64_t* offsets, int64_t n, int index_bits,
                      float* positions_sorted, float* masses_sorted, void* particle_indices,
                      void* inverse, cudaStream_t stream) {
  if (n < 1 || !positions || !order || !seg_sorted || !offsets || !positions_sorted ||
      (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  ygx::k_seg_reorder<<<ygx::grid_for(n, 256), 256, 0, stream>>>(
      positions, masses, order, seg_sorted, offsets, n, index_bits, positions_sorted,
      masses_sorted, particle_indices, inverse);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

// Leaf partitions of every set (local particle ranges [start, end), leaf
// codes, depths -1) and leaf_seg (int32, set of each global leaf).
int ygx_batch_leaves(const uint64_t* codes_sorted, const int64_t* offsets, const int64_t* leaf_off,
                     int64_t S, int64_t total_leaves, int64_t leaf_size, int index_bits,
                     void* leaf_starts, void* leaf_ends, uint64_t* leaf_codes, void* leaf_depths,
                     int32_t* leaf_seg, cudaStream_t stream) {
  if (S < 1 || total_leaves < S || leaf_size < 1 || (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  ygx::k_seg_leaves<<<ygx::grid_for(total_leaves, 256), 256, 0, stream>>>(
      codes_sorted, offsets, leaf_off, S, total_leaves, leaf_size, index_bits, leaf_starts,
      leaf_ends, leaf_codes, leaf_depths, leaf_seg);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

static ygx::TopoScratch carve_seg_topo(ygx::Arena& a, int64_t total, int64_t S,
                                       uint32_t** seg_hist, int32_t** seg_max,
                                       int32_t** node_seg_tmp) {
  ygx::TopoScratch s;
  s.status = a.take<uint32_t>(64);
  s.tree_flags = a.take<uint32_t>(64);
  s.changed = a.take<uint32_t>(128);
  s.stop = a.take<uint32_t>(64);
  s.level_hist = a.take<uint32_t>(64);
  s.max_level = a.take<int32_t>(64);
  *seg_hist = a.take<uint32_t>((size_t)S * 64);
  *seg_max = a.take<int32_t>(S);
  s.parent_claim = a.take<int32_t>(total);
  for (int b = 0; b < 2; ++b) { s.sc[b] = a.take<int32_t>(total); s.d[b] = a.take<int32_t>(total); }
  s.level_keys = a.take<uint64_t>(total);
  s.level_keys_sorted = a.take<uint64_t>(total);
  s.nbl_u32 = a.take<uint32_t>(total);
  *node_seg_tmp = nullptr;
  s.sort = ygx::carve_sort_scratch(a, total, 4);
  return s;
}

size_t ygx_batch_topology_workspace_size(int64_t total_leaves, int64_t S) {
  ygx::Arena a{nullptr, 0, 0};
  uint32_t* h;
  int32_t* m;
  int32_t* t;
  const int64_t total = total_leaves > S ? 2 * total_leaves - S : 1;
  carve_seg_topo(a, total, S > 0 ? S : 1, &h, &m, &t);
  return a.used + 256;
}

// The forest of S Karras trees (set s: leaves leaf_off[s] .. leaf_off[s+1],
// nodes at NO_s = 2 leaf_off[s] - s; total = 2 total_leaves - S).  Per-set
// outputs hold local values as ygx_build_topology gives them for the set
// alone: parent / node_ranges / node_level / nodes_by_level (total), left /
// right / flags (total_leaves - S), level_offsets (S x 65), num_levels (S).
// parent32 / left32 / right32 / nbl32 hold global node ids, node_seg32 the
// set of every node, leafpos32 the near-row position of every leaf (the
// sets' leaves back to back; -1 for internal nodes), node_base32 / leaf_base32
// the first node id of the set of every node / leaf, seg_flags (S)
// YGX_FLAG_MALFORMED per set and tree_flags_out (1 word) their union.
int ygx_batch_build_topology(const uint64_t* leaf_codes, const void* leaf_starts,
                             const void* leaf_ends, const int64_t* leaf_off,
                             const int32_t* leaf_seg, int64_t S, int64_t total_leaves,
                             int index_bits, void* parent, void* left, void* right,
                             uint8_t* left_is_leaf, uint8_t* right_is_leaf, void* node_ranges,
                             void* node_level, void* level_offsets, void* nodes_by_level,
                             void* num_levels, int32_t* parent32, int32_t* left32,
                             int32_t* right32, int32_t* level32, int32_t* nbl32,
                             int32_t* node_seg32, int32_t* leafpos32, int32_t* node_base32,
                             int32_t* leaf_base32, uint32_t* seg_flags, uint32_t* tree_flags_out,
                             void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (S < 1 || S > (1 << 16) || total_leaves < S || (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  const int64_t total = 2 * total_leaves - S;
  if (total >= (int64_t)INT32_MAX / 2) return YGX_ERR_ARG;
  if (ws_bytes < ygx_batch_topology_workspace_size(total_leaves, S)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  uint32_t* seg_hist;
  int32_t* seg_max;
  int32_t* unused;
  ygx::TopoScratch s = carve_seg_topo(a, total, S, &seg_hist, &seg_max, &unused);
  // flags, changed, stop, hist, max_level, seg_hist, seg_max are contiguous
  if (cudaMemsetAsync(s.tree_flags, 0, (char*)(seg_max + S) - (char*)s.tree_flags, stream) !=
          cudaSuccess ||
      cudaMemsetAsync(s.stop, 0xFF, 64 * sizeof(uint32_t), stream) != cudaSuccess ||
      cudaMemsetAsync(s.parent_claim, 0xFF, total * sizeof(int32_t), stream) != cudaSuccess ||
      cudaMemsetAsync(seg_flags, 0, S * sizeof(uint32_t), stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  ygx::k_seg_karras<<<ygx::grid_for(total_leaves, 256), 256, 0, stream>>>(
      leaf_codes, leaf_starts, leaf_ends, leaf_off, leaf_seg, total_leaves, index_bits, left,
      right, left_is_leaf, right_is_leaf, node_ranges, left32, right32, s.parent_claim,
      node_seg32, leafpos32, node_base32, leaf_base32);
  YGX_CHECK_LAUNCH();
  ygx::k_seg_parent_decode<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      s.parent_claim, node_seg32, leaf_off, total, index_bits, parent, parent32);
  YGX_CHECK_LAUNCH();
  ygx::k_seg_check_wellformed<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      parent32, left32, right32, node_seg32, leaf_off, total, seg_flags, s.tree_flags);
  YGX_CHECK_LAUNCH();
  int bl = 0;
  while (((int64_t)1 << bl) <= total) ++bl;
  const int rounds = bl + 1;
  ygx::k_depth_init<<<ygx::grid_for(total, 256), 256, 0, stream>>>(parent32, total, s.sc[0], s.d[0]);
  YGX_CHECK_LAUNCH();
  for (int r = 0; r < rounds; ++r) {
    ygx::k_depth_round<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
        s.sc[r & 1], s.d[r & 1], s.sc[(r + 1) & 1], s.d[(r + 1) & 1], total, r, s.changed, s.stop);
    YGX_CHECK_LAUNCH();
  }
  ygx::k_seg_depth_finish<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      s.sc[0], s.d[0], s.sc[1], s.d[1], total, s.stop, (uint32_t)rounds, node_seg32, leaf_off,
      index_bits, node_level, level32, s.level_keys, seg_hist, seg_max, seg_flags, s.tree_flags);
  YGX_CHECK_LAUNCH();
  ygx::k_seg_level_tables<<<ygx::grid_for(S, 128), 128, 0, stream>>>(
      seg_hist, seg_max, leaf_off, S, index_bits, level_offsets, num_levels);
  YGX_CHECK_LAUNCH();
  // nodes_by_level: stable sort by (set, level); sets < 2^16, levels < 2^16
  int rc = ygx::onesweep_sort(s.level_keys, nullptr, total, 0, 32, s.level_keys_sorted, s.nbl_u32,
                              s.sort, false, s.status, stream);
  if (rc) return rc;
  ygx::k_seg_nbl<<<ygx::grid_for(total, 256), 256, 0, stream>>>(s.nbl_u32, node_seg32, leaf_off,
                                                                total, index_bits,
                                                                nodes_by_level, nbl32);
  YGX_CHECK_LAUNCH();
  if (tree_flags_out &&
      cudaMemcpyAsync(tree_flags_out, s.tree_flags, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                      stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  return YGX_OK;
}

}  // extern "C"
