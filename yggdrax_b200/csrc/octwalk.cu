// Native octree walk: the dual-tree walk in explicit octree cell space
// (_dual_tree_walk_octree_impl, yggdrax/_interactions_impl.py:1908-2597),
// behind build_octree_native_far_pairs (:5556-5634) and
// build_octree_native_neighbor_lists (:5637-5717); and the cell box geometry
// those walks use (compute_explicit_octree_box_geometry,
// yggdrax/octree.py:422-476).
//
// The walk is breadth first from (root, root).  Each generation is a stable
// compaction (as the reference's cumsum pushes): one kernel evaluates every
// pair (MAC on the box centres and extents, accept / near / refine, split
// rule, number of children), two device-wide scans give every child and
// every accepted / near pair its slot, a second kernel writes the next
// wavefront and the pair log, and a one-thread kernel advances the
// counters.  The log of a generation holds its accepted pairs twice: first
// every pair as (row of the first cell, second cell) in wavefront order,
// then every pair as (row of the second cell, first cell) -- the
// reference's fwd and bwd blocks (:2243-2394).  A stable sort of the whole
// log by row therefore yields every row in (generation, block, wavefront)
// order, the reference's row order up to the order inside one block, which
// the reference leaves to an unstable argsort (:813-873).
#include "common.cuh"
#include "scan.cuh"

namespace ygx {

namespace {

constexpr uint32_t kOctFarOver = 1u << 0;    // a far row exceeded its capacity
constexpr uint32_t kOctNearOver = 1u << 1;   // a near row exceeded its capacity
constexpr uint32_t kOctQueueOver = 1u << 2;  // more children than the queue holds
constexpr uint32_t kOctBadInput = 1u << 3;   // a cell id out of range
constexpr uint32_t kOctWfShort = 1u << 4;    // children exceed the wavefront buffer
constexpr uint32_t kOctLogShort = 1u << 5;   // the pair log was too short (walk continues)
constexpr int kOctMaxGens = 1 << 16;

struct OctCtl {
  long long size;      // pairs in the current wavefront
  long long far_n;     // far log entries so far (2 per accepted pair)
  long long near_n;    // near log entries so far (2 per near pair)
  unsigned long long accept;  // decisions
  unsigned long long nearc;
  unsigned long long refine;
  long long wf_need;   // largest number of children of a generation
  unsigned int flags;
  unsigned int gens;
};

struct OctParams {
  const int32_t* children;     // [M][8] octant slots, -1 where empty
  const int32_t* child_count;  // [M]
  const float* centers;        // [M][3]
  const float* radii;          // [M]
  const float* max_extents;    // [M]
  const uint8_t* leaf;         // [M] leaf test of the node space in use
  const int32_t* far_row;      // [M] row key of a cell in the far log, or null
  const int32_t* near_row;     // [M] row key of a cell in the near log (-1: none), or null
  int32_t* far_cnt;            // [M]
  int32_t* near_cnt;           // [near rows]
  int64_t M;
  float theta_sq;
  float theta;
  float scale;                 // dehnen radius scale
  int mac;                     // 0 bh, 1 dehnen, 2 engblom
  int64_t far_cap;             // per-row capacities
  int64_t near_cap;
};

__device__ __forceinline__ float oct_ext(const OctParams& p, int32_t n) {
  // dehnen / engblom: box radius (dehnen scaled); bh: box max extent
  return p.mac == 0 ? p.max_extents[n] : (p.mac == 1 ? __fmul_rn(p.scale, p.radii[n]) : p.radii[n]);
}

// Children of a refined pair in _octree_refine_pairs_single order
// (:106-165): the first child_count octant slots of the split side(s), -1
// slots skipped.  kind: 1 both sides of the diagonal (a <= b), 2 both sides
// (target-major), 3 target only, 4 source only.  Calls f(k, x, y) for the
// k-th kept child (x, y) and returns the number kept.
template <typename F>
__device__ __forceinline__ int oct_children(const OctParams& p, int kind, int32_t t, int32_t s,
                                            F&& f) {
  int k = 0;
  const int32_t* ct = p.children + (int64_t)t * 8;
  const int32_t* cs = p.children + (int64_t)s * 8;
  const int nt = p.child_count[t], ns = p.child_count[s];
  if (kind == 1) {
    for (int a = 0; a < nt && a < 8; ++a)
      for (int b = a; b < nt && b < 8; ++b)
        if (ct[a] >= 0 && ct[b] >= 0) f(k++, ct[a], ct[b]);
  } else if (kind == 2) {
    for (int a = 0; a < nt && a < 8; ++a)
      for (int b = 0; b < ns && b < 8; ++b)
        if (ct[a] >= 0 && cs[b] >= 0) f(k++, ct[a], cs[b]);
  } else if (kind == 3) {
    for (int a = 0; a < nt && a < 8; ++a)
      if (ct[a] >= 0) f(k++, ct[a], s);
  } else if (kind == 4) {
    for (int b = 0; b < ns && b < 8; ++b)
      if (cs[b] >= 0) f(k++, t, cs[b]);
  }
  return k;
}

__global__ void k_oct_eval(const int32_t* __restrict__ cur_t, const int32_t* __restrict__ cur_s,
                           int64_t size, OctParams p, int32_t* __restrict__ nchild,
                           uint8_t* __restrict__ kind, int64_t* __restrict__ emit,
                           OctCtl* __restrict__ ctl) {
  unsigned long long n_acc = 0, n_near = 0, n_ref = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t t = cur_t[i], s = cur_s[i];
    int nc = 0, kd = 0;
    long long em = 0;
    if (t >= 0 && s >= 0 && t < p.M && s < p.M) {
      // delta = centers[t] - centers[s]; squares summed in written order
      const float dx = __fsub_rn(p.centers[3 * t], p.centers[3 * s]);
      const float dy = __fsub_rn(p.centers[3 * t + 1], p.centers[3 * s + 1]);
      const float dz = __fsub_rn(p.centers[3 * t + 2], p.centers[3 * s + 2]);
      const float d2 =
          __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
      const float et = oct_ext(p, t), es = oct_ext(p, s);
      bool ok;
      if (p.mac == 2) {
        const float big = fmaxf(et, es), small = fminf(et, es);
        const float lhs = __fadd_rn(big, __fmul_rn(p.theta, small));
        ok = __fmul_rn(lhs, lhs) <= __fmul_rn(p.theta_sq, d2);
      } else {
        const float sm = __fadd_rn(et, es);
        ok = __fmul_rn(sm, sm) <= __fmul_rn(p.theta_sq, d2);
      }
      const bool diff = t != s;
      const bool accept = diff && d2 > 0.0f && ok;
      const bool tl = p.leaf[t] != 0, sl = p.leaf[s] != 0;
      const bool is_near = !accept && tl && sl && diff;
      const bool refine = !accept && !is_near;
      const bool same = !diff;
      const bool split_t = refine && !tl && (same || sl || et >= es);
      const bool split_s = refine && !sl && (same || tl || es > et);
      kd = split_t && split_s ? (same ? 1 : 2) : split_t ? 3 : split_s ? 4 : 0;
      if (kd) nc = oct_children(p, kd, t, s, [](int, int32_t, int32_t) {});
      em = ((accept && p.far_row) ? 1ll : 0ll) | (((is_near && p.near_row) ? 1ll : 0ll) << 32);
      // decisions (all three kinds counted, collected or not)
      n_acc += accept ? 1 : 0;
      n_near += is_near ? 1 : 0;
      n_ref += refine ? 1 : 0;
    } else {
      atomicOr(&ctl->flags, kOctBadInput);
    }
    nchild[i] = nc;
    kind[i] = (uint8_t)kd;
    emit[i] = em;
  }
  for (int o = 16; o > 0; o >>= 1) {
    n_acc += __shfl_xor_sync(0xffffffffu, n_acc, o);
    n_near += __shfl_xor_sync(0xffffffffu, n_near, o);
    n_ref += __shfl_xor_sync(0xffffffffu, n_ref, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (n_acc) atomicAdd(&ctl->accept, n_acc);
    if (n_near) atomicAdd(&ctl->nearc, n_near);
    if (n_ref) atomicAdd(&ctl->refine, n_ref);
  }
}

__global__ void k_oct_emit(const int32_t* __restrict__ cur_t, const int32_t* __restrict__ cur_s,
                           int64_t size, OctParams p, const uint8_t* __restrict__ kind,
                           const int64_t* __restrict__ emit, const int64_t* __restrict__ child_off,
                           const int64_t* __restrict__ emit_off, const OctCtl* __restrict__ ctl,
                           int64_t wf_room, int32_t* __restrict__ nxt_t,
                           int32_t* __restrict__ nxt_s, int64_t log_cap,
                           uint64_t* __restrict__ far_key, uint32_t* __restrict__ far_val,
                           uint64_t* __restrict__ near_key, uint32_t* __restrict__ near_val,
                           unsigned int* __restrict__ flags) {
  const long long far_n = ctl->far_n, near_n = ctl->near_n;
  const long long tot = emit_off[size];
  const long long n_acc = tot & 0xffffffffll, n_near = tot >> 32;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t t = cur_t[i], s = cur_s[i];
    const long long em = emit[i];
    if (em & 1ll) {
      const long long r = emit_off[i] & 0xffffffffll;
      const long long fwd = far_n + r, bwd = far_n + n_acc + r;
      if (bwd < log_cap) {
        far_key[fwd] = (uint64_t)(uint32_t)p.far_row[t];
        far_val[fwd] = (uint32_t)s;
        far_key[bwd] = (uint64_t)(uint32_t)p.far_row[s];
        far_val[bwd] = (uint32_t)t;
      } else {
        atomicOr(flags, kOctLogShort);
      }
      if ((int64_t)atomicAdd(&p.far_cnt[t], 1) >= p.far_cap) atomicOr(flags, kOctFarOver);
      if ((int64_t)atomicAdd(&p.far_cnt[s], 1) >= p.far_cap) atomicOr(flags, kOctFarOver);
    }
    if (em >> 32) {
      const long long r = emit_off[i] >> 32;
      const long long fwd = near_n + r, bwd = near_n + n_near + r;
      const int32_t rt = p.near_row[t], rs = p.near_row[s];
      if (rt < 0 || rs < 0) {
        atomicOr(flags, kOctBadInput);
      } else {
        if (bwd < log_cap) {
          near_key[fwd] = (uint64_t)(uint32_t)rt;
          near_val[fwd] = (uint32_t)s;
          near_key[bwd] = (uint64_t)(uint32_t)rs;
          near_val[bwd] = (uint32_t)t;
        } else {
          atomicOr(flags, kOctLogShort);
        }
        if ((int64_t)atomicAdd(&p.near_cnt[rt], 1) >= p.near_cap) atomicOr(flags, kOctNearOver);
        if ((int64_t)atomicAdd(&p.near_cnt[rs], 1) >= p.near_cap) atomicOr(flags, kOctNearOver);
      }
    }
    const int kd = kind[i];
    if (kd == 0) continue;
    const int64_t base = child_off[i];
    oct_children(p, kd, t, s, [&](int k, int32_t x, int32_t y) {
      const int64_t slot = base + k;
      if (slot < wf_room) {
        nxt_t[slot] = x < y ? x : y;
        nxt_s[slot] = x < y ? y : x;
      }
    });
  }
}

// Counters after a generation: the log grows by both blocks, the wavefront
// keeps its first `queue` children (flagged when there were more), and a
// generation with more children than the wavefront buffer holds asks for a
// larger buffer.
__global__ void k_oct_advance(OctCtl* __restrict__ ctl, const int64_t* __restrict__ child_off,
                              const int64_t* __restrict__ emit_off, int64_t size, int64_t queue,
                              int64_t wf_room, const unsigned int* __restrict__ flags) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const long long children = child_off[size];
  const long long et = emit_off[size];
  ctl->far_n += 2 * (et & 0xffffffffll);
  ctl->near_n += 2 * (et >> 32);
  ctl->flags |= *flags;
  const long long kept = children < queue ? children : queue;
  if (children > queue) ctl->flags |= kOctQueueOver;
  if (kept > wf_room) ctl->flags |= kOctWfShort;
  if (kept > ctl->wf_need) ctl->wf_need = kept;
  ctl->size = kept;
  ctl->gens += 1;
}

__global__ void k_oct_i32(const void* __restrict__ in, int index_bits, int64_t n,
                          int32_t* __restrict__ out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    out[k] = (int32_t)load_idx(in, index_bits, k);
}

// Every third bit of a 64-bit word (the inverse of the Morton spread), by
// the standard mask-and-shift compaction.
__device__ __forceinline__ uint64_t compact3(uint64_t x) {
  x &= 0x1249249249249249ull;
  x = (x ^ (x >> 2)) & 0x10C30C30C30C30C3ull;
  x = (x ^ (x >> 4)) & 0x100F00F00F00F00Full;
  x = (x ^ (x >> 8)) & 0x001F0000FF0000FFull;
  x = (x ^ (x >> 16)) & 0x001F00000000FFFFull;
  x = (x ^ (x >> 32)) & 0x00000000001FFFFFull;
  return x;
}

// compute_explicit_octree_box_geometry (octree.py:422-476), fp32 with every
// operation rounded: cell = domain / 2^depth, mins = bmin + cell * index,
// maxs = mins + cell, centre 0.5 (mins + maxs), half 0.5 (maxs - mins),
// radius sqrt((h0^2 + h1^2) + h2^2), max extent max(h); zeros on invalid
// cells.
__global__ void k_oct_box(const uint8_t* __restrict__ valid, const uint64_t* __restrict__ codes,
                          const void* __restrict__ depths, int index_bits, int64_t M,
                          float bx0, float by0, float bz0, float dx, float dy, float dz,
                          float* __restrict__ centers, float* __restrict__ half,
                          float* __restrict__ radii, float* __restrict__ max_extents) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    float c[3] = {0.f, 0.f, 0.f}, h[3] = {0.f, 0.f, 0.f}, r = 0.f, mx = 0.f;
    if (valid[k]) {
      int64_t d = load_idx(depths, index_bits, k);
      d = d < 0 ? 0 : (d > 21 ? 21 : d);
      const uint64_t sh = (uint64_t)(21 - d);
      const uint64_t code = codes[k];
      const uint64_t q[3] = {compact3(code) >> sh, compact3(code >> 1) >> sh,
                             compact3(code >> 2) >> sh};
      const float cnt = (float)(1ull << d);
      const float b0[3] = {bx0, by0, bz0}, dom[3] = {dx, dy, dz};
      for (int a = 0; a < 3; ++a) {
        const float cell = __fdiv_rn(dom[a], cnt);
        const float lo = __fadd_rn(b0[a], __fmul_rn(cell, (float)q[a]));
        const float hi = __fadd_rn(lo, cell);
        c[a] = __fmul_rn(0.5f, __fadd_rn(lo, hi));
        h[a] = __fmul_rn(0.5f, __fsub_rn(hi, lo));
      }
      const float s = __fadd_rn(__fadd_rn(__fmul_rn(h[0], h[0]), __fmul_rn(h[1], h[1])),
                                __fmul_rn(h[2], h[2]));
      r = __fsqrt_rn(s);
      mx = fmaxf(fmaxf(h[0], h[1]), h[2]);
    }
    for (int a = 0; a < 3; ++a) {
      centers[3 * k + a] = c[a];
      half[3 * k + a] = h[a];
    }
    radii[k] = r;
    max_extents[k] = mx;
  }
}

struct OctScratch {
  OctCtl* ctl;
  unsigned int* flags;
  int32_t* children;
  int32_t* child_count;
  int32_t* wf_t[2];
  int32_t* wf_s[2];
  int32_t* nchild;
  uint8_t* kind;
  int64_t* emit;
  int64_t* child_off;
  int64_t* emit_off;
  int64_t* tmp;
};

OctScratch carve_oct(Arena& a, int64_t M, int64_t wf) {
  OctScratch s;
  s.ctl = a.take<OctCtl>(1);
  s.flags = a.take<unsigned int>(16);
  s.children = a.take<int32_t>(8 * M);
  s.child_count = a.take<int32_t>(M);
  for (int k = 0; k < 2; ++k) {
    s.wf_t[k] = a.take<int32_t>(wf);
    s.wf_s[k] = a.take<int32_t>(wf);
  }
  s.nchild = a.take<int32_t>(wf);
  s.kind = a.take<uint8_t>(wf);
  s.emit = a.take<int64_t>(wf);
  s.child_off = a.take<int64_t>(wf + 1);
  s.emit_off = a.take<int64_t>(wf + 1);
  s.tmp = a.take<int64_t>(scan_scratch_elems(wf));
  return s;
}

}  // namespace

}  // namespace ygx

extern "C" {

int ygx_octree_box_geometry(const uint8_t* valid, const uint64_t* codes, const void* depths,
                            int index_bits, int64_t M, const float* bounds_min,
                            const float* bounds_max, float* centers, float* half_extents,
                            float* radii, float* max_extents, cudaStream_t stream) {
  if (M < 0 || (index_bits != 32 && index_bits != 64) || !bounds_min || !bounds_max)
    return YGX_ERR_ARG;
  if (M == 0) return YGX_OK;
  if (!valid || !codes || !depths || !centers || !half_extents || !radii || !max_extents)
    return YGX_ERR_ARG;
  // domain = bounds_max - bounds_min in fp32 (host values)
  const float d0 = bounds_max[0] - bounds_min[0], d1 = bounds_max[1] - bounds_min[1],
              d2 = bounds_max[2] - bounds_min[2];
  ygx::k_oct_box<<<ygx::grid_for(M, 256), 256, 0, stream>>>(
      valid, codes, depths, index_bits, M, bounds_min[0], bounds_min[1], bounds_min[2], d0, d1,
      d2, centers, half_extents, radii, max_extents);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

size_t ygx_octree_walk_workspace_size(int64_t M, int64_t wf_capacity) {
  ygx::Arena a{nullptr, 0, 0};
  ygx::carve_oct(a, M > 0 ? M : 1, wf_capacity > 0 ? wf_capacity : 1);
  return a.used + 256;
}

int ygx_octree_walk(const void* children, const void* child_counts, int index_bits, int64_t M,
                    const float* centers, const float* radii, const float* max_extents,
                    const uint8_t* leaf_mask, const int32_t* far_row, const int32_t* near_row,
                    int64_t near_rows, int64_t root, int mac, float theta,
                    float dehnen_radius_scale, int64_t max_pair_queue, int64_t wf_capacity,
                    int64_t far_row_cap, int64_t near_row_cap, int64_t log_capacity,
                    uint64_t* far_key, uint32_t* far_val, uint64_t* near_key,
                    uint32_t* near_val, int32_t* far_cnt, int32_t* near_cnt,
                    int64_t* stats_out, uint32_t* flags_out, void* ws, size_t ws_bytes,
                    cudaStream_t stream) {
  if (M < 1 || M > INT32_MAX || root < 0 || root >= M || mac < 0 || mac > 2 ||
      max_pair_queue < 1 || wf_capacity < 1 || log_capacity < 1 ||
      (index_bits != 32 && index_bits != 64) || !children || !child_counts || !centers ||
      !radii || !max_extents || !leaf_mask || !stats_out || !flags_out || !ws ||
      (!far_row && !near_row) || (far_row && (!far_key || !far_val || !far_cnt)) ||
      (near_row && (near_rows < 1 || !near_key || !near_val || !near_cnt)))
    return YGX_ERR_ARG;
  if (ws_bytes < ygx_octree_walk_workspace_size(M, wf_capacity)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::OctScratch s = ygx::carve_oct(a, M, wf_capacity);
  ygx::k_oct_i32<<<ygx::grid_for(8 * M, 256), 256, 0, stream>>>(children, index_bits, 8 * M,
                                                               s.children);
  YGX_CHECK_LAUNCH();
  ygx::k_oct_i32<<<ygx::grid_for(M, 256), 256, 0, stream>>>(child_counts, index_bits, M,
                                                           s.child_count);
  YGX_CHECK_LAUNCH();
  if ((far_cnt && cudaMemsetAsync(far_cnt, 0, sizeof(int32_t) * M, stream) != cudaSuccess) ||
      (near_cnt && cudaMemsetAsync(near_cnt, 0, sizeof(int32_t) * near_rows, stream) !=
                       cudaSuccess) ||
      cudaMemsetAsync(s.flags, 0, 16 * sizeof(unsigned int), stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  ygx::OctParams p;
  p.children = s.children;
  p.child_count = s.child_count;
  p.centers = centers;
  p.radii = radii;
  p.max_extents = max_extents;
  p.leaf = leaf_mask;
  p.far_row = far_row;
  p.near_row = near_row;
  p.far_cnt = far_cnt;
  p.near_cnt = near_cnt;
  p.M = M;
  // theta^2 in fp32 (jnp.asarray(theta, centers.dtype) ** 2); engblom's theta
  // is sqrt(theta^2)
  const float th = theta;
  p.theta_sq = th * th;
  p.theta = sqrtf(p.theta_sq);
  p.scale = dehnen_radius_scale;
  p.mac = mac;
  p.far_cap = far_row_cap;
  p.near_cap = near_row_cap;
  const int64_t Q = max_pair_queue < 4 ? 4 : max_pair_queue;
  ygx::OctCtl init{1, 0, 0, 0, 0, 0, 1, 0u, 0u};
  const int32_t r32 = (int32_t)root;
  if (cudaMemcpyAsync(s.ctl, &init, sizeof(init), cudaMemcpyHostToDevice, stream) != cudaSuccess ||
      cudaMemcpyAsync(s.wf_t[0], &r32, sizeof(r32), cudaMemcpyHostToDevice, stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(s.wf_s[0], &r32, sizeof(r32), cudaMemcpyHostToDevice, stream) !=
          cudaSuccess)
    return YGX_ERR_CUDA;
  const uint32_t stop = ygx::kOctFarOver | ygx::kOctNearOver | ygx::kOctQueueOver |
                        ygx::kOctBadInput | ygx::kOctWfShort;
  ygx::OctCtl h = init;
  int cur = 0;
  int rc = YGX_OK;
  while (h.size > 0 && (h.flags & stop) == 0) {
    if (h.gens >= (unsigned)ygx::kOctMaxGens) {
      rc = YGX_ERR_QUEUE_OVERFLOW;
      break;
    }
    const int64_t n = h.size;
    const int grid = ygx::grid_for(n, 256);
    ygx::k_oct_eval<<<grid, 256, 0, stream>>>(s.wf_t[cur], s.wf_s[cur], n, p, s.nchild, s.kind,
                                              s.emit, s.ctl);
    YGX_CHECK_LAUNCH();
    rc = ygx::exclusive_scan<int32_t>(s.nchild, n, s.child_off, s.tmp, stream);
    if (rc) break;
    rc = ygx::exclusive_scan<int64_t>(s.emit, n, s.emit_off, s.tmp, stream);
    if (rc) break;
    ygx::k_oct_emit<<<grid, 256, 0, stream>>>(
        s.wf_t[cur], s.wf_s[cur], n, p, s.kind, s.emit, s.child_off, s.emit_off, s.ctl,
        wf_capacity, s.wf_t[cur ^ 1], s.wf_s[cur ^ 1], log_capacity, far_key, far_val, near_key,
        near_val, s.flags);
    YGX_CHECK_LAUNCH();
    ygx::k_oct_advance<<<1, 32, 0, stream>>>(s.ctl, s.child_off, s.emit_off, n, Q, wf_capacity,
                                             s.flags);
    YGX_CHECK_LAUNCH();
    if (cudaMemcpyAsync(&h, s.ctl, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
      return YGX_ERR_CUDA;
    cur ^= 1;
  }
  stats_out[0] = h.far_n;
  stats_out[1] = h.near_n;
  stats_out[2] = (int64_t)h.accept;
  stats_out[3] = (int64_t)h.nearc;
  stats_out[4] = (int64_t)h.refine;
  stats_out[5] = (int64_t)h.gens;
  stats_out[6] = h.wf_need;
  flags_out[0] = h.flags;
  if (h.flags & ygx::kOctBadInput) return YGX_ERR_ARG;
  return rc;
}

}  // extern "C"
