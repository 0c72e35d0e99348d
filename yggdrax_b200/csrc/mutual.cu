// Canonical mutual dual-tree walk: every unordered node pair once
// (dual_tree_walk_mutual, yggdrax/_interactions_impl.py:6357-6560).
//
// The reference walks a fixed-capacity wavefront breadth-first and appends
// accepted / near pairs to flat lists in wavefront order, children in the
// order of their parents, each parent's children in the refinement order of
// _count_refine_pairs_single (:174-221).  Those orders are part of its
// output, so each generation here is a stable compaction: one kernel
// evaluates every pair (MAC, action, number of children), two device-wide
// exclusive scans give every child, far and near pair its slot, and a second
// kernel writes them.  A one-thread kernel then advances the counters with
// the reference's overflow rules; the host reads them once per generation
// (the reference's while-loop condition).
#include "common.cuh"
#include "scan.cuh"

namespace ygx {

namespace {

constexpr uint32_t kMutFarOver = 1u << 0;
constexpr uint32_t kMutNearOver = 1u << 1;
constexpr uint32_t kMutQueueOver = 1u << 2;
constexpr uint32_t kMutBadInput = 1u << 3;
constexpr int kMutMaxGens = 1 << 16;

struct MutualCtl {
  long long size;    // pairs in the current wavefront
  long long far_n;   // far pairs the flat list would hold (counted past its capacity)
  long long near_n;
  unsigned int flags;
  unsigned int pad;
};

// Refinement cases (kind): 0 none, 1 both children of a diagonal pair,
// 2 both sides of an off-diagonal pair, 3 the first node only, 4 the second
// node only.
__global__ void k_mut_eval(const int32_t* __restrict__ cur_a, const int32_t* __restrict__ cur_b,
                           int64_t size, const int32_t* __restrict__ left,
                           const float* __restrict__ centers, const float* __restrict__ radii,
                           int64_t total, float theta_sq, int32_t* __restrict__ nchild,
                           uint8_t* __restrict__ kind, int64_t* __restrict__ emit,
                           MutualCtl* __restrict__ ctl) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t sa = cur_a[i], sb = cur_b[i];
    int nc = 0, kd = 0;
    long long em = 0;
    if (sa >= 0 && sb >= 0 && sa < total && sb < total) {
      const bool a_leaf = left[sa] < 0, b_leaf = left[sb] < 0, same = sa == sb;
      // delta = centers[b] - centers[a]; sum of squares in written order
      const float dx = __fsub_rn(centers[3 * sb], centers[3 * sa]);
      const float dy = __fsub_rn(centers[3 * sb + 1], centers[3 * sa + 1]);
      const float dz = __fsub_rn(centers[3 * sb + 2], centers[3 * sa + 2]);
      const float d2 =
          __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
      const float ra = radii[sa], rb = radii[sb];
      const float rs = __fadd_rn(ra, rb);
      // theta * d > r_a + r_b, squared, strict; never for a self-pair
      const bool accept = !same && __fmul_rn(theta_sq, d2) > __fmul_rn(rs, rs);
      const bool both_leaf = a_leaf && b_leaf;
      const bool is_near = !accept && both_leaf && !same;
      const bool refine = !accept && !both_leaf;
      const bool split_a = refine && !a_leaf && (same || b_leaf || ra >= rb);
      const bool split_b = refine && !b_leaf && (same || a_leaf || rb > ra);
      if (split_a && split_b) {
        kd = same ? 1 : 2;
        nc = same ? 3 : 4;
      } else if (split_a) {
        kd = 3;
        nc = 2;
      } else if (split_b) {
        kd = 4;
        nc = 2;
      }
      em = (accept ? 1ll : 0ll) | ((is_near ? 1ll : 0ll) << 32);
    } else if (sa >= total || sb >= total) {
      atomicOr(&ctl->flags, kMutBadInput);
    }
    nchild[i] = nc;
    kind[i] = (uint8_t)kd;
    emit[i] = em;
  }
}

template <typename T>
__device__ __forceinline__ void put_pair(void* a, void* b, long long slot, long long va,
                                         long long vb) {
  reinterpret_cast<T*>(a)[slot] = (T)va;
  reinterpret_cast<T*>(b)[slot] = (T)vb;
}

// Children at child_off[i] + k (first `cap` of them kept, canonical
// (min, max) order), far / near pairs at the list counters + their prefix.
__global__ void k_mut_emit(const int32_t* __restrict__ cur_a, const int32_t* __restrict__ cur_b,
                           int64_t size, const int32_t* __restrict__ left,
                           const int32_t* __restrict__ right, const uint8_t* __restrict__ kind,
                           const int64_t* __restrict__ emit,
                           const int64_t* __restrict__ child_off,
                           const int64_t* __restrict__ emit_off, const MutualCtl* __restrict__ ctl,
                           int64_t cap, int32_t* __restrict__ nxt_a, int32_t* __restrict__ nxt_b,
                           int64_t far_cap, int64_t near_cap, int index_bits, void* far_a,
                           void* far_b, void* near_a, void* near_b) {
  const long long far_n = ctl->far_n, near_n = ctl->near_n;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t sa = cur_a[i], sb = cur_b[i];
    const long long em = emit[i];
    if (em & 1ll) {
      const long long slot = far_n + (emit_off[i] & 0xffffffffll);
      if (slot < far_cap) {
        if (index_bits == 32) put_pair<int32_t>(far_a, far_b, slot, sa, sb);
        else put_pair<int64_t>(far_a, far_b, slot, sa, sb);
      }
    }
    if (em >> 32) {
      const long long slot = near_n + (emit_off[i] >> 32);
      if (slot < near_cap) {
        if (index_bits == 32) put_pair<int32_t>(near_a, near_b, slot, sa, sb);
        else put_pair<int64_t>(near_a, near_b, slot, sa, sb);
      }
    }
    const int kd = kind[i];
    if (kd == 0) continue;
    int32_t ca[4], cb[4];
    int nc = 0;
    const int32_t al = left[sa] , ar = right[sa];
    const int32_t bl = sb >= 0 ? left[sb] : -1, br = sb >= 0 ? right[sb] : -1;
    if (kd == 1) {
      ca[0] = al; cb[0] = al;
      ca[1] = al; cb[1] = ar;
      ca[2] = ar; cb[2] = ar;
      nc = 3;
    } else if (kd == 2) {
      ca[0] = al; cb[0] = bl;
      ca[1] = al; cb[1] = br;
      ca[2] = ar; cb[2] = bl;
      ca[3] = ar; cb[3] = br;
      nc = 4;
    } else if (kd == 3) {
      ca[0] = al; cb[0] = sb;
      ca[1] = ar; cb[1] = sb;
      nc = 2;
    } else {
      ca[0] = sa; cb[0] = bl;
      ca[1] = sa; cb[1] = br;
      nc = 2;
    }
    const int64_t base = child_off[i];
    for (int k = 0; k < nc; ++k) {
      const int64_t slot = base + k;
      if (slot < cap) {
        nxt_a[slot] = ca[k] < cb[k] ? ca[k] : cb[k];
        nxt_b[slot] = ca[k] < cb[k] ? cb[k] : ca[k];
      }
    }
  }
}

// Counters and flags after a generation (the reference's _flat_append and
// push rules): a list overflows when any of this generation's pairs got a
// slot at or past its capacity; the wavefront keeps its first `cap` children.
__global__ void k_mut_advance(MutualCtl* __restrict__ ctl, const int64_t* __restrict__ child_off,
                              const int64_t* __restrict__ emit_off, int64_t size, int64_t cap,
                              int64_t far_cap, int64_t near_cap) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const long long children = child_off[size];
  const long long et = emit_off[size];
  const long long nf = et & 0xffffffffll, nn = et >> 32;
  if (nf > 0 && ctl->far_n + nf > far_cap) ctl->flags |= kMutFarOver;
  if (nn > 0 && ctl->near_n + nn > near_cap) ctl->flags |= kMutNearOver;
  ctl->far_n += nf;
  ctl->near_n += nn;
  if (children > cap) ctl->flags |= kMutQueueOver;
  ctl->size = children < cap ? children : cap;
}

__global__ void k_mut_children_i32(const void* __restrict__ in, int index_bits, int64_t n,
                                   int32_t* __restrict__ out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    out[k] = (int32_t)load_idx(in, index_bits, k);
}

struct MutualScratch {
  MutualCtl* ctl;
  int32_t* left;
  int32_t* right;
  int32_t* wf_a[2];
  int32_t* wf_b[2];
  int32_t* nchild;
  uint8_t* kind;
  int64_t* emit;
  int64_t* child_off;
  int64_t* emit_off;
  int64_t* tmp;
};

MutualScratch carve_mutual(Arena& a, int64_t total, int64_t cap) {
  MutualScratch s;
  s.ctl = a.take<MutualCtl>(1);
  s.left = a.take<int32_t>(total);
  s.right = a.take<int32_t>(total);
  for (int k = 0; k < 2; ++k) {
    s.wf_a[k] = a.take<int32_t>(cap);
    s.wf_b[k] = a.take<int32_t>(cap);
  }
  s.nchild = a.take<int32_t>(cap);
  s.kind = a.take<uint8_t>(cap);
  s.emit = a.take<int64_t>(cap);
  s.child_off = a.take<int64_t>(cap + 1);
  s.emit_off = a.take<int64_t>(cap + 1);
  s.tmp = a.take<int64_t>(scan_scratch_elems(cap));
  return s;
}

}  // namespace

}  // namespace ygx

extern "C" {

size_t ygx_mutual_walk_workspace_size(int64_t total, int64_t max_pair_queue) {
  ygx::Arena a{nullptr, 0, 0};
  ygx::carve_mutual(a, total > 0 ? total : 1, max_pair_queue > 0 ? max_pair_queue : 1);
  return a.used + 256;
}

int ygx_mutual_walk(const void* left_full, const void* right_full, int index_bits,
                    const float* centers, const float* radii, int64_t total, float theta,
                    int64_t root, int64_t max_pair_queue, int64_t far_cap, int64_t near_cap,
                    void* far_a, void* far_b, void* near_a, void* near_b, int64_t* counts_out,
                    uint32_t* flags_out, int* gens_out, void* ws, size_t ws_bytes,
                    cudaStream_t stream) {
  if (total < 1 || total > INT32_MAX || root < 0 || root >= total || max_pair_queue < 1 ||
      max_pair_queue > INT32_MAX || far_cap < 1 || near_cap < 1 ||
      (index_bits != 32 && index_bits != 64) || !left_full || !right_full || !centers ||
      !radii || !far_a || !far_b || !near_a || !near_b || !counts_out || !flags_out || !ws)
    return YGX_ERR_ARG;
  if (ws_bytes < ygx_mutual_walk_workspace_size(total, max_pair_queue)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::MutualScratch s = ygx::carve_mutual(a, total, max_pair_queue);
  const int64_t Q = max_pair_queue;
  // theta^2 in fp32 (jnp.asarray(theta, centers.dtype) ** 2)
  const float th = theta;
  const float theta_sq = th * th;
  const size_t isz = index_bits == 32 ? 4 : 8;
  // -1 everywhere in the flat lists (all-ones bytes), zero counters
  if (cudaMemsetAsync(far_a, 0xff, isz * far_cap, stream) != cudaSuccess ||
      cudaMemsetAsync(far_b, 0xff, isz * far_cap, stream) != cudaSuccess ||
      cudaMemsetAsync(near_a, 0xff, isz * near_cap, stream) != cudaSuccess ||
      cudaMemsetAsync(near_b, 0xff, isz * near_cap, stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  ygx::k_mut_children_i32<<<ygx::grid_for(total, 256), 256, 0, stream>>>(left_full, index_bits,
                                                                        total, s.left);
  YGX_CHECK_LAUNCH();
  ygx::k_mut_children_i32<<<ygx::grid_for(total, 256), 256, 0, stream>>>(right_full, index_bits,
                                                                        total, s.right);
  YGX_CHECK_LAUNCH();
  ygx::MutualCtl init{1, 0, 0, 0u, 0u};
  const int32_t r32 = (int32_t)root;
  if (cudaMemcpyAsync(s.ctl, &init, sizeof(init), cudaMemcpyHostToDevice, stream) != cudaSuccess ||
      cudaMemcpyAsync(s.wf_a[0], &r32, sizeof(r32), cudaMemcpyHostToDevice, stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(s.wf_b[0], &r32, sizeof(r32), cudaMemcpyHostToDevice, stream) !=
          cudaSuccess)
    return YGX_ERR_CUDA;
  ygx::MutualCtl h = init;
  int gen = 0, cur = 0;
  int rc = YGX_OK;
  while (h.size > 0 && (h.flags & (ygx::kMutFarOver | ygx::kMutNearOver | ygx::kMutQueueOver |
                                   ygx::kMutBadInput)) == 0) {
    if (gen >= ygx::kMutMaxGens) {
      rc = YGX_ERR_QUEUE_OVERFLOW;
      break;
    }
    const int64_t n = h.size;
    const int grid = ygx::grid_for(n, 256);
    ygx::k_mut_eval<<<grid, 256, 0, stream>>>(s.wf_a[cur], s.wf_b[cur], n, s.left, centers,
                                              radii, total, theta_sq, s.nchild, s.kind, s.emit,
                                              s.ctl);
    YGX_CHECK_LAUNCH();
    rc = ygx::exclusive_scan<int32_t>(s.nchild, n, s.child_off, s.tmp, stream);
    if (rc) break;
    rc = ygx::exclusive_scan<int64_t>(s.emit, n, s.emit_off, s.tmp, stream);
    if (rc) break;
    ygx::k_mut_emit<<<grid, 256, 0, stream>>>(
        s.wf_a[cur], s.wf_b[cur], n, s.left, s.right, s.kind, s.emit, s.child_off, s.emit_off,
        s.ctl, Q, s.wf_a[cur ^ 1], s.wf_b[cur ^ 1], far_cap, near_cap, index_bits, far_a, far_b,
        near_a, near_b);
    YGX_CHECK_LAUNCH();
    ygx::k_mut_advance<<<1, 32, 0, stream>>>(s.ctl, s.child_off, s.emit_off, n, Q, far_cap,
                                             near_cap);
    YGX_CHECK_LAUNCH();
    if (cudaMemcpyAsync(&h, s.ctl, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
      return YGX_ERR_CUDA;
    cur ^= 1;
    ++gen;
  }
  if (cudaMemcpyAsync(&h, s.ctl, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  counts_out[0] = h.far_n;
  counts_out[1] = h.near_n;
  flags_out[0] = h.flags;
  if (gens_out) gens_out[0] = gen;
  if (h.flags & ygx::kMutBadInput) return YGX_ERR_ARG;
  return rc;
}

}  // extern "C"
