// Explicit octree tables derived from the radix topology (L1b).
//
// Replaces build_explicit_octree_metadata (octree.py:479-550) and
// build_explicit_octree_metadata_from_leaf_partitions (octree.py:204-419):
// the compressed octree cells are the leaf cells plus the lowest common
// ancestors of consecutive leaves (2L - 1 candidates), sorted by a
// depth-major address with the onesweep sort, deduplicated by a scan, then
// every table is filled by one thread per cell.
#include "scan.cuh"
#include "sort.cuh"

namespace ygx {
namespace {

constexpr uint64_t kU64Max = ~0ull;

// octree.py:113-133
__device__ __forceinline__ uint64_t oct_address(uint64_t code, int64_t depth) {
  uint64_t d = (uint64_t)(depth > 0 ? depth : 0);
  uint64_t bit_shift = 63ull - 3ull * d;  // wraps like the reference's uint64
  uint64_t pow8d = shl64(1ull, 3ull * d);
  return (pow8d - 1ull) / 7ull + shr64(code, bit_shift);
}
// octree.py:136-141
__device__ __forceinline__ uint64_t prefix_code(uint64_t code, int64_t depth) {
  if (depth <= 0) return 0;
  int64_t s = 63 - 3 * depth;
  s = s > 0 ? s : 0;
  return shl64(shr64(code, (uint64_t)s), (uint64_t)s);
}
// octree.py:144-149
__device__ __forceinline__ int64_t octant_at_depth(uint64_t code, int64_t depth) {
  if (depth <= 0) return 0;
  int64_t s = 63 - 3 * depth;
  s = s > 0 ? s : 0;
  return (int64_t)(shr64(code, (uint64_t)s) & 7ull);
}
// octree.py:152-165
__device__ __forceinline__ int64_t common_depth(uint64_t a, uint64_t b) {
  uint64_t x = a ^ b;
  int64_t bits = x == 0 ? 63 : (clz64(x) - 1 > 0 ? clz64(x) - 1 : 0);
  return bits / 3;
}
// x[idx] for a signed index: wrap negatives by n, clamp into [0, n-1].
__device__ __forceinline__ int64_t gather_index(int64_t idx, int64_t n) {
  if (idx < 0) idx += n;
  if (idx < 0) idx = 0;
  if (idx > n - 1) idx = n - 1;
  return idx;
}
// jnp.searchsorted(method="scan"): ceil(log2(n + 1)) halving steps over
// (low, high] from (0, n).  Used verbatim because the adaptive leaf cells
// searched in phase 3 need not be sorted.
__device__ __forceinline__ int64_t searchsorted_scan(const uint64_t* a, int64_t n, uint64_t q,
                                                     bool left) {
  if (n == 0) return 0;
  int levels = 0;
  while (((int64_t)1 << levels) < n + 1) ++levels;
  int64_t lo = 0, hi = n;
  for (int it = 0; it < levels; ++it) {
    int64_t mid = (int64_t)(((uint64_t)lo + (uint64_t)hi) >> 1);
    uint64_t v = a[mid];
    bool go_left = left ? (q <= v) : (q < v);
    if (go_left) hi = mid; else lo = mid;
  }
  return hi;
}
// Lower bound in a sorted array (same result as the scan search there).
__device__ __forceinline__ int64_t lower_bound(const uint64_t* a, int64_t n, uint64_t q) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] < q) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// octree.py:168-186 (_resolved_leaf_cells) + candidate leaves.
__global__ void k_leaf_cells(const void* ranges, int64_t ni, int64_t L, const uint64_t* codes,
                             int64_t n, const uint64_t* leaf_codes_raw, const void* leaf_depths_raw,
                             int index_bits, uint64_t* lcode, int32_t* ldepth, int64_t* lstart,
                             int64_t* lend, uint64_t* addr) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < L;
       j += (int64_t)gridDim.x * blockDim.x) {
    int64_t s = load_idx(ranges, index_bits, 2 * (ni + j));
    int64_t e = load_idx(ranges, index_bits, 2 * (ni + j) + 1);
    uint64_t first = codes[gather_index(s, n)];
    uint64_t last = codes[gather_index(e, n)];
    int64_t raw = load_idx(leaf_depths_raw, index_bits, j);
    int64_t d = raw >= 0 ? raw : common_depth(first, last);
    uint64_t c = prefix_code(raw >= 0 ? leaf_codes_raw[j] : first, d);
    lcode[j] = c;
    ldepth[j] = (int32_t)d;
    lstart[j] = s;
    lend[j] = e + 1;
    addr[j] = oct_address(c, d);
  }
}

// Consecutive-leaf LCAs (octree.py:275-281).
__global__ void k_lca_cells(const uint64_t* lcode, int64_t L, uint64_t* addr, uint64_t* ccode,
                            int32_t* cdepth) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j + 1 < L;
       j += (int64_t)gridDim.x * blockDim.x) {
    int64_t d = common_depth(lcode[j], lcode[j + 1]);
    uint64_t c = prefix_code(lcode[j], d);
    addr[L + j] = oct_address(c, d);
    ccode[j] = c;
    cdepth[j] = (int32_t)d;
  }
}

__global__ void k_is_new(const uint64_t* addr_sorted, int64_t C, int32_t* is_new) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < C;
       k += (int64_t)gridDim.x * blockDim.x)
    is_new[k] = (k == 0 || addr_sorted[k] != addr_sorted[k - 1]) ? 1 : 0;
}

// First occurrence of each address writes the cell (duplicates carry the
// same code and depth, so max-scatter reduces to a plain store).
__global__ void k_unique_cells(const uint64_t* addr_sorted, const uint32_t* order, int64_t C,
                               int64_t L, const int32_t* is_new, const int64_t* uidx,
                               const uint64_t* lcode, const int32_t* ldepth, const uint64_t* ccode,
                               const int32_t* cdepth, uint64_t* ocode, int32_t* odepth,
                               uint64_t* oaddr) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < C;
       k += (int64_t)gridDim.x * blockDim.x) {
    if (!is_new[k]) continue;
    uint32_t src = order[k];
    int64_t u = uidx[k];
    ocode[u] = src < L ? lcode[src] : ccode[src - L];
    odepth[u] = src < L ? ldepth[src] : cdepth[src - L];
    oaddr[u] = addr_sorted[k];
  }
}

__global__ void k_cells(int64_t M, const int64_t* num_unique_p, int64_t L, const uint64_t* lcode,
                        const int64_t* lstart, const int64_t* lend, uint64_t* ocode,
                        int32_t* odepth, uint64_t* oaddr, int index_bits, uint64_t* o_codes,
                        void* o_depths, void* o_ranges, uint8_t* o_valid, void* o_parent,
                        int32_t* parent32, void* o_nbl, uint32_t* level_hist,
                        int32_t* max_depth) {
  const int64_t U = *num_unique_p;
  __shared__ uint32_t s_hist[22];
  if (threadIdx.x < 22) s_hist[threadIdx.x] = 0;
  __syncthreads();
  int32_t mx = 0;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    const bool valid = k < U;
    uint64_t c = valid ? ocode[k] : 0ull;
    int64_t d = valid ? odepth[k] : -1;
    o_codes[k] = c;
    store_idx(o_depths, index_bits, k, d);
    o_valid[k] = valid;
    store_idx(o_nbl, index_bits, k, k);  // valid cells are depth-sorted already
    // Ranges (phase 3): [C, C | mask_d] searched in the leaf cells.
    uint64_t dep = (uint64_t)(d > 0 ? d : 0);
    uint64_t bs = 63ull - 3ull * dep;
    uint64_t bs_safe = bs < 62ull ? bs : 62ull;
    uint64_t mask = shl64(1ull, bs_safe) - 1ull;
    uint64_t endc = valid ? (c | mask) : 0ull;
    int64_t f = searchsorted_scan(lcode, L, c, true);
    int64_t l = searchsorted_scan(lcode, L, endc, false) - 1;
    int64_t bound = L - 1 > 0 ? L - 1 : 0;
    f = f < 0 ? 0 : (f > bound ? bound : f);
    l = l < 0 ? 0 : (l > bound ? bound : l);
    store_idx(o_ranges, index_bits, 2 * k, valid ? lstart[f] : 0);
    store_idx(o_ranges, index_bits, 2 * k + 1, valid ? lend[l] - 1 : -1);
    // Parent (phase 5): deepest existing strict ancestor.
    int64_t par = -1;
    if (valid) {
      for (int step = 1; step <= 21 && step <= d; ++step) {
        int64_t pd = d - step;
        uint64_t pa = oct_address(prefix_code(c, pd), pd);
        int64_t pos = lower_bound(oaddr, M, pa);
        int64_t safe = pos < M - 1 ? pos : M - 1;
        if (oaddr[safe] == pa) { par = pos; break; }
      }
      if (d >= 0) atomicAdd(&s_hist[d < 21 ? d : 21], 1u);
      mx = (int32_t)d > mx ? (int32_t)d : mx;
    }
    store_idx(o_parent, index_bits, k, par);
    parent32[k] = (int32_t)par;
  }
  __syncthreads();
  if (threadIdx.x < 22 && s_hist[threadIdx.x]) atomicAdd(&level_hist[threadIdx.x], s_hist[threadIdx.x]);
  atomicMax(max_depth, mx);
}

__global__ void k_children(int64_t M, const int64_t* num_unique_p, const uint64_t* ocode,
                           const int32_t* odepth, const int32_t* parent32, int32_t* cplus) {
  const int64_t U = *num_unique_p;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < U;
       k += (int64_t)gridDim.x * blockDim.x) {
    int32_t p = parent32[k];
    if (p < 0) continue;
    int64_t oc = octant_at_depth(ocode[k], odepth[k]);
    atomicMax(&cplus[(int64_t)p * 8 + oc], (int32_t)(k + 1));
  }
}

__global__ void k_child_tables(int64_t M, const int64_t* num_unique_p, const int32_t* cplus,
                               int index_bits, void* o_children, uint8_t* o_child_mask,
                               void* o_child_counts, uint8_t* o_leaf_mask, int32_t* leaf_flag) {
  const int64_t U = *num_unique_p;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    const bool valid = k < U;
    int cnt = 0;
    for (int c = 0; c < 8; ++c) {
      int64_t v = (int64_t)cplus[k * 8 + c] - 1;
      store_idx(o_children, index_bits, k * 8 + c, v);
      bool m = valid && v >= 0;
      o_child_mask[k * 8 + c] = m;
      cnt += m;
    }
    store_idx(o_child_counts, index_bits, k, cnt);
    bool leaf = valid && cnt == 0;
    o_leaf_mask[k] = leaf;
    leaf_flag[k] = leaf ? 1 : 0;
  }
}

__global__ void k_leaf_nodes(int64_t M, const int32_t* leaf_flag, const int64_t* leaf_pos,
                             int index_bits, void* o_leaf_nodes) {
  const int64_t nleaf = leaf_pos[M];
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < M;
       k += (int64_t)gridDim.x * blockDim.x) {
    if (leaf_flag[k]) store_idx(o_leaf_nodes, index_bits, leaf_pos[k], k);
    if (k >= nleaf) store_idx(o_leaf_nodes, index_bits, k, -1);
  }
}

__global__ void k_level_offsets(const uint32_t* level_hist, const int32_t* max_depth,
                                int index_bits, void* o_level_offsets, void* o_num_levels) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    int64_t acc = 0;
    store_idx(o_level_offsets, index_bits, 0, 0);
    for (int l = 0; l < 22; ++l) {
      acc += level_hist[l];
      store_idx(o_level_offsets, index_bits, l + 1, acc);
    }
    store_idx(o_num_levels, index_bits, 0, (int64_t)(*max_depth) + 1);
  }
}

// radix node -> cell (octree.py:513-532).
__global__ void k_radix_to_oct(const void* ranges, int64_t total, int64_t ni, const uint64_t* codes,
                               int64_t n, const uint64_t* lcode, const int32_t* ldepth,
                               const uint64_t* oaddr, int64_t M, int index_bits,
                               void* radix_node_to_oct, void* radix_leaf_to_oct) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < total;
       v += (int64_t)gridDim.x * blockDim.x) {
    int64_t d;
    uint64_t c;
    if (v >= ni) {
      d = ldepth[v - ni];
      c = lcode[v - ni];
    } else {
      uint64_t first = codes[gather_index(load_idx(ranges, index_bits, 2 * v), n)];
      uint64_t last = codes[gather_index(load_idx(ranges, index_bits, 2 * v + 1), n)];
      d = common_depth(first, last);
      c = prefix_code(first, d);
    }
    int64_t pos = lower_bound(oaddr, M, oct_address(c, d));
    store_idx(radix_node_to_oct, index_bits, v, pos);
    if (v >= ni) store_idx(radix_leaf_to_oct, index_bits, v - ni, pos);
  }
}

}  // namespace

struct OctScratch {
  uint32_t* status;
  uint32_t* level_hist;
  int32_t* max_depth;
  int64_t* num_unique;
  uint64_t* lcode;
  int32_t* ldepth;
  int64_t* lstart;
  int64_t* lend;
  uint64_t* ccode;
  int32_t* cdepth;
  uint64_t* addr;
  uint64_t* addr_sorted;
  uint32_t* order;
  int32_t* is_new;
  int64_t* uidx;
  int64_t* scan_tmp;
  uint64_t* ocode;
  int32_t* odepth;
  uint64_t* oaddr;
  int32_t* parent32;
  int32_t* cplus;
  int32_t* leaf_flag;
  int64_t* leaf_pos;
  SortScratch sort;
};

static OctScratch carve_oct(Arena& a, int64_t L) {
  const int64_t C = 2 * L - 1 > 1 ? 2 * L - 1 : 1;
  OctScratch s;
  s.status = a.take<uint32_t>(64);
  s.level_hist = a.take<uint32_t>(32);
  s.max_depth = a.take<int32_t>(32);
  s.num_unique = a.take<int64_t>(8);
  s.lcode = a.take<uint64_t>(L);
  s.ldepth = a.take<int32_t>(L);
  s.lstart = a.take<int64_t>(L);
  s.lend = a.take<int64_t>(L);
  s.ccode = a.take<uint64_t>(L);
  s.cdepth = a.take<int32_t>(L);
  s.addr = a.take<uint64_t>(C);
  s.addr_sorted = a.take<uint64_t>(C);
  s.order = a.take<uint32_t>(C);
  s.is_new = a.take<int32_t>(C);
  s.uidx = a.take<int64_t>(C + 1);
  s.scan_tmp = a.take<int64_t>(scan_scratch_elems(C));
  s.ocode = a.take<uint64_t>(C);
  s.odepth = a.take<int32_t>(C);
  s.oaddr = a.take<uint64_t>(C);
  s.parent32 = a.take<int32_t>(C);
  s.cplus = a.take<int32_t>(C * 8);
  s.leaf_flag = a.take<int32_t>(C);
  s.leaf_pos = a.take<int64_t>(C + 1);
  s.sort = carve_sort_scratch(a, C, 8);
  return s;
}

}  // namespace ygx

extern "C" {

size_t ygx_octree_workspace_size(int64_t num_leaves) {
  ygx::Arena a{nullptr, 0, 0};
  ygx::carve_oct(a, num_leaves);
  return a.used + 256;
}

int ygx_octree_tables(const void* node_ranges, int64_t total, const uint64_t* morton_codes,
                      int64_t n, const uint64_t* leaf_codes, const void* leaf_depths,
                      int max_cell_depth, int index_bits, void* oct_parent, void* oct_children,
                      void* oct_child_counts, uint8_t* oct_child_mask, uint8_t* oct_valid_mask,
                      uint64_t* oct_node_codes, void* oct_node_depths, void* oct_node_ranges,
                      void* oct_nodes_by_level, void* oct_level_offsets, void* oct_num_levels,
                      uint8_t* oct_leaf_mask, void* oct_leaf_nodes, void* radix_node_to_oct,
                      void* radix_leaf_to_oct, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (total < 1 || n < 1 || (index_bits != 32 && index_bits != 64)) return YGX_ERR_ARG;
  const int64_t ni = (total - 1) / 2;
  const int64_t L = total - ni;
  if (ws_bytes < ygx_octree_workspace_size(L)) return YGX_ERR_ARG;
  if (max_cell_depth < 0 || max_cell_depth > 21) max_cell_depth = 21;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::OctScratch s = ygx::carve_oct(a, L);
  const int64_t C = 2 * L - 1;
  const int64_t M = C > 1 ? C : 1;
  if (cudaMemsetAsync(s.level_hist, 0, (char*)(s.num_unique + 8) - (char*)s.level_hist, stream) !=
      cudaSuccess)
    return YGX_ERR_CUDA;
  if (cudaMemsetAsync(s.cplus, 0, sizeof(int32_t) * M * 8, stream) != cudaSuccess) return YGX_ERR_CUDA;
  ygx::k_leaf_cells<<<ygx::grid_for(L, 256), 256, 0, stream>>>(
      node_ranges, ni, L, morton_codes, n, leaf_codes, leaf_depths, index_bits, s.lcode, s.ldepth,
      s.lstart, s.lend, s.addr);
  YGX_CHECK_LAUNCH();
  if (L > 1) {
    ygx::k_lca_cells<<<ygx::grid_for(L, 256), 256, 0, stream>>>(s.lcode, L, s.addr, s.ccode, s.cdepth);
    YGX_CHECK_LAUNCH();
  }
  // Address bits for depth <= D: (8^D - 1)/7 + 8^D - 1 < 2^(3D + 1).
  const int bits = 3 * max_cell_depth + 1 > 64 ? 64 : 3 * max_cell_depth + 1;
  int rc = ygx::onesweep_sort(s.addr, nullptr, C, 0, bits < 1 ? 1 : bits, s.addr_sorted, s.order,
                              s.sort, false, s.status, stream);
  if (rc) return rc;
  ygx::k_is_new<<<ygx::grid_for(C, 256), 256, 0, stream>>>(s.addr_sorted, C, s.is_new);
  YGX_CHECK_LAUNCH();
  rc = ygx::exclusive_scan<int32_t>(s.is_new, C, s.uidx, s.scan_tmp, stream);
  if (rc) return rc;
  if (cudaMemcpyAsync(s.num_unique, s.uidx + C, sizeof(int64_t), cudaMemcpyDeviceToDevice,
                      stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  // oaddr beyond the unique cells is the uint64 max sentinel.
  if (cudaMemsetAsync(s.oaddr, 0xFF, sizeof(uint64_t) * M, stream) != cudaSuccess) return YGX_ERR_CUDA;
  ygx::k_unique_cells<<<ygx::grid_for(C, 256), 256, 0, stream>>>(
      s.addr_sorted, s.order, C, L, s.is_new, s.uidx, s.lcode, s.ldepth, s.ccode, s.cdepth, s.ocode,
      s.odepth, s.oaddr);
  YGX_CHECK_LAUNCH();
  ygx::k_cells<<<ygx::grid_for(M, 256), 256, 0, stream>>>(
      M, s.num_unique, L, s.lcode, s.lstart, s.lend, s.ocode, s.odepth, s.oaddr, index_bits,
      oct_node_codes, oct_node_depths, oct_node_ranges, oct_valid_mask, oct_parent, s.parent32,
      oct_nodes_by_level, s.level_hist, s.max_depth);
  YGX_CHECK_LAUNCH();
  ygx::k_children<<<ygx::grid_for(M, 256), 256, 0, stream>>>(M, s.num_unique, s.ocode, s.odepth,
                                                             s.parent32, s.cplus);
  YGX_CHECK_LAUNCH();
  ygx::k_child_tables<<<ygx::grid_for(M, 256), 256, 0, stream>>>(
      M, s.num_unique, s.cplus, index_bits, oct_children, oct_child_mask, oct_child_counts,
      oct_leaf_mask, s.leaf_flag);
  YGX_CHECK_LAUNCH();
  rc = ygx::exclusive_scan<int32_t>(s.leaf_flag, M, s.leaf_pos, s.scan_tmp, stream);
  if (rc) return rc;
  ygx::k_leaf_nodes<<<ygx::grid_for(M, 256), 256, 0, stream>>>(M, s.leaf_flag, s.leaf_pos,
                                                               index_bits, oct_leaf_nodes);
  YGX_CHECK_LAUNCH();
  ygx::k_level_offsets<<<1, 32, 0, stream>>>(s.level_hist, s.max_depth, index_bits,
                                             oct_level_offsets, oct_num_levels);
  YGX_CHECK_LAUNCH();
  ygx::k_radix_to_oct<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      node_ranges, total, ni, morton_codes, n, s.lcode, s.ldepth, s.oaddr, M, index_bits,
      radix_node_to_oct, radix_leaf_to_oct);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

}  // extern "C"
