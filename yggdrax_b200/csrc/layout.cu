// Row re-layouts of the traversal outputs (no counterpart kernels in the
// reference, which does these with jnp gathers / cumsum / nonzero):
//  * level-major far rows -> node-order rows (the count-then-fill layout that
//    DualTreeWalkResult / CompactTaggedFarPairs carry, _interactions_impl.py
//    :3561-3637, 5340-5390);
//  * the cells flagged by an index list, compacted in cell order with their
//    rank (the carrier cells of the native octree walk, :5411-5553);
//  * counts -> offsets (exclusive scan in the index dtype);
//  * a dense (rows x width) table of a row-mapped value per CSR entry, -1
//    padded (neighbor_leaf_positions, :3658-3688).
#include "scan.cuh"

namespace ygx {
namespace {

__global__ void k_load_counts(const void* counts, int index_bits, int64_t n,
                              int64_t* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = load_idx(counts, index_bits, i);
}

__global__ void k_store_offsets(const int64_t* __restrict__ off, int64_t n, int index_bits,
                                void* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n;
       i += (int64_t)gridDim.x * blockDim.x)
    store_idx(out, index_bits, i, off[i]);
}

// One warp per node: its row, read at its level-major start, written at its
// node-order start; targets = the node.
__global__ void __launch_bounds__(256)
    k_node_order_rows(const void* counts, const void* lm_offsets, const void* lm_sources,
                      const int64_t* __restrict__ no_off, int64_t total, int index_bits,
                      void* out_sources, void* out_targets) {
  const int lane = threadIdx.x & 31;
  const int64_t w0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = w0; v < total; v += nw) {
    const int64_t c = load_idx(counts, index_bits, v);
    const int64_t src = load_idx(lm_offsets, index_bits, v);
    const int64_t dst = no_off[v];
    for (int64_t k = lane; k < c; k += 32) {
      store_idx(out_sources, index_bits, dst + k, load_idx(lm_sources, index_bits, src + k));
      store_idx(out_targets, index_bits, dst + k, v);
    }
  }
}

__global__ void k_flag(const void* idx, int index_bits, int64_t n, int64_t M,
                       int32_t* __restrict__ flag, uint32_t* __restrict__ status) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = load_idx(idx, index_bits, i);
    if (c >= 0 && c < M) flag[c] = 1;
    else raise_flag(status, kFlagBadInput);
  }
}

__global__ void k_compact_flags(const int32_t* __restrict__ flag, const int64_t* __restrict__ pre,
                                int64_t M, int index_bits, int32_t* __restrict__ rank,
                                void* cells) {
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < M;
       c += (int64_t)gridDim.x * blockDim.x) {
    if (flag[c]) {
      rank[c] = (int32_t)pre[c];
      store_idx(cells, index_bits, pre[c], c);
    } else {
      rank[c] = -1;
    }
  }
}

__global__ void k_dense_rows(const void* offsets, const void* counts, int64_t rows,
                             const void* values, const int32_t* __restrict__ lookup,
                             int64_t lookup_n, int index_bits, int64_t width, void* out) {
  const int64_t n = rows * width;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = e / width, k = e - j * width;
    int64_t v = -1;
    if (k < load_idx(counts, index_bits, j)) {
      const int64_t x = load_idx(values, index_bits, load_idx(offsets, index_bits, j) + k);
      v = (x >= 0 && x < lookup_n) ? lookup[x] : -1;
    }
    store_idx(out, index_bits, e, v);
  }
}

__global__ void k_gather_idx(const void* table, const int64_t* __restrict__ idx, int64_t n,
                             int64_t table_n, int index_bits, void* out,
                             uint32_t* __restrict__ status) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = idx[i];
    int64_t v = -1;
    if (k >= 0 && k < table_n) v = load_idx(table, index_bits, k);
    else raise_flag(status, kFlagBadInput);
    store_idx(out, index_bits, i, v);
  }
}

// out[idx[i]] = i (a permutation's inverse); idx and out each int32 or int64.
__global__ void k_scatter_positions(const void* idx, int idx_bits, int64_t n, int64_t out_n,
                                    void* out, int out_bits, uint32_t* __restrict__ status) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = load_idx(idx, idx_bits, i);
    if (k >= 0 && k < out_n) store_idx(out, out_bits, k, i);
    else raise_flag(status, kFlagBadInput);
  }
}

struct LayoutScratch {
  uint32_t* status;
  int64_t* vals;  // n + 1
  int64_t* off;   // n + 1
  int32_t* flag;  // n
  int64_t* tmp;
};

LayoutScratch carve_layout(Arena& a, int64_t n) {
  LayoutScratch s;
  const int64_t m = n > 0 ? n : 1;
  s.status = a.take<uint32_t>(64);
  s.vals = a.take<int64_t>(m + 1);
  s.off = a.take<int64_t>(m + 1);
  s.flag = a.take<int32_t>(m);
  s.tmp = a.take<int64_t>(scan_scratch_elems(m));
  return s;
}

}  // namespace
}  // namespace ygx

extern "C" {

size_t ygx_layout_workspace_size(int64_t n) {
  ygx::Arena a{nullptr, 0, 0};
  ygx::carve_layout(a, n);
  return a.used + 256;
}

int ygx_counts_to_offsets(const void* counts, int64_t n, int index_bits, void* offsets_out,
                          void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (n < 0 || !offsets_out || !ws || (n > 0 && !counts) || (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  if (ws_bytes < ygx_layout_workspace_size(n)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::LayoutScratch s = ygx::carve_layout(a, n);
  if (n > 0) {
    ygx::k_load_counts<<<ygx::grid_for(n, 256), 256, 0, stream>>>(counts, index_bits, n, s.vals);
    YGX_CHECK_LAUNCH();
    int rc = ygx::exclusive_scan<int64_t>(s.vals, n, s.off, s.tmp, stream);
    if (rc) return rc;
  } else if (cudaMemsetAsync(s.off, 0, sizeof(int64_t), stream) != cudaSuccess) {
    return YGX_ERR_CUDA;
  }
  ygx::k_store_offsets<<<ygx::grid_for(n + 1, 256), 256, 0, stream>>>(s.off, n, index_bits,
                                                                     offsets_out);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

int ygx_node_order_far_rows(int64_t total, const void* far_counts, const void* node_offsets,
                            const void* sources, int index_bits, void* out_offsets,
                            void* out_sources, void* out_targets, void* ws, size_t ws_bytes,
                            cudaStream_t stream) {
  if (total < 1 || !far_counts || !node_offsets || !out_offsets || !ws ||
      (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  if (ws_bytes < ygx_layout_workspace_size(total)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::LayoutScratch s = ygx::carve_layout(a, total);
  ygx::k_load_counts<<<ygx::grid_for(total, 256), 256, 0, stream>>>(far_counts, index_bits,
                                                                   total, s.vals);
  YGX_CHECK_LAUNCH();
  int rc = ygx::exclusive_scan<int64_t>(s.vals, total, s.off, s.tmp, stream);
  if (rc) return rc;
  ygx::k_store_offsets<<<ygx::grid_for(total + 1, 256), 256, 0, stream>>>(s.off, total,
                                                                         index_bits, out_offsets);
  YGX_CHECK_LAUNCH();
  if (out_sources && out_targets && sources) {
    ygx::k_node_order_rows<<<ygx::grid_for(total * 32, 256, ygx::kNumSMs * 16), 256, 0, stream>>>(
        far_counts, node_offsets, sources, s.off, total, index_bits, out_sources, out_targets);
    YGX_CHECK_LAUNCH();
  }
  return YGX_OK;
}

int ygx_flag_compact(const void* idx, int64_t n_idx, int64_t M, int index_bits,
                     int32_t* rank_out, void* cells_out, int64_t* count_out, void* ws,
                     size_t ws_bytes, cudaStream_t stream) {
  if (M < 1 || n_idx < 0 || !rank_out || !cells_out || !count_out || !ws ||
      (n_idx > 0 && !idx) || (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  if (ws_bytes < ygx_layout_workspace_size(M)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::LayoutScratch s = ygx::carve_layout(a, M);
  if (cudaMemsetAsync(s.status, 0, sizeof(uint32_t), stream) != cudaSuccess ||
      cudaMemsetAsync(s.flag, 0, sizeof(int32_t) * M, stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  if (n_idx > 0) {
    ygx::k_flag<<<ygx::grid_for(n_idx, 256), 256, 0, stream>>>(idx, index_bits, n_idx, M, s.flag,
                                                              s.status);
    YGX_CHECK_LAUNCH();
  }
  int rc = ygx::exclusive_scan<int32_t>(s.flag, M, s.off, s.tmp, stream);
  if (rc) return rc;
  ygx::k_compact_flags<<<ygx::grid_for(M, 256), 256, 0, stream>>>(s.flag, s.off, M, index_bits,
                                                                 rank_out, cells_out);
  YGX_CHECK_LAUNCH();
  uint32_t flags = 0;
  if (cudaMemcpyAsync(count_out, s.off + M, sizeof(int64_t), cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(&flags, s.status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  return flags ? YGX_ERR_ARG : YGX_OK;
}

int ygx_dense_row_table(const void* offsets, const void* counts, int64_t rows, const void* values,
                        const int32_t* lookup, int64_t lookup_n, int index_bits, int64_t width,
                        void* out, cudaStream_t stream) {
  if (rows < 0 || width < 0 || (rows * width > 0 && (!offsets || !counts || !values || !lookup ||
                                                      !out)) ||
      (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  if (rows * width == 0) return YGX_OK;
  ygx::k_dense_rows<<<ygx::grid_for(rows * width, 256), 256, 0, stream>>>(
      offsets, counts, rows, values, lookup, lookup_n, index_bits, width, out);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

int ygx_gather_index(const void* table, int64_t table_n, const int64_t* idx, int64_t n,
                     int index_bits, void* out, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (n < 0 || table_n < 0 || !ws || (n > 0 && (!table || !idx || !out)) ||
      (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  if (ws_bytes < 256) return YGX_ERR_ARG;
  if (n == 0) return YGX_OK;
  uint32_t* status = (uint32_t*)ws;
  ygx::k_gather_idx<<<ygx::grid_for(n, 256), 256, 0, stream>>>(table, idx, n, table_n, index_bits,
                                                              out, status);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

int ygx_scatter_positions(const void* idx, int idx_bits, int64_t n, int64_t out_n, void* out,
                          int out_bits, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (n < 0 || out_n < 0 || !ws || ws_bytes < 256 || (n > 0 && (!idx || !out)) ||
      (idx_bits != 32 && idx_bits != 64) || (out_bits != 32 && out_bits != 64))
    return YGX_ERR_ARG;
  if (n == 0) return YGX_OK;
  ygx::k_scatter_positions<<<ygx::grid_for(n, 256), 256, 0, stream>>>(
      idx, idx_bits, n, out_n, out, out_bits, (uint32_t*)ws);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

}  // extern "C"
