/*
 * ygx.h -- C ABI of libygx.so, the sm_100a CUDA implementation of the
 * yggdrax tree pipeline (Morton encode + stable sort, Karras radix /
 * fixed-depth builds, octree tables, node geometry, dual-tree traversal).
 *
 * Conventions
 *  - Every array argument is a DEVICE pointer to caller-owned memory unless
 *    the comment says "host".  Nothing here allocates device memory.
 *  - Scratch memory is a caller-provided device workspace `ws` of at least
 *    the bytes returned by the matching *_workspace_size function.  Its first
 *    256 bytes hold a status word of YGX_FLAG_* bits that kernels OR into
 *    instead of trapping; clear it with ygx_workspace_init and read it with
 *    ygx_status_read.
 *  - Index outputs use the "index dtype" of the reference (int64 by default,
 *    int32 when index_bits == 32): arguments typed `void*` with an
 *    `index_bits` parameter are arrays of that dtype.
 *  - All work is enqueued on `stream`; functions synchronize the stream only
 *    where their comment says so (to return data-dependent sizes).
 *  - Return value: YGX_OK or one of the YGX_ERR_* codes below.
 *
 * Each entry point names the reference function (file:line in the yggdrax
 * project) whose behaviour it provides.
 */
#pragma once
#include <stddef.h>
#include <stdint.h>

typedef struct CUstream_st* cudaStream_t;

enum {
  YGX_OK = 0,
  YGX_ERR_ARG = 1,             /* bad argument / workspace too small          */
  YGX_ERR_CUDA = 2,            /* a CUDA runtime call or launch failed        */
  YGX_ERR_TIMEOUT = 3,         /* a bounded device spin gave up               */
  YGX_ERR_QUEUE_OVERFLOW = 4,  /* traversal wavefront capacity exceeded       */
  YGX_ERR_FAR_OVERFLOW = 5,    /* far-list capacity exceeded                  */
  YGX_ERR_NEAR_OVERFLOW = 6,   /* near-list capacity exceeded                 */
  YGX_ERR_INT32_TOTAL = 7,     /* pair totals exceed the int32 range          */
  YGX_ERR_MALFORMED = 8,       /* topology inconsistent (tied Morton codes)   */
  YGX_ERR_TOO_LARGE = 9        /* size above a fixed maximum                  */
};

/* status-word bits (device side) */
#define YGX_FLAG_TIMEOUT (1u << 0)
#define YGX_FLAG_QUEUE_OVERFLOW (1u << 1)
#define YGX_FLAG_FAR_OVERFLOW (1u << 2)
#define YGX_FLAG_NEAR_OVERFLOW (1u << 3)
#define YGX_FLAG_MALFORMED (1u << 4)
#define YGX_FLAG_BAD_INPUT (1u << 5)
#define YGX_FLAG_LOG_OVERFLOW (1u << 6)

/* launch-shape knobs (ygx_tune_set / ygx_tune_get); chosen by the autotuner */
#define YGX_TUNE_SORT_RANK 0   /* onesweep ranking: 0 ballots, 1 peer tables, 2 by skew */
#define YGX_TUNE_SORT_SKEW 1   /* policy 2 threshold: max digit share x 256 (1..256)    */
#define YGX_TUNE_WALK_BLOCKS 2 /* walk CTAs per SM (2..6)                              */
#define YGX_TUNE_REFIT_WARPS 3 /* warps per CTA of the leaf refit (2, 4, 8)            */
#define YGX_TUNE_ROW_GRID 4    /* CTAs per SM of the short-row finalize (4..32, pow2)  */
#define YGX_TUNE_SORT_TILE 5   /* onesweep tile: 0 16x256 keys 3/SM, 1 12x256 4/SM,     */
                               /* 2 20x256 2/SM, 3 24x256 2/SM                          */
#define YGX_TUNE_SPIN_LIMIT 6  /* iterations a device-side wait (sort look-back) spins   */
                               /* before it gives up and flags YGX_FLAG_TIMEOUT          */
                               /* (0..2^24; default 2^22); not a performance knob        */
#define YGX_TUNE_TARGET_BUDGET 7 /* steps one warp spends on a piece of a target before */
                                 /* handing the rest to other warps (1..4096; 128)     */
#define YGX_TUNE_SORT_BITS 8   /* onesweep digit width: 8, or 11 (2048 bins) for every  */
                               /* sort whose key range it covers in fewer passes        */
                               /* (63-bit Morton codes: 6 passes instead of 8)          */

/* traversal statistics words (host array of YGX_TSTAT_WORDS uint64) */
#define YGX_TSTAT_WORDS 16
#define YGX_TSTAT_FAR_TOTAL 0   /* directed far entries (sum of far counts)    */
#define YGX_TSTAT_NEAR_TOTAL 1  /* directed near entries                       */
#define YGX_TSTAT_MAX_FAR 2     /* largest far row                             */
#define YGX_TSTAT_MAX_NEAR 3    /* largest near row                            */
#define YGX_TSTAT_ACCEPT 4      /* accept decisions (canonical pairs)          */
#define YGX_TSTAT_NEAR 5        /* near decisions                              */
#define YGX_TSTAT_REFINE 6      /* refine decisions                            */
#define YGX_TSTAT_MAX_WF 7      /* largest wavefront                           */
#define YGX_TSTAT_GENS 8        /* wavefront generations                       */
#define YGX_TSTAT_WF_NEED 9     /* wf_capacity that would have fit             */
#define YGX_TSTAT_LOG_NEED 10   /* log_capacity that would have fit            */
#define YGX_TSTAT_OVF_ROWS 11   /* predicted walk: rows past their capacity    */
#define YGX_TSTAT_OVF_ENTRIES 12 /* predicted walk: entries past the capacities */
#define YGX_TSTAT_EXT_FAR 13    /* predicted walk: far extension entries       */
#define YGX_TSTAT_EXT_NEAR 14   /* predicted walk: near extension entries      */

#ifdef __cplusplus
extern "C" {
#endif

/* ---- workspace / status -------------------------------------------------- */

/* Zeroes the status word and bookkeeping header of a workspace. */
int ygx_workspace_init(void* ws, size_t ws_bytes, cudaStream_t stream);
/* Copies the status word to host *host_flags; synchronizes the stream. */
int ygx_status_read(const void* ws, uint32_t* host_flags, cudaStream_t stream);
/* Number of kernel launches this library has issued in this process. */
uint64_t ygx_launch_counter(void);
/* Launch-shape knobs (YGX_TUNE_*), process-wide.  No reference counterpart:
 * the reference tunes nothing at run time.  An illegal value is rejected with
 * YGX_ERR_ARG and leaves the knob unchanged.  Results never depend on a knob. */
int ygx_tune_set(int knob, int value);
int ygx_tune_get(int knob, int* value);

/* ---- L0: bounds, Morton codes, stable sort ------------------------------- */

/* infer_bounds (yggdrax/bounds.py:11-33): bounds_out = [min x,y,z, max x,y,z]
 * with the reference's padding.  ws: ygx_encode_sort_workspace_size(0). */
int ygx_bounds(const float* positions, int64_t n, float* bounds_out, void* ws, size_t ws_bytes,
               cudaStream_t stream);

/* morton_encode_impl (yggdrax/morton.py:43-77): 63-bit codes of positions
 * (n x 3 float32) in bounds (6 floats, device). */
int ygx_morton_encode(const float* positions, int64_t n, const float* bounds, uint64_t* codes,
                      cudaStream_t stream);

size_t ygx_encode_sort_workspace_size(int64_t n);
/* Fused infer_bounds (if bounds_in == NULL) + morton_encode_impl + the stable
 * argsort of the codes (yggdrax/_tree_impl.py:397-402, yggdrax/tree.py:401-404):
 * codes_sorted[k] = code of particle order[k], ascending, ties by index. */
int ygx_encode_sort(const float* positions, int64_t n, const float* bounds_in, float* bounds_out,
                    uint64_t* codes_sorted, uint32_t* order, void* ws, size_t ws_bytes,
                    cudaStream_t stream);

size_t ygx_sort_pairs_workspace_size(int64_t n);
/* Stable LSD radix sort of (uint64 key, uint32 value) pairs on key bits
 * [begin_bit, end_bit) -- the device equivalent of jnp.argsort(stable=True)
 * used throughout the reference (values_in == NULL: value = input index). */
int ygx_sort_pairs(const uint64_t* keys_in, const uint32_t* values_in, int64_t n, int begin_bit,
                   int end_bit, uint64_t* keys_out, uint32_t* values_out, void* ws,
                   size_t ws_bytes, cudaStream_t stream);

/* Same sort as ygx_sort_pairs, for callers that cannot allocate device
 * memory where they sort (e.g. an XLA custom-call handler without a scratch
 * request, whose framework has preallocated the GPU's memory pool): the
 * scratch lives in a 6 MiB array inside libygx.so that every GPU using the
 * library keeps until the process exits.  At most 262,144 keys per call;
 * larger n returns YGX_ERR_TOO_LARGE.  Nothing is allocated.  The first call
 * on a device looks up the array's device address (make it before any
 * stream capture, with the stream's device current).  All calls share the
 * array: calls that overlap on the GPU race, so order them on one stream.
 * No counterpart in the reference (it has no allocation-free sort entry). */
int ygx_sort_pairs_noalloc(const uint64_t* keys_in, const uint32_t* values_in, int64_t n,
                           int begin_bit, int end_bit, uint64_t* keys_out, uint32_t* values_out,
                           cudaStream_t stream);
/* Status word of the last ygx_sort_pairs_noalloc call on the stream's
 * device (YGX_FLAG_TIMEOUT: a look-back wait gave up; YGX_FLAG_BAD_INPUT: an
 * inconsistent digit histogram), copied to host *host_flags in stream order;
 * synchronizes the stream.  0 means the sort completed.  Allocates nothing.
 * No counterpart in the reference. */
int ygx_sort_pairs_noalloc_status(uint32_t* host_flags, cudaStream_t stream);

/* reorder_particles_by_indices / inverse_permutation
 * (yggdrax/_tree_impl.py:900-926): any output may be NULL. */
int ygx_reorder(const float* positions, const float* masses, const uint32_t* order, int64_t n,
                int index_bits, float* positions_sorted, float* masses_sorted,
                void* particle_indices, void* inverse, cudaStream_t stream);
/* The same reorder in two steps, for random-order inputs: ygx_pack_particles
 * writes (x, y, z, mass) float4 records (packed: n records, 16-byte aligned,
 * caller-owned), and ygx_reorder_packed gathers one aligned record per
 * particle (one memory sector instead of up to three).  Outputs as for
 * ygx_reorder; any output may be NULL. */
int ygx_pack_particles(const float* positions, const float* masses, int64_t n, void* packed,
                       cudaStream_t stream);
int ygx_reorder_packed(const void* packed, const uint32_t* order, int64_t n, int index_bits,
                       float* positions_sorted, float* masses_sorted, void* particle_indices,
                       void* inverse, cudaStream_t stream);

/* ---- L1: leaf partitions -------------------------------------------------- */

/* Fixed-size chunks of the sorted order (yggdrax/_tree_impl.py:404-406):
 * L = ceil(n / leaf_size) leaves; leaf_codes = codes_sorted[start];
 * leaf_depths (may be NULL) = -1. */
int ygx_leaves_adaptive(const uint64_t* codes_sorted, int64_t n, int64_t leaf_size, int index_bits,
                        void* leaf_starts, void* leaf_ends, uint64_t* leaf_codes,
                        void* leaf_depths, cudaStream_t stream);

/* _fixed_depth_leaf_partitions (yggdrax/_tree_impl.py:1373-1401), depth >= 1:
 * 8^depth dense buckets, empty ones kept. */
int ygx_leaves_fixed(const uint64_t* codes_sorted, int64_t n, int depth, int index_bits,
                     void* leaf_starts, void* leaf_ends, uint64_t* leaf_codes, void* leaf_depths,
                     cudaStream_t stream);

size_t ygx_refine_workspace_size(int64_t num_buckets);
/* _refine_leaf_partitions_by_aspect (yggdrax/_tree_impl.py:96-227), pass 1:
 * per-bucket refined-leaf counts; the total lands at device *total_out. */
int ygx_refine_count(const float* positions_sorted, const uint64_t* codes_sorted,
                     const void* starts, const void* ends, const uint64_t* codes,
                     const void* depths, int64_t L, int current_depth, int max_refine_levels,
                     double aspect_threshold, int min_leaf_particles, int index_bits,
                     int64_t* total_out, void* ws, size_t ws_bytes, cudaStream_t stream);
/* pass 2 (same arguments and workspace): the refined leaves in (start, code)
 * order. */
int ygx_refine_emit(const float* positions_sorted, const uint64_t* codes_sorted,
                    const void* starts, const void* ends, const uint64_t* codes,
                    const void* depths, int64_t L, int current_depth, int max_refine_levels,
                    double aspect_threshold, int min_leaf_particles, int index_bits,
                    void* out_starts, void* out_ends, uint64_t* out_codes, void* out_depths,
                    void* ws, size_t ws_bytes, cudaStream_t stream);

/* ---- L1: Karras topology and levels --------------------------------------- */

size_t ygx_topology_workspace_size(int64_t num_leaves);
/* _build_tree_from_leaf_partitions (yggdrax/_tree_impl.py:1009-1355) for
 * L >= 2 leaves, total = 2L - 1 nodes: parent, left/right children and leaf
 * flags, node_ranges (total x 2, inclusive), node_level, level_offsets (65),
 * nodes_by_level, num_levels (1) -- plus int32 copies used by the geometry
 * and traversal kernels (left32/right32 span all nodes, -1 on leaves).
 * *tree_flags_out (device word) gets YGX_FLAG_MALFORMED when tied leaf codes
 * produced a parent array that disagrees with the child arrays. */
int ygx_build_topology(const uint64_t* leaf_codes, const void* leaf_starts, const void* leaf_ends,
                       int64_t L, int index_bits, void* parent, void* left, void* right,
                       uint8_t* left_is_leaf, uint8_t* right_is_leaf, void* node_ranges,
                       void* node_level, void* level_offsets, void* nodes_by_level,
                       void* num_levels, int32_t* parent32, int32_t* left32, int32_t* right32,
                       int32_t* level32, int32_t* nbl32, uint32_t* tree_flags_out, void* ws,
                       size_t ws_bytes, cudaStream_t stream);

/* ---- L1b: explicit octree tables ------------------------------------------ */

size_t ygx_octree_workspace_size(int64_t num_leaves);
/* build_explicit_octree_metadata (yggdrax/octree.py:479-550) over a radix
 * topology of `total` nodes: M = 2L - 1 cell slots.  max_cell_depth bounds
 * every leaf cell depth (<= 21) and sizes the address sort. */
int ygx_octree_tables(const void* node_ranges, int64_t total, const uint64_t* morton_codes,
                      int64_t n, const uint64_t* leaf_codes, const void* leaf_depths,
                      int max_cell_depth, int index_bits, void* oct_parent, void* oct_children,
                      void* oct_child_counts, uint8_t* oct_child_mask, uint8_t* oct_valid_mask,
                      uint64_t* oct_node_codes, void* oct_node_depths, void* oct_node_ranges,
                      void* oct_nodes_by_level, void* oct_level_offsets, void* oct_num_levels,
                      uint8_t* oct_leaf_mask, void* oct_leaf_nodes, void* radix_node_to_oct,
                      void* radix_leaf_to_oct, void* ws, size_t ws_bytes, cudaStream_t stream);

/* ---- L2: node geometry ----------------------------------------------------- */

size_t ygx_geometry_workspace_size(int64_t total);
/* compute_tree_geometry (yggdrax/_geometry_impl.py:176-338): center (total x 3),
 * half_extent (total x 3), radius, max_extent (float32).  use_morton selects
 * Morton-cell leaf boxes; otherwise particle ranges with at most
 * max_leaf_size particles per leaf (< 0: no cap). */
int ygx_tree_geometry(const void* node_ranges, int64_t total, int index_bits,
                      const int32_t* parent32, const int32_t* left32, const int32_t* right32,
                      const int32_t* level32, const uint32_t* tree_flags,
                      const float* positions_sorted, int64_t n, int use_morton,
                      const float* bounds, const uint64_t* leaf_codes, const void* leaf_depths,
                      int64_t max_leaf_size, float* center, float* half_extent, float* radius,
                      float* max_extent, void* ws, size_t ws_bytes, cudaStream_t stream);

/* ---- L3: dual-tree traversal ------------------------------------------------ */

/* wf_capacity: wavefront pairs over all walk regions; log_capacity: logged
 * (accepted or near) pairs over all log regions.  The walk reports in
 * YGX_TSTAT_WF_NEED / YGX_TSTAT_LOG_NEED the capacities that would have fit. */
size_t ygx_traverse_workspace_size(int64_t total, int64_t num_leaves, int64_t wf_capacity,
                                   int64_t log_capacity);
/* The walk of build_interactions_and_neighbors: the count walk
 * (yggdrax/_interactions_impl.py:2600-2939 _dual_tree_walk_count_impl) and
 * the pair enumeration of the fill walk (:2942-3558) in one pass; every
 * accepted / near pair is logged once for ygx_traverse_fill.
 * mac 0 = "bh", 1 = "dehnen", 2 = "engblom".  stats_out / flags_out are HOST
 * arrays (YGX_TSTAT_WORDS / 1 words).  YGX_FLAG_QUEUE_OVERFLOW or
 * YGX_FLAG_LOG_OVERFLOW in *flags_out: re-run with larger capacities (the
 * walk is deterministic; the reported log need is exact).  gens_hint > 0:
 * the expected number of generations (a previous walk's YGX_TSTAT_GENS);
 * the wavefront is first checked after that many, then every 16.
 * Synchronizes the stream. */
#define YGX_WALK_LOG 0   /* one walk: row counts + a log of accepted / near pairs */
#define YGX_WALK_COUNT 1 /* plain two-pass mode, first walk: row counts only     */
int ygx_traverse_walk(const float* center, const float* radius, const float* max_extent,
                      const int32_t* left32, const int32_t* right32, const int32_t* leafpos32,
                      int64_t total, int64_t num_internal, int mac, float theta,
                      float dehnen_radius_scale, int root, int mode, int gens_hint,
                      int64_t wf_capacity, int64_t log_capacity, uint64_t* stats_out,
                      uint32_t* flags_out, void* ws, size_t ws_bytes, cudaStream_t stream);
/* Row layout of the fill walk (_dual_tree_walk_compact_fill_impl,
 * :2942-3558) and the offset tables of _result_to_interactions /
 * _result_to_neighbors (:3561-3837), from the walk's counts and pair log. */
int ygx_traverse_fill(int64_t total, int64_t num_internal, int64_t wf_capacity,
                      int64_t log_capacity, int64_t far_total, int64_t near_total,
                      const int32_t* nbl32, const int32_t* leafpos32,
                      const void* tree_level_offsets, int num_levels, int index_bits,
                      void* node_offsets, void* far_counts, void* level_offsets,
                      void* near_offsets, void* near_counts, int32_t* far_src32,
                      int32_t* near_nbr32, void* ws, size_t ws_bytes, cudaStream_t stream);
/* Plain two-pass mode, second walk (the reference's count-then-fill,
 * _dual_tree_walk_compact_fill_impl :2942-3558): after ygx_traverse_walk with
 * YGX_WALK_COUNT on the same workspace, the offset tables as in
 * ygx_traverse_fill and the raw rows written by walking the `gens`
 * generations again (entries at atomic row cursors). */
int ygx_traverse_fill_walk(int64_t total, int64_t num_internal, int mac, float theta, int root,
                           int64_t wf_capacity, int64_t log_capacity, int gens,
                           int64_t far_total, int64_t near_total, const int32_t* nbl32,
                           const void* tree_level_offsets, int num_levels, int index_bits,
                           void* node_offsets, void* far_counts, void* level_offsets,
                           void* near_offsets, void* near_counts, int32_t* far_src32,
                           int32_t* near_nbr32, void* ws, size_t ws_bytes, cudaStream_t stream);
/* Learned one-pass mode (no counterpart in the reference; it replaces the
 * count walk of count-then-fill, _interactions_impl.py:2600-2939, by the
 * capacities of ygx_predict_caps and stays exact by completing every row
 * that outgrew its capacity):
 * 1. ygx_traverse_pad_offsets: padded row offsets into the workspace;
 *    sums_out (host, 2 words) = padded far / near totals.
 * 2. ygx_traverse_walk_predicted: one walk writing the raw rows (buffers of
 *    at least the padded totals); entries past a row's capacity are logged.
 * 3. ygx_traverse_fill_predicted: offset tables, overflowed rows moved to the
 *    extension area (raw buffers of padded total + YGX_TSTAT_EXT_* entries)
 *    and completed; far_raw_off / near_raw_off receive the raw row starts for
 *    ygx_traverse_finalize. */
int ygx_traverse_pad_offsets(int64_t total, int64_t num_internal, int64_t wf_capacity,
                             int64_t log_capacity, const int32_t* far_cap32,
                             const int32_t* near_cap32, uint64_t* sums_out, void* ws,
                             size_t ws_bytes, cudaStream_t stream);
int ygx_traverse_walk_predicted(const float* center, const float* radius,
                                const float* max_extent, const int32_t* left32,
                                const int32_t* right32, const int32_t* leafpos32, int64_t total,
                                int64_t num_internal, int mac, float theta,
                                float dehnen_radius_scale, int root, int gens_hint,
                                int64_t wf_capacity, int64_t log_capacity,
                                const int32_t* far_cap32,
                                const int32_t* near_cap32, int32_t* far_raw32,
                                int32_t* near_raw32, uint64_t* stats_out, uint32_t* flags_out,
                                void* ws, size_t ws_bytes, cudaStream_t stream);
int ygx_traverse_fill_predicted(int64_t total, int64_t num_internal, int64_t wf_capacity,
                                int64_t log_capacity, const int32_t* far_cap32,
                                const int32_t* near_cap32, int64_t far_raw_cap,
                                int64_t near_raw_cap, const int32_t* nbl32,
                                const void* tree_level_offsets, int num_levels, int index_bits,
                                void* node_offsets, void* far_counts, void* level_offsets,
                                void* near_offsets, void* near_counts, int32_t* far_raw32,
                                int32_t* near_raw32, int64_t* far_raw_off, int64_t* near_raw_off,
                                void* ws, size_t ws_bytes, cudaStream_t stream);
/* Row finalize: canonical (ascending) order within each row, level-major
 * far sources/targets/target_levels, leaf-ordered near neighbours, and
 * optionally the dense neighbour_leaf_positions table (L x max_nbr).
 * far_raw_off / near_raw_off (device int64 per row, may be null) say where
 * each raw row starts when the raw rows are not at the output offsets (the
 * predicted walk's padded rows); far_row_base / near_row_base (int32 per
 * row, may be null) are subtracted from every node id written for the row
 * (the batched forest writes each set's lists in its local node ids). */
int ygx_traverse_finalize(int64_t total, int64_t num_internal, int64_t wf_capacity,
                          int64_t log_capacity, const int32_t* level32, const int32_t* leafpos32,
                          int index_bits, int32_t* far_src32, int32_t* near_nbr32,
                          const int64_t* far_raw_off, const int64_t* near_raw_off,
                          const int32_t* far_row_base, const int32_t* near_row_base,
                          void* far_sources,
                          void* far_targets, void* target_levels, void* neighbors,
                          void* neighbor_leaf_positions, int64_t max_nbr, void* ws,
                          size_t ws_bytes, cudaStream_t stream);
/* ---- per-target walk: the same exact lists, row by row -------------------
 * Replaces the count walk + compact fill walk of
 * build_interactions_and_neighbors (_interactions_impl.py:2600-3558; the
 * pair set of _dual_tree_walk_impl, :1119-1905) and the layouts of
 * _result_to_interactions / _result_to_neighbors (:3561-3837).  One warp
 * per target node walks the pairs {t, s} of the reference's symmetric walk
 * that involve t, from the parent's "split on my side" list; long
 * expansions are split into pieces run by other warps.  ordered != 0: the
 * warp walks its candidates in Morton order, so every row comes out in
 * ascending order with no sort; ordered == 0: every resolved candidate is
 * emitted at once and only refined ones are expanded (no re-popped lanes),
 * and ygx_target_walk_lists sorts the rows.  The same `ordered` must be
 * passed to all three calls of one walk.  Well-formed single
 * trees only (nodes 0..num_internal-1 internal, root `root`).
 * Predicted rows (unordered only; all six pointers, or none): far_rcap32
 * (per node) / near_rcap32 (per leaf position) are row capacities
 * (ygx_predict_caps), pad_far / pad_near their slots (ygx_target_pad), and
 * far_raw / near_raw int32 arrays of at least the padded totals plus the
 * extension the walk reports (YGX_TSTAT_EXT_FAR / _EXT_NEAR: the entries of
 * the rows that outgrew their capacity).  The walk writes every chunk that
 * fits its row's capacity in place; only the rest pass through the pools.
 * With predicted rows stats_out also carries YGX_TSTAT_OVF_ROWS /
 * _OVF_ENTRIES. 
 * caps (host, 8 int64): entry capacities of the far pool, near pool, split
 * lists, spill area; record capacities of far chunks, near chunks,
 * split-list chunks; continuation queue.  needs_out (host, 14 uint64): what
 * each of them needed (re-run with at least these when
 * YGX_FLAG_LOG_OVERFLOW is set), then the most chunks one split list had,
 * the warp cycles spent on pieces and waiting, the pieces run, the 32-wide
 * steps run and the candidates those steps held.
 * flags_out also reports YGX_FLAG_TIMEOUT (a bounded wait gave up) and
 * YGX_FLAG_MALFORMED (a split list had more chunks than can be ordered);
 * with either flag the lists are not produced: use ygx_traverse_walk.
 * stats_out as for ygx_traverse_walk (wf_need / log_need are 0).
 * Synchronizes the stream. */
size_t ygx_target_walk_workspace_size(int64_t total, int64_t num_leaves, const int64_t* caps,
                                      int ordered);
int ygx_target_walk(const float* center, const float* radius, const float* max_extent,
                    const int32_t* left32, const int32_t* right32, const int32_t* leafpos32,
                    const int32_t* parent32, const int32_t* level32, const int32_t* nbl32,
                    int64_t total, int64_t num_internal, int root, int mac, float theta,
                    float dehnen_radius_scale, const int64_t* caps, int ordered,
                    const int32_t* far_rcap32, const int32_t* near_rcap32,
                    const int64_t* pad_far, const int64_t* pad_near, int32_t* far_raw,
                    int32_t* near_raw, const void* tree_level_offsets, int num_levels,
                    int index_bits, uint64_t* stats_out, uint64_t* needs_out,
                    uint32_t* flags_out, void* ws, size_t ws_bytes, cudaStream_t stream);
/* After ygx_target_walk on the same workspace and capacities: the offset /
 * count tables and the rows (level-major far sources / targets /
 * target_levels, leaf-ordered near neighbours) in the index dtype, and
 * with max_nbr > 0 the dense neighbour_leaf_positions table (L x max_nbr).
 * far_records / near_records: needs_out[4] / needs_out[5] of the walk.
 * Unordered walks assemble and sort the rows in far_raw / near_raw (int32,
 * capacities far_raw_cap / near_raw_cap: at least far_total / near_total, or
 * with predicted rows the same arrays, capacities and pointers the walk had);
 * ordered walks take NULL / 0 for all of these. */
int ygx_target_walk_lists(int64_t total, int64_t num_internal, const int64_t* caps, int ordered,
                          const int32_t* far_rcap32, const int32_t* near_rcap32,
                          const int64_t* pad_far, const int64_t* pad_near, int32_t* far_raw,
                          int64_t far_raw_cap, int32_t* near_raw, int64_t near_raw_cap,
                          const int32_t* nbl32, const int32_t* level32,
                          const void* tree_level_offsets, int num_levels, int index_bits,
                          int64_t far_total, int64_t near_total, uint64_t far_records,
                          uint64_t near_records, void* node_offsets, void* far_counts,
                          void* level_offsets, void* sources, void* targets, void* target_levels,
                          void* near_offsets, void* near_counts, void* neighbors,
                          const int32_t* leafpos32, int64_t max_nbr,
                          void* neighbor_leaf_positions, void* ws, size_t ws_bytes,
                          cudaStream_t stream);
/* Padded row slots for predicted capacities (no reference counterpart: the
 * reference sizes rows by its count pass): pad_far[0..total] /
 * pad_near[0..num_leaves] = exclusive sums of far_rcap32 / near_rcap32 (int64,
 * device); sums_out (host, 2) = the padded totals.  Synchronizes the stream. */
size_t ygx_target_pad_workspace_size(int64_t total, int64_t num_leaves);
int ygx_target_pad(int64_t total, int64_t num_leaves, const int32_t* far_rcap32,
                   const int32_t* near_rcap32, int64_t* pad_far, int64_t* pad_near,
                   uint64_t* sums_out, void* ws, size_t ws_bytes, cudaStream_t stream);
/* ---- row re-layouts ---------------------------------------------------------
 * Device forms of the jnp gathers / cumsum / nonzero the reference uses to
 * re-lay its lists.  Index arrays are in the index dtype (index_bits). */
size_t ygx_layout_workspace_size(int64_t n);
/* offsets_out[0..n] = exclusive cumulative sum of counts[0..n) (the jnp.cumsum
 * row offsets of _result_to_neighbors, _interactions_impl.py:3640-3837). */
int ygx_counts_to_offsets(const void* counts, int64_t n, int index_bits, void* offsets_out,
                          void* ws, size_t ws_bytes, cudaStream_t stream);
/* Level-major far rows (node_offsets[v] = start of node v's row in sources)
 * -> the count-then-fill node-order layout: out_offsets[0..total] = node-order
 * row starts, out_sources / out_targets (may be NULL) the rows in node order
 * with every entry's target node (DualTreeWalkResult interaction_*,
 * CompactTaggedFarPairs; _interactions_impl.py:3561-3637, 5340-5390). */
int ygx_node_order_far_rows(int64_t total, const void* far_counts, const void* node_offsets,
                            const void* sources, int index_bits, void* out_offsets,
                            void* out_sources, void* out_targets, void* ws, size_t ws_bytes,
                            cudaStream_t stream);
/* The distinct cells named by idx[0..n_idx) in ascending order (cells_out,
 * capacity M) with rank_out[c] = position of cell c in that list or -1, and
 * their number in host *count_out -- jnp.nonzero of the carrier mask of the
 * native octree walk (_interactions_impl.py:5411-5553).  Synchronizes the
 * stream; an index outside [0, M) returns YGX_ERR_ARG. */
int ygx_flag_compact(const void* idx, int64_t n_idx, int64_t M, int index_bits,
                     int32_t* rank_out, void* cells_out, int64_t* count_out, void* ws,
                     size_t ws_bytes, cudaStream_t stream);
/* out[j * width + k] = lookup[values[offsets[j] + k]] for k < counts[j], else
 * -1 (rows x width): the dense neighbor_leaf_positions table
 * (_interactions_impl.py:3658-3688).  lookup is int32 over lookup_n values. */
int ygx_dense_row_table(const void* offsets, const void* counts, int64_t rows, const void* values,
                        const int32_t* lookup, int64_t lookup_n, int index_bits, int64_t width,
                        void* out, cudaStream_t stream);
/* out[i] = table[idx[i]] (idx int64; an index outside the table writes -1
 * and sets YGX_FLAG_BAD_INPUT in the status word at ws). */
int ygx_gather_index(const void* table, int64_t table_n, const int64_t* idx, int64_t n,
                     int index_bits, void* out, void* ws, size_t ws_bytes, cudaStream_t stream);
/* out[idx[i]] = i for i < n (a permutation's inverse, the jnp scatter of
 * inverse_permutation, _tree_impl.py:900-910); idx and out are int32 or int64
 * (idx_bits, out_bits); an index outside [0, out_n) sets YGX_FLAG_BAD_INPUT in
 * the status word at ws. */
int ygx_scatter_positions(const void* idx, int idx_bits, int64_t n, int64_t out_n, void* out,
                          int out_bits, void* ws, size_t ws_bytes, cudaStream_t stream);

/* ---- learned row-capacity predictor (no counterpart in the reference) -----
 * A per-node MLP (YGX_MLP_INPUTS -> 64 -> 64 -> 2, ReLU, fp32) that predicts
 * log2(1 + far row length) and log2(1 + near row length) from the node's
 * geometry, so the one-pass predicted walk can size its rows without the
 * count walk of count-then-fill (_interactions_impl.py:2600-2939).
 * Parameters: one float array of YGX_MLP_PARAMS (W1 [in x 64], b1, W2
 * [64 x 64], b2, W3 [64 x 2], b3; row-major). */
#define YGX_MLP_INPUTS 12
#define YGX_MLP_PARAMS 5122
int ygx_mlp_param_count(void);
size_t ygx_mlp_workspace_size(int64_t batch);
/* features[k * YGX_MLP_INPUTS + i] of every node (node_ranges inclusive,
 * index dtype).  mac as in ygx_traverse_walk. */
int ygx_node_features(const float* center, const float* radius, const float* max_extent,
                      const int32_t* level32, const int32_t* parent32, int64_t total,
                      int64_t num_internal, const void* node_ranges, int index_bits, int root,
                      float theta, int mac, float* features, cudaStream_t stream);
/* out[k * 2 + j] = MLP(features[k]). */
int ygx_mlp_forward(const float* params, const float* features, int64_t n, float* out,
                    cudaStream_t stream);
/* Masked mean-squared-error gradients of one batch (targets / mask [batch x 2]);
 * grads_out (YGX_MLP_PARAMS floats) and loss_out (1 float) are device
 * pointers, either may be null. */
int ygx_mlp_gradients(const float* params, const float* features, const float* targets,
                      const float* mask, int64_t batch, float* grads_out, float* loss_out,
                      void* ws, size_t ws_bytes, cudaStream_t stream);
/* One Adam step (step >= 1, betas 0.9 / 0.999) on a batch. */
int ygx_mlp_train_step(float* params, float* adam_m, float* adam_v, int step, float lr,
                       const float* features, const float* targets, const float* mask,
                       int64_t batch, float* loss_out, void* ws, size_t ws_bytes,
                       cudaStream_t stream);
/* Row capacities: far_cap32[node] and near_cap32[leaf position] =
 * ceil(2^(prediction + slack) - 1) + add. */
int ygx_predict_caps(const float* center, const float* radius, const float* max_extent,
                     const int32_t* level32, const int32_t* parent32, const int32_t* leafpos32,
                     int64_t total, int64_t num_internal, const void* node_ranges, int index_bits,
                     int root, float theta, int mac, const float* params, float slack_far,
                     float slack_near, int32_t add, int32_t* far_cap32, int32_t* near_cap32,
                     cudaStream_t stream);

/* ---- batched sets (no counterpart in the reference: many independent point
 * sets, stored back to back, built and walked together; every set's slice of
 * every output equals what the single-set entry points give for it) --------
 * Set s = points offsets[s] .. offsets[s+1] (device int64, S + 1), S <= 65536.
 * The forest: set s has L_s leaves at global leaf positions leaf_off[s] ..
 * leaf_off[s+1] and 2 L_s - 1 nodes at global node ids NO_s = 2 leaf_off[s] - s,
 * in the per-tree layout (internal nodes first). */
size_t ygx_batch_encode_sort_workspace_size(int64_t n);
/* infer_bounds / morton_encode_impl / the stable argsort
 * (bounds.py:11-33, morton.py:43-77, _tree_impl.py:401) of every set:
 * bounds_out (S x 6), codes_sorted and order_out (global input index) in
 * (set, code, index) order, seg_sorted_out (may be null) the set of each. */
int ygx_batch_encode_sort(const float* positions, int64_t n, const int64_t* offsets, int64_t S,
                          float* bounds_out, uint64_t* codes_sorted, uint32_t* order_out,
                          int32_t* seg_sorted_out, void* ws, size_t ws_bytes,
                          cudaStream_t stream);
/* _tree_impl.py:1047-1050, :900-910 per set (local particle_indices / inverse). */
int ygx_batch_reorder(const float* positions, const float* masses, const uint32_t* order,
                      const int32_t* seg_sorted, const int64_t* offsets, int64_t n, int index_bits,
                      float* positions_sorted, float* masses_sorted, void* particle_indices,
                      void* inverse, cudaStream_t stream);
size_t ygx_batch_leaf_offsets_workspace_size(int64_t S);
/* leaf_off (device, S + 1) = exclusive scan of ceil(n_s / leaf_size);
 * *total_leaves_out (host).  Synchronizes the stream. */
int ygx_batch_leaf_offsets(const int64_t* offsets, int64_t S, int64_t leaf_size,
                           int64_t* leaf_off, int64_t* total_leaves_out, void* ws,
                           size_t ws_bytes, cudaStream_t stream);
/* _tree_impl.py:405-406 per set; leaf_seg = set of each global leaf. */
int ygx_batch_leaves(const uint64_t* codes_sorted, const int64_t* offsets, const int64_t* leaf_off,
                     int64_t S, int64_t total_leaves, int64_t leaf_size, int index_bits,
                     void* leaf_starts, void* leaf_ends, uint64_t* leaf_codes, void* leaf_depths,
                     int32_t* leaf_seg, cudaStream_t stream);
size_t ygx_batch_topology_workspace_size(int64_t total_leaves, int64_t S);
/* _build_tree_from_leaf_partitions (_tree_impl.py:1009-1355) for every set:
 * per-set arrays with local values (parent / node_ranges / node_level /
 * nodes_by_level: 2 total_leaves - S; left / right / flags: total_leaves - S;
 * level_offsets S x 65; num_levels S), int32 copies with global node ids,
 * node_seg32 / leafpos32 / node_base32 (per node), leaf_base32 (per leaf),
 * seg_flags (S) and their union tree_flags_out. */
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
                             void* ws, size_t ws_bytes, cudaStream_t stream);
/* compute_tree_geometry (_geometry_impl.py:176-338) for every tree of the
 * forest (particle ranges; workspace ygx_geometry_workspace_size(total)). */
int ygx_batch_tree_geometry(const void* node_ranges, int64_t total, int64_t S,
                            const int64_t* leaf_off, const int32_t* leaf_seg,
                            int64_t total_leaves, const int64_t* offsets, int index_bits,
                            const int32_t* parent32, const int32_t* left32,
                            const int32_t* right32, const int32_t* level32,
                            const uint32_t* seg_flags, const float* positions_sorted,
                            int64_t max_leaf_size, float* center, float* half_extent,
                            float* radius, float* max_extent, void* ws, size_t ws_bytes,
                            cudaStream_t stream);
/* ygx_traverse_walk (YGX_WALK_LOG) over all trees of the forest at once;
 * ygx_traverse_fill / ygx_traverse_finalize (with the node / leaf bases as
 * row bases) follow on the same workspace. */
int ygx_batch_traverse_walk(const float* center, const float* radius, const float* max_extent,
                            const int32_t* left32, const int32_t* right32,
                            const int32_t* leafpos32, const int32_t* parent32, int64_t total,
                            const int64_t* leaf_off, int64_t S, const uint32_t* seg_flags,
                            int mac, float theta, float dehnen_radius_scale, int gens_hint,
                            int64_t wf_capacity, int64_t log_capacity, uint64_t* stats_out,
                            uint32_t* flags_out, void* ws, size_t ws_bytes, cudaStream_t stream);

/* The batched walk + fill + finalize in one call with every size fixed by
 * the caller (exactly `gens` generations; wavefront / log capacities;
 * far_capacity / near_capacity output entries) and no host synchronization
 * or copy, so that a CUDA graph can capture it.  What does not fit is
 * flagged in the workspace status (rows then left empty); read the flags and
 * the statistics with ygx_traverse_stats_read.  No reference counterpart. */
int ygx_batch_traverse_lists(
    const float* center, const float* radius, const float* max_extent, const int32_t* left32,
    const int32_t* right32, const int32_t* leafpos32, const int32_t* parent32,
    const int32_t* nbl32, const int32_t* level32, const int32_t* node_base32,
    const int32_t* leaf_base32, int64_t total, const int64_t* leaf_off, int64_t S,
    const uint32_t* seg_flags, int mac, float theta, float dehnen_radius_scale, int gens,
    int64_t wf_capacity, int64_t log_capacity, int64_t far_capacity, int64_t near_capacity,
    int index_bits, void* node_offsets, void* far_counts, void* near_offsets, void* near_counts,
    int32_t* far_src32, int32_t* near_nbr32, void* sources, void* targets, void* target_levels,
    void* neighbors, void* ws, size_t ws_bytes, cudaStream_t stream);

/* Statistics words (YGX_TSTAT_*) and status flags of a traversal workspace,
 * copied to the host; synchronizes the stream. */
int ygx_traverse_stats_read(int64_t total, int64_t num_leaves, int64_t wf_capacity,
                            int64_t log_capacity, const void* ws, size_t ws_bytes,
                            uint64_t* stats_out, uint32_t* flags_out, cudaStream_t stream);

int ygx_traverse_status(const void* ws, uint32_t* flags_out, cudaStream_t stream);

/* geometry_to_level_major (yggdrax/_geometry_impl.py:342-420): row l of the
 * (num_levels x max_nodes) outputs holds level l's nodes in nodes_by_level
 * order (nbl32), zero / -1 past the level's count. */
int ygx_level_major_geometry(const int32_t* nbl32, const void* level_offsets, int index_bits,
                             int num_levels, int64_t max_nodes, const float* center,
                             const float* half_extent, const float* radius,
                             const float* max_extent, float* o_center, float* o_half,
                             float* o_radius, float* o_max, void* o_nodes, cudaStream_t stream);

/* _dense_m2l_buffers (yggdrax/dense_interactions.py:34-146): for each of
 * `slots` level-major slots (node_idx, -1 = empty) and k < max_interactions:
 * the k-th source of the node's far row (-1 past its count), the mask, the
 * count per slot and the displacement centre[node] - centre[source]. */
int ygx_dense_m2l(const void* node_idx, int index_bits, int64_t slots, int64_t max_interactions,
                  const void* counts, const void* offsets, const void* sources,
                  const float* center, int64_t total, void* o_src, bool* o_mask, void* o_counts,
                  float* o_disp, cudaStream_t stream);

/* build_grouped_interactions_from_pairs (yggdrax/grouped_interactions.py:
 * 75-200) in two calls on one workspace: ygx_grouped_classes computes every
 * pair's class key (target level, source level, rint in float64 of the
 * displacement over the target level's cell, root_extent a host double[3]),
 * sorts the pairs stably by key and returns the number of classes (host);
 * ygx_grouped_emit then writes the class keys / displacements / offsets, the
 * pairs in class order and each input pair's class id.  Synchronizes. */
size_t ygx_grouped_workspace_size(int64_t num_pairs);
int ygx_grouped_classes(const void* sources, const void* targets, int index_bits,
                        int64_t num_pairs, const int32_t* level32, const float* center,
                        const double* root_extent, int64_t* num_classes_out, void* ws,
                        size_t ws_bytes, cudaStream_t stream);
int ygx_grouped_emit(const void* sources, const void* targets, int index_bits, int64_t num_pairs,
                     const double* root_extent, int32_t* class_keys, float* class_disp,
                     void* class_offsets, void* class_sources, void* class_targets,
                     void* class_ids, void* ws, size_t ws_bytes, cudaStream_t stream);

/* compute_tree_mass_moments / compute_tree_multipole_moments
 * (yggdrax/tree_moments.py:686-877): fp32 prefix sums of mass-weighted
 * monomials over the sorted particles, differenced at node_ranges (nodes x 2,
 * inclusive, index dtype), shifted to `centers` (null: the centres of mass).
 * o_mass / o_com always; with o_packed non-null also the packed coefficients
 * (nodes x C, C = total_coefficients(max_order)) and the tensors (dipole 3,
 * second / quadrupole 9, third / octupole 27, fourth / hexadecapole 81 per
 * node).  Does not synchronize. */
size_t ygx_moments_workspace_size(int64_t n, int max_order);
int ygx_tree_moments(const float* positions_sorted, const float* masses_sorted, int64_t n,
                     const void* node_ranges, int index_bits, int64_t nodes, int max_order,
                     const float* centers, float* o_mass, float* o_com, float* o_center,
                     float* o_packed, float* o_dipole, float* o_second, float* o_quad,
                     float* o_third, float* o_oct, float* o_fourth, float* o_hexa, void* ws,
                     size_t ws_bytes, cudaStream_t stream);

/* dual_tree_walk_mutual (yggdrax/_interactions_impl.py:6357-6560): the
 * symmetric walk that emits every unordered node pair once.  left_full /
 * right_full: children of all `total` nodes (-1 on leaves) in the index dtype;
 * centers (total x 3) and radii (total) are the caller's MAC inputs (accept
 * when theta * |c_b - c_a| > r_a + r_b, strict).  far_a/far_b (far_cap) and
 * near_a/near_b (near_cap) receive the canonical pairs (a < b) in the
 * reference's breadth-first emission order, -1 past the end.  counts_out[2]
 * (host) = far and near pairs the lists would hold (counted past the
 * capacities); flags_out (host): bit 0 far, bit 1 near, bit 2 wavefront
 * (max_pair_queue) overflow -- the walk stops after the generation that set
 * one, like the reference.  Synchronizes once per generation. */
size_t ygx_mutual_walk_workspace_size(int64_t total, int64_t max_pair_queue);
int ygx_mutual_walk(const void* left_full, const void* right_full, int index_bits,
                    const float* centers, const float* radii, int64_t total, float theta,
                    int64_t root, int64_t max_pair_queue, int64_t far_cap, int64_t near_cap,
                    void* far_a, void* far_b, void* near_a, void* near_b, int64_t* counts_out,
                    uint32_t* flags_out, int* gens_out, void* ws, size_t ws_bytes,
                    cudaStream_t stream);

/* compute_explicit_octree_box_geometry (yggdrax/octree.py:422-476): boxes of
 * M octree cells from their (code, depth); valid (uint8), codes (uint64) and
 * depths (index dtype) on the device, bounds_min / bounds_max (3 floats each)
 * on the HOST.  Writes centers / half_extents (M x 3), radii, max_extents
 * (M) in fp32, zeros on invalid cells. */
int ygx_octree_box_geometry(const uint8_t* valid, const uint64_t* codes, const void* depths,
                            int index_bits, int64_t M, const float* bounds_min,
                            const float* bounds_max, float* centers, float* half_extents,
                            float* radii, float* max_extents, cudaStream_t stream);

/* _dual_tree_walk_octree_impl (yggdrax/_interactions_impl.py:1908-2597), the
 * walk behind build_octree_native_far_pairs / build_octree_native_neighbor_lists
 * (:5556-5717), in octree cell space from (root, root).  children (M x 8
 * octant slots, -1 empty) and child_counts in the index dtype; centers /
 * radii / max_extents the cell boxes; leaf_mask (uint8) the leaf test of the
 * node space in use.  Exactly one of far_row / near_row is given: far_row
 * (M, int32) = the log row key of every cell (its position in the level
 * order); near_row (M, int32) = the row of a leaf cell (0..near_rows-1) or
 * -1.  mac 0 bh (box max extent), 1 dehnen (box radius x scale), 2 engblom
 * (box radius).  Every accepted (near) pair is logged twice, per generation
 * first as (row of t, s) then as (row of s, t), into *_key / *_val
 * (log_capacity entries); *_cnt receive the row lengths.  stats_out (host,
 * 8 x int64): far log entries, near log entries, accept, near, refine
 * decisions, generations, the largest wavefront kept.  flags_out (host):
 * bit 0 a far row above far_row_cap, bit 1 a near row above near_row_cap,
 * bit 2 more children than max_pair_queue (the walk stops after that
 * generation, like the reference), bit 4 more children than wf_capacity
 * (re-run with stats_out[6] or more), bit 5 the log was too short (the walk
 * ran on; re-run with stats_out[0] or [1] entries).  Synchronizes once per
 * generation.  A stable sort of the log by key gives the reference's rows. */
size_t ygx_octree_walk_workspace_size(int64_t M, int64_t wf_capacity);
int ygx_octree_walk(const void* children, const void* child_counts, int index_bits, int64_t M,
                    const float* centers, const float* radii, const float* max_extents,
                    const uint8_t* leaf_mask, const int32_t* far_row, const int32_t* near_row,
                    int64_t near_rows, int64_t root, int mac, float theta,
                    float dehnen_radius_scale, int64_t max_pair_queue, int64_t wf_capacity,
                    int64_t far_row_cap, int64_t near_row_cap, int64_t log_capacity,
                    uint64_t* far_key, uint32_t* far_val, uint64_t* near_key,
                    uint32_t* near_val, int32_t* far_cnt, int32_t* near_cnt,
                    int64_t* stats_out, uint32_t* flags_out, void* ws, size_t ws_bytes,
                    cudaStream_t stream);

#ifdef __cplusplus
}
#endif
