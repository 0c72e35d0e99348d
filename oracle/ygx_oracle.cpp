// CPU oracle for the yggdrax tree pipeline -- TEST INFRASTRUCTURE ONLY.
//
// This file restates, function by function, the reference algorithm of the
// yggdrax hot path (Morton encode, stable sort, leaf partitions, Karras
// build, levels, octree tables, geometry, dual-tree walk) in plain C++17 with
// OpenMP.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// legs may load it; the product (yggdrax_b200) never does.
//
// Each function cites the reference file:line it restates (paths relative
// to the reference project root).  Floating-point work is done in IEEE fp32
// with no contraction (the file is compiled with -ffp-contract=off) in the
// operation order the reference writes.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>
#include <deque>
#include <omp.h>

typedef int64_t i64;
typedef uint64_t u64;

namespace {

inline float fmin_nan(float a, float b) {
  // jnp.minimum / lax.min propagate NaN.
  if (std::isnan(a) || std::isnan(b)) return std::numeric_limits<float>::quiet_NaN();
  return a < b ? a : b;
}
inline float fmax_nan(float a, float b) {
  if (std::isnan(a) || std::isnan(b)) return std::numeric_limits<float>::quiet_NaN();
  return a > b ? a : b;
}
inline int clz64(u64 x) { return x ? __builtin_clzll(x) : 64; }

// Vector storage whose resize leaves new elements uninitialised (every
// element is written before it is read), so growing a buffer costs no
// serial zero fill.
template <class T>
struct UninitAlloc : std::allocator<T> {
  template <class U>
  struct rebind { using other = UninitAlloc<U>; };
  UninitAlloc() = default;
  template <class U>
  UninitAlloc(const UninitAlloc<U>&) {}
  template <class U>
  void construct(U* p) noexcept { ::new ((void*)p) U; }
  template <class U, class... A>
  void construct(U* p, A&&... a) { ::new ((void*)p) U(std::forward<A>(a)...); }
};
typedef std::vector<i64, UninitAlloc<i64>> ivec;

// Appends the per-thread buffers bufs[0..nt) to out in thread order (the
// order of the serial loop under a static schedule), copying in parallel.
void concat_parallel(ivec& out, std::vector<ivec>& bufs) {
  const int nt = (int)bufs.size();
  std::vector<size_t> off(nt + 1, out.size());
  for (int q = 0; q < nt; ++q) off[q + 1] = off[q] + bufs[q].size();
  out.resize(off[nt]);
#pragma omp parallel for schedule(static, 1)
  for (int q = 0; q < nt; ++q)
    if (!bufs[q].empty()) std::memcpy(out.data() + off[q], bufs[q].data(), bufs[q].size() * 8);
}


// morton.py:22-30 (_spread3_u64)
inline u64 spread3(u64 x) {
  x &= 0x1FFFFFull;
  x = (x | (x << 32)) & 0x1F00000000FFFFull;
  x = (x | (x << 16)) & 0x1F0000FF0000FFull;
  x = (x | (x << 8)) & 0x100F00F00F00F00Full;
  x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}
// morton.py:32-39 (_compact3_u64)
inline u64 compact3(u64 x) {
  x &= 0x1249249249249249ull;
  x = (x | (x >> 2)) & 0x10C30C30C30C30C3ull;
  x = (x | (x >> 4)) & 0x100F00F00F00F00Full;
  x = (x | (x >> 8)) & 0x1F0000FF0000FFull;
  x = (x | (x >> 16)) & 0x1F00000000FFFFull;
  x = (x | (x >> 32)) & 0x1FFFFFull;
  return x;
}

// XLA shift semantics: a shift by >= 64 gives 0.
inline u64 shr(u64 x, u64 s) { return s >= 64 ? 0 : (x >> s); }
inline u64 shl(u64 x, u64 s) { return s >= 64 ? 0 : (x << s); }

// octree.py:113-133 (_oct_address)
inline u64 oct_address(u64 code, i64 depth) {
  u64 d = (u64)std::max<i64>(0, depth);
  u64 bit_shift = (u64)63 - (u64)3 * d;  // wraps like uint64 for d > 21
  u64 level_prefix = shr(code, bit_shift);
  u64 pow8d = shl(1ull, 3ull * d);
  u64 level_offset = (pow8d - 1ull) / 7ull;
  return level_offset + level_prefix;
}
// octree.py:136-141 (_prefix_code)
inline u64 prefix_code(u64 code, i64 depth) {
  if (depth <= 0) return 0;
  i64 s = std::max<i64>(0, 63 - 3 * depth);
  return shl(shr(code, (u64)s), (u64)s);
}
// octree.py:144-149 (_octant_at_depth)
inline i64 octant_at_depth(u64 code, i64 depth) {
  if (depth <= 0) return 0;
  i64 s = std::max<i64>(0, 63 - 3 * depth);
  return (i64)(shr(code, (u64)s) & 7ull);
}
// octree.py:152-165 (_common_depth_from_codes)
inline i64 common_depth(u64 a, u64 b) {
  u64 x = a ^ b;
  i64 bits = x == 0 ? 63 : std::max<i64>(clz64(x) - 1, 0);
  return bits / 3;
}

// JAX gather index semantics for x[idx] with a signed index: a negative
// index is wrapped by the axis size, then the start index is clamped into
// [0, n-1] (XLA gather clamps out-of-bounds starts).
inline i64 jax_gather_index(i64 idx, i64 n) {
  if (idx < 0) idx += n;
  if (idx < 0) idx = 0;
  if (idx > n - 1) idx = n - 1;
  return idx;
}

// jnp.searchsorted(..., method="scan") restated: a fixed number of halving
// steps over (low, high] starting from (0, n).  For sorted inputs this is an
// ordinary lower/upper bound; the exact step sequence matters when the
// searched array is not sorted (adaptive octree leaf cells).
inline i64 searchsorted_scan(const u64* arr, i64 n, u64 q, bool left) {
  if (n == 0) return 0;
  int levels = 0;
  while ((1ll << levels) < n + 1) ++levels;  // ceil(log2(n + 1))
  i64 lo = 0, hi = n;
  for (int it = 0; it < levels; ++it) {
    i64 mid = (i64)(((u64)lo + (u64)hi) / 2ull);
    bool go_left = left ? (q <= arr[mid]) : (q < arr[mid]);
    if (go_left) hi = mid; else lo = mid;
  }
  return hi;
}

}  // namespace

extern "C" {

int ygo_num_threads() { return omp_get_max_threads(); }
void ygo_set_num_threads(int t) { if (t > 0) omp_set_num_threads(t); }

// ---------------------------------------------------------------------------
// bounds.py:29-33 (infer_bounds): per-axis min/max, padding
// max(span * 0.05f, 1e-6f), returned as (min - pad, max + pad) in fp32.
void ygo_infer_bounds(const float* pos, i64 n, float* out_min, float* out_max) {
  float mn[3] = {INFINITY, INFINITY, INFINITY};
  float mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  bool nan[3] = {false, false, false};
#pragma omp parallel
  {
    float lmn[3] = {INFINITY, INFINITY, INFINITY};
    float lmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    bool lnan[3] = {false, false, false};
#pragma omp for schedule(static)
    for (i64 i = 0; i < n; ++i) {
      for (int a = 0; a < 3; ++a) {
        float v = pos[3 * i + a];
        if (std::isnan(v)) { lnan[a] = true; continue; }
        lmn[a] = std::min(lmn[a], v);
        lmx[a] = std::max(lmx[a], v);
      }
    }
#pragma omp critical
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], lmn[a]);
      mx[a] = std::max(mx[a], lmx[a]);
      nan[a] = nan[a] || lnan[a];
    }
  }
  const float c005 = 0.05f, c1em6 = 1e-6f;
  for (int a = 0; a < 3; ++a) {
    float lo = nan[a] ? NAN : mn[a];
    float hi = nan[a] ? NAN : mx[a];
    float span = hi - lo;
    float pad = fmax_nan(span * c005, c1em6);
    out_min[a] = lo - pad;
    out_max[a] = hi + pad;
  }
}

// ---------------------------------------------------------------------------
// morton.py:43-77 (morton_encode_impl): norm = (p - min) / (max - min),
// clip to [0, 1.0f] (nextafter(1.0, 0.0) rounds to 1.0f against fp32 data),
// rint(norm * 2097151) half-to-even, spread and interleave x | y<<1 | z<<2.
void ygo_morton_encode(const float* pos, i64 n, const float* bmin, const float* bmax,
                       u64* codes) {
  float span[3];
  for (int a = 0; a < 3; ++a) span[a] = bmax[a] - bmin[a];
  const float maxv = 2097151.0f;
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < n; ++i) {
    u64 c[3];
    for (int a = 0; a < 3; ++a) {
      float norm = (pos[3 * i + a] - bmin[a]) / span[a];
      norm = fmin_nan(fmax_nan(norm, 0.0f), 1.0f);
      float v = std::nearbyint(norm * maxv);
      // NaN has no defined integer conversion; map it to 0.
      c[a] = std::isnan(v) ? 0ull : (u64)v;
    }
    codes[i] = spread3(c[0]) | (spread3(c[1]) << 1) | (spread3(c[2]) << 2);
  }
}

// morton.py:83-115 (morton_decode)
void ygo_morton_decode(const u64* codes, i64 n, const float* bmin, const float* bmax,
                       float* pos) {
  const float maxv = 2097151.0f;
  for (i64 i = 0; i < n; ++i) {
    u64 c = codes[i];
    u64 q[3] = {compact3(c), compact3(c >> 1), compact3(c >> 2)};
    for (int a = 0; a < 3; ++a) {
      float norm = (float)q[a] / maxv;
      pos[3 * i + a] = norm * (bmax[a] - bmin[a]) + bmin[a];
    }
  }
}

// ---------------------------------------------------------------------------
// jnp.argsort(codes, stable=True) (_tree_impl.py:401) and
// jnp.lexsort((orig_idx, codes)) (tree.py:403): the same permutation --
// ascending key, ties by original index.  Restated as an LSD radix sort
// (stable by construction) over the bits [0, key_bits).
void ygo_stable_argsort_u64(const u64* keys, i64 n, int key_bits, i64* order) {
  std::vector<i64> a(n), b(n);
  for (i64 i = 0; i < n; ++i) a[i] = i;
  std::vector<u64> ka(keys, keys + n), kb(n);
  if (key_bits <= 0) key_bits = 64;
  const int RB = 11;
  for (int shift = 0; shift < key_bits; shift += RB) {
    i64 cnt[1 << RB];
    std::memset(cnt, 0, sizeof(cnt));
    for (i64 i = 0; i < n; ++i) cnt[(ka[i] >> shift) & ((1 << RB) - 1)]++;
    i64 s = 0;
    for (int d = 0; d < (1 << RB); ++d) { i64 c = cnt[d]; cnt[d] = s; s += c; }
    for (i64 i = 0; i < n; ++i) {
      int d = (ka[i] >> shift) & ((1 << RB) - 1);
      i64 p = cnt[d]++;
      kb[p] = ka[i];
      b[p] = a[i];
    }
    std::swap(a, b);
    std::swap(ka, kb);
  }
  std::memcpy(order, a.data(), sizeof(i64) * n);
}

// ---------------------------------------------------------------------------
// _tree_impl.py:1373-1401 (_fixed_depth_leaf_partitions), depth >= 1:
// bucket = code >> (63 - 3d), bincount over 8^d buckets, exclusive scan,
// dense codes bucket << shift (empty buckets kept), depths = d.
void ygo_fixed_depth_partitions(const u64* sorted_codes, i64 n, int depth, i64* starts,
                                i64* ends, u64* codes, i64* depths) {
  const int shift = std::max(0, 63 - depth * 3);
  const i64 L = (i64)1 << (3 * depth);
  std::vector<i64> counts(L, 0);
  for (i64 i = 0; i < n; ++i) {
    u64 id = sorted_codes[i] >> shift;
    if ((i64)id < L) counts[id]++;
  }
  i64 s = 0;
  for (i64 b = 0; b < L; ++b) {
    starts[b] = s;
    s += counts[b];
    ends[b] = s;
    codes[b] = (u64)b << shift;
    depths[b] = depth;
  }
}

// _tree_impl.py:96-227 (_refine_leaf_partitions_by_aspect), including the
// entry shift 64 - 3*depth (one more than the partitioner's 63 - 3*depth),
// the float64 aspect arithmetic and the final (start, code) ordering.
// Returns the number of output leaves; writes them only if it fits in cap.
i64 ygo_refine(const float* pos_sorted, const u64* sorted_codes, const i64* starts,
               const i64* ends, const u64* codes, const i64* depths, i64 L,
               int current_depth, int max_refine_levels, double aspect_threshold,
               int min_leaf_particles, i64 cap, i64* o_starts, i64* o_ends, u64* o_codes,
               i64* o_depths) {
  struct Item { i64 s, e; u64 code; i64 depth; };
  std::vector<Item> out;
  std::deque<Item> queue;
  for (i64 i = 0; i < L; ++i) queue.push_back({starts[i], ends[i], codes[i], depths[i]});
  const double eps = 1e-12;
  const float eps_f = (float)eps;
  while (!queue.empty()) {
    Item it = queue.front();
    queue.pop_front();
    if (it.e <= it.s) { out.push_back(it); continue; }
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    bool nan[3] = {false, false, false};
    for (i64 p = it.s; p < it.e; ++p)
      for (int a = 0; a < 3; ++a) {
        float v = pos_sorted[3 * p + a];
        if (std::isnan(v)) nan[a] = true;
        mn[a] = std::min(mn[a], v);
        mx[a] = std::max(mx[a], v);
      }
    float ext[3];
    for (int a = 0; a < 3; ++a) ext[a] = nan[a] ? NAN : (mx[a] - mn[a]);
    // numpy .min()/.max() propagate NaN
    float emin = fmin_nan(fmin_nan(ext[0], ext[1]), ext[2]);
    float emax = fmax_nan(fmax_nan(ext[0], ext[1]), ext[2]);
    // max(emin, eps): Python keeps emin unless eps > emin, compared in fp32
    double min_axis = (eps_f > emin) ? eps : (double)emin;
    double max_axis = (double)emax;
    double aspect = (min_axis > 0) ? max_axis / min_axis : INFINITY;
    bool exceeded = (it.depth - current_depth) >= max_refine_levels;
    if (aspect <= aspect_threshold || exceeded) { out.push_back(it); continue; }
    i64 entry_shift = std::max<i64>(0, 64 - it.depth * 3);
    i64 child_depth = it.depth + 1;
    i64 child_shift = entry_shift - 3;
    if (child_shift < 0) { out.push_back(it); continue; }
    i64 cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (i64 p = it.s; p < it.e; ++p) cnt[(sorted_codes[p] >> child_shift) & 7ull]++;
    int nz = 0;
    for (int k = 0; k < 8; ++k) nz += cnt[k] != 0;
    if (nz <= 1) { out.push_back(it); continue; }
    i64 off = it.s;
    for (int sub = 0; sub < 8; ++sub) {
      if (cnt[sub] == 0) continue;
      Item c{off, off + cnt[sub], it.code | ((u64)sub << child_shift), child_depth};
      if (cnt[sub] <= min_leaf_particles) out.push_back(c); else queue.push_back(c);
      off = c.e;
    }
  }
  i64 m = (i64)out.size();
  if (m > cap) return m;
  std::vector<i64> ord(m);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](i64 a, i64 b) {
    if (out[a].s != out[b].s) return out[a].s < out[b].s;
    return out[a].code < out[b].code;
  });
  for (i64 k = 0; k < m; ++k) {
    const Item& it = out[ord[k]];
    o_starts[k] = it.s; o_ends[k] = it.e; o_codes[k] = it.code; o_depths[k] = it.depth;
  }
  return m;
}

// ---------------------------------------------------------------------------
// _tree_impl.py:1115-1270 (Karras 2012 LBVH over leaf codes, num_leaves >= 2).
// delta(i, j): -1 out of range; clz(ci ^ cj), or 64 + clz(i ^ j) for equal
// codes (index tie-break).  Direction, span by a greedy 31-step search,
// split by a codes-only LCP search, children (leaves are num_internal+id),
// and the parent scatter: left writes then right writes, the last writer in
// index order wins (serial scatter).
static inline i64 kdelta(const u64* c, i64 L, i64 i, i64 j) {
  if (j < 0 || j >= L) return -1;
  u64 ci = c[i], cj = c[j];
  if (ci == cj) return 64 + clz64((u64)i ^ (u64)j);
  return clz64(ci ^ cj);
}
static inline i64 lcp_codes(u64 a, u64 b) { return a == b ? 64 : clz64(a ^ b); }

void ygo_karras(const u64* leaf_codes, const i64* leaf_starts, const i64* leaf_ends, i64 L,
                i64* parent, i64* left, i64* right, uint8_t* left_is_leaf,
                uint8_t* right_is_leaf, i64* node_ranges) {
  const i64 ni = L - 1, total = 2 * L - 1;
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < ni; ++i) {
    i64 dp = kdelta(leaf_codes, L, i, i + 1);
    i64 dm = kdelta(leaf_codes, L, i, i - 1);
    i64 d = (dp - dm) > 0 ? 1 : ((dp - dm) < 0 ? -1 : 0);
    if (i == 0) d = 1;
    if (d == 0) d = 1;
    i64 dmin = kdelta(leaf_codes, L, i, i - d);
    i64 span = 0;
    for (int k = 30; k >= 0; --k) {
      i64 step = (i64)1 << k;
      i64 cand = i + (span + step) * d;
      if (cand >= 0 && cand < L && kdelta(leaf_codes, L, i, cand) > dmin) span += step;
    }
    i64 end = i + span * d;
    i64 first = std::min(i, end), last = std::max(i, end);
    node_ranges[2 * i] = leaf_starts[first];
    node_ranges[2 * i + 1] = leaf_ends[last] - 1;
    u64 fc = leaf_codes[first];
    i64 cp = lcp_codes(fc, leaf_codes[last]);
    i64 split = first;
    for (int k = 30; k >= 0; --k) {
      i64 step = (i64)1 << k;
      i64 mid = split + step;
      i64 safe_mid = mid < last ? mid : last;
      i64 cmp = lcp_codes(fc, leaf_codes[safe_mid]);
      if (mid < last && cmp > cp) split = mid;
    }
    bool ll = split == first, rl = split + 1 == last;
    left_is_leaf[i] = ll;
    right_is_leaf[i] = rl;
    left[i] = ll ? ni + first : split;
    right[i] = rl ? ni + last : split + 1;
  }
  for (i64 k = 0; k < total; ++k) parent[k] = -1;
  for (i64 i = 0; i < ni; ++i) parent[left[i]] = i;
  for (i64 i = 0; i < ni; ++i) parent[right[i]] = i;
  for (i64 j = 0; j < L; ++j) {
    node_ranges[2 * (ni + j)] = leaf_starts[j];
    node_ranges[2 * (ni + j) + 1] = leaf_ends[j] - 1;
  }
}

// _tree_impl.py:1272-1316: node depth by pointer doubling over a fixed
// bit_length(total)+1 rounds (synchronous updates), level counts over 64
// bins (out-of-range levels dropped), level offsets (65), nodes_by_level =
// stable argsort of node_level, num_levels = clip(max + 1, 1, 64).
void ygo_levels(const i64* parent, i64 total, i64* node_level, i64* level_offsets,
                i64* nodes_by_level, i64* num_levels) {
  std::vector<i64> sc(total), d(total), sc2(total), d2(total);
  for (i64 k = 0; k < total; ++k) {
    bool root = parent[k] < 0;
    sc[k] = root ? k : parent[k];
    d[k] = root ? 0 : 1;
  }
  int bl = 0;
  while (((i64)1 << bl) <= total) ++bl;  // int.bit_length()
  int rounds = std::max(1, bl + 1);
  for (int r = 0; r < rounds; ++r) {
#pragma omp parallel for schedule(static)
    for (i64 k = 0; k < total; ++k) {
      d2[k] = d[k] + d[sc[k]];
      sc2[k] = sc[sc[k]];
    }
    std::swap(sc, sc2);
    std::swap(d, d2);
  }
  i64 mx = 0;
  std::vector<i64> counts(64, 0);
  for (i64 k = 0; k < total; ++k) {
    node_level[k] = d[k];
    mx = std::max(mx, d[k]);
    if (d[k] >= 0 && d[k] < 64) counts[d[k]]++;
  }
  level_offsets[0] = 0;
  for (int l = 0; l < 64; ++l) level_offsets[l + 1] = level_offsets[l] + counts[l];
  std::vector<i64> ord(total);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](i64 a, i64 b) { return d[a] < d[b]; });
  std::memcpy(nodes_by_level, ord.data(), sizeof(i64) * total);
  *num_levels = std::min<i64>(std::max<i64>(mx + 1, 1), 64);
}

// ---------------------------------------------------------------------------
// octree.py:168-186 (_resolved_leaf_cells), 204-419
// (build_explicit_octree_metadata_from_leaf_partitions) and 479-550
// (build_explicit_octree_metadata): compressed octree cells = leaf cells plus
// consecutive-leaf LCAs, stable address sort + dedup, ranges by scan
// searchsorted over leaf codes, level tables, parent by deepest existing
// ancestor, children by max-scatter, leaf list, radix -> oct maps.
// M = 2L - 1 slots.  Returns num_unique.
i64 ygo_octree_metadata(const i64* node_ranges, i64 total, const u64* morton_codes,
                        i64 n, const u64* leaf_codes_raw, const i64* leaf_depths_raw,
                        i64* oct_parent, i64* oct_children, i64* oct_child_counts,
                        uint8_t* oct_child_mask, uint8_t* oct_valid_mask,
                        u64* oct_node_codes, i64* oct_node_depths, i64* oct_node_ranges,
                        i64* oct_nodes_by_level, i64* oct_level_offsets,
                        i64* oct_num_levels, uint8_t* oct_leaf_mask, i64* oct_leaf_nodes,
                        i64* radix_node_to_oct, i64* radix_leaf_to_oct) {
  const i64 ni = (total - 1) / 2;
  const i64 L = total - ni;
  std::vector<i64> lstart(L), lend(L), ldepth(L);
  std::vector<u64> lcode(L);
  for (i64 j = 0; j < L; ++j) {
    i64 s = node_ranges[2 * (ni + j)], e = node_ranges[2 * (ni + j) + 1];
    lstart[j] = s;
    lend[j] = e + 1;
    u64 first = morton_codes[jax_gather_index(s, n)];
    u64 last = morton_codes[jax_gather_index(e, n)];
    i64 raw = leaf_depths_raw[j];
    i64 dd = raw >= 0 ? raw : common_depth(first, last);
    ldepth[j] = dd;
    lcode[j] = raw >= 0 ? prefix_code(leaf_codes_raw[j], dd) : prefix_code(first, dd);
  }
  const i64 M = std::max<i64>(1, 2 * L - 1);
  std::vector<u64> all_codes(2 * L - 1);
  std::vector<i64> all_depths(2 * L - 1);
  for (i64 j = 0; j < L; ++j) { all_codes[j] = lcode[j]; all_depths[j] = ldepth[j]; }
  for (i64 j = 0; j + 1 < L; ++j) {
    i64 dd = common_depth(lcode[j], lcode[j + 1]);
    all_depths[L + j] = dd;
    all_codes[L + j] = prefix_code(lcode[j], dd);
  }
  const i64 C = 2 * L - 1;
  std::vector<u64> addr(C);
  for (i64 k = 0; k < C; ++k) addr[k] = oct_address(all_codes[k], all_depths[k]);
  std::vector<i64> ord(C);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](i64 a, i64 b) { return addr[a] < addr[b]; });
  for (i64 k = 0; k < M; ++k) {
    oct_node_codes[k] = 0;
    oct_node_depths[k] = -1;
    oct_valid_mask[k] = 0;
  }
  i64 uniq = -1;
  for (i64 k = 0; k < C; ++k) {
    i64 src = ord[k];
    if (k == 0 || addr[src] != addr[ord[k - 1]]) ++uniq;
    oct_node_codes[uniq] = std::max(oct_node_codes[uniq], all_codes[src]);
    oct_node_depths[uniq] = std::max(oct_node_depths[uniq], all_depths[src]);
  }
  const i64 num_unique = uniq + 1;
  for (i64 k = 0; k < M; ++k) oct_valid_mask[k] = k < num_unique;
  // ranges (phase 3)
  for (i64 k = 0; k < M; ++k) {
    bool valid = oct_valid_mask[k];
    u64 dep = (u64)std::max<i64>(oct_node_depths[k], 0);
    u64 bs = (u64)63 - 3ull * dep;
    u64 bs_safe = std::min<u64>(bs, 62);
    u64 mask = shl(1ull, bs_safe) - 1ull;
    u64 endc = valid ? (oct_node_codes[k] | mask) : 0ull;
    i64 f = searchsorted_scan(lcode.data(), L, oct_node_codes[k], true);
    i64 l = searchsorted_scan(lcode.data(), L, endc, false) - 1;
    i64 bound = std::max<i64>(L - 1, 0);
    f = std::min(std::max<i64>(f, 0), bound);
    l = std::min(std::max<i64>(l, 0), bound);
    if (valid) {
      oct_node_ranges[2 * k] = lstart[f];
      oct_node_ranges[2 * k + 1] = lend[l] - 1;
    } else {
      oct_node_ranges[2 * k] = 0;
      oct_node_ranges[2 * k + 1] = -1;
    }
  }
  // level structure (phase 4)
  i64 maxd = 0;
  std::vector<i64> lc(22, 0);
  for (i64 k = 0; k < M; ++k) {
    if (oct_valid_mask[k]) {
      maxd = std::max(maxd, oct_node_depths[k]);
      i64 cd = std::min<i64>(std::max<i64>(oct_node_depths[k], 0), 21);
      lc[cd]++;
    }
  }
  *oct_num_levels = maxd + 1;
  oct_level_offsets[0] = 0;
  for (int l = 0; l < 22; ++l) oct_level_offsets[l + 1] = oct_level_offsets[l] + lc[l];
  {
    std::vector<i64> o(M);
    std::iota(o.begin(), o.end(), 0);
    std::stable_sort(o.begin(), o.end(), [&](i64 a, i64 b) {
      i64 da = oct_valid_mask[a] ? oct_node_depths[a] : 22;
      i64 db = oct_valid_mask[b] ? oct_node_depths[b] : 22;
      return da < db;
    });
    std::memcpy(oct_nodes_by_level, o.data(), sizeof(i64) * M);
  }
  // parent (phase 5)
  const u64 U64MAX = std::numeric_limits<u64>::max();
  std::vector<u64> oaddr(M);
  for (i64 k = 0; k < M; ++k)
    oaddr[k] = oct_valid_mask[k] ? oct_address(oct_node_codes[k], oct_node_depths[k]) : U64MAX;
  for (i64 k = 0; k < M; ++k) oct_parent[k] = -1;
  for (int step = 1; step <= 21; ++step) {
    for (i64 k = 0; k < M; ++k) {
      if (!oct_valid_mask[k] || oct_parent[k] >= 0 || oct_node_depths[k] < step) continue;
      i64 pd = oct_node_depths[k] - step;
      u64 paddr = oct_address(prefix_code(oct_node_codes[k], pd), pd);
      i64 pos = searchsorted_scan(oaddr.data(), M, paddr, true);
      i64 safe = std::min<i64>(pos, M - 1);
      if (oaddr[safe] == paddr) oct_parent[k] = pos;
    }
  }
  // children (phase 6)
  std::vector<i64> cplus(M * 8, 0);
  for (i64 k = 0; k < M; ++k) {
    if (!(oct_valid_mask[k] && oct_parent[k] >= 0)) continue;
    i64 oc = octant_at_depth(oct_node_codes[k], oct_node_depths[k]);
    i64& slot = cplus[oct_parent[k] * 8 + oc];
    slot = std::max(slot, k + 1);
  }
  i64 nleaf = 0;
  for (i64 k = 0; k < M; ++k) {
    i64 cnt = 0;
    for (int c = 0; c < 8; ++c) {
      i64 v = cplus[k * 8 + c] - 1;
      oct_children[k * 8 + c] = v;
      bool m = oct_valid_mask[k] && v >= 0;
      oct_child_mask[k * 8 + c] = m;
      cnt += m;
    }
    oct_child_counts[k] = cnt;
    oct_leaf_mask[k] = oct_valid_mask[k] && cnt == 0;
  }
  for (i64 k = 0; k < M; ++k) oct_leaf_nodes[k] = -1;
  for (i64 k = 0; k < M; ++k)
    if (oct_leaf_mask[k]) oct_leaf_nodes[nleaf++] = k;
  // radix -> oct (build_explicit_octree_metadata, octree.py:513-532)
  for (i64 v = 0; v < total; ++v) {
    i64 dd;
    u64 cc;
    if (v >= ni) {
      dd = ldepth[v - ni];
      cc = lcode[v - ni];
    } else {
      u64 first = morton_codes[jax_gather_index(node_ranges[2 * v], n)];
      u64 last = morton_codes[jax_gather_index(node_ranges[2 * v + 1], n)];
      dd = common_depth(first, last);
      cc = prefix_code(first, dd);
    }
    radix_node_to_oct[v] = searchsorted_scan(oaddr.data(), M, oct_address(cc, dd), true);
  }
  for (i64 j = 0; j < L; ++j) radix_leaf_to_oct[j] = radix_node_to_oct[ni + j];
  return num_unique;
}

// ---------------------------------------------------------------------------
// _geometry_impl.py:176-338 (compute_tree_geometry).
// Leaf bounds: masked min/max over at most `cap` particles of each leaf's
// range (empty -> +FLT_MAX / -FLT_MAX), or Morton cells
// (mins = bmin + (domain / 2^depth) * idx, maxs = mins + cell).
// Upward pass: node depth from the parent array by pointer doubling until
// the shortcuts stop changing, then for level = max_depth-1 .. 0 every
// internal node at that level takes min/max of its children's current
// values (synchronous within a level; internal nodes start at 0).
// Final: center = 0.5*(mn+mx), half = max(0.5*(mx-mn), 1e-6),
// radius = sqrt((h0*h0 + h1*h1) + h2*h2), max_extent = max(h).
// Returns 0, or -1 if the parent array never converges (cyclic).
int ygo_geometry(const i64* node_ranges, i64 total, const i64* left, const i64* right,
                 const i64* parent, const float* pos_sorted, i64 n, int use_morton,
                 const float* bmin, const float* bmax, const u64* leaf_codes,
                 const i64* leaf_depths, i64 max_leaf_size, float* center, float* half,
                 float* radius, float* max_extent) {
  const i64 ni = (total - 1) / 2;
  const i64 L = total - ni;
  std::vector<float> mn(3 * total, 0.0f), mx(3 * total, 0.0f);
  if (use_morton) {
    float dom[3];
    for (int a = 0; a < 3; ++a) dom[a] = bmax[a] - bmin[a];
#pragma omp parallel for schedule(static)
    for (i64 j = 0; j < L; ++j) {
      i64 dc = std::min<i64>(std::max<i64>(leaf_depths[j], 0), 21);
      u64 sh = (u64)(21 - dc);
      u64 code = leaf_codes[j];
      u64 q[3] = {compact3(code) >> sh, compact3(code >> 1) >> sh, compact3(code >> 2) >> sh};
      float cnt = (float)(u64)(1ull << dc);
      for (int a = 0; a < 3; ++a) {
        float cell = dom[a] / cnt;
        float lo = bmin[a] + cell * (float)q[a];
        mn[3 * (ni + j) + a] = lo;
        mx[3 * (ni + j) + a] = lo + cell;
      }
    }
  } else {
    i64 cap = max_leaf_size;
    if (cap < 0) {
      cap = 0;
      for (i64 j = 0; j < L; ++j)
        cap = std::max(cap, node_ranges[2 * (ni + j) + 1] - node_ranges[2 * (ni + j)] + 1);
    }
    const float big = std::numeric_limits<float>::max();
#pragma omp parallel for schedule(static)
    for (i64 j = 0; j < L; ++j) {
      i64 s = node_ranges[2 * (ni + j)];
      i64 c = node_ranges[2 * (ni + j) + 1] - s + 1;
      float lo[3], hi[3];
      for (int a = 0; a < 3; ++a) {
        if (cap == 0) { lo[a] = INFINITY; hi[a] = -INFINITY; } else { lo[a] = big; hi[a] = -big; }
      }
      for (i64 k = 0; k < std::min(c, cap); ++k) {
        i64 p = s + k;
        for (int a = 0; a < 3; ++a) {
          float v = pos_sorted[3 * p + a];
          lo[a] = fmin_nan(lo[a], v);
          hi[a] = fmax_nan(hi[a], v);
        }
      }
      for (int a = 0; a < 3; ++a) { mn[3 * (ni + j) + a] = lo[a]; mx[3 * (ni + j) + a] = hi[a]; }
    }
  }
  if (ni > 0) {
    std::vector<i64> sc(total), d(total), sc2(total), d2(total);
    for (i64 k = 0; k < total; ++k) {
      bool root = parent[k] < 0;
      sc[k] = root ? k : parent[k];
      d[k] = root ? 0 : 1;
    }
    bool changed = true;
    int guard = 0;
    while (changed) {
      if (++guard > 200) return -1;
      changed = false;
      for (i64 k = 0; k < total; ++k) {
        d2[k] = d[k] + d[sc[k]];
        sc2[k] = sc[sc[k]];
        if (sc2[k] != sc[k]) changed = true;
      }
      std::swap(sc, sc2);
      std::swap(d, d2);
    }
    i64 maxd = 0;
    for (i64 k = 0; k < total; ++k) maxd = std::max(maxd, d[k]);
    std::vector<std::vector<i64>> by_level(std::max<i64>(maxd, 0) + 1);
    for (i64 i = 0; i < ni; ++i)
      if (d[i] >= 0 && d[i] <= maxd) by_level[d[i]].push_back(i);
    std::vector<float> tmp;
    for (i64 level = maxd - 1; level >= 0; --level) {
      const auto& nodes = by_level[level];
      tmp.resize(6 * nodes.size());
      for (size_t t = 0; t < nodes.size(); ++t) {
        i64 i = nodes[t];
        for (int a = 0; a < 3; ++a) {
          tmp[6 * t + a] = fmin_nan(mn[3 * left[i] + a], mn[3 * right[i] + a]);
          tmp[6 * t + 3 + a] = fmax_nan(mx[3 * left[i] + a], mx[3 * right[i] + a]);
        }
      }
      for (size_t t = 0; t < nodes.size(); ++t) {
        i64 i = nodes[t];
        for (int a = 0; a < 3; ++a) { mn[3 * i + a] = tmp[6 * t + a]; mx[3 * i + a] = tmp[6 * t + 3 + a]; }
      }
    }
  }
  const float c05 = 0.5f, cmin = 1e-6f;
#pragma omp parallel for schedule(static)
  for (i64 k = 0; k < total; ++k) {
    float h[3];
    for (int a = 0; a < 3; ++a) {
      float lo = mn[3 * k + a], hi = mx[3 * k + a];
      center[3 * k + a] = c05 * (lo + hi);
      h[a] = fmax_nan(c05 * (hi - lo), cmin);
      half[3 * k + a] = h[a];
    }
    float s = h[0] * h[0];
    s = s + h[1] * h[1];
    s = s + h[2] * h[2];
    radius[k] = std::sqrt(s);
    max_extent[k] = fmax_nan(fmax_nan(h[0], h[1]), h[2]);
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Dual-tree walk: _interactions_impl.py:338-395 (MAC), 713-728 (actions),
// 1262-1310 / 174-221 (refinement), 1119-1905 / 2600-3558 (wavefront walk
// from (root, root) with canonical (min, max) pairs).  The oracle runs the
// same BFS generations, records every accepted and near canonical pair
// once, and counts decisions.  mac: 0 = bh, 1 = dehnen, 2 = engblom;
// `ext` are the per-node MAC extents already selected and scaled.
// Pairs are packed as (first << 32) | second (node ids stay below 2^31); a
// pair with a missing (-1) node packs to -1 and is skipped when evaluated.
inline i64 pack2(i64 a, i64 b) {
  return (a < 0 || b < 0) ? -1 : (i64)(((u64)a << 32) | (u64)(uint32_t)b);
}
inline i64 first2(i64 p) { return (i64)((u64)p >> 32); }
inline i64 second2(i64 p) { return (i64)(uint32_t)(u64)p; }

struct WalkResult {
  ivec far, nearp;  // accepted / near canonical pairs (lo, hi), packed
  i64 accept = 0, nearc = 0, refine = 0, max_wf = 1, generations = 0;
};

void* ygo_walk(const float* center, const float* ext, const i64* left, const i64* right,
               i64 total, i64 ni, float theta_sq, int mac, i64 root) {
  WalkResult* R = new WalkResult();
  ivec wf{pack2(root, root)}, nwf;
  const float theta = std::sqrt(theta_sq);
  const int nt = omp_get_max_threads();
  // per-thread buffers, kept (with their capacity) across generations; each
  // thread fills private copies and swaps them in (no shared cache lines)
  std::vector<ivec> nt_w(nt), fl(nt), nl(nt);
  while (!wf.empty()) {
    R->generations++;
    const i64 W = (i64)wf.size();
    std::vector<i64> acc(nt, 0), nrc(nt, 0), ref(nt, 0);
#pragma omp parallel num_threads(nt)
    {
      const int tid = omp_get_thread_num();
      ivec Pw, Fl, Nl;
      Pw.swap(nt_w[tid]); Fl.swap(fl[tid]); Nl.swap(nl[tid]);
      Pw.clear(); Fl.clear(); Nl.clear();
      i64 a_ = 0, n_ = 0, r_ = 0;
#pragma omp for schedule(static)
      for (i64 k = 0; k < W; ++k) {
        if (wf[k] < 0) continue;
        const i64 t = first2(wf[k]), s = second2(wf[k]);
        float dx = center[3 * t] - center[3 * s];
        float dy = center[3 * t + 1] - center[3 * s + 1];
        float dz = center[3 * t + 2] - center[3 * s + 2];
        float d2 = dx * dx;
        d2 = d2 + dy * dy;
        d2 = d2 + dz * dz;
        bool diff = t != s;
        float et = ext[t], es = ext[s];
        bool ok;
        if (mac == 2) {
          float big = fmax_nan(et, es), small = fmin_nan(et, es);
          float lhs = big + theta * small;
          ok = lhs * lhs <= theta_sq * d2;
        } else {
          float sum = et + es;
          ok = sum * sum <= theta_sq * d2;
        }
        bool mac_ok = diff && (d2 > 0.0f) && ok;
        bool t_int = t < ni, s_int = s < ni;
        if (mac_ok) {
          a_++;
          Fl.push_back(pack2(t, s));
          continue;
        }
        if (!t_int && !s_int && diff) {
          n_++;
          Nl.push_back(pack2(t, s));
          continue;
        }
        r_++;
        bool same = t == s;
        bool st = t_int && (same || !s_int || et >= es);
        bool ss = s_int && (same || !t_int || es > et);
        auto push = [&](i64 a, i64 b) { Pw.push_back(pack2(std::min(a, b), std::max(a, b))); };
        if (st && ss) {
          if (same) {
            push(left[t], left[t]); push(left[t], right[t]); push(right[t], right[t]);
          } else {
            push(left[t], left[s]); push(left[t], right[s]);
            push(right[t], left[s]); push(right[t], right[s]);
          }
        } else if (st) {
          push(left[t], s); push(right[t], s);
        } else if (ss) {
          push(t, left[s]); push(t, right[s]);
        }
      }
      acc[tid] = a_; nrc[tid] = n_; ref[tid] = r_;
      nt_w[tid].swap(Pw); fl[tid].swap(Fl); nl[tid].swap(Nl);
    }
    nwf.clear();
    concat_parallel(nwf, nt_w);
    concat_parallel(R->far, fl);
    concat_parallel(R->nearp, nl);
    for (int q = 0; q < nt; ++q) { R->accept += acc[q]; R->nearc += nrc[q]; R->refine += ref[q]; }
    wf.swap(nwf);
    R->max_wf = std::max<i64>(R->max_wf, (i64)wf.size());
    if (R->generations > 100000) break;
  }
  return R;
}

// sizes: [num_far_pairs, num_near_pairs, accept, near, refine, max_wf, generations]
void ygo_walk_sizes(void* h, i64* out) {
  WalkResult* R = (WalkResult*)h;
  out[0] = (i64)R->far.size(); out[1] = (i64)R->nearp.size();
  out[2] = R->accept; out[3] = R->nearc; out[4] = R->refine; out[5] = R->max_wf;
  out[6] = R->generations;
}

// Directed lists in the reference's output layouts (_interactions_impl.py
// 3561-3637 and 3640-3837), rows in canonical (ascending) order:
//  far:  counts per node; entries ordered level-major by target rank in
//        nodes_by_level, sources ascending within a target;
//        node_offsets[node] = start of that node's slice.
//  near: counts per leaf position; CSR rows in leaf-position order,
//        neighbour node ids ascending within a row.
void ygo_walk_lists(void* h, i64 total, const i64* nodes_by_level, const i64* leaf_position,
                    i64 L, i64* far_counts, i64* node_offsets, i64* far_sources,
                    i64* far_targets, i64* near_counts, i64* near_offsets,
                    i64* near_neighbors) {
  // Rows are sorted at the end, so entries may be placed in any order: the
  // scatters run in parallel with atomic row cursors.
  WalkResult* R = (WalkResult*)h;
  const i64 P = (i64)R->far.size();
  const i64* fp = R->far.data();
  std::vector<i64> cnt(total, 0);
#pragma omp parallel for schedule(static)
  for (i64 k = 0; k < P; ++k) {
    __atomic_fetch_add(&cnt[first2(fp[k])], 1, __ATOMIC_RELAXED);
    __atomic_fetch_add(&cnt[second2(fp[k])], 1, __ATOMIC_RELAXED);
  }
  std::vector<i64> start(total + 1, 0);  // by rank
  for (i64 r = 0; r < total; ++r) start[r + 1] = start[r] + cnt[nodes_by_level[r]];
#pragma omp parallel for schedule(static)
  for (i64 r = 0; r < total; ++r) {
    const i64 v = nodes_by_level[r];
    far_counts[v] = cnt[v];
    node_offsets[v] = start[r];
  }
  node_offsets[total] = 2 * P;
  std::vector<i64> cur(node_offsets, node_offsets + total);
#pragma omp parallel for schedule(static)
  for (i64 k = 0; k < P; ++k) {
    const i64 a = first2(fp[k]), b = second2(fp[k]);
    const i64 pa = __atomic_fetch_add(&cur[a], 1, __ATOMIC_RELAXED);
    far_sources[pa] = b; far_targets[pa] = a;
    const i64 pb = __atomic_fetch_add(&cur[b], 1, __ATOMIC_RELAXED);
    far_sources[pb] = a; far_targets[pb] = b;
  }
#pragma omp parallel for schedule(dynamic, 256)
  for (i64 v = 0; v < total; ++v)
    std::sort(far_sources + node_offsets[v], far_sources + node_offsets[v] + cnt[v]);
  const i64 Q = (i64)R->nearp.size();
  const i64* np_ = R->nearp.data();
  std::vector<i64> ncnt(L, 0);
#pragma omp parallel for schedule(static)
  for (i64 k = 0; k < Q; ++k) {
    __atomic_fetch_add(&ncnt[leaf_position[first2(np_[k])]], 1, __ATOMIC_RELAXED);
    __atomic_fetch_add(&ncnt[leaf_position[second2(np_[k])]], 1, __ATOMIC_RELAXED);
  }
  near_offsets[0] = 0;
  for (i64 j = 0; j < L; ++j) { near_counts[j] = ncnt[j]; near_offsets[j + 1] = near_offsets[j] + ncnt[j]; }
  std::vector<i64> ncur(near_offsets, near_offsets + L);
#pragma omp parallel for schedule(static)
  for (i64 k = 0; k < Q; ++k) {
    const i64 a = first2(np_[k]), b = second2(np_[k]);
    near_neighbors[__atomic_fetch_add(&ncur[leaf_position[a]], 1, __ATOMIC_RELAXED)] = b;
    near_neighbors[__atomic_fetch_add(&ncur[leaf_position[b]], 1, __ATOMIC_RELAXED)] = a;
  }
#pragma omp parallel for schedule(dynamic, 256)
  for (i64 j = 0; j < L; ++j)
    std::sort(near_neighbors + near_offsets[j], near_neighbors + near_offsets[j + 1]);
}

void ygo_walk_free(void* h) { delete (WalkResult*)h; }

}  // extern "C"
