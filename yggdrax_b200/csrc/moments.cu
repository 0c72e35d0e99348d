// Per-node mass and multipole moments (yggdrax/tree_moments.py:686-877).
//
// The reference forms, for every particle, the mass-weighted monomials
// m x^a y^b z^c of all multi-indices up to the order (packed layout: level by
// level, multi_index_tuples order), takes their prefix sums over the
// Morton-sorted particles, differences them at each node's particle range,
// and shifts the raw sums to the node's expansion centre with the binomial
// stencil; the tensors (second ... fourth moments and their trace-free
// quadrupole / octupole / hexadecapole) follow per node.  Here:
//   k_monomials   one thread per particle, columns in a (C, N) layout,
//   k_col_scan_*  fp32 inclusive prefix per column (reduce, scan the tile
//                 sums, rescan), so the column sums are O(N) work,
//   k_node_moments one thread per node: range differences, centre of mass,
//                 the shift to the expansion centre and the STF tensors.
// Arithmetic follows the reference's written fp32 order (cumprod powers,
// left-to-right monomial products, sequential sums over the stencil); the
// prefix sums are a parallel scan, so values agree with the reference to fp32
// rounding of the prefix sums, not bit for bit.
#include "common.cuh"

namespace ygx {

namespace {

constexpr int kMaxOrder = 4;
constexpr int kMaxCoef = 35;  // total_coefficients(4)
constexpr int kScanTileF = 2048;

struct Combos {
  unsigned char a[kMaxCoef], b[kMaxCoef], c[kMaxCoef];
  int count;
};

// multi_index_tuples(level) for level 0..order, concatenated (multipole_utils.py)
Combos make_combos(int order) {
  Combos k{};
  int n = 0;
  for (int lv = 0; lv <= order; ++lv)
    for (int i = 0; i <= lv; ++i)
      for (int j = 0; j <= lv - i; ++j) {
        k.a[n] = (unsigned char)i;
        k.b[n] = (unsigned char)j;
        k.c[n] = (unsigned char)(lv - i - j);
        ++n;
      }
  k.count = n;
  return k;
}

// cumprod([1, v, v, v, v])[p]
__device__ __forceinline__ void powers(float v, float p[kMaxOrder + 1]) {
  p[0] = 1.0f;
  for (int k = 1; k <= kMaxOrder; ++k) p[k] = __fmul_rn(p[k - 1], v);
}

__global__ void k_monomials(const float* __restrict__ pos, const float* __restrict__ mass,
                            int64_t n, Combos cb, float* __restrict__ cols) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float px[kMaxOrder + 1], py[kMaxOrder + 1], pz[kMaxOrder + 1];
    powers(pos[3 * i], px);
    powers(pos[3 * i + 1], py);
    powers(pos[3 * i + 2], pz);
    const float m = mass[i];
    for (int c = 0; c < cb.count; ++c) {
      const float mono = __fmul_rn(__fmul_rn(px[cb.a[c]], py[cb.b[c]]), pz[cb.c[c]]);
      cols[(int64_t)c * n + i] = __fmul_rn(m, mono);
    }
  }
}

// Tile sums of every column: tile t of column c sums elements
// [t * kScanTileF, (t + 1) * kScanTileF).
__global__ void k_col_tile_sums(const float* __restrict__ cols, int64_t n, int64_t tiles,
                                float* __restrict__ tile_sums) {
  const int c = blockIdx.y;
  const float* col = cols + (int64_t)c * n;
  __shared__ float s_w[32];
  for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int64_t base = t * kScanTileF;
    float acc = 0.0f;
    for (int k = threadIdx.x; k < kScanTileF; k += blockDim.x)
      acc = __fadd_rn(acc, base + k < n ? col[base + k] : 0.0f);
    for (int o = 16; o > 0; o >>= 1) acc = __fadd_rn(acc, __shfl_xor_sync(0xffffffffu, acc, o));
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      float s = 0.0f;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s = __fadd_rn(s, s_w[w]);
      tile_sums[(int64_t)c * tiles + t] = s;
    }
    __syncthreads();
  }
}

// Exclusive prefix of each column's tile sums (one CTA per column, serial
// over the tiles in chunks of the block).
__global__ void k_col_tile_scan(float* __restrict__ tile_sums, int64_t tiles) {
  const int c = blockIdx.x;
  float* ts = tile_sums + (int64_t)c * tiles;
  __shared__ float s[1024];
  float carry = 0.0f;
  for (int64_t b0 = 0; b0 < tiles; b0 += blockDim.x) {
    const int64_t k = b0 + threadIdx.x;
    const float v = k < tiles ? ts[k] : 0.0f;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < (int)blockDim.x; off <<= 1) {
      const float add = (int)threadIdx.x >= off ? s[threadIdx.x - off] : 0.0f;
      __syncthreads();
      s[threadIdx.x] = __fadd_rn(s[threadIdx.x], add);
      __syncthreads();
    }
    const float incl = s[threadIdx.x];
    if (k < tiles) ts[k] = __fadd_rn(carry, __fsub_rn(incl, v));  // exclusive
    __syncthreads();
    carry = __fadd_rn(carry, s[blockDim.x - 1]);
    __syncthreads();
  }
}

// prefix[c][i + 1] = inclusive prefix of column c at element i; prefix[c][0] = 0.
__global__ void k_col_rescan(const float* __restrict__ cols, int64_t n, int64_t tiles,
                             const float* __restrict__ tile_off, float* __restrict__ prefix) {
  const int c = blockIdx.y;
  const float* col = cols + (int64_t)c * n;
  float* pre = prefix + (int64_t)c * (n + 1);
  __shared__ float s[kScanTileF];
  for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
    const int64_t base = t * kScanTileF;
    for (int k = threadIdx.x; k < kScanTileF; k += blockDim.x)
      s[k] = base + k < n ? col[base + k] : 0.0f;
    __syncthreads();
    // one thread per 8 consecutive elements: serial within, scan across
    constexpr int kPer = kScanTileF / 256;
    float loc[kPer];
    float run = 0.0f;
    const int t0 = threadIdx.x * kPer;
    for (int k = 0; k < kPer; ++k) {
      run = __fadd_rn(run, s[t0 + k]);
      loc[k] = run;
    }
    __shared__ float s_sum[256];
    s_sum[threadIdx.x] = run;
    __syncthreads();
    for (int off = 1; off < 256; off <<= 1) {
      const float add = (int)threadIdx.x >= off ? s_sum[threadIdx.x - off] : 0.0f;
      __syncthreads();
      s_sum[threadIdx.x] = __fadd_rn(s_sum[threadIdx.x], add);
      __syncthreads();
    }
    const float before = __fadd_rn(tile_off[(int64_t)c * tiles + t],
                                   threadIdx.x > 0 ? s_sum[threadIdx.x - 1] : 0.0f);
    for (int k = 0; k < kPer; ++k) {
      const int64_t i = base + t0 + k;
      if (i < n) pre[i + 1] = __fadd_rn(before, loc[k]);
    }
    if (t == 0 && threadIdx.x == 0) pre[0] = 0.0f;
    __syncthreads();
  }
}

struct Stencil {
  float binom[kMaxCoef * kMaxCoef];     // 0 where beta > alpha
  unsigned char gx[kMaxCoef * kMaxCoef], gy[kMaxCoef * kMaxCoef], gz[kMaxCoef * kMaxCoef];
};

// One thread per node: raw range sums, mass / centre of mass, the binomial
// shift to the expansion centre (centre of mass, or `centers` when given), and
// the tensors.  Outputs (per node): mass, com (3), center (3), packed (C),
// dipole (3), second (9), quad (9), third (27), oct (27), fourth (81), hexa (81).
__global__ void k_node_moments(const float* __restrict__ prefix, int64_t n,
                               const void* ranges, int index_bits, int64_t nodes, int order,
                               int C, int Ccols, Combos cb, const Stencil* __restrict__ st,
                               const float* __restrict__ centers, float* __restrict__ o_mass,
                               float* __restrict__ o_com, float* __restrict__ o_center,
                               float* __restrict__ o_packed, float* __restrict__ o_dipole,
                               float* __restrict__ o_second, float* __restrict__ o_quad,
                               float* __restrict__ o_third, float* __restrict__ o_oct,
                               float* __restrict__ o_fourth, float* __restrict__ o_hexa) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nodes;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = load_idx(ranges, index_bits, 2 * q);
    const int64_t e = load_idx(ranges, index_bits, 2 * q + 1) + 1;
    float raw[kMaxCoef];
    for (int c = 0; c < Ccols; ++c)
      raw[c] = __fsub_rn(prefix[(int64_t)c * (n + 1) + e], prefix[(int64_t)c * (n + 1) + s]);
    // compute_tree_mass_moments: mass, centre of mass (0 for massless nodes);
    // the weighted-position columns are the level-1 combos (1,0,0), (0,1,0),
    // (0,0,1) = packed indices 3, 2, 1
    const float m = raw[0];
    const float safe = m == 0.0f ? 1.0f : m;
    float com[3];
    if (Ccols >= 4) {
      com[0] = m == 0.0f ? 0.0f : __fdiv_rn(raw[3], safe);
      com[1] = m == 0.0f ? 0.0f : __fdiv_rn(raw[2], safe);
      com[2] = m == 0.0f ? 0.0f : __fdiv_rn(raw[1], safe);
    } else {
      com[0] = com[1] = com[2] = 0.0f;
    }
    o_mass[q] = m;
    if (o_com)
      for (int a = 0; a < 3; ++a) o_com[3 * q + a] = com[a];
    if (!o_packed) continue;
    float ctr[3];
    for (int a = 0; a < 3; ++a) ctr[a] = centers ? centers[3 * q + a] : com[a];
    for (int a = 0; a < 3; ++a) o_center[3 * q + a] = ctr[a];
    float px[kMaxOrder + 1], py[kMaxOrder + 1], pz[kMaxOrder + 1];
    powers(-ctr[0], px);
    powers(-ctr[1], py);
    powers(-ctr[2], pz);
    float pk[kMaxCoef];
    for (int i = 0; i < C; ++i) {
      float acc = 0.0f;
      for (int j = 0; j < C; ++j) {
        const int ij = i * kMaxCoef + j;
        const float b = st->binom[ij];
        float tr = 0.0f;
        if (b != 0.0f) {
          const float cf = __fmul_rn(__fmul_rn(px[st->gx[ij]], py[st->gy[ij]]), pz[st->gz[ij]]);
          tr = __fmul_rn(cf, b);  // (centre factor * mask) * binomial
        }
        acc = __fadd_rn(acc, __fmul_rn(tr, raw[j]));
      }
      pk[i] = acc;
      o_packed[q * C + i] = acc;
    }
    // tensors (_moments_from_raw_packed, :312-395); combo index by (i, j, k)
    auto idx = [&](int a, int b, int c) -> int {
      for (int t = 0; t < C; ++t)
        if (cb.a[t] == a && cb.b[t] == b && cb.c[t] == c) return t;
      return -1;
    };
    const bool zero = pk[0] == 0.0f;
    float dip[3] = {0.0f, 0.0f, 0.0f};
    if (order >= 1) {
      dip[0] = pk[idx(1, 0, 0)];
      dip[1] = pk[idx(0, 1, 0)];
      dip[2] = pk[idx(0, 0, 1)];
    }
    for (int a = 0; a < 3; ++a) o_dipole[3 * q + a] = zero ? 0.0f : dip[a];
    // symmetric tensors of order 2..4 from the packed level values
    float sec[9], thr[27], fou[81];
    for (int i = 0; i < 9; ++i) sec[i] = 0.0f;
    for (int i = 0; i < 27; ++i) thr[i] = 0.0f;
    for (int i = 0; i < 81; ++i) fou[i] = 0.0f;
    if (order >= 2)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
          int cnt[3] = {0, 0, 0};
          ++cnt[i];
          ++cnt[j];
          sec[3 * i + j] = pk[idx(cnt[0], cnt[1], cnt[2])];
        }
    if (order >= 3)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k) {
            int cnt[3] = {0, 0, 0};
            ++cnt[i];
            ++cnt[j];
            ++cnt[k];
            thr[9 * i + 3 * j + k] = pk[idx(cnt[0], cnt[1], cnt[2])];
          }
    if (order >= 4)
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k)
            for (int l = 0; l < 3; ++l) {
              int cnt[3] = {0, 0, 0};
              ++cnt[i];
              ++cnt[j];
              ++cnt[k];
              ++cnt[l];
              fou[27 * i + 9 * j + 3 * k + l] = pk[idx(cnt[0], cnt[1], cnt[2])];
            }
    // quadrupole = 3 S - tr(S) I
    const float trace = __fadd_rn(__fadd_rn(sec[0], sec[4]), sec[8]);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        float v = __fmul_rn(3.0f, sec[3 * i + j]);
        v = __fsub_rn(v, i == j ? trace : 0.0f);
        o_quad[9 * q + 3 * i + j] = zero ? 0.0f : v;
        o_second[9 * q + 3 * i + j] = zero ? 0.0f : sec[3 * i + j];
      }
    // octupole (:233-256)
    float r2rk[3];
    for (int k = 0; k < 3; ++k)
      r2rk[k] = __fadd_rn(__fadd_rn(thr[0 + k], thr[12 + k]), thr[24 + k]);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) {
          float v = 0.0f;
          if (order >= 3) {
            v = __fmul_rn(5.0f, thr[9 * i + 3 * j + k]);
            if (i == j) v = __fsub_rn(v, r2rk[k]);
            if (i == k) v = __fsub_rn(v, r2rk[j]);
            if (j == k) v = __fsub_rn(v, r2rk[i]);
          }
          o_oct[27 * q + 9 * i + 3 * j + k] = zero ? 0.0f : v;
          o_third[27 * q + 9 * i + 3 * j + k] = zero ? 0.0f : thr[9 * i + 3 * j + k];
        }
    // hexadecapole (:258-298)
    float r2[9];
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < 3; ++l)
        r2[3 * k + l] = __fadd_rn(__fadd_rn(fou[0 * 27 + 0 * 9 + 3 * k + l],
                                            fou[1 * 27 + 1 * 9 + 3 * k + l]),
                                  fou[2 * 27 + 2 * 9 + 3 * k + l]);
    const float r4 = __fadd_rn(
        __fadd_rn(__fadd_rn(fou[0], fou[40]), fou[80]),
        __fmul_rn(2.0f, __fadd_rn(__fadd_rn(fou[0 * 27 + 0 * 9 + 3 * 1 + 1],
                                            fou[0 * 27 + 0 * 9 + 3 * 2 + 2]),
                                  fou[1 * 27 + 1 * 9 + 3 * 2 + 2])));
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k)
          for (int l = 0; l < 3; ++l) {
            const int at = 27 * i + 9 * j + 3 * k + l;
            float v = 0.0f;
            if (order >= 4) {
              v = __fmul_rn(35.0f, fou[at]);
              float term = 0.0f;
              if (i == j) term = __fadd_rn(term, r2[3 * k + l]);
              if (i == k) term = __fadd_rn(term, r2[3 * j + l]);
              if (i == l) term = __fadd_rn(term, r2[3 * j + k]);
              if (j == k) term = __fadd_rn(term, r2[3 * i + l]);
              if (j == l) term = __fadd_rn(term, r2[3 * i + k]);
              if (k == l) term = __fadd_rn(term, r2[3 * i + j]);
              v = __fsub_rn(v, __fmul_rn(5.0f, term));
              int df = 0;
              if (i == j && k == l) ++df;
              if (i == k && j == l) ++df;
              if (i == l && j == k) ++df;
              if (df) v = __fadd_rn(v, __fmul_rn(r4, (float)df));
            }
            o_hexa[81 * q + at] = zero ? 0.0f : v;
            o_fourth[81 * q + at] = zero ? 0.0f : fou[at];
          }
  }
}

int64_t comb(int n, int k) {
  if (k < 0 || k > n) return 0;
  int64_t r = 1;
  for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
  return r;
}

}  // namespace

}  // namespace ygx

extern "C" {

size_t ygx_moments_workspace_size(int64_t n, int max_order) {
  if (max_order < 0 || max_order > ygx::kMaxOrder || n < 1) return 0;
  const int oc = max_order < 1 ? 1 : max_order;  // the centre of mass needs order 1
  const int C = (oc + 1) * (oc + 2) * (oc + 3) / 6;
  const int64_t tiles = (n + ygx::kScanTileF - 1) / ygx::kScanTileF;
  ygx::Arena a{nullptr, 0, 0};
  a.take<float>((size_t)C * n);
  a.take<float>((size_t)C * (n + 1));
  a.take<float>((size_t)C * tiles);
  a.take<ygx::Stencil>(1);
  return a.used + 256;
}

// Mass moments (compute_tree_mass_moments, tree_moments.py:686-744) when
// o_packed is null; otherwise also the multipole moments about `centers`
// (null: the centres of mass) through max_order (compute_tree_multipole_moments,
// :747-877).  ranges: the topology's node_ranges (nodes x 2, inclusive) in the
// index dtype.  Does not synchronize.
int ygx_tree_moments(const float* positions_sorted, const float* masses_sorted, int64_t n,
                     const void* node_ranges, int index_bits, int64_t nodes, int max_order,
                     const float* centers, float* o_mass, float* o_com, float* o_center,
                     float* o_packed, float* o_dipole, float* o_second, float* o_quad,
                     float* o_third, float* o_oct, float* o_fourth, float* o_hexa, void* ws,
                     size_t ws_bytes, cudaStream_t stream) {
  if (n < 1 || nodes < 1 || max_order < 0 || max_order > ygx::kMaxOrder || !positions_sorted ||
      !masses_sorted || !node_ranges || !o_mass || (index_bits != 32 && index_bits != 64))
    return YGX_ERR_ARG;
  if (o_packed && (!o_center || !o_dipole || !o_second || !o_quad || !o_third || !o_oct ||
                   !o_fourth || !o_hexa))
    return YGX_ERR_ARG;
  if (ws_bytes < ygx_moments_workspace_size(n, max_order)) return YGX_ERR_ARG;
  // columns through order max(max_order, 1): the centre of mass needs the
  // weighted positions; the packed output holds C coefficients
  const int order = o_packed ? max_order : 0;
  const int oc = max_order < 1 ? 1 : max_order;
  const int Ccols = (oc + 1) * (oc + 2) * (oc + 3) / 6;
  const int C = (order + 1) * (order + 2) * (order + 3) / 6;
  const int64_t tiles = (n + ygx::kScanTileF - 1) / ygx::kScanTileF;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  float* cols = a.take<float>((size_t)Ccols * n);
  float* prefix = a.take<float>((size_t)Ccols * (n + 1));
  float* tsum = a.take<float>((size_t)Ccols * tiles);
  ygx::Stencil* st = a.take<ygx::Stencil>(1);
  const ygx::Combos cb = ygx::make_combos(oc);
  // translation stencil: binomial(alpha, beta) and gamma = alpha - beta
  static thread_local ygx::Stencil h;
  for (int i = 0; i < ygx::kMaxCoef; ++i)
    for (int j = 0; j < ygx::kMaxCoef; ++j) {
      const int ij = i * ygx::kMaxCoef + j;
      h.binom[ij] = 0.0f;
      h.gx[ij] = h.gy[ij] = h.gz[ij] = 0;
      if (i < C && j < C && cb.a[i] >= cb.a[j] && cb.b[i] >= cb.b[j] && cb.c[i] >= cb.c[j]) {
        h.binom[ij] = (float)(ygx::comb(cb.a[i], cb.a[j]) * ygx::comb(cb.b[i], cb.b[j]) *
                              ygx::comb(cb.c[i], cb.c[j]));
        h.gx[ij] = (unsigned char)(cb.a[i] - cb.a[j]);
        h.gy[ij] = (unsigned char)(cb.b[i] - cb.b[j]);
        h.gz[ij] = (unsigned char)(cb.c[i] - cb.c[j]);
      }
    }
  if (o_packed &&
      cudaMemcpyAsync(st, &h, sizeof(h), cudaMemcpyHostToDevice, stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  ygx::k_monomials<<<ygx::grid_for(n, 256), 256, 0, stream>>>(positions_sorted, masses_sorted, n,
                                                              cb, cols);
  YGX_CHECK_LAUNCH();
  const dim3 g2((unsigned)(tiles < 65535 ? tiles : 65535), (unsigned)Ccols);
  ygx::k_col_tile_sums<<<g2, 256, 0, stream>>>(cols, n, tiles, tsum);
  YGX_CHECK_LAUNCH();
  ygx::k_col_tile_scan<<<Ccols, 1024, 0, stream>>>(tsum, tiles);
  YGX_CHECK_LAUNCH();
  ygx::k_col_rescan<<<g2, 256, 0, stream>>>(cols, n, tiles, tsum, prefix);
  YGX_CHECK_LAUNCH();
  ygx::k_node_moments<<<ygx::grid_for(nodes, 128), 128, 0, stream>>>(
      prefix, n, node_ranges, index_bits, nodes, order, C, Ccols, cb, st, centers, o_mass, o_com,
      o_center, o_packed, o_dipole, o_second, o_quad, o_third, o_oct, o_fourth, o_hexa);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

}  // extern "C"
