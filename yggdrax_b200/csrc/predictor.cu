// Learned row-capacity predictor for the traversal: per-node features from
// the geometry and topology, a small fp32 MLP (kIn -> 64 -> 64 -> 2,
// ReLU) that predicts log2(1 + far row length) and log2(1 + near row
// length), its training (tiled SGEMM forward / backward, masked MSE, Adam)
// and its inference fused with the capacity and padded-offset computation
// used by the one-pass predicted walk.  There is no counterpart in the
// reference: it replaces the count walk of count-then-fill
// (_interactions_impl.py:2600-2939) by a prediction; the lists stay exact
// because rows that outgrow their prediction are detected and completed.
#include "scan.cuh"

namespace ygx {
namespace {

constexpr int kIn = YGX_MLP_INPUTS;
constexpr int kHid = 64;
constexpr int kOut = 2;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kIn * kHid;
constexpr int kOffW2 = kOffB1 + kHid;
constexpr int kOffB2 = kOffW2 + kHid * kHid;
constexpr int kOffW3 = kOffB2 + kHid;
constexpr int kOffB3 = kOffW3 + kHid * kOut;
constexpr int kParams = kOffB3 + kOut;
static_assert(kParams == YGX_MLP_PARAMS, "parameter layout");

enum { kMacBH = 0, kMacDehnen = 1, kMacEngblom = 2 };

// Features of node k (all O(1) in magnitude):
//  0 log2(radius / root radius)        1 log2(max_extent / root max_extent)
//  2 level / 16                         3 leaf (0/1)
//  4 log2(particles) / 8                5 log2(parent radius / root radius)
//  6 log2(distance to root centre / root radius + 1e-3)
//  7 log2(MAC extent / (distance + 1e-3 root radius))
//  8 theta                              9 1 for the "bh" MAC, else 0
// 10 log2(leaves) / 20                  11 log2(particles / parent's particles)
__device__ __forceinline__ void node_features(
    int64_t k, const float* __restrict__ center, const float* __restrict__ radius,
    const float* __restrict__ max_extent, const int32_t* __restrict__ level32,
    const int32_t* __restrict__ parent32, int64_t total, int64_t ni, const void* ranges,
    int index_bits, int root, float theta, int mac, float* f) {
  const float rr = radius[root], er = max_extent[root];
  const float r = radius[k], e = max_extent[k];
  const float dx = center[3 * k] - center[3 * root];
  const float dy = center[3 * k + 1] - center[3 * root + 1];
  const float dz = center[3 * k + 2] - center[3 * root + 2];
  const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
  const int64_t s = load_idx(ranges, index_bits, 2 * k);
  const int64_t c = load_idx(ranges, index_bits, 2 * k + 1) - s + 1;
  const int32_t par = parent32[k] >= 0 ? parent32[k] : (int32_t)k;
  const int64_t ps = load_idx(ranges, index_bits, 2 * (int64_t)par);
  const int64_t pc = load_idx(ranges, index_bits, 2 * (int64_t)par + 1) - ps + 1;
  const float emac = mac == kMacBH ? e : r;
  f[0] = log2f(r / rr);
  f[1] = log2f(e / er);
  f[2] = (float)level32[k] * (1.0f / 16.0f);
  f[3] = k >= ni ? 1.0f : 0.0f;
  f[4] = log2f((float)(c > 1 ? c : 1)) * 0.125f;
  f[5] = log2f(radius[par] / rr);
  f[6] = log2f(dist / rr + 1e-3f);
  f[7] = log2f(emac / (dist + 1e-3f * rr));
  f[8] = theta;
  f[9] = mac == kMacBH ? 1.0f : 0.0f;
  f[10] = log2f((float)(total - ni)) * 0.05f;
  f[11] = log2f((float)(c > 1 ? c : 1) / (float)(pc > 1 ? pc : 1));
}

__global__ void k_node_features(const float* __restrict__ center, const float* __restrict__ radius,
                                const float* __restrict__ max_extent,
                                const int32_t* __restrict__ level32,
                                const int32_t* __restrict__ parent32, int64_t total, int64_t ni,
                                const void* ranges, int index_bits, int root, float theta,
                                int mac, float* __restrict__ X) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    float f[kIn];
    node_features(k, center, radius, max_extent, level32, parent32, total, ni, ranges, index_bits,
                  root, theta, mac, f);
#pragma unroll
    for (int i = 0; i < kIn; ++i) X[k * kIn + i] = f[i];
  }
}

// One sample through the MLP with the parameters in shared memory; h1 stays
// in registers, the second layer is folded straight into the output.
// The parameters in shared memory with W1 and W2 transposed (row j holds
// the weights into hidden unit j), so each unit's dot product reads 16-byte
// words -- a quarter of the shared-memory loads of the row-major layout.
// Inference uses fused multiply-adds (one instruction instead of two; the
// library otherwise builds without contraction): a capacity only sizes the
// padding of a row, the lists stay exact whatever it is.
static_assert(kIn % 4 == 0, "W1 rows are read as float4");
struct __align__(16) MlpSmem {
  float w1t[kHid][kIn];
  float w2t[kHid][kHid];
  float b1[kHid];
  float b2[kHid];
  float w3[kHid * kOut];
  float b3[kOut];
};

__device__ __forceinline__ void mlp_load(MlpSmem& s, const float* __restrict__ params) {
  for (int e = threadIdx.x; e < kIn * kHid; e += blockDim.x) {
    const int i = e / kHid, j = e % kHid;
    s.w1t[j][i] = params[kOffW1 + e];
  }
  for (int e = threadIdx.x; e < kHid * kHid; e += blockDim.x) {
    const int i = e / kHid, j = e % kHid;
    s.w2t[j][i] = params[kOffW2 + e];
  }
  for (int e = threadIdx.x; e < kHid; e += blockDim.x) {
    s.b1[e] = params[kOffB1 + e];
    s.b2[e] = params[kOffB2 + e];
  }
  for (int e = threadIdx.x; e < kHid * kOut; e += blockDim.x) s.w3[e] = params[kOffW3 + e];
  if (threadIdx.x < kOut) s.b3[threadIdx.x] = params[kOffB3 + threadIdx.x];
}

__device__ __forceinline__ void mlp_eval(const MlpSmem& s, const float* x, float* out) {
  float h1[kHid];
#pragma unroll
  for (int j = 0; j < kHid; ++j) {
    float a = s.b1[j];
#pragma unroll
    for (int i = 0; i < kIn; i += 4) {
      const float4 w = *reinterpret_cast<const float4*>(&s.w1t[j][i]);
      a = __fmaf_rn(x[i], w.x, a);
      a = __fmaf_rn(x[i + 1], w.y, a);
      a = __fmaf_rn(x[i + 2], w.z, a);
      a = __fmaf_rn(x[i + 3], w.w, a);
    }
    h1[j] = a > 0.0f ? a : 0.0f;
  }
  // four hidden units at a time: four independent summation chains, each in
  // the order of the row-major loop
  static_assert(kHid % 4 == 0, "units are taken four at a time");
  float o0 = s.b3[0], o1 = s.b3[1];
#pragma unroll 1
  for (int j = 0; j < kHid; j += 4) {
    float a[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) a[u] = s.b2[j + u];
#pragma unroll
    for (int i = 0; i < kHid; i += 4) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float4 w = *reinterpret_cast<const float4*>(&s.w2t[j + u][i]);
        a[u] = __fmaf_rn(h1[i], w.x, a[u]);
        a[u] = __fmaf_rn(h1[i + 1], w.y, a[u]);
        a[u] = __fmaf_rn(h1[i + 2], w.z, a[u]);
        a[u] = __fmaf_rn(h1[i + 3], w.w, a[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const float r = a[u] > 0.0f ? a[u] : 0.0f;
      o0 = __fmaf_rn(r, s.w3[(j + u) * kOut], o0);
      o1 = __fmaf_rn(r, s.w3[(j + u) * kOut + 1], o1);
    }
  }
  out[0] = o0;
  out[1] = o1;
}

__global__ void __launch_bounds__(128) k_mlp_infer(const float* __restrict__ X, int64_t n,
                                                   const float* __restrict__ params,
                                                   float* __restrict__ out) {
  __shared__ MlpSmem s_p;
  mlp_load(s_p, params);
  __syncthreads();
#pragma unroll 1
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    float x[kIn], o[kOut];
#pragma unroll
    for (int i = 0; i < kIn; ++i) x[i] = __ldg(X + k * kIn + i);
    mlp_eval(s_p, x, o);
    out[k * kOut] = o[0];
    out[k * kOut + 1] = o[1];
  }
}

// Capacity from a predicted log2(1 + length): 2^(pred + slack) - 1 rounded
// up, plus `add`, clamped to [add, 2^30].
__device__ __forceinline__ int32_t cap_of(float pred, float slack, int32_t add) {
  const float v = exp2f(fminf(pred + slack, 30.0f)) - 1.0f;
  const int32_t c = (int32_t)ceilf(fmaxf(v, 0.0f)) + add;
  return c < add ? add : c;
}

__global__ void __launch_bounds__(128)
    k_predict_caps(const float* __restrict__ center, const float* __restrict__ radius,
                   const float* __restrict__ max_extent, const int32_t* __restrict__ level32,
                   const int32_t* __restrict__ parent32, const int32_t* __restrict__ leafpos32,
                   int64_t total, int64_t ni, const void* ranges, int index_bits, int root,
                   float theta, int mac, const float* __restrict__ params, float slack_far,
                   float slack_near, int32_t add, int32_t* __restrict__ far_cap,
                   int32_t* __restrict__ near_cap) {
  __shared__ MlpSmem s_p;
  mlp_load(s_p, params);
  __syncthreads();
#pragma unroll 1
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += (int64_t)gridDim.x * blockDim.x) {
    float f[kIn], o[kOut];
    node_features(k, center, radius, max_extent, level32, parent32, total, ni, ranges, index_bits,
                  root, theta, mac, f);
    mlp_eval(s_p, f, o);
    far_cap[k] = cap_of(o[0], slack_far, add);
    if (k >= ni) near_cap[leafpos32[k]] = cap_of(o[1], slack_near, add);
  }
}

// ---- training ---------------------------------------------------------------

// C[M x N] (+)= op(A)[M x K] . op(B)[K x N], row-major, 64 x 64 tiles, 4 x 4
// outputs per thread.  op(A)[m][k] = TA ? A[k*lda+m] : A[m*lda+k], likewise
// B.  With split-K (gridDim.z > 1) every z-slice adds its partial product
// atomically into C, which must then start at zero.
template <bool TA, bool TB>
__global__ void __launch_bounds__(256)
    k_gemm(int M, int N, int K, const float* __restrict__ A, int lda, const float* __restrict__ B,
           int ldb, float* __restrict__ C, int ldc) {
  constexpr int T = 64, KT = 16;
  __shared__ float As[KT][T + 1], Bs[KT][T + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.y * T, n0 = blockIdx.x * T;
  const int kchunk = (K + gridDim.z - 1) / gridDim.z;
  const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
  float acc[4][4] = {};
  for (int k0 = kb; k0 < ke; k0 += KT) {
    for (int e = threadIdx.x; e < KT * T; e += 256) {
      const int kk = e / T, mm = e % T;
      const int gk = k0 + kk, gm = m0 + mm, gn = n0 + mm;
      As[kk][mm] = (gk < ke && gm < M) ? (TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk])
                                       : 0.0f;
      Bs[kk][mm] = (gk < ke && gn < N) ? (TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn])
                                       : 0.0f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < KT; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += a[i] * b[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + ty * 4 + i;
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + tx * 4 + j;
      if (n >= N) continue;
      if (gridDim.z > 1) atomicAdd(&C[(size_t)m * ldc + n], acc[i][j]);
      else C[(size_t)m * ldc + n] = acc[i][j];
    }
  }
}

__global__ void k_bias_act(float* __restrict__ Z, const float* __restrict__ b, int64_t M, int N,
                           bool relu) {
  const int64_t total = M * N;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    float v = Z[e] + b[e % N];
    Z[e] = relu && v < 0.0f ? 0.0f : v;
  }
}

// Masked mean-squared error: loss = sum(mask * (out - y)^2) / M, dOut = its
// gradient.
__global__ void k_loss_grad(const float* __restrict__ O, const float* __restrict__ Y,
                            const float* __restrict__ mask, int64_t M, float* __restrict__ dO,
                            float* __restrict__ loss) {
  float part = 0.0f;
  const float inv = 1.0f / (float)M;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < M * kOut;
       e += (int64_t)gridDim.x * blockDim.x) {
    const float d = (O[e] - Y[e]) * mask[e];
    dO[e] = 2.0f * d * inv;
    part += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, part * inv);
}

__global__ void k_relu_bwd(float* __restrict__ dH, const float* __restrict__ H, int64_t n) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    if (!(H[e] > 0.0f)) dH[e] = 0.0f;
}

// db[n] += sum over rows of dZ[:, n] (db must start at zero).
__global__ void k_colsum(const float* __restrict__ dZ, int64_t M, int N, float* __restrict__ db) {
  const int n = blockIdx.y;
  float part = 0.0f;
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < M;
       m += (int64_t)gridDim.x * blockDim.x)
    part += dZ[m * N + n];
  for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&db[n], part);
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

struct MlpScratch {
  float* H1;    // [B x 64] post-activation
  float* H2;    // [B x 64]
  float* O;     // [B x 2]
  float* dO;    // [B x 2]
  float* dH2;   // [B x 64]
  float* dH1;   // [B x 64]
  float* grads; // [kParams]
  float* loss;  // [1]
};

MlpScratch carve_mlp(Arena& a, int64_t B) {
  MlpScratch s;
  s.H1 = a.take<float>((size_t)B * kHid);
  s.H2 = a.take<float>((size_t)B * kHid);
  s.O = a.take<float>((size_t)B * kOut);
  s.dO = a.take<float>((size_t)B * kOut);
  s.dH2 = a.take<float>((size_t)B * kHid);
  s.dH1 = a.take<float>((size_t)B * kHid);
  s.grads = a.take<float>(kParams);
  s.loss = a.take<float>(1);
  return s;
}

template <bool TA, bool TB>
int gemm(int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc,
         int splits, cudaStream_t st) {
  if (splits > 1 &&
      cudaMemsetAsync(C, 0, sizeof(float) * (size_t)M * ldc, st) != cudaSuccess)
    return YGX_ERR_CUDA;
  dim3 grid((N + 63) / 64, (M + 63) / 64, splits);
  k_gemm<TA, TB><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

// Forward + backward over a batch: gradients into s.grads, loss into s.loss.
int mlp_grads(const float* params, const float* X, const float* Y, const float* mask, int64_t B,
              const MlpScratch& s, cudaStream_t st) {
  const int b = (int)B;
  const int splits = (int)((B + 8191) / 8192) < 64 ? (int)((B + 8191) / 8192) : 64;
  if (cudaMemsetAsync(s.grads, 0, sizeof(float) * kParams, st) != cudaSuccess ||
      cudaMemsetAsync(s.loss, 0, sizeof(float), st) != cudaSuccess)
    return YGX_ERR_CUDA;
  int rc;
  const int eg = grid_for((int64_t)B * kHid, 256);
  // forward
  if ((rc = gemm<false, false>(b, kHid, kIn, X, kIn, params + kOffW1, kHid, s.H1, kHid, 1, st)))
    return rc;
  k_bias_act<<<eg, 256, 0, st>>>(s.H1, params + kOffB1, B, kHid, true);
  YGX_CHECK_LAUNCH();
  if ((rc = gemm<false, false>(b, kHid, kHid, s.H1, kHid, params + kOffW2, kHid, s.H2, kHid, 1,
                               st)))
    return rc;
  k_bias_act<<<eg, 256, 0, st>>>(s.H2, params + kOffB2, B, kHid, true);
  YGX_CHECK_LAUNCH();
  if ((rc = gemm<false, false>(b, kOut, kHid, s.H2, kHid, params + kOffW3, kOut, s.O, kOut, 1,
                               st)))
    return rc;
  k_bias_act<<<grid_for(B * kOut, 256), 256, 0, st>>>(s.O, params + kOffB3, B, kOut, false);
  YGX_CHECK_LAUNCH();
  k_loss_grad<<<grid_for(B * kOut, 256), 256, 0, st>>>(s.O, Y, mask, B, s.dO, s.loss);
  YGX_CHECK_LAUNCH();
  // backward
  if ((rc = gemm<true, false>(kHid, kOut, b, s.H2, kHid, s.dO, kOut, s.grads + kOffW3, kOut,
                              splits, st)))
    return rc;
  k_colsum<<<dim3(grid_for(B, 256, 64), kOut), 256, 0, st>>>(s.dO, B, kOut, s.grads + kOffB3);
  YGX_CHECK_LAUNCH();
  if ((rc = gemm<false, true>(b, kHid, kOut, s.dO, kOut, params + kOffW3, kOut, s.dH2, kHid, 1,
                              st)))
    return rc;
  k_relu_bwd<<<eg, 256, 0, st>>>(s.dH2, s.H2, B * kHid);
  YGX_CHECK_LAUNCH();
  if ((rc = gemm<true, false>(kHid, kHid, b, s.H1, kHid, s.dH2, kHid, s.grads + kOffW2, kHid,
                              splits, st)))
    return rc;
  k_colsum<<<dim3(grid_for(B, 256, 64), kHid), 256, 0, st>>>(s.dH2, B, kHid, s.grads + kOffB2);
  YGX_CHECK_LAUNCH();
  if ((rc = gemm<false, true>(b, kHid, kHid, s.dH2, kHid, params + kOffW2, kHid, s.dH1, kHid, 1,
                              st)))
    return rc;
  k_relu_bwd<<<eg, 256, 0, st>>>(s.dH1, s.H1, B * kHid);
  YGX_CHECK_LAUNCH();
  if ((rc = gemm<true, false>(kIn, kHid, b, X, kIn, s.dH1, kHid, s.grads + kOffW1, kHid, splits,
                              st)))
    return rc;
  k_colsum<<<dim3(grid_for(B, 256, 64), kHid), 256, 0, st>>>(s.dH1, B, kHid, s.grads + kOffB1);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

}  // namespace
}  // namespace ygx

extern "C" {

int ygx_mlp_param_count(void) { return ygx::kParams; }

size_t ygx_mlp_workspace_size(int64_t batch) {
  ygx::Arena a{nullptr, 0, 0};
  ygx::carve_mlp(a, batch > 0 ? batch : 1);
  return a.used + 256;
}

int ygx_node_features(const float* center, const float* radius, const float* max_extent,
                      const int32_t* level32, const int32_t* parent32, int64_t total,
                      int64_t num_internal, const void* node_ranges, int index_bits, int root,
                      float theta, int mac, float* features, cudaStream_t stream) {
  if (total < 1 || num_internal < 0 || root < 0 || root >= total || mac < 0 || mac > 2 ||
      (index_bits != 32 && index_bits != 64) || !features)
    return YGX_ERR_ARG;
  ygx::k_node_features<<<ygx::grid_for(total, 256), 256, 0, stream>>>(
      center, radius, max_extent, level32, parent32, total, num_internal, node_ranges, index_bits,
      root, theta, mac, features);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

int ygx_mlp_forward(const float* params, const float* features, int64_t n, float* out,
                    cudaStream_t stream) {
  if (n < 0 || !params || (n > 0 && (!features || !out))) return YGX_ERR_ARG;
  if (n == 0) return YGX_OK;
  ygx::k_mlp_infer<<<ygx::grid_for(n, 128), 128, 0, stream>>>(features, n, params, out);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

int ygx_mlp_gradients(const float* params, const float* features, const float* targets,
                      const float* mask, int64_t batch, float* grads_out, float* loss_out,
                      void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (batch < 1 || batch > INT32_MAX || !params || !features || !targets || !mask)
    return YGX_ERR_ARG;
  if (ws_bytes < ygx_mlp_workspace_size(batch)) return YGX_ERR_ARG;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::MlpScratch s = ygx::carve_mlp(a, batch);
  int rc = ygx::mlp_grads(params, features, targets, mask, batch, s, stream);
  if (rc) return rc;
  if (grads_out && cudaMemcpyAsync(grads_out, s.grads, sizeof(float) * ygx::kParams,
                                   cudaMemcpyDeviceToDevice, stream) != cudaSuccess)
    return YGX_ERR_CUDA;
  if (loss_out &&
      cudaMemcpyAsync(loss_out, s.loss, sizeof(float), cudaMemcpyDeviceToDevice, stream) !=
          cudaSuccess)
    return YGX_ERR_CUDA;
  return YGX_OK;
}

int ygx_mlp_train_step(float* params, float* adam_m, float* adam_v, int step, float lr,
                       const float* features, const float* targets, const float* mask,
                       int64_t batch, float* loss_out, void* ws, size_t ws_bytes,
                       cudaStream_t stream) {
  if (step < 1 || !adam_m || !adam_v) return YGX_ERR_ARG;
  int rc = ygx_mlp_gradients(params, features, targets, mask, batch, nullptr, loss_out, ws,
                             ws_bytes, stream);
  if (rc) return rc;
  ygx::Arena a{(char*)ws, 0, ws_bytes};
  ygx::MlpScratch s = ygx::carve_mlp(a, batch);
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
  ygx::k_adam<<<ygx::grid_for(ygx::kParams, 256), 256, 0, stream>>>(
      params, s.grads, adam_m, adam_v, ygx::kParams, lr, b1, b2, 1e-8f, c1, c2);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

int ygx_predict_caps(const float* center, const float* radius, const float* max_extent,
                     const int32_t* level32, const int32_t* parent32, const int32_t* leafpos32,
                     int64_t total, int64_t num_internal, const void* node_ranges, int index_bits,
                     int root, float theta, int mac, const float* params, float slack_far,
                     float slack_near, int32_t add, int32_t* far_cap32, int32_t* near_cap32,
                     cudaStream_t stream) {
  if (total < 3 || num_internal < 1 || root < 0 || root >= total || mac < 0 || mac > 2 ||
      (index_bits != 32 && index_bits != 64) || add < 1 || !params || !far_cap32 || !near_cap32)
    return YGX_ERR_ARG;
  ygx::k_predict_caps<<<ygx::grid_for(total, 128), 128, 0, stream>>>(
      center, radius, max_extent, level32, parent32, leafpos32, total, num_internal, node_ranges,
      index_bits, root, theta, mac, params, slack_far, slack_near, add, far_cap32, near_cap32);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

}  // extern "C"
