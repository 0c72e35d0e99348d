#include "scan.cuh"

#include <atomic>

namespace ygx {
static std::atomic<unsigned long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
}  // namespace ygx

extern "C" uint64_t ygx_launch_counter(void) { return ygx::g_launches.load(); }

namespace ygx {
namespace {

__device__ __forceinline__ int64_t block_exclusive_sum(int64_t v, int64_t* s_warp, int64_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t incl = v;
  for (int off = 1; off < 32; off <<= 1) {
    int64_t o = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += o;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int64_t w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
    int64_t wi = w;
    for (int off = 1; off < 32; off <<= 1) {
      int64_t o = __shfl_up_sync(0xffffffffu, wi, off);
      if (lane >= off) wi += o;
    }
    if (lane < (int)(blockDim.x >> 5)) s_warp[lane] = wi - w;
    if (lane == 31) *total = wi;
  }
  __syncthreads();
  int64_t r = s_warp[warp] + incl - v;
  __syncthreads();
  return r;
}

template <typename InT>
__global__ void __launch_bounds__(kScanThreads)
    k_tile_sums(const InT* __restrict__ in, int64_t n, int64_t* __restrict__ sums) {
  __shared__ int64_t s_warp[32];
  __shared__ int64_t s_total;
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  int64_t acc = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
    if (i < n) acc += (int64_t)in[i];
  }
  block_exclusive_sum(acc, s_warp, &s_total);
  if (threadIdx.x == 0) sums[blockIdx.x] = s_total;
}

__global__ void __launch_bounds__(1024) k_scan_sums(int64_t* __restrict__ sums, int64_t m) {
  __shared__ int64_t s_warp[32];
  __shared__ int64_t s_total;
  int64_t carry = 0;
  for (int64_t base = 0; base < m; base += blockDim.x) {
    int64_t i = base + threadIdx.x;
    int64_t v = i < m ? sums[i] : 0;
    int64_t e = block_exclusive_sum(v, s_warp, &s_total);
    if (i < m) sums[i] = carry + e;
    carry += s_total;
  }
  if (threadIdx.x == 0) sums[m] = carry;
}

template <typename InT>
__global__ void __launch_bounds__(kScanThreads)
    k_tile_scan(const InT* __restrict__ in, int64_t n, const int64_t* __restrict__ sums,
                int64_t* __restrict__ out) {
  __shared__ int64_t s_warp[32];
  __shared__ int64_t s_total;
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  // Blocked arrangement: thread t owns items [t*K, t*K+K) of the tile.
  int64_t v[kScanItems];
  int64_t acc = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    v[k] = i < n ? (int64_t)in[i] : 0;
    acc += v[k];
  }
  int64_t run = sums[blockIdx.x] + block_exclusive_sum(acc, s_warp, &s_total);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + (int64_t)threadIdx.x * kScanItems + k;
    if (i < n) out[i] = run;
    run += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = sums[gridDim.x];
}

}  // namespace

template <typename InT>
int exclusive_scan(const InT* in, int64_t n, int64_t* out, int64_t* tmp, cudaStream_t st) {
  if (n <= 0) {
    if (cudaMemsetAsync(out, 0, sizeof(int64_t), st) != cudaSuccess) return YGX_ERR_CUDA;
    return YGX_OK;
  }
  const int64_t tiles = scan_tiles(n);
  k_tile_sums<InT><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, tmp);
  YGX_CHECK_LAUNCH();
  k_scan_sums<<<1, 1024, 0, st>>>(tmp, tiles);
  YGX_CHECK_LAUNCH();
  k_tile_scan<InT><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, tmp, out);
  YGX_CHECK_LAUNCH();
  return YGX_OK;
}

template int exclusive_scan<int32_t>(const int32_t*, int64_t, int64_t*, int64_t*, cudaStream_t);
template int exclusive_scan<int64_t>(const int64_t*, int64_t, int64_t*, int64_t*, cudaStream_t);
template int exclusive_scan<uint32_t>(const uint32_t*, int64_t, int64_t*, int64_t*, cudaStream_t);

}  // namespace ygx
