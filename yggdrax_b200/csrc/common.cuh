// Shared helpers for the yggdrax_b200 CUDA kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <atomic>

#include "../../include/ygx.h"

namespace ygx {

constexpr int kNumSMs = 148;

// Launch-shape knobs (set through ygx_tune_set; defaults are the measured
// best on B200 for the 16M-particle Plummer pipeline).
struct Tune {
  int sort_rank_policy = 2;    // onesweep ranking: 0 ballots, 1 peer tables, 2 by digit skew
  int sort_skew_q8 = 32;       // policy 2: peer tables while max digit share <= q8 / 256
  int walk_blocks_per_sm = 6;  // walk CTAs per SM (<= kWalkBlocksPerSM)
  int refit_warps = 8;         // warps per CTA of the leaf refit
  int row_grid_per_sm = 16;    // CTAs per SM of the short-row finalize kernels
  int sort_tile = 0;           // onesweep tile shape (index into kSortShape, sort.cuh)
  int spin_limit = 1 << 22;    // iterations of a device-side wait before it gives up
  int target_budget = 128;     // per-target walk: warp steps per piece before a hand-off
  int sort_bits = 8;           // onesweep digit width: 8, or 11 where it cuts passes
};
extern Tune g_tune;

// Device-side status word.  Kernels never trap: a bounded spin that gives up,
// or a capacity that is exceeded, ORs a flag in here and the kernel returns.
// Flags map one-to-one onto the YGX_ERR_* return codes.
enum StatusFlag : uint32_t {
  kFlagTimeout = 1u << 0,
  kFlagQueueOverflow = 1u << 1,
  kFlagFarOverflow = 1u << 2,
  kFlagNearOverflow = 1u << 3,
  kFlagMalformed = 1u << 4,
  kFlagBadInput = 1u << 5,
  kFlagLogOverflow = 1u << 6,
};

// Iteration limit of every device-side spin (decoupled look-back), passed to
// the kernels from g_tune.spin_limit (knob YGX_TUNE_SPIN_LIMIT).  A wait this
// long means a producer did not make progress; the waiter records
// kFlagTimeout and continues with what it has, so the launch always ends.
constexpr int kSpinLimitMax = 1 << 24;

__device__ __forceinline__ void raise_flag(uint32_t* status, uint32_t f) {
  if (status) atomicOr(status, f);
}

__device__ __forceinline__ int clz64(uint64_t x) { return x ? __clzll((long long)x) : 64; }

// 21-bit spread / compact with the interleave masks of a 63-bit Morton code.
__host__ __device__ __forceinline__ uint64_t spread3(uint64_t x) {
  x &= 0x1FFFFFull;
  x = (x | (x << 32)) & 0x1F00000000FFFFull;
  x = (x | (x << 16)) & 0x1F0000FF0000FFull;
  x = (x | (x << 8)) & 0x100F00F00F00F00Full;
  x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}
__host__ __device__ __forceinline__ uint64_t compact3(uint64_t x) {
  x &= 0x1249249249249249ull;
  x = (x | (x >> 2)) & 0x10C30C30C30C30C3ull;
  x = (x | (x >> 4)) & 0x100F00F00F00F00Full;
  x = (x | (x >> 8)) & 0x1F0000FF0000FFull;
  x = (x | (x >> 16)) & 0x1F00000000FFFFull;
  x = (x | (x >> 32)) & 0x1FFFFFull;
  return x;
}

// uint64 shifts with the "shift >= 64 gives 0" rule of the reference's
// uint64 arithmetic.
__host__ __device__ __forceinline__ uint64_t shr64(uint64_t x, uint64_t s) { return s >= 64 ? 0 : (x >> s); }
__host__ __device__ __forceinline__ uint64_t shl64(uint64_t x, uint64_t s) { return s >= 64 ? 0 : (x << s); }

// NaN-propagating min / max (the reference's minimum / maximum).
__device__ __forceinline__ float fmin_nan(float a, float b) {
  return (a != a || b != b) ? __int_as_float(0x7fc00000) : fminf(a, b);
}
__device__ __forceinline__ float fmax_nan(float a, float b) {
  return (a != a || b != b) ? __int_as_float(0x7fc00000) : fmaxf(a, b);
}

// Index outputs are INDEX_DTYPE: int64 by default, int32 on request.
template <typename T>
__device__ __forceinline__ void store_index(void* base, int64_t i, int64_t v) {
  reinterpret_cast<T*>(base)[i] = static_cast<T>(v);
}
__device__ __forceinline__ void store_idx(void* base, int index_bits, int64_t i, int64_t v) {
  if (index_bits == 32) reinterpret_cast<int32_t*>(base)[i] = (int32_t)v;
  else reinterpret_cast<int64_t*>(base)[i] = v;
}
__device__ __forceinline__ int64_t load_idx(const void* base, int index_bits, int64_t i) {
  if (index_bits == 32) return reinterpret_cast<const int32_t*>(base)[i];
  return reinterpret_cast<const int64_t*>(base)[i];
}

inline int grid_for(int64_t n, int block, int max_blocks = kNumSMs * 16) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > max_blocks) g = max_blocks;
  return (int)g;
}

inline size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

// Raises a kernel's dynamic shared-memory limit on the current device.  The
// attribute is per device, so `done` keeps one bit per device that has it
// (set from any host thread).
template <typename Kernel>
inline cudaError_t ensure_smem_limit(Kernel kernel, int bytes, std::atomic<uint64_t>& done) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return cudaErrorInvalidDevice;
  const uint64_t bit = 1ull << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
  const cudaError_t e =
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
  return e;
}

// Bump allocator over a caller-provided workspace.
struct Arena {
  char* base;
  size_t used;
  size_t cap;
  template <typename T>
  T* take(size_t count) {
    size_t off = align_up(used);
    used = off + count * sizeof(T);
    return base ? reinterpret_cast<T*>(base + off) : nullptr;
  }
};

}  // namespace ygx

namespace ygx {
// Host-side count of kernel launches issued by this library (all threads).
void note_launch();
}  // namespace ygx

// Called right after every kernel launch: counts it and reports launch errors.
#define YGX_CHECK_LAUNCH()                           \
  do {                                               \
    ygx::note_launch();                              \
    cudaError_t _e = cudaGetLastError();             \
    if (_e != cudaSuccess) return YGX_ERR_CUDA;      \
  } while (0)
