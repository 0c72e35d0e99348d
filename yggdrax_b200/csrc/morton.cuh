// Morton encode of one point (shared by the single-set and batched paths).
#pragma once
#include "common.cuh"

namespace ygx {

// morton.py:64-77 in fp32 with IEEE division and round-half-even.
__device__ __forceinline__ uint64_t encode_one(float x, float y, float z, const float* mn,
                                               const float* span) {
  float v[3] = {x, y, z};
  uint64_t q[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float norm = __fdiv_rn(__fsub_rn(v[a], mn[a]), span[a]);
    norm = fminf(fmaxf(norm, 0.0f), 1.0f);  // NaN -> 0 (no integer image)
    q[a] = __float2ull_rn(__fmul_rn(norm, 2097151.0f));
  }
  return spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
}

}  // namespace ygx
