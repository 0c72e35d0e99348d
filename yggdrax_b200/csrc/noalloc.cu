// ygx_sort_pairs_noalloc: the stable radix sort of ygx_sort_pairs with its
// scratch memory in a fixed device array instead of a caller workspace.
//
// Who needs it: code that cannot allocate device memory at the point where
// it sorts -- for example a JAX/XLA custom-call handler that was registered
// without a scratch-buffer request (XLA preallocates most of the GPU's memory
// for its own pool, so a cudaMalloc issued from inside the handler can fail
// or fragment that pool), or a host runtime with a fixed, pre-reserved
// memory budget.  Such callers still pass their own input and output
// buffers; only the sort's temporary storage comes from here.
//
// The scratch is one file-scope __device__ array of kNoAllocBytes bytes.
// Every GPU that loads this library holds that much device memory until the
// process exits, so the array is kept small: at most kNoAllocMaxKeys keys
// per call.  All calls on a device share the same array and it keeps the
// previous call's contents; each call clears the parts that must start at
// zero.  Two calls whose work overlaps on the GPU (different streams, or
// different host threads without ordering) race on the array and corrupt
// each other's results -- order such calls on one stream.
#include <mutex>

#include "sort.cuh"

namespace ygx {
namespace {

constexpr int64_t kNoAllocMaxKeys = int64_t(1) << 18;   // 262,144 keys per call
constexpr size_t kNoAllocBytes = size_t(4) << 20;      // 4 MiB per GPU

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device.  The host-side
// name of a __device__ array is only a stand-in, so the address is looked up
// once per device (with that device current) and cached.
int scratch_address(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return YGX_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return YGX_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return YGX_ERR_CUDA;
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return YGX_OK;
}

}  // namespace
}  // namespace ygx

extern "C" {

int ygx_sort_pairs_noalloc(const uint64_t* keys_in, const uint32_t* values_in, int64_t n,
                           int begin_bit, int end_bit, uint64_t* keys_out, uint32_t* values_out,
                           cudaStream_t stream) {
  if (n < 0 || (n > 0 && (!keys_in || !keys_out || !values_out))) return YGX_ERR_ARG;
  if (n > ygx::kNoAllocMaxKeys) return YGX_ERR_TOO_LARGE;
  if (ygx::onesweep_scratch_bytes(ygx::kNoAllocMaxKeys) + 256 > ygx::kNoAllocBytes)
    return YGX_ERR_ARG;  // layout does not fit (build-time sizing error)
  void* base = nullptr;
  int rc = ygx::scratch_address(&base);
  if (rc != YGX_OK) return rc;
  ygx::Arena a{(char*)base, 0, ygx::kNoAllocBytes};
  uint32_t* status = a.take<uint32_t>(64);
  ygx::SortScratch s = ygx::carve_sort_scratch(a, ygx::kNoAllocMaxKeys);
  if (a.used > ygx::kNoAllocBytes) return YGX_ERR_ARG;
  if (cudaMemsetAsync(status, 0, sizeof(uint32_t), stream) != cudaSuccess) return YGX_ERR_CUDA;
  return ygx::onesweep_sort(keys_in, values_in, n, begin_bit, end_bit, keys_out, values_out, s,
                            false, status, stream);
}

}  // extern "C"
