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
//
// The first 4 bytes of the array are the sort's status word (YGX_FLAG_*
// bits: a look-back wait that gave up, an inconsistent histogram).  Each
// call zeroes it before sorting; ygx_sort_pairs_noalloc_status reads it back
// after a call, so a caller can tell a complete sort from one that was cut
// short.
#include <mutex>

#include "sort.cuh"

namespace ygx {
namespace {

constexpr int64_t kNoAllocMaxKeys = int64_t(1) << 18;   // 262,144 keys per call
constexpr size_t kNoAllocBytes = size_t(6) << 20;      // 6 MiB per GPU

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// cuCtxGetCurrent, reached through the runtime's driver entry point so the
// library needs no link against libcuda.
typedef int (*CtxGetCurrentFn)(void** ctx);

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
struct ScratchSlot {
  void* ptr = nullptr;
  void* ctx = nullptr;  // context the address belongs to
};
ScratchSlot g_scratch[kMaxDevices];

CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (CtxGetCurrentFn) nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(p);
  }();
  return fn;
}

// Device address of g_noalloc_scratch on the current device.  In host code
// the array's name is only a stand-in, so the address is looked up with
// cudaGetSymbolAddress, with the device current, and cached per device
// together with the context it was taken in: after cudaDeviceReset the
// module is loaded again into a new context and the array may sit
// elsewhere, so a changed context triggers a fresh look-up.  (Where the
// driver entry point is unavailable the address is looked up on every call.)
// The stream must belong to the current device.
int scratch_address(cudaStream_t stream, void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return YGX_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return YGX_ERR_ARG;
  int sdev = -1;
  if (cudaStreamGetDevice(stream, &sdev) != cudaSuccess) return YGX_ERR_ARG;
  if (sdev != dev) return YGX_ERR_ARG;
  void* ctx = nullptr;
  CtxGetCurrentFn get = ctx_get_current();
  const bool have_ctx = get != nullptr && get(&ctx) == 0 && ctx != nullptr;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  ScratchSlot& s = g_scratch[dev];
  if (s.ptr == nullptr || !have_ctx || s.ctx != ctx) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return YGX_ERR_CUDA;
    s.ptr = p;
    s.ctx = have_ctx ? ctx : nullptr;
  }
  *out = s.ptr;
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
  int rc = ygx::scratch_address(stream, &base);
  if (rc != YGX_OK) return rc;
  ygx::Arena a{(char*)base, 0, ygx::kNoAllocBytes};
  uint32_t* status = a.take<uint32_t>(64);
  ygx::SortScratch s = ygx::carve_sort_scratch(a, ygx::kNoAllocMaxKeys);
  if (a.used > ygx::kNoAllocBytes) return YGX_ERR_ARG;
  if (cudaMemsetAsync(status, 0, sizeof(uint32_t), stream) != cudaSuccess) return YGX_ERR_CUDA;
  return ygx::onesweep_sort(keys_in, values_in, n, begin_bit, end_bit, keys_out, values_out, s,
                            false, status, stream);
}

int ygx_sort_pairs_noalloc_status(uint32_t* host_flags, cudaStream_t stream) {
  if (!host_flags) return YGX_ERR_ARG;
  void* base = nullptr;
  int rc = ygx::scratch_address(stream, &base);
  if (rc != YGX_OK) return rc;
  uint32_t v = 0;
  if (cudaMemcpyAsync(&v, base, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream) !=
      cudaSuccess)
    return YGX_ERR_CUDA;
  if (cudaStreamSynchronize(stream) != cudaSuccess) return YGX_ERR_CUDA;
  *host_flags = v;
  return YGX_OK;
}

}  // extern "C"
