// Allocation-free variant of the fused, broadcast-reducing backward of
// regularized_gamma_p.
//
// The regular entry point (tsb_regularized_gamma_p_backward) needs a device
// workspace for the per-tile partial sums of gradients that it reduces to a
// broadcast input's shape, and expects the caller to allocate it.  Some
// callers cannot: a host that reaches this library only through a plain C
// FFI (cgo, JNI, ctypes) may own no device allocator at all, and a
// latency-critical loop may not call cudaMalloc, which can synchronize the
// whole device.  This entry point serves them.  It allocates nothing: the
// partial sums live in a file-scope device array of fixed size
// (TSB_NOALLOC_SCRATCH_BYTES), which every GPU that loads the library holds
// until the process exits.
//
// Rules that follow from the shared array:
//   - the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current) and caches it; make
//     that first call before any stream capture.  The cache lives as long as
//     the process: cudaDeviceReset destroys the context that holds the array,
//     so after a reset this entry point must not be called again;
//   - every call uses the same array, so calls that overlap on the GPU (on
//     different streams, or from different host threads) race and must be
//     serialized by the caller;
//   - the array keeps the last call's partial sums; nothing needs clearing,
//     because a call writes every partial it later reads;
//   - a request whose partial sums do not fit is rejected with
//     TSB_ERR_WORKSPACE and nothing is launched.
#include <mutex>

#include "igamma_ops.cuh"

namespace tsb {
namespace {

__device__ __align__(256) unsigned char g_noalloc_scratch[TSB_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mutex;
void* g_noalloc_addr[64];  // device address of g_noalloc_scratch, per device ordinal

// Device address of the scratch array on the current device (looked up once
// per device; host code cannot use the symbol itself as a device pointer).
int32_t noalloc_scratch(void** addr) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(TSB_ERR_DEVICE, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  }
  if (dev < 0 || dev >= 64) return set_error(TSB_ERR_DEVICE, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      return set_error(TSB_ERR_DEVICE, "cudaGetSymbolAddress of the scratch array failed on device %d: %s", dev,
                       cudaGetErrorString(e));
    }
    g_noalloc_addr[dev] = p;
  }
  *addr = g_noalloc_addr[dev];
  return TSB_OK;
}

}  // namespace
}  // namespace tsb

extern "C" int32_t tsb_regularized_gamma_p_backward_noalloc(const tsb_tensor* in, int32_t n_in, const tsb_tensor* out,
                                                            int32_t n_out, int32_t precision, void* stream) {
  const int64_t need = tsb_workspace_bytes(in, n_in, out, n_out);
  if (need < 0) return static_cast<int32_t>(need);
  if (need > TSB_NOALLOC_SCRATCH_BYTES)
    return tsb::set_error(TSB_ERR_WORKSPACE,
                          "reducing these gradients needs %lld bytes of scratch; the allocation-free entry point has "
                          "%lld (use tsb_regularized_gamma_p_backward with a caller-provided workspace)",
                          (long long)need, (long long)TSB_NOALLOC_SCRATCH_BYTES);
  void* ws = nullptr;
  if (need > 0) {
    const int32_t st = tsb::noalloc_scratch(&ws);
    if (st) return st;
  }
  return tsb::run_op<tsb::GammaPBwd>(in, n_in, out, n_out, precision, ws, need, stream);
}
