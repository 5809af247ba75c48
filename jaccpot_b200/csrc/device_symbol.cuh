#pragma once
// Device addresses of file-scope __device__ arrays for host code.
//
// In host code the name of a __device__ variable is a host-side stand-in,
// not a device address; cudaGetSymbolAddress gives the address on the
// current device.  It is looked up once per device and cached, keyed by the
// device's current CUDA context: a context that was reset (cudaDeviceReset)
// reloads the module and may place the variable elsewhere, so a new context
// id triggers a new lookup.  The context id comes from the driver's
// cuCtxGetCurrent / cuCtxGetId, fetched through cudaGetDriverEntryPoint (no
// link-time dependency on libcuda); where those are unavailable the address
// is looked up on every call, which is always correct.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

namespace jb {

constexpr int kSymbolCacheDevices = 128;

struct SymbolCache {
  std::mutex mu;
  void* addr[kSymbolCacheDevices] = {};
  unsigned long long ctx[kSymbolCacheDevices] = {};
};

// Id of the calling thread's current context (0 when it cannot be read).
inline unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
    cudaGetLastError();  // a failed query leaves no sticky error behind
  });
  if (!get_current || !get_id) return 0;
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current(&c) != CUDA_SUCCESS || c == nullptr || get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// *out = device address of a __device__ symbol on the current device;
// `lookup(void**)` calls cudaGetSymbolAddress for it.  Returns the CUDA
// error of the lookup (cudaSuccess when found).
template <typename Lookup>
cudaError_t cached_symbol_address(SymbolCache& cache, Lookup&& lookup, void** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long ctx = current_context_id();
  if (dev < 0 || dev >= kSymbolCacheDevices || ctx == 0) return lookup(out);
  std::lock_guard<std::mutex> lock(cache.mu);
  if (cache.addr[dev] == nullptr || cache.ctx[dev] != ctx) {
    void* p = nullptr;
    e = lookup(&p);
    if (e != cudaSuccess) return e;
    cache.addr[dev] = p;
    cache.ctx[dev] = ctx;
  }
  *out = cache.addr[dev];
  return cudaSuccess;
}

// Device address of the leaf error word of the current device (fmm_capi.cu).
int leaf_error_word(int** out);

}  // namespace jb
