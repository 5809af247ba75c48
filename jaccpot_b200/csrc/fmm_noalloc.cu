// Leaf evaluation for callers that cannot allocate device memory
// (jb_leaf_eval_noalloc in include/jaccpot_b200.h).
//
// jb_leaf_eval needs a caller-provided scratch buffer for the partial results
// of leaves whose near list is split over several work units.  Some callers
// cannot provide one: a jax.ffi / XLA custom-call handler only sees the
// buffers XLA planned for it, and a cudaMalloc from inside it would
// synchronise the device in the middle of XLA's asynchronous schedule; code
// that runs inside a CUDA stream capture may not call cudaMalloc at all.  For
// them this file holds that scratch in a fixed-size device array that every
// GPU loading the library keeps until the process exits.
//
// The kernels are the ones jb_leaf_eval launches (the same near-field form,
// so the results are equal bit for bit); only the scratch pointer differs.
#include "device_symbol.cuh"
#include "fmm_adjoint.cuh"

#define JB_ORDERS_NA(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)
JB_ORDERS_NA(JB_DECLARE_ORDER)

namespace {

// 16384 slots x 64 particles x float4 = 16 MiB per device.
static __device__ __align__(256) float4 g_leaf_scratch[(int64_t)JB_LEAF_EVAL_NOALLOC_MAX_SLOTS * jb::kMaxLeaf];

jb::SymbolCache g_scratch_cache;

// Device address of g_leaf_scratch on the current device: in host code the
// array's name is only a host-side handle, so the address is looked up with
// that device current, once per device and context, and cached.
int scratch_address(void** out) {
  const cudaError_t e = jb::cached_symbol_address(
      g_scratch_cache, [](void** p) { return cudaGetSymbolAddress(p, g_leaf_scratch); }, out);
  return e == cudaSuccess ? JB_OK : jb::cuda_status(e);
}

template <template <int> class F, typename... A>
int dispatch_order(int p, A... args) {
  switch (p) {
#define JB_CASE_NA(PP) \
  case PP:             \
    return F<PP>::run(args...);
    JB_ORDERS_NA(JB_CASE_NA)
#undef JB_CASE_NA
    default:
      return JB_ERR_ORDER;
  }
}

}  // namespace

extern "C" JB_API int jb_leaf_eval_noalloc(int p, int p2p_mode, const float* pos4, int num_internal, int num_units,
                                           const int* units, const int* aux, const int* runs, const int* node_ranges,
                                           const float* centers, const float* locals, float G, float eps2,
                                           float* out_acc4, int num_slots, int num_split, const int* split,
                                           void* stream) {
  if (num_units < 0 || num_split < 0 || num_internal < 0 || num_slots < 0 ||
      (num_units > 0 && (!pos4 || !units || !aux || !runs || !node_ranges || !centers || !locals || !out_acc4)) ||
      (num_split > 0 && (!split || !out_acc4 || !node_ranges || num_slots == 0)))
    return JB_ERR_ARG;
  if (p2p_mode & ~(JB_P2P_KAHAN | JB_P2P_POTENTIAL)) return JB_ERR_ARG;
  if (p < 1 || p > JB_MAX_ORDER) return JB_ERR_ORDER;
  if (num_slots > JB_LEAF_EVAL_NOALLOC_MAX_SLOTS) return JB_ERR_WORKSPACE;
  // Every scratch row that the reduce reads is written earlier in the same
  // call, so nothing needs clearing between calls; slots at or beyond
  // num_slots are neither written nor read (JB_LEAF_ERR_SLOT).
  void* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != JB_OK) return rc;
  int* err = nullptr;
  rc = jb::leaf_error_word(&err);
  if (rc != JB_OK) return rc;
  return dispatch_order<jb::RunLeafEval>(p, p2p_mode, pos4, num_internal, num_units, units, aux, runs, node_ranges,
                                         centers, locals, G, eps2, out_acc4, static_cast<float*>(scratch),
                                         num_split, split, reinterpret_cast<cudaStream_t>(stream),
                                         (const int*)nullptr, (const float*)nullptr, 1, jb::g_leaf_flat != 0,
                                         num_slots, err);
}
