// C-ABI entry points (include/jaccpot_b200.h) and the order-independent kernels.
#include "fmm_kernels.cuh"

#define JB_ORDERS(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)
JB_ORDERS(JB_DECLARE_ORDER)

namespace jb {

static thread_local char g_err[256] = {0};

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return JB_OK;
  snprintf(g_err, sizeof(g_err), "%s", cudaGetErrorString(e));
  return JB_ERR_CUDA;
}

// ---------------------------------------------------------------------------
// Gather into Morton order.
// ---------------------------------------------------------------------------
__global__ void k_gather_sorted(int64_t n, const float* __restrict__ pos, const float* __restrict__ mass,
                                const int64_t* __restrict__ perm, float4* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t o = perm[i];
  out[i] = make_float4(pos[3 * o], pos[3 * o + 1], pos[3 * o + 2], mass[o]);
}

__global__ void k_scatter_unsorted(int64_t n, const float4* __restrict__ acc4, const int64_t* __restrict__ perm,
                                   float* __restrict__ out_acc, float* __restrict__ out_pot) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t o = perm[i];
  const float4 a = acc4[i];
  out_acc[3 * o] = a.x;
  out_acc[3 * o + 1] = a.y;
  out_acc[3 * o + 2] = a.z;
  if (out_pot) out_pot[o] = a.w;
}

// ---------------------------------------------------------------------------
// List validation (prepare time).
// ---------------------------------------------------------------------------
__global__ void k_validate(int num_nodes, int num_internal, const int* left, const int* right, const int64_t* far_off,
                           const int* far_src, int64_t num_far, const int64_t* near_off, const int* near_src,
                           int64_t num_near, int* bad) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int num_leaves = num_nodes - num_internal;
  int b = 0;
  for (int64_t i = tid; i < num_internal; i += stride) {
    if (left[i] <= i || left[i] >= num_nodes) ++b;
    if (right[i] <= i || right[i] >= num_nodes) ++b;
  }
  for (int64_t i = tid; i < num_far; i += stride)
    if (far_src[i] < 0 || far_src[i] >= num_nodes) ++b;
  for (int64_t i = tid; i < num_near; i += stride)
    if (near_src[i] < 0 || near_src[i] >= num_leaves) ++b;
  for (int64_t i = tid; i <= num_nodes; i += stride) {
    if (far_off[i] < 0 || far_off[i] > num_far) ++b;
    if (i > 0 && far_off[i] < far_off[i - 1]) ++b;
  }
  for (int64_t i = tid; i <= num_leaves; i += stride) {
    if (near_off[i] < 0 || near_off[i] > num_near) ++b;
    if (i > 0 && near_off[i] < near_off[i - 1]) ++b;
  }
  if (b) atomicAdd(bad, b);
}

// ---------------------------------------------------------------------------
// Dispatch over the compile-time order.
// ---------------------------------------------------------------------------

template <template <int> class F, typename... A>
static int dispatch(int p, A... args) {
  switch (p) {
#define JB_CASE(PP) \
  case PP:          \
    return F<PP>::run(args...);
    JB_ORDERS(JB_CASE)
#undef JB_CASE
    default:
      return JB_ERR_ORDER;
  }
}

static inline unsigned blocks_1d(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

}  // namespace jb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace jb;

#define ST(s) reinterpret_cast<cudaStream_t>(s)

extern "C" {

JB_API int jb_coeff_stride(int p) { return (p >= 1 && p <= JB_MAX_ORDER) ? cstride(p) : 0; }

JB_API const char* jb_last_cuda_error(void) { return g_err; }

JB_API int jb_gather_sorted(int64_t n, const float* pos, const float* mass, const int64_t* perm, float* out_pos4,
                            void* stream) {
  if (n < 0 || (n > 0 && (!pos || !mass || !perm || !out_pos4))) return JB_ERR_ARG;
  if (n == 0) return JB_OK;
  k_gather_sorted<<<blocks_1d(n, 256), 256, 0, ST(stream)>>>(n, pos, mass, perm, reinterpret_cast<float4*>(out_pos4));
  return launch_status();
}

JB_API int jb_scatter_unsorted(int64_t n, const float* acc4, const int64_t* perm, float* out_acc, float* out_pot,
                               void* stream) {
  if (n < 0 || (n > 0 && (!acc4 || !perm || !out_acc))) return JB_ERR_ARG;
  if (n == 0) return JB_OK;
  k_scatter_unsorted<<<blocks_1d(n, 256), 256, 0, ST(stream)>>>(n, reinterpret_cast<const float4*>(acc4), perm,
                                                                  out_acc, out_pot);
  return launch_status();
}

JB_API int jb_validate_lists(int num_nodes, int num_internal, const int* left, const int* right,
                             const int64_t* far_off, const int* far_src, int64_t num_far, const int64_t* near_off,
                             const int* near_src, int64_t num_near, int* bad_count_dev, void* stream) {
  if (num_nodes < 1 || num_internal < 0 || num_internal >= num_nodes || !far_off || !near_off || !bad_count_dev)
    return JB_ERR_ARG;
  if ((num_internal > 0 && (!left || !right)) || (num_far > 0 && !far_src) || (num_near > 0 && !near_src))
    return JB_ERR_ARG;
  cudaError_t e = cudaMemsetAsync(bad_count_dev, 0, sizeof(int), ST(stream));
  if (e != cudaSuccess) return cuda_status(e);
  k_validate<<<148 * 4, 256, 0, ST(stream)>>>(num_nodes, num_internal, left, right, far_off, far_src, num_far, near_off,
                                              near_src, num_near, bad_count_dev);
  return launch_status();
}

JB_API int jb_p2m(int p, const float* pos4, int num_nodes, int num_internal, const int* node_ranges, float* centers,
                  float* mult, void* stream) {
  if (!pos4 || !node_ranges || !centers || !mult || num_nodes < 1 || num_internal < 0) return JB_ERR_ARG;
  return dispatch<RunP2M>(p, pos4, num_nodes, num_internal, node_ranges, centers, mult, ST(stream));
}

JB_API int jb_m2m_level(int p, int first, int last, const int* left, const int* right, float* centers, float* mult,
                        void* stream) {
  if (first < 0 || last < first || (last > first && (!left || !right || !centers || !mult))) return JB_ERR_ARG;
  return dispatch<RunM2M>(p, first, last, left, right, centers, mult, ST(stream));
}

JB_API int jb_m2l(int p, int mode, int num_targets, const int* targets, const float* mult, const float* centers,
                  const int64_t* far_off, const int* far_src, float* locals, void* stream) {
  if (num_targets < 0 || (num_targets > 0 && (!targets || !mult || !centers || !far_off || !locals))) return JB_ERR_ARG;
  if (mode != JB_M2L_FP32) return JB_ERR_UNSUPPORTED;
  return dispatch<RunM2L>(p, num_targets, targets, mult, centers, far_off, far_src, locals, ST(stream));
}

JB_API int jb_l2l_level(int p, int first, int last, const int* left, const int* right, const float* centers,
                        float* locals, void* stream) {
  if (first < 0 || last < first || (last > first && (!left || !right || !centers || !locals))) return JB_ERR_ARG;
  return dispatch<RunL2L>(p, first, last, left, right, centers, locals, ST(stream));
}

JB_API int jb_leaf_eval(int p, int p2p_mode, const float* pos4, int num_internal, int num_leaves,
                        const int* node_ranges, const float* centers, const float* locals, const int64_t* near_off,
                        const int* near_src, float G, float eps2, float* out_acc4, void* stream) {
  if (!pos4 || !node_ranges || !centers || !locals || !near_off || !out_acc4 || num_leaves < 0 || num_internal < 0)
    return JB_ERR_ARG;
  if (p2p_mode != JB_P2P_FP32 && p2p_mode != JB_P2P_KAHAN) return JB_ERR_ARG;
  return dispatch<RunLeafEval>(p, p2p_mode, pos4, num_internal, num_leaves, node_ranges, centers, locals, near_off,
                               near_src, G, eps2, out_acc4, ST(stream));
}

JB_API int jb_eval_targets(int p, const float* pos4, int num_internal, const int* node_ranges, const float* centers,
                           const float* locals, const int64_t* near_off, const int* near_src, const int* leaf_of,
                           int64_t num_targets, const int* targets_sorted, float G, float eps2, float* out_acc4,
                           void* stream) {
  if (num_targets < 0 || (num_targets > 0 && (!pos4 || !node_ranges || !centers || !locals || !near_off || !leaf_of ||
                                               !targets_sorted || !out_acc4)))
    return JB_ERR_ARG;
  return dispatch<RunTargets>(p, pos4, num_internal, node_ranges, centers, locals, near_off, near_src, leaf_of,
                              num_targets, targets_sorted, G, eps2, out_acc4, ST(stream));
}

}  // extern "C"
