// C-ABI entry points (include/jaccpot_b200.h) and the order-independent kernels.
#include "device_symbol.cuh"
#include "fmm_adjoint.cuh"

#include <cooperative_groups.h>
#include <mutex>

namespace cg = cooperative_groups;

#define JB_ORDERS(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10)
JB_ORDERS(JB_DECLARE_ORDER)

namespace jb {

static thread_local char g_err[256] = {0};
int g_split_max_parents[2] = {1 << 30, 2048};  // measured at clustered N=4M, p=8
int g_leaf_flat = 1;
int g_m2l_coop = 1;

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return JB_OK;
  snprintf(g_err, sizeof(g_err), "%s", cudaGetErrorString(e));
  return JB_ERR_CUDA;
}

// Leaf error word (JB_LEAF_ERR_* bits) of each device, set by the leaf
// kernels when a precondition is broken, read by jb_leaf_eval_errors.
static __device__ int g_leaf_err;
static SymbolCache g_leaf_err_cache;

int leaf_error_word(int** out) {
  void* p = nullptr;
  const cudaError_t e = cached_symbol_address(
      g_leaf_err_cache, [](void** q) { return cudaGetSymbolAddress(q, g_leaf_err); }, &p);
  if (e != cudaSuccess) return cuda_status(e);
  *out = static_cast<int*>(p);
  return JB_OK;
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

// The same un-permute as a gather: out[j] = acc4[inv_perm[j]], so the 12-byte
// output rows are written in order (coalesced) and only the 16-byte reads
// scatter; the scatter form writes each row into a different place.
__global__ void k_gather_unsorted(int64_t n, const float4* __restrict__ acc4, const int64_t* __restrict__ inv_perm,
                                  float* __restrict__ out_acc, float* __restrict__ out_pot) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const float4 a = acc4[inv_perm[j]];
  out_acc[3 * j] = a.x;
  out_acc[3 * j + 1] = a.y;
  out_acc[3 * j + 2] = a.z;
  if (out_pot) out_pot[j] = a.w;
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

__global__ void k_validate_leaves(int num_nodes, int num_internal, const int2* __restrict__ ranges, int max_occ,
                                  int* bad) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int b = 0;
  for (int64_t i = num_internal + tid; i < num_nodes; i += stride) {
    const int2 r = ranges[i];
    const int64_t cnt = (int64_t)r.y - r.x + 1;
    if (r.x < 0 || cnt < 1 || cnt > max_occ) ++b;
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

#define JB_ADJ_ORDERS(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9)

template <typename Fn>
static int dispatch_adj(int p, Fn&& fn) {
  switch (p) {
#define JB_ACASE(PP) \
  case PP:           \
    return fn(RunAdj<PP>{});
    JB_ADJ_ORDERS(JB_ACASE)
#undef JB_ACASE
    default:
      return JB_ERR_ORDER;
  }
}

// ---------------------------------------------------------------------------
// Verification: FP64 direct sum on sampled targets (the error report every
// result carries; runtime/reference.py:292 semantics, self pair excluded).
// A cluster of kDirectParts blocks per target: block r of the cluster sums
// the sources of its r-th share with 256 threads in FP64 and reduces them
// in shared memory; after the cluster barrier, block 0 adds the blocks'
// sums in rank order through distributed shared memory, so the result does
// not depend on scheduling and needs no scratch.
// ---------------------------------------------------------------------------
constexpr int kDirectParts = 8;

__global__ void __cluster_dims__(kDirectParts, 1, 1) __launch_bounds__(256)
    k_direct_f64(int64_t n, const float4* __restrict__ pos4, int64_t nt, const int* __restrict__ tsorted, double G,
                 double eps2, double* __restrict__ out) {
  __shared__ double red[4][256];
  cg::cluster_group cluster = cg::this_cluster();
  const int part = (int)cluster.block_rank();
  const int64_t q = blockIdx.x / kDirectParts;  // every block of a cluster has the same target
  const int i = q < nt ? tsorted[q] : -1;
  double ax = 0, ay = 0, az = 0, ph = 0;
  if (q < nt) {
    const float4 ti = pos4[i];
    const double xi = ti.x, yi = ti.y, zi = ti.z;
    const int64_t j0 = n * part / kDirectParts, j1 = n * (part + 1) / kDirectParts;
    for (int64_t j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
      if (j == i) continue;
      const float4 s = pos4[j];
      const double dx = xi - s.x, dy = yi - s.y, dz = zi - s.z;
      const double d2 = dx * dx + dy * dy + dz * dz + eps2;
      const double ir = rsqrt(d2);
      const double w = (double)s.w * ir * ir * ir;
      ax += w * dx;
      ay += w * dy;
      az += w * dz;
      ph += (double)s.w * ir;
    }
  }
  red[0][threadIdx.x] = ax;
  red[1][threadIdx.x] = ay;
  red[2][threadIdx.x] = az;
  red[3][threadIdx.x] = ph;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + o];
    __syncthreads();
  }
  cluster.sync();  // every block's sum is in its shared memory
  if (part == 0 && q < nt && threadIdx.x < 4) {
    double sum = 0;
    for (int r = 0; r < kDirectParts; ++r) sum += cluster.map_shared_rank(&red[0][0], r)[threadIdx.x * 256];
    out[4 * q + threadIdx.x] = -G * sum;
  }
  cluster.sync();  // the other blocks' shared memory stays until block 0 has read it
}

// Throughput probe.  mode 0: FP32 FMA chains (8 independent per thread);
// 1: MUFU rsqrt chains; 2: packed f32x2 FMA chains (8 per thread); 3: the
// near field's particle-pair arithmetic on register-resident sources (the
// packed step of chunk_sums: 2 pairs per step, 3 targets' accumulators) --
// the pair rate the FP32 and MUFU pipes allow for that instruction mix.
__global__ void k_probe(int iters, int use_mufu, float* out) {
  if (use_mufu == 2) {
    f32x2 a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = f2(1.0f + 1e-3f * (threadIdx.x + k), 1.0f - 1e-3f * k);
    const f32x2 b = f2(0.999f, 0.999f), c = f2(1e-4f, 1e-4f);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
      for (int k = 0; k < 8; ++k) a[k] = f2_fma(a[k], b, c);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      float lo, hi;
      f2_split(a[k], lo, hi);
      s += lo + hi;
    }
    if (s == 12345.678f) out[threadIdx.x] = s;
    return;
  }
  if (use_mufu == 3) {
    f32x2 sx[4], sy[4], sz[4], sm[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      sx[k] = f2(0.1f * k + 1e-3f * threadIdx.x, 0.2f * k);
      sy[k] = f2(0.3f * k, 0.1f + 0.05f * k);
      sz[k] = f2(-0.2f * k, 0.4f);
      sm[k] = f2(1e-3f, 2e-3f);
    }
    const f32x2 E2 = f2(1e-4f, 1e-4f);
    f32x2 TX[3], TY[3], TZ[3], AX[3], AY[3], AZ[3];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      TX[t] = f2(1.f + t, 1.f + t);
      TY[t] = f2(2.f, 2.f);
      TZ[t] = f2(0.5f * t, 0.5f * t);
      AX[t] = AY[t] = AZ[t] = f2(0.f, 0.f);
    }
    const f32x2 step = f2(1e-6f, -1e-6f);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
      for (int t = 0; t < 3; ++t) {  // the targets move, so nothing is loop-invariant
        TX[t] = f2_add(TX[t], step);
        TY[t] = f2_add(TY[t], step);
        TZ[t] = f2_add(TZ[t], step);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
#pragma unroll
        for (int t = 0; t < 3; ++t) {
          const f32x2 dx = f2_sub(TX[t], sx[k]), dy = f2_sub(TY[t], sy[k]), dz = f2_sub(TZ[t], sz[k]);
          const f32x2 d2 = f2_fma(dx, dx, f2_fma(dy, dy, f2_fma(dz, dz, E2)));
          float d2a, d2b;
          f2_split(d2, d2a, d2b);
          const f32x2 ir = f2(rsqrt_ftz(d2a), rsqrt_ftz(d2b));
          const f32x2 w = f2_mul(f2_mul(sm[k], ir), f2_mul(ir, ir));
          AX[t] = f2_fma(w, dx, AX[t]);
          AY[t] = f2_fma(w, dy, AY[t]);
          AZ[t] = f2_fma(w, dz, AZ[t]);
        }
      }
    }
    float s = 0.f;
#pragma unroll
    for (int t = 0; t < 3; ++t) {
      float lo, hi;
      f2_split(f2_add(f2_add(AX[t], AY[t]), AZ[t]), lo, hi);
      s += lo + hi;
    }
    if (s == 12345.678f) out[threadIdx.x] = s;
    return;
  }
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = 1.0f + 1e-3f * (threadIdx.x + k);
  const float b = 0.999f, c = 1e-4f;
  if (use_mufu) {
    for (int it = 0; it < iters; ++it) {
#pragma unroll
      for (int k = 0; k < 8; ++k) a[k] = rsqrtf(a[k] + c);
    }
  } else {
    for (int it = 0; it < iters; ++it) {
#pragma unroll
      for (int k = 0; k < 8; ++k) a[k] = fmaf(a[k], b, c);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (s == 12345.678f) out[threadIdx.x] = s;  // keeps the chains live
}

// ---------------------------------------------------------------------------
// Near field: warp per leaf unit, lane = target particle.  For the pair
// (k, l), d = x_k - x_l, q = (|d|^2 + eps^2)^-1/2:
//   dL/dx_k += G [ -m_l q^3 w_k + m_k q^3 w_l + 3 q^5 (m_l (w_k.d) - m_k (w_l.d)) d ]
//   dL/dm_k += G q^3 (w_l . d)
// which needs l in near(k) <=> k in near(l) (the lists are symmetric).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void adj_near_pair(float4 tk, float4 wk, float4 s, float4 ws, float eps2, bool skip,
                                              float* a) {
  const float dx = tk.x - s.x, dy = tk.y - s.y, dz = tk.z - s.z;
  const float d2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
  const float q = skip ? 0.f : rsqrt_ftz(d2);
  const float q3 = q * q * q;
  const float q5 = q3 * q * q;
  const float wkd = wk.x * dx + wk.y * dy + wk.z * dz;
  const float wld = ws.x * dx + ws.y * dy + ws.z * dz;
  const float c = 3.f * q5 * (s.w * wkd - tk.w * wld);
  const float aml = -s.w * q3, amk = tk.w * q3;
  a[0] += aml * wk.x + amk * ws.x + c * dx;
  a[1] += aml * wk.y + amk * ws.y + c * dy;
  a[2] += aml * wk.z + amk * ws.z + c * dz;
  a[3] += q3 * wld;
}

static __global__ void __launch_bounds__(32 * kWarpsPerBlock) k_adj_near(
    const float4* __restrict__ pos4, const float4* __restrict__ w4, int num_internal, int num_units,
    const int4* __restrict__ units, const int2* __restrict__ aux, const int2* __restrict__ runs,
    const int2* __restrict__ ranges, float G, float eps2, float4* __restrict__ out, float4* __restrict__ partial) {
  __shared__ float4 sP[kWarpsPerBlock][32];
  __shared__ float4 sW[kWarpsPerBlock][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int u = blockIdx.x * kWarpsPerBlock + warp;
  if (u >= num_units) return;
  const int4 U = units[u];
  const int2 ax = aux[u];
  const int2 rg = ranges[num_internal + U.x];
  const int nt = rg.y - rg.x + 1;
  if (nt > kMaxLeaf) return;  // a split leaf's partial row holds kMaxLeaf targets (jb_validate_leaves)
  float a[4] = {0.f, 0.f, 0.f, 0.f};
  // targets beyond 32 particles take further passes
  for (int t0 = 0; t0 < nt; t0 += 32) {
    const int tl = t0 + lane;
    const bool active = tl < nt;
    const float4 tk = active ? pos4[rg.x + tl] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 wk = active ? w4[rg.x + tl] : make_float4(0.f, 0.f, 0.f, 0.f);
    a[0] = a[1] = a[2] = a[3] = 0.f;
    if (ax.y & 1) {
      for (int s0 = 0; s0 < nt; s0 += 32) {
        const int j = s0 + lane;
        sP[warp][lane] = (j < nt) ? pos4[rg.x + j] : JB_PAD4;
        sW[warp][lane] = (j < nt) ? w4[rg.x + j] : make_float4(0.f, 0.f, 0.f, 0.f);
        __syncwarp();
#pragma unroll 8
        for (int q = 0; q < 32; ++q)
          adj_near_pair(tk, wk, sP[warp][q], sW[warp][q], eps2, (s0 + q == tl) || (s0 + q >= nt), a);
        __syncwarp();
      }
    }
    const int nsrc = U.w;
    int r = U.y, rbase = 0;
    int2 run = (U.z > U.y) ? runs[r] : make_int2(0, 0);
    auto fetch = [&](int f, float4& p, float4& w) {  // source f of the unit (padding past the end)
      while (f >= rbase + run.y && r + 1 < U.z) {
        rbase += run.y;
        ++r;
        run = runs[r];
      }
      const bool ok = f < nsrc;
      p = ok ? pos4[run.x + (f - rbase)] : JB_PAD4;
      w = ok ? w4[run.x + (f - rbase)] : make_float4(0.f, 0.f, 0.f, 0.f);
    };
    float4 qp = JB_PAD4, qw = make_float4(0.f, 0.f, 0.f, 0.f);
    if (nsrc > 0) fetch(lane, qp, qw);
    for (int base = 0; base < nsrc; base += 32) {
      sP[warp][lane] = qp;
      sW[warp][lane] = qw;
      __syncwarp();
      if (base + 32 < nsrc) fetch(base + 32 + lane, qp, qw);  // the next chunk, while this one is used
#pragma unroll 8
      for (int q = 0; q < 32; ++q) adj_near_pair(tk, wk, sP[warp][q], sW[warp][q], eps2, base + q >= nsrc, a);
      __syncwarp();
    }
    if (active) {
      const float4 res = make_float4(G * a[0], G * a[1], G * a[2], G * a[3]);
      if (ax.x < 0) out[rg.x + tl] = res;
      else partial[(size_t)ax.x * kMaxLeaf + tl] = res;
    }
  }
}

// M2L centre-gradient gather, thread per node u: for every pair e = (u <- v)
// of u's list, g_e belongs to u as target and the reverse pair (v <- u)
// (index rev[e]) contributes -g_rev(e) to u as source.
__global__ void k_adj_m2l_gather(int num_nodes, const int64_t* __restrict__ far_off, const int* __restrict__ rev,
                                 const float4* __restrict__ g4, float4* __restrict__ cbar4) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= num_nodes) return;
  float x = 0.f, y = 0.f, z = 0.f;
  for (int64_t e = far_off[u]; e < far_off[u + 1]; ++e) {
    const float4 a = g4[e], b = g4[rev[e]];
    x += a.x - b.x;
    y += a.y - b.y;
    z += a.z - b.z;
  }
  float4 c = cbar4[u];
  c.x += x;
  c.y += y;
  c.z += z;
  cbar4[u] = c;
}

static inline unsigned blocks_1d(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

}  // namespace jb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace jb;

#define ST(s) reinterpret_cast<cudaStream_t>(s)

extern "C" {

JB_API int jb_set_level_split(int m2m_max_parents, int l2l_max_parents) {
  if (m2m_max_parents < 0 || l2l_max_parents < 0) return JB_ERR_ARG;
  jb::g_split_max_parents[0] = m2m_max_parents;
  jb::g_split_max_parents[1] = l2l_max_parents;
  return JB_OK;
}

JB_API int jb_set_leaf_form(int chunk_major) {
  if (chunk_major != 0 && chunk_major != 1) return JB_ERR_ARG;
  jb::g_leaf_flat = chunk_major;
  return JB_OK;
}

JB_API int jb_set_m2l_fetch(int warp_rows) {
  if (warp_rows != 0 && warp_rows != 1) return JB_ERR_ARG;
  jb::g_m2l_coop = warp_rows;
  return JB_OK;
}

JB_API int jb_coeff_stride(int p) { return (p >= 1 && p <= JB_MAX_ORDER) ? cstride(p) : 0; }

JB_API int jb_graph_instantiate(void* graph, int node_priority, void** exec) {
  if (!graph || !exec || (node_priority != 0 && node_priority != 1)) return JB_ERR_ARG;
  cudaGraphExec_t e = nullptr;
  const cudaError_t rc = cudaGraphInstantiateWithFlags(
      &e, static_cast<cudaGraph_t>(graph), node_priority ? cudaGraphInstantiateFlagUseNodePriority : 0);
  if (rc != cudaSuccess) return cuda_status(rc);
  *exec = e;
  return JB_OK;
}

JB_API int jb_graph_launch(void* exec, void* stream) {
  if (!exec) return JB_ERR_ARG;
  const cudaError_t rc = cudaGraphLaunch(static_cast<cudaGraphExec_t>(exec), ST(stream));
  return cuda_status(rc);
}

JB_API int jb_graph_exec_destroy(void* exec) {
  if (!exec) return JB_ERR_ARG;
  return cuda_status(cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(exec)));
}

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

JB_API int jb_gather_unsorted(int64_t n, const float* acc4, const int64_t* inv_perm, float* out_acc, float* out_pot,
                              void* stream) {
  if (n < 0 || (n > 0 && (!acc4 || !inv_perm || !out_acc))) return JB_ERR_ARG;
  if (n == 0) return JB_OK;
  k_gather_unsorted<<<blocks_1d(n, 256), 256, 0, ST(stream)>>>(n, reinterpret_cast<const float4*>(acc4), inv_perm,
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

JB_API int jb_validate_leaves(int num_nodes, int num_internal, const int* node_ranges, int max_occupancy,
                              int* bad_count_dev, void* stream) {
  if (num_nodes < 1 || num_internal < 0 || num_internal >= num_nodes || !node_ranges || !bad_count_dev ||
      max_occupancy < 1 || max_occupancy > kMaxLeaf)
    return JB_ERR_ARG;
  const cudaError_t e = cudaMemsetAsync(bad_count_dev, 0, sizeof(int), ST(stream));
  if (e != cudaSuccess) return cuda_status(e);
  k_validate_leaves<<<148 * 4, 256, 0, ST(stream)>>>(num_nodes, num_internal, reinterpret_cast<const int2*>(node_ranges),
                                                     max_occupancy, bad_count_dev);
  return launch_status();
}

JB_API int jb_leaf_eval_errors(int* flags, int clear, void* stream) {
  if (!flags) return JB_ERR_ARG;
  int* w = nullptr;
  int rc = leaf_error_word(&w);
  if (rc != JB_OK) return rc;
  cudaError_t e = cudaMemcpyAsync(flags, w, sizeof(int), cudaMemcpyDeviceToHost, ST(stream));
  if (e == cudaSuccess && clear) e = cudaMemsetAsync(w, 0, sizeof(int), ST(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(ST(stream));
  return cuda_status(e);
}

JB_API int jb_direct_f64(int64_t n, const float* pos4, int64_t num_targets, const int* targets_sorted, double G,
                         double eps2, double* out4, void* stream) {
  if (n < 1 || num_targets < 0 || (num_targets > 0 && (!pos4 || !targets_sorted || !out4))) return JB_ERR_ARG;
  if (num_targets == 0) return JB_OK;
  if (num_targets > (int64_t)0x7fffffff / kDirectParts) return JB_ERR_ARG;
  k_direct_f64<<<(unsigned)(num_targets * kDirectParts), 256, 0, ST(stream)>>>(
      n, reinterpret_cast<const float4*>(pos4), num_targets, targets_sorted, G, eps2, out4);
  return launch_status();
}

JB_API int jb_probe_throughput(int blocks, int iters, int use_mufu, float* sink, void* stream) {
  if (blocks < 1 || iters < 1 || !sink) return JB_ERR_ARG;
  k_probe<<<blocks, 256, 0, ST(stream)>>>(iters, use_mufu, sink);
  return launch_status();
}

JB_API int jb_p2m(int p, const float* pos4, int num_nodes, int num_internal, const int* node_ranges, float* centers,
                  float* mult, void* stream) {
  if (!pos4 || !node_ranges || !centers || !mult || num_nodes < 1 || num_internal < 0) return JB_ERR_ARG;
  return dispatch<RunP2M>(p, pos4, num_nodes, num_internal, node_ranges, centers, mult, ST(stream));
}

JB_API int jb_m2m_level(int p, int first, int last, const int* left, const int* right, const int* node_ranges,
                        float* centers, float* mult, void* stream) {
  if (first < 0 || last < first || (last > first && (!left || !right || !node_ranges || !centers || !mult)))
    return JB_ERR_ARG;
  return dispatch<RunM2M>(p, first, last, left, right, node_ranges, centers, mult, ST(stream));
}

JB_API int jb_m2l(int p, int mode, int num_units, const int* units, const float* mult, const float* centers,
                  const int* far_src, float* locals, float* partials, int num_split, const int* split,
                  void* stream) {
  if (num_units < 0 || num_split < 0 ||
      (num_units > 0 && (!units || !mult || !centers || !far_src || !locals)) ||
      (num_split > 0 && (!split || !partials || !locals)))
    return JB_ERR_ARG;
  if (mode != JB_M2L_FP32) return JB_ERR_UNSUPPORTED;
  return dispatch<RunM2L>(p, num_units, units, mult, centers, far_src, locals, partials, num_split, split,
                          ST(stream));
}

JB_API int jb_m2l_weighted(int p, int num_units, const int* units, const float* mult, const float* centers,
                           const int* far_src, const float* far_w, float* locals, float* partials, int num_split,
                           const int* split, void* stream) {
  if (num_units < 0 || num_split < 0 ||
      (num_units > 0 && (!units || !mult || !centers || !far_src || !far_w || !locals)) ||
      (num_split > 0 && (!split || !partials || !locals)))
    return JB_ERR_ARG;
  return dispatch<RunM2L>(p, num_units, units, mult, centers, far_src, locals, partials, num_split, split,
                          ST(stream), false, 0, far_w);
}

}  // extern "C"

namespace jb {
// Side streams of the gear M2L, one set per device, made on first use: the
// gears' launches touch disjoint rows (a target split over several units,
// whatever their gears, writes only its own partial rows), so they run side
// by side instead of one after the other, joined back by events.
struct GearStreams {
  cudaStream_t s[8];
  cudaEvent_t fork, join[8];
};

static int gear_streams(GearStreams** out) {
  static std::mutex mu;
  static GearStreams per_dev[64];
  static bool made[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e);
  if (dev < 0 || dev >= 64) return JB_ERR_CUDA;
  std::lock_guard<std::mutex> lk(mu);
  if (!made[dev]) {
    GearStreams& g = per_dev[dev];
    e = cudaEventCreateWithFlags(&g.fork, cudaEventDisableTiming);
    for (int i = 0; i < 8 && e == cudaSuccess; ++i) {
      e = cudaStreamCreateWithFlags(&g.s[i], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g.join[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) return cuda_status(e);
    made[dev] = true;
  }
  *out = &per_dev[dev];
  return JB_OK;
}
}  // namespace jb

extern "C" {

JB_API int jb_m2l_gears(int p_max, int mode, int num_gears, const int* gear_orders, const int64_t* gear_unit_offsets,
                        const int* units, const float* mult, const float* centers, const int* far_src,
                        float* locals, float* partials, int num_split, const int* split, void* stream) {
  if (p_max < 1 || p_max > JB_MAX_ORDER) return JB_ERR_ORDER;
  if (num_gears < 1 || !gear_orders || !gear_unit_offsets || num_split < 0 || (num_split > 0 && (!split || !partials)))
    return JB_ERR_ARG;
  if (mode != JB_M2L_FP32) return JB_ERR_UNSUPPORTED;
  const int rs = cstride(p_max);
  for (int g = 0; g < num_gears; ++g) {
    const int pg = gear_orders[g];
    const int64_t u0 = gear_unit_offsets[g], u1 = gear_unit_offsets[g + 1];
    if (pg < 1 || pg > p_max || u0 < 0 || u1 < u0) return JB_ERR_ARG;
    if (u1 > u0 && (!units || !mult || !centers || !far_src || !locals)) return JB_ERR_ARG;
  }
  // the last gear (the highest order, most of the work) on the caller's
  // stream, the others on side streams forked from it and joined back
  GearStreams* gs = nullptr;
  const bool side = num_gears > 1 && num_gears <= 9;
  if (side) {
    const int rc = gear_streams(&gs);
    if (rc) return rc;
    const cudaError_t e = cudaEventRecord(gs->fork, ST(stream));
    if (e != cudaSuccess) return cuda_status(e);
  }
  for (int g = 0; g < num_gears; ++g) {
    const int64_t u0 = gear_unit_offsets[g], u1 = gear_unit_offsets[g + 1];
    if (u1 == u0) continue;
    cudaStream_t st = ST(stream);
    if (side && g < num_gears - 1) {
      st = gs->s[g];
      const cudaError_t e = cudaStreamWaitEvent(st, gs->fork, 0);
      if (e != cudaSuccess) return cuda_status(e);
    }
    const int rc = dispatch<RunM2L>(gear_orders[g], (int)(u1 - u0), units + 4 * u0, mult, centers, far_src, locals,
                                    partials, 0, (const int*)nullptr, st, false, rs);
    if (rc) return rc;
    if (side && g < num_gears - 1) {
      cudaError_t e = cudaEventRecord(gs->join[g], st);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(ST(stream), gs->join[g], 0);
      if (e != cudaSuccess) return cuda_status(e);
    }
  }
  if (num_split > 0) {
    k_m2l_reduce<<<blocks_1d((int64_t)num_split * rs, 256), 256, 0, ST(stream)>>>(
        num_split, reinterpret_cast<const int4*>(split), partials, locals, rs);
    return launch_status();
  }
  return JB_OK;
}

JB_API int jb_m2l_mixed(int p_max, int num_units, const int* units, const int* bounds, const float* mult,
                        const float* centers, const int* far_src, float* locals, float* partials, int num_split,
                        const int* split, void* stream) {
  if (p_max < 1 || p_max > JB_MAX_ORDER) return JB_ERR_ORDER;
  if (num_units < 0 || num_split < 0 || (num_split > 0 && (!split || !partials)))
    return JB_ERR_ARG;
  if (num_units > 0 && (!units || !bounds || !mult || !centers || !far_src || !locals)) return JB_ERR_ARG;
  return dispatch<RunM2LMixed>(p_max, num_units, units, bounds, mult, centers, far_src, locals, partials, num_split,
                               split, ST(stream));
}

JB_API int jb_l2l_leaves(int p, int num_units, const int* units, const int* anc, const float* centers,
                         float* locals, void* stream) {
  if (num_units < 0 || (num_units > 0 && (!units || !anc || !centers || !locals))) return JB_ERR_ARG;
  return dispatch<RunL2LLeaves>(p, num_units, units, anc, centers, locals, ST(stream));
}

JB_API int jb_l2l_level(int p, int first, int last, const int* left, const int* right, const float* centers,
                        float* locals, void* stream) {
  if (first < 0 || last < first || (last > first && (!left || !right || !centers || !locals))) return JB_ERR_ARG;
  return dispatch<RunL2L>(p, first, last, left, right, centers, locals, ST(stream));
}

JB_API int jb_leaf_eval_weighted(int p, int p2p_mode, const float* pos4, const int* rung, int num_level_weights,
                                 const float* level_weights, int num_internal, int num_units, const int* units,
                                 const int* aux, const int* runs, const int* node_ranges, const float* centers,
                                 const float* locals, float G, float eps2, float* out_acc4, float* partials,
                                 int num_split, const int* split, void* stream) {
  if (num_units < 0 || num_split < 0 || num_internal < 0 || !rung || !level_weights || num_level_weights < 1 ||
      num_level_weights > 32 ||
      (num_units > 0 && (!pos4 || !units || !aux || !runs || !node_ranges || !centers || !locals || !out_acc4)) ||
      (num_split > 0 && (!split || !partials || !out_acc4 || !node_ranges)))
    return JB_ERR_ARG;
  if (p2p_mode & ~(JB_P2P_KAHAN | JB_P2P_POTENTIAL | JB_P2P_FAR_ONLY | JB_P2P_NEAR_ONLY)) return JB_ERR_ARG;
  if ((p2p_mode & JB_P2P_FAR_ONLY) && (p2p_mode & JB_P2P_NEAR_ONLY)) return JB_ERR_ARG;
  int* err = nullptr;
  const int rc = leaf_error_word(&err);
  if (rc != JB_OK) return rc;
  return dispatch<RunLeafEval>(p, p2p_mode, pos4, num_internal, num_units, units, aux, runs, node_ranges, centers,
                               locals, G, eps2, out_acc4, partials, num_split, split, ST(stream), rung,
                               level_weights, num_level_weights, false, 0x7fffffff, err);
}

JB_API int jb_leaf_eval(int p, int p2p_mode, const float* pos4, int num_internal, int num_units, const int* units,
                        const int* aux, const int* runs, const int* node_ranges, const float* centers,
                        const float* locals, float G, float eps2, float* out_acc4, float* partials, int num_split,
                        const int* split, void* stream) {
  if (num_units < 0 || num_split < 0 || num_internal < 0 ||
      (num_units > 0 && (!pos4 || !units || !aux || !runs || !node_ranges || !centers || !locals || !out_acc4)) ||
      (num_split > 0 && (!split || !partials || !out_acc4 || !node_ranges)))
    return JB_ERR_ARG;
  constexpr int parts = JB_P2P_FAR_ONLY | JB_P2P_NEAR_ONLY | JB_P2P_NEAR_FIRST | JB_P2P_FAR_AFTER;
  if (p2p_mode & ~(JB_P2P_KAHAN | JB_P2P_POTENTIAL | parts)) return JB_ERR_ARG;
  if (__builtin_popcount(p2p_mode & parts) > 1) return JB_ERR_ARG;  // at most one of the four
  int* err = nullptr;
  const int rc = leaf_error_word(&err);
  if (rc != JB_OK) return rc;
  return dispatch<RunLeafEval>(p, p2p_mode, pos4, num_internal, num_units, units, aux, runs, node_ranges, centers,
                               locals, G, eps2, out_acc4, partials, num_split, split, ST(stream), nullptr, nullptr,
                               1, jb::g_leaf_flat != 0, 0x7fffffff, err);
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

// ---------------------------------------------------------------------------
// Adjoint (VJP) of the pass at fixed topology.
// ---------------------------------------------------------------------------
JB_API int jb_adj_near(const float* pos4, const float* w4, int num_internal, int num_units, const int* units,
                       const int* aux, const int* runs, const int* node_ranges, float G, float eps2, float* out_xm4,
                       float* partials, int num_split, const int* split, void* stream) {
  if (num_units < 0 || num_split < 0 || num_internal < 0 ||
      (num_units > 0 && (!pos4 || !w4 || !units || !aux || !runs || !node_ranges || !out_xm4)) ||
      (num_split > 0 && (!split || !partials || !out_xm4 || !node_ranges)))
    return JB_ERR_ARG;
  if (num_units > 0) {
    k_adj_near<<<blocks_1d(num_units, kWarpsPerBlock), 32 * kWarpsPerBlock, 0, ST(stream)>>>(
        reinterpret_cast<const float4*>(pos4), reinterpret_cast<const float4*>(w4), num_internal, num_units,
        reinterpret_cast<const int4*>(units), reinterpret_cast<const int2*>(aux), reinterpret_cast<const int2*>(runs),
        reinterpret_cast<const int2*>(node_ranges), G, eps2, reinterpret_cast<float4*>(out_xm4),
        reinterpret_cast<float4*>(partials));
    const int rc = launch_status();
    if (rc) return rc;
  }
  if (num_split > 0) {
    k_leaf_reduce<false><<<blocks_1d((int64_t)num_split * kMaxLeaf, 256), 256, 0, ST(stream)>>>(
        num_split, reinterpret_cast<const int4*>(split), num_internal, reinterpret_cast<const int2*>(node_ranges),
        reinterpret_cast<const float4*>(partials), reinterpret_cast<float4*>(out_xm4), 0x7fffffff, nullptr);
    return launch_status();
  }
  return JB_OK;
}

JB_API int jb_adj_leaf_far(int p, const float* pos4, const float* w4, int num_nodes, int num_internal,
                           const int* node_ranges, const float* centers, const float* locals, float G, float* xm4,
                           float* lbar, float* cbar4, void* stream) {
  if (!pos4 || !w4 || !node_ranges || !centers || !locals || !xm4 || !lbar || !cbar4 || num_nodes < 1 ||
      num_internal < 0 || num_internal >= num_nodes)
    return JB_ERR_ARG;
  return dispatch_adj(p, [&](auto R) {
    return decltype(R)::leaf_far(pos4, w4, num_nodes, num_internal, node_ranges, centers, locals, G, xm4, lbar,
                                 cbar4, ST(stream));
  });
}

JB_API int jb_adj_l2l_level(int p, int first, int last, const int* left, const int* right, const float* centers,
                            const float* locals, float* lbar, float* cbar4, void* stream) {
  if (first < 0 || last < first || (last > first && (!left || !right || !centers || !locals || !lbar || !cbar4)))
    return JB_ERR_ARG;
  return dispatch_adj(p, [&](auto R) {
    return decltype(R)::l2l_level(first, last, left, right, centers, locals, lbar, cbar4, ST(stream));
  });
}

JB_API int jb_adj_m2l(int p, int num_units, const int* units, const float* lbar, const float* centers,
                      const int* far_src, float* mbar, float* partials, int num_split, const int* split,
                      void* stream) {
  if (num_units < 0 || num_split < 0 || (num_units > 0 && (!units || !lbar || !centers || !far_src || !mbar)) ||
      (num_split > 0 && (!split || !partials || !mbar)))
    return JB_ERR_ARG;
  if (p < 1 || p > JB_ADJ_MAX_ORDER) return JB_ERR_ORDER;
  return dispatch<RunM2L>(p, num_units, units, lbar, centers, far_src, mbar, partials, num_split, split, ST(stream),
                          true);
}

JB_API int jb_adj_m2l_centers(int p, int num_nodes, int64_t num_pairs, const int* pair_tgt, const int* far_src,
                              const int64_t* far_off, const int* rev, const float* mult, const float* lbar,
                              const float* centers, float* g4, float* cbar4, void* stream) {
  if (num_nodes < 1 || num_pairs < 0 || !far_off || !cbar4 ||
      (num_pairs > 0 && (!pair_tgt || !far_src || !rev || !mult || !lbar || !centers || !g4)))
    return JB_ERR_ARG;
  if (num_pairs == 0) return (p >= 1 && p <= JB_ADJ_MAX_ORDER) ? JB_OK : JB_ERR_ORDER;
  const int rc = dispatch_adj(p, [&](auto R) {
    return decltype(R)::m2l_pairs(num_pairs, pair_tgt, far_src, mult, lbar, centers, g4, ST(stream));
  });
  if (rc) return rc;
  k_adj_m2l_gather<<<blocks_1d(num_nodes, 128), 128, 0, ST(stream)>>>(
      num_nodes, far_off, rev, reinterpret_cast<const float4*>(g4), reinterpret_cast<float4*>(cbar4));
  return launch_status();
}

JB_API int jb_adj_m2m_level(int p, int first, int last, const int* left, const int* right, const float* centers,
                            const float* mult, float* mbar, float* cbar4, void* stream) {
  if (first < 0 || last < first || (last > first && (!left || !right || !centers || !mult || !mbar || !cbar4)))
    return JB_ERR_ARG;
  return dispatch_adj(p, [&](auto R) {
    return decltype(R)::m2m_level(first, last, left, right, centers, mult, mbar, cbar4, ST(stream));
  });
}

JB_API int jb_adj_p2m(int p, const float* pos4, int num_nodes, int num_internal, const int* node_ranges,
                      const float* centers, const float* mbar, const float* cbar4, float* xm4, void* stream) {
  if (!pos4 || !node_ranges || !centers || !mbar || !cbar4 || !xm4 || num_nodes < 1 || num_internal < 0 ||
      num_internal >= num_nodes)
    return JB_ERR_ARG;
  return dispatch_adj(p, [&](auto R) {
    return decltype(R)::p2m(pos4, num_nodes, num_internal, node_ranges, centers, mbar, cbar4, xm4, ST(stream));
  });
}

}  // extern "C"
