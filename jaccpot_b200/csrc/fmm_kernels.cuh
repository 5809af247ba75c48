#pragma once
// sm_100a kernels of the FMM evaluation pass, templated on the expansion order.
// Each order is instantiated in its own translation unit (fmm_order.cu built
// with -DJB_ORDER=P); the C-ABI entry points live in fmm_capi.cu.
//
// Work decomposition (nothing here uses atomics; every output element has one
// writer, so results are run-to-run deterministic):
//   P2M        warp per leaf: COM by warp reduction, U_n^m per lane, transpose
//              reduction of the (p+1)^2 coefficients through shared memory;
//   M2M / L2L  thread per (parent) / (parent, child), one launch per level;
//   M2L        thread per target node walking its CSR source list, targets
//              pre-sorted by list length so warps stay converged; the
//              per-thread local accumulates in a shared-memory column;
//   leaf eval  warp per target leaf: L2P (lane = particle, the leaf's local
//              staged once in shared memory) fused with the P2P near field,
//              source leaves staged 32 particles at a time in shared memory.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <cstring>

#include "../../include/jaccpot_b200.h"
#include "fmm_ops.cuh"

namespace jb {

// Defined in fmm_capi.cu.
int cuda_status(cudaError_t e);
inline int launch_status() { return cuda_status(cudaGetLastError()); }

// ---------------------------------------------------------------------------
// P2M (+ leaf COM).
// ---------------------------------------------------------------------------
constexpr int kWarpsPerBlock = 4;

template <int P>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_p2m(const float4* __restrict__ pos4, int num_nodes, int num_internal,
                                                              const int2* __restrict__ ranges, float4* __restrict__ centers,
                                                              float* __restrict__ mult) {
  constexpr int C = csize(P), CS = cstride(P), CP = C + 1;
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* red = smem + warp * 32 * CP;
  const int leaf = blockIdx.x * kWarpsPerBlock + warp;
  const int node = num_internal + leaf;
  if (node >= num_nodes) return;
  const int2 rg = ranges[node];
  // COM
  float sm = 0.f, sx = 0.f, sy = 0.f, sz = 0.f;
  for (int i = rg.x + lane; i <= rg.y; i += 32) {
    const float4 q = pos4[i];
    sm += q.w;
    sx = fmaf(q.w, q.x, sx);
    sy = fmaf(q.w, q.y, sy);
    sz = fmaf(q.w, q.z, sz);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sm += __shfl_xor_sync(0xffffffffu, sm, o);
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
    sz += __shfl_xor_sync(0xffffffffu, sz, o);
  }
  float cx, cy, cz;
  if (sm > 0.f) {
    const float inv = 1.f / sm;
    cx = sx * inv;
    cy = sy * inv;
    cz = sz * inv;
  } else {
    cx = cy = cz = 0.f;
    int cnt = 0;
    for (int i = rg.x + lane; i <= rg.y; i += 32) {
      const float4 q = pos4[i];
      cx += q.x;
      cy += q.y;
      cz += q.z;
      ++cnt;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      cx += __shfl_xor_sync(0xffffffffu, cx, o);
      cy += __shfl_xor_sync(0xffffffffu, cy, o);
      cz += __shfl_xor_sync(0xffffffffu, cz, o);
      cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    }
    const float inv = 1.f / (float)cnt;
    cx *= inv;
    cy *= inv;
    cz *= inv;
  }
  if (lane == 0) centers[node] = make_float4(cx, cy, cz, sm);
  // P2M: per-lane partial sums, then reduce across lanes through shared memory.
  float acc[C];
#pragma unroll
  for (int k = 0; k < C; ++k) acc[k] = 0.f;
  for (int i = rg.x + lane; i <= rg.y; i += 32) {
    const float4 q = pos4[i];
    float U[C];
    solid_harmonics<P>(q.x - cx, q.y - cy, q.z - cz, U);
#pragma unroll
    for (int k = 0; k < C; ++k) acc[k] = fmaf(q.w, U[k], acc[k]);
  }
#pragma unroll
  for (int k = 0; k < C; ++k) red[lane * CP + k] = acc[k];
  __syncwarp();
  float* out = mult + (size_t)node * CS;
  for (int k = lane; k < CS; k += 32) {
    float s = 0.f;
    if (k < C) {
#pragma unroll 8
      for (int j = 0; j < 32; ++j) s += red[j * CP + k];
    }
    out[k] = s;
  }
}

// ---------------------------------------------------------------------------
// M2M, one level (+ internal COM from the children).
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(128) k_m2m_level(int first, int last, const int* __restrict__ left,
                                                   const int* __restrict__ right, float4* __restrict__ centers,
                                                   float* __restrict__ mult) {
  constexpr int C = csize(P), CS = cstride(P);
  const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= last) return;
  const int a = left[i], b = right[i];
  const float4 ca = centers[a], cb = centers[b];
  const float m = ca.w + cb.w;
  float4 c;
  if (m > 0.f) {
    const float inv = 1.f / m;
    c = make_float4((ca.w * ca.x + cb.w * cb.x) * inv, (ca.w * ca.y + cb.w * cb.y) * inv,
                    (ca.w * ca.z + cb.w * cb.z) * inv, m);
  } else {
    c = make_float4(0.5f * (ca.x + cb.x), 0.5f * (ca.y + cb.y), 0.5f * (ca.z + cb.z), 0.f);
  }
  centers[i] = c;
  float acc[C];
  {
    float v[C];
    const float* src = mult + (size_t)a * CS;
#pragma unroll
    for (int k = 0; k < C; ++k) v[k] = src[k];
    m2m_pair<P>(v, ca.x - c.x, ca.y - c.y, ca.z - c.z);
#pragma unroll
    for (int k = 0; k < C; ++k) acc[k] = v[k];
  }
  {
    float v[C];
    const float* src = mult + (size_t)b * CS;
#pragma unroll
    for (int k = 0; k < C; ++k) v[k] = src[k];
    m2m_pair<P>(v, cb.x - c.x, cb.y - c.y, cb.z - c.z);
#pragma unroll
    for (int k = 0; k < C; ++k) acc[k] += v[k];
  }
  float* dst = mult + (size_t)i * CS;
#pragma unroll
  for (int k = 0; k < C; ++k) dst[k] = acc[k];
#pragma unroll
  for (int k = C; k < CS; ++k) dst[k] = 0.f;
}

// ---------------------------------------------------------------------------
// M2L: thread per target.
// ---------------------------------------------------------------------------
constexpr int kM2LThreads = 128;

template <int P>
__global__ void __launch_bounds__(kM2LThreads) k_m2l_fp32(int num_targets, const int* __restrict__ targets,
                                                          const float* __restrict__ mult, const float4* __restrict__ centers,
                                                          const int64_t* __restrict__ far_off, const int* __restrict__ far_src,
                                                          float* __restrict__ locals) {
  constexpr int C = csize(P), CS = cstride(P);
  extern __shared__ float sacc[];  // [C][kM2LThreads]
  const int t = blockIdx.x * kM2LThreads + threadIdx.x;
  if (t >= num_targets) return;
  const int tgt = targets[t];
#pragma unroll
  for (int k = 0; k < C; ++k) sacc[k * kM2LThreads + threadIdx.x] = 0.f;
  const float4 ct = centers[tgt];
  const int64_t e0 = far_off[tgt], e1 = far_off[tgt + 1];
  for (int64_t e = e0; e < e1; ++e) {
    const int s = far_src[e];
    const float4 cs = centers[s];
    float v[C], w[C];
    const float4* src = reinterpret_cast<const float4*>(mult + (size_t)s * CS);
#pragma unroll
    for (int k = 0; k < CS / 4; ++k) {
      const float4 q = __ldg(src + k);
      if (4 * k + 0 < C) v[4 * k + 0] = q.x;
      if (4 * k + 1 < C) v[4 * k + 1] = q.y;
      if (4 * k + 2 < C) v[4 * k + 2] = q.z;
      if (4 * k + 3 < C) v[4 * k + 3] = q.w;
    }
    m2l_pair<P>(v, w, ct.x - cs.x, ct.y - cs.y, ct.z - cs.z);
#pragma unroll
    for (int k = 0; k < C; ++k) sacc[k * kM2LThreads + threadIdx.x] += w[k];
  }
  float* dst = locals + (size_t)tgt * CS;
#pragma unroll
  for (int k = 0; k < C; ++k) dst[k] = sacc[k * kM2LThreads + threadIdx.x];
#pragma unroll
  for (int k = C; k < CS; ++k) dst[k] = 0.f;
}

// ---------------------------------------------------------------------------
// L2L, one level: thread per (parent, child).
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(128) k_l2l_level(int first, int last, const int* __restrict__ left,
                                                   const int* __restrict__ right, const float4* __restrict__ centers,
                                                   float* __restrict__ locals) {
  constexpr int C = csize(P), CS = cstride(P);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = first + (tid >> 1);
  if (i >= last) return;
  const int ch = (tid & 1) ? right[i] : left[i];
  const float4 cp = centers[i], cc = centers[ch];
  float v[C];
  const float* src = locals + (size_t)i * CS;
#pragma unroll
  for (int k = 0; k < C; ++k) v[k] = src[k];
  l2l_pair<P>(v, cp.x - cc.x, cp.y - cc.y, cp.z - cc.z);
  float* dst = locals + (size_t)ch * CS;
#pragma unroll
  for (int k = 0; k < C; ++k) dst[k] += v[k];
}

// ---------------------------------------------------------------------------
// Leaf evaluation: L2P + P2P, warp per target leaf.
// ---------------------------------------------------------------------------
struct SmemF {
  const float* f;
  __device__ __forceinline__ float operator()(int k) const { return f[k]; }
};

template <bool KAHAN>
struct Acc4 {
  float x = 0.f, y = 0.f, z = 0.f, w = 0.f;
  float cx = 0.f, cy = 0.f, cz = 0.f, cw = 0.f;
  __device__ __forceinline__ static void add(float& s, float& c, float v) {
    if (KAHAN) {
      const float y = v - c;
      const float t = s + y;
      c = (t - s) - y;
      s = t;
    } else {
      s += v;
    }
  }
  __device__ __forceinline__ void add(float ax, float ay, float az, float aw) {
    add(x, cx, ax);
    add(y, cy, ay);
    add(z, cz, az);
    add(w, cw, aw);
  }
};

template <bool KAHAN>
__device__ __forceinline__ void p2p_block(const float4* __restrict__ spos, int ns, int self_j, float4 ti, float eps2,
                                          Acc4<KAHAN>& a) {
  for (int j = 0; j < ns; ++j) {
    const float4 s = spos[j];
    const float dx = ti.x - s.x, dy = ti.y - s.y, dz = ti.z - s.z;
    const float d2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
    const float ir = rsqrtf(d2);
    const bool self = (j == self_j);
    const float mir = self ? 0.f : s.w * ir;
    const float w = self ? 0.f : mir * ir * ir;
    a.add(w * dx, w * dy, w * dz, mir);
  }
}

template <int P, bool KAHAN>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_leaf_eval(const float4* __restrict__ pos4, int num_internal,
                                                                   int leaf_first, int leaf_last,
                                                                   const int2* __restrict__ ranges,
                                                                   const float4* __restrict__ centers,
                                                                   const float* __restrict__ locals,
                                                                   const int64_t* __restrict__ near_off,
                                                                   const int* __restrict__ near_src, float G, float eps2,
                                                                   float4* __restrict__ out) {
  constexpr int C = csize(P), CS = cstride(P);
  __shared__ float sF[kWarpsPerBlock][CS];
  __shared__ float4 sP[kWarpsPerBlock][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int leaf = leaf_first + blockIdx.x * kWarpsPerBlock + warp;
  if (leaf >= leaf_last) return;
  const int node = num_internal + leaf;
  const int2 rg = ranges[node];
  const float4 c = centers[node];
  for (int k = lane; k < CS; k += 32) sF[warp][k] = locals[(size_t)node * CS + k];
  __syncwarp();
  const int64_t e0 = near_off[leaf], e1 = near_off[leaf + 1];
  for (int tb = rg.x; tb <= rg.y; tb += 32) {
    const int ti_idx = tb + lane;
    const bool active = ti_idx <= rg.y;
    const float4 ti = active ? pos4[ti_idx] : make_float4(0.f, 0.f, 0.f, 0.f);
    Acc4<KAHAN> a;
    // self leaf (all chunks), excluding the diagonal
    for (int sb = rg.x; sb <= rg.y; sb += 32) {
      const int ns = min(32, rg.y - sb + 1);
      __syncwarp();
      if (lane < ns) sP[warp][lane] = pos4[sb + lane];
      __syncwarp();
      p2p_block<KAHAN>(sP[warp], ns, ti_idx - sb, ti, eps2, a);
    }
    for (int64_t e = e0; e < e1; ++e) {
      const int2 sr = ranges[num_internal + near_src[e]];
      for (int sb = sr.x; sb <= sr.y; sb += 32) {
        const int ns = min(32, sr.y - sb + 1);
        __syncwarp();
        if (lane < ns) sP[warp][lane] = pos4[sb + lane];
        __syncwarp();
        p2p_block<KAHAN>(sP[warp], ns, -1, ti, eps2, a);
      }
    }
    // far field
    float U[C];
    solid_harmonics<P>(c.x - ti.x, c.y - ti.y, c.z - ti.z, U);
    float phi, g[3];
    l2p_eval<P>(SmemF{sF[warp]}, U, &phi, g);
    if (active) {
      out[ti_idx] = make_float4(-G * a.x - G * g[0], -G * a.y - G * g[1], -G * a.z - G * g[2],
                                -G * a.w - G * phi);
    }
  }
}

// ---------------------------------------------------------------------------
// Target subset: warp per target.
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(128) k_eval_targets(const float4* __restrict__ pos4, int num_internal,
                                                      const int2* __restrict__ ranges, const float4* __restrict__ centers,
                                                      const float* __restrict__ locals, const int64_t* __restrict__ near_off,
                                                      const int* __restrict__ near_src, const int* __restrict__ leaf_of,
                                                      int64_t num_targets, const int* __restrict__ tsorted, float G,
                                                      float eps2, float4* __restrict__ out) {
  constexpr int C = csize(P), CS = cstride(P);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t q = (int64_t)blockIdx.x * 4 + warp;
  if (q >= num_targets) return;
  const int i = tsorted[q];
  const int leaf = leaf_of[i];
  const int node = num_internal + leaf;
  const float4 ti = pos4[i];
  float ax = 0.f, ay = 0.f, az = 0.f, aw = 0.f;
  const int64_t e0 = near_off[leaf], e1 = near_off[leaf + 1];
  for (int64_t e = e0 - 1; e < e1; ++e) {
    const int2 sr = (e < e0) ? ranges[node] : ranges[num_internal + near_src[e]];
    for (int j = sr.x + lane; j <= sr.y; j += 32) {
      const float4 s = pos4[j];
      const float dx = ti.x - s.x, dy = ti.y - s.y, dz = ti.z - s.z;
      const float d2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
      const float ir = rsqrtf(d2);
      const bool self = (j == i);
      const float mir = self ? 0.f : s.w * ir;
      const float w = self ? 0.f : mir * ir * ir;
      ax = fmaf(w, dx, ax);
      ay = fmaf(w, dy, ay);
      az = fmaf(w, dz, az);
      aw += mir;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ax += __shfl_xor_sync(0xffffffffu, ax, o);
    ay += __shfl_xor_sync(0xffffffffu, ay, o);
    az += __shfl_xor_sync(0xffffffffu, az, o);
    aw += __shfl_xor_sync(0xffffffffu, aw, o);
  }
  if (lane == 0) {
    const float4 c = centers[node];
    float U[C];
    solid_harmonics<P>(c.x - ti.x, c.y - ti.y, c.z - ti.z, U);
    const float* F = locals + (size_t)node * CS;
    float phi, g[3];
    l2p_eval<P>(SmemF{F}, U, &phi, g);
    out[q] = make_float4(-G * ax - G * g[0], -G * ay - G * g[1], -G * az - G * g[2], -G * aw - G * phi);
  }
}

static inline unsigned blocks_for(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }

template <int P>
struct RunP2M {
  static int run(const float* pos4, int num_nodes, int num_internal, const int* ranges, float* centers, float* mult,
                 cudaStream_t st) {
    const int L = num_nodes - num_internal;
    if (L <= 0) return JB_OK;
    const size_t sm = sizeof(float) * kWarpsPerBlock * 32 * (csize(P) + 1);
    cudaFuncSetAttribute(k_p2m<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_p2m<P><<<blocks_for(L, kWarpsPerBlock), 32 * kWarpsPerBlock, sm, st>>>(
        reinterpret_cast<const float4*>(pos4), num_nodes, num_internal, reinterpret_cast<const int2*>(ranges),
        reinterpret_cast<float4*>(centers), mult);
    return launch_status();
  }
};

template <int P>
struct RunM2M {
  static int run(int first, int last, const int* left, const int* right, float* centers, float* mult, cudaStream_t st) {
    if (last <= first) return JB_OK;
    k_m2m_level<P><<<blocks_for(last - first, 128), 128, 0, st>>>(first, last, left, right,
                                                                   reinterpret_cast<float4*>(centers), mult);
    return launch_status();
  }
};

template <int P>
struct RunM2L {
  static int run(int num_targets, const int* targets, const float* mult, const float* centers, const int64_t* far_off,
                 const int* far_src, float* locals, cudaStream_t st) {
    if (num_targets <= 0) return JB_OK;
    const size_t sm = sizeof(float) * csize(P) * kM2LThreads;
    cudaFuncSetAttribute(k_m2l_fp32<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_m2l_fp32<P><<<blocks_for(num_targets, kM2LThreads), kM2LThreads, sm, st>>>(
        num_targets, targets, mult, reinterpret_cast<const float4*>(centers), far_off, far_src, locals);
    return launch_status();
  }
};

template <int P>
struct RunL2L {
  static int run(int first, int last, const int* left, const int* right, const float* centers, float* locals,
                 cudaStream_t st) {
    if (last <= first) return JB_OK;
    k_l2l_level<P><<<blocks_for(2 * (int64_t)(last - first), 128), 128, 0, st>>>(
        first, last, left, right, reinterpret_cast<const float4*>(centers), locals);
    return launch_status();
  }
};

template <int P>
struct RunLeafEval {
  static int run(int mode, const float* pos4, int num_internal, int leaf_first, int leaf_last, const int* ranges,
                 const float* centers, const float* locals, const int64_t* near_off, const int* near_src, float G,
                 float eps2, float* out, cudaStream_t st) {
    if (leaf_last <= leaf_first) return JB_OK;
    const unsigned nb = blocks_for(leaf_last - leaf_first, kWarpsPerBlock);
    if (mode == JB_P2P_KAHAN) {
      k_leaf_eval<P, true><<<nb, 32 * kWarpsPerBlock, 0, st>>>(
          reinterpret_cast<const float4*>(pos4), num_internal, leaf_first, leaf_last, reinterpret_cast<const int2*>(ranges),
          reinterpret_cast<const float4*>(centers), locals, near_off, near_src, G, eps2, reinterpret_cast<float4*>(out));
    } else {
      k_leaf_eval<P, false><<<nb, 32 * kWarpsPerBlock, 0, st>>>(
          reinterpret_cast<const float4*>(pos4), num_internal, leaf_first, leaf_last, reinterpret_cast<const int2*>(ranges),
          reinterpret_cast<const float4*>(centers), locals, near_off, near_src, G, eps2, reinterpret_cast<float4*>(out));
    }
    return launch_status();
  }
};

template <int P>
struct RunTargets {
  static int run(const float* pos4, int num_internal, const int* ranges, const float* centers, const float* locals,
                 const int64_t* near_off, const int* near_src, const int* leaf_of, int64_t nt, const int* ts, float G,
                 float eps2, float* out, cudaStream_t st) {
    if (nt <= 0) return JB_OK;
    k_eval_targets<P><<<blocks_for(nt, 4), 128, 0, st>>>(
        reinterpret_cast<const float4*>(pos4), num_internal, reinterpret_cast<const int2*>(ranges),
        reinterpret_cast<const float4*>(centers), locals, near_off, near_src, leaf_of, nt, ts, G, eps2,
        reinterpret_cast<float4*>(out));
    return launch_status();
  }
};

}  // namespace jb


#define JB_DECLARE_ORDER(PP)                 \
  extern template struct jb::RunP2M<PP>;      \
  extern template struct jb::RunM2M<PP>;      \
  extern template struct jb::RunM2L<PP>;      \
  extern template struct jb::RunL2L<PP>;      \
  extern template struct jb::RunLeafEval<PP>; \
  extern template struct jb::RunTargets<PP>;
