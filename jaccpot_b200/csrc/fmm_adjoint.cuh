#pragma once
// Adjoint (vector-Jacobian product) of the evaluation pass at fixed topology:
// given w (one 3-vector per sorted particle), the gradient of
// L = sum_i w_i . a_i with respect to the sorted positions and masses, with the
// COM expansion centres differentiated too.  This is what the reference's
// differentiable_accelerations gives jax.grad (runtime/fmm_evaluate.py:542-731,
// :1175-1250; analytic near-field VJP nearfield/grad.py:726-869; analytic L2P
// VJP operators/real_p2m_l2p.py:402-491), written as hand-made reverse kernels.
//
// Reverse order (each stage one launch or one launch per level):
//   near      P2P adjoint, gathered over the (symmetric) neighbour lists
//   leaf far  L2P adjoint: Lbar_leaf = -G sum_i (w_i . grad) U, and the
//             Hessian-vector product for the particle, centre terms
//   L2L       deepest parents first: Lbar_p += L2L(d)^T Lbar_c = M2M(d) Lbar_c
//   M2L       Mbar_u += sum_v M2L(c_v - c_u) Lbar_v (M2L is symmetric), and
//             the displacement derivative -D(order p+1 M2L) per pair
//   M2M       root first: Mbar_c += M2M(d)^T Mbar_p = L2L(d) Mbar_p, then the
//             COM chain c_p = (mu_a c_a + mu_b c_b) / mu_p pushed to children
//   P2M       per particle: mass and position terms, leaf COM
// Transposes come for free: the real M2L matrix is symmetric and
// M2M(d)^T = L2L(d) for the same displacement (both checked in the tests).
// Every output element has one writer per launch (no atomics).
//
// cbar4[node] = (dL/dc_x, dL/dc_y, dL/dc_z, dL/dmu) accumulates over stages;
// xm4[i] = (dL/dx, dL/dy, dL/dz, dL/dm) per sorted particle.
#include "fmm_kernels.cuh"

namespace jb {

struct ArrF {
  const float* f;
  __device__ __forceinline__ float operator()(int k) const { return f[k]; }
};

// ---------------------------------------------------------------------------
// Leaf far field (L2P adjoint): warp per leaf, lane = particle.
//   Lbar_leaf  = -G sum_i sum_a w_ia D_a^T U(delta_i)
//   deltabar_i = -G grad_delta ( (sum_a w_ia D_a F) . U(delta_i) )
//   xbar_i -= deltabar_i ;  cbar_leaf += sum_i deltabar_i        (delta = c - x)
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_adj_leaf_far(
    const float4* __restrict__ pos4, const float4* __restrict__ w4, int num_nodes, int num_internal,
    const int2* __restrict__ ranges, const float4* __restrict__ centers, const float* __restrict__ locals, float G,
    float4* __restrict__ xm4, float* __restrict__ lbar, float4* __restrict__ cbar4) {
  constexpr int C = csize(P), CS = cstride(P), CP = C + 1;
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* red = smem + warp * 32 * CP;
  float* sF = smem + kWarpsPerBlock * 32 * CP + warp * CS;
  const int node = num_internal + blockIdx.x * kWarpsPerBlock + warp;
  if (node >= num_nodes) return;
  const int2 rg = ranges[node];
  const float4 c = centers[node];
  for (int k = lane; k < CS; k += 32) sF[k] = locals[(size_t)node * CS + k];
  float* myred = red + lane * CP;
#pragma unroll
  for (int k = 0; k < C; ++k) myred[k] = 0.f;
  __syncwarp();
  float cb0 = 0.f, cb1 = 0.f, cb2 = 0.f;
  for (int i = rg.x + lane; i <= rg.y; i += 32) {
    const float4 q = pos4[i];
    const float4 wv = w4[i];
    float U[C];
    solid_harmonics<P>(c.x - q.x, c.y - q.y, c.z - q.z, U);
    float Gw[C];
#pragma unroll
    for (int k = 0; k < C; ++k) Gw[k] = 0.f;
    for_ladder<P>([&](int a, int row, int col, float val) {
      const float wa = (a == 0) ? wv.x : ((a == 1) ? wv.y : wv.z);
      myred[col] += (-G * wa * val) * U[row];
      Gw[row] += (wa * val) * sF[col];
    });
    float phi, g[3];
    l2p_eval<P>(ArrF{Gw}, U, &phi, g);
    const float dbx = -G * g[0], dby = -G * g[1], dbz = -G * g[2];
    float4 x = xm4[i];
    x.x -= dbx;
    x.y -= dby;
    x.z -= dbz;
    xm4[i] = x;
    cb0 += dbx;
    cb1 += dby;
    cb2 += dbz;
  }
  __syncwarp();
  float* out = lbar + (size_t)node * CS;
  for (int k = lane; k < CS; k += 32) {
    float s = 0.f;
    if (k < C) {
#pragma unroll 8
      for (int j = 0; j < 32; ++j) s += red[j * CP + k];
    }
    out[k] = s;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cb0 += __shfl_xor_sync(0xffffffffu, cb0, o);
    cb1 += __shfl_xor_sync(0xffffffffu, cb1, o);
    cb2 += __shfl_xor_sync(0xffffffffu, cb2, o);
  }
  if (lane == 0) {
    float4 cb = cbar4[node];
    cb.x += cb0;
    cb.y += cb1;
    cb.z += cb2;
    cbar4[node] = cb;
  }
}

// ---------------------------------------------------------------------------
// L2L adjoint, one level (parents in [first, last)), thread per parent:
//   X = L2L(d)^T Lbar_c = M2M(d) Lbar_c,  d = c_p - c_c
//   Lbar_p = X_left + X_right ;  g = X . D F_p ;  cbar_p += g, cbar_c -= g
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(128) k_adj_l2l_level(int first, int last, const int* __restrict__ left,
                                                       const int* __restrict__ right,
                                                       const float4* __restrict__ centers,
                                                       const float* __restrict__ locals, float* __restrict__ lbar,
                                                       float4* __restrict__ cbar4) {
  constexpr int C = csize(P), CS = cstride(P);
  const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= last) return;
  const float4 cp = centers[i];
  const float* Fp = locals + (size_t)i * CS;
  float* Lp = lbar + (size_t)i * CS;
  float4 cbp = cbar4[i];
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const int ch = side ? right[i] : left[i];
    const float4 cc = centers[ch];
    float X[C];
    const float* src = lbar + (size_t)ch * CS;
#pragma unroll
    for (int k = 0; k < C; ++k) X[k] = src[k];
    m2m_pair<P>(X, cp.x - cc.x, cp.y - cc.y, cp.z - cc.z);
    if (side == 0) {
#pragma unroll
      for (int k = 0; k < C; ++k) Lp[k] = X[k];
#pragma unroll
      for (int k = C; k < CS; ++k) Lp[k] = 0.f;
    } else {
#pragma unroll
      for (int k = 0; k < C; ++k) Lp[k] += X[k];
    }
    float g[3];
    ladder_dot3<P>(ArrF{X}, ArrF{Fp}, g);
    cbp.x += g[0];
    cbp.y += g[1];
    cbp.z += g[2];
    float4 cbc = cbar4[ch];
    cbc.x -= g[0];
    cbc.y -= g[1];
    cbc.z -= g[2];
    cbar4[ch] = cbc;
  }
  cbar4[i] = cbp;
}

// ---------------------------------------------------------------------------
// M2L displacement derivative, thread per far pair e = (t <- s):
//   g_e = Lbar_t . d/dd [M2L_p(d) M_s] = -Lbar_t . D (M2L_{p+1}(d) M_s),  d = c_t - c_s
// (the order p+1 triangular M2L carries exactly the degree n+1 terms that
// the derivative of the truncated degree-n coefficient needs).
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(128) k_adj_m2l_pairs(int64_t num_pairs, const int* __restrict__ pair_tgt,
                                                       const int* __restrict__ far_src,
                                                       const float* __restrict__ mult,
                                                       const float* __restrict__ lbar,
                                                       const float4* __restrict__ centers, float4* __restrict__ g4) {
  constexpr int C = csize(P), CS = cstride(P), C1 = csize(P + 1);
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= num_pairs) return;
  const int t = pair_tgt[e], s = far_src[e];
  const float4 ct = centers[t], cs = centers[s];
  float v[C1];
  const float* Ms = mult + (size_t)s * CS;
#pragma unroll
  for (int k = 0; k < C1; ++k) v[k] = (k < C) ? Ms[k] : 0.f;
  m2l_kfold<P + 1>(v, ct.x - cs.x, ct.y - cs.y, ct.z - cs.z);
  float g[3];
  ladder_dot3<P + 1>(ArrF{lbar + (size_t)t * CS}, ArrF{v}, g);
  g4[e] = make_float4(-g[0], -g[1], -g[2], 0.f);
}

// ---------------------------------------------------------------------------
// M2M adjoint + COM chain, one level (parents in [first, last)), root first:
//   Mbar_c += M2M(d)^T Mbar_p = L2L(d) Mbar_p,  d = c_c - c_p
//   g = (M2M(d) M_c) . D Mbar_p ; cbar_c += g, cbar_p -= g
//   then cbar_c += (mu_c / mu_p) cbar_p, mubar_c = mubar_p + (c_c - c_p).cbar_p / mu_p
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(128) k_adj_m2m_level(int first, int last, const int* __restrict__ left,
                                                       const int* __restrict__ right,
                                                       const float4* __restrict__ centers,
                                                       const float* __restrict__ mult, float* __restrict__ mbar,
                                                       float4* __restrict__ cbar4) {
  constexpr int C = csize(P), CS = cstride(P);
  const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= last) return;
  const float4 cp = centers[i];
  const float* Mbp = mbar + (size_t)i * CS;
  float4 cbp = cbar4[i];
  int chs[2] = {left[i], right[i]};
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const int ch = chs[side];
    const float4 cc = centers[ch];
    float Y[C];
#pragma unroll
    for (int k = 0; k < C; ++k) Y[k] = Mbp[k];
    l2l_pair<P>(Y, cc.x - cp.x, cc.y - cp.y, cc.z - cp.z);
    float* Mbc = mbar + (size_t)ch * CS;
#pragma unroll
    for (int k = 0; k < C; ++k) Mbc[k] += Y[k];
    const float* Mc = mult + (size_t)ch * CS;
#pragma unroll
    for (int k = 0; k < C; ++k) Y[k] = Mc[k];
    m2m_pair<P>(Y, cc.x - cp.x, cc.y - cp.y, cc.z - cp.z);
    float g[3];
    ladder_dot3<P>(ArrF{Y}, ArrF{Mbp}, g);
    float4 cbc = cbar4[ch];
    cbc.x += g[0];
    cbc.y += g[1];
    cbc.z += g[2];
    cbar4[ch] = cbc;
    cbp.x -= g[0];
    cbp.y -= g[1];
    cbp.z -= g[2];
  }
  cbar4[i] = cbp;
  const float inv = cp.w > 0.f ? 1.f / cp.w : 0.f;
#pragma unroll
  for (int side = 0; side < 2; ++side) {
    const int ch = chs[side];
    const float4 cc = centers[ch];
    const float f = cc.w * inv;
    float4 cbc = cbar4[ch];
    cbc.x += f * cbp.x;
    cbc.y += f * cbp.y;
    cbc.z += f * cbp.z;
    cbc.w = cbp.w + ((cc.x - cp.x) * cbp.x + (cc.y - cp.y) * cbp.y + (cc.z - cp.z) * cbp.z) * inv;
    cbar4[ch] = cbc;
  }
}

// ---------------------------------------------------------------------------
// P2M + leaf COM adjoint, warp per leaf, lane = particle, y = x - c:
//   gM = grad_y (Mbar . U(y)) ; cbar_tot = cbar_leaf - sum_j m_j gM_j
//   mbar_j += Mbar . U(y) + mubar + y . cbar_tot / mu
//   xbar_j += m_j gM + (m_j / mu) cbar_tot
// ---------------------------------------------------------------------------
template <int P>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_adj_p2m(const float4* __restrict__ pos4, int num_nodes,
                                                                  int num_internal, const int2* __restrict__ ranges,
                                                                  const float4* __restrict__ centers,
                                                                  const float* __restrict__ mbar,
                                                                  const float4* __restrict__ cbar4,
                                                                  float4* __restrict__ xm4) {
  constexpr int C = csize(P), CS = cstride(P);
  __shared__ float sM[kWarpsPerBlock][CS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int node = num_internal + blockIdx.x * kWarpsPerBlock + warp;
  if (node >= num_nodes) return;
  const int2 rg = ranges[node];
  const float4 c = centers[node];
  const float4 cb = cbar4[node];
  for (int k = lane; k < CS; k += 32) sM[warp][k] = mbar[(size_t)node * CS + k];
  __syncwarp();
  // pass 1: centre term
  float s0 = 0.f, s1 = 0.f, s2 = 0.f;
  for (int i = rg.x + lane; i <= rg.y; i += 32) {
    const float4 q = pos4[i];
    float U[C];
    solid_harmonics<P>(q.x - c.x, q.y - c.y, q.z - c.z, U);
    float phi, g[3];
    l2p_eval<P>(SmemF{sM[warp]}, U, &phi, g);
    s0 = fmaf(q.w, g[0], s0);
    s1 = fmaf(q.w, g[1], s1);
    s2 = fmaf(q.w, g[2], s2);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  const float tx = cb.x - s0, ty = cb.y - s1, tz = cb.z - s2;
  const float inv = c.w > 0.f ? 1.f / c.w : 0.f;
  // pass 2: particle terms
  for (int i = rg.x + lane; i <= rg.y; i += 32) {
    const float4 q = pos4[i];
    const float yx = q.x - c.x, yy = q.y - c.y, yz = q.z - c.z;
    float U[C];
    solid_harmonics<P>(yx, yy, yz, U);
    float phi, g[3];
    l2p_eval<P>(SmemF{sM[warp]}, U, &phi, g);
    float4 x = xm4[i];
    x.x += q.w * g[0] + q.w * inv * tx;
    x.y += q.w * g[1] + q.w * inv * ty;
    x.z += q.w * g[2] + q.w * inv * tz;
    x.w += phi + cb.w + (yx * tx + yy * ty + yz * tz) * inv;
    xm4[i] = x;
  }
}

// ---------------------------------------------------------------------------
template <int P>
struct RunAdj {
  static int leaf_far(const float* pos4, const float* w4, int num_nodes, int num_internal, const int* ranges,
                      const float* centers, const float* locals, float G, float* xm4, float* lbar, float* cbar4,
                      cudaStream_t st) {
    const int L = num_nodes - num_internal;
    if (L <= 0) return JB_OK;
    const size_t sm = sizeof(float) * kWarpsPerBlock * (32 * (csize(P) + 1) + cstride(P));
    cudaFuncSetAttribute(k_adj_leaf_far<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_adj_leaf_far<P><<<blocks_for(L, kWarpsPerBlock), 32 * kWarpsPerBlock, sm, st>>>(
        reinterpret_cast<const float4*>(pos4), reinterpret_cast<const float4*>(w4), num_nodes, num_internal,
        reinterpret_cast<const int2*>(ranges), reinterpret_cast<const float4*>(centers), locals, G,
        reinterpret_cast<float4*>(xm4), lbar, reinterpret_cast<float4*>(cbar4));
    return launch_status();
  }
  static int l2l_level(int first, int last, const int* left, const int* right, const float* centers,
                       const float* locals, float* lbar, float* cbar4, cudaStream_t st) {
    if (last <= first) return JB_OK;
    k_adj_l2l_level<P><<<blocks_for(last - first, 128), 128, 0, st>>>(
        first, last, left, right, reinterpret_cast<const float4*>(centers), locals, lbar,
        reinterpret_cast<float4*>(cbar4));
    return launch_status();
  }
  static int m2l_pairs(int64_t num_pairs, const int* pair_tgt, const int* far_src, const float* mult,
                       const float* lbar, const float* centers, float* g4, cudaStream_t st) {
    if (num_pairs <= 0) return JB_OK;
    k_adj_m2l_pairs<P><<<blocks_for(num_pairs, 128), 128, 0, st>>>(
        num_pairs, pair_tgt, far_src, mult, lbar, reinterpret_cast<const float4*>(centers),
        reinterpret_cast<float4*>(g4));
    return launch_status();
  }
  static int m2m_level(int first, int last, const int* left, const int* right, const float* centers,
                       const float* mult, float* mbar, float* cbar4, cudaStream_t st) {
    if (last <= first) return JB_OK;
    k_adj_m2m_level<P><<<blocks_for(last - first, 128), 128, 0, st>>>(
        first, last, left, right, reinterpret_cast<const float4*>(centers), mult, mbar,
        reinterpret_cast<float4*>(cbar4));
    return launch_status();
  }
  static int p2m(const float* pos4, int num_nodes, int num_internal, const int* ranges, const float* centers,
                 const float* mbar, const float* cbar4, float* xm4, cudaStream_t st) {
    const int L = num_nodes - num_internal;
    if (L <= 0) return JB_OK;
    k_adj_p2m<P><<<blocks_for(L, kWarpsPerBlock), 32 * kWarpsPerBlock, 0, st>>>(
        reinterpret_cast<const float4*>(pos4), num_nodes, num_internal, reinterpret_cast<const int2*>(ranges),
        reinterpret_cast<const float4*>(centers), mbar, reinterpret_cast<const float4*>(cbar4),
        reinterpret_cast<float4*>(xm4));
    return launch_status();
  }
};

}  // namespace jb
