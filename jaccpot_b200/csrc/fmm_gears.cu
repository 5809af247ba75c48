// Learned gear (per-interaction expansion order) selector: features, error
// labels, and a 12 -> 64 -> 64 -> 4 GELU MLP with hand-written training
// (forward + backward + Adam) and a fused per-pair inference kernel.
//
// The reference chooses each far pair's order from an analytic error proxy
// (Dehnen 2014 eq. 15, runtime/_adaptive_policy.py:249-372) and runs the M2L
// bucketed by gear (runtime/fmm_prepare.py:2400-2480).  Here the proxy is
// replaced by a network trained on the errors the FMM itself makes: for
// sampled far pairs, the force error of each gear's M2L against an order-10
// M2L of the same multipole, at the near and far side of the target's
// bounding sphere, relative to the smallest particle force in the target
// node.  Inference picks the lowest gear whose predicted cumulative
// probability of being within budget reaches 1 - eps; with a thin margin it
// falls back to the highest gear.
//
// Parameter layout (floats): W1[64][12] b1[64] W2[64][64] b2[64] W3[4][64] b3[4].
#include <cuda_bf16.h>

#include "fmm_adjoint.cuh"

namespace jb {
namespace gears {

constexpr int kIn = 12, kH = 64, kOut = 4;
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kOut * kH, kParams = oB3 + kOut;
static_assert(kParams == 5252, "parameter layout");
constexpr int kPowDeg = 8;  // per-degree power features for n = 1..8

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float x) {
  return 0.5f * (1.f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

__host__ __device__ constexpr double factd2(int n) { return n <= 1 ? 1.0 : (double)n * factd2(n - 1); }

// Per node: log10 of Dehnen's per-degree power P_n (real basis, m != 0
// weights doubled; _adaptive_policy.py:161-214) over mu r^n, n = 1..8.
template <int P>
__global__ void k_node_powers(int num_nodes, const float* __restrict__ mult, const float4* __restrict__ centers,
                              const float* __restrict__ radii, float* __restrict__ feat) {
  constexpr int CS = cstride(P);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= num_nodes) return;
  const float* M = mult + (size_t)i * CS;
  const float mu = fmaxf(centers[i].w, 1e-30f);
  const float r = fmaxf(radii[i], 1e-30f);
  float rn = 1.f;
#pragma unroll
  for (int n = 1; n <= kPowDeg; ++n) {
    rn *= r;
    float out = -30.f;
    if (n <= P) {
      float s = 0.f;
#pragma unroll
      for (int m = -n; m <= n; ++m) {
        const int am = m < 0 ? -m : m;
        const float w = (float)(factd2(n - am) * factd2(n + am) * (m != 0 ? 2.0 : 1.0));
        const float c = M[shi(n, m)];
        s = fmaf(w * c, c, s);
      }
      out = log10f(fmaxf(sqrtf(s), 1e-37f) / fmaxf(mu * rn, 1e-37f));
      out = fmaxf(out, -30.f);
    }
    feat[(size_t)i * kPowDeg + (n - 1)] = out;
  }
}

// Smallest particle force magnitude per leaf, then per internal node (level by level).
__global__ void k_leaf_force_min(int num_nodes, int num_internal, const int2* __restrict__ ranges,
                                 const float4* __restrict__ acc4, float* __restrict__ scale) {
  const int node = num_internal + blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= num_nodes) return;
  const int2 rg = ranges[node];
  float a = 3.0e38f;
  for (int i = rg.x; i <= rg.y; ++i) {
    const float4 v = acc4[i];
    a = fminf(a, sqrtf(v.x * v.x + v.y * v.y + v.z * v.z));
  }
  scale[node] = a;
}

__global__ void k_force_min_level(int first, int last, const int* __restrict__ left, const int* __restrict__ right,
                                  float* __restrict__ scale) {
  const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= last) return;
  scale[i] = fminf(scale[left[i]], scale[right[i]]);
}

// Dehnen's per-degree power P_l = sqrt(sum_m w_lm M_l^m^2), w_lm = (l-|m|)!
// (l+|m|)! doubled for m != 0 in the real no-sqrt2 packing
// (_adaptive_policy.py:161-214 dehnen_multipole_power_by_degree), in FP64 for
// l = 0..p (a point mass m at distance r has P_l = m r^l).
__global__ void k_dehnen_power(int p, int num_nodes, const float* __restrict__ mult, int rs,
                               double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= num_nodes) return;
  const float* M = mult + (size_t)i * rs;
  for (int l = 0; l <= p; ++l) {
    double acc = 0.0;
    for (int m = -l; m <= l; ++m) {
      const int am = m < 0 ? -m : m;
      const double w = factd2(l - am) * factd2(l + am) * (m != 0 ? 2.0 : 1.0);
      const double c = (double)M[l * l + l + m];
      acc += w * c * c;
    }
    out[(size_t)i * (p + 1) + l] = sqrt(acc);
  }
}

// The 12 features of far pair (t <- s).
__device__ __forceinline__ void pair_features(int t, int s, const float4* __restrict__ centers,
                                              const float* __restrict__ radii, const float* __restrict__ node_feat,
                                              const float* __restrict__ scale, float G, float* f) {
  const float4 ct = centers[t], cs = centers[s];
  const float dx = ct.x - cs.x, dy = ct.y - cs.y, dz = ct.z - cs.z;
  const float d = fmaxf(sqrtf(dx * dx + dy * dy + dz * dz), 1e-30f);
  const float rt = radii[t], rs = radii[s];
  f[0] = (rs + rt) / d;                          // opening ratio
  f[1] = rt / fmaxf(rs + rt, 1e-30f);            // share of the target in it
#pragma unroll
  for (int n = 0; n < kPowDeg; ++n) f[2 + n] = node_feat[(size_t)s * kPowDeg + n];  // source shape
  f[10] = log10f(fmaxf(ct.w, 1e-30f) / fmaxf(cs.w, 1e-30f));                      // target-cell mass
  f[11] = log10f(fmaxf(scale[t], 1e-30f) * d * d / fmaxf(G * cs.w, 1e-30f));     // target force scale
}

__global__ void k_pair_features(int64_t n, const int64_t* __restrict__ pair_ids, const int* __restrict__ pair_tgt,
                                const int* __restrict__ far_src, const float4* __restrict__ centers,
                                const float* __restrict__ radii, const float* __restrict__ node_feat,
                                const float* __restrict__ scale, float G, float* __restrict__ out) {
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int64_t e = pair_ids ? pair_ids[q] : q;
  float f[kIn];
  pair_features(pair_tgt[e], far_src[e], centers, radii, node_feat, scale, G, f);
#pragma unroll
  for (int k = 0; k < kIn; ++k) out[q * kIn + k] = f[k];
}

// grad_delta of sum L U(delta) at delta = +-h (near / far side of the target sphere).
template <int P>
__device__ __forceinline__ void two_side_grads(const float* L, float hx, float hy, float hz, float* g) {
  float U[csize(P)];
  float phi;
  solid_harmonics<P>(hx, hy, hz, U);
  l2p_eval<P>(ArrF{L}, U, &phi, g);
  solid_harmonics<P>(-hx, -hy, -hz, U);
  l2p_eval<P>(ArrF{L}, U, &phi, g + 3);
}

template <int PG>
__device__ __forceinline__ float gear_error(const float* Mrow, float dx, float dy, float dz, float hx, float hy,
                                            float hz, const float* gref) {
  float v[csize(PG)];
#pragma unroll
  for (int k = 0; k < csize(PG); ++k) v[k] = Mrow[k];
  m2l_kfold<PG>(v, dx, dy, dz);
  float g[6];
  two_side_grads<PG>(v, hx, hy, hz, g);
  const float e0 = sqrtf((g[0] - gref[0]) * (g[0] - gref[0]) + (g[1] - gref[1]) * (g[1] - gref[1]) +
                         (g[2] - gref[2]) * (g[2] - gref[2]));
  const float e1 = sqrtf((g[3] - gref[3]) * (g[3] - gref[3]) + (g[4] - gref[4]) * (g[4] - gref[4]) +
                         (g[5] - gref[5]) * (g[5] - gref[5]));
  return fmaxf(e0, e1);
}

// log10(force error / smallest target force) of each gear, against the
// order-10 M2L; mult10 holds order-10 multipoles (stride cstride(10)).
__global__ void __launch_bounds__(64) k_gear_errors(int64_t n, const int64_t* __restrict__ pair_ids,
                                                    const int* __restrict__ pair_tgt,
                                                    const int* __restrict__ far_src,
                                                    const float* __restrict__ mult10,
                                                    const float4* __restrict__ centers,
                                                    const float* __restrict__ radii,
                                                    const float* __restrict__ scale, float G,
                                                    float* __restrict__ out) {
  constexpr int PR = 10, CR = csize(PR), CSR = cstride(PR);
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int64_t e = pair_ids[q];
  const int t = pair_tgt[e], s = far_src[e];
  const float4 ct = centers[t], cs = centers[s];
  const float dx = ct.x - cs.x, dy = ct.y - cs.y, dz = ct.z - cs.z;
  const float d = fmaxf(sqrtf(dx * dx + dy * dy + dz * dz), 1e-30f);
  const float rt = radii[t];
  // delta = c_t - y for y = c_t + rt * dhat (far side) and c_t - rt * dhat (near side)
  const float hx = -rt * dx / d, hy = -rt * dy / d, hz = -rt * dz / d;
  const float* Mrow = mult10 + (size_t)s * CSR;
  float gref[6];
  {
    float v[CR];
#pragma unroll
    for (int k = 0; k < CR; ++k) v[k] = Mrow[k];
    m2l_kfold<PR>(v, dx, dy, dz);
    two_side_grads<PR>(v, hx, hy, hz, gref);
  }
  const float inv = 1.f / fmaxf(scale[t], 1e-30f);
  const float ge[kOut] = {gear_error<2>(Mrow, dx, dy, dz, hx, hy, hz, gref) * G,
                          gear_error<4>(Mrow, dx, dy, dz, hx, hy, hz, gref) * G,
                          gear_error<6>(Mrow, dx, dy, dz, hx, hy, hz, gref) * G,
                          gear_error<8>(Mrow, dx, dy, dz, hx, hy, hz, gref) * G};
#pragma unroll
  for (int k = 0; k < kOut; ++k) out[q * kOut + k] = log10f(fmaxf(ge[k] * inv, 1e-30f));
}

// ---------------------------------------------------------------------------
// MLP.  Forward for one sample with parameters W (bf16-rounded floats) in
// shared memory; z1, z2 are the pre-activations.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mlp_forward(const float* __restrict__ W, const float* x, float* z1, float* z2,
                                            float* o) {
#pragma unroll 4
  for (int i = 0; i < kH; ++i) {
    float a = W[oB1 + i];
#pragma unroll
    for (int k = 0; k < kIn; ++k) a = fmaf(W[oW1 + i * kIn + k], x[k], a);
    z1[i] = a;
  }
  float h1[kH];
#pragma unroll
  for (int i = 0; i < kH; ++i) h1[i] = gelu(z1[i]);
#pragma unroll 2
  for (int i = 0; i < kH; ++i) {
    float a = W[oB2 + i];
#pragma unroll
    for (int k = 0; k < kH; ++k) a = fmaf(W[oW2 + i * kH + k], h1[k], a);
    z2[i] = a;
  }
#pragma unroll
  for (int j = 0; j < kOut; ++j) {
    float a = W[oB3 + j];
#pragma unroll
    for (int k = 0; k < kH; ++k) a = fmaf(W[oW3 + j * kH + k], gelu(z2[k]), a);
    o[j] = a;
  }
}

constexpr int kTrainThreads = 128;

// One training step's gradients over a chunk of the batch: block b takes
// samples [b*128, b*128+128) of this batch, writes its parameter-gradient sum
// to gpart[b][kParams] and its loss sum to lpart[b].  Softmax cross-entropy
// on the label (lowest gear within budget).
__global__ void __launch_bounds__(kTrainThreads) k_mlp_grad(int n, const float* __restrict__ X,
                                                            const int* __restrict__ labels,
                                                            const float* __restrict__ Wq,
                                                            float* __restrict__ gpart, float* __restrict__ lpart) {
  extern __shared__ float sm[];
  float* W = sm;                                   // kParams
  float* sX = W + kParams;                         // [kIn][T]
  float* sH1 = sX + kIn * kTrainThreads;           // [kH][T]
  float* sD1 = sH1 + kH * kTrainThreads;           // [kH][T]
  float* sH2 = sD1 + kH * kTrainThreads;           // [kH][T]
  float* sD2 = sH2 + kH * kTrainThreads;           // [kH][T]
  float* sD3 = sD2 + kH * kTrainThreads;           // [kOut][T]
  float* sL = sD3 + kOut * kTrainThreads;          // [T]
  const int tid = threadIdx.x;
  for (int k = tid; k < kParams; k += kTrainThreads) W[k] = Wq[k];
  __syncthreads();
  const int q = blockIdx.x * kTrainThreads + tid;
  const bool valid = q < n;
  float x[kIn];
#pragma unroll
  for (int k = 0; k < kIn; ++k) x[k] = valid ? X[(size_t)q * kIn + k] : 0.f;
  float z1[kH], z2[kH], o[kOut];
  mlp_forward(W, x, z1, z2, o);
  // softmax cross-entropy
  float mx = o[0];
#pragma unroll
  for (int j = 1; j < kOut; ++j) mx = fmaxf(mx, o[j]);
  float se = 0.f, pr[kOut];
#pragma unroll
  for (int j = 0; j < kOut; ++j) {
    pr[j] = expf(o[j] - mx);
    se += pr[j];
  }
  const int lab = valid ? labels[q] : 0;
  float loss = 0.f;
#pragma unroll
  for (int j = 0; j < kOut; ++j) {
    pr[j] /= se;
    const float d3 = valid ? (pr[j] - (j == lab ? 1.f : 0.f)) : 0.f;
    sD3[j * kTrainThreads + tid] = d3;
    if (j == lab) loss = valid ? -logf(fmaxf(pr[j], 1e-30f)) : 0.f;
  }
  sL[tid] = loss;
  // dz2 = (W3^T d3) * gelu'(z2)
#pragma unroll
  for (int k = 0; k < kH; ++k) {
    float a = 0.f;
#pragma unroll
    for (int j = 0; j < kOut; ++j) a = fmaf(W[oW3 + j * kH + k], sD3[j * kTrainThreads + tid], a);
    const float d2 = a * gelu_d(z2[k]);
    sD2[k * kTrainThreads + tid] = d2;
    sH2[k * kTrainThreads + tid] = gelu(z2[k]);
  }
  // dz1 = (W2^T dz2) * gelu'(z1)
  float dh1[kH];
#pragma unroll
  for (int k = 0; k < kH; ++k) dh1[k] = 0.f;
#pragma unroll 2
  for (int i = 0; i < kH; ++i) {
    const float d2 = sD2[i * kTrainThreads + tid];
#pragma unroll
    for (int k = 0; k < kH; ++k) dh1[k] = fmaf(W[oW2 + i * kH + k], d2, dh1[k]);
  }
#pragma unroll
  for (int k = 0; k < kH; ++k) {
    sD1[k * kTrainThreads + tid] = dh1[k] * gelu_d(z1[k]);
    sH1[k * kTrainThreads + tid] = gelu(z1[k]);
  }
#pragma unroll
  for (int k = 0; k < kIn; ++k) sX[k * kTrainThreads + tid] = x[k];
  __syncthreads();
  // parameter gradients: sums over the block's samples
  float* gout = gpart + (size_t)blockIdx.x * kParams;
  for (int pidx = tid; pidx < kParams; pidx += kTrainThreads) {
    const float* a;
    const float* b = nullptr;
    if (pidx < oB1) {
      a = sD1 + (pidx / kIn) * kTrainThreads;
      b = sX + (pidx % kIn) * kTrainThreads;
    } else if (pidx < oW2) {
      a = sD1 + (pidx - oB1) * kTrainThreads;
    } else if (pidx < oB2) {
      const int r = pidx - oW2;
      a = sD2 + (r / kH) * kTrainThreads;
      b = sH1 + (r % kH) * kTrainThreads;
    } else if (pidx < oW3) {
      a = sD2 + (pidx - oB2) * kTrainThreads;
    } else if (pidx < oB3) {
      const int r = pidx - oW3;
      a = sD3 + (r / kH) * kTrainThreads;
      b = sH2 + (r % kH) * kTrainThreads;
    } else {
      a = sD3 + (pidx - oB3) * kTrainThreads;
    }
    float s = 0.f;
    if (b) {
      for (int j = 0; j < kTrainThreads; ++j) s = fmaf(a[j], b[j], s);
    } else {
      for (int j = 0; j < kTrainThreads; ++j) s += a[j];
    }
    gout[pidx] = s;
  }
  if (tid == 0) {
    float s = 0.f;
    for (int j = 0; j < kTrainThreads; ++j) s += sL[j];
    lpart[blockIdx.x] = s;
  }
}

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Adam on the FP32 master weights; Wq is their BF16-rounded copy used by the
// forward passes (training and inference alike).
__global__ void k_mlp_adam(int nblocks, const float* __restrict__ gpart, float inv_batch, float lr, float beta1,
                           float beta2, float eps, int step, float* __restrict__ master, float* __restrict__ m1,
                           float* __restrict__ m2, float* __restrict__ Wq) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kParams) return;
  float g = 0.f;
  for (int b = 0; b < nblocks; ++b) g += gpart[(size_t)b * kParams + k];
  g *= inv_batch;
  const float a = beta1 * m1[k] + (1.f - beta1) * g;
  const float v = beta2 * m2[k] + (1.f - beta2) * g * g;
  m1[k] = a;
  m2[k] = v;
  const float ah = a / (1.f - powf(beta1, (float)step));
  const float vh = v / (1.f - powf(beta2, (float)step));
  const float w = master[k] - lr * ah / (sqrtf(vh) + eps);
  master[k] = w;
  Wq[k] = bf16_round(w);
}

// Fused inference: features -> normalisation -> MLP -> gear, thread per pair.
// gear = lowest g with P(label <= g) >= conf; if the winning class's
// probability is below min_top the margin is thin and the pair keeps the
// highest gear.
__global__ void __launch_bounds__(128) k_gear_select(int64_t n, const int* __restrict__ pair_tgt,
                                                     const int* __restrict__ far_src,
                                                     const float4* __restrict__ centers,
                                                     const float* __restrict__ radii,
                                                     const float* __restrict__ node_feat,
                                                     const float* __restrict__ scale, float G,
                                                     const float* __restrict__ Wq, const float* __restrict__ norm,
                                                     float conf, float min_top, int* __restrict__ gear_out) {
  __shared__ float W[kParams + 2 * kIn];
  for (int k = threadIdx.x; k < kParams; k += blockDim.x) W[k] = Wq[k];
  for (int k = threadIdx.x; k < 2 * kIn; k += blockDim.x) W[kParams + k] = norm[k];
  __syncthreads();
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  float x[kIn];
  pair_features(pair_tgt[e], far_src[e], centers, radii, node_feat, scale, G, x);
#pragma unroll
  for (int k = 0; k < kIn; ++k) x[k] = (x[k] - W[kParams + k]) * W[kParams + kIn + k];
  float z1[kH], z2[kH], o[kOut];
  mlp_forward(W, x, z1, z2, o);
  float mx = o[0];
#pragma unroll
  for (int j = 1; j < kOut; ++j) mx = fmaxf(mx, o[j]);
  float pr[kOut], se = 0.f;
#pragma unroll
  for (int j = 0; j < kOut; ++j) {
    pr[j] = expf(o[j] - mx);
    se += pr[j];
  }
  float cum = 0.f, top = 0.f;
  int g = kOut - 1;
  bool found = false;
#pragma unroll
  for (int j = 0; j < kOut; ++j) {
    const float pj = pr[j] / se;
    top = fmaxf(top, pj);
    cum += pj;
    if (!found && cum >= conf) {
      g = j;
      found = true;
    }
  }
  if (top < min_top) g = kOut - 1;
  gear_out[e] = g;
}

}  // namespace gears
}  // namespace jb

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace jb;
using namespace jb::gears;

static inline unsigned gblocks(int64_t n, int per) { return (unsigned)((n + per - 1) / per); }
#define GST(s) reinterpret_cast<cudaStream_t>(s)

extern "C" {

JB_API int jb_gear_param_count(void) { return kParams; }

JB_API int jb_gear_node_features(int p, int num_nodes, int num_internal, const int* left, const int* right,
                                 const int* level_offsets_host, int num_levels, const int* node_ranges,
                                 const float* mult, const float* centers, const float* radii, const float* acc4,
                                 float* node_feat, float* scale, void* stream) {
  if (num_nodes < 1 || num_internal < 0 || !mult || !centers || !radii || !acc4 || !node_feat || !scale ||
      !node_ranges || (num_internal > 0 && (!left || !right || !level_offsets_host)))
    return JB_ERR_ARG;
  cudaStream_t st = GST(stream);
  switch (p) {
#define JB_NP(PP)                                                                                             \
  case PP:                                                                                                    \
    k_node_powers<PP><<<gblocks(num_nodes, 128), 128, 0, st>>>(num_nodes, mult,                              \
                                                               reinterpret_cast<const float4*>(centers), radii, \
                                                               node_feat);                                     \
    break;
    JB_NP(1) JB_NP(2) JB_NP(3) JB_NP(4) JB_NP(5) JB_NP(6) JB_NP(7) JB_NP(8) JB_NP(9) JB_NP(10)
#undef JB_NP
    default:
      return JB_ERR_ORDER;
  }
  int rc = launch_status();
  if (rc) return rc;
  const int L = num_nodes - num_internal;
  k_leaf_force_min<<<gblocks(L, 128), 128, 0, st>>>(num_nodes, num_internal,
                                                   reinterpret_cast<const int2*>(node_ranges),
                                                   reinterpret_cast<const float4*>(acc4), scale);
  rc = launch_status();
  if (rc) return rc;
  for (int lev = num_levels - 1; lev >= 0; --lev) {
    const int a = level_offsets_host[lev], b = level_offsets_host[lev + 1];
    if (b <= a) continue;
    k_force_min_level<<<gblocks(b - a, 128), 128, 0, st>>>(a, b, left, right, scale);
    rc = launch_status();
    if (rc) return rc;
  }
  return JB_OK;
}

JB_API int jb_node_dehnen_power(int p, int num_nodes, const float* mult, int row_stride, double* out, void* stream) {
  if (p < 0 || p > JB_MAX_ORDER || num_nodes < 0 || row_stride < (p + 1) * (p + 1) ||
      (num_nodes > 0 && (!mult || !out)))
    return JB_ERR_ARG;
  if (num_nodes == 0) return JB_OK;
  k_dehnen_power<<<gblocks(num_nodes, 128), 128, 0, GST(stream)>>>(p, num_nodes, mult, row_stride, out);
  return launch_status();
}

JB_API int jb_node_force_scale(int num_nodes, int num_internal, const int* left, const int* right,
                               const int* level_offsets_host, int num_levels, const int* node_ranges,
                               const float* acc4, float* scale, void* stream) {
  if (num_nodes < 1 || num_internal < 0 || num_internal >= num_nodes || !node_ranges || !acc4 || !scale ||
      (num_internal > 0 && (!left || !right || !level_offsets_host || num_levels < 1)))
    return JB_ERR_ARG;
  cudaStream_t st = GST(stream);
  const int L = num_nodes - num_internal;
  k_leaf_force_min<<<gblocks(L, 128), 128, 0, st>>>(num_nodes, num_internal, reinterpret_cast<const int2*>(node_ranges),
                                                   reinterpret_cast<const float4*>(acc4), scale);
  int rc = launch_status();
  if (rc) return rc;
  for (int lev = num_levels - 1; lev >= 0; --lev) {
    const int a = level_offsets_host[lev], b = level_offsets_host[lev + 1];
    if (b <= a) continue;
    k_force_min_level<<<gblocks(b - a, 128), 128, 0, st>>>(a, b, left, right, scale);
    rc = launch_status();
    if (rc) return rc;
  }
  return JB_OK;
}

JB_API int jb_gear_pair_features(int64_t n, const int64_t* pair_ids, const int* pair_tgt, const int* far_src,
                                 const float* centers, const float* radii, const float* node_feat,
                                 const float* scale, float G, float* out, void* stream) {
  if (n < 0 || (n > 0 && (!pair_tgt || !far_src || !centers || !radii || !node_feat || !scale || !out)))
    return JB_ERR_ARG;
  if (n == 0) return JB_OK;
  k_pair_features<<<gblocks(n, 128), 128, 0, GST(stream)>>>(n, pair_ids, pair_tgt, far_src,
                                                             reinterpret_cast<const float4*>(centers), radii,
                                                             node_feat, scale, G, out);
  return launch_status();
}

JB_API int jb_gear_errors(int64_t n, const int64_t* pair_ids, const int* pair_tgt, const int* far_src,
                          const float* mult10, const float* centers, const float* radii, const float* scale, float G,
                          float* out, void* stream) {
  if (n < 0 || (n > 0 && (!pair_ids || !pair_tgt || !far_src || !mult10 || !centers || !radii || !scale || !out)))
    return JB_ERR_ARG;
  if (n == 0) return JB_OK;
  k_gear_errors<<<gblocks(n, 64), 64, 0, GST(stream)>>>(n, pair_ids, pair_tgt, far_src, mult10,
                                                        reinterpret_cast<const float4*>(centers), radii, scale, G,
                                                        out);
  return launch_status();
}

JB_API int jb_gear_train_grad(int n, const float* X, const int* labels, const float* Wq, float* gpart, float* lpart,
                              void* stream) {
  if (n < 1 || !X || !labels || !Wq || !gpart || !lpart) return JB_ERR_ARG;
  const size_t sm = sizeof(float) * (kParams + (kIn + 4 * kH + kOut + 1) * kTrainThreads);
  cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_mlp_grad<<<gblocks(n, kTrainThreads), kTrainThreads, sm, GST(stream)>>>(n, X, labels, Wq, gpart, lpart);
  return launch_status();
}

JB_API int jb_gear_adam(int nblocks, const float* gpart, float inv_batch, float lr, float beta1, float beta2,
                        float eps, int step, float* master, float* m1, float* m2, float* Wq, void* stream) {
  if (nblocks < 1 || !gpart || !master || !m1 || !m2 || !Wq || step < 1) return JB_ERR_ARG;
  k_mlp_adam<<<gblocks(kParams, 256), 256, 0, GST(stream)>>>(nblocks, gpart, inv_batch, lr, beta1, beta2, eps, step,
                                                             master, m1, m2, Wq);
  return launch_status();
}

JB_API int jb_gear_select(int64_t n, const int* pair_tgt, const int* far_src, const float* centers,
                          const float* radii, const float* node_feat, const float* scale, float G, const float* Wq,
                          const float* norm, float conf, float min_top, int* gear_out, void* stream) {
  if (n < 0 || (n > 0 && (!pair_tgt || !far_src || !centers || !radii || !node_feat || !scale || !Wq || !norm ||
                          !gear_out)))
    return JB_ERR_ARG;
  if (n == 0) return JB_OK;
  k_gear_select<<<gblocks(n, 128), 128, 0, GST(stream)>>>(n, pair_tgt, far_src,
                                                           reinterpret_cast<const float4*>(centers), radii,
                                                           node_feat, scale, G, Wq, norm, conf, min_top, gear_out);
  return launch_status();
}

}  // extern "C"
