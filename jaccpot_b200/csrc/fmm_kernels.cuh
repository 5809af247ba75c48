#pragma once
// sm_100a kernels of the FMM evaluation pass, templated on the expansion order.
// Each order is instantiated in its own translation unit (fmm_order.cu built
// with -DJB_ORDER=P); the C-ABI entry points live in fmm_capi.cu.
//
// Work decomposition (nothing here uses atomics; every output element has one
// writer, so results are run-to-run deterministic):
//   P2M        warp per leaf: COM by warp reduction, U_n^m per lane, transpose
//              reduction of the (p+1)^2 coefficients through shared memory;
//   M2M / L2L  one launch per level: each translation's degrees split over
//              four warps (k_*_level_split), or thread per (parent, child) on
//              the wide L2L levels;
//   M2L        thread per work unit (<= 512 pairs of one target's CSR list),
//              units sorted by length so warps stay converged; the local
//              accumulates in registers;
//   leaf eval  L2P warp per leaf (lane = particle, the leaf's local staged in
//              shared memory), then P2P warp per work unit (a leaf and a slice
//              of its neighbour list), sources staged 32 at a time in shared
//              memory.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <cstring>
#include <type_traits>

#include "../../include/jaccpot_b200.h"
#include "fmm_ops.cuh"

namespace jb {

// Defined in fmm_capi.cu.
int cuda_status(cudaError_t e);
// Levels with at most this many parents use the degree-split M2M [0] / L2L
// [1] kernels, wider ones the thread-per-translation kernels
// (jb_set_level_split).
extern int g_split_max_parents[2];
// Nonzero: leaves of more than 16 particles take the chunk-major near-field
// form (k_leaf_units_flat) in jb_leaf_eval (jb_set_leaf_form).
extern int g_leaf_flat;
// Nonzero: the single-order FP32 M2L fetches source rows with the whole warp
// (k_m2l_units_coop) rather than thread by thread (jb_set_m2l_fetch).
extern int g_m2l_coop;
inline int launch_status() { return cuda_status(cudaGetLastError()); }

// Most particles a leaf may hold: the near-field kernels give each target of
// a leaf one lane (or a lane group) of a warp, a leaf of more than 32 in two
// passes of at most 32 targets, and each split leaf one partial row of
// kMaxLeaf float4.  A unit whose leaf holds more writes nothing and sets
// JB_LEAF_ERR_OCCUPANCY in the error word; a partial-row slot at or beyond
// the caller's slot count is skipped and sets JB_LEAF_ERR_SLOT
// (jb_leaf_eval_errors reads the word).
constexpr int kMaxLeaf = JB_MAX_LEAF_OCCUPANCY;
static_assert(kMaxLeaf == 64, "leaves are evaluated in at most two passes of 32 targets");
__device__ __forceinline__ void leaf_error(int* err, int bit) {
  if (err) atomicOr(err, bit);
}

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
// Two adjacent threads per parent (one per child): each shifts its child's
// multipole, the pair adds the two through one shuffle per coefficient (the
// same sum in both lanes), and the even lane writes the parent.
template <int P>
__global__ void __launch_bounds__(128) k_m2m_level(int first, int last, const int* __restrict__ left,
                                                   const int* __restrict__ right, const int2* __restrict__ ranges,
                                                   float4* __restrict__ centers, float* __restrict__ mult) {
  constexpr int C = csize(P), CS = cstride(P);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = first + (tid >> 1);
  const bool ok = i < last;
  const int side = tid & 1;
  float v[C];
  float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
  if (ok) {
    const int a = left[i], b = right[i];
    const float4 ca = centers[a], cb = centers[b];
    const float m = ca.w + cb.w;
    if (m > 0.f) {
      const float inv = 1.f / m;
      c = make_float4((ca.w * ca.x + cb.w * cb.x) * inv, (ca.w * ca.y + cb.w * cb.y) * inv,
                      (ca.w * ca.z + cb.w * cb.z) * inv, m);
    } else {
      // no mass below: the mean particle position (mutual/topology.py:500-516),
      // from the children's means weighted by their particle counts
      const int2 ra = ranges[a], rb = ranges[b];
      const float na = (float)(ra.y - ra.x + 1), nb = (float)(rb.y - rb.x + 1);
      const float inv = 1.f / (na + nb);
      c = make_float4((na * ca.x + nb * cb.x) * inv, (na * ca.y + nb * cb.y) * inv, (na * ca.z + nb * cb.z) * inv,
                      0.f);
    }
    const float4 cc = side ? cb : ca;
    const float* src = mult + (size_t)(side ? b : a) * CS;
#pragma unroll
    for (int k = 0; k < C; ++k) v[k] = src[k];
    m2m_pair<P>(v, cc.x - c.x, cc.y - c.y, cc.z - c.z);
  } else {
#pragma unroll
    for (int k = 0; k < C; ++k) v[k] = 0.f;
  }
#pragma unroll
  for (int k = 0; k < C; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], 1);
  if (ok && side == 0) {
    centers[i] = c;
    float* dst = mult + (size_t)i * CS;
#pragma unroll
    for (int k = 0; k < C; ++k) dst[k] = v[k];
#pragma unroll
    for (int k = C; k < CS; ++k) dst[k] = 0.f;
  }
}

// ---------------------------------------------------------------------------
// M2L over work units.  A unit is (target, first pair, end pair, slot): at
// most a fixed number of consecutive pairs of one target's CSR list, so no
// thread walks an arbitrarily long list.  slot < 0: the unit holds the
// target's whole list and writes locals[target]; slot >= 0: it writes the
// partial row partials[slot], and k_m2l_reduce sums a target's partial rows
// in slot order.  Thread per unit, units sorted longest first.
//
// The next pair's multipole row is fetched into a per-thread shared-memory
// row with cp.async while the current pair is rotated back, which hides the
// L2 gather latency; the row stride is an odd number of 16-byte words so the
// per-thread LDS.128 reads are bank-conflict free.  The local accumulates in
// registers (255 per thread, 8 warps per SM).
// ---------------------------------------------------------------------------
constexpr int kM2LThreads = 64;

__host__ __device__ constexpr int row4(int p) { return (cstride(p) / 4) | 1; }  // float4 per smem row (odd)

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// NEG = true evaluates M2L(c_source - c_target) instead (the displacement of
// the reverse pair), which is what the adjoint's transposed M2L needs: the
// real M2L matrix is symmetric, so sum_v M2L(c_v - c_u)^T Lbar_v is this
// kernel run over u's own list with Lbar in place of the multipoles.
//
// W: pair e's contribution is scaled by far_w[e] (the block-step level weight
// of the mutual lane); the unweighted instantiations do not read it.
template <int P, bool NEG, bool W = false>
__global__ void __launch_bounds__(kM2LThreads, 4) k_m2l_units(int num_units, const int4* __restrict__ units,
                                                              const float* __restrict__ mult,
                                                              const float4* __restrict__ centers,
                                                              const int* __restrict__ far_src,
                                                              float* __restrict__ locals,
                                                              float* __restrict__ partials, int rs,
                                                              const float* __restrict__ far_w = nullptr) {
  // rs: row stride (floats) of mult / locals / partials, >= cstride(P); a
  // lower-order pass (gear) reads the prefix of each row (degrees <= P).
  constexpr int C = csize(P), CS = cstride(P), R4 = row4(P);
  extern __shared__ float4 m2l_smem[];
  float4* row = m2l_smem + threadIdx.x * R4;
  const int u = blockIdx.x * kM2LThreads + threadIdx.x;
  if (u >= num_units) return;
  const int4 U = units[u];
  const int tgt = U.x, e0 = U.y, e1 = U.z, slot = U.w;
  float acc[C];
#pragma unroll
  for (int k = 0; k < C; ++k) acc[k] = 0.f;
  const float4 ct = centers[tgt];
  // source ids run two pairs ahead and centres one pair ahead of the row
  // copies, so no load feeds an address in the same iteration
  const int s0 = far_src[e0];
  int s1 = (e0 + 1 < e1) ? far_src[e0 + 1] : s0;
  {
    const float4* src = reinterpret_cast<const float4*>(mult + (size_t)s0 * rs);
#pragma unroll
    for (int k = 0; k < CS / 4; ++k) cp_async16(row + k, src + k);
    cp_async_commit();
  }
  float4 cs = centers[s0];
  float4 cs1 = centers[s1];
  for (int e = e0; e < e1; ++e) {
    float v[C];
    cp_async_wait_all();
#pragma unroll
    for (int k = 0; k < CS / 4; ++k) {
      const float4 q = row[k];
      if (4 * k + 0 < C) v[4 * k + 0] = q.x;
      if (4 * k + 1 < C) v[4 * k + 1] = q.y;
      if (4 * k + 2 < C) v[4 * k + 2] = q.z;
      if (4 * k + 3 < C) v[4 * k + 3] = q.w;
    }
    // every value read from `row` is in registers: refill it for the next pair
    if (e + 1 < e1) {
      const float4* src = reinterpret_cast<const float4*>(mult + (size_t)s1 * rs);
#pragma unroll
      for (int k = 0; k < CS / 4; ++k) cp_async16(row + k, src + k);
      cp_async_commit();
    }
    const int s2 = (e + 2 < e1) ? __ldg(far_src + e + 2) : s1;
    const float dx = NEG ? cs.x - ct.x : ct.x - cs.x;
    const float dy = NEG ? cs.y - ct.y : ct.y - cs.y;
    const float dz = NEG ? cs.z - ct.z : ct.z - cs.z;
    m2l_kfold_acc<P, W>(v, acc, dx, dy, dz, W ? __ldg(far_w + e) : 1.f);
    cs = cs1;
    cs1 = centers[s2];
    s1 = s2;
  }
  float* dst = (slot < 0) ? locals + (size_t)tgt * rs : partials + (size_t)slot * rs;
#pragma unroll
  for (int k = 0; k < C; ++k) dst[k] = acc[k];
  for (int k = C; k < rs; ++k) dst[k] = 0.f;
}

// The warp's next source rows, fetched together: lane j's row s_j (-1: none)
// goes to wrows + j * R4, one cp.async instruction per row, lane k copying
// 16-byte word k (k < NW); one cp.async group.  ids: the warp's 32 ints of
// shared memory.  The caller has made sure every lane is done with its row
// and with the previous ids (a __syncwarp after the last read).
template <int NW, int R4>
__device__ __forceinline__ void warp_rows_fetch(float4* wrows, int* ids, int lane, int s, const float* mult, int rs) {
  ids[lane] = s;
  __syncwarp();
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int4 sq = reinterpret_cast<const int4*>(ids)[q];
    const int sj[4] = {sq.x, sq.y, sq.z, sq.w};
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (sj[i] >= 0 && lane < NW)
        cp_async16(wrows + (4 * q + i) * R4 + lane, reinterpret_cast<const float4*>(mult + (size_t)sj[i] * rs) + lane);
  }
  cp_async_commit();
}

// k_m2l_units with each source row fetched by the whole warp: per pair the
// lanes publish their next source ids, and for each of the warp's 32 rows one
// cp.async instruction copies it, lane k taking 16-byte word k.  A row is then
// 2-3 cache lines for one instruction, where a thread copying its own row
// issues one instruction per word with all 32 lanes on different lines (32
// L1 wavefronts each).  The lanes step through their units together (units
// are sorted longest first, so a warp's lengths are close); a lane past its
// unit's end only takes part in the copies.  The same arithmetic as
// k_m2l_units (the compiler may fuse a multiply and an add differently in the
// two kernels: the sums agree to FP32 rounding).  At the headline workload
// this fetch takes the M2L from 2.96 to 2.68 ms (order 8).  The mixed-order
// kernel keeps the per-thread fetch: there the lanes' segment lengths differ
// more, and stepping them together measured slower (5.88 -> 5.94 ms).
template <int P, bool NEG, bool W = false>
__global__ void __launch_bounds__(kM2LThreads, 4) k_m2l_units_coop(int num_units, const int4* __restrict__ units,
                                                                   const float* __restrict__ mult,
                                                                   const float4* __restrict__ centers,
                                                                   const int* __restrict__ far_src,
                                                                   float* __restrict__ locals,
                                                                   float* __restrict__ partials, int rs,
                                                                   const float* __restrict__ far_w = nullptr) {
  constexpr int C = csize(P), CS = cstride(P), R4 = row4(P), NW = CS / 4;
  static_assert(NW <= 32, "one warp instruction copies a row");
  extern __shared__ float4 m2l_smem[];
  const int lane = threadIdx.x & 31;
  float4* wrows = m2l_smem + (threadIdx.x & ~31) * R4;  // the warp's 32 rows
  float4* row = wrows + lane * R4;
  int* ids = reinterpret_cast<int*>(m2l_smem + kM2LThreads * R4) + (threadIdx.x & ~31);
  const int u = blockIdx.x * kM2LThreads + threadIdx.x;
  const bool ok = u < num_units;
  const int4 U = ok ? units[u] : make_int4(0, 0, 0, -1);
  const int tgt = U.x, e0 = U.y, slot = U.w;
  const int n = ok ? U.z - U.y : 0;
  const int nmax = __reduce_max_sync(0xffffffffu, n);
  auto fetch = [&](int s) { warp_rows_fetch<NW, R4>(wrows, ids, lane, s, mult, rs); };
  float acc[C];
#pragma unroll
  for (int k = 0; k < C; ++k) acc[k] = 0.f;
  const float4 ct = ok ? centers[tgt] : make_float4(0.f, 0.f, 0.f, 0.f);
  int s0 = -1, s1 = -1;
  float4 cs = ct, cs1 = ct;
  if (n > 0) {
    s0 = far_src[e0];
    s1 = (n > 1) ? far_src[e0 + 1] : s0;
    cs = centers[s0];
    cs1 = centers[s1];
  }
  fetch(s0);
  for (int it = 0; it < nmax; ++it) {
    const bool act = it < n;
    float v[C];
    cp_async_wait_all();
    __syncwarp();  // the copies every lane issued into the warp's rows have landed
    if (act) {
#pragma unroll
      for (int k = 0; k < CS / 4; ++k) {
        const float4 q = row[k];
        if (4 * k + 0 < C) v[4 * k + 0] = q.x;
        if (4 * k + 1 < C) v[4 * k + 1] = q.y;
        if (4 * k + 2 < C) v[4 * k + 2] = q.z;
        if (4 * k + 3 < C) v[4 * k + 3] = q.w;
      }
    }
    __syncwarp();  // every row (and every id) read before the next copies
    fetch(act && it + 1 < n ? s1 : -1);
    if (act) {
      const int e = e0 + it;
      const int s2 = (it + 2 < n) ? __ldg(far_src + e + 2) : s1;
      const float dx = NEG ? cs.x - ct.x : ct.x - cs.x;
      const float dy = NEG ? cs.y - ct.y : ct.y - cs.y;
      const float dz = NEG ? cs.z - ct.z : ct.z - cs.z;
      m2l_kfold_acc<P, W>(v, acc, dx, dy, dz, W ? __ldg(far_w + e) : 1.f);
      cs = cs1;
      cs1 = centers[s2];
      s1 = s2;
    }
  }
  cp_async_wait_all();  // nothing in flight (the last fetch copies nothing)
  if (!ok) return;
  float* dst = (slot < 0) ? locals + (size_t)tgt * rs : partials + (size_t)slot * rs;
#pragma unroll
  for (int k = 0; k < C; ++k) dst[k] = acc[k];
  for (int k = C; k < rs; ++k) dst[k] = 0.f;
}

// L2L straight to the leaves (jb_l2l_leaves): a leaf's local is its own M2L
// sum plus, for each ancestor a that received far pairs, L2L(a -> leaf) of a's
// own M2L sum.  Shifting the centre of a degree-P local expansion is exact,
// so this equals the level-by-level cascade up to rounding, and only the
// leaves' locals -- all that L2P reads -- are formed; the internal nodes keep
// their own M2L sums.  units[u] = (leaf node, first, end, unused) over anc[]
// (the leaf's ancestors with far pairs, nearest first); thread per leaf, the
// warp's ancestor rows fetched together as in k_m2l_units_coop.  One launch
// with every leaf's chain in parallel, where the cascade runs one dependent
// launch per level.
template <int P>
__global__ void __launch_bounds__(kM2LThreads, 4) k_l2l_leaves(int num_units, const int4* __restrict__ units,
                                                               const int* __restrict__ anc,
                                                               const float4* __restrict__ centers,
                                                               float* __restrict__ locals) {
  constexpr int C = csize(P), CS = cstride(P), R4 = row4(P), NW = CS / 4;
  extern __shared__ float4 m2l_smem[];
  const int lane = threadIdx.x & 31;
  float4* wrows = m2l_smem + (threadIdx.x & ~31) * R4;
  float4* row = wrows + lane * R4;
  int* ids = reinterpret_cast<int*>(m2l_smem + kM2LThreads * R4) + (threadIdx.x & ~31);
  const int u = blockIdx.x * kM2LThreads + threadIdx.x;
  const bool ok = u < num_units;
  const int4 U = ok ? units[u] : make_int4(0, 0, 0, -1);
  const int leaf = U.x, e0 = U.y;
  const int n = ok ? U.z - U.y : 0;
  const int nmax = __reduce_max_sync(0xffffffffu, n);
  float acc[C];
#pragma unroll
  for (int k = 0; k < C; ++k) acc[k] = 0.f;
  const float4 cl = ok ? centers[leaf] : make_float4(0.f, 0.f, 0.f, 0.f);
  int s0 = -1, s1 = -1;
  float4 ca = cl, ca1 = cl;
  if (n > 0) {
    s0 = anc[e0];
    s1 = (n > 1) ? anc[e0 + 1] : s0;
    ca = centers[s0];
    ca1 = centers[s1];
  }
  warp_rows_fetch<NW, R4>(wrows, ids, lane, s0, locals, CS);
  for (int it = 0; it < nmax; ++it) {
    const bool act = it < n;
    float v[C];
    cp_async_wait_all();
    __syncwarp();  // the copies every lane issued into the warp's rows have landed
    if (act) {
#pragma unroll
      for (int k = 0; k < CS / 4; ++k) {
        const float4 q = row[k];
        if (4 * k + 0 < C) v[4 * k + 0] = q.x;
        if (4 * k + 1 < C) v[4 * k + 1] = q.y;
        if (4 * k + 2 < C) v[4 * k + 2] = q.z;
        if (4 * k + 3 < C) v[4 * k + 3] = q.w;
      }
    }
    __syncwarp();  // every row (and every id) read before the next copies
    warp_rows_fetch<NW, R4>(wrows, ids, lane, act && it + 1 < n ? s1 : -1, locals, CS);
    if (act) {
      const int s2 = (it + 2 < n) ? __ldg(anc + e0 + it + 2) : s1;
      l2l_pair<P>(v, ca.x - cl.x, ca.y - cl.y, ca.z - cl.z);
#pragma unroll
      for (int k = 0; k < C; ++k) acc[k] += v[k];
      ca = ca1;
      ca1 = centers[s2];
      s1 = s2;
    }
  }
  cp_async_wait_all();
  if (!ok || n == 0) return;
  float* dst = locals + (size_t)leaf * CS;
#pragma unroll
  for (int k = 0; k < C; ++k) dst[k] += acc[k];
}

// Sums the partial rows of targets whose list was split: split[i] =
// (target, first slot, number of slots, unused).  Thread per (target, coefficient).
static __global__ void __launch_bounds__(256) k_m2l_reduce(int num_split, const int4* __restrict__ split,
                                                           const float* __restrict__ partials,
                                                           float* __restrict__ locals, int CS) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(t / CS), k = (int)(t % CS);
  if (i >= num_split) return;
  const int4 sp = split[i];
  float a = 0.f;
  for (int q = 0; q < sp.z; ++q) a += partials[(size_t)(sp.y + q) * CS + k];
  locals[(size_t)sp.x * CS + k] = a;
}

// ---------------------------------------------------------------------------
// M2L with per-pair orders (gears) in one launch.  The orders form the ladder
// P, P-2, P-4, P-6 (those >= 1; kMixedSegs(P) of them).  A unit is a slice of
// one target's far list whose pairs are sorted by order, highest first, so it
// holds up to four segments: units[u] = (target, first pair, end pair, slot)
// and bounds[u] = (b1, b2, b3, end): segment j = [b_j, b_{j+1}) with b_0 =
// first pair, evaluated at order P - 2j into the same registers (a lower
// order adds only to the degrees it has).  Thread per unit; every lane of a
// warp finishes segment j (__syncwarp) before any starts segment j+1, so
// lanes only diverge inside a segment.  Units are sorted by their segment
// lengths (highest order first), so the lanes of a warp have similar ones.
// Slots and the split reduce are k_m2l_units'.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int kMixedSegs(int P) { return (P + 1) / 2 < 4 ? (P + 1) / 2 : 4; }

template <int P>
__device__ __forceinline__ void m2l_segment(int e0, int e1, const float* __restrict__ mult,
                                            const float4* __restrict__ centers, const int* __restrict__ far_src,
                                            int rs, float4 ct, float4* row, float* acc) {
  constexpr int C = csize(P), CS = cstride(P);
  if (e1 <= e0) return;
  const int s0 = far_src[e0];
  int s1 = (e0 + 1 < e1) ? far_src[e0 + 1] : s0;
  {
    const float4* src = reinterpret_cast<const float4*>(mult + (size_t)s0 * rs);
#pragma unroll
    for (int k = 0; k < CS / 4; ++k) cp_async16(row + k, src + k);
    cp_async_commit();
  }
  float4 cs = centers[s0];
  float4 cs1 = centers[s1];
  for (int e = e0; e < e1; ++e) {
    float v[C];
    cp_async_wait_all();
#pragma unroll
    for (int k = 0; k < CS / 4; ++k) {
      const float4 q = row[k];
      if (4 * k + 0 < C) v[4 * k + 0] = q.x;
      if (4 * k + 1 < C) v[4 * k + 1] = q.y;
      if (4 * k + 2 < C) v[4 * k + 2] = q.z;
      if (4 * k + 3 < C) v[4 * k + 3] = q.w;
    }
    if (e + 1 < e1) {
      const float4* src = reinterpret_cast<const float4*>(mult + (size_t)s1 * rs);
#pragma unroll
      for (int k = 0; k < CS / 4; ++k) cp_async16(row + k, src + k);
      cp_async_commit();
    }
    const int s2 = (e + 2 < e1) ? __ldg(far_src + e + 2) : s1;
    m2l_kfold_acc<P, false>(v, acc, ct.x - cs.x, ct.y - cs.y, ct.z - cs.z, 1.f);
    cs = cs1;
    cs1 = centers[s2];
    s1 = s2;
  }
}

template <int P, int J = 0>
__device__ __forceinline__ void m2l_segments(const int* b, const float* __restrict__ mult,
                                             const float4* __restrict__ centers, const int* __restrict__ far_src,
                                             int rs, float4 ct, float4* row, float* acc) {
  if constexpr (J < kMixedSegs(P)) {
    m2l_segment<P - 2 * J>(b[J], b[J + 1], mult, centers, far_src, rs, ct, row, acc);
    __syncwarp();
    m2l_segments<P, J + 1>(b, mult, centers, far_src, rs, ct, row, acc);
  }
}

template <int P>
__global__ void __launch_bounds__(kM2LThreads, 4) k_m2l_mixed(int num_units, const int4* __restrict__ units,
                                                              const int4* __restrict__ bounds,
                                                              const float* __restrict__ mult,
                                                              const float4* __restrict__ centers,
                                                              const int* __restrict__ far_src,
                                                              float* __restrict__ locals,
                                                              float* __restrict__ partials, int rs) {
  constexpr int C = csize(P);
  extern __shared__ float4 m2l_smem[];
  float4* row = m2l_smem + threadIdx.x * row4(P);
  const int u = blockIdx.x * kM2LThreads + threadIdx.x;
  const bool ok = u < num_units;  // lanes past the end run empty segments to the warp barriers
  const int4 U = ok ? units[u] : make_int4(0, 0, 0, -1);
  const int4 B = ok ? bounds[u] : make_int4(0, 0, 0, 0);
  const int b[5] = {U.y, B.x, B.y, B.z, B.w};
  float acc[C];
#pragma unroll
  for (int k = 0; k < C; ++k) acc[k] = 0.f;
  const float4 ct = ok ? centers[U.x] : make_float4(0.f, 0.f, 0.f, 0.f);
  m2l_segments<P>(b, mult, centers, far_src, rs, ct, row, acc);
  if (!ok) return;
  float* dst = (U.w < 0) ? locals + (size_t)U.x * rs : partials + (size_t)U.w * rs;
#pragma unroll
  for (int k = 0; k < C; ++k) dst[k] = acc[k];
  for (int k = C; k < rs; ++k) dst[k] = 0.f;
}

// ---------------------------------------------------------------------------
// M2M / L2L, one level, degrees split over four warps.
//
// A translation's rotations and B products act on each degree separately;
// only the z-shift mixes degrees.  So a block of four warps takes 32
// translations (lane = translation) and warp q works on a fixed set of
// degrees (kDegSet: the degrees dealt greedily by (2l+1)^2, largest first, so
// the four chains are about equally long), exchanging the rotated vectors
// once through shared memory for the z-shift.  Each warp's chain is about a
// quarter of the single-thread one, which is what bounds these levels: even
// the widest level here holds only ~31 k translations, far too few for the
// single-thread form to fill the GPU.  The operations, their order and their
// constants are those of m2m_pair / l2l_pair.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr unsigned kDegSet(int P, int q) {
  int tot[4] = {0, 0, 0, 0};
  unsigned mask[4] = {0u, 0u, 0u, 0u};
  for (int l = P; l >= 0; --l) {
    int best = 0;
    for (int k = 1; k < 4; ++k)
      if (tot[k] < tot[best]) best = k;
    tot[best] += (2 * l + 1) * (2 * l + 1);
    mask[best] |= 1u << l;
  }
  return mask[q];
}

// f(integral_constant<int, l>) for every degree l <= P in MASK, ascending.
template <int P, unsigned MASK, int L = 0>
struct ForDeg {
  template <typename F>
  static __device__ __forceinline__ void run(F&& f) {
    if constexpr (L <= P) {
      if constexpr (((MASK >> L) & 1u) != 0u) f(std::integral_constant<int, L>{});
      ForDeg<P, MASK, L + 1>::run(f);
    }
  }
};

// dz_rot restricted to degree L (the same angle recurrence, so the same values).
template <int L, bool NEG>
__device__ __forceinline__ void dz_rot_deg(float* v, float c1, float s1) {
  const float sa = NEG ? -s1 : s1;
  float c = c1, s = sa;
#pragma unroll
  for (int m = 1; m <= L; ++m) {
    if (m > 1) {
      const float cn = c * c1 - s * sa;
      s = fmaf(s, c1, c * sa);
      c = cn;
    }
    const int ip = shi(L, m), im = shi(L, -m);
    const float vp = v[ip], vm = v[im];
    v[ip] = c * vp - s * vm;
    v[im] = fmaf(s, vp, c * vm);
  }
}

constexpr int kSplitItems = 32;  // translations per block (lane = translation)
__host__ __device__ constexpr int xrow(int P) { return csize(P) | 1; }  // odd row: conflict-free exchange

// One translation's degrees MASK of v (indexed by the full packed layout):
// IS_M2M selects m2m_pair's chain (delta = child - parent), else l2l_pair's
// (delta = parent - child).  xr: this translation's exchange row.
template <int P, unsigned MASK, bool IS_M2M>
__device__ __forceinline__ void split_translate(float* v, float dx, float dy, float dz, float* xr) {
  float caz, saz, cax, sax, r;
  align_cs(dx, dy, dz, caz, saz, cax, sax, r);
  const float d = r < 1e-30f ? 0.f : r;
  ForDeg<P, MASK>::run([&](auto lc) {
    constexpr int L = decltype(lc)::value;
    dz_rot_deg<L, false>(v, caz, saz);
    BDeg<L, !IS_M2M>::apply(v);
    dz_rot_deg<L, true>(v, cax, sax);
    BDeg<L, !IS_M2M>::apply(v);
#pragma unroll
    for (int m = -L; m <= L; ++m) xr[shi(L, m)] = v[shi(L, m)];
  });
  __syncthreads();
  float dk[P + 1];
  dk[0] = 1.f;
#pragma unroll
  for (int k = 1; k <= P; ++k) dk[k] = dk[k - 1] * d * (float)(1.0 / (double)k);
  ForDeg<P, MASK>::run([&](auto lc) {
    constexpr int n = decltype(lc)::value;
#pragma unroll
    for (int m = -n; m <= n; ++m) {
      float acc = v[shi(n, m)];
      if (IS_M2M) {
#pragma unroll
        for (int k = 1; k <= n - iabs(m); ++k) acc = fmaf(dk[k], xr[shi(n - k, m)], acc);
      } else {
#pragma unroll
        for (int k = 1; k <= P - n; ++k) acc = fmaf(dk[k], xr[shi(n + k, m)], acc);
      }
      v[shi(n, m)] = acc;
    }
    BDeg<n, !IS_M2M>::apply(v);
    dz_rot_deg<n, false>(v, cax, sax);
    BDeg<n, !IS_M2M>::apply(v);
    dz_rot_deg<n, true>(v, caz, saz);
  });
}

// Item i of the level: parent first + i/2, child side i&1 (as the
// single-thread kernels).  Inactive items still reach the block barrier.
template <int P, unsigned MASK>
__device__ __forceinline__ void m2m_split_warp(int first, int last, const int* __restrict__ left,
                                               const int* __restrict__ right, const int2* __restrict__ ranges,
                                               float4* __restrict__ centers, float* __restrict__ mult, float* xr,
                                               bool write_center) {
  constexpr int C = csize(P), CS = cstride(P);
  const int lane = threadIdx.x & 31;
  const int i = first + (int)(blockIdx.x * kSplitItems + lane) / 2;
  const bool ok = i < last;
  const int side = lane & 1;
  float v[C];
  float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 cc = c;
  if (ok) {
    const int a = left[i], b = right[i];
    const float4 ca = centers[a], cb = centers[b];
    const float m = ca.w + cb.w;
    if (m > 0.f) {
      const float inv = 1.f / m;
      c = make_float4((ca.w * ca.x + cb.w * cb.x) * inv, (ca.w * ca.y + cb.w * cb.y) * inv,
                      (ca.w * ca.z + cb.w * cb.z) * inv, m);
    } else {
      const int2 ra = ranges[a], rb = ranges[b];
      const float na = (float)(ra.y - ra.x + 1), nb = (float)(rb.y - rb.x + 1);
      const float inv = 1.f / (na + nb);
      c = make_float4((na * ca.x + nb * cb.x) * inv, (na * ca.y + nb * cb.y) * inv, (na * ca.z + nb * cb.z) * inv,
                      0.f);
    }
    cc = side ? cb : ca;
    const float* src = mult + (size_t)(side ? b : a) * CS;
    ForDeg<P, MASK>::run([&](auto lc) {
      constexpr int L = decltype(lc)::value;
#pragma unroll
      for (int m = -L; m <= L; ++m) v[shi(L, m)] = src[shi(L, m)];
    });
  } else {
    ForDeg<P, MASK>::run([&](auto lc) {
      constexpr int L = decltype(lc)::value;
#pragma unroll
      for (int m = -L; m <= L; ++m) v[shi(L, m)] = 0.f;
    });
  }
  split_translate<P, MASK, true>(v, cc.x - c.x, cc.y - c.y, cc.z - c.z, xr);
  ForDeg<P, MASK>::run([&](auto lc) {
    constexpr int L = decltype(lc)::value;
#pragma unroll
    for (int m = -L; m <= L; ++m) v[shi(L, m)] += __shfl_xor_sync(0xffffffffu, v[shi(L, m)], 1);
  });
  if (ok && side == 0) {
    float* dst = mult + (size_t)i * CS;
    ForDeg<P, MASK>::run([&](auto lc) {
      constexpr int L = decltype(lc)::value;
#pragma unroll
      for (int m = -L; m <= L; ++m) dst[shi(L, m)] = v[shi(L, m)];
    });
    if (write_center) {
      centers[i] = c;
#pragma unroll
      for (int k = C; k < CS; ++k) dst[k] = 0.f;
    }
  }
}

template <int P>
__global__ void __launch_bounds__(128) k_m2m_level_split(int first, int last, const int* __restrict__ left,
                                                         const int* __restrict__ right, const int2* __restrict__ ranges,
                                                         float4* __restrict__ centers, float* __restrict__ mult) {
  __shared__ float xs[kSplitItems * xrow(P)];
  float* xr = xs + (threadIdx.x & 31) * xrow(P);
  switch (threadIdx.x >> 5) {
    case 0: m2m_split_warp<P, kDegSet(P, 0)>(first, last, left, right, ranges, centers, mult, xr, true); break;
    case 1: m2m_split_warp<P, kDegSet(P, 1)>(first, last, left, right, ranges, centers, mult, xr, false); break;
    case 2: m2m_split_warp<P, kDegSet(P, 2)>(first, last, left, right, ranges, centers, mult, xr, false); break;
    default: m2m_split_warp<P, kDegSet(P, 3)>(first, last, left, right, ranges, centers, mult, xr, false); break;
  }
}

template <int P, unsigned MASK>
__device__ __forceinline__ void l2l_split_warp(int first, int last, const int* __restrict__ left,
                                               const int* __restrict__ right, const float4* __restrict__ centers,
                                               float* __restrict__ locals, float* xr) {
  constexpr int C = csize(P), CS = cstride(P);
  const int lane = threadIdx.x & 31;
  const int i = first + (int)(blockIdx.x * kSplitItems + lane) / 2;
  const bool ok = i < last;
  float v[C];
  int ch = 0;
  float4 cp = make_float4(0.f, 0.f, 0.f, 0.f), cc = cp;
  if (ok) {
    ch = (lane & 1) ? right[i] : left[i];
    cp = centers[i];
    cc = centers[ch];
    const float* src = locals + (size_t)i * CS;
    ForDeg<P, MASK>::run([&](auto lc) {
      constexpr int L = decltype(lc)::value;
#pragma unroll
      for (int m = -L; m <= L; ++m) v[shi(L, m)] = src[shi(L, m)];
    });
  } else {
    ForDeg<P, MASK>::run([&](auto lc) {
      constexpr int L = decltype(lc)::value;
#pragma unroll
      for (int m = -L; m <= L; ++m) v[shi(L, m)] = 0.f;
    });
  }
  split_translate<P, MASK, false>(v, cp.x - cc.x, cp.y - cc.y, cp.z - cc.z, xr);
  if (ok) {
    float* dst = locals + (size_t)ch * CS;
    ForDeg<P, MASK>::run([&](auto lc) {
      constexpr int L = decltype(lc)::value;
#pragma unroll
      for (int m = -L; m <= L; ++m) dst[shi(L, m)] += v[shi(L, m)];
    });
  }
  (void)C;
}

template <int P>
__global__ void __launch_bounds__(128) k_l2l_level_split(int first, int last, const int* __restrict__ left,
                                                         const int* __restrict__ right,
                                                         const float4* __restrict__ centers,
                                                         float* __restrict__ locals) {
  __shared__ float xs[kSplitItems * xrow(P)];
  float* xr = xs + (threadIdx.x & 31) * xrow(P);
  switch (threadIdx.x >> 5) {
    case 0: l2l_split_warp<P, kDegSet(P, 0)>(first, last, left, right, centers, locals, xr); break;
    case 1: l2l_split_warp<P, kDegSet(P, 1)>(first, last, left, right, centers, locals, xr); break;
    case 2: l2l_split_warp<P, kDegSet(P, 2)>(first, last, left, right, centers, locals, xr); break;
    default: l2l_split_warp<P, kDegSet(P, 3)>(first, last, left, right, centers, locals, xr); break;
  }
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
// Leaf evaluation over work units: the far field (L2P, k_leaf_l2p, warp per
// leaf) and then the near field (P2P, k_leaf_units, warp per unit).
//
// A unit is one target leaf and a slice of its near list, stored as runs of
// consecutive source leaves (= contiguous particle ranges, runs[r] = (first
// particle, count)); units[u] = (leaf, first run, end run, source count),
// aux[u] = (slot, flags).  flags & 1: the unit also does the leaf's self block
// (diagonal excluded), and k_leaf_l2p evaluates the leaf's far field for it.
// slot < 0: the unit covers the whole leaf and adds its sum to out_acc4;
// otherwise it writes partial[slot][lane] and k_leaf_reduce adds a leaf's
// slots to out_acc4 in order.
//
// Sources stream through the warp in packed chunks of 32 (the runs are
// concatenated; each lane tracks its own run), staged in shared memory and
// broadcast; the next chunk's loads are issued before the current chunk is
// consumed.  Leaves with <= 16 (<= 8) particles give each target 2 (4)
// lanes that split every chunk, so most lanes do useful work.  KAHAN adds
// each chunk's partial sums into compensated per-target accumulators.
// ---------------------------------------------------------------------------
struct SmemF {
  const float* f;
  __device__ __forceinline__ float operator()(int k) const { return f[k]; }
};

// A leaf's near and far parts are each rounded to FP32 on their own, then
// added with one rounded add.  Written out so the compiler fuses neither the
// scaling nor the add into an FMA: the sum then has the same bits whichever
// part is written first (the near field before the far field when the two
// run on separate streams, JB_P2P_NEAR_FIRST / JB_P2P_FAR_AFTER).
__device__ __forceinline__ float4 near_scaled(float G, const float* v) {
  return make_float4(__fmul_rn(-G, v[0]), __fmul_rn(-G, v[1]), __fmul_rn(-G, v[2]), __fmul_rn(-G, v[3]));
}
__device__ __forceinline__ float4 add_rn(float4 a, float4 b) {
  return make_float4(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z), __fadd_rn(a.w, b.w));
}

template <bool KAHAN>
struct NearAcc {
  float s[4] = {0.f, 0.f, 0.f, 0.f};
  float c[4] = {0.f, 0.f, 0.f, 0.f};
  __device__ __forceinline__ void add(int i, float v) {
    if (KAHAN) {
      const float y = v - c[i];
      const float t = s[i] + y;
      c[i] = (t - s[i]) - y;
      s[i] = t;
    } else {
      s[i] += v;
    }
  }
  __device__ __forceinline__ float value(int i) const { return KAHAN ? s[i] - c[i] : s[i]; }
};

#define JB_PAD4 make_float4(1e18f, 1e18f, 1e18f, 0.f)

// Packed FP32x2 arithmetic (sm_100 add/sub/mul/fma .f32x2): one instruction
// for two lanes of work, so the near-field loop handles two sources per step
// with half the issue slots of scalar code.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 f2(float lo, float hi) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_split(f32x2 v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 f2_sub(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 f2_add(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 f2_mul(f32x2 a, f32x2 b) {
  f32x2 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f32x2 f2_fma(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// The 32 sources of one chunk, staged per coordinate in the order the lane
// groups read them: source j sits at position (j % G) * (32 / G) + j / G, so
// group h's sources are one contiguous run and four of them load as one
// 16-byte vector that splits into two packed pairs with no register moves.
struct alignas(16) NearStage {
  float x[32], y[32], z[32], m[32];
  int r[32];  // block-step rung of each staged source (weighted form only)
};

template <int G>
__device__ __forceinline__ void stage_source(NearStage& s, int j, float4 v) {
  const int k = (j % G) * (32 / G) + j / G;
  s.x[k] = v.x;
  s.y[k] = v.y;
  s.z[k] = v.z;
  s.m[k] = v.w;
}

template <int G>
__device__ __forceinline__ void stage_rung(NearStage& s, int j, int r) {
  s.r[(j % G) * (32 / G) + j / G] = r;
}

// Level weights of the mutual lane's block-step form: a particle pair belongs
// to the level of its finer endpoint, max(rung_i, rung_j), and is scaled by
// that level's weight (rungs clamped to the table when staged).
struct PairWeights {
  const float* tbl;  // shared memory, one weight per level
  int rt;            // this lane's target rung
};

// One chunk of 32 staged sources for this lane's target: the lane's 32/G
// sources (j = q*G + h), two per packed step; the two partial sums are added
// at the end of the chunk (and into the compensated accumulator when KAHAN).
template <int G, bool KAHAN, bool POT, bool SELF, bool W = false, bool FTZ = false>
__device__ __forceinline__ void near_chunk(const NearStage& st, float4 ti, int h, int self_j, float eps2,
                                           NearAcc<KAHAN>& a, PairWeights pw = PairWeights{nullptr, 0}) {
  constexpr int R = 32 / G;
  const ulonglong2* X = reinterpret_cast<const ulonglong2*>(st.x + h * R);
  const ulonglong2* Y = reinterpret_cast<const ulonglong2*>(st.y + h * R);
  const ulonglong2* Z = reinterpret_cast<const ulonglong2*>(st.z + h * R);
  const ulonglong2* M = reinterpret_cast<const ulonglong2*>(st.m + h * R);
  const f32x2 TX = f2(ti.x, ti.x), TY = f2(ti.y, ti.y), TZ = f2(ti.z, ti.z), E2 = f2(eps2, eps2);
  f32x2 AX = f2(0.f, 0.f), AY = AX, AZ = AX, AW = AX;
  auto step = [&](f32x2 sx, f32x2 sy, f32x2 sz, f32x2 sm, int q) {
    const f32x2 dx = f2_sub(TX, sx);
    const f32x2 dy = f2_sub(TY, sy);
    const f32x2 dz = f2_sub(TZ, sz);
    const f32x2 d2 = f2_fma(dx, dx, f2_fma(dy, dy, f2_fma(dz, dz, E2)));
    float d2a, d2b;
    f2_split(d2, d2a, d2b);
    const f32x2 ir = FTZ ? f2(rsqrt_ftz(d2a), rsqrt_ftz(d2b)) : f2(rsqrtf(d2a), rsqrtf(d2b));
    f32x2 mir = f2_mul(sm, ir);
    f32x2 w = f2_mul(mir, f2_mul(ir, ir));
    if (W) {
      const int k0 = h * R + q;
      const f32x2 lw = f2(pw.tbl[max(pw.rt, st.r[k0])], pw.tbl[max(pw.rt, st.r[k0 + 1])]);
      mir = f2_mul(mir, lw);
      w = f2_mul(w, lw);
    }
    if (SELF) {
      const int j0 = q * G + h, j1 = j0 + G;
      float m0, m1, w0, w1;
      f2_split(mir, m0, m1);
      f2_split(w, w0, w1);
      m0 = (j0 == self_j) ? 0.f : m0;
      w0 = (j0 == self_j) ? 0.f : w0;
      m1 = (j1 == self_j) ? 0.f : m1;
      w1 = (j1 == self_j) ? 0.f : w1;
      mir = f2(m0, m1);
      w = f2(w0, w1);
    }
    AX = f2_fma(w, dx, AX);
    AY = f2_fma(w, dy, AY);
    AZ = f2_fma(w, dz, AZ);
    if (POT) AW = f2_add(AW, mir);
  };
#pragma unroll
  for (int v = 0; v < R / 4; ++v) {
    const ulonglong2 x = X[v], y = Y[v], z = Z[v], m = M[v];
    step(x.x, y.x, z.x, m.x, 4 * v);
    step(x.y, y.y, z.y, m.y, 4 * v + 2);
  }
  float x0, x1, y0, y1, z0, z1;
  f2_split(AX, x0, x1);
  f2_split(AY, y0, y1);
  f2_split(AZ, z0, z1);
  a.add(0, x0 + x1);
  a.add(1, y0 + y1);
  a.add(2, z0 + z1);
  if (POT) {
    float w0, w1;
    f2_split(AW, w0, w1);
    a.add(3, w0 + w1);
  }
}

// The targets rg (at most 32: the leaf, or one of its two halves) of the
// leaf whose particles are lr; row: where this pass's targets start in the
// leaf's partial row (0 or 32).
template <int G, bool KAHAN, bool POT, bool W, bool FTZ>
__device__ __forceinline__ void leaf_unit(const float4* __restrict__ pos4, int2 rg, int4 U, int2 aux,
                                          const int2* __restrict__ runs, NearStage& sP, int lane, float G_,
                                          float eps2, float4* __restrict__ out, float4* __restrict__ partial,
                                          int max_slots, int* err, const int* __restrict__ rung = nullptr,
                                          const float* tbl = nullptr, int nlw = 1, int2 lr = make_int2(0, -1),
                                          int row = 0) {
  if (lr.y < lr.x) lr = rg;
  const int tl = lane / G, h = lane % G;
  const int nt = rg.y - rg.x + 1;
  const bool active = tl < nt;
  const float4 ti = active ? pos4[rg.x + tl] : make_float4(0.f, 0.f, 0.f, 0.f);
  auto clamp_rung = [&](int r) { return min(max(r, 0), nlw - 1); };
  PairWeights pw{tbl, 0};
  if (W) pw.rt = active ? clamp_rung(rung[rg.x + tl]) : 0;
  NearAcc<KAHAN> a;
  if (aux.y & 1) {  // the self block: the leaf's particles in chunks of 32, the diagonal excluded
    for (int b = lr.x; b <= lr.y; b += 32) {
      const int j = b + lane;
      stage_source<G>(sP, lane, (j <= lr.y) ? pos4[j] : JB_PAD4);
      if (W) stage_rung<G>(sP, lane, (j <= lr.y) ? clamp_rung(rung[j]) : 0);
      __syncwarp();
      near_chunk<G, KAHAN, POT, true, W, FTZ>(sP, ti, h, rg.x + tl - b, eps2, a, pw);
      __syncwarp();
    }
  }
  const int nsrc = U.w;
  if (nsrc > 0) {
    int r = U.y, rbase = 0;
    int2 run = runs[r];
    auto fetch_index = [&](int f) -> int {  // particle of source f, -1 past the end
      while (f >= rbase + run.y && r + 1 < U.z) {
        rbase += run.y;
        ++r;
        run = runs[r];
      }
      return (f < nsrc) ? run.x + (f - rbase) : -1;
    };
    int qi = fetch_index(lane);
    float4 qn = qi >= 0 ? pos4[qi] : JB_PAD4;
    int qr = (W && qi >= 0) ? clamp_rung(rung[qi]) : 0;
    for (int base = 0; base < nsrc; base += 32) {
      stage_source<G>(sP, lane, qn);
      if (W) stage_rung<G>(sP, lane, qr);
      __syncwarp();
      if (base + 32 < nsrc) {
        qi = fetch_index(base + 32 + lane);
        qn = qi >= 0 ? pos4[qi] : JB_PAD4;
        if (W) qr = qi >= 0 ? clamp_rung(rung[qi]) : 0;
      }
      near_chunk<G, KAHAN, POT, false, W, FTZ>(sP, ti, h, -1, eps2, a, pw);
      __syncwarp();
    }
  }
  float v[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    v[i] = (POT || i < 3) ? a.value(i) : 0.f;
    if (G >= 2) v[i] += __shfl_xor_sync(0xffffffffu, v[i], 1);
    if (G >= 4) v[i] += __shfl_xor_sync(0xffffffffu, v[i], 2);
  }
  const float4 res = near_scaled(G_, v);
  if (active && h == 0) {
    if (aux.x < 0) {
      const float4 f = out[rg.x + tl];  // the far field k_leaf_l2p wrote
      out[rg.x + tl] = add_rn(f, res);
    } else if (aux.x < max_slots) {
      partial[(size_t)aux.x * kMaxLeaf + row + tl] = res;
    } else {
      leaf_error(err, JB_LEAF_ERR_SLOT);
    }
  }
}

// Near field (P2P) of the work units, added to the far field already in out
// (whole leaves) or written to the partial rows (split leaves).
//
// W: the block-step weighted form of the mutual lane -- every pair scaled by
// lw[max(rung_i, rung_j)] (rung: per sorted particle, lw: nlw <= 32 weights).
// FTZ: 1/r from rsqrt_ftz (the pass's forms all use it; false gives rsqrtf).
template <bool KAHAN, bool POT, bool W = false, bool FTZ = true>
static __global__ void __launch_bounds__(32 * kWarpsPerBlock, POT ? 6 : 8) k_leaf_units(
    const float4* __restrict__ pos4, int num_internal, int num_units, const int4* __restrict__ units,
    const int2* __restrict__ aux, const int2* __restrict__ runs, const int2* __restrict__ ranges, float G,
    float eps2, float4* __restrict__ out, float4* __restrict__ partial, int max_slots, int* err,
    const int* __restrict__ rung = nullptr, const float* __restrict__ lw = nullptr, int nlw = 1) {
  __shared__ NearStage sP[kWarpsPerBlock];
  __shared__ float tbl[32];
  if (W) {
    if (threadIdx.x < 32) tbl[threadIdx.x] = threadIdx.x < (unsigned)nlw ? lw[threadIdx.x] : 0.f;
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int u = blockIdx.x * kWarpsPerBlock + warp;
  if (u >= num_units) return;
  const int4 U = units[u];
  const int2 ax = aux[u];
  const int2 rg = ranges[num_internal + U.x];
  const int ntl = rg.y - rg.x + 1;
  if (ntl > kMaxLeaf) {
    if (lane == 0) leaf_error(err, JB_LEAF_ERR_OCCUPANCY);
    return;
  }
  for (int row = 0; row < ntl; row += 32) {  // a leaf of more than 32 particles in two passes
    const int2 rt = make_int2(rg.x + row, min(rg.y, rg.x + row + 31));
    const int nt = rt.y - rt.x + 1;
    if (row > 0) __syncwarp();  // the first pass's reads of the stage are done
    if (nt <= 8)
      leaf_unit<4, KAHAN, POT, W, FTZ>(pos4, rt, U, ax, runs, sP[warp], lane, G, eps2, out, partial, max_slots, err,
                                       rung, tbl, nlw, rg, row);
    else if (nt <= 16)
      leaf_unit<2, KAHAN, POT, W, FTZ>(pos4, rt, U, ax, runs, sP[warp], lane, G, eps2, out, partial, max_slots, err,
                                       rung, tbl, nlw, rg, row);
    else
      leaf_unit<1, KAHAN, POT, W, FTZ>(pos4, rt, U, ax, runs, sP[warp], lane, G, eps2, out, partial, max_slots, err,
                                       rung, tbl, nlw, rg, row);
  }
}

// ---------------------------------------------------------------------------
// Near field with every lane busy, for leaves of 17..32 particles.
//
// One lane per target leaves 32 - nt lanes idle.  Here a unit's work, nt
// targets x C source chunks of kFlatChunk (64), is walked chunk-major: item
// f = c * nt + t, 32 items per warp step, lane l of step s takes item 32 s + l
// (target f mod nt against chunk f / nt).  A step spans at most three
// consecutive chunks (nt >= 17), so the chunks sit in a ring of four
// shared-memory slots, padded so that the slots one load instruction reads
// fall in different banks.  Each chunk is copied into its slot by cp.async
// (four 4-byte copies per source: the ring is one array per coordinate, so
// that a 16-byte load yields two packed source pairs), one chunk ahead of the
// chunks the step reads, so no register holds a source in flight.  The
// per-target sums live in shared memory: lane l < nt owns its item's target
// and, when lane l + nt holds the same target's next chunk, adds that partial
// straight after its own, so every target receives its chunk partials in
// chunk order through one (compensated) add per 64 sources.
// ---------------------------------------------------------------------------
constexpr int kFlatChunk = 64;                // sources per chunk (item)
constexpr int kFlatSlot = kFlatChunk + 4;     // slot stride (floats): the three slots one load reads use distinct banks
struct alignas(16) FlatStage {
  float x[4][kFlatSlot], y[4][kFlatSlot], z[4][kFlatSlot], m[4][kFlatSlot];  // source chunk ring
  float4 tp[32];                                                            // target positions
  float4 s[32], c[32];                                                      // per-target sums and compensations
};

union WarpStage {
  NearStage n;
  FlatStage f;
};

__device__ __forceinline__ void cp_async4(float* smem_dst, const float* gmem_src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Sums of one chunk of NS sources for one target, the arithmetic of
// near_chunk with one lane per target (packed pairs j, j + 1; the two halves
// added at the end).
template <bool POT, bool SELF, int NS = 32>
__device__ __forceinline__ float4 chunk_sums(const float* xs, const float* ys, const float* zs, const float* ms,
                                             float4 ti, int self_j, float eps2) {
  const ulonglong2* X = reinterpret_cast<const ulonglong2*>(xs);
  const ulonglong2* Y = reinterpret_cast<const ulonglong2*>(ys);
  const ulonglong2* Z = reinterpret_cast<const ulonglong2*>(zs);
  const ulonglong2* M = reinterpret_cast<const ulonglong2*>(ms);
  const f32x2 TX = f2(ti.x, ti.x), TY = f2(ti.y, ti.y), TZ = f2(ti.z, ti.z), E2 = f2(eps2, eps2);
  f32x2 AX = f2(0.f, 0.f), AY = AX, AZ = AX, AW = AX;
  auto step = [&](f32x2 sx, f32x2 sy, f32x2 sz, f32x2 sm, int j0) {
    const f32x2 dx = f2_sub(TX, sx);
    const f32x2 dy = f2_sub(TY, sy);
    const f32x2 dz = f2_sub(TZ, sz);
    const f32x2 d2 = f2_fma(dx, dx, f2_fma(dy, dy, f2_fma(dz, dz, E2)));
    float d2a, d2b;
    f2_split(d2, d2a, d2b);
    const f32x2 ir = f2(rsqrt_ftz(d2a), rsqrt_ftz(d2b));
    f32x2 mir = f2_mul(sm, ir);
    f32x2 w = f2_mul(mir, f2_mul(ir, ir));
    if (SELF) {
      float m0, m1, w0, w1;
      f2_split(mir, m0, m1);
      f2_split(w, w0, w1);
      m0 = (j0 == self_j) ? 0.f : m0;
      w0 = (j0 == self_j) ? 0.f : w0;
      m1 = (j0 + 1 == self_j) ? 0.f : m1;
      w1 = (j0 + 1 == self_j) ? 0.f : w1;
      mir = f2(m0, m1);
      w = f2(w0, w1);
    }
    AX = f2_fma(w, dx, AX);
    AY = f2_fma(w, dy, AY);
    AZ = f2_fma(w, dz, AZ);
    if (POT) AW = f2_add(AW, mir);
  };
#pragma unroll
  for (int v = 0; v < NS / 4; ++v) {
    const ulonglong2 x = X[v], y = Y[v], z = Z[v], m = M[v];
    step(x.x, y.x, z.x, m.x, 4 * v);
    step(x.y, y.y, z.y, m.y, 4 * v + 2);
  }
  float x0, x1, y0, y1, z0, z1, w0 = 0.f, w1 = 0.f;
  f2_split(AX, x0, x1);
  f2_split(AY, y0, y1);
  f2_split(AZ, z0, z1);
  if (POT) f2_split(AW, w0, w1);
  return make_float4(x0 + x1, y0 + y1, z0 + z1, POT ? w0 + w1 : 0.f);
}

// Adds one chunk's sums into target t's accumulator in shared memory.
template <bool KAHAN, bool POT>
__device__ __forceinline__ void flat_add(FlatStage& S, int t, float4 v) {
  NearAcc<KAHAN> a;
  const float4 s = S.s[t];
  a.s[0] = s.x, a.s[1] = s.y, a.s[2] = s.z, a.s[3] = s.w;
  if (KAHAN) {
    const float4 c = S.c[t];
    a.c[0] = c.x, a.c[1] = c.y, a.c[2] = c.z, a.c[3] = c.w;
  }
  a.add(0, v.x);
  a.add(1, v.y);
  a.add(2, v.z);
  if (POT) a.add(3, v.w);
  S.s[t] = make_float4(a.s[0], a.s[1], a.s[2], a.s[3]);
  if (KAHAN) S.c[t] = make_float4(a.c[0], a.c[1], a.c[2], a.c[3]);
}

template <bool KAHAN, bool POT>
__device__ __forceinline__ void leaf_unit_flat(const float4* __restrict__ pos4, int2 rg, int4 U, int2 aux,
                                               const int2* __restrict__ runs, FlatStage& S, int lane, float G_,
                                               float eps2, float4* __restrict__ out, float4* __restrict__ partial,
                                               int max_slots, int* err, int2 lr, int row) {
  constexpr int CH = kFlatChunk;
  const int nt = rg.y - rg.x + 1;  // 17..32 targets (the leaf lr, or one of its halves)
  const bool tgt = lane < nt;
  const float4 me = tgt ? pos4[rg.x + lane] : JB_PAD4;
  S.tp[lane] = me;
  S.s[lane] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (KAHAN) S.c[lane] = make_float4(0.f, 0.f, 0.f, 0.f);
  if (aux.y & 1) {  // the self block: the leaf's particles in chunks of 32, the diagonal excluded
    const float4 ti = tgt ? me : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int b = lr.x; b <= lr.y; b += 32) {
      const float4 q = (b + lane <= lr.y) ? pos4[b + lane] : JB_PAD4;
      __syncwarp();  // the previous chunk's reads are done
      S.x[0][lane] = q.x;
      S.y[0][lane] = q.y;
      S.z[0][lane] = q.z;
      S.m[0][lane] = q.w;
      __syncwarp();
      const float4 v = chunk_sums<POT, true>(S.x[0], S.y[0], S.z[0], S.m[0], ti, rg.x + lane - b, eps2);
      if (tgt) flat_add<KAHAN, POT>(S, lane, v);
    }
  }
  const int nsrc = U.w;
  if (nsrc > 0) {
    const int C = (nsrc + CH - 1) / CH;
    const int total = nt * C;
    int r = U.y, rbase = 0;
    int2 run = runs[r];
    // copies source f of the unit (padding past the end) into position q of
    // ring slot sl; a lane's f only grow, so its run cursor only advances
    auto stage_src = [&](int f, int sl, int q) {
      while (f >= rbase + run.y && r + 1 < U.z) {
        rbase += run.y;
        ++r;
        run = runs[r];
      }
      if (f < nsrc) {
        const float* src = reinterpret_cast<const float*>(pos4 + run.x + (f - rbase));
        cp_async4(&S.x[sl][q], src);
        cp_async4(&S.y[sl][q], src + 1);
        cp_async4(&S.z[sl][q], src + 2);
        cp_async4(&S.m[sl][q], src + 3);
      } else {
        S.x[sl][q] = 1e18f;
        S.y[sl][q] = 1e18f;
        S.z[sl][q] = 1e18f;
        S.m[sl][q] = 0.f;
      }
    };
    auto stage_chunk = [&](int k) {  // one cp.async group per chunk
      const int sl = k & 3;
      stage_src(k * CH + lane, sl, lane);
      stage_src(k * CH + 32 + lane, sl, 32 + lane);
      cp_async_commit();
    };
    int staged = 0;
    int c = (lane >= nt) ? 1 : 0, t = lane - c * nt;  // item f = lane
    __syncwarp();  // the self block's reads of slot 0 are done
    for (int base = 0; base < total; base += 32) {
      const int chi = min(__shfl_sync(0xffffffffu, c, 31), C - 1);
      __syncwarp();  // the previous step's reads and adds are done
      // chunks up to chi are needed now; chi + 1 is copied ahead.  The slot
      // of chunk k held chunk k - 4 <= chi - 3, older than any chunk a step
      // spanning at most three chunks reads.
      const int want = min(chi + 1, C - 1);
      while (staged <= want) stage_chunk(staged++);
      if (staged - 1 > chi)
        cp_async_wait_one();  // all but the chunk copied ahead
      else
        cp_async_wait_all();
      __syncwarp();
      const int sl = c & 3;
      const float4 v = chunk_sums<POT, false, CH>(S.x[sl], S.y[sl], S.z[sl], S.m[sl], S.tp[t], -1, eps2);
      float4 v2;
      v2.x = __shfl_down_sync(0xffffffffu, v.x, nt);
      v2.y = __shfl_down_sync(0xffffffffu, v.y, nt);
      v2.z = __shfl_down_sync(0xffffffffu, v.z, nt);
      v2.w = POT ? __shfl_down_sync(0xffffffffu, v.w, nt) : 0.f;
      if (tgt && base + lane < total) {
        NearAcc<KAHAN> a;  // one read and one write of the target's sums for both adds
        const float4 s0 = S.s[t];
        a.s[0] = s0.x, a.s[1] = s0.y, a.s[2] = s0.z, a.s[3] = s0.w;
        if (KAHAN) {
          const float4 c0 = S.c[t];
          a.c[0] = c0.x, a.c[1] = c0.y, a.c[2] = c0.z, a.c[3] = c0.w;
        }
        a.add(0, v.x);
        a.add(1, v.y);
        a.add(2, v.z);
        if (POT) a.add(3, v.w);
        if (lane + nt < 32 && base + lane + nt < total) {  // lane + nt holds (t, c + 1)
          a.add(0, v2.x);
          a.add(1, v2.y);
          a.add(2, v2.z);
          if (POT) a.add(3, v2.w);
        }
        S.s[t] = make_float4(a.s[0], a.s[1], a.s[2], a.s[3]);
        if (KAHAN) S.c[t] = make_float4(a.c[0], a.c[1], a.c[2], a.c[3]);
      }
      t += 32 - nt;  // item f + 32
      c += 1;
      if (t >= nt) {
        t -= nt;
        c += 1;
      }
    }
    cp_async_wait_all();  // nothing left in flight (the ring is reused by the next unit)
  }
  __syncwarp();
  if (tgt) {
    NearAcc<KAHAN> a;
    const float4 s = S.s[lane];
    a.s[0] = s.x, a.s[1] = s.y, a.s[2] = s.z, a.s[3] = s.w;
    if (KAHAN) {
      const float4 cc = S.c[lane];
      a.c[0] = cc.x, a.c[1] = cc.y, a.c[2] = cc.z, a.c[3] = cc.w;
    }
    float v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = (POT || i < 3) ? a.value(i) : 0.f;
    const float4 res = near_scaled(G_, v);
    if (aux.x < 0) {
      const float4 f = out[rg.x + lane];  // the far field k_leaf_l2p wrote
      out[rg.x + lane] = add_rn(f, res);
    } else if (aux.x < max_slots) {
      partial[(size_t)aux.x * kMaxLeaf + row + lane] = res;
    } else {
      leaf_error(err, JB_LEAF_ERR_SLOT);
    }
  }
}

// k_leaf_units with the chunk-major form for leaves of more than 16
// particles (the lane-group forms below that) and rsqrt_ftz.  Same results
// for squared distances in the normal FP32 range.
template <bool KAHAN, bool POT>
static __global__ void __launch_bounds__(32 * kWarpsPerBlock, POT ? 6 : 8) k_leaf_units_flat(
    const float4* __restrict__ pos4, int num_internal, int num_units, const int4* __restrict__ units,
    const int2* __restrict__ aux, const int2* __restrict__ runs, const int2* __restrict__ ranges, float G,
    float eps2, float4* __restrict__ out, float4* __restrict__ partial, int max_slots, int* err) {
  __shared__ WarpStage sW[kWarpsPerBlock];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int u = blockIdx.x * kWarpsPerBlock + warp;
  if (u >= num_units) return;
  const int4 U = units[u];
  const int2 ax = aux[u];
  const int2 rg = ranges[num_internal + U.x];
  const int ntl = rg.y - rg.x + 1;
  if (ntl > kMaxLeaf) {
    if (lane == 0) leaf_error(err, JB_LEAF_ERR_OCCUPANCY);
    return;
  }
  for (int row = 0; row < ntl; row += 32) {  // a leaf of more than 32 particles in two passes
    const int2 rt = make_int2(rg.x + row, min(rg.y, rg.x + row + 31));
    const int nt = rt.y - rt.x + 1;
    if (row > 0) __syncwarp();  // the first pass's reads of the stage are done
    if (nt <= 8)
      leaf_unit<4, KAHAN, POT, false, true>(pos4, rt, U, ax, runs, sW[warp].n, lane, G, eps2, out, partial,
                                            max_slots, err, nullptr, nullptr, 1, rg, row);
    else if (nt <= 16)
      leaf_unit<2, KAHAN, POT, false, true>(pos4, rt, U, ax, runs, sW[warp].n, lane, G, eps2, out, partial,
                                            max_slots, err, nullptr, nullptr, 1, rg, row);
    else
      leaf_unit_flat<KAHAN, POT>(pos4, rt, U, ax, runs, sW[warp].f, lane, G, eps2, out, partial, max_slots, err, rg,
                                 row);
  }
}

// Far field (L2P) of every leaf: warp per leaf (its unit with flags & 1),
// lane per particle, the local expansion staged in shared memory.  Writes
// out = -G (grad phi, phi); runs before k_leaf_units, which adds the near
// field.  Kept out of the near-field kernel so that kernel's register count
// is set by the P2P loop alone (about half, and twice the resident warps).
// mode kL2PZero: write zeros instead (the near field alone, JB_P2P_NEAR_ONLY
// and JB_P2P_NEAR_FIRST); kL2PAdd: add the far field to what out holds (the
// near field a JB_P2P_NEAR_FIRST launch wrote), with the rounding of the
// near-field kernel's own add.
enum { kL2PWrite = 0, kL2PZero = 1, kL2PAdd = 2 };
template <int P>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_leaf_l2p(
    const float4* __restrict__ pos4, int num_internal, int num_units, const int4* __restrict__ units,
    const int2* __restrict__ aux, const int2* __restrict__ ranges, const float4* __restrict__ centers,
    const float* __restrict__ locals, float G, float4* __restrict__ out, int mode) {
  constexpr int C = csize(P), CS = cstride(P);
  __shared__ float sF[kWarpsPerBlock][CS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int u = blockIdx.x * kWarpsPerBlock + warp;
  if (u >= num_units || !(aux[u].y & 1)) return;
  const int node = num_internal + units[u].x;
  const int2 rg = ranges[node];
  if (rg.y - rg.x + 1 > kMaxLeaf) return;  // refused by the near-field kernel, which flags it
  if (mode == kL2PZero) {  // near field alone: the sums start from zero
    for (int i = rg.x + lane; i <= rg.y; i += 32) out[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    return;
  }
  // the first particle and the centre are fetched alongside the local's staging
  const float4 c = centers[node];
  const float4 t0 = (rg.x + lane <= rg.y) ? pos4[rg.x + lane] : c;
  for (int k = lane; k < CS; k += 32) sF[warp][k] = locals[(size_t)node * CS + k];
  __syncwarp();
  for (int i = rg.x + lane; i <= rg.y; i += 32) {  // two rounds for a leaf of more than 32
    const float4 ti = (i == rg.x + lane) ? t0 : pos4[i];
    float U_[C];
    solid_harmonics<P>(c.x - ti.x, c.y - ti.y, c.z - ti.z, U_);
    float phi, g[3];
    l2p_eval<P>(SmemF{sF[warp]}, U_, &phi, g);
    const float4 f = make_float4(__fmul_rn(-G, g[0]), __fmul_rn(-G, g[1]), __fmul_rn(-G, g[2]), __fmul_rn(-G, phi));
    out[i] = mode == kL2PAdd ? add_rn(f, out[i]) : f;
  }
}

// Sums the partial results of leaves whose work was split: split[i] = (leaf,
// first slot, number of slots, unused).  Thread per (leaf, particle slot).
// ACCUM: the sum starts from what out holds (the far field), else from zero.
template <bool ACCUM>
static __global__ void __launch_bounds__(256) k_leaf_reduce(int num_split, const int4* __restrict__ split, int num_internal,
                                                     const int2* __restrict__ ranges, const float4* __restrict__ partial,
                                                     float4* __restrict__ out, int max_slots, int* err) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(t / kMaxLeaf), l = (int)(t % kMaxLeaf);
  if (i >= num_split) return;
  const int4 sp = split[i];
  const int2 rg = ranges[num_internal + sp.x];
  if (rg.y - rg.x + 1 > kMaxLeaf) return;  // flagged by the near-field kernel
  if (sp.y < 0 || sp.z < 0 || (int64_t)sp.y + sp.z > max_slots) {
    if (l == 0) leaf_error(err, JB_LEAF_ERR_SLOT);
    return;
  }
  if (rg.x + l > rg.y) return;
  float4 a = ACCUM ? out[rg.x + l] : make_float4(0.f, 0.f, 0.f, 0.f);
  for (int q = 0; q < sp.z; ++q) {
    const float4 v = partial[(size_t)(sp.y + q) * kMaxLeaf + l];
    a.x += v.x;
    a.y += v.y;
    a.z += v.z;
    a.w += v.w;
  }
  out[rg.x + l] = a;
}

// ---------------------------------------------------------------------------
// Target subset: warp per target, lane per source leaf.
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
  // lane k takes the k-th source leaf of each group of 32 (the target's own
  // leaf first) and runs through its particles: the leaves' range lookups
  // overlap instead of following one another
  const int64_t e0 = near_off[leaf], e1 = near_off[leaf + 1];
  for (int64_t eb = e0 - 1; eb < e1; eb += 32) {
    const int64_t e = eb + lane;
    if (e >= e1) continue;
    const int2 sr = (e < e0) ? ranges[node] : ranges[num_internal + near_src[e]];
    for (int j = sr.x; j <= sr.y; ++j) {
      const float4 s = pos4[j];
      const float dx = ti.x - s.x, dy = ti.y - s.y, dz = ti.z - s.z;
      const float d2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
      const float ir = rsqrt_ftz(d2);
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
  static int run(int first, int last, const int* left, const int* right, const int* ranges, float* centers,
                 float* mult, cudaStream_t st) {
    if (last <= first) return JB_OK;
    if (last - first <= g_split_max_parents[0]) {
      k_m2m_level_split<P><<<blocks_for(2 * (int64_t)(last - first), kSplitItems), 128, 0, st>>>(
          first, last, left, right, reinterpret_cast<const int2*>(ranges), reinterpret_cast<float4*>(centers), mult);
    } else {
      k_m2m_level<P><<<blocks_for(2 * (int64_t)(last - first), 128), 128, 0, st>>>(
          first, last, left, right, reinterpret_cast<const int2*>(ranges), reinterpret_cast<float4*>(centers), mult);
    }
    return launch_status();
  }
};

template <int P>
struct RunM2L {
  static int run(int num_units, const int* units, const float* mult, const float* centers, const int* far_src,
                 float* locals, float* partials, int num_split, const int* split, cudaStream_t st, bool neg = false,
                 int rs = 0, const float* far_w = nullptr) {
    if (rs <= 0) rs = cstride(P);
    if (num_units > 0) {
      const bool coop = g_m2l_coop != 0;
      const size_t sm = sizeof(float4) * kM2LThreads * row4(P) + (coop ? sizeof(int) * kM2LThreads : 0);
      auto kern = coop ? (far_w ? k_m2l_units_coop<P, false, true>
                                : (neg ? k_m2l_units_coop<P, true> : k_m2l_units_coop<P, false>))
                       : (far_w ? k_m2l_units<P, false, true> : (neg ? k_m2l_units<P, true> : k_m2l_units<P, false>));
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      kern<<<blocks_for(num_units, kM2LThreads), kM2LThreads, sm, st>>>(
          num_units, reinterpret_cast<const int4*>(units), mult, reinterpret_cast<const float4*>(centers), far_src,
          locals, partials, rs, far_w);
      const int rc = launch_status();
      if (rc) return rc;
    }
    if (num_split > 0) {
      k_m2l_reduce<<<blocks_for((int64_t)num_split * rs, 256), 256, 0, st>>>(
          num_split, reinterpret_cast<const int4*>(split), partials, locals, rs);
      return launch_status();
    }
    return JB_OK;
  }
};

template <int P>
struct RunM2LMixed {
  static int run(int num_units, const int* units, const int* bounds, const float* mult, const float* centers,
                 const int* far_src, float* locals, float* partials, int num_split, const int* split, cudaStream_t st) {
    const int rs = cstride(P);
    if (num_units > 0) {
      const size_t sm = sizeof(float4) * kM2LThreads * row4(P);
      cudaFuncSetAttribute(k_m2l_mixed<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      k_m2l_mixed<P><<<blocks_for(num_units, kM2LThreads), kM2LThreads, sm, st>>>(
          num_units, reinterpret_cast<const int4*>(units), reinterpret_cast<const int4*>(bounds), mult,
          reinterpret_cast<const float4*>(centers), far_src, locals, partials, rs);
      const int rc = launch_status();
      if (rc) return rc;
    }
    if (num_split > 0) {
      k_m2l_reduce<<<blocks_for((int64_t)num_split * rs, 256), 256, 0, st>>>(
          num_split, reinterpret_cast<const int4*>(split), partials, locals, rs);
      return launch_status();
    }
    return JB_OK;
  }
};

template <int P>
struct RunL2L {
  static int run(int first, int last, const int* left, const int* right, const float* centers, float* locals,
                 cudaStream_t st) {
    if (last <= first) return JB_OK;
    if (last - first <= g_split_max_parents[1]) {
      k_l2l_level_split<P><<<blocks_for(2 * (int64_t)(last - first), kSplitItems), 128, 0, st>>>(
          first, last, left, right, reinterpret_cast<const float4*>(centers), locals);
    } else {
      k_l2l_level<P><<<blocks_for(2 * (int64_t)(last - first), 128), 128, 0, st>>>(
          first, last, left, right, reinterpret_cast<const float4*>(centers), locals);
    }
    return launch_status();
  }
};

template <int P>
struct RunL2LLeaves {
  static int run(int num_units, const int* units, const int* anc, const float* centers, float* locals,
                 cudaStream_t st) {
    if (num_units <= 0) return JB_OK;
    const size_t sm = sizeof(float4) * kM2LThreads * row4(P) + sizeof(int) * kM2LThreads;
    cudaFuncSetAttribute(k_l2l_leaves<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_l2l_leaves<P><<<blocks_for(num_units, kM2LThreads), kM2LThreads, sm, st>>>(
        num_units, reinterpret_cast<const int4*>(units), anc, reinterpret_cast<const float4*>(centers), locals);
    return launch_status();
  }
};

template <int P>
struct RunLeafEval {
  template <bool K, bool PT>
  static void go(unsigned nb, cudaStream_t st, const float4* pos4, int num_internal, int num_units, const int4* units,
                 const int2* aux, const int2* runs, const int2* ranges, float G, float eps2, float4* out,
                 float4* partial, const int* rung, const float* lw, int nlw, bool flat, int max_slots, int* err) {
    if (rung)
      k_leaf_units<K, PT, true><<<nb, 32 * kWarpsPerBlock, 0, st>>>(pos4, num_internal, num_units, units, aux, runs,
                                                                    ranges, G, eps2, out, partial, max_slots, err,
                                                                    rung, lw, nlw);
    else if (flat) {
      // 23.5 KB of shared memory per block: ask for the carveout that holds
      // the eight blocks per SM the launch bounds allow.
      static const cudaError_t carve = cudaFuncSetAttribute(
          k_leaf_units_flat<K, PT>, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
      (void)carve;
      k_leaf_units_flat<K, PT><<<nb, 32 * kWarpsPerBlock, 0, st>>>(pos4, num_internal, num_units, units, aux, runs,
                                                                   ranges, G, eps2, out, partial, max_slots, err);
    }
    else
      k_leaf_units<K, PT><<<nb, 32 * kWarpsPerBlock, 0, st>>>(pos4, num_internal, num_units, units, aux, runs, ranges,
                                                              G, eps2, out, partial, max_slots, err);
  }
  static int run(int mode, const float* pos4, int num_internal, int num_units, const int* units, const int* aux,
                 const int* runs, const int* ranges, const float* centers, const float* locals, float G, float eps2,
                 float* out, float* partial, int num_split, const int* split, cudaStream_t st,
                 const int* rung = nullptr, const float* lw = nullptr, int nlw = 1, bool flat = false,
                 int max_slots = 0x7fffffff, int* err = nullptr) {
    if (num_units > 0) {
      const unsigned nb = blocks_for(num_units, kWarpsPerBlock);
      auto a0 = reinterpret_cast<const float4*>(pos4);
      auto a1 = reinterpret_cast<const int4*>(units);
      auto a2 = reinterpret_cast<const int2*>(aux);
      auto a3 = reinterpret_cast<const int2*>(runs);
      auto a4 = reinterpret_cast<const int2*>(ranges);
      auto o = reinterpret_cast<float4*>(out);
      auto pt = reinterpret_cast<float4*>(partial);
      const bool far_only = (mode & JB_P2P_FAR_ONLY) != 0, far_after = (mode & JB_P2P_FAR_AFTER) != 0;
      const bool zero = (mode & (JB_P2P_NEAR_ONLY | JB_P2P_NEAR_FIRST)) != 0;
      k_leaf_l2p<P><<<nb, 32 * kWarpsPerBlock, 0, st>>>(a0, num_internal, num_units, a1, a2, a4,
                                                        reinterpret_cast<const float4*>(centers), locals, G, o,
                                                        zero ? kL2PZero : far_after ? kL2PAdd : kL2PWrite);
      int rc = launch_status();
      if (rc) return rc;
      if (far_only) return JB_OK;
      if (!far_after) {  // FAR_AFTER: the near field is already in out (and partials)
        const bool kahan = (mode & JB_P2P_KAHAN) != 0, pot = (mode & JB_P2P_POTENTIAL) != 0;
        if (kahan && pot) go<true, true>(nb, st, a0, num_internal, num_units, a1, a2, a3, a4, G, eps2, o, pt, rung, lw, nlw, flat, max_slots, err);
        else if (kahan) go<true, false>(nb, st, a0, num_internal, num_units, a1, a2, a3, a4, G, eps2, o, pt, rung, lw, nlw, flat, max_slots, err);
        else if (pot) go<false, true>(nb, st, a0, num_internal, num_units, a1, a2, a3, a4, G, eps2, o, pt, rung, lw, nlw, flat, max_slots, err);
        else go<false, false>(nb, st, a0, num_internal, num_units, a1, a2, a3, a4, G, eps2, o, pt, rung, lw, nlw, flat, max_slots, err);
        rc = launch_status();
        if (rc) return rc;
      }
    }
    if (num_split > 0 && !(mode & JB_P2P_NEAR_FIRST)) {  // NEAR_FIRST: summed by the FAR_AFTER call
      k_leaf_reduce<true><<<blocks_for((int64_t)num_split * kMaxLeaf, 256), 256, 0, st>>>(
          num_split, reinterpret_cast<const int4*>(split), num_internal, reinterpret_cast<const int2*>(ranges),
          reinterpret_cast<const float4*>(partial), reinterpret_cast<float4*>(out), max_slots, err);
      return launch_status();
    }
    return JB_OK;
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
  extern template struct jb::RunM2LMixed<PP>; \
  extern template struct jb::RunL2L<PP>;      \
  extern template struct jb::RunL2LLeaves<PP>; \
  extern template struct jb::RunLeafEval<PP>; \
  extern template struct jb::RunTargets<PP>;  \
  JB_DECLARE_ADJ_##PP

// The adjoint needs the order p+1 M2L, so it is built for p <= 9.
#define JB_DECLARE_ADJ_1 extern template struct jb::RunAdj<1>;
#define JB_DECLARE_ADJ_2 extern template struct jb::RunAdj<2>;
#define JB_DECLARE_ADJ_3 extern template struct jb::RunAdj<3>;
#define JB_DECLARE_ADJ_4 extern template struct jb::RunAdj<4>;
#define JB_DECLARE_ADJ_5 extern template struct jb::RunAdj<5>;
#define JB_DECLARE_ADJ_6 extern template struct jb::RunAdj<6>;
#define JB_DECLARE_ADJ_7 extern template struct jb::RunAdj<7>;
#define JB_DECLARE_ADJ_8 extern template struct jb::RunAdj<8>;
#define JB_DECLARE_ADJ_9 extern template struct jb::RunAdj<9>;
#define JB_DECLARE_ADJ_10
#define JB_ADJ_MAX_ORDER 9
