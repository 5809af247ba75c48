// Device prepare: the tree and the interaction lists of tree_build.cpp, built
// on the GPU from device arrays, bit for bit the same arrays.
//
// Same algorithm as the host stand-in for yggdrax (tree_build.cpp; used where
// jaccpot calls yggdrax at runtime/fmm_prepare.py:823 and :1411):
//   1. bounding cube, 63-bit Morton codes (21 bits per axis), stable sort of
//      (code, input index)                       -> k_bbox_*, k_morton, radix sort;
//   2. breadth-first radix split: a range of more than leaf_size particles is
//      split at the highest differing code bit (duplicates at the midpoint);
//      internal ids in BFS order, leaves renumbered in particle order
//                                                -> one k_level_* pair per level;
//   3. FP64 COM and bounding radius, leaves from their particles, internal
//      nodes from their children, deepest level first -> k_leaf_com, k_internal_com;
//   4. dual walk from (root, root): (A, A) opens into its children's three
//      pairs; (A, B) is far when d^2 > 0 and (r_A + r_B)^2 <= theta^2 d^2,
//      near when both are leaves, else the larger-radius internal node is
//      split; far and near pairs are emitted in both directions
//                                                -> breadth-first k_walk_*;
//   5. target-major CSR with sources ascending   -> key radix sort + row counts.
// The walk visits the same pairs as the host's depth-first recursion (every
// decision depends on the pair alone); sorting the emitted pairs gives the
// host's CSR order.  The floating-point steps are the host's, operation for
// operation, and this file is compiled with -fmad=false so no multiply-add is
// contracted: the COM, radii and MAC decisions are the host's to the last bit.
//
// Work decomposition: thread per particle / range / node / pair; prefix sums
// by a three-kernel tile scan; the sort is an LSD radix sort with 8-bit digits
// whose scatter ranks keys by warp match masks in index order (stable).  The
// only atomics are shared-memory digit counts, row counts and a max, all
// order-independent, so every output is run-to-run identical.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/jaccpot_b200.h"

#include "dev_prims.cuh"

namespace jbdev {

cudaError_t pool(cudaMemPool_t* out) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[dev]) {
    cudaMemPoolProps pr = {};
    pr.allocType = cudaMemAllocationTypePinned;
    pr.handleTypes = cudaMemHandleTypeNone;
    pr.location.type = cudaMemLocationTypeDevice;
    pr.location.id = dev;
    e = cudaMemPoolCreate(&pools[dev], &pr);
    if (e != cudaSuccess) return e;
    uint64_t keep = 4ull << 30;
    e = cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
  }
  *out = pools[dev];
  return cudaSuccess;
}

}  // namespace jbdev

namespace {

// ---------------------------------------------------------------------------
// 1. Morton codes.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_bbox_partial(const double* __restrict__ pos, int64_t n, double* __restrict__ part) {
  __shared__ double sm[6][256];
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    for (int k = 0; k < 3; ++k) {
      const double x = pos[3 * i + k];
      lo[k] = fmin(lo[k], x);
      hi[k] = fmax(hi[k], x);
    }
  for (int k = 0; k < 3; ++k) {
    sm[k][threadIdx.x] = lo[k];
    sm[3 + k][threadIdx.x] = hi[k];
  }
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < 3; ++k) {
        sm[k][threadIdx.x] = fmin(sm[k][threadIdx.x], sm[k][threadIdx.x + w]);
        sm[3 + k][threadIdx.x] = fmax(sm[3 + k][threadIdx.x], sm[3 + k][threadIdx.x + w]);
      }
    __syncthreads();
  }
  if (threadIdx.x < 6) part[6 * blockIdx.x + threadIdx.x] = sm[threadIdx.x][0];
}

__global__ void k_bbox_final(const double* __restrict__ part, int nblk, double* __restrict__ bb) {
  if (threadIdx.x >= 6) return;
  const int k = threadIdx.x;
  double v = part[k];
  for (int b = 1; b < nblk; ++b) v = (k < 3) ? fmin(v, part[6 * b + k]) : fmax(v, part[6 * b + k]);
  bb[k] = v;
}

__device__ __forceinline__ uint64_t spread21(uint64_t v) {
  v &= 0x1fffffULL;
  v = (v | (v << 32)) & 0x1f00000000ffffULL;
  v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
  v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
  v = (v | (v << 2)) & 0x1249249249249249ULL;
  return v;
}

__global__ void k_morton(const double* __restrict__ pos, int64_t n, const double* __restrict__ bb,
                         uint64_t* __restrict__ codes, int* __restrict__ idx) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double ext = fmax(bb[3] - bb[0], fmax(bb[4] - bb[1], bb[5] - bb[2]));
  if (!(ext > 0)) ext = 1.0;
  const double qmax = (double)((1 << 21) - 1);
  const double scale = qmax / ext;
  uint64_t q[3];
  for (int k = 0; k < 3; ++k) {
    double f = (pos[3 * i + k] - bb[k]) * scale;
    f = fmin(fmax(f, 0.0), qmax);
    q[k] = (uint64_t)f;
  }
  codes[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
  idx[i] = (int)i;
}

// ---------------------------------------------------------------------------
// 2. Breadth-first radix split.
// ---------------------------------------------------------------------------
struct Pending {
  int s, e, parent, side;
};

__device__ __forceinline__ int split_point(const uint64_t* __restrict__ c, int s, int e) {
  const uint64_t a = c[s], b = c[e];
  if (a == b) return (int)(((int64_t)s + e + 1) / 2);
  const int bit = 63 - __clzll((long long)(a ^ b));
  const uint64_t mask = 1ULL << bit;
  int lo = s + 1, hi = e;  // first index whose code has `bit` set
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if (c[mid] & mask) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

__global__ void k_level_flags(const Pending* __restrict__ fr, int F, int leaf_size, int* __restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < F) flag[i] = (fr[i].e - fr[i].s + 1 > leaf_size) ? 1 : 0;
}

struct LeafRec {
  int s, e, parent, side, level;
};

__global__ void k_level_emit(const Pending* __restrict__ fr, int F, const int* __restrict__ flag,
                             const int* __restrict__ rank, int int_base, int leaf_base, int level,
                             const uint64_t* __restrict__ codes, int* __restrict__ int_ranges, int* __restrict__ int_parent,
                             int* __restrict__ int_level, int* __restrict__ left, int* __restrict__ right,
                             Pending* __restrict__ next, LeafRec* __restrict__ leaves) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= F) return;
  const Pending pd = fr[i];
  const int r = rank[i];
  if (flag[i]) {
    const int id = int_base + r;
    int_ranges[2 * id] = pd.s;
    int_ranges[2 * id + 1] = pd.e;
    int_parent[id] = pd.parent;
    int_level[id] = level;
    left[id] = -1;
    right[id] = -1;
    if (pd.parent >= 0) (pd.side == 0 ? left : right)[pd.parent] = id;
    const int sp = split_point(codes, pd.s, pd.e);
    next[2 * r] = Pending{pd.s, sp - 1, id, 0};
    next[2 * r + 1] = Pending{sp, pd.e, id, 1};
  } else {
    leaves[leaf_base + (i - r)] = LeafRec{pd.s, pd.e, pd.parent, pd.side, level};
  }
}

__global__ void k_mark_leaf_starts(const LeafRec* __restrict__ lv, int L, int* __restrict__ flag) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < L) flag[lv[j].s] = 1;
}

__global__ void k_leaf_of(const int* __restrict__ flag, const int* __restrict__ lidx, int64_t n, int* __restrict__ leaf_of) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) leaf_of[i] = lidx[i] + flag[i] - 1;
}

__global__ void k_place_leaves(const LeafRec* __restrict__ lv, int L, const int* __restrict__ lidx, int num_internal,
                               int* __restrict__ ranges, int* __restrict__ parent, int* __restrict__ level,
                               int* __restrict__ left, int* __restrict__ right) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= L) return;
  const LeafRec r = lv[j];
  const int id = num_internal + lidx[r.s];
  ranges[2 * id] = r.s;
  ranges[2 * id + 1] = r.e;
  parent[id] = r.parent;
  level[id] = r.level;
  if (r.parent >= 0) (r.side == 0 ? left : right)[r.parent] = id;
}

__global__ void k_widen_perm(const int* __restrict__ v, int64_t n, int64_t* __restrict__ perm) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) perm[i] = v[i];
}

__global__ void k_max_occupancy(const int* __restrict__ ranges, int num_internal, int L, int* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= L) return;
  const int id = num_internal + j;
  atomicMax(out, ranges[2 * id + 1] - ranges[2 * id] + 1);
}

// ---------------------------------------------------------------------------
// 3. COM and bounding radii (FP64, the host's operation order).
// ---------------------------------------------------------------------------
__global__ void k_leaf_com(int L, int num_internal, const int* __restrict__ ranges, const int* __restrict__ perm,
                           const double* __restrict__ pos, const double* __restrict__ mass, double* __restrict__ com,
                           double* __restrict__ radius, double* __restrict__ nmass) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= L) return;
  const int id = num_internal + j;
  const int s = ranges[2 * id], e = ranges[2 * id + 1];
  double sm = 0, sx = 0, sy = 0, sz = 0;
  for (int i = s; i <= e; ++i) {
    const int64_t o = perm[i];
    const double m = mass[o];
    sm += m;
    sx += m * pos[3 * o];
    sy += m * pos[3 * o + 1];
    sz += m * pos[3 * o + 2];
  }
  double c[3];
  if (sm > 0) {
    c[0] = sx / sm;
    c[1] = sy / sm;
    c[2] = sz / sm;
  } else {  // massless leaf: mean position of its particles
    c[0] = c[1] = c[2] = 0;
    for (int i = s; i <= e; ++i)
      for (int k = 0; k < 3; ++k) c[k] += pos[3 * (int64_t)perm[i] + k];
    for (int k = 0; k < 3; ++k) c[k] /= (double)(e - s + 1);
  }
  double rmax = 0;
  for (int i = s; i <= e; ++i) {
    const int64_t o = perm[i];
    const double dx = pos[3 * o] - c[0], dy = pos[3 * o + 1] - c[1], dz = pos[3 * o + 2] - c[2];
    rmax = fmax(rmax, sqrt(dx * dx + dy * dy + dz * dz));
  }
  nmass[id] = sm;
  radius[id] = rmax;
  for (int k = 0; k < 3; ++k) com[3 * (int64_t)id + k] = c[k];
}

__global__ void k_internal_com(int first, int last, const int* __restrict__ left, const int* __restrict__ right,
                               const int* __restrict__ ranges, double* __restrict__ com, double* __restrict__ radius,
                               double* __restrict__ nmass) {
  const int i = first + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= last) return;
  const int a = left[i], b = right[i];
  const double ma = nmass[a], mb = nmass[b], sm = ma + mb;
  const double na = (double)(ranges[2 * a + 1] - ranges[2 * a] + 1);
  const double nb = (double)(ranges[2 * b + 1] - ranges[2 * b] + 1);
  double c[3];
  for (int k = 0; k < 3; ++k)
    c[k] = sm > 0 ? (ma * com[3 * (int64_t)a + k] + mb * com[3 * (int64_t)b + k]) / sm
                  : (na * com[3 * (int64_t)a + k] + nb * com[3 * (int64_t)b + k]) / (na + nb);
  double r = 0;
  const int ch[2] = {a, b};
  for (int q = 0; q < 2; ++q) {
    double d2 = 0;
    for (int k = 0; k < 3; ++k) {
      const double dd = com[3 * (int64_t)ch[q] + k] - c[k];
      d2 += dd * dd;
    }
    r = fmax(r, sqrt(d2) + radius[ch[q]]);
  }
  nmass[i] = sm;
  radius[i] = r;
  for (int k = 0; k < 3; ++k) com[3 * (int64_t)i + k] = c[k];
}

// ---------------------------------------------------------------------------
// 4. Dual walk, breadth-first over node pairs.
// ---------------------------------------------------------------------------
enum : int { kNone = 0, kSelf = 1, kFar = 2, kNear = 3, kSplitA = 4, kSplitB = 5 };
constexpr int kMaxGears = 8;
constexpr int kMaxGearOrder = 24;
constexpr int kGearShift = 56;  // far keys of the adaptive walk carry the gear in bits 56..63

struct WalkCtx {
  const int* left;
  const int* right;
  const double* com;
  const double* radius;
  int num_internal;
  double theta2;
  // error-controlled, target-centric walk (jb_dtree_adaptive_walk); unused
  // by the symmetric theta walk
  const double* power;  // Dehnen per-degree source power P_l, num_nodes x npow
  const float* fscale;  // force scale of each target node (smallest |a| under it)
  int npow;             // degrees 0..npow-1 of power
  int num_gears;
  int gear_order[kMaxGears];
  double G, eps, theta_max;
};

__device__ __forceinline__ int walk_decide(const WalkCtx& w, int a, int b) {
  const bool la = a >= w.num_internal, lb = b >= w.num_internal;
  if (a == b) return la ? kNone : kSelf;
  double d2 = 0;
  for (int k = 0; k < 3; ++k) {
    const double dd = w.com[3 * (int64_t)a + k] - w.com[3 * (int64_t)b + k];
    d2 += dd * dd;
  }
  const double ra = w.radius[a], rb = w.radius[b];
  const double rs = ra + rb;
  if (d2 > 0 && rs * rs <= w.theta2 * d2) return kFar;
  if (la && lb) return kNear;
  return (!la && (lb || ra >= rb)) ? kSplitA : kSplitB;
}

__global__ void k_walk_count(const int2* __restrict__ fr, int F, WalkCtx w, I3* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= F) return;
  const int d = walk_decide(w, fr[i].x, fr[i].y);
  cnt[i] = I3{d == kSelf ? 3 : (d >= kSplitA ? 2 : 0), d == kFar ? 2 : 0, d == kNear ? 2 : 0};
}

__global__ void k_walk_emit(const int2* __restrict__ fr, int F, WalkCtx w, const I3* __restrict__ off,
                            int2* __restrict__ next, uint64_t* __restrict__ far_keys, int far_shift,
                            uint64_t* __restrict__ near_keys, int near_shift) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= F) return;
  const I3 o3 = off[i];
  const int a = fr[i].x, b = fr[i].y;
  const int d = walk_decide(w, a, b);
  if (d == kSelf) {
    const int l = w.left[a], r = w.right[a];
    int2* o = next + o3.a;
    o[0] = make_int2(l, l);
    o[1] = make_int2(r, r);
    o[2] = make_int2(l, r);
  } else if (d == kSplitA) {
    next[o3.a] = make_int2(w.left[a], b);
    next[o3.a + 1] = make_int2(w.right[a], b);
  } else if (d == kSplitB) {
    next[o3.a] = make_int2(a, w.left[b]);
    next[o3.a + 1] = make_int2(a, w.right[b]);
  } else if (d == kFar) {
    far_keys[o3.b] = ((uint64_t)a << far_shift) | (uint64_t)b;
    far_keys[o3.b + 1] = ((uint64_t)b << far_shift) | (uint64_t)a;
  } else if (d == kNear) {
    const uint64_t la = (uint64_t)(a - w.num_internal), lb = (uint64_t)(b - w.num_internal);
    near_keys[o3.c] = (la << near_shift) | lb;
    near_keys[o3.c + 1] = (lb << near_shift) | la;
  }
}

// Error-controlled acceptance of the far pair (target t <- source s), the
// reference's Dehnen eq. (15)/(16a) policy (runtime/_adaptive_policy.py:
// 267-376 dehnen_paper_pair_error_by_order, :2285-2338 the directional test):
//   E_p   = sum_{l=0}^{p} C(p, l) P_l(s) rho_t^(p-l)        (eq. 15, binomial sum)
//   dF_p  = 8 max(rho_s, rho_t) / (rho_s + rho_t) * G E_p / d^(p+2)
// (the source mass of E_p / (M_s d^p) and of G M_s / d^2 cancels), accepted
// when (rho_s + rho_t) < theta_max d and the highest gear passes
// dF < max(eps * fscale[t], 1e-24); the gear is the lowest passing one.
// Returns the gear index, or -1.  Every step is a separately rounded FP64
// operation (this file is compiled with -fmad=false), in the order the
// oracle's restatement (oracle/adaptive_walk.py) uses.
__device__ int error_gear(const WalkCtx& w, int t, int s, double d, double rt, double rs) {
  double rtp[kMaxGearOrder + 1], dp[kMaxGearOrder + 3];
  const int pmax = w.gear_order[w.num_gears - 1];
  rtp[0] = 1.0;
  for (int k = 1; k <= pmax; ++k) rtp[k] = rtp[k - 1] * rt;
  dp[0] = 1.0;
  for (int k = 1; k <= pmax + 2; ++k) dp[k] = dp[k - 1] * d;
  const double den = fmax(rs + rt, 1e-24);
  const double imp = (8.0 * fmax(rs, rt)) / den;
  const double thr = fmax(w.eps * (double)w.fscale[t], 1e-24);
  const double* P = w.power + (int64_t)s * w.npow;
  int first = -1;
  bool pass = false;
  for (int g = 0; g < w.num_gears; ++g) {
    const int p = w.gear_order[g];
    double e = 0.0, c = 1.0;  // c = C(p, l)
    for (int l = 0; l <= p && l < w.npow; ++l) {
      if (l > 0) c = (c * (double)(p - l + 1)) / (double)l;
      e = e + (c * P[l]) * rtp[p - l];
    }
    const double ferr = ((w.G * imp) * e) / dp[p + 2];
    pass = ferr < thr;
    if (pass && first < 0) first = g;
  }
  return pass ? first : -1;  // the highest gear must pass
}

__device__ __forceinline__ int adaptive_decide(const WalkCtx& w, int t, int s, int* gear) {
  const bool lt = t >= w.num_internal, ls = s >= w.num_internal;
  if (t == s) return lt ? kNone : kSelf;
  double d2 = 0;
  for (int k = 0; k < 3; ++k) {
    const double dd = w.com[3 * (int64_t)t + k] - w.com[3 * (int64_t)s + k];
    d2 += dd * dd;
  }
  const double rt = w.radius[t], rs = w.radius[s];
  if (d2 > 0) {
    const double d = sqrt(d2);
    if (rs + rt < w.theta_max * d) {
      const int g = error_gear(w, t, s, d, rt, rs);
      if (g >= 0) {
        *gear = g;
        return kFar;
      }
    }
  }
  if (lt && ls) return kNear;
  return (!lt && (ls || rt >= rs)) ? kSplitA : kSplitB;
}

__global__ void k_awalk_count(const int2* __restrict__ fr, int F, WalkCtx w, I3* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= F) return;
  int g = 0;
  const int d = adaptive_decide(w, fr[i].x, fr[i].y, &g);
  cnt[i] = I3{d == kSelf ? 4 : (d >= kSplitA ? 2 : 0), d == kFar ? 1 : 0, d == kNear ? 1 : 0};
}

__global__ void k_awalk_emit(const int2* __restrict__ fr, int F, WalkCtx w, const I3* __restrict__ off,
                             int2* __restrict__ next, uint64_t* __restrict__ far_keys, int far_shift,
                             uint64_t* __restrict__ near_keys, int near_shift) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= F) return;
  const I3 o3 = off[i];
  const int t = fr[i].x, s = fr[i].y;
  int g = 0;
  const int d = adaptive_decide(w, t, s, &g);
  if (d == kSelf) {
    const int l = w.left[t], r = w.right[t];
    int2* o = next + o3.a;
    o[0] = make_int2(l, l);
    o[1] = make_int2(r, r);
    o[2] = make_int2(l, r);
    o[3] = make_int2(r, l);
  } else if (d == kSplitA) {
    next[o3.a] = make_int2(w.left[t], s);
    next[o3.a + 1] = make_int2(w.right[t], s);
  } else if (d == kSplitB) {
    next[o3.a] = make_int2(t, w.left[s]);
    next[o3.a + 1] = make_int2(t, w.right[s]);
  } else if (d == kFar) {
    far_keys[o3.b] = ((uint64_t)g << kGearShift) | ((uint64_t)t << far_shift) | (uint64_t)s;
  } else if (d == kNear) {
    near_keys[o3.c] = ((uint64_t)(t - w.num_internal) << near_shift) | (uint64_t)(s - w.num_internal);
  }
}

// The lowest gear whose eq. (15) estimate passes, for the given far pairs of
// a fixed list (the analytic per-pair order choice the reference makes for
// its gear buckets, with dehnen_paper); the highest gear where even it fails.
__global__ void k_far_dehnen_gears(int64_t n, const int* __restrict__ pair_tgt, const int* __restrict__ far_src,
                                   WalkCtx w, int* __restrict__ gears) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int t = pair_tgt[e], s = far_src[e];
  double d2 = 0;
  for (int k = 0; k < 3; ++k) {
    const double dd = w.com[3 * (int64_t)t + k] - w.com[3 * (int64_t)s + k];
    d2 += dd * dd;
  }
  const int g = d2 > 0 ? error_gear(w, t, s, sqrt(d2), w.radius[t], w.radius[s]) : -1;
  gears[e] = g < 0 ? w.num_gears - 1 : g;
}

// Moves the gear bits of sorted far keys into gears[] (CSR order).
__global__ void k_take_gears(uint64_t* __restrict__ keys, int64_t n, int* __restrict__ gears) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t k = keys[i];
  gears[i] = (int)(k >> kGearShift);
  keys[i] = k & ((1ULL << kGearShift) - 1);
}

// ---------------------------------------------------------------------------
// 5. CSR from sorted (row << shift | col) keys.
// ---------------------------------------------------------------------------
// keys sorted; thread i writes column i and, where the row changes between
// keys i-1 and i, the offsets of the rows in between; rows before the first
// key start at 0, rows after the last at n.
__global__ void k_csr(const uint64_t* __restrict__ keys, int64_t n, int shift, int rows, int* __restrict__ cols,
                      int64_t* __restrict__ off) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= rows) {
    const int64_t r0 = (int64_t)(keys[0] >> shift), r1 = (int64_t)(keys[n - 1] >> shift);
    if (i <= r0) off[i] = 0;
    else if (i > r1) off[i] = n;
  }
  if (i < n) {
    const uint64_t k = keys[i];
    cols[i] = (int)(k & ((1ULL << shift) - 1));
    if (i > 0) {
      const int64_t r = (int64_t)(k >> shift), rp = (int64_t)(keys[i - 1] >> shift);
      for (int64_t q = rp + 1; q <= r; ++q) off[q] = i;
    }
  }
}

inline int bits_for(int64_t v) {  // bits to hold values in [0, v)
  int b = 1;
  while (b < 62 && ((int64_t)1 << b) < v) ++b;
  return b;
}

}  // namespace

// ---------------------------------------------------------------------------
// The handle: every output array in device memory.
// ---------------------------------------------------------------------------
struct jb_dtree {
  jb_tree_info_t info{};
  DBuf perm, ranges, left, right, parent, level, level_off, leaf_of, far_off, far_src, near_off, near_src, com, radius;
  DBuf far_gear;  // gear index per far pair (CSR order) after jb_dtree_adaptive_walk
  int walk_kind = 0;  // 0: symmetric theta walk, 1: error-controlled target-centric walk
};

namespace {

// Steps 4 and 5: the dual walk from (root, root) and the CSR lists built from
// what it emits, into t.far_off/far_src/near_off/near_src (and t.far_gear for
// the adaptive walk).  Sets t.info.num_far_pairs / num_near_pairs.
int64_t walk_lists(jb_dtree& t, const WalkCtx& w, bool adaptive, int NN, int L, Scratch& s, int* d_total32,
                   cudaStream_t st) {
  const int far_shift = bits_for(NN), near_shift = bits_for(std::max(L, 1));
  DBuf w0, w1, cnt3, off3, far_keys, near_keys;
  int64_t n_far = 0, n_near = 0;
  if (NN > 1) {
    const int64_t cap = std::max<int64_t>(1 << 16, 4 * (int64_t)NN);
    ck(w0.alloc(cap * sizeof(int2)));
    ck(w1.alloc(cap * sizeof(int2)));
    ck(cnt3.alloc(cap * sizeof(I3)));
    ck(off3.alloc(cap * sizeof(I3)));
    ck(far_keys.alloc((size_t)std::max<int64_t>(1 << 16, 256 * (int64_t)NN) * 8));
    ck(near_keys.alloc((size_t)std::max<int64_t>(1 << 16, 256 * (int64_t)L) * 8));
    I3* d_tot3 = reinterpret_cast<I3*>(d_total32);
    const int2 root = make_int2(0, 0);
    ck(cudaMemcpyAsync(w0.p, &root, sizeof(root), cudaMemcpyHostToDevice, st));
    DBuf* wc = &w0;
    DBuf* wn = &w1;
    int64_t Fw = 1;
    while (Fw > 0) {
      if ((size_t)Fw * sizeof(I3) > cnt3.bytes) {
        ck(cnt3.alloc((size_t)Fw * 2 * sizeof(I3)));
        ck(off3.alloc((size_t)Fw * 2 * sizeof(I3)));
      }
      if (adaptive)
        k_awalk_count<<<nblocks(Fw, 256), 256, 0, st>>>(wc->as<int2>(), (int)Fw, w, cnt3.as<I3>());
      else
        k_walk_count<<<nblocks(Fw, 256), 256, 0, st>>>(wc->as<int2>(), (int)Fw, w, cnt3.as<I3>());
      ck_launch();
      exclusive_scan<I3>(cnt3.as<I3>(), off3.as<I3>(), Fw, d_tot3, s, st);
      const I3 tot = read_word(d_tot3, st);
      // grow the next frontier and the key buffers as needed (stream-ordered)
      ck(wn->grow((size_t)tot.a * 2 * sizeof(int2), 0, st));
      const size_t need_far = (size_t)(n_far + tot.b) * 8, need_near = (size_t)(n_near + tot.c) * 8;
      if (need_far > far_keys.bytes) ck(far_keys.grow(std::max(need_far, 2 * far_keys.bytes), (size_t)n_far * 8, st));
      if (need_near > near_keys.bytes)
        ck(near_keys.grow(std::max(need_near, 2 * near_keys.bytes), (size_t)n_near * 8, st));
      if (adaptive)
        k_awalk_emit<<<nblocks(Fw, 256), 256, 0, st>>>(wc->as<int2>(), (int)Fw, w, off3.as<I3>(), wn->as<int2>(),
                                                       far_keys.as<uint64_t>() + n_far, far_shift,
                                                       near_keys.as<uint64_t>() + n_near, near_shift);
      else
        k_walk_emit<<<nblocks(Fw, 256), 256, 0, st>>>(wc->as<int2>(), (int)Fw, w, off3.as<I3>(), wn->as<int2>(),
                                                      far_keys.as<uint64_t>() + n_far, far_shift,
                                                      near_keys.as<uint64_t>() + n_near, near_shift);
      ck_launch();
      n_far += tot.b;
      n_near += tot.c;
      Fw = tot.a;
      std::swap(wc, wn);
    }
  }
  w0.release();
  w1.release();
  cnt3.release();
  off3.release();

  auto to_csr = [&](DBuf& keys, int64_t m, int shift, int rows, DBuf& off, DBuf& col, DBuf* gears) {
    ck(off.alloc((size_t)(rows + 1) * 8));
    ck(col.alloc((size_t)std::max<int64_t>(m, 1) * 4));
    if (gears) ck(gears->alloc((size_t)std::max<int64_t>(m, 1) * 4));
    if (m == 0) {
      ck(cudaMemsetAsync(off.p, 0, (size_t)(rows + 1) * 8, st));
      return;
    }
    DBuf tmp;
    ck(tmp.alloc((size_t)m * 8));
    radix_sort(keys.as<uint64_t>(), nullptr, tmp.as<uint64_t>(), nullptr, m, 2 * shift, s, st);
    if (gears) {
      k_take_gears<<<nblocks(m, 256), 256, 0, st>>>(keys.as<uint64_t>(), m, gears->as<int>());
      ck_launch();
    }
    k_csr<<<nblocks(std::max<int64_t>(m, rows + 1), 256), 256, 0, st>>>(keys.as<uint64_t>(), m, shift, rows,
                                                                       col.as<int>(), off.as<int64_t>());
    ck_launch();
  };
  if (NN > 1) {
    to_csr(far_keys, n_far, far_shift, NN, t.far_off, t.far_src, adaptive ? &t.far_gear : nullptr);
    far_keys.release();
    to_csr(near_keys, n_near, near_shift, L, t.near_off, t.near_src, nullptr);
    near_keys.release();
  } else {
    ck(t.far_off.alloc((size_t)(NN + 1) * 8));
    ck(cudaMemsetAsync(t.far_off.p, 0, (size_t)(NN + 1) * 8, st));
    ck(t.near_off.alloc((size_t)(L + 1) * 8));
    ck(cudaMemsetAsync(t.near_off.p, 0, (size_t)(L + 1) * 8, st));
    ck(t.far_src.alloc(4));
    ck(t.near_src.alloc(4));
    if (adaptive) ck(t.far_gear.alloc(4));
  }
  t.info.num_far_pairs = n_far;
  t.info.num_near_pairs = n_near;
  return 0;
}

void build(jb_dtree& t, int64_t n, const double* pos, const double* mass, int leaf_size, double theta, cudaStream_t st) {
  tl_stream = st;
  Scratch s;
  ck(s.total.alloc(64));
  int64_t* d_total64 = s.total.as<int64_t>();
  int* d_total32 = reinterpret_cast<int*>(d_total64 + 4);

  // 1. Morton codes, sorted with their input index.
  DBuf part, bb, k0, k1, v0, v1;
  const int nb_bb = 296;
  ck(part.alloc(6 * nb_bb * sizeof(double)));
  ck(bb.alloc(6 * sizeof(double)));
  k_bbox_partial<<<nb_bb, 256, 0, st>>>(pos, n, part.as<double>());
  ck_launch();
  k_bbox_final<<<1, 32, 0, st>>>(part.as<double>(), nb_bb, bb.as<double>());
  ck_launch();
  ck(k0.alloc((size_t)n * 8));
  ck(k1.alloc((size_t)n * 8));
  ck(v0.alloc((size_t)n * 4));
  ck(v1.alloc((size_t)n * 4));
  k_morton<<<nblocks(n, 256), 256, 0, st>>>(pos, n, bb.as<double>(), k0.as<uint64_t>(), v0.as<int>());
  ck_launch();
  radix_sort(k0.as<uint64_t>(), v0.as<int>(), k1.as<uint64_t>(), v1.as<int>(), n, 63, s, st);
  const uint64_t* codes = k0.as<uint64_t>();
  const int* sperm = v0.as<int>();  // sorted slot -> input index

  // 2. Breadth-first split, one level at a time.
  DBuf fr0, fr1, flag, rank, int_ranges, int_parent, int_level, leaves, left, right;
  ck(fr0.alloc((size_t)n * sizeof(Pending)));
  ck(fr1.alloc((size_t)n * sizeof(Pending)));
  ck(flag.alloc((size_t)(n + 1) * 4));
  ck(rank.alloc((size_t)(n + 1) * 4));
  ck(int_ranges.alloc((size_t)n * 8));
  ck(int_parent.alloc((size_t)n * 4));
  ck(int_level.alloc((size_t)n * 4));
  ck(left.alloc((size_t)n * 4));
  ck(right.alloc((size_t)n * 4));
  ck(leaves.alloc((size_t)n * sizeof(LeafRec)));
  {
    const Pending root{0, (int)n - 1, -1, 0};
    ck(cudaMemcpyAsync(fr0.p, &root, sizeof(root), cudaMemcpyHostToDevice, st));
  }
  Pending* cur = fr0.as<Pending>();
  Pending* nxt = fr1.as<Pending>();
  int F = 1, int_base = 0, leaf_base = 0, level = 0;
  std::vector<int> level_off;
  while (F > 0) {
    level_off.push_back(int_base);
    k_level_flags<<<nblocks(F, 256), 256, 0, st>>>(cur, F, leaf_size, flag.as<int>());
    ck_launch();
    exclusive_scan<int>(flag.as<int>(), rank.as<int>(), F, d_total32, s, st);
    const int n_int = read_word(d_total32, st);
    k_level_emit<<<nblocks(F, 256), 256, 0, st>>>(cur, F, flag.as<int>(), rank.as<int>(), int_base, leaf_base, level,
                                                  codes, int_ranges.as<int>(), int_parent.as<int>(), int_level.as<int>(),
                                                  left.as<int>(), right.as<int>(), nxt, leaves.as<LeafRec>());
    ck_launch();
    int_base += n_int;
    leaf_base += F - n_int;
    F = 2 * n_int;
    std::swap(cur, nxt);
    ++level;
  }
  const int NI = int_base, L = leaf_base, NN = NI + L;
  while (level_off.size() > 1 && level_off.back() == NI) level_off.pop_back();
  level_off.push_back(NI);
  int num_levels = NI > 0 ? (int)level_off.size() - 1 : 0;
  if (NI == 0) level_off.assign(1, 0);

  // Leaves in particle order; node arrays.
  ck(cudaMemsetAsync(flag.p, 0, (size_t)n * 4, st));
  k_mark_leaf_starts<<<nblocks(L, 256), 256, 0, st>>>(leaves.as<LeafRec>(), L, flag.as<int>());
  ck_launch();
  exclusive_scan<int>(flag.as<int>(), rank.as<int>(), n, nullptr, s, st);
  ck(t.leaf_of.alloc((size_t)n * 4));
  k_leaf_of<<<nblocks(n, 256), 256, 0, st>>>(flag.as<int>(), rank.as<int>(), n, t.leaf_of.as<int>());
  ck_launch();
  ck(t.ranges.alloc((size_t)NN * 8));
  ck(t.parent.alloc((size_t)NN * 4));
  ck(t.level.alloc((size_t)NN * 4));
  ck(t.left.alloc((size_t)std::max(NI, 1) * 4));
  ck(t.right.alloc((size_t)std::max(NI, 1) * 4));
  if (NI > 0) {
    ck(cudaMemcpyAsync(t.ranges.p, int_ranges.p, (size_t)NI * 8, cudaMemcpyDeviceToDevice, st));
    ck(cudaMemcpyAsync(t.parent.p, int_parent.p, (size_t)NI * 4, cudaMemcpyDeviceToDevice, st));
    ck(cudaMemcpyAsync(t.level.p, int_level.p, (size_t)NI * 4, cudaMemcpyDeviceToDevice, st));
    ck(cudaMemcpyAsync(t.left.p, left.p, (size_t)NI * 4, cudaMemcpyDeviceToDevice, st));
    ck(cudaMemcpyAsync(t.right.p, right.p, (size_t)NI * 4, cudaMemcpyDeviceToDevice, st));
  }
  k_place_leaves<<<nblocks(L, 256), 256, 0, st>>>(leaves.as<LeafRec>(), L, rank.as<int>(), NI, t.ranges.as<int>(),
                                                  t.parent.as<int>(), t.level.as<int>(), t.left.as<int>(),
                                                  t.right.as<int>());
  ck_launch();
  ck(t.level_off.alloc(level_off.size() * 4));
  ck(cudaMemcpyAsync(t.level_off.p, level_off.data(), level_off.size() * 4, cudaMemcpyHostToDevice, st));
  ck(t.perm.alloc((size_t)n * 8));
  k_widen_perm<<<nblocks(n, 256), 256, 0, st>>>(sperm, n, t.perm.as<int64_t>());
  ck_launch();
  ck(cudaMemsetAsync(d_total32, 0, 4, st));
  k_max_occupancy<<<nblocks(L, 256), 256, 0, st>>>(t.ranges.as<int>(), NI, L, d_total32);
  ck_launch();
  const int max_occ = read_word(d_total32, st);

  // 3. COM and radii.
  DBuf nmass;
  ck(t.com.alloc((size_t)NN * 3 * 8));
  ck(t.radius.alloc((size_t)NN * 8));
  ck(nmass.alloc((size_t)NN * 8));
  k_leaf_com<<<nblocks(L, 128), 128, 0, st>>>(L, NI, t.ranges.as<int>(), sperm, pos, mass, t.com.as<double>(),
                                              t.radius.as<double>(), nmass.as<double>());
  ck_launch();
  for (int lv = num_levels - 1; lv >= 0; --lv) {
    const int a = level_off[lv], b = level_off[lv + 1];
    if (b <= a) continue;
    k_internal_com<<<nblocks(b - a, 128), 128, 0, st>>>(a, b, t.left.as<int>(), t.right.as<int>(), t.ranges.as<int>(),
                                                        t.com.as<double>(), t.radius.as<double>(), nmass.as<double>());
    ck_launch();
  }
  // free the split buffers before the walk
  fr0.release();
  fr1.release();
  int_ranges.release();
  int_parent.release();
  int_level.release();
  leaves.release();
  left.release();
  right.release();
  k1.release();
  v1.release();

  // 4./5. Dual walk (only when the root is split, as the host) and CSR lists.
  {
    WalkCtx w{};
    w.left = t.left.as<int>();
    w.right = t.right.as<int>();
    w.com = t.com.as<double>();
    w.radius = t.radius.as<double>();
    w.num_internal = NI;
    w.theta2 = theta * theta;
    walk_lists(t, w, false, NN, L, s, d_total32, st);
  }
  ck(cudaStreamSynchronize(st));

  t.info.num_particles = n;
  t.info.num_nodes = NN;
  t.info.num_internal = NI;
  t.info.num_leaves = L;
  t.info.num_levels = num_levels;
  t.info.max_leaf_occupancy = max_occ;
}

const DBuf* field_buf(const jb_dtree* t, int field) {
  switch (field) {
    case JB_TREE_PERMUTATION: return &t->perm;
    case JB_TREE_NODE_RANGES: return &t->ranges;
    case JB_TREE_LEFT_CHILD: return &t->left;
    case JB_TREE_RIGHT_CHILD: return &t->right;
    case JB_TREE_PARENT: return &t->parent;
    case JB_TREE_NODE_LEVEL: return &t->level;
    case JB_TREE_LEVEL_OFFSETS: return &t->level_off;
    case JB_TREE_LEAF_OF_PARTICLE: return &t->leaf_of;
    case JB_TREE_FAR_OFFSETS: return &t->far_off;
    case JB_TREE_FAR_SOURCES: return &t->far_src;
    case JB_TREE_NEAR_OFFSETS: return &t->near_off;
    case JB_TREE_NEAR_SOURCES: return &t->near_src;
    case JB_TREE_CENTERS_F64: return &t->com;
    case JB_TREE_RADII_F64: return &t->radius;
    case JB_TREE_FAR_GEARS: return t->walk_kind == 1 ? &t->far_gear : nullptr;
    default: return nullptr;
  }
}

size_t field_bytes(const jb_dtree* t, int field) {
  const jb_tree_info_t& i = t->info;
  switch (field) {
    case JB_TREE_PERMUTATION: return (size_t)i.num_particles * 8;
    case JB_TREE_NODE_RANGES: return (size_t)i.num_nodes * 8;
    case JB_TREE_LEFT_CHILD:
    case JB_TREE_RIGHT_CHILD: return (size_t)i.num_internal * 4;
    case JB_TREE_PARENT:
    case JB_TREE_NODE_LEVEL: return (size_t)i.num_nodes * 4;
    case JB_TREE_LEVEL_OFFSETS: return (size_t)(i.num_levels + 1) * 4;
    case JB_TREE_LEAF_OF_PARTICLE: return (size_t)i.num_particles * 4;
    case JB_TREE_FAR_OFFSETS: return (size_t)(i.num_nodes + 1) * 8;
    case JB_TREE_FAR_SOURCES: return (size_t)i.num_far_pairs * 4;
    case JB_TREE_NEAR_OFFSETS: return (size_t)(i.num_leaves + 1) * 8;
    case JB_TREE_NEAR_SOURCES: return (size_t)i.num_near_pairs * 4;
    case JB_TREE_CENTERS_F64: return (size_t)i.num_nodes * 24;
    case JB_TREE_RADII_F64: return (size_t)i.num_nodes * 8;
    case JB_TREE_FAR_GEARS: return t->walk_kind == 1 ? (size_t)i.num_far_pairs * 4 : 0;
    default: return 0;
  }
}

}  // namespace

extern "C" {

JB_API int jb_tree_build_device(int64_t n, const double* pos, const double* mass, int leaf_size, double theta,
                                void* stream, jb_dtree** out) {
  if (!out) return JB_ERR_ARG;
  *out = nullptr;
  if (n <= 0 || n > (int64_t)0x7fffffff || !pos || !mass || leaf_size < 1 || !(theta > 0) || !(theta < 1.0))
    return JB_ERR_ARG;
  jb_dtree* t = new (std::nothrow) jb_dtree();
  if (!t) return JB_ERR_ALLOC;
  try {
    build(*t, n, pos, mass, leaf_size, theta, reinterpret_cast<cudaStream_t>(stream));
  } catch (const Fail& f) {
    delete t;
    return f.rc;
  } catch (const std::bad_alloc&) {
    delete t;
    return JB_ERR_ALLOC;
  }
  *out = t;
  return JB_OK;
}

JB_API int jb_dtree_adaptive_walk(jb_dtree* t, int num_degrees, const double* power, const float* force_scale,
                                  double G, double eps, double theta_max, int num_gears, const int* gear_orders,
                                  void* stream) {
  if (!t || !power || !force_scale || num_degrees < 1 || num_gears < 1 || num_gears > kMaxGears || !gear_orders ||
      !(eps > 0) || !(theta_max > 0) || theta_max > 1.0 || !(G > 0))
    return JB_ERR_ARG;
  for (int g = 0; g < num_gears; ++g) {
    const int p = gear_orders[g];
    if (p < 0 || p > kMaxGearOrder || p >= num_degrees || (g > 0 && p <= gear_orders[g - 1])) return JB_ERR_ARG;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  try {
    tl_stream = st;
    Scratch s;
    ck(s.total.alloc(64));
    int* d_total32 = reinterpret_cast<int*>(s.total.as<int64_t>() + 4);
    WalkCtx w{};
    w.left = t->left.as<int>();
    w.right = t->right.as<int>();
    w.com = t->com.as<double>();
    w.radius = t->radius.as<double>();
    w.num_internal = t->info.num_internal;
    w.power = power;
    w.fscale = force_scale;
    w.npow = num_degrees;
    w.num_gears = num_gears;
    for (int g = 0; g < num_gears; ++g) w.gear_order[g] = gear_orders[g];
    w.G = G;
    w.eps = eps;
    w.theta_max = theta_max;
    t->far_off.release();
    t->far_src.release();
    t->near_off.release();
    t->near_src.release();
    t->far_gear.release();
    walk_lists(*t, w, true, t->info.num_nodes, t->info.num_leaves, s, d_total32, st);
    t->walk_kind = 1;
    ck(cudaStreamSynchronize(st));
  } catch (const Fail& f) {
    return f.rc;
  } catch (const std::bad_alloc&) {
    return JB_ERR_ALLOC;
  }
  return JB_OK;
}

JB_API int jb_far_dehnen_gears(int64_t num_pairs, const int* pair_tgt, const int* far_src, const double* com,
                               const double* radius, int num_degrees, const double* power, const float* force_scale,
                               double G, double eps, int num_gears, const int* gear_orders, int* gears,
                               void* stream) {
  if (num_pairs < 0 || num_degrees < 1 || num_gears < 1 || num_gears > kMaxGears || !gear_orders || !(eps > 0) ||
      !(G > 0) || (num_pairs > 0 && (!pair_tgt || !far_src || !com || !radius || !power || !force_scale || !gears)))
    return JB_ERR_ARG;
  for (int g = 0; g < num_gears; ++g) {
    const int p = gear_orders[g];
    if (p < 0 || p > kMaxGearOrder || p >= num_degrees || (g > 0 && p <= gear_orders[g - 1])) return JB_ERR_ARG;
  }
  if (num_pairs == 0) return JB_OK;
  WalkCtx w{};
  w.com = com;
  w.radius = radius;
  w.power = power;
  w.fscale = force_scale;
  w.npow = num_degrees;
  w.num_gears = num_gears;
  for (int g = 0; g < num_gears; ++g) w.gear_order[g] = gear_orders[g];
  w.G = G;
  w.eps = eps;
  w.theta_max = 1.0;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  k_far_dehnen_gears<<<nblocks(num_pairs, 256), 256, 0, st>>>(num_pairs, pair_tgt, far_src, w, gears);
  return jb::cuda_status(cudaGetLastError());
}

JB_API int jb_dtree_info(const jb_dtree* t, jb_tree_info_t* info) {
  if (!t || !info) return JB_ERR_ARG;
  *info = t->info;
  return JB_OK;
}

JB_API const void* jb_dtree_field(const jb_dtree* t, int field) {
  if (!t) return nullptr;
  const DBuf* b = field_buf(t, field);
  return b ? b->p : nullptr;
}

JB_API int jb_dtree_copy(const jb_dtree* t, int field, void* dst) {
  if (!t || !dst) return JB_ERR_ARG;
  const DBuf* b = field_buf(t, field);
  if (!b) return JB_ERR_ARG;
  const size_t bytes = field_bytes(t, field);
  if (bytes == 0) return JB_OK;
  return jb::cuda_status(cudaMemcpy(dst, b->p, bytes, cudaMemcpyDeviceToHost));
}

JB_API void jb_dtree_free(jb_dtree* t) { delete t; }

}  // extern "C"
