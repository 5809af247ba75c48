// Split-BF16 M2L on the 5th-generation tensor cores (tcgen05, TMEM).
//
// The per-pair rotate+scale chain of the real-basis M2L
// (operators/m2l_real_rot_scale.py:288-386) is
//   Dz(az) -> B -> Dz(-ax) r^-k -> K -> r^-(n+1) Dz(ax) -> B^T -> Dz(-az)
// with three constant products (B, K = B^T Z0 B, B^T) between per-pair
// diagonal steps.  A CTA takes tiles of 128 consecutive far pairs (pair i of
// the tile = thread i = MMA row i = TMEM lane i).  Each thread applies the
// diagonal steps to its pair's 81-vector in registers, splits it into BF16
// hi and lo parts and writes them as the A operand (K-major core matrices in
// shared memory); one thread issues the products as block-diagonal 16/32-wide
// tcgen05.mma tiles (kind::f16, BF16 inputs, FP32 accumulation in TMEM),
// three per tile: A_hi W_hi + A_lo W_hi + A_hi W_lo; the results come back
// with tcgen05.ld.  The products' hi/lo weight tiles are generated on the
// host (jaccpot_b200/_tables.py, generated/tc_plans.h).
//
// Accumulation onto targets: the tile's outputs go to shared memory and the
// runs of equal target (the far list is sorted by target) are summed by
// column; targets whose whole list lies in one tile write their local row,
// the others write scratch rows that k_m2l_reduce sums in slot order.  Every
// wait on the MMA barrier is bounded: on timeout the kernel records status 1,
// drains its outstanding commit (bounded), frees TMEM and returns; status 2
// means the drain timed out as well (the TMEM was released while an MMA may
// still write it: the context is not to be used further).
#include <cuda_bf16.h>

#include "fmm_kernels.cuh"
#include "generated/tc_plans.h"

namespace jb {
namespace tc {

constexpr int kThreads = 128;
constexpr int kASbo = (kTcRow / 8) * 128;          // bytes between 8-row groups of the A operand
constexpr int kAPartBytes = 128 * kTcRow * 2;      // one BF16 part of a 128 x kTcRow tile
constexpr int kTmemCols = 128;
constexpr unsigned kSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t su32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version 1; base offset 0, no swizzle
  return d;
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
// K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(id), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

// Bounded wait on the barrier phase; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
  for (unsigned it = 0; it < kSpinLimit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* f) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int k = 0; k < 16; ++k) f[k] = __uint_as_float(r[k]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // a -> low half (lower address)
  return *reinterpret_cast<uint32_t*>(&h);
}

// Writes row `row` of the A operand (hi and lo parts) for product G of plan P
// from the coefficient vector v: padded column c holds v[inp_G(c)] (or 0).
template <int P, int G>
__device__ __forceinline__ void write_a(const float* v, unsigned char* a_hi, unsigned char* a_lo, int row) {
  using PL = TcPlan<P>;
  constexpr int NP = G == 0 ? PL::kNpad0 : (G == 1 ? PL::kNpad1 : PL::kNpad2);
  const int base = (row >> 3) * kASbo + (row & 7) * 16;
#pragma unroll
  for (int q = 0; q < NP / 8; ++q) {
    float x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int k = G == 0 ? PL::inp0(8 * q + j) : (G == 1 ? PL::inp1(8 * q + j) : PL::inp2(8 * q + j));
      x[j] = k >= 0 ? v[k] : 0.f;
    }
    uint32_t h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      __nv_bfloat162 hb = __floats2bfloat162_rn(x[2 * j], x[2 * j + 1]);
      const float2 hf = __bfloat1622float2(hb);
      h[j] = *reinterpret_cast<uint32_t*>(&hb);
      l[j] = pack2(x[2 * j] - hf.x, x[2 * j + 1] - hf.y);
    }
    *reinterpret_cast<uint4*>(a_hi + base + q * 128) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(a_lo + base + q * 128) = make_uint4(l[0], l[1], l[2], l[3]);
  }
}

// Reads this thread's accumulator row of product G back into coefficient order.
template <int P, int G>
__device__ __forceinline__ void read_d(uint32_t tmem_row, float* v) {
  using PL = TcPlan<P>;
  constexpr int NP = G == 0 ? PL::kNpad0 : (G == 1 ? PL::kNpad1 : PL::kNpad2);
  float d[kTcRow];
#pragma unroll
  for (int q = 0; q < NP / 16; ++q) tmem_ld16(tmem_row + 16 * q, d + 16 * q);
  tmem_wait_ld();
#pragma unroll
  for (int k = 0; k < csize(P); ++k) v[k] = 0.f;
#pragma unroll
  for (int c = 0; c < NP; ++c) {
    const int k = G == 0 ? PL::out0(c) : (G == 1 ? PL::out1(c) : PL::out2(c));
    if (k >= 0) v[k] = d[c];
  }
}

// One product, issued by a single thread: for every diagonal tile, the three
// split products, K in steps of 16.
template <int P, int G>
__device__ __forceinline__ void issue(uint32_t tmem, uint32_t a_hi, uint32_t a_lo, uint32_t w_base) {
  using PL = TcPlan<P>;
  constexpr int NT = G == 0 ? PL::kNumTiles0 : (G == 1 ? PL::kNumTiles1 : PL::kNumTiles2);
#pragma unroll
  for (int j = 0; j < NT; ++j) {
    const int col = G == 0 ? PL::tile_col0(j) : (G == 1 ? PL::tile_col1(j) : PL::tile_col2(j));
    const int w = G == 0 ? PL::tile_w0(j) : (G == 1 ? PL::tile_w1(j) : PL::tile_w2(j));
    const int off = G == 0 ? PL::tile_off0(j) : (G == 1 ? PL::tile_off1(j) : PL::tile_off2(j));
    const uint32_t wsbo = (uint32_t)(w / 8) * 128u;
    const uint32_t w_hi = w_base + (uint32_t)off, w_lo = w_hi + (uint32_t)(w * w * 2);
    const uint32_t id = idesc(w);
#pragma unroll
    for (int pr = 0; pr < 3; ++pr) {
      const uint32_t a = pr == 1 ? a_lo : a_hi;
      const uint32_t b = pr == 2 ? w_lo : w_hi;
#pragma unroll
      for (int ks = 0; ks < w / 16; ++ks) {
        const uint64_t ad = sdesc(a + (uint32_t)(col / 8 + 2 * ks) * 128u, 128u, (uint32_t)kASbo);
        const uint64_t bd = sdesc(b + (uint32_t)(2 * ks) * 128u, 128u, wsbo);
        mma_bf16(tmem + (uint32_t)col, ad, bd, id, (pr == 0 && ks == 0) ? 0u : 1u);
      }
    }
  }
}

// KONLY = true: only the K product runs on the tensor cores and B / B^T run
// as literal-constant FMAs in registers (one MMA round trip per tile instead
// of three); false: all three products on the tensor cores.
template <int P, bool KONLY>
__global__ void __launch_bounds__(kThreads) k_m2l_tc(int num_tiles, int64_t num_pairs, const int* __restrict__ pair_tgt,
                                                     const int* __restrict__ far_src, const int* __restrict__ seg_off,
                                                     const int4* __restrict__ segs, const float* __restrict__ mult,
                                                     const float4* __restrict__ centers, float* __restrict__ locals,
                                                     float* __restrict__ partials, int* __restrict__ status) {
  using PL = TcPlan<P>;
  constexpr int C = csize(P), CS = cstride(P), YS = C | 1;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  unsigned char* a_hi = sm;
  unsigned char* a_lo = sm + kAPartBytes;
  unsigned char* w_s = sm + 2 * kAPartBytes;
  float* ys = reinterpret_cast<float*>(sm);  // output rows alias the A parts once the last product is done
  __shared__ uint64_t s_mbar;
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5;

  // constant weight tiles -> shared memory (only K's when the others run in registers)
  {
    constexpr int w0 = KONLY ? PL::kGemmOff1 : 0;
    constexpr int w1 = KONLY ? PL::kGemmOff2 : PL::kWBytes;
    const uint4* src = reinterpret_cast<const uint4*>(PL::weights()) + w0 / 16;
    uint4* dst = reinterpret_cast<uint4*>(w_s);
    for (int k = tid; k < (w1 - w0) / 16; k += kThreads) dst[k] = src[k];
  }
  const uint32_t mbar = su32(&s_mbar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&s_tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t tmem_row = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t sa_hi = su32(a_hi), sa_lo = su32(a_lo);
  // tile offsets are relative to the whole weight array; with KONLY only K's
  // part is resident, so its base is shifted back by K's offset
  const uint32_t sw = su32(w_s) - (KONLY ? (uint32_t)PL::kGemmOff1 : 0u);
  uint32_t phase = 0;
  bool aborted = false;
  bool pending = false;  // a commit whose barrier phase has not been consumed

  for (int tile = blockIdx.x; tile < num_tiles && !aborted; tile += gridDim.x) {
    const int64_t e = (int64_t)tile * 128 + tid;
    const bool valid = e < num_pairs;
    float v[C];
    float caz = 1.f, saz = 0.f, cax = 1.f, sax = 0.f, s = 1.f;
    if (valid) {
      const int src = far_src[e], tgt = pair_tgt[e];
      const float4 ct = centers[tgt], cs = centers[src];
      const float dx = ct.x - cs.x, dy = ct.y - cs.y, dz = ct.z - cs.z;
      const float rho2 = dx * dx + dy * dy, r2 = rho2 + dz * dz;
      const float rho = sqrtf(rho2), r = sqrtf(r2);
      if (rho2 > 0.f) {
        const float ir = 1.f / rho;
        caz = dy * ir;
        saz = dx * ir;
      }
      if (r2 > 0.f) {
        const float ir = 1.f / r;
        cax = dz * ir;
        sax = rho * ir;
      }
      s = 1.f / fmaxf(r, 1.0e-30f);
      const float4* row = reinterpret_cast<const float4*>(mult + (size_t)src * CS);
#pragma unroll
      for (int k = 0; k < CS / 4; ++k) {
        const float4 q = __ldg(row + k);
        if (4 * k + 0 < C) v[4 * k + 0] = q.x;
        if (4 * k + 1 < C) v[4 * k + 1] = q.y;
        if (4 * k + 2 < C) v[4 * k + 2] = q.z;
        if (4 * k + 3 < C) v[4 * k + 3] = q.w;
      }
      dz_rot<P, false>(v, caz, saz);
    } else {
#pragma unroll
      for (int k = 0; k < C; ++k) v[k] = 0.f;
    }

    if (KONLY) {
      BApply<P, false>::apply(v);
    } else {
      // ---- product 1: B
      write_a<P, 0>(v, a_hi, a_lo, tid);
      fence_proxy_async();
      fence_before();
      __syncthreads();
      if (tid == 0) {
        fence_after();
        issue<P, 0>(tmem, sa_hi, sa_lo, sw);
        mma_commit(mbar);
      }
      pending = true;
      const bool ok1 = mbar_wait(mbar, phase);
      if (__syncthreads_or(!ok1)) {
        aborted = true;
        break;
      }
      phase ^= 1u;
      pending = false;
      fence_after();
      read_d<P, 0>(tmem_row, v);
    }
    dz_rot<P, true>(v, cax, sax);
    scale_degrees<P, 0>(v, s);

    // ---- product 2: K
    write_a<P, 1>(v, a_hi, a_lo, tid);
    fence_proxy_async();
    fence_before();
    __syncthreads();
    if (tid == 0) {
      fence_after();
      issue<P, 1>(tmem, sa_hi, sa_lo, sw);
      mma_commit(mbar);
    }
    pending = true;
    const bool ok2 = mbar_wait(mbar, phase);
    if (__syncthreads_or(!ok2)) {
      aborted = true;
      break;
    }
    phase ^= 1u;
    pending = false;
    fence_after();
    read_d<P, 1>(tmem_row, v);
    scale_degrees<P, 1>(v, s);
    dz_rot<P, false>(v, cax, sax);

    if (KONLY) {
      BApply<P, true>::apply(v);
    } else {
      // ---- product 3: B^T
      write_a<P, 2>(v, a_hi, a_lo, tid);
      fence_proxy_async();
      fence_before();
      __syncthreads();
      if (tid == 0) {
        fence_after();
        issue<P, 2>(tmem, sa_hi, sa_lo, sw);
        mma_commit(mbar);
      }
      pending = true;
      const bool ok3 = mbar_wait(mbar, phase);
      if (__syncthreads_or(!ok3)) {
        aborted = true;
        break;
      }
      phase ^= 1u;
      pending = false;
      fence_after();
      read_d<P, 2>(tmem_row, v);
    }
    dz_rot<P, true>(v, caz, saz);

    // ---- accumulate runs of equal target (rows of the tile are pairs in list order)
#pragma unroll
    for (int k = 0; k < C; ++k) ys[tid * YS + k] = v[k];
    __syncthreads();
    const int s0 = seg_off[tile], s1 = seg_off[tile + 1];
    if (tid < CS) {
      for (int sg = s0; sg < s1; ++sg) {
        const int4 S = segs[sg];
        float acc = 0.f;
        if (tid < C)
          for (int r = S.y; r < S.z; ++r) acc += ys[r * YS + tid];
        float* dst = (S.w < 0) ? locals + (size_t)S.x * CS : partials + (size_t)S.w * CS;
        dst[tid] = acc;
      }
    }
    fence_before();
    __syncthreads();
  }

  if (aborted) {
    if (tid == 0) atomicMax(status, 1);
    // drain the outstanding commit before TMEM is released (bounded as well);
    // status 2: the drain timed out too, so the MMA may still be writing the
    // TMEM freed below and the context must be treated as unusable
    if (pending && !mbar_wait(mbar, phase) && tid == 0) atomicMax(status, 2);
    fence_before();
  }
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

template <int P>
int run(int num_tiles, int64_t num_pairs, const int* pair_tgt, const int* far_src, const int* seg_off, const int* segs,
        const float* mult, const float* centers, float* locals, float* partials, int num_split, const int* split,
        int* status, bool konly, cudaStream_t st) {
  using PL = TcPlan<P>;
  const size_t wbytes = konly ? (size_t)(PL::kGemmOff2 - PL::kGemmOff1) : (size_t)PL::kWBytes;
  const size_t sm = 128 + 2 * (size_t)kAPartBytes + wbytes;
  static_assert(128 * (csize(P) | 1) * 4 <= 2 * kAPartBytes, "output rows must fit in the A region");
  auto kern = konly ? k_m2l_tc<P, true> : k_m2l_tc<P, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return cuda_status(e);
  if (num_tiles > 0) {
    // CTAs resident per SM: shared memory bound, and 128 TMEM columns each (<= 512)
    const int per_sm = sm <= 56 * 1024 ? 4 : 3;
    const int grid = num_tiles < 148 * per_sm ? num_tiles : 148 * per_sm;
    kern<<<grid, kThreads, sm, st>>>(num_tiles, num_pairs, pair_tgt, far_src, seg_off,
                                             reinterpret_cast<const int4*>(segs), mult,
                                             reinterpret_cast<const float4*>(centers), locals, partials, status);
    const int rc = launch_status();
    if (rc) return rc;
  }
  if (num_split > 0) {
    const int cs = cstride(P);
    k_m2l_reduce<<<(unsigned)(((int64_t)num_split * cs + 255) / 256), 256, 0, st>>>(
        num_split, reinterpret_cast<const int4*>(split), partials, locals, cs);
    return launch_status();
  }
  return JB_OK;
}


// Unit layout: thread t of a CTA owns work unit t of its group of 128 (at most
// 64 consecutive pairs of one target, the same units as k_m2l_units, sorted
// longest first so a group's units have similar lengths).  Step j of the
// group handles the j-th pair of every unit: each thread runs the rotations,
// B and B^T in registers, the K product of all 128 pairs is one set of
// tensor-core tiles (MMA row = thread), and the local accumulates in
// registers, so no cross-thread reduction is needed.  The next pair's source
// row is fetched with cp.async into a per-thread shared row while the current
// one is processed.
template <int P>
__global__ void __launch_bounds__(kThreads, 2) k_m2l_tc_units(int num_units, const int4* __restrict__ units,
                                                              const float* __restrict__ mult,
                                                              const float4* __restrict__ centers,
                                                              const int* __restrict__ far_src,
                                                              float* __restrict__ locals,
                                                              float* __restrict__ partials, int* __restrict__ status) {
  using PL = TcPlan<P>;
  constexpr int C = csize(P), CS = cstride(P), R4 = row4(P);
  constexpr int WB = PL::kGemmOff2 - PL::kGemmOff1;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  unsigned char* a_hi = sm;
  unsigned char* a_lo = sm + kAPartBytes;
  unsigned char* w_s = sm + 2 * kAPartBytes;
  float4* rows = reinterpret_cast<float4*>(w_s + WB);
  __shared__ uint64_t s_mbar;
  __shared__ uint32_t s_tmem;
  __shared__ int s_steps;
  const int tid = threadIdx.x, warp = tid >> 5;
  float4* row = rows + tid * R4;
  {
    const uint4* src = reinterpret_cast<const uint4*>(PL::weights()) + PL::kGemmOff1 / 16;
    uint4* dst = reinterpret_cast<uint4*>(w_s);
    for (int k = tid; k < WB / 16; k += kThreads) dst[k] = src[k];
  }
  const uint32_t mbar = su32(&s_mbar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(&s_tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = s_tmem;
  const uint32_t tmem_row = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t sa_hi = su32(a_hi), sa_lo = su32(a_lo);
  const uint32_t sw = su32(w_s) - (uint32_t)PL::kGemmOff1;
  uint32_t phase = 0;
  bool aborted = false, pending = false;
  const int num_groups = (num_units + kThreads - 1) / kThreads;

  for (int g = blockIdx.x; g < num_groups && !aborted; g += gridDim.x) {
    const int u = g * kThreads + tid;
    const bool has = u < num_units;
    const int4 U = has ? units[u] : make_int4(0, 0, 0, -1);
    const int len = U.z - U.y;
    // steps = the group's longest unit (units come sorted longest first, but
    // the maximum is taken anyway so any order is correct)
    if (tid == 0) s_steps = 0;
    __syncthreads();
    if (len > 0) atomicMax(&s_steps, len);
    __syncthreads();
    const int steps = s_steps;
    const float4 ct = has ? centers[U.x] : make_float4(0.f, 0.f, 0.f, 0.f);
    float acc[C];
#pragma unroll
    for (int k = 0; k < C; ++k) acc[k] = 0.f;
    int sidx = (len > 0) ? far_src[U.y] : 0;
    if (len > 0) {
      const float4* src = reinterpret_cast<const float4*>(mult + (size_t)sidx * CS);
#pragma unroll
      for (int k = 0; k < CS / 4; ++k) cp_async16(row + k, src + k);
      cp_async_commit();
    }
    float4 cs = (len > 0) ? centers[sidx] : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int j = 0; j < steps; ++j) {
      const bool act = j < len;
      float v[C];
      float caz = 1.f, saz = 0.f, cax = 1.f, sax = 0.f, s = 1.f;
      if (act) {
        cp_async_wait_all();
#pragma unroll
        for (int k = 0; k < CS / 4; ++k) {
          const float4 q = row[k];
          if (4 * k + 0 < C) v[4 * k + 0] = q.x;
          if (4 * k + 1 < C) v[4 * k + 1] = q.y;
          if (4 * k + 2 < C) v[4 * k + 2] = q.z;
          if (4 * k + 3 < C) v[4 * k + 3] = q.w;
        }
        const float dx = ct.x - cs.x, dy = ct.y - cs.y, dz = ct.z - cs.z;
        if (j + 1 < len) {
          sidx = __ldg(far_src + U.y + j + 1);
          const float4* src = reinterpret_cast<const float4*>(mult + (size_t)sidx * CS);
#pragma unroll
          for (int k = 0; k < CS / 4; ++k) cp_async16(row + k, src + k);
          cp_async_commit();
          cs = centers[sidx];
        }
        float r;
        align_cs(dx, dy, dz, caz, saz, cax, sax, r);
        s = 1.f / fmaxf(r, 1.0e-30f);
        dz_rot<P, false>(v, caz, saz);
        BApply<P, false>::apply(v);
        dz_rot<P, true>(v, cax, sax);
        scale_degrees<P, 0>(v, s);
      } else {
#pragma unroll
        for (int k = 0; k < C; ++k) v[k] = 0.f;
      }
      write_a<P, 1>(v, a_hi, a_lo, tid);
      fence_proxy_async();
      fence_before();
      __syncthreads();
      if (tid == 0) {
        fence_after();
        issue<P, 1>(tmem, sa_hi, sa_lo, sw);
        mma_commit(mbar);
      }
      pending = true;
      const bool ok = mbar_wait(mbar, phase);
      if (__syncthreads_or(!ok)) {
        aborted = true;
        break;
      }
      phase ^= 1u;
      pending = false;
      fence_after();
      read_d<P, 1>(tmem_row, v);
      if (act) {
        scale_degrees<P, 1>(v, s);
        dz_rot<P, false>(v, cax, sax);
        BApply<P, true>::apply(v);
        dz_rot<P, true>(v, caz, saz);
#pragma unroll
        for (int k = 0; k < C; ++k) acc[k] += v[k];
      }
    }
    if (aborted) break;
    if (has && len > 0) {
      float* dst = (U.w < 0) ? locals + (size_t)U.x * CS : partials + (size_t)U.w * CS;
#pragma unroll
      for (int k = 0; k < C; ++k) dst[k] = acc[k];
#pragma unroll
      for (int k = C; k < CS; ++k) dst[k] = 0.f;
    }
  }
  if (aborted) {
    if (tid == 0) atomicMax(status, 1);
    if (pending && !mbar_wait(mbar, phase) && tid == 0) atomicMax(status, 2);  // as in k_m2l_tc
  }
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

template <int P>
int run_units(int num_units, const int* units, const float* mult, const float* centers, const int* far_src,
              float* locals, float* partials, int num_split, const int* split, int* status, cudaStream_t st) {
  using PL = TcPlan<P>;
  const size_t sm = 128 + 2 * (size_t)kAPartBytes + (size_t)(PL::kGemmOff2 - PL::kGemmOff1) +
                    (size_t)kThreads * row4(P) * 16;
  cudaError_t e = cudaFuncSetAttribute(k_m2l_tc_units<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return cuda_status(e);
  if (num_units > 0) {
    const int groups = (num_units + kThreads - 1) / kThreads;
    const int grid = groups < 148 * 2 ? groups : 148 * 2;
    k_m2l_tc_units<P><<<grid, kThreads, sm, st>>>(num_units, reinterpret_cast<const int4*>(units), mult,
                                                   reinterpret_cast<const float4*>(centers), far_src, locals,
                                                   partials, status);
    const int rc = launch_status();
    if (rc) return rc;
  }
  if (num_split > 0) {
    const int cs = cstride(P);
    k_m2l_reduce<<<(unsigned)(((int64_t)num_split * cs + 255) / 256), 256, 0, st>>>(
        num_split, reinterpret_cast<const int4*>(split), partials, locals, cs);
    return launch_status();
  }
  return JB_OK;
}

}  // namespace tc
}  // namespace jb

extern "C" JB_API int jb_m2l_split(int p, int products, int num_tiles, int64_t num_pairs, const int* pair_tgt,
                                   const int* far_src, const int* seg_off, const int* segs, const float* mult,
                                   const float* centers, float* locals, float* partials, int num_split,
                                   const int* split, int* status, void* stream) {
  if ((products != 1 && products != 3) || num_tiles < 0 || num_pairs < 0 || num_split < 0 || !status ||
      (num_tiles > 0 && (!pair_tgt || !far_src || !seg_off || !segs || !mult || !centers || !locals)) ||
      (num_split > 0 && (!split || !partials)) || (int64_t)num_tiles * 128 < num_pairs)
    return JB_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  switch (p) {
#define JB_TC_CASE(PP) \
  case PP:             \
    return jb::tc::run<PP>(num_tiles, num_pairs, pair_tgt, far_src, seg_off, segs, mult, centers, locals, partials, \
                           num_split, split, status, products == 1, st);
    JB_TC_CASE(2) JB_TC_CASE(3) JB_TC_CASE(4) JB_TC_CASE(5) JB_TC_CASE(6) JB_TC_CASE(7) JB_TC_CASE(8)
#undef JB_TC_CASE
    default:
      return JB_ERR_UNSUPPORTED;
  }
}

extern "C" JB_API int jb_m2l_split_units(int p, int num_units, const int* units, const float* mult,
                                         const float* centers, const int* far_src, float* locals, float* partials,
                                         int num_split, const int* split, int* status, void* stream) {
  if (num_units < 0 || num_split < 0 || !status ||
      (num_units > 0 && (!units || !mult || !centers || !far_src || !locals)) ||
      (num_split > 0 && (!split || !partials || !locals)))
    return JB_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  switch (p) {
#define JB_TCU_CASE(PP) \
  case PP:              \
    return jb::tc::run_units<PP>(num_units, units, mult, centers, far_src, locals, partials, num_split, split, \
                                 status, st);
    JB_TCU_CASE(2) JB_TCU_CASE(3) JB_TCU_CASE(4) JB_TCU_CASE(5) JB_TCU_CASE(6) JB_TCU_CASE(7) JB_TCU_CASE(8)
#undef JB_TCU_CASE
    default:
      return JB_ERR_UNSUPPORTED;
  }
}
