#pragma once
// Device primitives of the GPU prepare (tree build, work-unit schedules):
// pool-backed device buffers, a three-kernel exclusive scan and a stable LSD
// radix sort of 64-bit keys.  Everything is in an anonymous namespace, so each
// translation unit that includes this has its own kernels; the memory pool is
// shared (jbdev::pool, defined in tree_gpu.cu).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/jaccpot_b200.h"

namespace jb {
int cuda_status(cudaError_t e);
}

namespace jbdev {
// Stream-ordered memory pool of the current device that keeps up to 4 GiB
// cached between calls.
cudaError_t pool(cudaMemPool_t* out);
}  // namespace jbdev

namespace {

constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------
// Device buffers owned by the builder / the handle, stream-ordered from a
// library memory pool per device that keeps up to 4 GiB cached between
// builds (a rebuild on a moved particle set allocates nothing new).
// ---------------------------------------------------------------------------
thread_local cudaStream_t tl_stream = nullptr;  // the stream of the build in progress on this thread

struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    bytes = 0;
  }
  cudaError_t alloc(size_t b) {
    release();
    if (b == 0) b = 16;
    cudaMemPool_t pool;
    cudaError_t e = jbdev::pool(&pool);
    if (e != cudaSuccess) return e;
    st = tl_stream;
    e = cudaMallocFromPoolAsync(&p, b, pool, st);
    if (e == cudaSuccess) bytes = b;
    else p = nullptr;
    return e;
  }
  // Grows to at least b bytes, keeping the first `keep` bytes (stream-ordered).
  cudaError_t grow(size_t b, size_t keep, cudaStream_t) {
    if (b <= bytes) return cudaSuccess;
    cudaMemPool_t pool;
    cudaError_t e = jbdev::pool(&pool);
    if (e != cudaSuccess) return e;
    void* q = nullptr;
    e = cudaMallocFromPoolAsync(&q, b, pool, tl_stream);
    if (e != cudaSuccess) return e;
    if (keep && p) {
      e = cudaMemcpyAsync(q, p, keep, cudaMemcpyDeviceToDevice, tl_stream);
      if (e != cudaSuccess) {
        cudaFreeAsync(q, tl_stream);
        return e;
      }
    }
    release();
    p = q;
    bytes = b;
    st = tl_stream;
    return cudaSuccess;
  }
  template <typename T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

struct Fail {
  int rc;
};

inline void ck(cudaError_t e) {
  if (e != cudaSuccess) throw Fail{jb::cuda_status(e)};
}
inline void ck_launch() { ck(cudaGetLastError()); }

inline unsigned nblocks(int64_t n, int per) { return (unsigned)std::max<int64_t>(1, (n + per - 1) / per); }

// ---------------------------------------------------------------------------
// Exclusive prefix sum: tiles of 4096 (1024 threads x 4), tile totals scanned
// recursively, then added back.
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 1024, kScanItems = 4, kScanTile = kScanThreads * kScanItems;

// Three counters scanned together (the dual walk's children / far / near).
struct I3 {
  int a, b, c;
};
__device__ __forceinline__ I3 operator+(I3 x, I3 y) { return I3{x.a + y.a, x.b + y.b, x.c + y.c}; }
__device__ __forceinline__ I3 operator-(I3 x, I3 y) { return I3{x.a - y.a, x.b - y.b, x.c - y.c}; }
template <typename T>
__device__ __forceinline__ T zero() {
  return T(0);
}
template <>
__device__ __forceinline__ I3 zero<I3>() {
  return I3{0, 0, 0};
}
template <typename T>
__device__ __forceinline__ T shfl_up(T v, int o) {
  return __shfl_up_sync(kFull, v, o);
}
template <>
__device__ __forceinline__ I3 shfl_up<I3>(I3 v, int o) {
  return I3{__shfl_up_sync(kFull, v.a, o), __shfl_up_sync(kFull, v.b, o), __shfl_up_sync(kFull, v.c, o)};
}

// Exclusive scan of one tile per block; the tile's sum goes to tile_sums
// (and to *total when the whole input is one tile).
template <typename T>
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const T* __restrict__ in, T* __restrict__ out,
                                                             T* __restrict__ tile_sums, T* __restrict__ total,
                                                             int64_t n) {
  __shared__ T warp_sums[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  T v[kScanItems];
  T s = zero<T>();
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    v[i] = (base + i < n) ? in[base + i] : zero<T>();
    s = s + v[i];
  }
  T incl = s;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = shfl_up<T>(incl, o);
    if (lane >= o) incl = incl + y;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const T w = warp_sums[lane];
    T wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = shfl_up<T>(wi, o);
      if (lane >= o) wi = wi + y;
    }
    warp_sums[lane] = wi - w;
  }
  __syncthreads();
  T run = warp_sums[warp] + incl - s;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i < n) out[base + i] = run;
    run = run + v[i];
  }
  if (threadIdx.x == kScanThreads - 1) {
    tile_sums[blockIdx.x] = run;
    if (total && gridDim.x == 1) *total = run;
  }
}

template <typename T>
__global__ void k_scan_add(T* __restrict__ out, const T* __restrict__ tile_off, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && i >= kScanTile) out[i] = out[i] + tile_off[i / kScanTile];
}

// ---------------------------------------------------------------------------
// LSD radix sort of 64-bit keys (optional int32 values), 8-bit digits.
// A block owns 2,048 consecutive keys; warp w owns 256 of them, in rounds of
// 32.  The scatter ranks a key among the same-digit keys before it by the
// warp's match mask, so equal digits keep their order (stable).
// ---------------------------------------------------------------------------
constexpr int kRsThreads = 256, kRsWarps = kRsThreads / 32, kRsRounds = 8, kRsTile = kRsThreads * kRsRounds;

__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const uint64_t* __restrict__ keys, int64_t n, int shift,
                                                        int* __restrict__ hist, int nblk) {
  __shared__ int cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * kRsTile + warp * (32 * kRsRounds);
#pragma unroll
  for (int r = 0; r < kRsRounds; ++r) {
    const int64_t i = base + r * 32 + lane;
    if (i < n) atomicAdd(&cnt[(int)((keys[i] >> shift) & 255u)], 1);
  }
  __syncthreads();
  hist[(int64_t)threadIdx.x * nblk + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const uint64_t* __restrict__ kin, const int* __restrict__ vin,
                                                           uint64_t* __restrict__ kout, int* __restrict__ vout, int64_t n,
                                                           int shift, const int* __restrict__ hist_off, int nblk) {
  __shared__ int wcnt[kRsWarps][256];
  for (int t = threadIdx.x; t < kRsWarps * 256; t += kRsThreads) (&wcnt[0][0])[t] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t base = (int64_t)blockIdx.x * kRsTile + warp * (32 * kRsRounds);
  uint64_t k[kRsRounds];
  int v[kRsRounds], d[kRsRounds];
#pragma unroll
  for (int r = 0; r < kRsRounds; ++r) {
    const int64_t i = base + r * 32 + lane;
    const bool ok = i < n;
    k[r] = ok ? kin[i] : 0ull;
    v[r] = (ok && vin) ? vin[i] : 0;
    d[r] = ok ? (int)((k[r] >> shift) & 255u) : 256;
    const unsigned peers = __match_any_sync(kFull, d[r]);
    if (d[r] < 256 && lane == __ffs(peers) - 1) wcnt[warp][d[r]] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {
    const int t = threadIdx.x;  // one digit per thread
    int run = hist_off[(int64_t)t * nblk + blockIdx.x];
#pragma unroll
    for (int w = 0; w < kRsWarps; ++w) {
      const int c = wcnt[w][t];
      wcnt[w][t] = run;
      run += c;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kRsRounds; ++r) {
    const unsigned peers = __match_any_sync(kFull, d[r]);
    if (d[r] < 256) {
      const int pos = wcnt[warp][d[r]] + __popc(peers & lt);
      kout[pos] = k[r];
      if (vout) vout[pos] = v[r];
    }
    __syncwarp();
    if (d[r] < 256 && lane == __ffs(peers) - 1) wcnt[warp][d[r]] += __popc(peers);
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Builder state.
// ---------------------------------------------------------------------------
struct Scratch {
  DBuf scan_tiles;  // tile sums of every recursion level
  DBuf total;       // 8 x int64 result words
  DBuf hist;        // radix histograms
};

// Tile-sum scratch of a scan of n elements: (2 * tiles + 8) words per
// recursion level.
template <typename T>
size_t scan_scratch_bytes(int64_t n) {
  size_t b = 0;
  while (n > 0) {
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    b += (size_t)(2 * tiles + 8) * sizeof(T);
    if (tiles <= 1) break;
    n = tiles;
  }
  return b;
}

template <typename T>
void scan_rec(const T* in, T* out, int64_t n, T* total, T* scratch, cudaStream_t st) {
  const int64_t tiles = (n + kScanTile - 1) / kScanTile;
  T* sums = scratch;
  T* sums_x = sums + tiles;
  k_scan_tiles<T><<<(unsigned)tiles, kScanThreads, 0, st>>>(in, out, sums, total, n);
  ck_launch();
  if (tiles > 1) {  // the tile sums' total is the total
    scan_rec<T>(sums, sums_x, tiles, total, sums + 2 * tiles + 8, st);
    k_scan_add<T><<<nblocks(n, 256), 256, 0, st>>>(out, sums_x, n);
    ck_launch();
  }
}

// out = exclusive prefix sum of in[0, n); *total (when given) = the sum.
template <typename T>
void exclusive_scan(const T* in, T* out, int64_t n, T* total, Scratch& s, cudaStream_t st) {
  if (n <= 0) {
    if (total) ck(cudaMemsetAsync(total, 0, sizeof(T), st));
    return;
  }
  const size_t need = scan_scratch_bytes<T>(n);
  if (need > s.scan_tiles.bytes) ck(s.scan_tiles.grow(std::max(need, 2 * s.scan_tiles.bytes), 0, st));
  scan_rec<T>(in, out, n, total, s.scan_tiles.as<T>(), st);
}

template <typename T>
T read_word(const T* d, cudaStream_t st) {
  T h;
  ck(cudaMemcpyAsync(&h, d, sizeof(T), cudaMemcpyDeviceToHost, st));
  ck(cudaStreamSynchronize(st));
  return h;
}

// Sorts keys[0, n) (and values) on bits [0, bits); the result is left in
// (k0, v0).  k1 / v1 are scratch of the same size.
void radix_sort(uint64_t* k0, int* v0, uint64_t* k1, int* v1, int64_t n, int bits, Scratch& s, cudaStream_t st) {
  if (n <= 1) return;
  const int nblk = (int)((n + kRsTile - 1) / kRsTile);
  const size_t hbytes = (size_t)256 * nblk * sizeof(int);
  if (s.hist.bytes < 2 * hbytes) ck(s.hist.alloc(2 * hbytes));
  int* hist = s.hist.as<int>();
  int* hoff = hist + (size_t)256 * nblk;
  const int passes = (bits + 7) / 8;
  for (int ps = 0; ps < passes; ++ps) {
    const int shift = 8 * ps;
    k_rs_hist<<<nblk, kRsThreads, 0, st>>>(k0, n, shift, hist, nblk);
    ck_launch();
    exclusive_scan<int>(hist, hoff, (int64_t)256 * nblk, nullptr, s, st);
    k_rs_scatter<<<nblk, kRsThreads, 0, st>>>(k0, v0, k1, v1, n, shift, hoff, nblk);
    ck_launch();
    std::swap(k0, k1);
    std::swap(v0, v1);
  }
  if (passes & 1) {  // result sits in the scratch pair: copy back
    ck(cudaMemcpyAsync(k1, k0, (size_t)n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
    if (v0 && v1) ck(cudaMemcpyAsync(v1, v0, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, st));
  }
}

}  // namespace
