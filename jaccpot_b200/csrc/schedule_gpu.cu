// Work-unit schedules built on the GPU from the device-resident lists: the
// same arrays, entry for entry, as the host builders in schedule.py
// (m2l_schedule, leaf_schedule, gear_m2l_schedule), which they replace at
// prepare time when the pass runs on a GPU.
//
// * M2L: the targets with far pairs, longest list first (stable), each list
//   cut into units of at most max_pairs consecutive pairs; units ordered by
//   decreasing length (stable); targets with more than one unit get
//   consecutive scratch slots (in target order) and a split entry.
// * Leaf evaluation: a target leaf's neighbour list cut where the running
//   source count crosses a multiple of max_sources; inside a unit, runs of
//   consecutive source leaves merge into one particle range; leaves without
//   neighbours get a unit of their own (self block + far field); a leaf's
//   units are numbered in list order for the slots, and all units are then
//   ordered by decreasing work (stable).
// * Gears: each target's far pairs regrouped by gear (stable), cut per
//   (target, gear) into units of at most max_pairs; slots numbered per target;
//   units ordered by gear, then decreasing length (stable).
// * Mixed gears (gear_m2l_mixed_schedule): each target's far pairs sorted by
//   order, highest first (stable), the list cut into units of at most
//   max_pairs with their segment bounds; slots numbered per target; units
//   ordered by decreasing segment lengths, highest order first (stable).
// Stable orders come from the LSD radix sort (keys with the index order as
// the tie-break), prefix sums from the tile scan of dev_prims.cuh; integer
// work only, and the only atomics are order-independent counts and maxima.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <new>
#include <vector>

#include "../../include/jaccpot_b200.h"
#include "dev_prims.cuh"

struct jb_dsched {
  jb_sched_info_t info{};
  DBuf units, aux, runs, split, far_src, gear_offsets, targets, pairs_per_gear;
};

namespace {

constexpr int kMaxLeafOcc = JB_MAX_LEAF_OCCUPANCY;

inline int bits_for(int64_t v) {  // bits to hold values in [0, v)
  int b = 1;
  while (b < 62 && ((int64_t)1 << b) < v) ++b;
  return b;
}

__global__ void k_iota(int* __restrict__ v, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = (int)i;
}

template <typename V>
__global__ void k_gather_rows(const V* __restrict__ src, const int* __restrict__ idx, int64_t n, V* __restrict__ dst) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

__global__ void k_row_counts(const int64_t* __restrict__ off, int rows, int64_t* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < rows) cnt[i] = off[i + 1] - off[i];
}

__global__ void k_max64(const int64_t* __restrict__ v, int64_t n, unsigned long long* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicMax(out, (unsigned long long)v[i]);
}

// Expands CSR offsets into the row of every entry (thread per row).
__global__ void k_expand_rows(const int64_t* __restrict__ off, int r0, int r1, int64_t base, int* __restrict__ row) {
  const int r = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= r1) return;
  for (int64_t e = off[r]; e < off[r + 1]; ++e) row[e - base] = r;
}

int* tot32(Scratch& s) { return reinterpret_cast<int*>(s.total.as<int64_t>() + 4); }

// ---------------------------------------------------------------------------
// M2L schedule.
// ---------------------------------------------------------------------------
__global__ void k_count_keys(const int64_t* __restrict__ cnt, int n, int64_t maxc, uint64_t* __restrict__ key) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) key[i] = (uint64_t)(maxc - cnt[i]);  // ascending key = descending count
}

__global__ void k_count_nonempty(const int64_t* __restrict__ cnt, int n, int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && cnt[i] > 0) atomicAdd(out, 1);
}

__global__ void k_flag_nonempty(const int* __restrict__ tg, int n, const int64_t* __restrict__ cnt, int* __restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = cnt[tg[i]] > 0 ? 1 : 0;
}

__global__ void k_compact(const int* __restrict__ src, int n, const int* __restrict__ flag, const int* __restrict__ pos,
                          int* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && flag[i]) dst[pos[i]] = src[i];
}

__global__ void k_m2l_nu(const int* __restrict__ tg, int T, const int64_t* __restrict__ cnt, int max_pairs,
                         int* __restrict__ nu, int* __restrict__ multi_nu, int* __restrict__ multi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T) return;
  const int u = (int)((cnt[tg[i]] + max_pairs - 1) / max_pairs);
  nu[i] = u;
  multi[i] = u > 1 ? 1 : 0;
  multi_nu[i] = u > 1 ? u : 0;
}

__global__ void k_m2l_emit(const int* __restrict__ tg, int T, const int64_t* __restrict__ off, int max_pairs,
                           const int* __restrict__ nu, const int* __restrict__ unit_off, const int* __restrict__ slot_base,
                           int4* __restrict__ units, uint64_t* __restrict__ key) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T) return;
  const int t = tg[i], n = nu[i];
  const int64_t a = off[t], b = off[t + 1];
  for (int k = 0; k < n; ++k) {
    const int u = unit_off[i] + k;
    const int64_t s = a + (int64_t)k * max_pairs, e = min(s + (int64_t)max_pairs, b);
    units[u] = make_int4(t, (int)s, (int)e, n > 1 ? slot_base[i] + k : -1);
    key[u] = (uint64_t)(max_pairs - (int)(e - s));
  }
}

__global__ void k_m2l_split(const int* __restrict__ tg, int T, const int* __restrict__ nu, const int* __restrict__ multi,
                            const int* __restrict__ split_pos, const int* __restrict__ slot_base,
                            int4* __restrict__ split) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < T && multi[i]) split[split_pos[i]] = make_int4(tg[i], slot_base[i], nu[i], 0);
}

void build_m2l(jb_dsched& d, int num_nodes, const int64_t* far_off, int max_pairs, int num_targets,
               const int* targets, cudaStream_t st) {
  Scratch s;
  ck(s.total.alloc(64));
  int* d_tot = tot32(s);
  DBuf cnt, tg;
  ck(cnt.alloc((size_t)std::max(num_nodes, 1) * 8));
  k_row_counts<<<nblocks(num_nodes, 256), 256, 0, st>>>(far_off, num_nodes, cnt.as<int64_t>());
  ck_launch();
  int T = 0;
  if (targets) {  // the caller's target list in its order, empty lists dropped
    DBuf flag, pos;
    const int n = std::max(num_targets, 1);
    ck(flag.alloc((size_t)n * 4));
    ck(pos.alloc((size_t)n * 4));
    ck(tg.alloc((size_t)n * 4));
    if (num_targets > 0) {
      k_flag_nonempty<<<nblocks(num_targets, 256), 256, 0, st>>>(targets, num_targets, cnt.as<int64_t>(),
                                                                   flag.as<int>());
      ck_launch();
      exclusive_scan<int>(flag.as<int>(), pos.as<int>(), num_targets, d_tot, s, st);
      T = read_word(d_tot, st);
      k_compact<<<nblocks(num_targets, 256), 256, 0, st>>>(targets, num_targets, flag.as<int>(), pos.as<int>(),
                                                           tg.as<int>());
      ck_launch();
    }
  } else if (num_nodes > 0) {  // every node with far pairs, longest list first (stable)
    DBuf mx, key0, key1, v1;
    ck(mx.alloc(8));
    ck(cudaMemsetAsync(mx.p, 0, 8, st));
    k_max64<<<nblocks(num_nodes, 256), 256, 0, st>>>(cnt.as<int64_t>(), num_nodes, mx.as<unsigned long long>());
    ck_launch();
    ck(cudaMemsetAsync(d_tot, 0, 4, st));
    k_count_nonempty<<<nblocks(num_nodes, 256), 256, 0, st>>>(cnt.as<int64_t>(), num_nodes, d_tot);
    ck_launch();
    const int64_t maxc = (int64_t)read_word(mx.as<unsigned long long>(), st);
    T = read_word(d_tot, st);
    ck(key0.alloc((size_t)num_nodes * 8));
    ck(key1.alloc((size_t)num_nodes * 8));
    ck(tg.alloc((size_t)num_nodes * 4));
    ck(v1.alloc((size_t)num_nodes * 4));
    k_count_keys<<<nblocks(num_nodes, 256), 256, 0, st>>>(cnt.as<int64_t>(), num_nodes, maxc, key0.as<uint64_t>());
    ck_launch();
    k_iota<<<nblocks(num_nodes, 256), 256, 0, st>>>(tg.as<int>(), num_nodes);
    ck_launch();
    radix_sort(key0.as<uint64_t>(), tg.as<int>(), key1.as<uint64_t>(), v1.as<int>(), num_nodes, bits_for(maxc + 1),
               s, st);
  }
  d.info.num_targets = T;
  ck(d.targets.alloc((size_t)std::max(T, 1) * 4));
  if (T == 0) {
    ck(d.units.alloc(16));
    ck(d.split.alloc(16));
    return;
  }
  ck(cudaMemcpyAsync(d.targets.p, tg.p, (size_t)T * 4, cudaMemcpyDeviceToDevice, st));
  DBuf nu, multi_nu, multi, unit_off, slot_base, split_pos;
  for (DBuf* b : {&nu, &multi_nu, &multi, &unit_off, &slot_base, &split_pos}) ck(b->alloc((size_t)T * 4));
  k_m2l_nu<<<nblocks(T, 256), 256, 0, st>>>(tg.as<int>(), T, cnt.as<int64_t>(), max_pairs, nu.as<int>(),
                                             multi_nu.as<int>(), multi.as<int>());
  ck_launch();
  exclusive_scan<int>(nu.as<int>(), unit_off.as<int>(), T, d_tot, s, st);
  exclusive_scan<int>(multi_nu.as<int>(), slot_base.as<int>(), T, d_tot + 1, s, st);
  exclusive_scan<int>(multi.as<int>(), split_pos.as<int>(), T, d_tot + 2, s, st);
  int tot[3];
  ck(cudaMemcpyAsync(tot, d_tot, sizeof(tot), cudaMemcpyDeviceToHost, st));
  ck(cudaStreamSynchronize(st));
  const int U = tot[0], S = tot[2];
  d.info.num_units = U;
  d.info.num_slots = tot[1];
  d.info.num_split = S;
  DBuf raw, k0, k1, idx0, idx1;
  ck(raw.alloc((size_t)U * 16));
  ck(k0.alloc((size_t)U * 8));
  ck(k1.alloc((size_t)U * 8));
  ck(idx0.alloc((size_t)U * 4));
  ck(idx1.alloc((size_t)U * 4));
  k_m2l_emit<<<nblocks(T, 128), 128, 0, st>>>(tg.as<int>(), T, far_off, max_pairs, nu.as<int>(), unit_off.as<int>(),
                                              slot_base.as<int>(), raw.as<int4>(), k0.as<uint64_t>());
  ck_launch();
  k_iota<<<nblocks(U, 256), 256, 0, st>>>(idx0.as<int>(), U);
  ck_launch();
  radix_sort(k0.as<uint64_t>(), idx0.as<int>(), k1.as<uint64_t>(), idx1.as<int>(), U, bits_for(max_pairs + 1), s, st);
  ck(d.units.alloc((size_t)U * 16));
  k_gather_rows<int4><<<nblocks(U, 256), 256, 0, st>>>(raw.as<int4>(), idx0.as<int>(), U, d.units.as<int4>());
  ck_launch();
  ck(d.split.alloc((size_t)std::max(S, 1) * 16));
  k_m2l_split<<<nblocks(T, 256), 256, 0, st>>>(tg.as<int>(), T, nu.as<int>(), multi.as<int>(), split_pos.as<int>(),
                                               slot_base.as<int>(), d.split.as<int4>());
  ck_launch();
  ck(cudaStreamSynchronize(st));
}

// ---------------------------------------------------------------------------
// Leaf schedule.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int leaf_count(const int* ranges, int num_internal, int j) {
  return ranges[2 * (num_internal + j) + 1] - ranges[2 * (num_internal + j)] + 1;
}

__global__ void k_edge_w(const int* __restrict__ near_src, int64_t e0, int64_t E, const int* __restrict__ ranges,
                         int num_internal, int64_t* __restrict__ w) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < E) w[e] = leaf_count(ranges, num_internal, near_src[e0 + e]);
}

// unit index of every edge inside its leaf, and the run breaks
__global__ void k_edge_uil(const int* __restrict__ tgt, const int* __restrict__ near_src, const int64_t* __restrict__ near_off,
                           int64_t e0, int64_t E, const int64_t* __restrict__ cs, int max_sources,
                           int* __restrict__ uil, int* __restrict__ brk) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const int t = tgt[e];
  const int64_t cum = cs[e] - cs[near_off[t] - e0];
  const int u = (int)(cum / max_sources);
  uil[e] = u;
  if (e == 0) {
    brk[e] = 1;
    return;
  }
  const int tp = tgt[e - 1];
  const int64_t cump = cs[e - 1] - cs[near_off[tp] - e0];
  const int up = (int)(cump / max_sources);
  brk[e] = (t != tp || u != up || near_src[e0 + e] != near_src[e0 + e - 1] + 1) ? 1 : 0;
}

__global__ void k_mark(const int* __restrict__ flag, const int* __restrict__ pos, int64_t n, int* __restrict__ first) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && flag[i]) first[pos[i]] = (int)i;
}

__global__ void k_run_fill(const int* __restrict__ rfirst, int R, int64_t E, const int64_t* __restrict__ cs,
                           int64_t total_w, const int* __restrict__ tgt, const int* __restrict__ uil,
                           const int* __restrict__ near_src, int64_t e0, const int* __restrict__ ranges, int num_internal,
                           int2* __restrict__ runs, int* __restrict__ run_tgt, int* __restrict__ run_uil,
                           int* __restrict__ ubrk) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= R) return;
  const int a = rfirst[r];
  const int64_t b = (r + 1 < R) ? rfirst[r + 1] : E;
  const int64_t end_cs = (b < E) ? cs[b] : total_w;
  runs[r] = make_int2(ranges[2 * (num_internal + near_src[e0 + a])], (int)(end_cs - cs[a]));
  run_tgt[r] = tgt[a];
  run_uil[r] = uil[a];
  ubrk[r] = (r == 0 || tgt[a] != tgt[rfirst[r - 1]] || uil[a] != uil[rfirst[r - 1]]) ? 1 : 0;
}

struct EdgeUnit {
  int leaf, rb, re, ns, first;
};

__global__ void k_edge_units(const int* __restrict__ ufirst, int Ue, int R, const int* __restrict__ rfirst, int64_t E,
                             const int64_t* __restrict__ cs, int64_t total_w, const int* __restrict__ run_tgt,
                             const int* __restrict__ run_uil, int lo, EdgeUnit* __restrict__ eu, int* __restrict__ n_per,
                             int* __restrict__ first_u) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= Ue) return;
  const int rb = ufirst[u], re = (u + 1 < Ue) ? ufirst[u + 1] : R;
  const int64_t ca = cs[rfirst[rb]], cb = (re < R) ? cs[rfirst[re]] : total_w;
  const int leaf = run_tgt[rb];
  eu[u] = EdgeUnit{leaf, rb, re, (int)(cb - ca), run_uil[rb] == 0 ? 1 : 0};
  atomicAdd(&n_per[leaf - lo], 1);
  if (u == 0 || run_tgt[ufirst[u - 1]] != leaf) first_u[leaf - lo] = u;
}

__global__ void k_lone(const int64_t* __restrict__ near_off, int lo, int hi, int* __restrict__ n_per) {
  const int j = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (j < hi && near_off[j + 1] == near_off[j]) n_per[j - lo] = 1;
}

__global__ void k_leaf_multi(const int* __restrict__ n_per, int NL, int* __restrict__ mnp, int* __restrict__ sflag) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= NL) return;
  mnp[j] = n_per[j] > 1 ? n_per[j] : 0;
  sflag[j] = n_per[j] > 1 ? 1 : 0;
}

__global__ void k_place_edge_units(const EdgeUnit* __restrict__ eu, int Ue, int lo, const int* __restrict__ base,
                                   const int* __restrict__ first_u, const int* __restrict__ n_per,
                                   const int* __restrict__ slot_base, const int* __restrict__ ranges, int num_internal,
                                   int4* __restrict__ units, int2* __restrict__ aux, int* __restrict__ work) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= Ue) return;
  const EdgeUnit x = eu[u];
  const int j = x.leaf - lo, k = u - first_u[j];
  const int pos = base[j] + k;
  units[pos] = make_int4(x.leaf, x.rb, x.re, x.ns);
  aux[pos] = make_int2(n_per[j] > 1 ? slot_base[j] + k : -1, x.first);
  work[pos] = x.ns + (x.first ? leaf_count(ranges, num_internal, x.leaf) : 0);
}

__global__ void k_place_lone(const int64_t* __restrict__ near_off, int lo, int hi, const int* __restrict__ base,
                             const int* __restrict__ ranges, int num_internal, int4* __restrict__ units,
                             int2* __restrict__ aux, int* __restrict__ work) {
  const int j = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= hi || near_off[j + 1] != near_off[j]) return;
  const int pos = base[j - lo];
  units[pos] = make_int4(j, 0, 0, 0);
  aux[pos] = make_int2(-1, 1);
  work[pos] = leaf_count(ranges, num_internal, j);
}

__global__ void k_max32(const int* __restrict__ v, int n, int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicMax(out, v[i]);
}

__global__ void k_work_keys(const int* __restrict__ work, int n, int maxw, uint64_t* __restrict__ key) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) key[i] = (uint64_t)(maxw - work[i]);
}

__global__ void k_leaf_split(int NL, int lo, const int* __restrict__ n_per, const int* __restrict__ spos,
                             const int* __restrict__ slot_base, int4* __restrict__ split) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < NL && n_per[j] > 1) split[spos[j]] = make_int4(lo + j, slot_base[j], n_per[j], 0);
}

// Largest leaf occupancy in [lo, hi) (atomicMax into *occ, zeroed first).
__global__ void k_leaf_max_occ(const int* __restrict__ ranges, int num_internal, int lo, int hi, int* __restrict__ occ) {
  const int j = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= hi) return;
  const int n = num_internal + j;
  atomicMax(occ, ranges[2 * n + 1] - ranges[2 * n] + 1);
}

void build_leaf(jb_dsched& d, int num_internal, const int* ranges, const int64_t* near_off, const int* near_src, int lo,
                int hi, int max_sources, cudaStream_t st) {
  Scratch s;
  ck(s.total.alloc(64));
  int* d_tot = tot32(s);
  int64_t* d_tot64 = s.total.as<int64_t>();
  const int NL = hi - lo;
  // the leaf kernels hold at most kMaxLeafOcc targets per leaf: refuse more
  if (NL > 0) {
    ck(cudaMemsetAsync(d_tot, 0, sizeof(int), st));
    k_leaf_max_occ<<<nblocks(NL, 256), 256, 0, st>>>(ranges, num_internal, lo, hi, d_tot);
    ck_launch();
    if (read_word(d_tot, st) > kMaxLeafOcc) throw Fail{JB_ERR_ARG};
  }
  int64_t ends[2] = {0, 0};
  ck(cudaMemcpyAsync(&ends[0], near_off + lo, 8, cudaMemcpyDeviceToHost, st));
  ck(cudaMemcpyAsync(&ends[1], near_off + hi, 8, cudaMemcpyDeviceToHost, st));
  ck(cudaStreamSynchronize(st));
  const int64_t e0 = ends[0], E = ends[1] - ends[0];
  DBuf tgt, w, cs, uil, brk, rpos, rfirst, runs_raw, run_tgt, run_uil, ubrk, upos, ufirst, eu, n_per, first_u;
  int R = 0, Ue = 0;
  int64_t total_w = 0;
  ck(n_per.alloc((size_t)std::max(NL, 1) * 4));
  ck(first_u.alloc((size_t)std::max(NL, 1) * 4));
  ck(cudaMemsetAsync(n_per.p, 0, (size_t)std::max(NL, 1) * 4, st));
  if (E > 0) {
    const size_t e = (size_t)E;
    ck(tgt.alloc(e * 4));
    ck(w.alloc(e * 8));
    ck(cs.alloc(e * 8));
    ck(uil.alloc(e * 4));
    ck(brk.alloc(e * 4));
    ck(rpos.alloc(e * 4));
    k_expand_rows<<<nblocks(NL, 128), 128, 0, st>>>(near_off, lo, hi, e0, tgt.as<int>());
    ck_launch();
    k_edge_w<<<nblocks(E, 256), 256, 0, st>>>(near_src, e0, E, ranges, num_internal, w.as<int64_t>());
    ck_launch();
    exclusive_scan<int64_t>(w.as<int64_t>(), cs.as<int64_t>(), E, d_tot64, s, st);
    k_edge_uil<<<nblocks(E, 256), 256, 0, st>>>(tgt.as<int>(), near_src, near_off, e0, E, cs.as<int64_t>(),
                                                max_sources, uil.as<int>(), brk.as<int>());
    ck_launch();
    exclusive_scan<int>(brk.as<int>(), rpos.as<int>(), E, d_tot, s, st);
    total_w = read_word(d_tot64, st);
    R = read_word(d_tot, st);
    ck(rfirst.alloc((size_t)R * 4));
    k_mark<<<nblocks(E, 256), 256, 0, st>>>(brk.as<int>(), rpos.as<int>(), E, rfirst.as<int>());
    ck_launch();
    ck(runs_raw.alloc((size_t)R * 8));
    ck(run_tgt.alloc((size_t)R * 4));
    ck(run_uil.alloc((size_t)R * 4));
    ck(ubrk.alloc((size_t)R * 4));
    ck(upos.alloc((size_t)R * 4));
    k_run_fill<<<nblocks(R, 256), 256, 0, st>>>(rfirst.as<int>(), R, E, cs.as<int64_t>(), total_w, tgt.as<int>(),
                                                uil.as<int>(), near_src, e0, ranges, num_internal, runs_raw.as<int2>(),
                                                run_tgt.as<int>(), run_uil.as<int>(), ubrk.as<int>());
    ck_launch();
    exclusive_scan<int>(ubrk.as<int>(), upos.as<int>(), R, d_tot, s, st);
    Ue = read_word(d_tot, st);
    ck(ufirst.alloc((size_t)Ue * 4));
    k_mark<<<nblocks(R, 256), 256, 0, st>>>(ubrk.as<int>(), upos.as<int>(), R, ufirst.as<int>());
    ck_launch();
    ck(eu.alloc((size_t)Ue * sizeof(EdgeUnit)));
    k_edge_units<<<nblocks(Ue, 256), 256, 0, st>>>(ufirst.as<int>(), Ue, R, rfirst.as<int>(), E, cs.as<int64_t>(),
                                                   total_w, run_tgt.as<int>(), run_uil.as<int>(), lo,
                                                   eu.as<EdgeUnit>(), n_per.as<int>(), first_u.as<int>());
    ck_launch();
  }
  ck(d.runs.alloc((size_t)std::max(R, 1) * 8));
  if (R > 0) ck(cudaMemcpyAsync(d.runs.p, runs_raw.p, (size_t)R * 8, cudaMemcpyDeviceToDevice, st));
  d.info.num_runs = R;
  if (NL <= 0) {
    ck(d.units.alloc(16));
    ck(d.aux.alloc(16));
    ck(d.split.alloc(16));
    ck(cudaStreamSynchronize(st));
    return;
  }
  k_lone<<<nblocks(NL, 256), 256, 0, st>>>(near_off, lo, hi, n_per.as<int>());
  ck_launch();
  DBuf base, mnp, sflag, slot_base, spos;
  for (DBuf* b : {&base, &mnp, &sflag, &slot_base, &spos}) ck(b->alloc((size_t)NL * 4));
  k_leaf_multi<<<nblocks(NL, 256), 256, 0, st>>>(n_per.as<int>(), NL, mnp.as<int>(), sflag.as<int>());
  ck_launch();
  exclusive_scan<int>(n_per.as<int>(), base.as<int>(), NL, d_tot, s, st);
  exclusive_scan<int>(mnp.as<int>(), slot_base.as<int>(), NL, d_tot + 1, s, st);
  exclusive_scan<int>(sflag.as<int>(), spos.as<int>(), NL, d_tot + 2, s, st);
  int tot[3];
  ck(cudaMemcpyAsync(tot, d_tot, sizeof(tot), cudaMemcpyDeviceToHost, st));
  ck(cudaStreamSynchronize(st));
  const int U = tot[0], S = tot[2];
  d.info.num_units = U;
  d.info.num_slots = tot[1];
  d.info.num_split = S;
  DBuf cu, ca, work, mx, k0, k1, idx0, idx1;
  ck(cu.alloc((size_t)U * 16));
  ck(ca.alloc((size_t)U * 8));
  ck(work.alloc((size_t)U * 4));
  if (Ue > 0) {
    k_place_edge_units<<<nblocks(Ue, 256), 256, 0, st>>>(eu.as<EdgeUnit>(), Ue, lo, base.as<int>(), first_u.as<int>(),
                                                         n_per.as<int>(), slot_base.as<int>(), ranges, num_internal,
                                                         cu.as<int4>(), ca.as<int2>(), work.as<int>());
    ck_launch();
  }
  k_place_lone<<<nblocks(NL, 256), 256, 0, st>>>(near_off, lo, hi, base.as<int>(), ranges, num_internal, cu.as<int4>(),
                                                 ca.as<int2>(), work.as<int>());
  ck_launch();
  ck(mx.alloc(4));
  ck(cudaMemsetAsync(mx.p, 0, 4, st));
  k_max32<<<nblocks(U, 256), 256, 0, st>>>(work.as<int>(), U, mx.as<int>());
  ck_launch();
  const int maxw = read_word(mx.as<int>(), st);
  ck(k0.alloc((size_t)U * 8));
  ck(k1.alloc((size_t)U * 8));
  ck(idx0.alloc((size_t)U * 4));
  ck(idx1.alloc((size_t)U * 4));
  k_work_keys<<<nblocks(U, 256), 256, 0, st>>>(work.as<int>(), U, maxw, k0.as<uint64_t>());
  ck_launch();
  k_iota<<<nblocks(U, 256), 256, 0, st>>>(idx0.as<int>(), U);
  ck_launch();
  radix_sort(k0.as<uint64_t>(), idx0.as<int>(), k1.as<uint64_t>(), idx1.as<int>(), U, bits_for((int64_t)maxw + 1), s,
             st);
  ck(d.units.alloc((size_t)U * 16));
  ck(d.aux.alloc((size_t)U * 8));
  k_gather_rows<int4><<<nblocks(U, 256), 256, 0, st>>>(cu.as<int4>(), idx0.as<int>(), U, d.units.as<int4>());
  ck_launch();
  k_gather_rows<int2><<<nblocks(U, 256), 256, 0, st>>>(ca.as<int2>(), idx0.as<int>(), U, d.aux.as<int2>());
  ck_launch();
  ck(d.split.alloc((size_t)std::max(S, 1) * 16));
  k_leaf_split<<<nblocks(NL, 256), 256, 0, st>>>(NL, lo, n_per.as<int>(), spos.as<int>(), slot_base.as<int>(),
                                                 d.split.as<int4>());
  ck_launch();
  ck(cudaStreamSynchronize(st));
}

// ---------------------------------------------------------------------------
// Gear schedule.
// ---------------------------------------------------------------------------
// A gear outside [0, num_gears) is counted in *bad and sorts as gear 0 (the
// call then fails with JB_ERR_INDEX).
// Per-gear pair counts go through a shared-memory histogram (one global add
// per block and gear), since every pair hits one of a few counters.
__global__ void __launch_bounds__(256) k_gear_keys(const int* __restrict__ row, const int* __restrict__ gears, int64_t P,
                                                   int gb, int num_gears, uint64_t* __restrict__ key,
                                                   unsigned long long* __restrict__ ppg, int* __restrict__ bad) {
  __shared__ unsigned int hist[64];
  if (threadIdx.x < 64) hist[threadIdx.x] = 0;
  __syncthreads();
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < P) {
    int g = gears[e];
    if (g < 0 || g >= num_gears) {
      atomicAdd(bad, 1);
      g = 0;
    }
    key[e] = ((uint64_t)row[e] << gb) | (uint64_t)g;
    atomicAdd(&hist[g], 1u);
  }
  __syncthreads();
  if ((int)threadIdx.x < num_gears && hist[threadIdx.x]) atomicAdd(&ppg[threadIdx.x], (unsigned long long)hist[threadIdx.x]);
}

__global__ void k_seg_brk(const uint64_t* __restrict__ key, int64_t P, int* __restrict__ brk) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < P) brk[i] = (i == 0 || key[i] != key[i - 1]) ? 1 : 0;
}

__global__ void k_seg_nu(const int* __restrict__ sfirst, int NS, int64_t P, int max_pairs, int* __restrict__ nu) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NS) return;
  const int64_t a = sfirst[i], b = (i + 1 < NS) ? sfirst[i + 1] : P;
  nu[i] = (int)((b - a + max_pairs - 1) / max_pairs);
}

struct GearUnit {
  int t, g, s, e;
};

__global__ void __launch_bounds__(128) k_gear_units(const int* __restrict__ sfirst, int NS, int64_t P,
                                                    const uint64_t* __restrict__ key, int gb, int max_pairs,
                                                    const int* __restrict__ nu, const int* __restrict__ unit_off,
                                                    GearUnit* __restrict__ gu, int* __restrict__ n_per,
                                                    int* __restrict__ tfirst, int* __restrict__ gcount) {
  __shared__ int hist[64];
  if (threadIdx.x < 64) hist[threadIdx.x] = 0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < NS) {
    const int64_t a = sfirst[i], b = (i + 1 < NS) ? sfirst[i + 1] : P;
    const uint64_t k = key[a];
    const int t = (int)(k >> gb), g = (int)(k & ((1ull << gb) - 1));
    const int n = nu[i];
    const bool first_seg_of_target = (i == 0) || (int)(key[sfirst[i - 1]] >> gb) != t;
    if (first_seg_of_target) tfirst[t] = unit_off[i];
    for (int q = 0; q < n; ++q) {
      const int64_t s = a + (int64_t)q * max_pairs, e = min(s + (int64_t)max_pairs, b);
      gu[unit_off[i] + q] = GearUnit{t, g, (int)s, (int)e};
    }
    atomicAdd(&n_per[t], n);
    atomicAdd(&hist[g], n);
  }
  __syncthreads();
  if (threadIdx.x < 64 && hist[threadIdx.x]) atomicAdd(&gcount[threadIdx.x], hist[threadIdx.x]);
}

__global__ void k_node_multi(const int* __restrict__ n_per, int nodes, int* __restrict__ mnp, int* __restrict__ sflag) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nodes) return;
  mnp[t] = n_per[t] > 1 ? n_per[t] : 0;
  sflag[t] = n_per[t] > 1 ? 1 : 0;
}

__global__ void k_gear_emit(const GearUnit* __restrict__ gu, int U, const int* __restrict__ n_per,
                            const int* __restrict__ tfirst, const int* __restrict__ slot_base, int max_pairs, int lb,
                            int4* __restrict__ units, uint64_t* __restrict__ key) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= U) return;
  const GearUnit x = gu[u];
  const int slot = n_per[x.t] > 1 ? slot_base[x.t] + (u - tfirst[x.t]) : -1;
  units[u] = make_int4(x.t, x.s, x.e, slot);
  key[u] = ((uint64_t)x.g << lb) | (uint64_t)(max_pairs - (x.e - x.s));
}

__global__ void k_node_split(int nodes, const int* __restrict__ n_per, const int* __restrict__ spos,
                             const int* __restrict__ slot_base, int4* __restrict__ split) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nodes && n_per[t] > 1) split[spos[t]] = make_int4(t, slot_base[t], n_per[t], 0);
}

void build_gears(jb_dsched& d, int num_nodes, const int64_t* far_off, const int* far_src, const int* gears,
                 int num_gears, int max_pairs, cudaStream_t st) {
  Scratch s;
  ck(s.total.alloc(64));
  int* d_tot = tot32(s);
  int64_t P = 0;
  ck(cudaMemcpyAsync(&P, far_off + num_nodes, 8, cudaMemcpyDeviceToHost, st));
  ck(cudaStreamSynchronize(st));
  const int gb = bits_for(num_gears);
  ck(d.pairs_per_gear.alloc((size_t)num_gears * 8));
  ck(cudaMemsetAsync(d.pairs_per_gear.p, 0, (size_t)num_gears * 8, st));
  ck(d.gear_offsets.alloc((size_t)(num_gears + 1) * 8));
  ck(d.far_src.alloc((size_t)std::max<int64_t>(P, 1) * 4));
  if (P == 0) {
    ck(cudaMemsetAsync(d.gear_offsets.p, 0, (size_t)(num_gears + 1) * 8, st));
    ck(d.units.alloc(16));
    ck(d.split.alloc(16));
    ck(cudaStreamSynchronize(st));
    return;
  }
  DBuf row, k0, k1, v0, v1, brk, spos, sfirst, nu, unit_off;
  ck(row.alloc((size_t)P * 4));
  k_expand_rows<<<nblocks(num_nodes, 128), 128, 0, st>>>(far_off, 0, num_nodes, 0, row.as<int>());
  ck_launch();
  ck(k0.alloc((size_t)P * 8));
  ck(k1.alloc((size_t)P * 8));
  ck(v0.alloc((size_t)P * 4));
  ck(v1.alloc((size_t)P * 4));
  ck(cudaMemsetAsync(d_tot + 3, 0, 4, st));
  k_gear_keys<<<nblocks(P, 256), 256, 0, st>>>(row.as<int>(), gears, P, gb, num_gears, k0.as<uint64_t>(),
                                               d.pairs_per_gear.as<unsigned long long>(), d_tot + 3);
  ck_launch();
  if (read_word(d_tot + 3, st) != 0) throw Fail{JB_ERR_INDEX};
  k_iota<<<nblocks(P, 256), 256, 0, st>>>(v0.as<int>(), P);
  ck_launch();
  radix_sort(k0.as<uint64_t>(), v0.as<int>(), k1.as<uint64_t>(), v1.as<int>(), P, bits_for(num_nodes) + gb, s, st);
  k_gather_rows<int><<<nblocks(P, 256), 256, 0, st>>>(far_src, v0.as<int>(), P, d.far_src.as<int>());
  ck_launch();
  row.release();
  k1.release();
  v1.release();
  ck(brk.alloc((size_t)P * 4));
  ck(spos.alloc((size_t)P * 4));
  k_seg_brk<<<nblocks(P, 256), 256, 0, st>>>(k0.as<uint64_t>(), P, brk.as<int>());
  ck_launch();
  exclusive_scan<int>(brk.as<int>(), spos.as<int>(), P, d_tot, s, st);
  const int NS = read_word(d_tot, st);
  ck(sfirst.alloc((size_t)NS * 4));
  k_mark<<<nblocks(P, 256), 256, 0, st>>>(brk.as<int>(), spos.as<int>(), P, sfirst.as<int>());
  ck_launch();
  brk.release();
  spos.release();
  ck(nu.alloc((size_t)NS * 4));
  ck(unit_off.alloc((size_t)NS * 4));
  k_seg_nu<<<nblocks(NS, 256), 256, 0, st>>>(sfirst.as<int>(), NS, P, max_pairs, nu.as<int>());
  ck_launch();
  exclusive_scan<int>(nu.as<int>(), unit_off.as<int>(), NS, d_tot, s, st);
  const int U = read_word(d_tot, st);
  DBuf gu, n_per, tfirst, gcount, mnp, sflag, slot_base, spos2;
  ck(gu.alloc((size_t)U * sizeof(GearUnit)));
  for (DBuf* b : {&n_per, &tfirst, &mnp, &sflag, &slot_base, &spos2}) ck(b->alloc((size_t)num_nodes * 4));
  ck(gcount.alloc((size_t)(num_gears + 1) * 8));
  ck(cudaMemsetAsync(n_per.p, 0, (size_t)num_nodes * 4, st));
  ck(cudaMemsetAsync(gcount.p, 0, (size_t)(num_gears + 1) * 8, st));
  k_gear_units<<<nblocks(NS, 128), 128, 0, st>>>(sfirst.as<int>(), NS, P, k0.as<uint64_t>(), gb, max_pairs,
                                                 nu.as<int>(), unit_off.as<int>(), gu.as<GearUnit>(), n_per.as<int>(),
                                                 tfirst.as<int>(), gcount.as<int>());
  ck_launch();
  k_node_multi<<<nblocks(num_nodes, 256), 256, 0, st>>>(n_per.as<int>(), num_nodes, mnp.as<int>(), sflag.as<int>());
  ck_launch();
  exclusive_scan<int>(mnp.as<int>(), slot_base.as<int>(), num_nodes, d_tot, s, st);
  exclusive_scan<int>(sflag.as<int>(), spos2.as<int>(), num_nodes, d_tot + 1, s, st);
  int tot[2];
  ck(cudaMemcpyAsync(tot, d_tot, sizeof(tot), cudaMemcpyDeviceToHost, st));
  ck(cudaStreamSynchronize(st));
  const int S = tot[1];
  d.info.num_units = U;
  d.info.num_slots = tot[0];
  d.info.num_split = S;
  // gear offsets: exclusive sums of the per-gear unit counts (int32 counts
  // widened by a scan over int64 copies)
  {
    std::vector<int> gc((size_t)num_gears + 1, 0);
    ck(cudaMemcpyAsync(gc.data(), gcount.p, (size_t)num_gears * 4, cudaMemcpyDeviceToHost, st));
    ck(cudaStreamSynchronize(st));
    std::vector<int64_t> go((size_t)num_gears + 1, 0);
    for (int g = 0; g < num_gears; ++g) go[(size_t)g + 1] = go[(size_t)g] + gc[(size_t)g];
    ck(cudaMemcpyAsync(d.gear_offsets.p, go.data(), go.size() * 8, cudaMemcpyHostToDevice, st));
    ck(cudaStreamSynchronize(st));
  }
  DBuf raw, uk0, uk1, idx0, idx1;
  ck(raw.alloc((size_t)U * 16));
  ck(uk0.alloc((size_t)U * 8));
  ck(uk1.alloc((size_t)U * 8));
  ck(idx0.alloc((size_t)U * 4));
  ck(idx1.alloc((size_t)U * 4));
  const int lb = bits_for(max_pairs + 1);
  k_gear_emit<<<nblocks(U, 256), 256, 0, st>>>(gu.as<GearUnit>(), U, n_per.as<int>(), tfirst.as<int>(),
                                               slot_base.as<int>(), max_pairs, lb, raw.as<int4>(), uk0.as<uint64_t>());
  ck_launch();
  k_iota<<<nblocks(U, 256), 256, 0, st>>>(idx0.as<int>(), U);
  ck_launch();
  radix_sort(uk0.as<uint64_t>(), idx0.as<int>(), uk1.as<uint64_t>(), idx1.as<int>(), U, lb + gb, s, st);
  ck(d.units.alloc((size_t)U * 16));
  k_gather_rows<int4><<<nblocks(U, 256), 256, 0, st>>>(raw.as<int4>(), idx0.as<int>(), U, d.units.as<int4>());
  ck_launch();
  ck(d.split.alloc((size_t)std::max(S, 1) * 16));
  k_node_split<<<nblocks(num_nodes, 256), 256, 0, st>>>(num_nodes, n_per.as<int>(), spos2.as<int>(),
                                                        slot_base.as<int>(), d.split.as<int4>());
  ck_launch();
  ck(cudaStreamSynchronize(st));
}

// ---------------------------------------------------------------------------
// Mixed gear schedule (jb_m2l_mixed): each target's pairs sorted by segment
// (order, highest first; stable inside), the whole list cut into units of at
// most max_pairs, each unit's segment bounds read off the sorted keys.
// ---------------------------------------------------------------------------
constexpr int kMixedSegMax = JB_MIXED_GEAR_SEGMENTS;

struct GearSegments {
  int seg[64];  // segment of each gear index
};

__global__ void __launch_bounds__(256) k_mixed_keys(const int* __restrict__ row, const int* __restrict__ gears,
                                                    int64_t P, int num_gears, GearSegments gs,
                                                    uint64_t* __restrict__ key, unsigned long long* __restrict__ ppg,
                                                    int* __restrict__ bad) {
  __shared__ unsigned int hist[64];
  if (threadIdx.x < 64) hist[threadIdx.x] = 0;
  __syncthreads();
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e < P) {
    int g = gears[e];
    if (g < 0 || g >= num_gears) {
      atomicAdd(bad, 1);
      g = 0;
    }
    key[e] = ((uint64_t)row[e] << 2) | (uint64_t)gs.seg[g];
    atomicAdd(&hist[g], 1u);
  }
  __syncthreads();
  if ((int)threadIdx.x < num_gears && hist[threadIdx.x]) atomicAdd(&ppg[threadIdx.x], (unsigned long long)hist[threadIdx.x]);
}

__global__ void k_mixed_nu(const int64_t* __restrict__ off, int nodes, int max_pairs, int* __restrict__ nu,
                           int* __restrict__ mnp, int* __restrict__ sflag) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nodes) return;
  const int u = (int)((off[t + 1] - off[t] + max_pairs - 1) / max_pairs);
  nu[t] = u;
  mnp[t] = u > 1 ? u : 0;
  sflag[t] = u > 1 ? 1 : 0;
}

// Thread per target: the segment starts by binary search in its sorted keys
// (the low two bits, non-decreasing inside a row), then its units.
__global__ void k_mixed_emit(const int64_t* __restrict__ off, int nodes, const uint64_t* __restrict__ key,
                             int max_pairs, int nb, const int* __restrict__ nu, const int* __restrict__ unit_off,
                             const int* __restrict__ slot_base, int4* __restrict__ units, int4* __restrict__ bounds,
                             uint64_t* __restrict__ ukey) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nodes) return;
  const int a = (int)off[t], b = (int)off[t + 1];
  if (a == b) return;
  int sb[kMixedSegMax + 1];
  sb[0] = a;
  sb[kMixedSegMax] = b;
  for (int j = 1; j < kMixedSegMax; ++j) {
    int lo = a, hi = b;
    while (lo < hi) {
      const int mid = lo + (hi - lo) / 2;
      if ((int)(key[mid] & 3u) < j) lo = mid + 1;
      else hi = mid;
    }
    sb[j] = lo;
  }
  const int n = nu[t];
  for (int q = 0; q < n; ++q) {
    const int u = unit_off[t] + q;
    const int s = a + q * max_pairs, e = min(s + max_pairs, b);
    int bd[kMixedSegMax + 1];
    bd[0] = s;
    bd[kMixedSegMax] = e;
    for (int j = 1; j < kMixedSegMax; ++j) bd[j] = min(max(sb[j], s), e);
    units[u] = make_int4(t, s, e, n > 1 ? slot_base[t] + q : -1);
    bounds[u] = make_int4(bd[1], bd[2], bd[3], e);
    uint64_t k = 0;
    for (int j = 0; j < kMixedSegMax; ++j) k = (k << nb) | (uint64_t)(max_pairs - (bd[j + 1] - bd[j]));
    ukey[u] = k;
  }
}

void build_gears_mixed(jb_dsched& d, int num_nodes, const int64_t* far_off, const int* far_src, const int* gears,
                       int num_gears, const GearSegments& gs, int max_pairs, cudaStream_t st) {
  Scratch s;
  ck(s.total.alloc(64));
  int* d_tot = tot32(s);
  int64_t P = 0;
  ck(cudaMemcpyAsync(&P, far_off + num_nodes, 8, cudaMemcpyDeviceToHost, st));
  ck(cudaStreamSynchronize(st));
  if (P > (int64_t)0x7fffffff - max_pairs) throw Fail{JB_ERR_ARG};  // unit bounds are int32
  ck(d.pairs_per_gear.alloc((size_t)num_gears * 8));
  ck(cudaMemsetAsync(d.pairs_per_gear.p, 0, (size_t)num_gears * 8, st));
  ck(d.far_src.alloc((size_t)std::max<int64_t>(P, 1) * 4));
  if (P == 0) {
    ck(d.units.alloc(16));
    ck(d.aux.alloc(16));
    ck(d.split.alloc(16));
    ck(cudaStreamSynchronize(st));
    return;
  }
  DBuf row, k0, k1, v0, v1;
  ck(row.alloc((size_t)P * 4));
  k_expand_rows<<<nblocks(num_nodes, 128), 128, 0, st>>>(far_off, 0, num_nodes, 0, row.as<int>());
  ck_launch();
  ck(k0.alloc((size_t)P * 8));
  ck(k1.alloc((size_t)P * 8));
  ck(v0.alloc((size_t)P * 4));
  ck(v1.alloc((size_t)P * 4));
  ck(cudaMemsetAsync(d_tot + 3, 0, 4, st));
  k_mixed_keys<<<nblocks(P, 256), 256, 0, st>>>(row.as<int>(), gears, P, num_gears, gs, k0.as<uint64_t>(),
                                                d.pairs_per_gear.as<unsigned long long>(), d_tot + 3);
  ck_launch();
  if (read_word(d_tot + 3, st) != 0) throw Fail{JB_ERR_INDEX};
  k_iota<<<nblocks(P, 256), 256, 0, st>>>(v0.as<int>(), P);
  ck_launch();
  radix_sort(k0.as<uint64_t>(), v0.as<int>(), k1.as<uint64_t>(), v1.as<int>(), P, bits_for(num_nodes) + 2, s, st);
  k_gather_rows<int><<<nblocks(P, 256), 256, 0, st>>>(far_src, v0.as<int>(), P, d.far_src.as<int>());
  ck_launch();
  row.release();
  k1.release();
  v1.release();
  v0.release();
  DBuf nu, mnp, sflag, unit_off, slot_base, spos;
  for (DBuf* b : {&nu, &mnp, &sflag, &unit_off, &slot_base, &spos}) ck(b->alloc((size_t)std::max(num_nodes, 1) * 4));
  k_mixed_nu<<<nblocks(num_nodes, 256), 256, 0, st>>>(far_off, num_nodes, max_pairs, nu.as<int>(), mnp.as<int>(),
                                                     sflag.as<int>());
  ck_launch();
  exclusive_scan<int>(nu.as<int>(), unit_off.as<int>(), num_nodes, d_tot, s, st);
  exclusive_scan<int>(mnp.as<int>(), slot_base.as<int>(), num_nodes, d_tot + 1, s, st);
  exclusive_scan<int>(sflag.as<int>(), spos.as<int>(), num_nodes, d_tot + 2, s, st);
  int tot[3];
  ck(cudaMemcpyAsync(tot, d_tot, sizeof(tot), cudaMemcpyDeviceToHost, st));
  ck(cudaStreamSynchronize(st));
  const int U = tot[0], S = tot[2];
  d.info.num_units = U;
  d.info.num_slots = tot[1];
  d.info.num_split = S;
  const int nb = bits_for(max_pairs + 1);
  DBuf raw_u, raw_b, uk0, uk1, idx0, idx1;
  ck(raw_u.alloc((size_t)U * 16));
  ck(raw_b.alloc((size_t)U * 16));
  ck(uk0.alloc((size_t)U * 8));
  ck(uk1.alloc((size_t)U * 8));
  ck(idx0.alloc((size_t)U * 4));
  ck(idx1.alloc((size_t)U * 4));
  k_mixed_emit<<<nblocks(num_nodes, 128), 128, 0, st>>>(far_off, num_nodes, k0.as<uint64_t>(), max_pairs, nb,
                                                       nu.as<int>(), unit_off.as<int>(), slot_base.as<int>(),
                                                       raw_u.as<int4>(), raw_b.as<int4>(), uk0.as<uint64_t>());
  ck_launch();
  k0.release();
  k_iota<<<nblocks(U, 256), 256, 0, st>>>(idx0.as<int>(), U);
  ck_launch();
  radix_sort(uk0.as<uint64_t>(), idx0.as<int>(), uk1.as<uint64_t>(), idx1.as<int>(), U, kMixedSegMax * nb, s, st);
  ck(d.units.alloc((size_t)U * 16));
  ck(d.aux.alloc((size_t)U * 16));
  k_gather_rows<int4><<<nblocks(U, 256), 256, 0, st>>>(raw_u.as<int4>(), idx0.as<int>(), U, d.units.as<int4>());
  ck_launch();
  k_gather_rows<int4><<<nblocks(U, 256), 256, 0, st>>>(raw_b.as<int4>(), idx0.as<int>(), U, d.aux.as<int4>());
  ck_launch();
  ck(d.split.alloc((size_t)std::max(S, 1) * 16));
  k_node_split<<<nblocks(num_nodes, 256), 256, 0, st>>>(num_nodes, nu.as<int>(), spos.as<int>(), slot_base.as<int>(),
                                                        d.split.as<int4>());
  ck_launch();
  ck(cudaStreamSynchronize(st));
}

// ---------------------------------------------------------------------------
// Reverse index of a symmetric far list: rev[e] for the pair e = (t <- s) is
// the entry (s <- t), found by binary search in row s (rows are sorted).
// Thread per row; a missing reverse is counted in *bad.
// ---------------------------------------------------------------------------
__global__ void k_far_reverse(const int64_t* __restrict__ off, int num_nodes, const int* __restrict__ src,
                              int* __restrict__ rev, int* __restrict__ bad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= num_nodes) return;
  for (int64_t e = off[t]; e < off[t + 1]; ++e) {
    const int s = src[e];
    int64_t lo = off[s], hi = off[s + 1];
    while (lo < hi) {
      const int64_t mid = lo + (hi - lo) / 2;
      if (src[mid] < t) lo = mid + 1;
      else hi = mid;
    }
    if (lo < off[s + 1] && src[lo] == t) {
      rev[e] = (int)lo;
    } else {
      rev[e] = -1;
      atomicAdd(bad, 1);
    }
  }
}

const DBuf* sched_field(const jb_dsched* d, int field) {
  switch (field) {
    case JB_SCHED_UNITS: return &d->units;
    case JB_SCHED_AUX: return &d->aux;
    case JB_SCHED_RUNS: return &d->runs;
    case JB_SCHED_SPLIT: return &d->split;
    case JB_SCHED_FAR_SOURCES: return &d->far_src;
    case JB_SCHED_GEAR_OFFSETS: return &d->gear_offsets;
    case JB_SCHED_TARGETS: return &d->targets;
    case JB_SCHED_PAIRS_PER_GEAR: return &d->pairs_per_gear;
    default: return nullptr;
  }
}

template <typename F>
int run_builder(jb_dsched** out, cudaStream_t st, F&& fn) {
  if (!out) return JB_ERR_ARG;
  *out = nullptr;
  jb_dsched* d = new (std::nothrow) jb_dsched();
  if (!d) return JB_ERR_ALLOC;
  tl_stream = st;
  try {
    fn(*d);
  } catch (const Fail& f) {
    delete d;
    return f.rc;
  } catch (const std::bad_alloc&) {
    delete d;
    return JB_ERR_ALLOC;
  }
  *out = d;
  return JB_OK;
}

}  // namespace

extern "C" {

JB_API int jb_m2l_schedule_device(int num_nodes, const int64_t* far_off, int max_pairs, int num_targets,
                                  const int* targets, void* stream, jb_dsched** out) {
  if (num_nodes < 0 || !far_off || max_pairs < 1 || (targets && num_targets < 0)) return JB_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return run_builder(out, st, [&](jb_dsched& d) {
    build_m2l(d, num_nodes, far_off, max_pairs, num_targets, targets, st);
  });
}

JB_API int jb_leaf_schedule_device(int num_internal, int num_leaves, const int* node_ranges, const int64_t* near_off,
                                   const int* near_src, int leaf_lo, int leaf_hi, int max_sources, void* stream,
                                   jb_dsched** out) {
  if (num_internal < 0 || num_leaves < 0 || !node_ranges || !near_off || !near_src || leaf_lo < 0 ||
      leaf_hi < leaf_lo || leaf_hi > num_leaves || max_sources < 1)
    return JB_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return run_builder(out, st, [&](jb_dsched& d) {
    build_leaf(d, num_internal, node_ranges, near_off, near_src, leaf_lo, leaf_hi, max_sources, st);
  });
}

JB_API int jb_gear_schedule_device(int num_nodes, const int64_t* far_off, const int* far_src, const int* gears,
                                   int num_gears, int max_pairs, void* stream, jb_dsched** out) {
  if (num_nodes < 0 || !far_off || !far_src || !gears || num_gears < 1 || num_gears > 64 || max_pairs < 1)
    return JB_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return run_builder(out, st, [&](jb_dsched& d) {
    build_gears(d, num_nodes, far_off, far_src, gears, num_gears, max_pairs, st);
  });
}

JB_API int jb_gear_mixed_schedule_device(int num_nodes, const int64_t* far_off, const int* far_src, const int* gears,
                                         int num_gears, const int* gear_orders, int p_max, int max_pairs,
                                         void* stream, jb_dsched** out) {
  if (num_nodes < 0 || !far_off || !far_src || !gears || !gear_orders || num_gears < 1 || num_gears > 64 ||
      max_pairs < 1 || max_pairs > 65535 || p_max < 1 || p_max > JB_MAX_ORDER)
    return JB_ERR_ARG;
  const int nseg = std::min(kMixedSegMax, (p_max + 1) / 2);
  GearSegments gs{};
  for (int g = 0; g < num_gears; ++g) {
    const int o = gear_orders[g], d = p_max - o;
    if (o < 1 || d < 0 || (d & 1) || d / 2 >= nseg) return JB_ERR_ARG;
    gs.seg[g] = d / 2;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  return run_builder(out, st, [&](jb_dsched& d) {
    build_gears_mixed(d, num_nodes, far_off, far_src, gears, num_gears, gs, max_pairs, st);
  });
}

JB_API int jb_far_reverse_index(int num_nodes, const int64_t* far_off, const int* far_src, int* rev, void* stream) {
  if (num_nodes < 0 || !far_off || !far_src || !rev) return JB_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  tl_stream = st;
  try {
    DBuf bad;
    ck(bad.alloc(4));
    ck(cudaMemsetAsync(bad.p, 0, 4, st));
    if (num_nodes > 0) {
      k_far_reverse<<<nblocks(num_nodes, 128), 128, 0, st>>>(far_off, num_nodes, far_src, rev, bad.as<int>());
      ck_launch();
    }
    if (read_word(bad.as<int>(), st) != 0) return JB_ERR_INDEX;
  } catch (const Fail& f) {
    return f.rc;
  }
  return JB_OK;
}

JB_API int jb_dsched_info(const jb_dsched* d, jb_sched_info_t* info) {
  if (!d || !info) return JB_ERR_ARG;
  *info = d->info;
  return JB_OK;
}

JB_API const void* jb_dsched_field(const jb_dsched* d, int field) {
  if (!d) return nullptr;
  const DBuf* b = sched_field(d, field);
  return b ? b->p : nullptr;
}

JB_API void jb_dsched_free(jb_dsched* d) { delete d; }

}  // extern "C"
