// Host-side prepare: Morton order, binary radix tree with bucketed leaves, COM
// centres, bounding radii and the dual-tree traversal that yields the far-pair
// (M2L) and leaf-neighbour (P2P) lists.
//
// This is the stand-in for the artefacts jaccpot takes from yggdrax
// (yggdrax.morton / tree build / compute_tree_mass_moments / dual traversal;
// used at jaccpot/runtime/fmm_prepare.py:19-40, :823, :1411 and
// jaccpot/runtime/kernels/_downward_prep.py:268).  yggdrax is not vendored in
// the reference, so its lists cannot be reproduced bit for bit; the layout
// produced here is the one the reference's kernels consume:
//   * node ids: internal nodes [0, num_internal) in breadth-first order (root
//     = 0), leaves [num_internal, num_nodes) in particle order; every internal
//     node has exactly two children (num_nodes = 2 * num_leaves - 1);
//   * node_ranges[n] = inclusive [start, end] in Morton-sorted order
//     (upward/real_tree_expansions.py:158);
//   * far pairs: target-centric CSR (offsets over all nodes, source node ids);
//   * near pairs: target-leaf CSR of source leaf indices, self excluded (the
//     self block is always evaluated, nearfield/_kernels.py:40-141).
// Traversal: symmetric dual walk (modelled on jaccpot/mutual/topology.py:265-407):
// accept (A, B) when (r_A + r_B)^2 <= theta^2 |c_A - c_B|^2 (the "dehnen" sum
// form, experimental/treecode_walk.py:47-64) with r = bounding radius about
// the COM; otherwise split the larger node; two leaves that fail become a
// near pair.  Both directions of every accepted pair are emitted.

#include "tree_build.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <parallel/algorithm>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline uint64_t spread21(uint64_t v) {
  v &= 0x1fffffULL;
  v = (v | (v << 32)) & 0x1f00000000ffffULL;
  v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
  v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
  v = (v | (v << 2)) & 0x1249249249249249ULL;
  return v;
}

struct Tree {
  int64_t N = 0;
  int leaf_size = 0;
  int num_nodes = 0, num_internal = 0, num_leaves = 0, num_levels = 0;
  std::vector<int64_t> perm;  // sorted slot -> original index
  std::vector<uint64_t> codes;
  std::vector<int32_t> ranges;  // 2 * num_nodes
  std::vector<int32_t> left, right, parent, level, level_off;
  std::vector<int32_t> leaf_of;  // sorted particle -> leaf index
  std::vector<double> com, radius, mass;
  std::vector<int64_t> far_off;
  std::vector<int32_t> far_src;
  std::vector<int64_t> near_off;
  std::vector<int32_t> near_src;
};

// Splits sorted codes [s, e] at the highest differing bit (the Karras radix
// split); duplicate codes split at the midpoint.
int split_point(const std::vector<uint64_t>& c, int s, int e) {
  const uint64_t a = c[s], b = c[e];
  if (a == b) return (s + e + 1) / 2;
  const int bit = 63 - __builtin_clzll(a ^ b);
  const uint64_t mask = 1ULL << bit;
  int lo = s + 1, hi = e;  // first index whose code has `bit` set
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if (c[mid] & mask) hi = mid; else lo = mid + 1;
  }
  return lo;
}

void build_topology(Tree& t, const double* pos, const double* mass) {
  const int64_t N = t.N;
  // Morton codes over the bounding cube.
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = 0; i < N; ++i)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], pos[3 * i + k]);
      hi[k] = std::max(hi[k], pos[3 * i + k]);
    }
  double ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
  if (!(ext > 0)) ext = 1.0;
  const double scale = (double)((1 << 21) - 1) / ext;
  std::vector<std::pair<uint64_t, int64_t>> kv((size_t)N);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < N; ++i) {
    uint64_t q[3];
    for (int k = 0; k < 3; ++k) {
      double f = (pos[3 * i + k] - lo[k]) * scale;
      f = std::min(std::max(f, 0.0), (double)((1 << 21) - 1));
      q[k] = (uint64_t)f;
    }
    kv[(size_t)i] = {(spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]), i};
  }
  __gnu_parallel::sort(kv.begin(), kv.end());
  t.perm.resize((size_t)N);
  t.codes.resize((size_t)N);
  for (int64_t i = 0; i < N; ++i) {
    t.codes[(size_t)i] = kv[(size_t)i].first;
    t.perm[(size_t)i] = kv[(size_t)i].second;
  }
  std::vector<std::pair<uint64_t, int64_t>>().swap(kv);

  // Breadth-first split.  Internal ids are handed out in BFS order; leaves are
  // renumbered afterwards in particle order.
  struct Pending { int s, e, parent, side, level; };
  std::vector<Pending> cur, nxt;
  cur.push_back({0, (int)N - 1, -1, 0, 0});
  std::vector<int32_t> int_ranges, int_parent, int_level, int_left, int_right;
  struct LeafRec { int s, e, parent, side, level; };
  std::vector<LeafRec> leaves;
  int level = 0;
  t.level_off.clear();
  while (!cur.empty()) {
    t.level_off.push_back((int)int_ranges.size() / 2);
    nxt.clear();
    for (const Pending& pd : cur) {
      const int cnt = pd.e - pd.s + 1;
      if (cnt <= t.leaf_size) {
        leaves.push_back({pd.s, pd.e, pd.parent, pd.side, pd.level});
        continue;
      }
      const int id = (int)int_ranges.size() / 2;
      int_ranges.push_back(pd.s);
      int_ranges.push_back(pd.e);
      int_parent.push_back(pd.parent);
      int_level.push_back(pd.level);
      int_left.push_back(-1);
      int_right.push_back(-1);
      if (pd.parent >= 0) (pd.side == 0 ? int_left : int_right)[pd.parent] = id;
      const int sp = split_point(t.codes, pd.s, pd.e);
      nxt.push_back({pd.s, sp - 1, id, 0, pd.level + 1});
      nxt.push_back({sp, pd.e, id, 1, pd.level + 1});
    }
    cur.swap(nxt);
    ++level;
  }
  const int num_internal = (int)int_ranges.size() / 2;
  // Trim trailing levels that hold no internal node.
  while (t.level_off.size() > 1 && t.level_off.back() == num_internal) t.level_off.pop_back();
  t.level_off.push_back(num_internal);
  t.num_levels = num_internal > 0 ? (int)t.level_off.size() - 1 : 0;
  if (num_internal == 0) t.level_off.assign(1, 0);

  std::sort(leaves.begin(), leaves.end(), [](const LeafRec& a, const LeafRec& b) { return a.s < b.s; });
  const int L = (int)leaves.size();
  t.num_internal = num_internal;
  t.num_leaves = L;
  t.num_nodes = num_internal + L;
  t.ranges.assign(2 * (size_t)t.num_nodes, 0);
  t.parent.assign(t.num_nodes, -1);
  t.level.assign(t.num_nodes, 0);
  t.left = int_left;
  t.right = int_right;
  for (int i = 0; i < num_internal; ++i) {
    t.ranges[2 * i] = int_ranges[2 * i];
    t.ranges[2 * i + 1] = int_ranges[2 * i + 1];
    t.parent[i] = int_parent[i];
    t.level[i] = int_level[i];
  }
  t.leaf_of.assign((size_t)N, 0);
  for (int j = 0; j < L; ++j) {
    const int id = num_internal + j;
    const LeafRec& lr = leaves[j];
    t.ranges[2 * id] = lr.s;
    t.ranges[2 * id + 1] = lr.e;
    t.parent[id] = lr.parent;
    t.level[id] = lr.level;
    if (lr.parent >= 0) (lr.side == 0 ? t.left : t.right)[lr.parent] = id;
    for (int i = lr.s; i <= lr.e; ++i) t.leaf_of[(size_t)i] = j;
  }

  // COM (mass-weighted, float64) and a bounding radius about it, leaves from
  // their particles, internal nodes bottom-up (children have larger BFS ids).
  t.com.assign(3 * (size_t)t.num_nodes, 0.0);
  t.radius.assign(t.num_nodes, 0.0);
  t.mass.assign(t.num_nodes, 0.0);
#pragma omp parallel for schedule(dynamic, 64)
  for (int j = 0; j < L; ++j) {
    const int id = num_internal + j;
    double sm = 0, sx = 0, sy = 0, sz = 0;
    for (int i = t.ranges[2 * id]; i <= t.ranges[2 * id + 1]; ++i) {
      const int64_t o = t.perm[(size_t)i];
      const double m = mass[o];
      sm += m; sx += m * pos[3 * o]; sy += m * pos[3 * o + 1]; sz += m * pos[3 * o + 2];
    }
    double c[3];
    if (sm > 0) { c[0] = sx / sm; c[1] = sy / sm; c[2] = sz / sm; }
    else {  // massless leaf: geometric mean of its particles
      const int s = t.ranges[2 * id], e = t.ranges[2 * id + 1];
      c[0] = c[1] = c[2] = 0;
      for (int i = s; i <= e; ++i) for (int k = 0; k < 3; ++k) c[k] += pos[3 * t.perm[(size_t)i] + k];
      for (int k = 0; k < 3; ++k) c[k] /= (double)(e - s + 1);
    }
    double rmax = 0;
    for (int i = t.ranges[2 * id]; i <= t.ranges[2 * id + 1]; ++i) {
      const int64_t o = t.perm[(size_t)i];
      const double dx = pos[3 * o] - c[0], dy = pos[3 * o + 1] - c[1], dz = pos[3 * o + 2] - c[2];
      rmax = std::max(rmax, std::sqrt(dx * dx + dy * dy + dz * dz));
    }
    t.mass[id] = sm;
    t.radius[id] = rmax;
    for (int k = 0; k < 3; ++k) t.com[3 * (size_t)id + k] = c[k];
  }
  for (int i = num_internal - 1; i >= 0; --i) {
    const int a = t.left[i], b = t.right[i];
    const double ma = t.mass[a], mb = t.mass[b], sm = ma + mb;
    double c[3];
    // massless subtree: mean particle position, from the children's means
    // weighted by their particle counts (as mutual/topology.py:500-516)
    const double na = (double)(t.ranges[2 * a + 1] - t.ranges[2 * a] + 1);
    const double nb = (double)(t.ranges[2 * b + 1] - t.ranges[2 * b] + 1);
    for (int k = 0; k < 3; ++k)
      c[k] = sm > 0 ? (ma * t.com[3 * (size_t)a + k] + mb * t.com[3 * (size_t)b + k]) / sm
                    : (na * t.com[3 * (size_t)a + k] + nb * t.com[3 * (size_t)b + k]) / (na + nb);
    double r = 0;
    for (int ch : {a, b}) {
      double d2 = 0;
      for (int k = 0; k < 3; ++k) { const double dd = t.com[3 * (size_t)ch + k] - c[k]; d2 += dd * dd; }
      r = std::max(r, std::sqrt(d2) + t.radius[ch]);
    }
    t.mass[i] = sm;
    t.radius[i] = r;
    for (int k = 0; k < 3; ++k) t.com[3 * (size_t)i + k] = c[k];
  }
}

struct PairOut {
  std::vector<std::pair<int32_t, int32_t>> far;   // (target, source) node ids
  std::vector<std::pair<int32_t, int32_t>> near;  // (target leaf, source leaf)
};

struct Walker {
  const Tree& t;
  double theta2;
  PairOut* out;
  bool is_leaf(int n) const { return n >= t.num_internal; }
  void emit_far(int a, int b) { out->far.push_back({a, b}); out->far.push_back({b, a}); }
  void emit_near(int a, int b) {
    const int la = a - t.num_internal, lb = b - t.num_internal;
    out->near.push_back({la, lb});
    out->near.push_back({lb, la});
  }
  void walk(int a, int b) {
    if (a == b) {
      if (is_leaf(a)) return;
      const int l = t.left[a], r = t.right[a];
      walk(l, l);
      walk(r, r);
      walk(l, r);
      return;
    }
    double d2 = 0;
    for (int k = 0; k < 3; ++k) {
      const double dd = t.com[3 * (size_t)a + k] - t.com[3 * (size_t)b + k];
      d2 += dd * dd;
    }
    const double rs = t.radius[a] + t.radius[b];
    if (d2 > 0 && rs * rs <= theta2 * d2) { emit_far(a, b); return; }
    const bool la = is_leaf(a), lb = is_leaf(b);
    if (la && lb) { emit_near(a, b); return; }
    const bool split_a = !la && (lb || t.radius[a] >= t.radius[b]);
    if (split_a) { walk(t.left[a], b); walk(t.right[a], b); }
    else { walk(a, t.left[b]); walk(a, t.right[b]); }
  }
};

// Expands the top of the walk breadth-first into independent (A, B) tasks,
// emitting whatever the first levels decide, until there is enough parallel work.
void collect_tasks(const Tree& t, double theta2, std::vector<std::pair<int, int>>& tasks, PairOut& top) {
  Walker w{t, theta2, &top};
  std::vector<std::pair<int, int>> frontier{{0, 0}}, next;
  for (int round = 0; round < 64 && !frontier.empty() && frontier.size() < 8192; ++round) {
    next.clear();
    for (const auto& ab : frontier) {
      const int a = ab.first, b = ab.second;
      if (a == b) {
        if (w.is_leaf(a)) continue;
        const int l = t.left[a], r = t.right[a];
        next.push_back({l, l});
        next.push_back({r, r});
        next.push_back({l, r});
        continue;
      }
      double d2 = 0;
      for (int k = 0; k < 3; ++k) { const double dd = t.com[3 * (size_t)a + k] - t.com[3 * (size_t)b + k]; d2 += dd * dd; }
      const double rs = t.radius[a] + t.radius[b];
      if (d2 > 0 && rs * rs <= theta2 * d2) { w.emit_far(a, b); continue; }
      const bool la = w.is_leaf(a), lb = w.is_leaf(b);
      if (la && lb) { w.emit_near(a, b); continue; }
      const bool split_a = !la && (lb || t.radius[a] >= t.radius[b]);
      if (split_a) { next.push_back({t.left[a], b}); next.push_back({t.right[a], b}); }
      else { next.push_back({a, t.left[b]}); next.push_back({a, t.right[b]}); }
    }
    frontier.swap(next);
  }
  tasks = frontier;
}

template <typename K>
void to_csr(std::vector<std::pair<int32_t, int32_t>>& pairs, int n_rows, std::vector<int64_t>& off, std::vector<int32_t>& col) {
  __gnu_parallel::sort(pairs.begin(), pairs.end());
  off.assign((size_t)n_rows + 1, 0);
  col.resize(pairs.size());
  for (size_t i = 0; i < pairs.size(); ++i) {
    off[(size_t)pairs[i].first + 1]++;
    col[i] = pairs[i].second;
  }
  for (int r = 0; r < n_rows; ++r) off[(size_t)r + 1] += off[(size_t)r];
}

void build_lists(Tree& t, double theta) {
  const double theta2 = theta * theta;
  PairOut top;
  std::vector<std::pair<int, int>> tasks;
  if (t.num_nodes > 1) collect_tasks(t, theta2, tasks, top);
  const int nthreads =
#ifdef _OPENMP
      omp_get_max_threads();
#else
      1;
#endif
  std::vector<PairOut> outs((size_t)nthreads);
#pragma omp parallel for schedule(dynamic, 1)
  for (size_t k = 0; k < tasks.size(); ++k) {
    int tid = 0;
#ifdef _OPENMP
    tid = omp_get_thread_num();
#endif
    Walker w{t, theta2, &outs[(size_t)tid]};
    w.walk(tasks[k].first, tasks[k].second);
  }
  std::vector<std::pair<int32_t, int32_t>> far = std::move(top.far), near = std::move(top.near);
  for (auto& o : outs) {
    far.insert(far.end(), o.far.begin(), o.far.end());
    near.insert(near.end(), o.near.begin(), o.near.end());
    std::vector<std::pair<int32_t, int32_t>>().swap(o.far);
    std::vector<std::pair<int32_t, int32_t>>().swap(o.near);
  }
  to_csr<int>(far, t.num_nodes, t.far_off, t.far_src);
  to_csr<int>(near, t.num_leaves, t.near_off, t.near_src);
}

}  // namespace

extern "C" {

JB_API int jb_tree_build(int64_t n, const double* pos, const double* mass, int leaf_size, double theta, jb_tree** out) {
  if (!out) return JB_ERR_ARG;
  *out = nullptr;
  if (n <= 0 || n > (int64_t)0x7fffffff || !pos || !mass || leaf_size < 1 || !(theta > 0) || !(theta < 1.0))
    return JB_ERR_ARG;
  for (int64_t i = 0; i < 3 * n; ++i)
    if (!std::isfinite(pos[i])) return JB_ERR_NONFINITE;
  for (int64_t i = 0; i < n; ++i)
    if (!std::isfinite(mass[i])) return JB_ERR_NONFINITE;
  Tree* t = new (std::nothrow) Tree();
  if (!t) return JB_ERR_ALLOC;
  try {
    t->N = n;
    t->leaf_size = leaf_size;
    build_topology(*t, pos, mass);
    build_lists(*t, theta);
  } catch (const std::bad_alloc&) {
    delete t;
    return JB_ERR_ALLOC;
  }
  *out = reinterpret_cast<jb_tree*>(t);
  return JB_OK;
}

JB_API int jb_tree_info(const jb_tree* h, jb_tree_info_t* info) {
  if (!h || !info) return JB_ERR_ARG;
  const Tree* t = reinterpret_cast<const Tree*>(h);
  info->num_particles = t->N;
  info->num_nodes = t->num_nodes;
  info->num_internal = t->num_internal;
  info->num_leaves = t->num_leaves;
  info->num_levels = t->num_levels;
  info->num_far_pairs = (int64_t)t->far_src.size();
  info->num_near_pairs = (int64_t)t->near_src.size();
  int w = 0;
  for (int j = 0; j < t->num_leaves; ++j) {
    const int id = t->num_internal + j;
    w = std::max(w, t->ranges[2 * id + 1] - t->ranges[2 * id] + 1);
  }
  info->max_leaf_occupancy = w;
  return JB_OK;
}

#define COPY(field, ptr_t, vec)                                          \
  case field: {                                                          \
    std::memcpy(dst, t->vec.data(), sizeof(ptr_t) * t->vec.size());      \
    return JB_OK;                                                        \
  }

JB_API int jb_tree_copy(const jb_tree* h, int field, void* dst) {
  if (!h || !dst) return JB_ERR_ARG;
  const Tree* t = reinterpret_cast<const Tree*>(h);
  switch (field) {
    COPY(JB_TREE_PERMUTATION, int64_t, perm)
    COPY(JB_TREE_NODE_RANGES, int32_t, ranges)
    COPY(JB_TREE_LEFT_CHILD, int32_t, left)
    COPY(JB_TREE_RIGHT_CHILD, int32_t, right)
    COPY(JB_TREE_PARENT, int32_t, parent)
    COPY(JB_TREE_NODE_LEVEL, int32_t, level)
    COPY(JB_TREE_LEVEL_OFFSETS, int32_t, level_off)
    COPY(JB_TREE_LEAF_OF_PARTICLE, int32_t, leaf_of)
    COPY(JB_TREE_FAR_OFFSETS, int64_t, far_off)
    COPY(JB_TREE_FAR_SOURCES, int32_t, far_src)
    COPY(JB_TREE_NEAR_OFFSETS, int64_t, near_off)
    COPY(JB_TREE_NEAR_SOURCES, int32_t, near_src)
    COPY(JB_TREE_CENTERS_F64, double, com)
    COPY(JB_TREE_RADII_F64, double, radius)
    default:
      return JB_ERR_ARG;
  }
}

JB_API void jb_tree_free(jb_tree* h) { delete reinterpret_cast<Tree*>(h); }

}  // extern "C"
