// Tree + interaction lists of the prepare step, restated for the oracle --
// TEST INFRASTRUCTURE ONLY (loaded by tests/ and bench.py's CPU legs, never
// by the product).
//
// A C++ transcription of oracle/tree.py (the scalar restatement of the
// yggdrax stand-in that jaccpot calls at runtime/fmm_prepare.py:823 and
// :1411), serial and in the same float64 operation order, so its arrays equal
// that module's -- and the product builders' -- bit for bit, but fast enough
// for the benchmark's 4M-particle CPU leg:
//   * Morton: 21 bits per axis over the bounding cube, (pos - lo) * (2^21-1)/ext
//     truncated; (code, input index) sorted;
//   * breadth-first radix split at the highest differing code bit (equal
//     codes: midpoint); internal ids in BFS order, leaves in particle order;
//   * COM (massless: mean position, count-weighted for internal nodes as
//     mutual/topology.py:500-516) and the bounding radius about it;
//   * dual walk from (root, root): far when d^2 > 0 and (r_A + r_B)^2 <=
//     theta^2 d^2 (experimental/treecode_walk.py:47-64), near when both are
//     leaves, else split the larger radius (mutual/topology.py:265-407); both
//     directions emitted; target-major CSR with sources ascending.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

namespace {

struct OTree {
  int64_t n = 0;
  int num_nodes = 0, num_internal = 0, num_leaves = 0, num_levels = 0;
  std::vector<int64_t> perm;
  std::vector<int32_t> ranges, left, right, parent, level, level_off, leaf_of;
  std::vector<int64_t> far_off, near_off;
  std::vector<int32_t> far_src, near_src;
  std::vector<double> com, rad;
};

uint64_t spread21(uint64_t v) {
  uint64_t out = 0;
  for (int b = 0; b < 21; ++b) out |= ((v >> b) & 1ULL) << (3 * b);
  return out;
}

int split_point(const std::vector<uint64_t>& c, int s, int e) {
  const uint64_t a = c[s], b = c[e];
  if (a == b) return (s + e + 1) / 2;
  int bit = 63;
  while (!(((a ^ b) >> bit) & 1ULL)) --bit;
  int lo = s + 1, hi = e;  // first index whose code has the bit set
  while (lo < hi) {
    const int mid = (lo + hi) / 2;
    if ((c[mid] >> bit) & 1ULL) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

void build(OTree& t, int64_t n, const double* pos, const double* mass, int leaf_size, double theta) {
  t.n = n;
  double lo[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = hi[k] = pos[k];
    for (int64_t i = 1; i < n; ++i) {
      lo[k] = std::min(lo[k], pos[3 * i + k]);
      hi[k] = std::max(hi[k], pos[3 * i + k]);
    }
  }
  double ext = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
  if (!(ext > 0)) ext = 1.0;
  const double qmax = (double)((1 << 21) - 1), scale = qmax / ext;
  std::vector<std::pair<uint64_t, int64_t>> keys((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    uint64_t q[3];
    for (int k = 0; k < 3; ++k) {
      double f = (pos[3 * i + k] - lo[k]) * scale;
      f = std::min(std::max(f, 0.0), qmax);
      q[k] = (uint64_t)f;
    }
    keys[(size_t)i] = {(spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]), i};
  }
  std::sort(keys.begin(), keys.end());
  std::vector<uint64_t> codes((size_t)n);
  t.perm.resize((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    codes[(size_t)i] = keys[(size_t)i].first;
    t.perm[(size_t)i] = keys[(size_t)i].second;
  }
  keys.clear();
  keys.shrink_to_fit();

  struct Pend { int s, e, par, side; };
  struct Leaf { int s, e, par, side, lv; };
  std::vector<Pend> cur{{0, (int)n - 1, -1, 0}}, nxt;
  std::vector<int32_t> iranges, ipar, ilev;
  std::vector<Leaf> leaves;
  std::vector<int32_t> level_off;
  int lev = 0;
  while (!cur.empty()) {
    level_off.push_back((int32_t)ipar.size());
    nxt.clear();
    for (const Pend& p : cur) {
      if (p.e - p.s + 1 <= leaf_size) {
        leaves.push_back({p.s, p.e, p.par, p.side, lev});
        continue;
      }
      const int nid = (int)ipar.size();
      iranges.push_back(p.s);
      iranges.push_back(p.e);
      ipar.push_back(p.par);
      ilev.push_back(lev);
      t.left.push_back(-1);
      t.right.push_back(-1);
      if (p.par >= 0) (p.side == 0 ? t.left : t.right)[(size_t)p.par] = nid;
      const int sp = split_point(codes, p.s, p.e);
      nxt.push_back({p.s, sp - 1, nid, 0});
      nxt.push_back({sp, p.e, nid, 1});
    }
    std::swap(cur, nxt);
    ++lev;
  }
  const int ni = (int)ipar.size();
  while (level_off.size() > 1 && level_off.back() == ni) level_off.pop_back();
  level_off.push_back(ni);
  t.num_levels = ni > 0 ? (int)level_off.size() - 1 : 0;
  if (ni == 0) level_off.assign(1, 0);
  t.level_off = level_off;
  std::sort(leaves.begin(), leaves.end(), [](const Leaf& a, const Leaf& b) { return a.s < b.s; });
  const int L = (int)leaves.size(), nodes = ni + L;
  t.num_internal = ni;
  t.num_leaves = L;
  t.num_nodes = nodes;
  t.ranges = iranges;
  t.ranges.resize(2 * (size_t)nodes);
  t.parent = ipar;
  t.parent.resize((size_t)nodes);
  t.level = ilev;
  t.level.resize((size_t)nodes);
  t.leaf_of.assign((size_t)n, 0);
  for (int j = 0; j < L; ++j) {
    const Leaf& lf = leaves[(size_t)j];
    const int nid = ni + j;
    t.ranges[2 * (size_t)nid] = lf.s;
    t.ranges[2 * (size_t)nid + 1] = lf.e;
    t.parent[(size_t)nid] = lf.par;
    t.level[(size_t)nid] = lf.lv;
    if (lf.par >= 0) (lf.side == 0 ? t.left : t.right)[(size_t)lf.par] = nid;
    for (int i = lf.s; i <= lf.e; ++i) t.leaf_of[(size_t)i] = j;
  }

  // COM and radii, float64, particle by particle
  t.com.assign(3 * (size_t)nodes, 0.0);
  t.rad.assign((size_t)nodes, 0.0);
  std::vector<double> msum((size_t)nodes, 0.0);
  for (int j = 0; j < L; ++j) {
    const int nid = ni + j, s = t.ranges[2 * (size_t)nid], e = t.ranges[2 * (size_t)nid + 1];
    double sm = 0, sx = 0, sy = 0, sz = 0;
    for (int i = s; i <= e; ++i) {
      const int64_t o = t.perm[(size_t)i];
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
    } else {
      c[0] = c[1] = c[2] = 0.0;
      for (int i = s; i <= e; ++i)
        for (int k = 0; k < 3; ++k) c[k] += pos[3 * t.perm[(size_t)i] + k];
      for (int k = 0; k < 3; ++k) c[k] = c[k] / (double)(e - s + 1);
    }
    double r = 0.0;
    for (int i = s; i <= e; ++i) {
      const int64_t o = t.perm[(size_t)i];
      const double dx = pos[3 * o] - c[0], dy = pos[3 * o + 1] - c[1], dz = pos[3 * o + 2] - c[2];
      r = std::max(r, std::sqrt(dx * dx + dy * dy + dz * dz));
    }
    msum[(size_t)nid] = sm;
    t.rad[(size_t)nid] = r;
    for (int k = 0; k < 3; ++k) t.com[3 * (size_t)nid + k] = c[k];
  }
  for (int i = ni - 1; i >= 0; --i) {
    const int a = t.left[(size_t)i], b = t.right[(size_t)i];
    const double ma = msum[(size_t)a], mb = msum[(size_t)b], sm = ma + mb;
    const double na = (double)(t.ranges[2 * (size_t)a + 1] - t.ranges[2 * (size_t)a] + 1);
    const double nb = (double)(t.ranges[2 * (size_t)b + 1] - t.ranges[2 * (size_t)b] + 1);
    double c[3];
    for (int k = 0; k < 3; ++k)
      c[k] = sm > 0 ? (ma * t.com[3 * (size_t)a + k] + mb * t.com[3 * (size_t)b + k]) / sm
                    : (na * t.com[3 * (size_t)a + k] + nb * t.com[3 * (size_t)b + k]) / (na + nb);
    double r = 0.0;
    for (int ch : {a, b}) {
      double d2 = 0.0;
      for (int k = 0; k < 3; ++k) {
        const double dd = t.com[3 * (size_t)ch + k] - c[k];
        d2 += dd * dd;
      }
      r = std::max(r, std::sqrt(d2) + t.rad[(size_t)ch]);
    }
    msum[(size_t)i] = sm;
    t.rad[(size_t)i] = r;
    for (int k = 0; k < 3; ++k) t.com[3 * (size_t)i + k] = c[k];
  }

  // dual walk
  const double theta2 = theta * theta;
  std::vector<std::pair<int32_t, int32_t>> far, near;
  if (nodes > 1) {
    std::vector<std::pair<int, int>> stack{{0, 0}};
    while (!stack.empty()) {
      const auto [a, b] = stack.back();
      stack.pop_back();
      const bool la = a >= ni, lb = b >= ni;
      if (a == b) {
        if (!la) {
          const int l = t.left[(size_t)a], r = t.right[(size_t)a];
          stack.push_back({l, l});
          stack.push_back({r, r});
          stack.push_back({l, r});
        }
        continue;
      }
      double d2 = 0.0;
      for (int k = 0; k < 3; ++k) {
        const double dd = t.com[3 * (size_t)a + k] - t.com[3 * (size_t)b + k];
        d2 += dd * dd;
      }
      const double rs = t.rad[(size_t)a] + t.rad[(size_t)b];
      if (d2 > 0 && rs * rs <= theta2 * d2) {
        far.push_back({a, b});
        far.push_back({b, a});
      } else if (la && lb) {
        near.push_back({a - ni, b - ni});
        near.push_back({b - ni, a - ni});
      } else if (!la && (lb || t.rad[(size_t)a] >= t.rad[(size_t)b])) {
        stack.push_back({t.left[(size_t)a], b});
        stack.push_back({t.right[(size_t)a], b});
      } else {
        stack.push_back({a, t.left[(size_t)b]});
        stack.push_back({a, t.right[(size_t)b]});
      }
    }
  }
  auto csr = [](std::vector<std::pair<int32_t, int32_t>>& pairs, int rows, std::vector<int64_t>& off,
                std::vector<int32_t>& col) {
    std::sort(pairs.begin(), pairs.end());
    off.assign((size_t)rows + 1, 0);
    col.resize(pairs.size());
    for (size_t q = 0; q < pairs.size(); ++q) {
      ++off[(size_t)pairs[q].first + 1];
      col[q] = pairs[q].second;
    }
    for (int r = 0; r < rows; ++r) off[(size_t)r + 1] += off[(size_t)r];
  };
  csr(far, nodes, t.far_off, t.far_src);
  csr(near, L, t.near_off, t.near_src);
}

}  // namespace

#define ORC_TREE_EXPORT extern "C" __attribute__((visibility("default")))

// Builds the tree of n float64 particles; returns an opaque handle (NULL on
// bad arguments).  sizes: num_nodes, num_internal, num_leaves, num_levels,
// num_far, num_near.
ORC_TREE_EXPORT void* oracle_tree_build(int64_t n, const double* pos, const double* mass, int leaf_size,
                                        double theta, int64_t* sizes) {
  if (n <= 0 || !pos || !mass || leaf_size < 1 || !(theta > 0) || !sizes) return nullptr;
  OTree* t = new OTree();
  build(*t, n, pos, mass, leaf_size, theta);
  sizes[0] = t->num_nodes;
  sizes[1] = t->num_internal;
  sizes[2] = t->num_leaves;
  sizes[3] = t->num_levels;
  sizes[4] = (int64_t)t->far_src.size();
  sizes[5] = (int64_t)t->near_src.size();
  return t;
}

// Field ids as jb_tree_copy's (permutation 0 ... radii 13).
ORC_TREE_EXPORT int oracle_tree_copy(void* h, int field, void* dst) {
  const OTree* t = static_cast<const OTree*>(h);
  if (!t || !dst) return 1;
  auto put = [&](const auto& v) {
    if (!v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    return 0;
  };
  switch (field) {
    case 0: return put(t->perm);
    case 1: return put(t->ranges);
    case 2: return put(t->left);
    case 3: return put(t->right);
    case 4: return put(t->parent);
    case 5: return put(t->level);
    case 6: return put(t->level_off);
    case 7: return put(t->leaf_of);
    case 8: return put(t->far_off);
    case 9: return put(t->far_src);
    case 10: return put(t->near_off);
    case 11: return put(t->near_src);
    case 12: return put(t->com);
    case 13: return put(t->rad);
    default: return 1;
  }
}

ORC_TREE_EXPORT void oracle_tree_free(void* h) { delete static_cast<OTree*>(h); }
