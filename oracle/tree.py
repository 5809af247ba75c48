"""Pure-Python restatement of the prepare step (tree + interaction lists) —
TEST INFRASTRUCTURE ONLY (imported by tests/ and nothing in the product).

The product builds the tree twice, on the host (csrc/tree_build.cpp,
``jb_tree_build``) and on the GPU (csrc/tree_gpu.cu, ``jb_tree_build_device``);
both stand in for the yggdrax calls jaccpot makes at runtime/fmm_prepare.py:823
(``_build_tree_with_config``) and :1411 (``_build_dual_tree_artifacts``).
yggdrax is not vendored, so its lists cannot be pinned; this module pins the
stand-in's own definition, step by step, in scalar float64 arithmetic whose
operation order is written out (sums run particle by particle), so its arrays
must equal both builders' bit for bit:

  * Morton: 21 bits per axis over the bounding cube, (pos - lo) * (2^21-1)/ext
    truncated; codes sorted with the input index as tie-break;
  * breadth-first radix split of ranges with more than leaf_size particles at
    the highest differing code bit (equal codes: midpoint); internal ids in
    BFS order, leaves in particle order;
  * COM (mass-weighted; massless: mean position, count-weighted for internal
    nodes as mutual/topology.py:500-516) and the bounding radius about it;
  * dual walk from (root, root) with the "dehnen" sum MAC
    (r_A + r_B)^2 <= theta^2 d^2 (experimental/treecode_walk.py:47-64),
    splitting the larger-radius node (mutual/topology.py:265-407); leaf pairs
    that fail are near; both directions emitted; CSR sorted by (target, source).

Pure Python loops: for N up to a few thousand.
"""

from __future__ import annotations

import math

import numpy as np


def _spread21(v: int) -> int:
    out = 0
    for b in range(21):
        out |= ((v >> b) & 1) << (3 * b)
    return out


def morton_order(pos: np.ndarray):
    pos = np.asarray(pos, np.float64)
    n = pos.shape[0]
    lo = [min(float(pos[i, k]) for i in range(n)) for k in range(3)]
    hi = [max(float(pos[i, k]) for i in range(n)) for k in range(3)]
    ext = max(hi[0] - lo[0], max(hi[1] - lo[1], hi[2] - lo[2]))
    if not ext > 0:
        ext = 1.0
    qmax = float((1 << 21) - 1)
    scale = qmax / ext
    keys = []
    for i in range(n):
        q = []
        for k in range(3):
            f = (float(pos[i, k]) - lo[k]) * scale
            f = min(max(f, 0.0), qmax)
            q.append(int(f))
        keys.append(((_spread21(q[0]) << 2) | (_spread21(q[1]) << 1) | _spread21(q[2]), i))
    keys.sort()
    return [k for k, _ in keys], [i for _, i in keys]


def _split_point(c, s, e):
    a, b = c[s], c[e]
    if a == b:
        return (s + e + 1) // 2
    bit = (a ^ b).bit_length() - 1
    for i in range(s + 1, e + 1):
        if c[i] >> bit & 1:
            return i
    raise AssertionError("sorted codes")


def build(pos, mass, leaf_size: int, theta: float) -> dict:
    """Every array of jb_tree_build for the same float64 inputs."""
    pos = np.asarray(pos, np.float64).reshape(-1, 3)
    mass = np.asarray(mass, np.float64).reshape(-1)
    n = pos.shape[0]
    codes, perm = morton_order(pos)

    # breadth-first split
    cur = [(0, n - 1, -1, 0)]
    int_ranges, int_parent, int_level, left, right = [], [], [], [], []
    leaves = []
    level_off = []
    level = 0
    while cur:
        level_off.append(len(int_ranges))
        nxt = []
        for s, e, par, side in cur:
            if e - s + 1 <= leaf_size:
                leaves.append((s, e, par, side, level))
                continue
            nid = len(int_ranges)
            int_ranges.append((s, e))
            int_parent.append(par)
            int_level.append(level)
            left.append(-1)
            right.append(-1)
            if par >= 0:
                (left if side == 0 else right)[par] = nid
            sp = _split_point(codes, s, e)
            nxt.append((s, sp - 1, nid, 0))
            nxt.append((sp, e, nid, 1))
        cur = nxt
        level += 1
    ni = len(int_ranges)
    while len(level_off) > 1 and level_off[-1] == ni:
        level_off.pop()
    level_off.append(ni)
    num_levels = len(level_off) - 1 if ni > 0 else 0
    if ni == 0:
        level_off = [0]
    leaves.sort(key=lambda r: r[0])
    L = len(leaves)
    nodes = ni + L
    ranges = list(int_ranges) + [None] * L
    parent = list(int_parent) + [0] * L
    nlevel = list(int_level) + [0] * L
    leaf_of = [0] * n
    for j, (s, e, par, side, lv) in enumerate(leaves):
        nid = ni + j
        ranges[nid] = (s, e)
        parent[nid] = par
        nlevel[nid] = lv
        if par >= 0:
            (left if side == 0 else right)[par] = nid
        for i in range(s, e + 1):
            leaf_of[i] = j

    # COM and radii, float64, particle by particle
    com = [[0.0, 0.0, 0.0] for _ in range(nodes)]
    rad = [0.0] * nodes
    msum = [0.0] * nodes
    P = [[float(pos[o, k]) for k in range(3)] for o in perm]
    M = [float(mass[o]) for o in perm]
    for j in range(L):
        nid = ni + j
        s, e = ranges[nid]
        sm = sx = sy = sz = 0.0
        for i in range(s, e + 1):
            sm += M[i]
            sx += M[i] * P[i][0]
            sy += M[i] * P[i][1]
            sz += M[i] * P[i][2]
        if sm > 0:
            c = [sx / sm, sy / sm, sz / sm]
        else:
            c = [0.0, 0.0, 0.0]
            for i in range(s, e + 1):
                for k in range(3):
                    c[k] += P[i][k]
            c = [c[k] / float(e - s + 1) for k in range(3)]
        r = 0.0
        for i in range(s, e + 1):
            dx, dy, dz = P[i][0] - c[0], P[i][1] - c[1], P[i][2] - c[2]
            r = max(r, math.sqrt(dx * dx + dy * dy + dz * dz))
        msum[nid], rad[nid], com[nid] = sm, r, c
    for i in range(ni - 1, -1, -1):
        a, b = left[i], right[i]
        ma, mb = msum[a], msum[b]
        sm = ma + mb
        na = float(ranges[a][1] - ranges[a][0] + 1)
        nb = float(ranges[b][1] - ranges[b][0] + 1)
        if sm > 0:
            c = [(ma * com[a][k] + mb * com[b][k]) / sm for k in range(3)]
        else:
            c = [(na * com[a][k] + nb * com[b][k]) / (na + nb) for k in range(3)]
        r = 0.0
        for ch in (a, b):
            d2 = 0.0
            for k in range(3):
                dd = com[ch][k] - c[k]
                d2 += dd * dd
            r = max(r, math.sqrt(d2) + rad[ch])
        msum[i], rad[i], com[i] = sm, r, c

    # dual walk
    theta2 = theta * theta
    far, near = [], []
    if nodes > 1:
        stack = [(0, 0)]
        while stack:
            a, b = stack.pop()
            la, lb = a >= ni, b >= ni
            if a == b:
                if not la:
                    l, r = left[a], right[a]
                    stack += [(l, l), (r, r), (l, r)]
                continue
            d2 = 0.0
            for k in range(3):
                dd = com[a][k] - com[b][k]
                d2 += dd * dd
            rs = rad[a] + rad[b]
            if d2 > 0 and rs * rs <= theta2 * d2:
                far += [(a, b), (b, a)]
            elif la and lb:
                near += [(a - ni, b - ni), (b - ni, a - ni)]
            elif not la and (lb or rad[a] >= rad[b]):
                stack += [(left[a], b), (right[a], b)]
            else:
                stack += [(a, left[b]), (a, right[b])]

    def csr(pairs, rows):
        pairs.sort()
        off = np.zeros(rows + 1, np.int64)
        for t, _ in pairs:
            off[t + 1] += 1
        return np.cumsum(off), np.array([s for _, s in pairs], np.int32)

    far_off, far_src = csr(far, nodes)
    near_off, near_src = csr(near, L)
    return {
        "permutation": np.array(perm, np.int64),
        "node_ranges": np.array(ranges, np.int32).reshape(-1, 2),
        "left_child": np.array(left, np.int32),
        "right_child": np.array(right, np.int32),
        "parent": np.array(parent, np.int32),
        "node_level": np.array(nlevel, np.int32),
        "level_offsets": np.array(level_off, np.int32),
        "leaf_of_particle": np.array(leaf_of, np.int32),
        "far_offsets": far_off,
        "far_sources": far_src,
        "near_offsets": near_off,
        "near_leaves": near_src,
        "centers_f64": np.array(com, np.float64).reshape(-1, 3),
        "radii_f64": np.array(rad, np.float64),
        "num_levels": num_levels,
    }
