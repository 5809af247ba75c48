"""Error-controlled dual walk -- TEST INFRASTRUCTURE ONLY.

Scalar-for-scalar numpy restatement of jb_dtree_adaptive_walk
(jaccpot_b200/csrc/tree_gpu.cu): the reference's Dehnen eq. (15)/(16a)
acceptance policy (jaccpot runtime/_adaptive_policy.py:267-376
``dehnen_paper_pair_error_by_order``, :2285-2338 the directional test of
``adaptive_pair_policy``), evaluated for ordered (target <- source) node
pairs.  Every floating-point step is a separately rounded FP64 operation in
the order the CUDA file uses, so given the same inputs (centres, radii,
powers, force scales) the lists and gears are identical bit for bit.

Only ``tests/`` may import this module.
"""

from __future__ import annotations

import math

import numpy as np


def error_gears(t, s, d, rt, rs, power, fscale, G, eps, orders):
    """Gear index per pair (-1: not accepted), eq. (15)/(16a)."""
    orders = [int(o) for o in orders]
    npow = power.shape[1]
    pmax = orders[-1]
    rtp = [np.ones_like(rt)]
    for _ in range(pmax):
        rtp.append(rtp[-1] * rt)
    dp = [np.ones_like(d)]
    for _ in range(pmax + 2):
        dp.append(dp[-1] * d)
    den = np.maximum(rs + rt, 1e-24)
    imp = (8.0 * np.maximum(rs, rt)) / den
    thr = np.maximum(eps * fscale[t].astype(np.float64), 1e-24)
    first = np.full(t.shape, -1, dtype=np.int64)
    passed = np.zeros(t.shape, dtype=bool)
    for g, p in enumerate(orders):
        e = np.zeros_like(d)
        c = 1.0
        for ell in range(min(p, npow - 1) + 1):
            if ell > 0:
                c = (c * float(p - ell + 1)) / float(ell)
            e = e + (c * power[s, ell]) * rtp[p - ell]
        ferr = ((G * imp) * e) / dp[p + 2]
        passed = ferr < thr
        first = np.where(passed & (first < 0), g, first)
    return np.where(passed, first, -1)


def adaptive_walk(left, right, com, radius, num_internal, power, fscale, *, G, eps, theta_max, orders):
    """Returns (far_off, far_src, far_gear, near_off, near_src): target-major
    CSR lists (sources ascending) as jb_dtree_adaptive_walk produces them."""
    num_nodes = com.shape[0]
    num_leaves = num_nodes - num_internal
    far_t, far_s, far_g, near_t, near_s = [], [], [], [], []
    T = np.zeros(1, np.int64)
    S = np.zeros(1, np.int64)
    if num_nodes == 1:
        T = T[:0]
        S = S[:0]
    while T.size:
        self_pair = T == S
        st = T[self_pair]
        st = st[st < num_internal]
        lc, rc = left[st].astype(np.int64), right[st].astype(np.int64)
        nT = [lc, rc, lc, rc]
        nS = [lc, rc, rc, lc]
        t, s = T[~self_pair], S[~self_pair]
        d2 = np.zeros(t.shape)
        for k in range(3):
            dd = com[t, k] - com[s, k]
            d2 = d2 + dd * dd
        rt, rs = radius[t], radius[s]
        d = np.sqrt(d2)
        conv = (d2 > 0) & (rs + rt < theta_max * d)
        gear = np.full(t.shape, -1, dtype=np.int64)
        if conv.any():
            idx = np.nonzero(conv)[0]
            gear[idx] = error_gears(t[idx], s[idx], d[idx], rt[idx], rs[idx], power, fscale, G, eps, orders)
        far = gear >= 0
        far_t.append(t[far])
        far_s.append(s[far])
        far_g.append(gear[far])
        lt, ls = t >= num_internal, s >= num_internal
        near = ~far & lt & ls
        near_t.append(t[near] - num_internal)
        near_s.append(s[near] - num_internal)
        rest = ~far & ~near
        t, s, lt, ls, rt, rs = t[rest], s[rest], lt[rest], ls[rest], rt[rest], rs[rest]
        split_t = ~lt & (ls | (rt >= rs))
        a, b = t[split_t], s[split_t]
        nT += [left[a].astype(np.int64), right[a].astype(np.int64)]
        nS += [b, b]
        a, b = t[~split_t], s[~split_t]
        nT += [a, a]
        nS += [left[b].astype(np.int64), right[b].astype(np.int64)]
        T = np.concatenate(nT)
        S = np.concatenate(nS)

    def csr(rows, cols, nrows, extra=None):
        rows = np.concatenate(rows) if rows else np.zeros(0, np.int64)
        cols = np.concatenate(cols) if cols else np.zeros(0, np.int64)
        order = np.lexsort((cols, rows))
        off = np.zeros(nrows + 1, np.int64)
        np.add.at(off, rows + 1, 1)
        off = np.cumsum(off)
        ex = None if extra is None else np.concatenate(extra)[order].astype(np.int32)
        return off, cols[order].astype(np.int32), ex

    far_off, far_src, far_gear = csr(far_t, far_s, num_nodes, far_g)
    near_off, near_src, _ = csr(near_t, near_s, num_leaves)
    return far_off, far_src, far_gear, near_off, near_src


def dehnen_power(mult, p):
    """Dehnen's per-degree power P_l (real packing, m != 0 weights doubled),
    FP64, l = 0..p (_adaptive_policy.py:161-214)."""
    mult = np.asarray(mult, dtype=np.float64)
    out = np.zeros((mult.shape[0], p + 1))
    for ell in range(p + 1):
        acc = np.zeros(mult.shape[0])
        for m in range(-ell, ell + 1):
            w = math.factorial(ell - abs(m)) * math.factorial(ell + abs(m)) * (2.0 if m else 1.0)
            c = mult[:, ell * ell + ell + m]
            acc = acc + w * c * c
        out[:, ell] = np.sqrt(acc)
    return out
