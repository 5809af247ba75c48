"""The error-controlled walk's restatement (oracle/adaptive_walk.py) on the
CPU: its lists cover every (target, source) particle pair exactly once --
through a far pair of one of the target's ancestors (or itself), a near pair
of its leaf, or the leaf's self block -- for loose and tight error targets;
Dehnen's power is m r^l for a point mass; and tightening eps only moves work
from the far field to the near field."""

from __future__ import annotations

import numpy as np
import pytest

from jaccpot_b200 import tree, workloads
from oracle import adaptive_walk as aw


def _inputs(n=3000, seed=1, leaf=8, theta=0.6, p=6):
    import oracle

    pos, mass = workloads.clustered(n, seed, clumps=6)
    topo = tree.build_topology(pos, mass, leaf_size=leaf, theta=theta)
    ps = pos[topo.permutation].astype(np.float64)
    ms = mass[topo.permutation].astype(np.float64)
    res = oracle.Pass(topo, np.float64).run(p, ps, ms)
    power = aw.dehnen_power(res["multipoles"], p)
    amag = np.linalg.norm(res["acc"], axis=1)
    fs = np.empty(topo.num_nodes, np.float32)
    for i in range(topo.num_nodes):
        a, b = topo.node_ranges[i]
        fs[i] = amag[a:b + 1].min()
    return topo, power, fs


def _coverage(topo, far_off, far_src, near_off, near_src):
    """count[i, j] = how many times particle pair (i <- j) is covered."""
    n = topo.num_particles
    cnt = np.zeros((n, n), np.int32)
    rng = topo.node_ranges
    for t in range(topo.num_nodes):
        a, b = rng[t]
        for e in range(far_off[t], far_off[t + 1]):
            c, d = rng[far_src[e]]
            cnt[a:b + 1, c:d + 1] += 1
    for lf in range(topo.num_leaves):
        a, b = rng[topo.num_internal + lf]
        cnt[a:b + 1, a:b + 1] += 1  # self block
        for e in range(near_off[lf], near_off[lf + 1]):
            c, d = rng[topo.num_internal + near_src[e]]
            cnt[a:b + 1, c:d + 1] += 1
    return cnt


@pytest.mark.parametrize("eps,orders,theta_max", [(1e-2, (2, 4, 6), 1.0), (1e-6, (4, 6), 0.8), (1e-9, (6,), 1.0)])
def test_lists_cover_every_particle_pair_once(eps, orders, theta_max):
    topo, power, fs = _inputs(n=1500)
    far_off, far_src, far_gear, near_off, near_src = aw.adaptive_walk(
        topo.left_child, topo.right_child, topo.centers_f64, topo.radii_f64, topo.num_internal, power, fs,
        G=1.0, eps=eps, theta_max=theta_max, orders=orders)
    assert far_gear.shape == far_src.shape
    assert far_gear.size == 0 or (far_gear.min() >= 0 and far_gear.max() < len(orders))
    cnt = _coverage(topo, far_off, far_src, near_off, near_src)
    assert (cnt == 1).all()


def test_tighter_eps_moves_work_to_the_near_field():
    topo, power, fs = _inputs(n=3000)
    res = {}
    for eps in (1e-3, 1e-6):
        fo, fsrc, fg, no, ns = aw.adaptive_walk(topo.left_child, topo.right_child, topo.centers_f64,
                                                topo.radii_f64, topo.num_internal, power, fs, G=1.0, eps=eps,
                                                theta_max=1.0, orders=(2, 4, 6))
        res[eps] = (fsrc.size, ns.size, np.bincount(fg, minlength=3))
    assert res[1e-6][1] > res[1e-3][1]  # more near pairs
    # the loose target uses the low gears more
    lo = lambda r: r[2][:2].sum() / max(1, r[2].sum())
    assert lo(res[1e-3]) > lo(res[1e-6])


def test_dehnen_power_of_a_point_mass():
    import oracle

    p = 7
    d = np.array([[0.3, -0.2, 0.5], [0.0, 0.0, -1.5], [2.0, 1.0, 0.0]])
    m = np.array([2.0, 0.5, 1.5])
    mult = oracle.p2m(p, d, m)
    P = aw.dehnen_power(mult, p)
    r = np.linalg.norm(d, axis=1)
    want = m[:, None] * r[:, None] ** np.arange(p + 1)[None, :]
    np.testing.assert_allclose(P, want, rtol=1e-12)
