"""Host prepare (tree + lists + work-unit schedules): structural invariants
and completeness of the interaction lists -- every (target leaf, source
particle) pair is covered exactly once, either directly (self or near list) or
through exactly one far pair of an ancestor."""

from __future__ import annotations

import numpy as np
import pytest

from jaccpot_b200 import _lib, schedule, tree, workloads

CASES = [("uniform", 5000, 16, 0.6), ("clustered", 8000, 32, 0.5), ("plummer", 6000, 8, 0.7)]


@pytest.fixture(scope="module", params=CASES, ids=lambda c: f"{c[0]}-{c[1]}")
def topo(request):
    gen, n, leaf, th = request.param
    pos, mass = workloads.GENERATORS[gen](n, 3)
    return tree.build_topology(pos, mass, leaf_size=leaf, theta=th), pos.astype(np.float64), mass


def test_structure(topo):
    t, pos, _ = topo
    ni, nn, nl = t.num_internal, t.num_nodes, t.num_leaves
    assert nn == 2 * nl - 1 and ni == nl - 1
    assert np.array_equal(np.sort(t.permutation), np.arange(t.num_particles))
    assert np.array_equal(t.inverse_permutation[t.permutation], np.arange(t.num_particles))
    r = t.node_ranges
    assert r[0, 0] == 0 and r[0, 1] == t.num_particles - 1
    cnt = r[:, 1] - r[:, 0] + 1
    assert np.all(cnt[ni:] <= t.leaf_size) and np.all(cnt[:ni] > t.leaf_size)
    # leaves tile the sorted particles in order
    assert np.array_equal(r[ni:, 0], np.concatenate([[0], r[ni:-1, 1] + 1]))
    for i in range(ni):
        a, b = t.left_child[i], t.right_child[i]
        assert a > i and b > i
        assert r[a, 0] == r[i, 0] and r[b, 1] == r[i, 1] and r[a, 1] + 1 == r[b, 0]
        assert t.parent[a] == i and t.parent[b] == i
        assert t.node_level[a] == t.node_level[i] + 1
    lo = t.level_offsets
    assert lo[0] == 0 and lo[-1] == ni and np.all(np.diff(lo) > 0)
    for lev in range(t.num_levels):
        assert np.all(t.node_level[lo[lev]:lo[lev + 1]] == lev)
    leaf_of = np.repeat(np.arange(nl), cnt[ni:])
    assert np.array_equal(t.leaf_of_particle, leaf_of)
    # Morton order is spatially coherent: leaves are compact relative to the box
    ext = np.ptp(pos, axis=0).max()
    assert np.median(t.radii_f64[ni:]) < 0.2 * ext


def test_mac_and_symmetry(topo):
    t, _, _ = topo
    c, rad = t.centers_f64, t.radii_f64
    tg = np.repeat(np.arange(t.num_nodes), np.diff(t.far_offsets))
    sr = t.far_sources
    d = np.linalg.norm(c[tg] - c[sr], axis=1)
    th = t.theta
    assert np.all(rad[tg] + rad[sr] <= th * d * (1 + 1e-12))
    assert set(zip(tg.tolist(), sr.tolist())) == set(zip(sr.tolist(), tg.tolist()))
    ni = t.num_internal
    nt = np.repeat(np.arange(t.num_leaves), np.diff(t.near_offsets))
    ns = t.near_leaves
    assert np.all(nt != ns)
    dn = np.linalg.norm(c[ni + nt] - c[ni + ns], axis=1)
    assert np.all((rad[ni + nt] + rad[ni + ns] > th * dn) | (dn == 0))
    assert set(zip(nt.tolist(), ns.tolist())) == set(zip(ns.tolist(), nt.tolist()))


def test_lists_cover_every_pair_exactly_once(topo):
    t, _, _ = topo
    ni, nl = t.num_internal, t.num_leaves
    r = t.node_ranges
    leaf_lo = t.leaf_of_particle[r[:, 0]]
    leaf_hi = t.leaf_of_particle[r[:, 1]]
    for T in range(0, nl, max(1, nl // 200)):
        cov = np.zeros(nl, dtype=np.int64)
        cov[T] += 1
        cov[t.near_leaves[t.near_offsets[T]:t.near_offsets[T + 1]]] += 1
        node = ni + T
        while node >= 0:
            for s in t.far_sources[t.far_offsets[node]:t.far_offsets[node + 1]]:
                cov[leaf_lo[s]:leaf_hi[s] + 1] += 1
            node = t.parent[node]
        assert np.all(cov == 1), (T, np.unique(cov))


def test_work_unit_schedules_cover_the_lists(topo):
    t, _, _ = topo
    ms = schedule.m2l_schedule(t, max_pairs=16)
    cov = np.zeros(t.num_far_pairs, dtype=np.int64)
    for tg, a, b, slot in ms.units:
        assert t.far_offsets[tg] <= a < b <= t.far_offsets[tg + 1] and b - a <= 16
        cov[a:b] += 1
    assert np.all(cov == 1)
    for tg, first, cnt, _ in ms.split:
        assert sorted(ms.units[ms.units[:, 0] == tg][:, 3].tolist()) == list(range(first, first + cnt))
    ls = schedule.leaf_schedule(t, max_sources=64)
    ni = t.num_internal
    for lf in range(t.num_leaves):
        us = ls.units[ls.units[:, 0] == lf]
        ax = ls.aux[ls.units[:, 0] == lf]
        assert ax[:, 1].sum() == 1
        parts = [np.arange(s, s + c) for u in us for s, c in ls.runs[u[1]:u[2]]]
        got = np.sort(np.concatenate(parts)) if parts else np.zeros(0, np.int64)
        nb = t.near_leaves[t.near_offsets[lf]:t.near_offsets[lf + 1]]
        want = np.sort(np.concatenate([np.arange(t.node_ranges[ni + j, 0], t.node_ranges[ni + j, 1] + 1)
                                       for j in nb])) if nb.size else np.zeros(0, np.int64)
        assert np.array_equal(got, want)
        assert np.array_equal(np.sort(us[:, 3]), np.sort([ls.runs[u[1]:u[2], 1].sum() for u in us]))


@pytest.mark.parametrize("leaf_range", [None, (3, 40)])
def test_leaf_ancestor_schedule(topo, leaf_range):
    """engine.l2l_leaf_schedule (the units of jb_l2l_leaves): one unit per leaf
    of the range that has an ancestor with far pairs, listing exactly those
    ancestors, nearest first; longest lists first.  With the far lists the
    chains cover every far pair whose target contains the leaf, once."""
    from jaccpot_b200 import engine

    t, _, _ = topo
    rng = (0, t.num_leaves) if leaf_range is None else leaf_range
    units, anc = engine.l2l_leaf_schedule(t, rng)
    ni = t.num_internal
    has_far = np.diff(t.far_offsets) > 0
    lens = units[:, 2] - units[:, 1]
    assert (lens > 0).all() and (np.diff(lens) <= 0).all() and (units[:, 3] == -1).all()
    seen = set()
    for leaf, a, b, _ in units:
        assert rng[0] <= leaf - ni < rng[1] and leaf not in seen
        seen.add(int(leaf))
        chain, c = [], int(t.parent[leaf])
        while c >= 0:
            if has_far[c]:
                chain.append(c)
            c = int(t.parent[c])
        assert list(anc[a:b]) == chain
    for lf in range(rng[0], rng[1]):  # leaves left out have no such ancestor
        if ni + lf not in seen:
            c = int(t.parent[ni + lf])
            while c >= 0:
                assert not has_far[c]
                c = int(t.parent[c])


def test_single_leaf_tree():
    pos = np.random.default_rng(0).normal(size=(10, 3))
    t = tree.build_topology(pos, np.ones(10), leaf_size=16, theta=0.6)
    assert t.num_nodes == 1 and t.num_internal == 0 and t.num_levels == 0
    assert t.num_far_pairs == 0 and t.num_near_pairs == 0


def test_bad_inputs_raise():
    pos = np.zeros((4, 3))
    with pytest.raises(_lib.JBError):
        tree.build_topology(pos, np.ones(4), leaf_size=0)
    with pytest.raises(_lib.JBError):
        tree.build_topology(pos, np.ones(4), theta=1.0)
    bad = pos.copy()
    bad[1, 2] = np.nan
    with pytest.raises(_lib.JBError):
        tree.build_topology(bad, np.ones(4))
    with pytest.raises(ValueError):
        tree.build_topology(pos, np.ones(3))


def test_duplicate_positions_terminate():
    pos = np.zeros((100, 3))
    t = tree.build_topology(pos, np.ones(100), leaf_size=8, theta=0.5)
    cnt = t.node_ranges[:, 1] - t.node_ranges[:, 0] + 1
    assert cnt[t.num_internal:].max() <= 8 and t.num_far_pairs == 0
