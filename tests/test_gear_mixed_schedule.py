"""The mixed gear schedule (one-launch gear M2L) on the CPU: its units cover
every target's far list exactly once, in order; the pairs of each segment
carry that segment's order; slots and split entries are consistent; units
are sorted by decreasing segment lengths, highest order first."""

from __future__ import annotations

import numpy as np
import pytest

from jaccpot_b200 import schedule, tree, workloads

ORDERS = (2, 4, 6, 8)


@pytest.fixture(scope="module")
def topo():
    pos, mass = workloads.clustered(6000, seed=3)
    return tree.build_topology(pos, mass, leaf_size=16, theta=0.6)


def _gears(t, ng, seed):
    rng = np.random.default_rng(seed)
    g = rng.integers(0, ng, size=t.num_far_pairs)
    g[: g.size // 3] = np.sort(g[: g.size // 3])  # runs of equal gears, as a walk emits them
    return g


def test_ladder():
    assert schedule.mixed_ladder(8) == (8, 6, 4, 2)
    assert schedule.mixed_ladder(10) == (10, 8, 6, 4)
    assert schedule.mixed_ladder(5) == (5, 3, 1)
    assert schedule.mixed_ladder(2) == (2,)


@pytest.mark.parametrize("orders,max_pairs", [(ORDERS, 128), (ORDERS, 7), ((4, 8), 32), ((8,), 64)])
def test_units_cover_lists_by_segment(topo, orders, max_pairs):
    t = topo
    ng = len(orders)
    g = _gears(t, ng, 11)
    gs = schedule.gear_m2l_mixed_schedule(t, g, orders, 8, max_pairs=max_pairs)
    off = t.far_offsets
    seg_of = np.array([(8 - o) // 2 for o in orders])
    tgt = np.repeat(np.arange(t.num_nodes), np.diff(off))
    order = np.lexsort((seg_of[g], tgt))
    seg_sorted = seg_of[g][order]
    assert np.array_equal(gs.far_src, t.far_sources[order])
    assert np.array_equal(gs.pairs_per_gear, np.bincount(g, minlength=ng))
    u, b = gs.units, gs.bounds
    assert u.shape == b.shape
    # every target's list is covered once by its units, which are at most max_pairs long
    covered = np.zeros(t.num_far_pairs, np.int64)
    for (tt, s, e, _), bb in zip(u, b):
        assert off[tt] <= s < e <= off[tt + 1] and e - s <= max_pairs
        bd = [s, *bb[:3], bb[3]]
        assert bb[3] == e and all(bd[j] <= bd[j + 1] for j in range(4))
        for j in range(4):
            assert np.all(seg_sorted[bd[j]:bd[j + 1]] == j)
        covered[s:e] += 1
    assert np.all(covered == 1)
    # slots: a target with several units owns consecutive slots, summed by its split entry
    n_units = np.bincount(u[:, 0], minlength=t.num_nodes)
    multi = n_units > 1
    assert np.all(u[~multi[u[:, 0]], 3] == -1)
    assert gs.num_slots == int(n_units[multi].sum())
    assert gs.split.shape[0] == int(multi.sum())
    for tt, first, n, _ in gs.split:
        slots = np.sort(u[u[:, 0] == tt, 3])
        assert n == n_units[tt] and np.array_equal(slots, np.arange(first, first + n))
    # sorted by segment lengths, highest order first (lexicographically non-increasing)
    c = np.diff(np.concatenate([u[:, 1:2], b], axis=1), axis=1)
    for a, bb in zip(c[:-1], c[1:]):
        assert tuple(a) >= tuple(bb)


def test_orders_off_the_ladder_are_refused(topo):
    g = _gears(topo, 3, 2)
    with pytest.raises(ValueError):
        schedule.gear_m2l_mixed_schedule(topo, g, (3, 5, 8), 8)
    with pytest.raises(ValueError):
        schedule.gear_m2l_mixed_schedule(topo, g[:, None].repeat(2, 1).ravel(), (4, 6, 8), 8)
