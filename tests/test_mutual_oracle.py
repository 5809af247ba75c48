"""The property the mutual lane rests on, checked with the FP64 oracle on the
host-built lists: with symmetric far/near lists, centre-of-mass expansions and
the triangular M2L truncation, the pass's forces sum to zero to round-off at
every order -- the reference's mutual claim (mutual/farfield.py: |F_A + F_B|
~4e-16 relative, flat in theta and order) -- and the canonical lists hold
every pair exactly once."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from jaccpot_b200 import mutual, tree, workloads


@pytest.fixture(scope="module")
def built():
    O.build()
    return True


@pytest.mark.parametrize("kind", ["uniform", "plummer", "clustered"])
@pytest.mark.parametrize("p", [2, 4, 8])
def test_pass_conserves_momentum_to_round_off(built, kind, p):
    pos, mass = workloads.GENERATORS[kind](4096, 5)
    pos, mass = pos.astype(np.float64), mass.astype(np.float64)
    t = tree.build_topology(pos, mass, leaf_size=16, theta=0.6)
    out = O.Pass(t, np.float64).run(p, pos[t.permutation], mass[t.permutation], G=1.0, eps2=1e-6)
    F = mass[t.permutation][:, None] * out["acc"][:, :3]
    assert mutual.momentum_residual(F) < 1e-13


def test_canonical_lists_hold_every_pair_once():
    pos, mass = workloads.clustered(6000, 2)
    t = tree.build_topology(pos, mass, leaf_size=16, theta=0.55)
    mt = mutual.build_mutual_topology_from_tree(t, order=6)
    assert (mt.far_a < mt.far_b).all() and (mt.near_a < mt.near_b).all()
    assert 2 * mt.far_a.size == t.num_far_pairs and 2 * mt.near_a.size == t.num_near_pairs
    canon = set(zip(mt.far_a.tolist(), mt.far_b.tolist()))
    tgt = t.far_pair_targets()
    both = {(min(a, b), max(a, b)) for a, b in zip(tgt.tolist(), t.far_sources.tolist())}
    assert canon == both and len(canon) == mt.far_a.size
    assert mt.self_leaves.size == t.num_leaves and mt.leaf_nodes[0] == t.num_internal


def test_block_step_bookkeeping():
    """Boundary weights of a 2**k_max sub-step base step (force.py:685-883
    there): ends kick every level with half weight, inner boundaries kick the
    levels at or above the trailing-zero floor."""
    k = 3
    assert mutual.n_sub(k) == 8
    assert mutual.is_sync_boundary(0, k) and mutual.is_sync_boundary(8, k) and not mutual.is_sync_boundary(4, k)
    assert [mutual.active_level_floor(s, k) for s in range(9)] == [0, 3, 2, 3, 1, 3, 2, 3, 0]
    w = mutual.boundary_level_weights(0, k, 1.0)
    assert np.allclose(w, [0.5, 0.25, 0.125, 0.0625])
    assert np.allclose(mutual.boundary_level_weights(2, k, 1.0), [0, 0, 0.25, 0.125])
    table = mutual.boundary_weight_table(k, 2.0)
    assert table.shape == (9, 4) and np.allclose(table[4], [0, 1.0, 0.5, 0.25])
    # every level receives dt_max / 2**k per its own sub-step over the base step
    assert np.allclose(table.sum(0), 2.0)
