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
