"""Pins the host tree builder (jb_tree_build) to the pure-Python restatement in
oracle/tree.py: every array -- permutation, node ranges, children, parents,
levels, leaf map, far / near CSR lists, FP64 centres and radii -- must be
equal bit for bit.  The GPU builder is pinned to the host one (and to this
oracle) in tests/test_gpu_tree.py."""

from __future__ import annotations

import numpy as np
import pytest

from jaccpot_b200 import tree, workloads
from oracle import tree as OT

FIELDS = ("permutation", "node_ranges", "left_child", "right_child", "parent", "node_level", "level_offsets",
          "leaf_of_particle", "far_offsets", "far_sources", "near_offsets", "near_leaves", "centers_f64",
          "radii_f64")


def _inputs(kind: str, n: int, seed: int):
    rng = np.random.default_rng(seed)
    if kind in workloads.GENERATORS:
        pos, mass = workloads.GENERATORS[kind](n, seed)
        return np.asarray(pos, np.float64), np.asarray(mass, np.float64)
    if kind == "duplicates":  # four distinct points, repeated
        pts = rng.uniform(-1, 1, size=(4, 3))
        return pts[rng.integers(0, 4, size=n)], rng.uniform(0.5, 1.5, size=n)
    if kind == "massless":  # a quarter of the particles without mass, one massless clump
        pos = rng.uniform(-1, 1, size=(n, 3))
        mass = rng.uniform(0.5, 1.5, size=n)
        mass[rng.random(n) < 0.25] = 0.0
        pos[: n // 8] = rng.normal(2.0, 0.01, size=(n // 8, 3))
        mass[: n // 8] = 0.0
        return pos, mass
    if kind == "zero_mass":
        return rng.uniform(-1, 1, size=(n, 3)), np.zeros(n)
    raise ValueError(kind)


CASES = [("uniform", 1500, 8, 0.5), ("clustered", 2500, 16, 0.6), ("plummer", 2000, 32, 0.55),
         ("duplicates", 300, 8, 0.6), ("massless", 1200, 8, 0.5), ("zero_mass", 600, 16, 0.6),
         ("uniform", 1, 8, 0.6), ("uniform", 16, 16, 0.6), ("uniform", 17, 16, 0.6), ("uniform", 200, 1, 0.7)]


def compare(got, want, where: str):
    for f in FIELDS:
        a, b = np.asarray(got[f]), np.asarray(want[f])
        assert a.shape == b.shape, (where, f, a.shape, b.shape)
        assert a.dtype == b.dtype, (where, f, a.dtype, b.dtype)
        assert np.array_equal(a.view(np.uint8) if a.dtype == np.float64 else a,
                              b.view(np.uint8) if b.dtype == np.float64 else b), (where, f)


def topo_fields(t) -> dict:
    return {f: getattr(t, f) for f in FIELDS}


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}-leaf{c[2]}")
def test_host_builder_matches_the_oracle_bit_for_bit(case):
    kind, n, leaf, theta = case
    pos, mass = _inputs(kind, n, 7)
    want = OT.build(pos, mass, leaf, theta)
    t = tree.build_topology(pos, mass, leaf_size=leaf, theta=theta)
    compare(topo_fields(t), want, str(case))
    assert t.num_levels == want["num_levels"]


@pytest.mark.parametrize("kind,n,leaf,theta", [("clustered", 3000, 8, 0.6), ("uniform", 2000, 16, 0.5),
                                               ("plummer", 4000, 32, 0.7), ("uniform", 1, 8, 0.6)])
def test_compiled_oracle_tree_equals_the_scalar_restatement(kind, n, leaf, theta):
    """oracle/tree_oracle.cpp (the oracle's fast tree, used by the benchmark's
    CPU legs) transcribes oracle/tree.py: the same arrays bit for bit."""
    import oracle
    from jaccpot_b200 import workloads
    from oracle import tree as otree

    pos, mass = workloads.GENERATORS[kind](n, 3)
    a = oracle.tree_build(pos, mass, leaf, theta)
    b = otree.build(pos, mass, leaf, theta)
    for k, v in b.items():
        if k == "num_levels":
            assert a.num_levels == v
        else:
            assert np.array_equal(getattr(a, k), v), k


def test_compiled_oracle_tree_equals_the_product_host_builder():
    import oracle
    from jaccpot_b200 import tree, workloads

    pos, mass = workloads.clustered(100_000, 9)
    a = oracle.tree_build(pos, mass, 32, 0.55)
    h = tree.build_topology(pos, mass, leaf_size=32, theta=0.55)
    for k in ("permutation", "node_ranges", "left_child", "right_child", "parent", "node_level", "level_offsets",
              "leaf_of_particle", "far_offsets", "far_sources", "near_offsets", "near_leaves", "centers_f64",
              "radii_f64"):
        assert np.array_equal(getattr(a, k), getattr(h, k)), k
