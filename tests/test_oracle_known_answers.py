"""The CPU oracle against the reference's known-answer identities
(jaccpot tests/unit/operators/test_real_harmonics.py) and physics anchors
(tests/integration/test_real_basis_runtime.py).  These pin the oracle's
conventions (normalisation, signs, delta directions) independently of any
tree or list."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from jaccpot_b200 import _tables, tree


def shi(n, m):
    return n * n + n + m


def test_sh_layout():
    assert [O.sh_size(p) for p in (0, 1, 4, 8, 12)] == [1, 4, 25, 81, 169]
    idx = [shi(n, m) for n in range(7) for m in range(-n, n + 1)]
    assert idx == list(range(49))


def test_dehnen_table3_degree_one():
    # test_real_harmonics.py:91-118: U_1^-1 = y/2, U_1^0 = z, U_1^1 = x/2
    for d in [(1.0, 0, 0), (0, 1.0, 0), (0, 0, 1.0), (0.3, -0.7, 0.2)]:
        u = O.p2m(1, np.array(d), [1.0])[0]
        assert u[0] == pytest.approx(1.0)
        assert u[1] == pytest.approx(d[1] / 2, abs=1e-14)
        assert u[2] == pytest.approx(d[2], abs=1e-14)
        assert u[3] == pytest.approx(d[0] / 2, abs=1e-14)


def test_p2m_monopole_and_linearity():
    rng = np.random.default_rng(0)
    d = rng.normal(size=3)
    a = O.p2m(6, d, [2.5])[0]
    b = O.p2m(6, d, [1.0])[0]
    assert a[0] == pytest.approx(2.5)
    np.testing.assert_allclose(a, 2.5 * b, rtol=1e-14)
    z = O.p2m(6, np.zeros(3), [3.0])[0]
    assert z[0] == 3.0 and np.all(np.abs(z[1:]) < 1e-50)  # radius floored at 1e-30


def _fd_jacobian(p, d, h=1e-6):
    J = np.zeros((O.sh_size(p), 3))
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        J[:, k] = (O.p2m(p, d + e, [1.0])[0] - O.p2m(p, d - e, [1.0])[0]) / (2 * h)
    return J


def test_z_derivative_lowers_the_degree():
    # test_real_harmonics.py:150-189: dU_n^m/dz = U_{n-1}^m
    rng = np.random.default_rng(20260806)
    p = 6
    for _ in range(3):
        d = rng.normal(size=3)
        U = O.p2m(p, d, [1.0])[0]
        J = _fd_jacobian(p, d)
        for n in range(1, p + 1):
            for m in range(-n, n + 1):
                want = U[shi(n - 1, m)] if abs(m) <= n - 1 else 0.0
                assert J[shi(n, m), 2] == pytest.approx(want, abs=2e-8 * max(1.0, abs(want)))


def test_l2p_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    for p in (2, 4, 8):
        F = rng.normal(size=O.sh_size(p))
        d = rng.normal(size=3)
        _, g = O.l2p(p, F, d)
        h = 1e-6
        for k in range(3):
            e = np.zeros(3)
            e[k] = h
            fd = (O.l2p(p, F, d + e)[0] - O.l2p(p, F, d - e)[0]) / (2 * h)
            assert g[0, k] == pytest.approx(fd[0], rel=1e-6, abs=1e-8)


@pytest.mark.parametrize("ell", range(0, 11))
def test_b_matrix_is_an_involution(ell):
    # test_real_harmonics.py:426
    B = O.bu_matrix(ell)
    np.testing.assert_allclose(B @ B, np.eye(2 * ell + 1), atol=1e-12)


@pytest.mark.parametrize("ell", range(0, 11))
def test_kernel_table_matches_oracle_and_sparsity_rule(ell):
    Bg = _tables.bu_matrix(ell)
    Bo = O.bu_matrix(ell)
    np.testing.assert_allclose(Bg, Bo, atol=1e-13)
    w = 2 * ell + 1
    for i in range(w):
        for j in range(w):
            if not _tables.bu_nonzero(ell, i, j):
                assert abs(Bo[i, j]) < 1e-13


def test_m2l_monopole_gives_inverse_distance():
    # test_real_harmonics.py:528-538
    M = O.p2m(6, np.zeros(3), [1.0])
    for d in ([0.0, 0.0, 2.0], [1.5, -0.5, 0.25], [0.0, 3.0, 0.0]):
        L = O.m2l(6, M, np.array(d))
        assert L[0, 0] == pytest.approx(1.0 / np.linalg.norm(d), rel=1e-13)


def _potential_via_expansions(p, src, mass, c_src, c_tgt, x):
    M = O.p2m(p, src - c_src, mass).sum(axis=0)
    L = O.m2l(p, M, c_tgt - c_src)
    phi, g = O.l2p(p, L[0], c_tgt - x)
    return phi[0], g[0]


def test_m2l_converges_with_order():
    # test_real_harmonics.py:541 (z axis) and :1216 (rotated geometry)
    rng = np.random.default_rng(5)
    src = rng.uniform(-0.3, 0.3, size=(20, 3))
    mass = rng.uniform(0.5, 1.5, size=20)
    c_src = np.average(src, axis=0, weights=mass)
    c_tgt = c_src + np.array([1.6, -0.9, 1.1])
    x = c_tgt + np.array([0.1, -0.2, 0.15])
    exact = np.sum(mass / np.linalg.norm(x - src, axis=1))
    errs = [abs(_potential_via_expansions(p, src, mass, c_src, c_tgt, x)[0] - exact) / exact for p in (2, 4, 6, 8, 10)]
    assert all(b < a for a, b in zip(errs, errs[1:]))
    assert errs[-1] < 1e-7


def test_single_particle_pipeline_force():
    # test_real_harmonics.py:991: P2M -> M2L -> L2P reproduces 1/r and its gradient
    y = np.array([0.05, -0.02, 0.03])
    c_src = np.zeros(3)
    c_tgt = np.array([2.0, 1.0, -1.5])
    x = c_tgt + np.array([-0.05, 0.04, 0.02])
    phi, g = _potential_via_expansions(10, y[None], [1.0], c_src, c_tgt, x)
    r = x - y
    assert phi == pytest.approx(1.0 / np.linalg.norm(r), rel=1e-9)
    # grad w.r.t. delta = centre - x is minus the gradient w.r.t. x
    np.testing.assert_allclose(-g, -r / np.linalg.norm(r) ** 3, rtol=1e-7)


def test_m2m_is_exact_for_truncated_multipoles():
    # M2M(P2M(x - c1), c1 - c2) == P2M(x - c2): translations of regular harmonics are exact
    rng = np.random.default_rng(11)
    for p in (3, 6, 9):
        x = rng.normal(size=3)
        c1 = rng.normal(size=3)
        c2 = rng.normal(size=3)
        a = O.m2m(p, O.p2m(p, x - c1, [1.3]), c1 - c2)[0]
        b = O.p2m(p, x - c2, [1.3])[0]
        np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-12 * np.abs(b).max())


def test_l2l_preserves_evaluation():
    # test_real_harmonics.py:944: a truncated local re-expanded about a child
    # centre evaluates to the same polynomial
    rng = np.random.default_rng(13)
    for p in (2, 5, 8):
        F = rng.normal(size=O.sh_size(p)) * 0.3 ** np.repeat(np.arange(p + 1), 2 * np.arange(p + 1) + 1)
        c1 = rng.normal(size=3)
        c2 = c1 + 0.3 * rng.normal(size=3)
        F2 = O.l2l(p, F, c1 - c2)[0]
        for _ in range(3):
            x = c2 + 0.2 * rng.normal(size=3)
            a, ga = O.l2p(p, F, c1 - x)
            b, gb = O.l2p(p, F2, c2 - x)
            assert a[0] == pytest.approx(b[0], rel=1e-11, abs=1e-12)
            np.testing.assert_allclose(ga[0], gb[0], rtol=1e-9, atol=1e-11)


def test_m2l_delta_sign_convention():
    # test_real_harmonics.py:1761: delta = target - source; the wrong sign is worse
    rng = np.random.default_rng(17)
    src = rng.uniform(-0.2, 0.2, size=(10, 3))
    mass = np.ones(10)
    c_src = src.mean(axis=0)
    c_tgt = np.array([1.5, 0.7, -0.4])
    x = c_tgt + np.array([0.05, 0.05, -0.05])
    exact = np.sum(1.0 / np.linalg.norm(x - src, axis=1))
    M = O.p2m(6, src - c_src, mass).sum(axis=0)
    good = O.l2p(6, O.m2l(6, M, c_tgt - c_src)[0], c_tgt - x)[0][0]
    bad = O.l2p(6, O.m2l(6, M, c_src - c_tgt)[0], c_tgt - x)[0][0]
    assert abs(good - exact) / exact < 1e-6
    assert abs(bad - exact) / exact > 1e-2


def _fmm(pos, mass, p, leaf, theta, eps2, dtype=np.float64):
    t = tree.build_topology(pos, mass, leaf_size=leaf, theta=theta)
    r = O.Pass(t, dtype).run(p, pos[t.permutation], mass[t.permutation], G=1.0, eps2=eps2)
    acc = np.empty_like(r["acc"], dtype=np.float64)
    acc[t.permutation] = r["acc"]
    return acc, t


def test_physics_anchor_small_system():
    # test_real_basis_runtime.py:52-77: N=96, leaf 8, p=4, softening 1e-2: rel-L2 < 5e-3
    rng = np.random.default_rng(0)
    pos = rng.uniform(-1, 1, size=(96, 3))
    mass = rng.uniform(0.5, 1.5, size=96)
    acc, t = _fmm(pos, mass, 4, 8, 0.5, 1e-4)
    d, _ = O.direct_sum(pos, mass, eps2=1e-4)
    assert t.num_far_pairs > 0
    assert np.linalg.norm(acc - d) / np.linalg.norm(d) < 5e-3


def test_fmm_converges_with_order():
    # test_real_basis_runtime.py:80-120
    rng = np.random.default_rng(1)
    pos = rng.uniform(-1, 1, size=(2000, 3))
    mass = rng.uniform(0.5, 1.5, size=2000)
    d, _ = O.direct_sum(pos, mass)
    errs = []
    for p in (2, 4, 6, 8):
        acc, _ = _fmm(pos, mass, p, 16, 0.5, 0.0)
        errs.append(np.linalg.norm(acc - d) / np.linalg.norm(d))
    assert all(b < 0.5 * a for a, b in zip(errs, errs[1:]))
    assert errs[-1] < 1e-5


def test_float32_oracle_tracks_float64():
    rng = np.random.default_rng(2)
    pos = rng.uniform(-1, 1, size=(3000, 3))
    mass = rng.uniform(0.5, 1.5, size=3000)
    a64, _ = _fmm(pos, mass, 6, 16, 0.6, 0.0, np.float64)
    a32, _ = _fmm(pos, mass, 6, 16, 0.6, 0.0, np.float32)
    e = np.linalg.norm(a32 - a64, axis=1) / np.linalg.norm(a64, axis=1)
    assert np.percentile(e, 99) < 1e-5
