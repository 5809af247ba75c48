"""The float64 adjoint oracle (oracle/adjoint.py) against central finite
differences of the oracle's own forward pass at fixed topology, and against
the reference's committed gradient goldens (jaccpot
tests/characterization/golden_grad/*.npz: grad of sum(w * accel) for
uniform N=128/256, p=2/4, leaf 4, theta 0.5, softening 1e-2, w =
normal(PRNGKey(7), (N,3))) at FMM-accuracy level, with the reference's own
physics anchors against the direct-sum gradient (test_fmm_grad_golden.py)."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from oracle import adjoint as A
from jaccpot_b200 import tree, workloads

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import jax_prng  # noqa: E402

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "reference_goldens.npz")


def _setup(gen, n, p, leaf, theta=0.5, eps=1e-2, seed=0):
    pos, mass = workloads.GENERATORS[gen](n, seed)
    t = tree.build_topology(pos, mass, leaf_size=leaf, theta=theta)
    ps = pos[t.permutation].astype(np.float64)
    ms = mass[t.permutation].astype(np.float64)
    w = np.random.default_rng(seed + 11).normal(size=(n, 3))
    return t, ps, ms, w, eps * eps


@pytest.mark.parametrize("gen,n,p,leaf,hrel", [("uniform", 400, 4, 8, 1e-5), ("clustered", 1200, 6, 16, 1e-6)])
def test_adjoint_oracle_matches_finite_differences(gen, n, p, leaf, hrel):
    t, ps, ms, w, eps2 = _setup(gen, n, p, leaf)
    assert t.num_far_pairs > 0
    P = O.Pass(t, np.float64)

    def loss(x, m):
        return float((w * P.run(p, x, m, G=1.0, eps2=eps2)["acc"]).sum())

    xb, mb = A.fmm_vjp(t, p, ps, ms, w, 1.0, eps2)
    rng = np.random.default_rng(5)
    for i in rng.choice(n, 6, replace=False):
        for a in range(3):
            h = hrel * max(1.0, abs(ps[i, a]))
            x1, x2 = ps.copy(), ps.copy()
            x1[i, a] += h
            x2[i, a] -= h
            fd = (loss(x1, ms) - loss(x2, ms)) / (2 * h)
            assert abs(fd - xb[i, a]) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(xb).max())
        h = 1e-5 * ms[i]
        m1, m2 = ms.copy(), ms.copy()
        m1[i] += h
        m2[i] -= h
        fd = (loss(ps, m1) - loss(ps, m2)) / (2 * h)
        assert abs(fd - mb[i]) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(mb).max())


def test_translation_transposes():
    # the identities the GPU adjoint relies on
    rng = np.random.default_rng(0)
    d = rng.normal(size=(4, 3))
    for p in (3, 6):
        m2l = A._op_matrices(O.m2l, p, d)
        m2m = A._op_matrices(O.m2m, p, d)
        l2l = A._op_matrices(O.l2l, p, d)
        assert np.allclose(m2l, np.transpose(m2l, (0, 2, 1)), rtol=1e-12, atol=1e-12 * np.abs(m2l).max())
        assert np.allclose(np.transpose(m2m, (0, 2, 1)), l2l, rtol=1e-12, atol=1e-12 * np.abs(l2l).max())


def _direct_grad(pos, mass, w, eps2):
    """Analytic gradient of sum_i w_i . a_i(direct sum) w.r.t. positions and masses."""
    d = pos[:, None, :] - pos[None, :, :]
    r2 = (d * d).sum(-1) + eps2
    np.fill_diagonal(r2, 1.0)
    q = 1.0 / np.sqrt(r2)
    np.fill_diagonal(q, 0.0)
    q3, q5 = q ** 3, q ** 5
    wd_i = np.einsum("ia,ija->ij", w, d)
    wd_j = np.einsum("ja,ija->ij", w, d)
    gx = (-mass[None, :, None] * q3[..., None] * w[:, None, :] + mass[:, None, None] * q3[..., None] * w[None, :, :]
          + 3 * q5[..., None] * (mass[None, :] * wd_i - mass[:, None] * wd_j)[..., None] * d).sum(1)
    gm = (q3 * wd_j).sum(1)
    return gx, gm


@pytest.mark.parametrize("name,n,p", [("uni_real_n128_p2", 128, 2), ("uni_real_n128_p4", 128, 4),
                                      ("uni_real_n256_p4", 256, 4)])
def test_adjoint_oracle_against_reference_gradient_goldens(name, n, p):
    pos, mass = jax_prng.golden_inputs("uniform", n)
    w = jax_prng.normal(jax_prng.key(7), (n, 3))
    eps2 = 1e-4
    t = tree.build_topology(pos, mass, leaf_size=4, theta=0.5)
    assert t.num_far_pairs > 0
    perm = t.permutation
    xb_s, mb_s = A.fmm_vjp(t, p, pos[perm], mass[perm], w[perm], 1.0, eps2)
    xb, mb = np.empty_like(xb_s), np.empty_like(mb_s)
    xb[perm], mb[perm] = xb_s, mb_s
    gx_d, gm_d = _direct_grad(pos, mass, w, eps2)
    gold_x, gold_m = GOLD[f"grad_{name}/grad_positions"], GOLD[f"grad_{name}/grad_masses"]
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    # the golden is the reference's gradient of the same loss on the same inputs
    assert rel(gold_x, gx_d) < {2: 5e-3, 4: 2e-3}[p]
    # the reference's anchors (test_fmm_grad_golden.py ANCHOR_REL_L2_BY_ORDER)
    assert rel(xb, gx_d) < {2: 5e-3, 4: 2e-3}[p]
    assert rel(mb, gm_d) < {2: 2e-2, 4: 1e-2}[p]
    # and the two FMM gradients agree to within their truncation errors
    assert rel(xb, gold_x) <= rel(xb, gx_d) + rel(gold_x, gx_d) + 1e-12
    assert rel(mb, gold_m) <= rel(mb, gm_d) + rel(gold_m, gm_d) + 1e-12
