"""The two near-field forms of jb_leaf_eval (jb_set_leaf_form): one lane per
target over 32-source chunks, or, for leaves of more than 16 particles, the
chunk-major walk over all 32 lanes with 64-source chunks.  They sum the same
particle pairs with the same per-pair arithmetic (1/r from the flush-to-zero
instruction in both) but group the partial sums differently, so they agree to
FP32 rounding -- for whole and split leaves, with and without compensation,
with and without a self block (target-range passes).  Leaves of at most 16
particles take the same lane-group code in both forms: bit-identical there."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import _lib, engine, tree, workloads  # noqa: E402

CASES = [("clustered", 262_144, 32, 0.55, 4096), ("plummer", 131_072, 32, 0.6, 96),
         ("uniform", 65_536, 24, 0.5, 4096), ("clustered", 50_000, 20, 0.7, 40),
         ("uniform", 3_000, 32, 0.6, 33), ("plummer", 131_072, 64, 0.6, 256),
         ("clustered", 65_536, 48, 0.55, 100)]


def _pass(kind, n, leaf, theta, unit_sources, p2p_mode, leaf_range=None):
    pos, mass = workloads.GENERATORS[kind](n, 4)
    mass[::11] = 0.0
    topo = tree.build_topology(pos, mass, leaf_size=leaf, theta=theta, device="cuda")
    dt = engine.DeviceTopology(topo, "cuda")
    ps = engine.Pass(dt, 4, G=1.0, eps2=1e-7, p2p_mode=p2p_mode, leaf_unit_sources=unit_sources,
                     leaf_range=leaf_range)
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    ps.upward()
    ps.downward()  # the locals the far field reads
    return ps, topo


def _both(ps, **kw):
    lb = _lib.lib()
    out = []
    try:
        for form in (0, 1):
            _lib.check(lb.jb_set_leaf_form(form), "jb_set_leaf_form")
            out.append(ps.evaluate(**kw).clone())
            torch.cuda.synchronize()
    finally:
        lb.jb_set_leaf_form(1)
    return out


def _agree(a, b, topo):
    """FP32-rounding agreement of two results; bit-identical on the particles
    of leaves of at most 16 (the same code in both forms)."""
    assert torch.isfinite(a).all() and torch.isfinite(b).all()
    an = torch.linalg.vector_norm(a[:, :3], dim=1).clamp_min(1e-30)
    rel = (torch.linalg.vector_norm(a[:, :3] - b[:, :3], dim=1) / an).double().cpu().numpy()
    assert np.percentile(rel, 99) <= 2e-6 and np.percentile(rel, 99.9) <= 2e-5, np.percentile(rel, [99, 99.9, 100])
    occ = topo.node_ranges[topo.num_internal:, 1] - topo.node_ranges[topo.num_internal:, 0] + 1
    small = np.repeat(occ <= 16, occ)
    idx = torch.from_numpy(np.nonzero(small)[0]).cuda()
    assert torch.equal(a[idx], b[idx])


@pytest.mark.parametrize("mode", ["fp32", "kahan"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}-leaf{c[2]}-u{c[4]}")
def test_chunk_major_form_agrees(case, mode):
    p2p = _lib.JB_P2P_KAHAN if mode == "kahan" else _lib.JB_P2P_FP32
    ps, topo = _pass(*case, p2p)
    occ = topo.node_ranges[topo.num_internal:, 1] - topo.node_ranges[topo.num_internal:, 0] + 1
    assert (occ > 16).any()  # the chunk-major form runs
    for pot in (False, True):
        a, b = _both(ps, potential=pot)
        _agree(a, b, topo)
    a, b = _both(ps, part="near")
    _agree(a, b, topo)


def test_chunk_major_form_on_a_leaf_range():
    ps, topo = _pass("clustered", 131_072, 32, 0.55, 200, _lib.JB_P2P_KAHAN,
                     leaf_range=(1000, 2500))
    a, b = _both(ps)
    lo = int(topo.node_ranges[topo.num_internal + 1000, 0])
    hi = int(topo.node_ranges[topo.num_internal + 2499, 1]) + 1
    sub = lambda x: x[lo:hi]
    occ = topo.node_ranges[topo.num_internal + 1000:topo.num_internal + 2500]
    occ = occ[:, 1] - occ[:, 0] + 1
    an = torch.linalg.vector_norm(sub(a)[:, :3], dim=1).clamp_min(1e-30)
    rel = (torch.linalg.vector_norm(sub(a)[:, :3] - sub(b)[:, :3], dim=1) / an).double().cpu().numpy()
    assert np.percentile(rel, 99) <= 2e-6


def test_leaf_form_argument_is_checked():
    lb = _lib.lib()
    assert lb.jb_set_leaf_form(2) == 1
    assert lb.jb_set_leaf_form(-1) == 1
    assert lb.jb_set_leaf_form(1) == 0
