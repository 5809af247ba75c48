"""The two near-field forms of jb_leaf_eval (jb_set_leaf_form): one lane per
target, or the chunk-major walk over all 32 lanes for leaves of more than 16
particles.  Both add the same per-chunk sums in the same order, and 1/r from
the flush-to-zero instruction equals rsqrtf for the normal squared distances
these inputs have, so the accelerations (and potentials) must be equal bit
for bit, for whole and
split leaves, with and without compensation, with and without a self block
(target-range passes)."""

from __future__ import annotations

import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import _lib, engine, tree, workloads  # noqa: E402

CASES = [("clustered", 262_144, 32, 0.55, 4096), ("plummer", 131_072, 32, 0.6, 96),
         ("uniform", 65_536, 24, 0.5, 4096), ("clustered", 50_000, 20, 0.7, 40),
         ("uniform", 3_000, 32, 0.6, 33)]


def _pass(kind, n, leaf, theta, unit_sources, p2p_mode, leaf_range=None):
    pos, mass = workloads.GENERATORS[kind](n, 4)
    mass[::11] = 0.0
    topo = tree.build_topology(pos, mass, leaf_size=leaf, theta=theta, device="cuda")
    dt = engine.DeviceTopology(topo, "cuda")
    ps = engine.Pass(dt, 4, G=1.0, eps2=1e-7, p2p_mode=p2p_mode, leaf_unit_sources=unit_sources,
                     leaf_range=leaf_range)
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
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


@pytest.mark.parametrize("mode", ["fp32", "kahan"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}-leaf{c[2]}-u{c[4]}")
def test_chunk_major_form_is_bit_identical(case, mode):
    p2p = _lib.JB_P2P_KAHAN if mode == "kahan" else _lib.JB_P2P_FP32
    ps, topo = _pass(*case, p2p)
    occ = topo.node_ranges[topo.num_internal:, 1] - topo.node_ranges[topo.num_internal:, 0] + 1
    assert (occ > 16).any()  # the chunk-major form runs
    for pot in (False, True):
        a, b = _both(ps, potential=pot)
        assert torch.isfinite(a).all()
        assert torch.equal(a, b), (a - b).abs().max().item()
    a, b = _both(ps, part="near")
    assert torch.equal(a, b)


def test_chunk_major_form_on_a_leaf_range():
    ps, topo = _pass("clustered", 131_072, 32, 0.55, 200, _lib.JB_P2P_KAHAN,
                     leaf_range=(1000, 2500))
    a, b = _both(ps)
    assert torch.equal(a, b)


def test_leaf_form_argument_is_checked():
    lb = _lib.lib()
    assert lb.jb_set_leaf_form(2) == 1
    assert lb.jb_set_leaf_form(-1) == 1
    assert lb.jb_set_leaf_form(1) == 0
