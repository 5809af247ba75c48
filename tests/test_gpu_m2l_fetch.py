"""The two source-row fetches of the single-order FP32 M2L (jb_set_m2l_fetch):
each thread copying its own row in 16-byte pieces, or the warp copying its 32
rows together, one instruction per row.  Only the copy differs; the
arithmetic is the same, compiled into two kernels (which may fuse a multiply
and an add differently), so the results agree to FP32 rounding: plain units
at several orders and unit lengths, the per-gear launches (and the mixed-order
launch, which fetches per thread either way), a target-range pass, the
weighted (block-step) M2L, the adjoint's transposed M2L (through the VJP) and
the whole pass."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import _lib, engine, tree, workloads  # noqa: E402


def _pass(kind, n, p, theta, leaf=32, seed=3, **kw):
    pos, mass = workloads.GENERATORS[kind](n, seed)
    mass[::13] = 0.0
    topo = tree.build_topology(pos, mass, leaf_size=leaf, theta=theta, device="cuda")
    dt = engine.DeviceTopology(topo, "cuda")
    ps = engine.Pass(dt, p, G=1.0, eps2=1e-7, **kw)
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    ps.upward()
    return ps, topo, pos


def _both(fn, p99=1e-5, worst=1e-4):
    lb = _lib.lib()
    out = []
    try:
        for warp_rows in (0, 1):
            _lib.check(lb.jb_set_m2l_fetch(warp_rows), "jb_set_m2l_fetch")
            r = fn()
            torch.cuda.synchronize()
            out.append([x.clone() for x in r] if isinstance(r, (tuple, list)) else [r.clone()])
    finally:
        lb.jb_set_m2l_fetch(1)
    for a, b in zip(*out):
        assert torch.isfinite(a).all() and torch.isfinite(b).all() and (a != 0).any()
        a2, b2 = a.reshape(a.shape[0], -1).double(), b.reshape(b.shape[0], -1).double()
        scale = a2.abs().max(dim=1).values
        rel = ((a2 - b2).abs().max(dim=1).values / scale.clamp_min(1e-300))[scale > 0].cpu().numpy()
        assert np.percentile(rel, 99) <= p99 and rel.max() <= worst, (np.percentile(rel, 99), rel.max())


def _locals(ps):
    def f():
        ps.m2l()
        return ps.ws.locals
    return f


@pytest.mark.parametrize("p", [1, 2, 4, 6, 8, 10])
def test_plain_units(p):
    ps, *_ = _pass("clustered", 65_536, p, 0.6)
    _both(_locals(ps))


@pytest.mark.parametrize("unit_pairs", [1, 7, 64])
def test_unit_lengths_and_a_leaf_range(unit_pairs):
    ps, *_ = _pass("plummer", 40_000, 6, 0.6, leaf=24, m2l_unit_pairs=unit_pairs, leaf_range=(50, 700))
    _both(_locals(ps))


@pytest.mark.parametrize("gear_form", ["mixed", "per_gear"])
def test_gear_units(gear_form):
    ps, topo, _ = _pass("clustered", 65_536, 8, 0.6, gear_form=gear_form)
    rng = np.random.default_rng(8)
    ps.set_gears(rng.integers(0, 4, topo.num_far_pairs), (2, 4, 6, 8))
    _both(_locals(ps))


def test_weighted_m2l():
    ps, topo, _ = _pass("uniform", 30_000, 5, 0.6)
    w = torch.rand(topo.num_far_pairs, device="cuda", dtype=torch.float32)

    def f():
        ps.m2l_weighted(w)
        return ps.ws.locals
    _both(f)


def test_whole_pass_and_vjp():
    ps, topo, pos = _pass("clustered", 32_768, 6, 0.6)
    n = pos.shape[0]
    gen = torch.Generator(device="cuda").manual_seed(3)
    w = torch.randn((n, 3), device="cuda", generator=gen)

    def f():
        acc = ps.run().clone()
        gp = torch.zeros((n, 3), device="cuda")
        gm = torch.zeros((n,), device="cuda")
        ps.vjp(w, gp, gm)
        return acc, gp, gm
    _both(f, p99=1e-5, worst=1e-2)  # gradients: sums with cancellation


def test_fetch_argument_is_checked():
    lb = _lib.lib()
    assert lb.jb_set_m2l_fetch(2) == 1
    assert lb.jb_set_m2l_fetch(-1) == 1
    assert lb.jb_set_m2l_fetch(1) == 0
