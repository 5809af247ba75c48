"""The mutual (momentum-conserving) lane on the GPU: its accelerations are the
facade's (massless particles reported as zero), its forces sum to zero to FP32
round-off -- near part, far part and total -- and the learned gears keep that
only when symmetrised; the device reverse index equals the host one."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import engine, gears, mutual, tree, workloads  # noqa: E402
from jaccpot_b200.solver import FastMultipoleMethod  # noqa: E402

ROUND_OFF = 1e-7  # FP32 sums over ~1e5..1e6 particles; the force error is ~1e-4


@pytest.mark.parametrize("kind", ["plummer", "clustered"])
def test_mutual_accelerations_conserve_momentum(kind):
    pos, mass = workloads.GENERATORS[kind](262_144, 4)
    mass[::97] = 0.0
    mt, st0 = mutual.build_mutual_topology(pos, mass, theta=0.55, order=6, leaf_size=32)
    st = mutual.build_mutual_state(mt, softening=1e-3)
    res = mutual.mutual_accelerations(st, pos, mass, return_parts=True)
    acc, near, far = res
    assert np.isfinite(acc).all()
    assert (acc[mass == 0] == 0).all()
    # the facade's accelerations at the same settings (positive masses)
    fmm = FastMultipoleMethod(theta=0.55, G=1.0, softening=1e-3, nearfield_compensated=True)
    ref = fmm.evaluate_prepared_state(fmm.prepare_state(pos, mass, leaf_size=32, max_order=6))
    pm = mass > 0
    scale = np.sqrt((ref[pm] ** 2).sum(1).mean())
    assert np.abs(acc[pm] - ref[pm]).max() <= 1e-5 * scale
    for f in (near, far, near + far):
        assert mutual.momentum_residual(f) < ROUND_OFF
    # parts add up to the total
    F = mass[:, None] * acc
    assert np.abs(near + far - F).max() <= 1e-5 * np.abs(F).max()


def test_symmetric_gears_keep_momentum():
    pos, mass = workloads.clustered(262_144, 9)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=0.55, device="cuda")
    dt = engine.DeviceTopology(topo, "cuda")
    rev = dt.far_reverse_index().cpu().numpy()
    assert np.array_equal(rev, topo.far_reverse_index())
    d_pos, d_mass = torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda()
    m = d_mass[dt.perm].double()
    model = gears.GearModel.load()
    out = {}
    for sym in (False, True):
        ps = engine.Pass(dt, 8, G=1.0, eps2=0.0)
        ps.load_particles(d_pos, d_mass)
        g = gears.apply_gears(ps, model, symmetric=sym)
        if sym:
            assert np.array_equal(g, g[rev])
        out[sym] = mutual.momentum_residual(m[:, None] * ps.run()[:, :3].double())
    assert out[True] < ROUND_OFF
    assert out[False] > out[True]  # per-direction orders break the pairwise balance


def test_block_step_weights():
    """The rung-weighted form: unit weights give the full acceleration, the
    per-level accelerations add up to it, and any weights keep momentum."""
    n = 131_072
    pos, mass = workloads.plummer(n, 12)
    rng = np.random.default_rng(3)
    rung = rng.integers(0, 4, size=n).astype(np.int32)
    mt, _ = mutual.build_mutual_topology(pos, mass, theta=0.55, order=6, leaf_size=32)
    st = mutual.build_mutual_state(mt, softening=1e-3)
    full = mutual.mutual_accelerations(st, pos, mass)
    scale = np.sqrt((full ** 2).sum(1).mean())
    ones = mutual.mutual_accelerations(st, pos, mass, rung=rung, level_weights=np.ones(4, np.float32))
    assert np.abs(ones - full).max() <= 1e-6 * scale
    levels = [mutual.mutual_level_accelerations(st, pos, mass, rung=rung, level=k, k_max=3) for k in range(4)]
    assert np.abs(sum(levels) - full).max() <= 1e-5 * scale
    assert all(np.abs(a).max() > 0 for a in levels)
    w = mutual.boundary_level_weights(0, 3, 0.01).astype(np.float32)
    res = mutual.mutual_accelerations(st, pos, mass, rung=rung, level_weights=w, return_parts=True)
    for f in (res.near_forces, res.far_forces, res.near_forces + res.far_forces):
        assert mutual.momentum_residual(f) < ROUND_OFF
    with pytest.raises(ValueError):
        mutual.mutual_accelerations(st, pos, mass, rung=rung)
