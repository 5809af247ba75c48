"""The two forms of the level sweeps (one thread per M2M / L2L translation,
or each translation's degrees split over four warps, jb_set_level_split) do
the same operations; their multipoles and locals agree to FP32 rounding, and
the default mix of the two is what the parity tests check against the oracle."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import _lib, engine, tree, workloads  # noqa: E402

DEFAULT = (1 << 30, 2048)


@pytest.mark.parametrize("p", [3, 6, 8, 10])
def test_split_and_thread_level_kernels_agree(p):
    pos, mass = workloads.clustered(131_072, seed=8)
    mass[::7] = 0.0  # massless nodes take the mean-position centre
    topo = tree.build_topology(pos, mass, leaf_size=16, theta=0.5, device="cuda")
    dt = engine.DeviceTopology(topo, "cuda")
    ps = engine.Pass(dt, p, G=1.0, eps2=1e-6)
    d_pos, d_mass = torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda()
    lb = _lib.lib()
    out = {}
    try:
        for name, thr in (("thread", 0), ("split", 1 << 30)):
            _lib.check(lb.jb_set_level_split(thr, thr), "jb_set_level_split")
            ps.load_particles(d_pos, d_mass)
            ps.upward()
            ps.m2l()
            ps.l2l(cascade=True)  # the level kernels
            torch.cuda.synchronize()
            out[name] = (ps.ws.centers.clone(), ps.ws.mult.clone(), ps.ws.locals.clone())
    finally:
        lb.jb_set_level_split(*DEFAULT)
    (c0, m0, l0), (c1, m1, l1) = out["thread"], out["split"]
    assert torch.equal(c0, c1)  # the centres are computed identically
    for a, b in ((m0, m1), (l0, l1)):
        scale = a.abs().amax(dim=1, keepdim=True).clamp_min(1e-30)
        rel = ((a - b).abs() / scale).double().cpu().numpy()
        assert np.isfinite(rel).all()
        assert np.percentile(rel, 99.9) <= 1e-5 and rel.max() <= 1e-4, (np.percentile(rel, 99.9), rel.max())
    assert lb.jb_set_level_split(-1, 0) == 1
