"""The L2L sweep starts at the shallowest internal far target (the levels
above it hold only zero locals): the pass is bit-identical to one that runs
every level, on shallow, deep (clustered) and single-leaf trees."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import engine, tree, workloads  # noqa: E402

CASES = [("uniform", 20_000, 16, 0.6, 6), ("clustered", 300_000, 32, 0.55, 8), ("plummer", 100_000, 8, 0.5, 4),
         ("uniform", 40, 64, 0.6, 8)]


@pytest.mark.parametrize("kind,n,leaf,theta,p", CASES, ids=lambda c: str(c))
def test_skipped_l2l_levels_change_nothing(kind, n, leaf, theta, p):
    pos, mass = workloads.GENERATORS[kind](n, 4)
    topo = tree.build_topology(pos, mass, leaf_size=leaf, theta=theta, device="cuda")
    dt = engine.DeviceTopology(topo, "cuda")
    lev = np.asarray(topo.node_level)
    ni = topo.num_internal
    tgt = np.nonzero(np.diff(topo.far_offsets)[:ni] > 0)[0]
    assert dt.l2l_first_level == (lev[tgt].min() if tgt.size else topo.num_levels)
    ps = engine.Pass(dt, p, G=1.0, eps2=1e-6)
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    a = ps.run(cascade=True).clone()  # the level-by-level sweep (the one that skips levels)
    la = ps.ws.locals.clone()
    first = dt.l2l_first_level
    dt.l2l_first_level = 0
    try:
        b = ps.run(cascade=True).clone()
        lb = ps.ws.locals.clone()
    finally:
        dt.l2l_first_level = first
    assert torch.equal(a, b) and torch.equal(la, lb)
