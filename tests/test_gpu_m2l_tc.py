"""Split-BF16 M2L on the tensor cores (jb_m2l_split, tcgen05) against the
float64 oracle: accumulated locals per target and the whole pass."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oracle as O  # noqa: E402
from jaccpot_b200 import _lib, engine, tree, workloads  # noqa: E402

# BF16 hi/lo 3-product: ~16 significant bits per product, so coefficient rows
# carry ~1e-4 relative error; forces (which the near field dominates) ~1e-6.
SPLIT_ROW_P99 = 1e-3
ACC_P99 = 1e-5


def _row_rel(a, b):
    return np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-300)


@pytest.mark.parametrize("p,layout,products", [(4, "units", 1), (6, "units", 1), (8, "units", 1),
                                               (4, "tiles", 1), (8, "tiles", 1), (4, "tiles", 3), (8, "tiles", 3)])
def test_split_m2l_matches_oracle(p, layout, products):
    pos, mass = workloads.clustered(32768, seed=5)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=0.6)
    dt = engine.DeviceTopology(topo, "cuda")
    ps = engine.Pass(dt, p, G=1.0, eps2=0.0, m2l_mode=_lib.JB_M2L_SPLIT_BF16)
    ps.tc_layout = layout
    ps.tc_products = products
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    ps.upward()
    ps.m2l()
    torch.cuda.synchronize()
    assert ps.tc_status() == 0
    C = (p + 1) ** 2
    got = ps.ws.locals.double().cpu().numpy()[:, :C]
    mult = ps.ws.mult.double().cpu().numpy()[:, :C]
    cen = ps.ws.centers.double().cpu().numpy()[:, :3]
    ref = O.Pass(topo, np.float64).m2l_accumulate(p, mult, cen)
    has = np.diff(topo.far_offsets) > 0
    assert np.all(got[~has] == 0)
    err = _row_rel(got[has], ref[has])
    assert np.isfinite(got).all()
    assert np.percentile(err, 99) <= SPLIT_ROW_P99, np.percentile(err, [50, 99, 100])
    assert err.max() <= 10 * SPLIT_ROW_P99


def test_split_pass_accuracy():
    pos, mass = workloads.clustered(65536, seed=9)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=0.6)
    dt = engine.DeviceTopology(topo, "cuda")
    ps = engine.Pass(dt, 8, G=1.0, eps2=0.0, m2l_mode=_lib.JB_M2L_SPLIT_BF16, p2p_mode=_lib.JB_P2P_KAHAN)
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    got = ps.run().double().cpu().numpy()[:, :3]
    assert ps.tc_status() == 0
    p_s = pos[topo.permutation].astype(np.float64)
    m_s = mass[topo.permutation].astype(np.float64)
    ref = O.Pass(topo, np.float64).run(8, p_s, m_s)["acc"]
    err = workloads.relative_errors(got, ref)
    assert np.percentile(err, 99) <= ACC_P99, np.percentile(err, [50, 99, 100])
    rng = np.random.default_rng(4)
    tg = rng.choice(65536, 2048, replace=False)
    direct, _ = O.direct_sum(p_s, m_s, targets=tg)
    e_gpu = workloads.relative_errors(got[tg], direct)
    e_orc = workloads.relative_errors(ref[tg], direct)
    assert np.percentile(e_gpu, 99) <= np.percentile(e_orc, 99) * 1.05 + 2e-6


def test_split_pass_is_deterministic():
    pos, mass = workloads.uniform_cube(16384, seed=2)
    topo = tree.build_topology(pos, mass, leaf_size=16, theta=0.6)
    dt = engine.DeviceTopology(topo, "cuda")
    ps = engine.Pass(dt, 6, G=1.0, eps2=0.0, m2l_mode=_lib.JB_M2L_SPLIT_BF16)
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    a = ps.run().clone()
    b = ps.run().clone()
    torch.cuda.synchronize()
    assert ps.tc_status() == 0
    assert torch.equal(a, b)
