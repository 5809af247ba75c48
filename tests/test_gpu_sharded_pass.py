"""The multi-GPU form's compute on one GPU: passes over contiguous leaf ranges
(Pass(leaf_range=...), M2L restricted to the target nodes that meet the range,
L2P + P2P for its leaves, the gear schedule cut to the same targets) give,
row for row, the whole pass's accelerations for their particles -- bit for bit,
since each range runs the same work units -- and together tile the output.
(The collectives around it -- broadcast of the sources, all_gather of the
slices -- are tested with gloo ranks in tests/test_sharding.py.)"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import _lib, engine, gears, sharding, tree, workloads  # noqa: E402


@pytest.mark.parametrize("form", ["plain", "chosen", "split_bf16"])
def test_leaf_range_passes_tile_the_whole_pass(form):
    pos, mass = workloads.clustered(262_144, seed=6)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=0.55, device="cuda")
    dt = engine.DeviceTopology(topo, "cuda")
    kw = {"plain": dict(m2l_mode=_lib.JB_M2L_FP32, p2p_mode=_lib.JB_P2P_FP32),
          "chosen": dict(m2l_mode=_lib.JB_M2L_FP32, p2p_mode=_lib.JB_P2P_KAHAN),
          "split_bf16": dict(m2l_mode=_lib.JB_M2L_SPLIT_BF16, p2p_mode=_lib.JB_P2P_KAHAN)}[form]
    d_pos, d_mass = torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda()
    full = engine.Pass(dt, 8, G=1.0, eps2=0.0, **kw)
    full.load_particles(d_pos, d_mass)
    g = None
    if form == "chosen":
        g = gears.apply_gears(full, gears.GearModel.load())
    want = full.run().clone()
    out = torch.full_like(want, float("nan"))
    for lo, hi in sharding.leaf_ranges(topo.num_leaves, 3):
        ps = engine.Pass(dt, 8, G=1.0, eps2=0.0, leaf_range=(lo, hi), **kw)
        if g is not None:
            ps.set_gears(g, gears.GearModel.load().orders)
            assert ps.gear_sched.units.shape[0] < full.gear_sched.units.shape[0]
        ps.load_particles(d_pos, d_mass)
        acc = ps.run()
        b, e = sharding.particle_range(topo, lo, hi)
        out[b:e] = acc[b:e]
    assert torch.equal(out, want)
