"""The learned selector's training labels against an FP64 order-12 reference.

jb_gear_errors labels a far pair with each gear's force error measured
against the order-10 FP32 M2L of the same multipole (on the near and far
side of the target's sphere, relative to the target's smallest force).  Here
the same quantity is restated in FP64 with order-12 multipoles (the oracle's
upward pass about the GPU's own centres) and an order-12 reference M2L: the
log errors agree where they matter and the labels at the model's budgets are
the same for 99.5% of pairs, so the FP32 order-10 reference does not bias
what the network learns."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oracle as O  # noqa: E402
from jaccpot_b200 import _lib, engine, gears, tree, workloads  # noqa: E402

ORDERS = (2, 4, 6, 8)


def test_labels_match_an_fp64_order12_reference():
    n, seed = 32768, 7
    pos, mass = workloads.clustered(n, seed)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=0.6)
    dt = engine.DeviceTopology(topo, "cuda")
    d_pos, d_mass = torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda()
    ps = engine.Pass(dt, 8, G=1.0, eps2=0.0)
    ps.load_particles(d_pos, d_mass)
    ps.run()
    ctx = gears.GearContext(ps)
    ctx.node_features()
    p10 = engine.Pass(dt, 10, G=1.0, eps2=0.0)
    p10.load_particles(d_pos, d_mass)
    p10.upward()
    rng = np.random.default_rng(3)
    m = min(4096, topo.num_far_pairs)
    ids_np = np.sort(rng.choice(topo.num_far_pairs, m, replace=False)).astype(np.int64)
    ids = torch.from_numpy(ids_np).cuda()
    Y = torch.empty((m, len(ORDERS)), device="cuda", dtype=torch.float32)
    _lib.check(_lib.lib().jb_gear_errors(m, ids.data_ptr(), ctx.pair_tgt.data_ptr(), dt.far_src.data_ptr(),
                                         p10.ws.mult.data_ptr(), ps.ws.centers.data_ptr(), ctx.radii.data_ptr(),
                                         ctx.scale.data_ptr(), 1.0, Y.data_ptr(),
                                         torch.cuda.current_stream().cuda_stream), "jb_gear_errors")
    torch.cuda.synchronize()
    Y = Y.cpu().numpy().astype(np.float64)
    # the FP64 order-12 restatement, about the same (FP32) centres
    centers = ps.ws.centers[:, :3].double().cpu().numpy()
    radii = ctx.radii.double().cpu().numpy()
    scale = ctx.scale.double().cpu().numpy()
    perm = topo.permutation
    opass = O.Pass(topo, np.float64)
    M12 = opass.upward(12, pos[perm].astype(np.float32).astype(np.float64),
                       mass[perm].astype(np.float32).astype(np.float64), centers)
    tgt = topo.far_pair_targets()[ids_np].astype(np.int64)
    src = topo.far_sources[ids_np].astype(np.int64)
    d = centers[tgt] - centers[src]
    dn = np.linalg.norm(d, axis=1, keepdims=True)
    h = -radii[tgt][:, None] * d / dn
    Ms = M12[src]

    def grads(p, L):
        _, g_far = O.l2p(p, L, h)
        _, g_near = O.l2p(p, L, -h)
        return g_far, g_near

    ref_far, ref_near = grads(12, O.m2l(12, Ms, d))
    Y64 = np.empty_like(Y)
    for k, p in enumerate(ORDERS):
        C = (p + 1) ** 2
        gf, gn = grads(p, O.m2l(p, Ms[:, :C], d))
        err = np.maximum(np.linalg.norm(gf - ref_far, axis=1), np.linalg.norm(gn - ref_near, axis=1))
        Y64[:, k] = np.log10(np.maximum(err / np.maximum(scale[tgt], 1e-30), 1e-30))
    # where a gear's error is above the FP32 floor the two references agree:
    # to 0.01 / 0.02 / 0.06 dex (p99) at orders 2 / 4 / 6; at order 8 the
    # order-10 reference, two orders above, understates the error by ~0.06 dex
    # (median; 0.15 at p99) -- and the labels are all but unchanged (measured
    # 99.5-99.7% identical at these budgets, the rest moving either way)
    live = Y64 > -7.0
    dY = Y - Y64
    for k, tol in enumerate((0.03, 0.05, 0.1, 0.25)):
        lv = live[:, k]
        assert np.percentile(np.abs(dY[lv, k]), 99) < tol, (ORDERS[k], np.percentile(np.abs(dY[lv, k]), 99))
    assert abs(np.median(dY[live[:, 3], 3])) < 0.1
    for budget in (1e-6, 3e-6, 1e-5, 3e-5):
        agree = np.mean(gears.labels_for(Y, budget) == gears.labels_for(Y64, budget))
        assert agree >= 0.99, (budget, agree)
