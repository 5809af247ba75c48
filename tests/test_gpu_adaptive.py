"""Error-controlled walk (jb_dtree_adaptive_walk) and the gear pass on it.

* the GPU walk equals its restatement (oracle/adaptive_walk.py) bit for bit
  -- far CSR, gears, near CSR -- on the same centres, radii, powers and force
  scales;
* the Dehnen power kernel equals the restatement's formula;
* the pass over the adaptive lists, every far pair at its gear, matches the
  FP64 oracle evaluating the same lists at the same gears (p99 <= 1e-5);
* its error against an FP64 direct sum follows the accuracy target.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oracle  # noqa: E402
from jaccpot_b200 import _lib, adaptive, engine, tree, workloads  # noqa: E402
from oracle import adaptive_walk as aw  # noqa: E402

ORDERS = (2, 4, 6, 8)


def _prepass(pos, mass, leaf=16, theta=0.6, p=8):
    dtree = tree.DeviceTree(pos, mass, leaf_size=leaf, theta=theta, device="cuda")
    topo0 = dtree.topology()
    dt0 = engine.DeviceTopology(topo0, "cuda")
    pre = engine.Pass(dt0, p)
    pre.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    pre.run()
    return dtree, topo0, pre


@pytest.mark.parametrize("kind,n,leaf,eps,tmax,orders", [
    ("clustered", 40_000, 16, 1e-5, 1.0, ORDERS),
    ("plummer", 20_000, 32, 3e-4, 0.8, (4, 8)),
    ("uniform", 8_000, 8, 1e-7, 1.0, (6,)),
])
def test_walk_matches_the_oracle_bit_for_bit(kind, n, leaf, eps, tmax, orders):
    pos, mass = workloads.GENERATORS[kind](n, 11)
    dtree, topo0, pre = _prepass(pos, mass, leaf=leaf, p=max(orders))
    power = adaptive.node_dehnen_power(pre)
    fs = adaptive.node_force_scale(pre)
    pw_h, fs_h = power.cpu().numpy(), fs.cpu().numpy()
    dtree.adaptive_walk(power, fs, G=1.0, eps=eps, theta_max=tmax, gear_orders=orders)
    topo = dtree.topology()
    dtree.free()
    want = aw.adaptive_walk(topo0.left_child, topo0.right_child, topo0.centers_f64, topo0.radii_f64,
                            topo0.num_internal, pw_h, fs_h, G=1.0, eps=eps, theta_max=tmax, orders=orders)
    got = (topo.far_offsets, topo.far_sources, topo.far_gears, topo.near_offsets, topo.near_leaves)
    for name, g, w in zip(("far_off", "far_src", "far_gear", "near_off", "near_src"), got, want):
        assert np.array_equal(np.asarray(g), np.asarray(w)), name
    # the tree itself is untouched
    assert np.array_equal(topo.node_ranges, topo0.node_ranges)
    assert np.array_equal(topo.centers_f64, topo0.centers_f64)
    assert topo.gear_orders == tuple(orders)


def test_power_kernel_matches_the_formula():
    pos, mass = workloads.clustered(20_000, 2)
    dtree, topo0, pre = _prepass(pos, mass, p=8)
    dtree.free()
    power = adaptive.node_dehnen_power(pre).cpu().numpy()
    mult = pre.ws.mult[:, :81].cpu().numpy()
    np.testing.assert_allclose(power, aw.dehnen_power(mult, 8), rtol=1e-12, atol=0)


def _oracle_gear_pass(topo, pos_s, mass_s, orders, p_top):
    """FP64 oracle over the adaptive lists, far pair e at order orders[gear[e]]."""
    P = oracle.Pass(topo, np.float64)
    centers = P.com(pos_s, mass_s)
    mult = P.upward(p_top, pos_s, mass_s, centers)
    loc = np.zeros_like(mult)
    tgt = topo.far_pair_targets()
    for gi, p in enumerate(orders):
        m = topo.far_gears == gi
        if not m.any():
            continue
        off = np.zeros(topo.num_nodes + 1, np.int64)
        np.add.at(off, tgt[m].astype(np.int64) + 1, 1)
        sub = SimpleNamespace(**{k: getattr(topo, k) for k in (
            "num_nodes", "num_internal", "num_levels", "node_ranges", "left_child", "right_child",
            "level_offsets", "near_offsets", "near_leaves", "leaf_of_particle")})
        sub.far_offsets, sub.far_sources = np.cumsum(off), topo.far_sources[m]
        C = (p + 1) ** 2
        part = oracle.Pass(sub, np.float64).m2l_accumulate(p, np.ascontiguousarray(mult[:, :C]), centers)
        loc[:, :C] += part
    loc = P.l2l_cascade(p_top, centers, loc)
    acc, _ = P.evaluate(p_top, pos_s, mass_s, centers, loc, 1.0, 0.0)
    return acc


@pytest.mark.parametrize("orders", [ORDERS, (4, 6, 8, 10)])
def test_gear_pass_matches_the_oracle_on_the_same_lists(orders):
    pos, mass = workloads.clustered(32_768, 5)
    prep = adaptive.prepare(pos, mass, leaf_size=32, orders=orders, eps=3e-5, theta_max=1.0, device="cuda")
    ps, topo = prep.pass_, prep.topology
    assert topo.far_gears is not None and topo.num_far_pairs > 0
    frac = np.bincount(topo.far_gears, minlength=len(orders)) / topo.num_far_pairs
    assert (frac > 0).sum() >= 2  # several gears in use
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    got = ps.run()[:, :3].double().cpu().numpy()
    perm = topo.permutation
    want = _oracle_gear_pass(topo, pos[perm].astype(np.float64), mass[perm].astype(np.float64), orders,
                             max(orders))
    err = workloads.relative_errors(got, want)
    assert np.percentile(err, 99) <= 1e-5, np.percentile(err, [50, 99, 100])


def test_error_follows_the_accuracy_target():
    n = 131_072
    pos, mass = workloads.clustered(n, 7)
    rng = np.random.default_rng(3)
    tg = rng.choice(n, 4096, replace=False)
    ref, _ = oracle.direct_sum(pos.astype(np.float64), mass.astype(np.float64), targets=tg)
    p99 = {}
    for eps in (1e-4, 1e-6):
        prep = adaptive.prepare(pos, mass, leaf_size=32, orders=ORDERS, eps=eps, device="cuda")
        ps = prep.pass_
        ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
        ps.run()
        acc = torch.empty((n, 3), device="cuda")
        ps.unsort(acc, None)
        e = workloads.relative_errors(acc.double().cpu().numpy()[tg], ref)
        p99[eps] = float(np.percentile(e, 99))
    assert p99[1e-6] < p99[1e-4]
    assert p99[1e-6] <= 1e-5, p99
    assert p99[1e-4] <= 1e-3, p99
