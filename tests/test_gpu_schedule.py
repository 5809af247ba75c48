"""Work-unit schedules built on the GPU (csrc/schedule_gpu.cu) against the
host builders of schedule.py: every array equal, on several topologies, unit
sizes, leaf ranges and random gear assignments, and the pass through either
schedule gives bit-identical accelerations."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import _lib, engine, schedule, tree, workloads  # noqa: E402

CASES = [("uniform", 20_000, 16, 0.6), ("clustered", 200_000, 32, 0.55), ("plummer", 100_000, 8, 0.5),
         ("clustered", 3_000, 32, 0.3)]


@pytest.fixture(scope="module", params=CASES, ids=lambda c: f"{c[0]}-{c[1]}-leaf{c[2]}-th{c[3]}")
def topo(request):
    kind, n, leaf, theta = request.param
    pos, mass = workloads.GENERATORS[kind](n, 21)
    t = tree.build_topology(pos, mass, leaf_size=leaf, theta=theta, device="cuda")
    return engine.DeviceTopology(t, "cuda"), pos, mass


def same(dev, host, what):
    d = dev.cpu().numpy() if torch.is_tensor(dev) else np.asarray(dev)
    h = np.asarray(host)
    assert d.shape == h.shape, (what, d.shape, h.shape)
    assert np.array_equal(d, h), what


@pytest.mark.parametrize("part", [None, (0.25, 0.6)])
def test_leaf_ancestor_schedule(topo, part):
    """The direct L2L's (leaf -> ancestors with far pairs) units: the device
    builder equals the host one entry for entry, whole and on a leaf range."""
    dt = topo[0]
    L = dt.topo.num_leaves
    rng = (0, L) if part is None else (int(part[0] * L), int(part[1] * L))
    hu, ha = engine.l2l_leaf_schedule(dt.topo, rng)
    du, da = engine.l2l_leaf_schedule_device(dt, rng)
    same(du.reshape(-1, 4), hu, "units")
    if hu.shape[0]:
        same(da, ha, "ancestors")


@pytest.mark.parametrize("max_pairs", [64, 16, 1])
def test_m2l_schedule(topo, max_pairs):
    dt = topo[0]
    want = schedule.m2l_schedule(dt.topo, max_pairs=max_pairs)
    got = schedule.m2l_schedule_device(dt, max_pairs=max_pairs)
    same(got.units, want.units, "units")
    same(got.split, want.split, "split")
    assert got.num_slots == want.num_slots
    # a target subset, in a given order (the leaf-range form)
    tg = dt.topo.m2l_targets[::3].copy()
    np.random.default_rng(0).shuffle(tg)
    tg = np.concatenate([tg, np.arange(3, dtype=np.int32)])  # nodes without far pairs are dropped
    want = schedule.m2l_schedule(dt.topo, max_pairs=max_pairs, targets=tg)
    got = schedule.m2l_schedule_device(dt, max_pairs=max_pairs, targets=tg)
    same(got.units, want.units, "units (targets)")
    same(got.split, want.split, "split (targets)")
    assert got.num_slots == want.num_slots


@pytest.mark.parametrize("max_sources", [4096, 256, 64, 1])
def test_leaf_schedule(topo, max_sources):
    dt = topo[0]
    L = dt.topo.num_leaves
    for rng in (None, (0, L // 3), (L // 3, L), (L // 2, L // 2 + 1), (5, 5)):
        want = schedule.leaf_schedule(dt.topo, max_sources=max_sources, leaf_range=rng)
        got = schedule.leaf_schedule_device(dt, max_sources=max_sources, leaf_range=rng)
        for f in ("units", "aux", "runs", "split"):
            same(getattr(got, f), getattr(want, f), f"{f} {rng}")
        assert got.num_slots == want.num_slots


@pytest.mark.parametrize("ng", [4, 1, 3])
def test_gear_schedule(topo, ng):
    dt = topo[0]
    rng = np.random.default_rng(ng)
    gears = rng.integers(0, ng, size=dt.topo.num_far_pairs)
    # runs of equal gears inside lists, as the selector produces
    gears[: gears.size // 2] = np.sort(gears[: gears.size // 2])
    orders = tuple(range(2, 2 + 2 * ng, 2))
    want = schedule.gear_m2l_schedule(dt.topo, gears, orders)
    got = schedule.gear_m2l_schedule_device(dt, gears, orders)
    for f in ("units", "split", "far_src", "gear_offsets", "pairs_per_gear"):
        same(getattr(got, f), getattr(want, f), f)
    assert got.num_slots == want.num_slots
    bad = gears.copy()
    bad[7] = ng
    with pytest.raises(_lib.JBError):
        schedule.gear_m2l_schedule_device(dt, bad, orders)


@pytest.mark.parametrize("orders,max_pairs", [((2, 4, 6, 8), 128), ((2, 4, 6, 8), 5), ((6, 8), 64), ((8,), 128)])
def test_mixed_gear_schedule(topo, orders, max_pairs):
    dt = topo[0]
    ng = len(orders)
    rng = np.random.default_rng(ng + max_pairs)
    gears = rng.integers(0, ng, size=dt.topo.num_far_pairs)
    gears[: gears.size // 2] = np.sort(gears[: gears.size // 2])
    want = schedule.gear_m2l_mixed_schedule(dt.topo, gears, orders, 8, max_pairs=max_pairs)
    got = schedule.gear_m2l_mixed_schedule_device(dt, gears, orders, 8, max_pairs=max_pairs)
    for f in ("units", "bounds", "split", "far_src", "pairs_per_gear"):
        same(getattr(got, f), getattr(want, f), f)
    assert got.num_slots == want.num_slots
    bad = gears.copy()
    bad[5] = ng
    with pytest.raises(_lib.JBError):
        schedule.gear_m2l_mixed_schedule_device(dt, bad, orders, 8)
    with pytest.raises(ValueError):
        schedule.gear_m2l_mixed_schedule_device(dt, gears, tuple(o - 1 for o in orders), 8)


def test_pass_is_identical_through_either_schedule(topo):
    dt, pos, mass = topo
    ps = engine.Pass(dt, 6, G=1.0, eps2=1e-6, p2p_mode=_lib.JB_P2P_KAHAN)  # device schedules
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    a = ps.run().clone()
    host = engine.Pass(dt, 6, G=1.0, eps2=1e-6, p2p_mode=_lib.JB_P2P_KAHAN)
    t = dt.topo
    host.m2l_sched = schedule.m2l_schedule(t, max_pairs=ps.m2l_unit_pairs)
    host.leaf_sched = schedule.leaf_schedule(t, max_sources=ps.leaf_unit_sources)
    up = lambda x: torch.from_numpy(x if x.size else np.zeros(4, np.int32)).cuda()
    host.d_m2l_units, host.d_m2l_split = up(host.m2l_sched.units), up(host.m2l_sched.split)
    host.d_leaf_units, host.d_leaf_aux = up(host.leaf_sched.units), up(host.leaf_sched.aux)
    host.d_leaf_runs, host.d_leaf_split = up(host.leaf_sched.runs), up(host.leaf_sched.split)
    host.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    b = host.run()
    assert torch.equal(a, b)
