"""The near field on one stream while the upward sweep, M2L and L2L run on a
high-priority one (Pass.run(overlap=True), JB_P2P_NEAR_FIRST then
JB_P2P_FAR_AFTER): the leaf's near and far parts are each rounded on their
own and added with one rounded add, so the two-stream order gives the
one-stream bits -- eagerly, as a torch graph and as a graph that keeps the
streams' priorities (PassGraph) -- with split leaves, the compensated sums
and the potential."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import FastMultipoleMethod, _lib, engine, tree, workloads  # noqa: E402


def _step(ps, pos, mass, overlap, potential):
    acc = torch.empty_like(pos)
    pot = torch.empty_like(mass) if potential else None
    ps.load_particles(pos, mass)
    ps.run(potential=potential, overlap=overlap)
    ps.unsort(acc, pot)
    torch.cuda.synchronize()
    return acc, pot


@pytest.fixture(scope="module")
def clustered():
    pos, mass = workloads.clustered(80_000, 5)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=0.6, device="cuda")
    return pos, mass, engine.DeviceTopology(topo, "cuda")


@pytest.mark.parametrize("p,mode,potential", [(8, _lib.JB_P2P_KAHAN, True), (8, _lib.JB_P2P_KAHAN, False),
                                              (4, _lib.JB_P2P_FP32, True)])
def test_two_streams_give_the_one_stream_bits(clustered, p, mode, potential):
    pos, mass, dt = clustered
    # short leaf units: many leaves split over several units (partials summed last)
    ps = engine.Pass(dt, p, G=1.0, eps2=1e-6, p2p_mode=mode, leaf_unit_sources=256)
    assert ps.leaf_sched.split.shape[0] > 0
    d_pos, d_mass = torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda()
    a1, u1 = _step(ps, d_pos, d_mass, False, potential)
    a2, u2 = _step(ps, d_pos, d_mass, True, potential)
    assert torch.equal(a1, a2)
    if potential:
        assert torch.equal(u1, u2)
    # the halves alone: near_first holds the near field of unsplit leaves
    ps.load_particles(d_pos, d_mass)
    ps.upward()
    ps.downward()
    near = ps.evaluate(part="near").clone()
    ps.evaluate(part="near_first")
    torch.cuda.synchronize()
    unsplit = torch.ones(near.shape[0], dtype=torch.bool, device=near.device)
    sp = ps.leaf_sched.split
    sp = sp if torch.is_tensor(sp) else torch.from_numpy(np.ascontiguousarray(sp))
    nr = dt.topo.node_ranges  # (num_nodes, 2) first / last sorted particle
    for lo, hi in nr[dt.topo.num_internal + sp[:, 0].cpu().numpy().astype(np.int64)].tolist():
        unsplit[lo:hi + 1] = False
    assert torch.equal(ps.ws.acc4[unsplit, :3], near[unsplit, :3])
    assert torch.count_nonzero(ps.ws.acc4[~unsplit]) == 0


def test_far_after_half_gives_the_one_call_bits(clustered):
    pos, mass, dt = clustered
    ps = engine.Pass(dt, 8, G=1.0, eps2=1e-6, p2p_mode=_lib.JB_P2P_KAHAN, leaf_unit_sources=256)
    d_pos, d_mass = torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda()
    ps.load_particles(d_pos, d_mass)
    ps.upward()
    ps.downward()
    one = ps.evaluate(potential=True).clone()
    ps.evaluate(potential=True, part="near_first")
    ps.evaluate(potential=True, part="far_after")
    torch.cuda.synchronize()
    assert torch.equal(ps.ws.acc4, one)


def test_two_streams_on_a_leaf_range(clustered):
    pos, mass, dt = clustered
    nl = dt.topo.num_leaves
    ps = engine.Pass(dt, 6, G=1.0, eps2=1e-6, p2p_mode=_lib.JB_P2P_KAHAN, leaf_range=(nl // 3, 2 * nl // 3),
                     leaf_unit_sources=256)
    d_pos, d_mass = torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda()
    t = dt.topo
    lo = int(t.node_ranges[t.num_internal + nl // 3, 0])
    hi = int(t.node_ranges[t.num_internal + 2 * nl // 3 - 1, 1]) + 1
    ps.load_particles(d_pos, d_mass)
    a1 = ps.run(overlap=False)[lo:hi].clone()
    ps.ws.acc4.fill_(3.0)
    ps.load_particles(d_pos, d_mass)
    a2 = ps.run(overlap=True)
    torch.cuda.synchronize()
    assert torch.equal(a2[lo:hi], a1)
    assert bool((a2[:lo] == 3.0).all()) and bool((a2[hi:] == 3.0).all())  # outside the range: untouched


@pytest.mark.parametrize("node_priority", [True, False])
def test_overlapped_graph_replays_the_eager_bits(clustered, node_priority):
    pos, mass, dt = clustered
    ps = engine.Pass(dt, 8, G=1.0, eps2=1e-6, p2p_mode=_lib.JB_P2P_KAHAN, leaf_unit_sources=512)
    d_pos, d_mass = torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda()
    ref, _ = _step(ps, d_pos, d_mass, False, False)
    acc = torch.empty_like(d_pos)
    g = ps.capture(d_pos, d_mass, acc, overlap=True, node_priority=node_priority)
    assert isinstance(g, engine.PassGraph) == node_priority
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(acc, ref)
    moved = d_pos + 1e-4 * torch.randn_like(d_pos)
    d_pos.copy_(moved)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(acc, _step(ps, moved.clone(), d_mass, False, False)[0])
    g.reset()


def test_overlap_on_the_error_controlled_pass():
    pos, mass = workloads.clustered(60_000, 6)
    kw = dict(theta=0.6, softening=0.0, adaptive_order=True, p_gears=(8,), adaptive_error_model="dehnen_paper",
              adaptive_eps=5e-5, mac_force_scale_mode="paper")
    fmm = FastMultipoleMethod(**kw, advanced={"nearfield_compensated": True})
    st = fmm.prepare_state(pos, mass, leaf_size=32, max_order=8)
    assert st.pass_.overlap  # the default
    st.pass_.overlap = False
    a1 = fmm.differentiable_accelerations(st, pos, mass)
    st.pass_.overlap = True
    a2 = fmm.differentiable_accelerations(st, pos, mass)
    assert np.array_equal(np.asarray(a1), np.asarray(a2))


def test_two_halves_refuse_to_combine():
    lb = _lib.lib()
    both = _lib.JB_P2P_NEAR_FIRST | _lib.JB_P2P_FAR_AFTER
    rc = lb.jb_leaf_eval(8, both, None, 0, 0, None, None, None, None, None, None, 1.0, 0.0, None, None, 0, None, None)
    assert rc == 1
    rc = lb.jb_leaf_eval(8, _lib.JB_P2P_NEAR_ONLY | _lib.JB_P2P_FAR_AFTER, None, 0, 0, None, None, None, None, None,
                         None, 1.0, 0.0, None, None, 0, None, None)
    assert rc == 1


def test_stages_order_their_own_fills_on_the_given_stream(clustered):
    """Every stage enqueues all its work on the stream it is given: the
    locals' zeroing before the M2L included.  The current stream is held
    busy (a bounded spin) while the M2L runs on another stream; a zeroing
    left on the current stream would land after the M2L and wipe it."""
    pos, mass, dt = clustered
    ps = engine.Pass(dt, 6, G=1.0, eps2=1e-6)
    d_pos, d_mass = torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda()
    ps.load_particles(d_pos, d_mass)
    ps.upward()
    ps.m2l()
    torch.cuda.synchronize()
    ref = ps.ws.locals.clone()
    ps.ws.locals.fill_(7.0)
    torch.cuda.synchronize()
    other = torch.cuda.Stream()
    torch.cuda._sleep(20_000_000)  # ~10 ms on the current stream
    ps.m2l(other)
    other.synchronize()
    torch.cuda.synchronize()
    assert torch.equal(ps.ws.locals, ref)
