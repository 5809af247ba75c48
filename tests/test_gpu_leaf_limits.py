"""Leaf-occupancy and slot preconditions of the leaf kernels, through the C
ABI: leaves of more than JB_MAX_LEAF_OCCUPANCY (64) particles get a status,
not a write -- the GPU leaf schedule refuses them, jb_validate_leaves counts
them, and a hand-made unit that names one writes nothing and sets the leaf
error word; a partial-row slot beyond jb_leaf_eval_noalloc's num_slots is
neither written nor read and sets JB_LEAF_ERR_SLOT."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import _lib, engine, tree, workloads  # noqa: E402


def _errors(clear=True):
    f = ctypes.c_int(-1)
    _lib.check(_lib.lib().jb_leaf_eval_errors(ctypes.byref(f), 1 if clear else 0,
                                              torch.cuda.current_stream().cuda_stream), "jb_leaf_eval_errors")
    return f.value


def _topology_with_big_leaves():
    pos, mass = workloads.uniform_cube(20000, seed=5)
    topo = tree.build_topology(pos, mass, leaf_size=96, theta=0.6)
    occ = topo.node_ranges[topo.num_internal:, 1] - topo.node_ranges[topo.num_internal:, 0] + 1
    assert occ.max() > 64
    return pos, mass, topo, occ


def test_over_full_leaves_get_a_status_not_a_write():
    pos, mass, topo, occ = _topology_with_big_leaves()
    lb = _lib.lib()
    st = torch.cuda.current_stream().cuda_stream
    ranges = torch.from_numpy(topo.node_ranges.reshape(-1).astype(np.int32)).cuda()
    bad = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.check(lb.jb_validate_leaves(topo.num_nodes, topo.num_internal, ranges.data_ptr(), 64, bad.data_ptr(), st),
               "jb_validate_leaves")
    assert int(bad.item()) == int((occ > 64).sum())
    # the engine refuses the topology up front
    with pytest.raises(ValueError):
        engine.Pass(engine.DeviceTopology(topo, "cuda"), 4)
    with pytest.raises(_lib.JBError):
        engine.DeviceTopology(topo, "cuda").validate()
    # the GPU leaf schedule builder refuses it
    near_off = torch.from_numpy(topo.near_offsets).cuda()
    near_src = torch.from_numpy(topo.near_leaves if topo.num_near_pairs else np.zeros(1, np.int32)).cuda()
    h = ctypes.c_void_p()
    rc = lb.jb_leaf_schedule_device(topo.num_internal, topo.num_leaves, ranges.data_ptr(), near_off.data_ptr(),
                                    near_src.data_ptr(), 0, topo.num_leaves, 4096, st, ctypes.byref(h))
    assert rc == 1 and not h.value
    # a hand-made unit naming the over-full leaf (self block only): no write, a flag
    big = int(np.argmax(occ))
    r0, r1 = topo.node_ranges[topo.num_internal + big]
    n = topo.num_particles
    pos4 = torch.zeros((n, 4), device="cuda")
    pos4[:, :3] = torch.from_numpy(pos[topo.permutation]).cuda()
    pos4[:, 3] = torch.from_numpy(mass[topo.permutation]).cuda()
    cs = _lib.coeff_stride(4)
    centers = torch.zeros((topo.num_nodes, 4), device="cuda")
    locs = torch.zeros((topo.num_nodes, cs), device="cuda")
    units = torch.tensor([[big, 0, 0, 0]], dtype=torch.int32, device="cuda")
    aux = torch.tensor([[-1, 1]], dtype=torch.int32, device="cuda")
    runs = torch.zeros((1, 2), dtype=torch.int32, device="cuda")
    out = torch.full((n, 4), 7.0, device="cuda")
    partials = torch.zeros((64, 4), device="cuda")
    _errors()
    _lib.check(lb.jb_leaf_eval(4, 0, pos4.data_ptr(), topo.num_internal, 1, units.data_ptr(), aux.data_ptr(),
                               runs.data_ptr(), ranges.data_ptr(), centers.data_ptr(), locs.data_ptr(), 1.0, 0.0,
                               out.data_ptr(), partials.data_ptr(), 0, None, st), "jb_leaf_eval")
    assert _errors() & _lib.JB_LEAF_ERR_OCCUPANCY
    assert bool((out == 7.0).all())
    assert _errors() == 0  # cleared


def test_noalloc_slot_beyond_num_slots_is_skipped_and_flagged():
    pos, mass = workloads.clustered(32768, seed=3)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=0.5)
    dt = engine.DeviceTopology(topo, "cuda")
    ps = engine.Pass(dt, 4, G=1.0, eps2=1e-6, leaf_unit_sources=256)
    sc = ps.leaf_sched
    assert sc.num_slots > 1
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    ps.upward()
    ps.downward()
    lb = _lib.lib()
    st = torch.cuda.current_stream().cuda_stream
    _errors()
    out = torch.zeros_like(ps.ws.acc4)
    # one slot too few: the last slot is not written, its reduce entry not read
    _lib.check(lb.jb_leaf_eval_noalloc(ps.p, 0, ps.ws.pos4.data_ptr(), topo.num_internal,
                                       int(sc.units.shape[0]), ps.d_leaf_units.data_ptr(), ps.d_leaf_aux.data_ptr(),
                                       ps.d_leaf_runs.data_ptr(), dt.node_ranges.data_ptr(),
                                       ps.ws.centers.data_ptr(), ps.ws.locals.data_ptr(), ps.G, ps.eps2,
                                       out.data_ptr(), int(sc.num_slots) - 1, int(sc.split.shape[0]),
                                       ps.d_leaf_split.data_ptr(), st), "jb_leaf_eval_noalloc")
    assert _errors() & _lib.JB_LEAF_ERR_SLOT
    # with the right count nothing is flagged
    _lib.check(lb.jb_leaf_eval_noalloc(ps.p, 0, ps.ws.pos4.data_ptr(), topo.num_internal,
                                       int(sc.units.shape[0]), ps.d_leaf_units.data_ptr(), ps.d_leaf_aux.data_ptr(),
                                       ps.d_leaf_runs.data_ptr(), dt.node_ranges.data_ptr(),
                                       ps.ws.centers.data_ptr(), ps.ws.locals.data_ptr(), ps.G, ps.eps2,
                                       out.data_ptr(), int(sc.num_slots), int(sc.split.shape[0]),
                                       ps.d_leaf_split.data_ptr(), st), "jb_leaf_eval_noalloc")
    assert _errors() == 0
    want = ps.evaluate().clone()
    assert torch.equal(out[:, :3], want[:, :3])
