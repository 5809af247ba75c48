"""GPU tree build (jb_tree_build_device) against the host builder and the
pure-Python oracle: every array bit for bit, on the oracle's small cases and
edge cases (one particle, one leaf, duplicates, massless particles and
clumps, leaf size 1) and on larger workloads where only the host builder is
fast enough to compare against; and the pass run on the GPU-built topology."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import _lib, tree, workloads  # noqa: E402
from oracle import tree as OT  # noqa: E402

from test_tree_oracle import CASES, FIELDS, _inputs, compare, topo_fields  # noqa: E402


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}-{c[1]}-leaf{c[2]}")
def test_device_builder_matches_the_oracle(case):
    kind, n, leaf, theta = case
    pos, mass = _inputs(kind, n, 7)
    want = OT.build(pos, mass, leaf, theta)
    t = tree.build_topology(pos, mass, leaf_size=leaf, theta=theta, device="cuda")
    compare(topo_fields(t), want, str(case))
    assert t.num_levels == want["num_levels"]


BIG = [("uniform", 100_000, 16, 0.6), ("plummer", 1_048_576, 32, 0.6), ("clustered", 1_048_576, 32, 0.55),
       ("clustered", 262_144, 8, 0.4)]


@pytest.mark.parametrize("case", BIG, ids=lambda c: f"{c[0]}-{c[1]}-leaf{c[2]}-th{c[3]}")
def test_device_builder_matches_the_host_builder(case):
    kind, n, leaf, theta = case
    pos, mass = workloads.GENERATORS[kind](n, 11)
    host = tree.build_topology(pos, mass, leaf_size=leaf, theta=theta)
    dev = tree.build_topology(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda(), leaf_size=leaf,
                              theta=theta, device="cuda")
    compare(topo_fields(dev), topo_fields(host), str(case))
    for k in ("num_nodes", "num_internal", "num_leaves", "num_levels", "max_leaf_occupancy"):
        assert getattr(dev, k) == getattr(host, k), k
    assert np.array_equal(dev.m2l_targets, host.m2l_targets)


def test_device_fields_are_device_pointers_and_repeatable():
    pos, mass = workloads.clustered(50_000, seed=5)
    p = torch.from_numpy(pos).double().cuda()
    m = torch.from_numpy(mass).double().cuda()
    lb = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for _ in range(2):
        h = ctypes.c_void_p()
        _lib.check(lb.jb_tree_build_device(p.shape[0], p.data_ptr(), m.data_ptr(), 32, 0.55, stream, ctypes.byref(h)),
                   "jb_tree_build_device")
        try:
            info = _lib.TreeInfo()
            _lib.check(lb.jb_dtree_info(h, ctypes.byref(info)), "jb_dtree_info")
            ptr = lb.jb_dtree_field(h, _lib.TREE_FIELDS["far_sources"][0])
            assert ptr
            assert not lb.jb_dtree_field(h, 99)
            a = np.empty(info.num_far_pairs, np.int32)
            _lib.check(lb.jb_dtree_copy(h, _lib.TREE_FIELDS["far_sources"][0], a.ctypes.data), "copy")
            outs.append(a)
        finally:
            lb.jb_dtree_free(h)
    assert np.array_equal(outs[0], outs[1])
    # bad arguments are refused before any launch
    h = ctypes.c_void_p()
    assert lb.jb_tree_build_device(0, p.data_ptr(), m.data_ptr(), 32, 0.55, stream, ctypes.byref(h)) == 1
    assert lb.jb_tree_build_device(10, p.data_ptr(), m.data_ptr(), 32, 1.5, stream, ctypes.byref(h)) == 1
    assert lb.jb_tree_build_device(10, p.data_ptr(), m.data_ptr(), 0, 0.5, stream, ctypes.byref(h)) == 1


def test_pass_on_the_device_built_topology():
    """The facade on a CUDA device builds the tree on the GPU (the host
    builder's arrays) and its pass agrees with the FP64 oracle pass on that
    topology; both sit at the method's truncation error against a direct sum."""
    import oracle as O
    from jaccpot_b200.solver import FastMultipoleMethod

    n = 65_536
    pos, mass = workloads.plummer(n, seed=2)
    fmm = FastMultipoleMethod(theta=0.6, G=1.0, softening=0.0)
    st = fmm.prepare_state(pos, mass, leaf_size=32, max_order=6)
    topo = st.topology
    host = tree.build_topology(pos, mass, leaf_size=32, theta=0.6)
    compare(topo_fields(topo), topo_fields(host), "facade")
    got = st.pass_.evaluate()[:, :3].double().cpu().numpy()
    O.build()
    want = O.Pass(topo, np.float64).run(6, pos[topo.permutation].astype(np.float64),
                                        mass[topo.permutation].astype(np.float64), G=1.0, eps2=0.0)["acc"][:, :3]
    scale = np.sqrt((want * want).sum(1).mean())
    e = np.linalg.norm(got - want, axis=1) / scale
    assert np.percentile(e, 99) <= 1e-5, np.percentile(e, [50, 99, 100])
    # and the truncation error against an FP64 direct sum on 1,024 targets
    tg = np.random.default_rng(0).choice(n, 1024, replace=False)
    ts = torch.from_numpy(topo.inverse_permutation[tg].astype(np.int32)).cuda()
    ref = torch.empty((1024, 4), device="cuda", dtype=torch.float64)
    _lib.check(_lib.lib().jb_direct_f64(n, st.pass_.ws.pos4.data_ptr(), 1024, ts.data_ptr(), 1.0, 0.0,
                                        ref.data_ptr(), torch.cuda.current_stream().cuda_stream), "direct")
    r = ref[:, :3].cpu().numpy()
    e = np.linalg.norm(got[ts.cpu().numpy()] - r, axis=1) / np.sqrt((r * r).sum(1).mean())
    assert np.percentile(e, 99) <= 5e-4, np.percentile(e, [50, 99])  # oracle FP64: 3.5e-4
