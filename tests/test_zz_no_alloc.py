"""jb_leaf_eval_noalloc: the leaf evaluation for callers that cannot allocate
device memory (an XLA custom-call handler that only sees the buffers XLA
planned for it, or code running under CUDA stream capture).  Its scratch is a
static device array inside the library instead of a caller buffer.

Checked through the C ABI against jb_leaf_eval (caller-provided scratch) on a
schedule that splits many leaves, so the scratch path is exercised, on two
calls in a row (the second call sees the first call's leftovers in the shared
array).  This file is collected last so that a run stopping at the first
failure has already run every other test.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import _lib, engine, tree, workloads  # noqa: E402

ACC_P99 = 1e-5  # the tolerance of the other leaf-evaluation parity tests


def _ptr(t):
    return t.data_ptr()


def test_noalloc_leaf_eval_matches_the_scratch_buffer_version():
    pos, mass = workloads.clustered(32768, seed=3)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=0.5)
    dt = engine.DeviceTopology(topo, "cuda")
    dt.validate()
    # small units: most leaves are split, so the partial rows are used
    ps = engine.Pass(dt, 6, G=1.0, eps2=1e-6, leaf_unit_sources=256)
    sc = ps.leaf_sched
    assert sc.split.shape[0] > 0 and 0 < sc.num_slots <= _lib.JB_LEAF_EVAL_NOALLOC_MAX_SLOTS
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    ps.upward()
    ps.downward()
    want = ps.evaluate(potential=True).clone()

    lb = _lib.lib()
    t, ws = topo, ps.ws
    stream = torch.cuda.current_stream().cuda_stream
    mode = _lib.JB_P2P_POTENTIAL
    for _ in range(2):
        out = torch.full_like(ws.acc4, float("nan"))
        rc = lb.jb_leaf_eval_noalloc(ps.p, mode, _ptr(ws.pos4), t.num_internal, int(sc.units.shape[0]),
                                     _ptr(ps.d_leaf_units), _ptr(ps.d_leaf_aux), _ptr(ps.d_leaf_runs),
                                     _ptr(dt.node_ranges), _ptr(ws.centers), _ptr(ws.locals), ps.G, ps.eps2,
                                     _ptr(out), int(sc.num_slots), int(sc.split.shape[0]), _ptr(ps.d_leaf_split),
                                     stream)
        _lib.check(rc, "jb_leaf_eval_noalloc")
        torch.cuda.synchronize()
        got = out.double().cpu().numpy()
        ref = want.double().cpu().numpy()
        assert np.isfinite(got).all()
        err = workloads.relative_errors(got[:, :3], ref[:, :3])
        assert np.percentile(err, 99) <= ACC_P99, np.percentile(err, [50, 99, 100])
        perr = np.abs(got[:, 3] - ref[:, 3]) / np.abs(ref[:, 3])
        assert np.percentile(perr, 99) <= ACC_P99

    # more slots than the static array holds: refused before any launch
    rc = lb.jb_leaf_eval_noalloc(ps.p, mode, _ptr(ws.pos4), t.num_internal, int(sc.units.shape[0]),
                                 _ptr(ps.d_leaf_units), _ptr(ps.d_leaf_aux), _ptr(ps.d_leaf_runs),
                                 _ptr(dt.node_ranges), _ptr(ws.centers), _ptr(ws.locals), ps.G, ps.eps2,
                                 _ptr(ws.acc4), _lib.JB_LEAF_EVAL_NOALLOC_MAX_SLOTS + 1,
                                 int(sc.split.shape[0]), _ptr(ps.d_leaf_split), stream)
    assert rc == 5  # JB_ERR_WORKSPACE
