"""The step as a CUDA graph (Pass.capture and the facade's cuda_graph option):
a replay launches the eager step's kernels with its arguments, so it gives
the eager step's bits -- on the captured inputs and on new inputs copied into
the captured buffers -- for the plain pass and the error-controlled pass
with its one-launch mixed-order M2L."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import FastMultipoleMethod, engine, tree, workloads  # noqa: E402


def _eager(ps, pos, mass):
    acc = torch.empty_like(pos)
    ps.load_particles(pos, mass)
    ps.run()
    ps.unsort(acc, None)
    return acc


def test_replay_equals_eager_plain():
    pos, mass = workloads.clustered(60_000, 3)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=0.6, device="cuda")
    ps = engine.Pass(engine.DeviceTopology(topo, "cuda"), 8, G=1.0, eps2=1e-6)
    d_pos, d_mass = torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda()
    acc = torch.empty_like(d_pos)
    g = ps.capture(d_pos, d_mass, acc)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(acc, _eager(ps, d_pos, d_mass))
    # new particles of the same topology, copied into the captured buffers
    moved = d_pos + 1e-4 * torch.randn_like(d_pos)
    d_pos.copy_(moved)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(acc, _eager(ps, moved.clone(), d_mass))


def test_facade_graph_path_equals_eager_for_the_error_controlled_form():
    pos, mass = workloads.clustered(60_000, 4)
    kw = dict(theta=0.6, softening=0.0, adaptive_order=True, p_gears=(2, 4, 6, 8), adaptive_error_model="dehnen_paper",
              adaptive_eps=3e-5, mac_force_scale_mode="paper")
    f_g = FastMultipoleMethod(**kw, advanced={"cuda_graph": True, "nearfield_compensated": True})
    f_e = FastMultipoleMethod(**kw, advanced={"nearfield_compensated": True})
    st_g = f_g.prepare_state(pos, mass, leaf_size=32, max_order=8)
    st_e = f_e.prepare_state(pos, mass, leaf_size=32, max_order=8)
    assert type(st_g.pass_.gear_sched).__name__ == "MixedGearM2LSchedule"
    rng = np.random.default_rng(1)
    for k in range(3):
        p = (pos + 1e-4 * k * rng.standard_normal(pos.shape)).astype(np.float32)
        a = f_g.differentiable_accelerations(st_g, p, mass)
        b = f_e.differentiable_accelerations(st_e, p, mass)
        assert torch.equal(a, b), k
    d = f_g.get_runtime_diagnostics()
    assert d["graph_captures"] == 1 and d["graph_replays"] == 3
    # device inputs give a device result from the same graph
    dev_out = f_g.differentiable_accelerations(st_g, torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    assert dev_out.is_cuda and torch.equal(dev_out.cpu(), f_e.differentiable_accelerations(st_e, pos, mass))
