"""Facade paths beyond prepare/evaluate, on the GPU: reuse_topology /
rebuild_every, strict_run_v2 (velocity Verlet, refresh every step),
strict_run_segmented, prepare_upward_sweep, differentiable_step_fn with
target_indices, and the error-controlled lane (adaptive_error_model=
"dehnen_paper") with its cached force scale."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oracle  # noqa: E402
from jaccpot_b200 import FastMultipoleMethod, workloads  # noqa: E402

KW = dict(theta=0.6, G=1.0, softening=1e-3)


def test_reuse_topology_holds_the_lists_for_rebuild_every_calls():
    pos, mass = workloads.plummer(30_000, 1)
    fmm = FastMultipoleMethod(reuse_topology=True, rebuild_every=3, **KW)
    ref = FastMultipoleMethod(**KW)
    rng = np.random.default_rng(0)
    for call in range(4):
        p = (pos + rng.normal(0, 1e-3, size=pos.shape)).astype(np.float32)
        acc = fmm.compute_accelerations(p, mass, leaf_size=16, max_order=4)
        held = fmm._reuse["state"]
        # every call equals the whole pass on the held (fixed) topology
        want = ref.differentiable_accelerations(held, p, mass)
        assert np.array_equal(acc, np.asarray(want))
    d = fmm.get_runtime_diagnostics()
    assert d["reuse_rebuilds"] == 2 and d["reuse_hits"] == 2


def test_strict_run_v2_is_velocity_verlet_with_a_refresh_each_step():
    n = 20_000
    pos, mass = workloads.plummer(n, 2)
    vel = np.random.default_rng(1).normal(0, 0.1, size=(n, 3)).astype(np.float32)
    state = np.stack([pos, vel], axis=1)
    dt, steps = 1e-3, 3
    fmm = FastMultipoleMethod(**KW)
    out, st, hist = fmm.strict_run_v2(state=state, masses=mass, dt=dt, num_steps=steps, refresh_every=1,
                                      leaf_size=16, max_order=4, return_history=True)
    assert out.shape == (n, 2, 3) and hist.shape == (steps, n, 2, 3) and st is not None
    # the same integration through prepare_state + evaluate
    man = FastMultipoleMethod(**KW)
    x = torch.from_numpy(pos).cuda().clone()
    v = torch.from_numpy(vel).cuda().clone()
    m = torch.from_numpy(mass).cuda()
    a = man.evaluate_prepared_state(man.prepare_state(x, m, leaf_size=16, max_order=4), as_numpy=False)
    for _ in range(steps):
        v.add_(a, alpha=0.5 * dt)
        x.add_(v, alpha=dt)
        a = man.evaluate_prepared_state(man.prepare_state(x, m, leaf_size=16, max_order=4), as_numpy=False)
        v.add_(a, alpha=0.5 * dt)
    np.testing.assert_allclose(out[:, 0], x.cpu().numpy(), rtol=0, atol=1e-6)
    np.testing.assert_allclose(out[:, 1], v.cpu().numpy(), rtol=0, atol=1e-5)
    np.testing.assert_array_equal(hist[-1], out)


def test_strict_run_segmented_refreshes_per_segment():
    n = 10_000
    pos, mass = workloads.uniform_cube(n, 3)
    fmm = FastMultipoleMethod(**KW)
    calls = []

    def runner(state, acc, k):
        calls.append(k)
        return state + 1e-4 * k * np.asarray(acc), float(np.abs(acc).sum())

    out, st, hist = fmm.strict_run_segmented(state=pos.copy(), masses=mass, num_steps=7, refresh_every=3,
                                             segment_runner=runner, positions_getter=lambda s: s,
                                             leaf_size=16, max_order=4, collect_history=True)
    assert calls == [3, 3, 1] and len(hist) == 3 and out.shape == pos.shape and st is not None


def test_upward_sweep_seam_and_step_fn_with_targets():
    n = 40_000
    pos, mass = workloads.clustered(n, 4)
    fmm = FastMultipoleMethod(**KW)
    st = fmm.prepare_state(pos, mass, leaf_size=32, max_order=6)
    t = st.topology
    up = fmm.prepare_upward_sweep(t, pos[t.permutation], mass[t.permutation], max_order=6)
    st.pass_.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    st.pass_.upward()
    assert torch.equal(up["multipoles"], st.pass_.ws.mult[:, :49])
    assert torch.equal(up["centers"], st.pass_.ws.centers)
    step = fmm.differentiable_step_fn(st, compile_now=(pos, mass))
    full = np.asarray(step(pos, mass))
    tg = np.random.default_rng(5).choice(n, 1000, replace=False)
    sub = fmm.differentiable_accelerations(st, pos, mass, target_indices=tg)
    assert np.array_equal(np.asarray(sub), full[tg])


def test_error_controlled_lane_through_the_facade():
    n = 131_072
    pos, mass = workloads.clustered(n, 6)
    fmm = FastMultipoleMethod(theta=0.6, G=1.0, softening=0.0, adaptive_order=True, p_gears=(2, 4, 6, 8),
                              adaptive_error_model="dehnen_paper", adaptive_eps=3e-5)
    st = fmm.prepare_state(pos, mass, leaf_size=32, max_order=8)
    assert st.topology.far_gears is not None and "adaptive" in st.scratch
    acc = fmm.evaluate_prepared_state(st)
    tg = np.random.default_rng(7).choice(n, 2048, replace=False)
    oracle.build()
    ref, _ = oracle.direct_sum(pos.astype(np.float64), mass.astype(np.float64), targets=tg)
    err = workloads.relative_errors(acc[tg], ref)
    assert np.percentile(err, 99) <= 1e-4, np.percentile(err, [50, 99])
    # 'prev': the next prepare takes its force scale from this evaluation
    d0 = fmm.get_runtime_diagnostics()
    st2 = fmm.prepare_state(pos, mass, leaf_size=32, max_order=8)
    d1 = fmm.get_runtime_diagnostics()
    assert d1["force_scale_reused"] == d0["force_scale_reused"] + 1
    assert d1["force_scale_prepasses"] == d0["force_scale_prepasses"]
    acc2 = fmm.evaluate_prepared_state(st2)
    err2 = workloads.relative_errors(acc2[tg], ref)
    assert np.percentile(err2, 99) <= 1e-4
    with pytest.raises(ValueError):  # the top gear must be the pass order
        fmm.prepare_state(pos, mass, leaf_size=32, max_order=6)
