"""refresh_prepared_state (the reference's same-topology refresh,
solver.py:1604 / runtime/fmm_strict_run.py:1152): a hit reuses the state's
schedules and gives exactly what a fresh prepare_state gives on the new
inputs; a changed topology or changed parameters fall back to a full prepare;
the old state stays valid."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import workloads  # noqa: E402
from jaccpot_b200.solver import FastMultipoleMethod  # noqa: E402

N = 200_000


def _fresh(fmm_kw, pos, mass, **kw):
    fmm = FastMultipoleMethod(**fmm_kw)
    st = fmm.prepare_state(pos, mass, **kw)
    return fmm.evaluate_prepared_state(st)


@pytest.mark.parametrize("adaptive", [False, True])
def test_refresh_hit_equals_a_fresh_prepare(adaptive):
    pos, mass = workloads.clustered(N, seed=4)
    kw = dict(theta=0.55, G=1.0, softening=0.0, nearfield_compensated=True, adaptive_order=adaptive)
    prep = dict(leaf_size=32, max_order=8)
    fmm = FastMultipoleMethod(**kw)
    st0 = fmm.prepare_state(pos, mass, **prep)
    acc0 = fmm.evaluate_prepared_state(st0)
    # doubled masses: the same Morton order and (exactly) the same centres, so
    # the same lists -- a hit
    st1 = fmm.refresh_prepared_state(st0, pos, 2 * mass)
    assert fmm.refresh_stats["hits"] == 1 and st1 is not st0
    assert st1.pass_.ws.mult.data_ptr() != st0.pass_.ws.mult.data_ptr()
    acc1 = fmm.evaluate_prepared_state(st1)
    want = _fresh(kw, pos, 2 * mass, **prep)
    assert np.array_equal(acc1, want)
    # the old state still evaluates its own particles
    assert np.array_equal(fmm.evaluate_prepared_state(st0), acc0)


def test_refresh_miss_on_a_moved_particle_set_and_on_new_parameters():
    pos, mass = workloads.clustered(N, seed=4)
    kw = dict(theta=0.55, G=1.0, softening=0.0)
    fmm = FastMultipoleMethod(**kw)
    st0 = fmm.prepare_state(pos, mass, leaf_size=32, max_order=6)
    rng = np.random.default_rng(1)
    moved = (pos + rng.normal(0, 0.05, size=pos.shape)).astype(np.float32)
    st1 = fmm.refresh_prepared_state(st0, moved, mass)
    assert fmm.refresh_stats["miss_topology"] == 1 and fmm.refresh_stats["hits"] == 0
    assert np.array_equal(fmm.evaluate_prepared_state(st1), _fresh(kw, moved, mass, leaf_size=32, max_order=6))
    st2 = fmm.refresh_prepared_state(st1, moved, mass, max_order=4)
    assert fmm.refresh_stats["miss_config"] == 1 and st2.max_order == 4
    assert np.array_equal(fmm.evaluate_prepared_state(st2), _fresh(kw, moved, mass, leaf_size=32, max_order=4))


def test_strict_loop_prepares_then_refreshes():
    pos, mass = workloads.plummer(50_000, seed=9)
    fmm = FastMultipoleMethod(theta=0.6, G=1.0, softening=1e-3)
    st, a0 = fmm.strict_prepare_refresh_and_evaluate(None, pos, mass, leaf_size=16, max_order=4)
    st, a1 = fmm.strict_prepare_refresh_and_evaluate(st, pos, 3 * mass, leaf_size=16, max_order=4)
    assert fmm.refresh_stats["hits"] == 1
    scale = np.sqrt((a0 * a0).sum(1).mean())
    np.testing.assert_allclose(a1, 3 * a0, rtol=0, atol=3e-5 * scale)
