"""The facade's sampled error monitor (advanced={"error_monitor": ...}): every
`every`-th whole-pass evaluation is checked against an FP64 direct sum on a
random target sample; the recorded percentiles are recomputed here from the
returned accelerations and an independent FP64 direct sum (the oracle's)."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oracle as O  # noqa: E402
from jaccpot_b200 import FastMultipoleMethod, workloads  # noqa: E402


def test_monitor_records_the_sampled_error():
    pos, mass = workloads.clustered(20_000, 9)
    soft = 1e-3
    f = FastMultipoleMethod(theta=0.6, softening=soft, advanced={"error_monitor": {"targets": 96, "every": 2}})
    st = f.prepare_state(pos, mass, leaf_size=32, max_order=6)
    accs = [f.evaluate_prepared_state(st) for _ in range(3)]
    assert [r["evaluation"] for r in f.error_history] == [1, 3]
    # the sample of check 3: the same generator over sorted indices
    rng = np.random.default_rng((0, 3))
    ts = rng.choice(pos.shape[0], size=96, replace=False)
    orig = st.topology.permutation[ts]
    d, _ = O.direct_sum(pos.astype(np.float32).astype(np.float64), mass.astype(np.float32).astype(np.float64),
                        eps2=soft * soft, targets=orig)
    got = accs[2][orig].astype(np.float64)
    e = np.linalg.norm(got - d, axis=1) / np.linalg.norm(d, axis=1)
    rec = f.error_history[-1]
    assert rec["p99"] == pytest.approx(np.percentile(e, 99), rel=1e-3)
    assert rec["max"] == pytest.approx(e.max(), rel=1e-3)
    assert rec["within_bound"] == (rec["p99"] <= 1e-4)
    assert f.get_runtime_diagnostics()["error_checks"] == 2
    assert rec["p99"] < 5e-3  # order 6, theta 0.6 on a clustered set


def test_monitor_runs_on_the_reevaluation_path():
    pos, mass = workloads.uniform_cube(8_000, 3)
    f = FastMultipoleMethod(theta=0.5, softening=1e-2, advanced={"error_monitor": 32})
    st = f.prepare_state(pos, mass, leaf_size=16, max_order=6)
    f.differentiable_accelerations(st, pos, mass)
    assert len(f.error_history) == 1 and f.error_history[0]["p99"] < 1e-3
