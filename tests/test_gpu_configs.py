"""The benchmark configurations at their full sizes, checked through
size-independent properties (the oracle cannot run them in seconds)."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from jaccpot_b200 import FastMultipoleMethod, _lib, workloads  # noqa: E402


def test_targets_at_plummer_1m_p6_match_the_full_evaluation():
    """Plummer N=1,048,576, p=6, leaf 32: evaluate_prepared_state on 65,536
    int32 targets drawn without replacement equals the full evaluation at
    those particles (same lists, same locals)."""
    n = 1048576
    pos, mass = workloads.plummer(n, 0)
    fmm = FastMultipoleMethod(preset="large_n_gpu", theta=0.6, G=1.0, softening=0.0)
    st = fmm.prepare_state(pos, mass, leaf_size=32, max_order=6)
    full = fmm.evaluate_prepared_state(st)
    tg = np.random.default_rng(0).choice(n, 65536, replace=False).astype(np.int32)
    sub = fmm.evaluate_prepared_state(st, target_indices=tg)
    assert sub.shape == (65536, 3) and np.isfinite(sub).all()
    err = workloads.relative_errors(sub, full[tg])
    assert err.max() <= 2e-5, err.max()


def test_clustered_4m_pass_against_direct_sum():
    """Clustered N=4,194,304, p=8, leaf 32, theta 0.55 (the headline workload):
    plain and split-BF16 forms against an FP64 direct sum on 4,096 targets."""
    n = 4194304
    pos, mass = workloads.clustered(n, 0)
    fmm = FastMultipoleMethod(theta=0.55, G=1.0, softening=0.0)
    st = fmm.prepare_state(pos, mass, leaf_size=32, max_order=8)
    from jaccpot_b200 import engine

    rng = np.random.default_rng(3)
    tg = rng.choice(n, 4096, replace=False)
    ts = torch.from_numpy(st.topology.inverse_permutation[tg].astype(np.int32)).cuda()
    ref = torch.empty((4096, 4), device="cuda", dtype=torch.float64)
    ps = st.pass_
    _lib.check(_lib.lib().jb_direct_f64(n, ps.ws.pos4.data_ptr(), 4096, ts.data_ptr(), 1.0, 0.0, ref.data_ptr(),
                                        torch.cuda.current_stream().cuda_stream), "direct")
    ref = ref[:, :3].cpu().numpy()
    for mode in (_lib.JB_M2L_FP32, _lib.JB_M2L_SPLIT_BF16):
        p2 = engine.Pass(st.device_topology, 8, G=1.0, eps2=0.0, m2l_mode=mode, p2p_mode=_lib.JB_P2P_KAHAN)
        p2.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
        acc = p2.run()[ts.long(), :3].double().cpu().numpy()
        e = workloads.relative_errors(acc, ref)
        assert np.percentile(e, 99) <= 1e-4, (mode, np.percentile(e, [50, 99]))
