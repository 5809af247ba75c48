"""The FP64 direct sum on sampled targets (jb_direct_f64, a thread-block
cluster per target) against the oracle's FP64 direct sum: the error report,
the bench's selection and the facade's error monitor all rest on it."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oracle as O  # noqa: E402
from jaccpot_b200 import _lib  # noqa: E402


@pytest.mark.parametrize("n,nt,eps2", [(1, 1, 0.0), (5, 5, 1e-4), (7, 3, 0.0), (20_000, 257, 0.0),
                                       (100_003, 64, 1e-6)])
def test_direct_f64_matches_the_oracle(n, nt, eps2):
    rng = np.random.default_rng(n)
    pos = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    mass = rng.uniform(0.5, 1.5, n).astype(np.float32)
    ts = np.sort(rng.choice(n, size=nt, replace=False)).astype(np.int32)
    pos4 = torch.from_numpy(np.concatenate([pos, mass[:, None]], axis=1)).cuda()
    d_ts = torch.from_numpy(ts).cuda()
    out = torch.empty((nt, 4), device="cuda", dtype=torch.float64)
    _lib.check(_lib.lib().jb_direct_f64(n, pos4.data_ptr(), nt, d_ts.data_ptr(), 1.5, eps2, out.data_ptr(),
                                        torch.cuda.current_stream().cuda_stream), "jb_direct_f64")
    acc, pot = O.direct_sum(pos.astype(np.float64), mass.astype(np.float64), targets=ts, G=1.5, eps2=eps2)
    got = out.cpu().numpy()
    if n == 1:
        assert np.all(got == 0.0)
        return
    scale = np.abs(acc).max(axis=1, keepdims=True)
    assert np.abs(got[:, :3] - acc).max() <= 1e-12 * scale.max()
    assert np.allclose(got[:, 3], pot, rtol=1e-12, atol=0.0)
