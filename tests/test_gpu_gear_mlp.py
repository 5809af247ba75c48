"""The gear selector's hand-written MLP kernels against the float64 numpy
restatement (oracle/mlp.py): batch gradients, the Adam step, the fused
per-pair inference; and a short training run on FMM-generated labels."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from oracle import mlp as M  # noqa: E402
from jaccpot_b200 import _lib, engine, gears, tree, workloads  # noqa: E402


def _ptr(t):
    return t.data_ptr()


def _rand_params(seed=0):
    return gears.bf16_round(gears.init_params(np.random.default_rng(seed)) * 1.5)


def test_gradient_kernel_matches_oracle():
    rng = np.random.default_rng(1)
    n = 1000  # not a multiple of the 128-sample block: the tail block is masked
    X = rng.normal(size=(n, 12)).astype(np.float32)
    lab = rng.integers(0, 4, size=n).astype(np.int32)
    W = _rand_params()
    nb = (n + 127) // 128
    gpart = torch.empty((nb, gears.N_PARAMS), device="cuda")
    lpart = torch.empty((nb,), device="cuda")
    dX, dL, dW = torch.from_numpy(X).cuda(), torch.from_numpy(lab).cuda(), torch.from_numpy(W).cuda()
    _lib.check(_lib.lib().jb_gear_train_grad(n, _ptr(dX), _ptr(dL), _ptr(dW), _ptr(gpart), _ptr(lpart),
                                             torch.cuda.current_stream().cuda_stream), "grad")
    torch.cuda.synchronize()
    g = gpart.double().sum(0).cpu().numpy()
    loss = float(lpart.double().sum())
    ref_loss, ref_g = M.loss_and_grad(W.astype(np.float64), X.astype(np.float64), lab)
    assert abs(loss - ref_loss) <= 1e-4 * abs(ref_loss)
    assert np.linalg.norm(g - ref_g) <= 1e-4 * np.linalg.norm(ref_g)
    # every block's share, not just the total
    assert np.abs(g - ref_g).max() <= 1e-3 * np.abs(ref_g).max()


def test_adam_step_matches_numpy():
    rng = np.random.default_rng(2)
    P = gears.N_PARAMS
    master = rng.normal(size=P).astype(np.float32)
    m1 = (rng.normal(size=P) * 1e-2).astype(np.float32)
    m2 = (rng.uniform(size=P) * 1e-3).astype(np.float32)
    gp = rng.normal(size=(3, P)).astype(np.float32)
    d = {k: torch.from_numpy(v.copy()).cuda() for k, v in dict(master=master, m1=m1, m2=m2, gp=gp).items()}
    Wq = torch.empty(P, device="cuda")
    _lib.check(_lib.lib().jb_gear_adam(3, _ptr(d["gp"]), 0.25, 1e-3, 0.9, 0.999, 1e-8, 5, _ptr(d["master"]),
                                       _ptr(d["m1"]), _ptr(d["m2"]), _ptr(Wq),
                                       torch.cuda.current_stream().cuda_stream), "adam")
    torch.cuda.synchronize()
    g = gp.astype(np.float64).sum(0) * 0.25
    a = 0.9 * m1 + 0.1 * g
    v = 0.999 * m2 + 0.001 * g * g
    w = master - 1e-3 * (a / (1 - 0.9 ** 5)) / (np.sqrt(v / (1 - 0.999 ** 5)) + 1e-8)
    assert np.allclose(d["master"].cpu().numpy(), w, rtol=1e-5, atol=1e-6)
    assert np.array_equal(Wq.cpu().numpy(), gears.bf16_round(d["master"].cpu().numpy()))


@pytest.fixture(scope="module")
def system():
    pos, mass = workloads.clustered(65536, seed=21)
    topo = tree.build_topology(pos, mass, leaf_size=32, theta=0.6)
    dt = engine.DeviceTopology(topo, "cuda")
    ps = engine.Pass(dt, 8, G=1.0, eps2=0.0)
    ps.load_particles(torch.from_numpy(pos).cuda(), torch.from_numpy(mass).cuda())
    ps.run()
    ctx = gears.GearContext(ps)
    ctx.node_features()
    return ps, ctx


def test_fused_inference_matches_host_network(system):
    ps, ctx = system
    X = ctx.pair_features().cpu().numpy()
    rng = np.random.default_rng(3)
    model = gears.GearModel(params=_rand_params(4), norm=np.concatenate([X.mean(0), 1 / (X.std(0) + 1e-6)]).astype(
        np.float32), conf=0.6, min_top=0.3)
    got = ctx.select(model).cpu().numpy()
    want = gears.predict(model, X)
    assert got.shape == want.shape
    assert (got == want).mean() >= 0.999
    assert set(np.unique(got)) <= {0, 1, 2, 3}
    del rng


def test_training_on_fmm_labels_reduces_the_loss(system):
    X, Y = gears.make_samples(7, n=65536, per_seed=40000)
    assert X.shape == (40000, 12) and Y.shape == (40000, 4) and np.isfinite(X).all() and np.isfinite(Y).all()
    # errors fall with the order for almost every pair
    assert np.mean(Y[:, 0] >= Y[:, 3]) > 0.99
    lab = gears.labels_for(Y, 1e-5)
    Wq, norm, hist = gears.train(X, lab, epochs=6, batch=2048)
    assert hist[-1] < 0.7 * hist[0]
    model = gears.GearModel(params=Wq, norm=norm, budget=1e-5)
    # the network learns the labels ...
    acc = (gears.probabilities(model, X).argmax(1) == lab).mean()
    assert acc > 0.8, acc
    # ... and the conservative selection rule rarely picks a gear below the label
    assert (gears.predict(model, X) < lab).mean() < 0.02
