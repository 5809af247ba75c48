"""GPU adjoint (hand-written VJP kernels through the C ABI) against the float64
adjoint oracle, against FP64 central finite differences of the oracle's
forward pass (relative step 1e-3), and through torch.autograd."""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oracle as O  # noqa: E402
from oracle import adjoint as A  # noqa: E402
from jaccpot_b200 import engine, tree, workloads  # noqa: E402
from jaccpot_b200.autodiff import fmm_accelerations  # noqa: E402

GRAD_P99 = 1e-4  # per-particle relative difference of the FP32 gradient vs the FP64 oracle

CASES = [("uniform", 2048, 16, 0.5, 4), ("plummer", 4096, 16, 0.5, 6), ("clustered", 8192, 32, 0.6, 6),
         ("plummer", 8192, 64, 0.6, 4)]


def _ids(c):
    return f"{c[0]}-n{c[1]}-leaf{c[2]}-th{c[3]}-p{c[4]}"


class Case:
    def __init__(self, gen, n, leaf, theta, p, eps=1e-2, seed=0):
        self.pos, self.mass = workloads.GENERATORS[gen](n, seed)
        self.topo = tree.build_topology(self.pos, self.mass, leaf_size=leaf, theta=theta)
        self.dt = engine.DeviceTopology(self.topo, "cuda")
        self.p, self.eps2 = p, eps * eps
        self.ps = engine.Pass(self.dt, p, G=1.0, eps2=self.eps2)
        self.w = np.random.default_rng(seed + 3).normal(size=(n, 3)).astype(np.float32)
        self.perm = self.topo.permutation

    def gpu_grad(self):
        d_pos = torch.from_numpy(self.pos).cuda()
        d_mass = torch.from_numpy(self.mass).cuda()
        self.ps.load_particles(d_pos, d_mass)
        gx = torch.empty_like(d_pos)
        gm = torch.empty_like(d_mass)
        self.ps.vjp(torch.from_numpy(self.w).cuda(), gx, gm)
        torch.cuda.synchronize()
        return gx.double().cpu().numpy(), gm.double().cpu().numpy()

    def oracle_grad(self):
        p = self.perm
        xb, mb = A.fmm_vjp(self.topo, self.p, self.pos[p].astype(np.float64), self.mass[p].astype(np.float64),
                           self.w[p].astype(np.float64), 1.0, self.eps2)
        gx, gm = np.empty_like(xb), np.empty_like(mb)
        gx[p], gm[p] = xb, mb
        return gx, gm


def _rel_rows(a, b):
    a, b = np.atleast_2d(a.T).T, np.atleast_2d(b.T).T
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_gpu_adjoint_matches_oracle_adjoint(case):
    c = Case(*case)
    gx, gm = c.gpu_grad()
    ox, om = c.oracle_grad()
    ex = _rel_rows(gx, ox)
    em = np.abs(gm - om) / np.maximum(np.abs(om), 1e-300)
    assert np.isfinite(gx).all() and np.isfinite(gm).all()
    assert np.percentile(ex, 99) <= GRAD_P99, np.percentile(ex, [50, 99, 100])
    assert np.percentile(em, 99) <= GRAD_P99, np.percentile(em, [50, 99, 100])
    assert np.linalg.norm(gx - ox) / np.linalg.norm(ox) <= 1e-5
    assert np.linalg.norm(gm - om) / np.linalg.norm(om) <= 1e-5


def fd_richardson(f, h):
    """Central difference with step h, Richardson-extrapolated with h/2
    (error O(h^4) instead of O(h^2))."""
    d1 = (f(h) - f(-h)) / (2 * h)
    d2 = (f(h / 2) - f(-h / 2)) / h
    return (4 * d2 - d1) / 3


def test_gpu_adjoint_matches_central_finite_differences():
    """64 random coordinates at N=8192, FP64 central differences of the oracle's
    forward pass (fixed topology) with relative step 1e-3 (Richardson
    extrapolated: particles closer than the step would otherwise leave the
    difference quotient's own truncation error above the 1e-4 bar)."""
    c = Case("plummer", 8192, 16, 0.5, 6)
    gx, gm = c.gpu_grad()
    p = c.perm
    xs, ms = c.pos[p].astype(np.float64), c.mass[p].astype(np.float64)
    ws = c.w[p].astype(np.float64)
    P = O.Pass(c.topo, np.float64)

    def loss(x, m):
        return float((ws * P.run(c.p, x, m, G=1.0, eps2=c.eps2)["acc"]).sum())

    rng = np.random.default_rng(17)
    inv = c.topo.inverse_permutation
    picks = rng.choice(8192 * 4, 64, replace=False)
    scale_x, scale_m = np.abs(gx).max(), np.abs(gm).max()
    for k in picks:
        i, a = divmod(int(k), 4)
        s = inv[i]
        if a < 3:
            h = 1e-3 * max(abs(xs[s, a]), 1e-3)

            def f(dh, s=s, a=a):
                x1 = xs.copy()
                x1[s, a] += dh
                return loss(x1, ms)

            fd = fd_richardson(f, h)
            assert abs(fd - gx[i, a]) <= 1e-4 * max(abs(fd), 1e-2 * scale_x), (i, a, fd, gx[i, a])
        else:
            h = 1e-3 * ms[s]

            def f(dh, s=s):
                m1 = ms.copy()
                m1[s] += dh
                return loss(xs, m1)

            fd = fd_richardson(f, h)
            assert abs(fd - gm[i]) <= 1e-4 * max(abs(fd), 1e-2 * scale_m), (i, fd, gm[i])


def test_autograd_function_runs_the_adjoint():
    c = Case(*CASES[0])
    pos = torch.from_numpy(c.pos).cuda().requires_grad_(True)
    mass = torch.from_numpy(c.mass).cuda().requires_grad_(True)
    w = torch.from_numpy(c.w).cuda()
    for keep in (1 << 30, 0):  # coefficients kept from the forward / recomputed in the backward
        pos.grad = None
        mass.grad = None
        acc = fmm_accelerations(pos, mass, c.ps, keep_bytes=keep)
        (w * acc).sum().backward()
        gx, gm = c.gpu_grad()
        assert torch.allclose(pos.grad.double().cpu(), torch.from_numpy(gx), rtol=1e-5, atol=1e-6 * np.abs(gx).max())
        assert torch.allclose(mass.grad.double().cpu(), torch.from_numpy(gm), rtol=1e-5, atol=1e-6 * np.abs(gm).max())
