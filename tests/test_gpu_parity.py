"""GPU parity of every stage of the pass against the CPU oracle (float64),
called through the C ABI on the same topology and the same inputs.

Stage tests feed the oracle the GPU's own inputs for that stage (centres,
multipoles, locals promoted to float64), so each comparison isolates one
kernel.  The end-to-end test compares the whole GPU pass to the whole oracle
pass and both to an FP64 direct sum.  List handling is checked with integer
pair counts.
"""

from __future__ import annotations

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import oracle as O  # noqa: E402
from jaccpot_b200 import _lib, engine, tree, workloads  # noqa: E402

# Tolerances (float32 kernels vs float64 oracle).
COEF_RTOL = 2e-5   # per-row max-norm relative error of coefficient arrays, 99th percentile
ACC_P99 = 1e-5     # per-particle relative force difference, 99th percentile (FP32 mode)
ACC_MAX = 1e-3

CASES = [
    ("uniform", 16384, 16, 0.6, 4),
    ("uniform", 16384, 16, 0.6, 8),
    ("plummer", 20000, 32, 0.6, 6),
    ("clustered", 32768, 32, 0.5, 8),
    # leaves of 33..64 particles: evaluated in two passes of at most 32 targets
    ("plummer", 40000, 64, 0.6, 6),
    ("clustered", 32768, 48, 0.55, 8),
]


def _ids(c):
    return f"{c[0]}-n{c[1]}-leaf{c[2]}-th{c[3]}-p{c[4]}"


class Setup:
    def __init__(self, gen, n, leaf, theta, p, G=1.0, eps=0.0, seed=0):
        self.pos, self.mass = workloads.GENERATORS[gen](n, seed)
        self.topo = tree.build_topology(self.pos, self.mass, leaf_size=leaf, theta=theta)
        self.dt = engine.DeviceTopology(self.topo, "cuda")
        self.dt.validate()
        self.p = p
        self.G = G
        self.eps2 = eps * eps
        self.ps = engine.Pass(self.dt, p, G=G, eps2=self.eps2)
        self.ps.load_particles(torch.from_numpy(self.pos).cuda(), torch.from_numpy(self.mass).cuda())
        self.pos_s = self.pos[self.topo.permutation].astype(np.float64)
        self.mass_s = self.mass[self.topo.permutation].astype(np.float64)
        self.orc = O.Pass(self.topo, np.float64)
        self.C = (p + 1) ** 2

    def coeffs(self, t):
        return t[:, : self.C].double().cpu().numpy()


_cache = {}


def setup(case):
    if case not in _cache:
        _cache.clear()
        _cache[case] = Setup(*case)
    return _cache[case]


def row_rel(a, b):
    num = np.abs(a - b).max(axis=1)
    den = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return num / den


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_gather_is_exact_permutation(case):
    s = setup(case)
    got = s.ps.ws.pos4.cpu().numpy()
    want = np.concatenate([s.pos[s.topo.permutation], s.mass[s.topo.permutation][:, None]], axis=1)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_upward_parity(case):
    s = setup(case)
    s.ps.upward()
    torch.cuda.synchronize()
    cen = s.ps.ws.centers.double().cpu().numpy()
    com = s.orc.com(s.pos_s, s.mass_s)
    scale = np.abs(s.pos_s).max()
    assert np.abs(cen[:, :3] - com).max() <= 1e-5 * scale
    tot = np.array([s.mass_s[a:b + 1].sum() for a, b in s.topo.node_ranges])
    assert np.allclose(cen[:, 3], tot, rtol=1e-5)
    # multipoles: oracle P2M + M2M on the GPU's centres
    mult_ref = s.orc.upward(s.p, s.pos_s, s.mass_s, cen[:, :3])
    err = row_rel(s.coeffs(s.ps.ws.mult), mult_ref)
    assert np.percentile(err, 99) <= COEF_RTOL, np.percentile(err, [50, 99, 100])
    assert err.max() <= 50 * COEF_RTOL


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_m2l_parity(case):
    s = setup(case)
    s.ps.upward()
    s.ps.m2l()
    torch.cuda.synchronize()
    cen = s.ps.ws.centers.double().cpu().numpy()[:, :3]
    mult = s.coeffs(s.ps.ws.mult)
    ref = s.orc.m2l_accumulate(s.p, mult, cen)
    got = s.coeffs(s.ps.ws.locals)
    has = np.diff(s.topo.far_offsets) > 0
    assert np.all(got[~has] == 0.0)
    err = row_rel(got[has], ref[has])
    assert np.percentile(err, 99) <= COEF_RTOL, np.percentile(err, [50, 99, 100])
    assert err.max() <= 50 * COEF_RTOL


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_l2l_parity(case):
    s = setup(case)
    s.ps.upward()
    s.ps.m2l()
    torch.cuda.synchronize()
    cen = s.ps.ws.centers.double().cpu().numpy()[:, :3]
    loc0 = s.coeffs(s.ps.ws.locals)
    s.ps.l2l(cascade=True)
    torch.cuda.synchronize()
    ref = s.orc.l2l_cascade(s.p, cen, loc0)
    got = s.coeffs(s.ps.ws.locals)
    nz = np.abs(ref).max(axis=1) > 0
    err = row_rel(got[nz], ref[nz])
    assert np.percentile(err, 99) <= COEF_RTOL, np.percentile(err, [50, 99, 100])
    assert err.max() <= 50 * COEF_RTOL


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_l2l_straight_to_the_leaves_parity(case):
    """jb_l2l_leaves (the pass's default downward sweep): every leaf's local
    against the oracle's level-by-level cascade; the internal nodes keep their
    own M2L sums."""
    s = setup(case)
    s.ps.upward()
    s.ps.m2l()
    torch.cuda.synchronize()
    cen = s.ps.ws.centers.double().cpu().numpy()[:, :3]
    loc0 = s.coeffs(s.ps.ws.locals)
    s.ps.l2l_direct = True  # the kernel, whatever the order's default
    try:
        s.ps.l2l()
    finally:
        s.ps.l2l_direct = s.p <= 8
    torch.cuda.synchronize()
    ref = s.orc.l2l_cascade(s.p, cen, loc0)
    got = s.coeffs(s.ps.ws.locals)
    ni = s.ps.dt.topo.num_internal
    assert np.array_equal(got[:ni], loc0[:ni])
    gl, rl = got[ni:], ref[ni:]
    nz = np.abs(rl).max(axis=1) > 0
    err = row_rel(gl[nz], rl[nz])
    assert np.percentile(err, 99) <= COEF_RTOL, np.percentile(err, [50, 99, 100])
    assert err.max() <= 50 * COEF_RTOL


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_leaf_eval_parity(case):
    s = setup(case)
    s.ps.upward()
    s.ps.downward()
    acc4 = s.ps.evaluate(potential=True)
    torch.cuda.synchronize()
    cen = s.ps.ws.centers.double().cpu().numpy()[:, :3]
    loc = s.coeffs(s.ps.ws.locals)
    ref, pot = s.orc.evaluate(s.p, s.pos_s, s.mass_s, cen, loc, s.G, s.eps2)
    got = acc4.double().cpu().numpy()
    err = workloads.relative_errors(got[:, :3], ref)
    assert np.percentile(err, 99) <= ACC_P99, np.percentile(err, [50, 99, 100])
    assert err.max() <= ACC_MAX
    perr = np.abs(got[:, 3] - pot) / np.abs(pot)
    assert np.percentile(perr, 99) <= ACC_P99


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_end_to_end_vs_oracle_and_direct(case):
    s = setup(case)
    acc4 = s.ps.run()
    torch.cuda.synchronize()
    got = acc4.double().cpu().numpy()[:, :3]
    ref = s.orc.run(s.p, s.pos_s, s.mass_s, G=s.G, eps2=s.eps2)["acc"]
    err = workloads.relative_errors(got, ref)
    assert np.percentile(err, 99) <= ACC_P99, np.percentile(err, [50, 99, 100])
    rng = np.random.default_rng(1)
    tg = rng.choice(s.topo.num_particles, size=min(2048, s.topo.num_particles), replace=False)
    direct, _ = O.direct_sum(s.pos_s, s.mass_s, targets=tg, G=s.G, eps2=s.eps2)
    e_gpu = workloads.relative_errors(got[tg], direct)
    e_orc = workloads.relative_errors(ref[tg], direct)
    # the GPU's truncation error is the oracle's up to FP32 round-off
    assert np.percentile(e_gpu, 99) <= np.percentile(e_orc, 99) * 1.05 + 2e-6


@pytest.mark.parametrize("case", CASES[:2], ids=_ids)
def test_near_field_pair_counts_are_exact(case):
    """Unit masses, G = 1, huge softening: every near pair contributes the
    same -rsqrt(eps2) to the potential, so -pot / rsqrt(eps2) is the integer
    number of source particles the kernel summed for each target."""
    s = setup(case)
    eps2 = float(2.0 ** 100)
    ps = engine.Pass(s.dt, s.p, G=1.0, eps2=eps2)
    n = s.topo.num_particles
    ps.load_particles(torch.from_numpy(s.pos).cuda(), torch.ones(n, device="cuda"))
    ps.ws.centers.zero_()
    ps.ws.locals.zero_()
    acc4 = ps.evaluate(potential=True)
    torch.cuda.synchronize()
    c = float(2.0 ** -50)
    got = np.rint(-acc4[:, 3].double().cpu().numpy() / c).astype(np.int64)
    t = s.topo
    cnt = (t.node_ranges[:, 1] - t.node_ranges[:, 0] + 1).astype(np.int64)[t.num_internal:]
    csum = np.concatenate([[0], np.cumsum(cnt[t.near_leaves])])
    per_leaf = cnt - 1 + (csum[t.near_offsets[1:]] - csum[t.near_offsets[:-1]])
    want = per_leaf[t.leaf_of_particle]
    assert np.array_equal(got, want)


@pytest.mark.parametrize("case", CASES[1:2], ids=_ids)
def test_targets_match_full_evaluation(case):
    s = setup(case)
    s.ps.run()
    full = s.ps.ws.acc4.double().cpu().numpy()
    rng = np.random.default_rng(7)
    ts = rng.choice(s.topo.num_particles, size=4096, replace=False).astype(np.int32)
    out = s.ps.evaluate_targets(torch.from_numpy(ts).cuda())
    torch.cuda.synchronize()
    got = out.double().cpu().numpy()
    err = workloads.relative_errors(got[:, :3], full[ts, :3])
    assert err.max() <= 2e-5
    # and against the oracle's own target path
    cen = s.ps.ws.centers.double().cpu().numpy()[:, :3]
    loc = s.coeffs(s.ps.ws.locals)
    ref, _ = s.orc.evaluate_targets(s.p, s.pos_s, s.mass_s, cen, loc, ts, s.G, s.eps2)
    assert np.percentile(workloads.relative_errors(got[:, :3], ref), 99) <= ACC_P99


def test_pass_is_deterministic():
    s = setup(CASES[1])
    a = s.ps.run().clone()
    b = s.ps.run().clone()
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_compensated_near_field_is_not_worse():
    s = setup(CASES[1])
    ps = engine.Pass(s.dt, s.p, G=1.0, eps2=0.0, p2p_mode=_lib.JB_P2P_KAHAN)
    ps.load_particles(torch.from_numpy(s.pos).cuda(), torch.from_numpy(s.mass).cuda())
    got_k = ps.run().double().cpu().numpy()[:, :3]
    got = s.ps.run().double().cpu().numpy()[:, :3]
    ref = s.orc.run(s.p, s.pos_s, s.mass_s)["acc"]
    ek = workloads.relative_errors(got_k, ref)
    e = workloads.relative_errors(got, ref)
    assert np.percentile(ek, 99) <= np.percentile(e, 99) * 1.1


def test_errors_are_reported_not_trapped():
    s = setup(CASES[0])
    lb = _lib.lib()
    assert lb.jb_p2m(11, 0, 1, 0, 0, 0, 0, 0) == _lib.JB_OK + 1  # null pointers -> JB_ERR_ARG
    assert lb.jb_m2l(s.p, 7, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0) == 8  # unknown mode
    with pytest.raises(_lib.JBError):
        _lib.coeff_stride(0)


@pytest.mark.parametrize("with_pot", [False, True])
def test_unsort_gather_equals_scatter(with_pot):
    """jb_gather_unsorted (out[j] = acc4[inv_perm[j]]) moves the same values as
    jb_scatter_unsorted (out[perm[i]] = acc4[i]), bit for bit."""
    lb = _lib.lib()
    n = 100_003
    rng = np.random.default_rng(5)
    perm = rng.permutation(n).astype(np.int64)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(n)
    d_perm, d_inv = torch.from_numpy(perm).cuda(), torch.from_numpy(inv).cuda()
    acc4 = torch.randn((n, 4), device="cuda")
    outs = []
    for fn, idx in ((lb.jb_scatter_unsorted, d_perm), (lb.jb_gather_unsorted, d_inv)):
        a = torch.full((n, 3), float("nan"), device="cuda")
        p = torch.full((n,), float("nan"), device="cuda")
        _lib.check(fn(n, acc4.data_ptr(), idx.data_ptr(), a.data_ptr(), p.data_ptr() if with_pot else None,
                      torch.cuda.current_stream().cuda_stream), "unsort")
        outs.append((a, p))
    torch.cuda.synchronize()
    assert torch.equal(outs[0][0], outs[1][0])
    assert torch.equal(outs[0][0], acc4[torch.from_numpy(inv).cuda(), :3])
    if with_pot:
        assert torch.equal(outs[0][1], outs[1][1])
