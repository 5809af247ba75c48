"""Reverse-mode (VJP) restatement of the FMM pass at fixed topology, float64 —
TEST INFRASTRUCTURE ONLY (imported by tests/ and nothing in the product).

Computes the gradient of L = sum_i w_i . a_i with respect to the sorted
positions and masses, where a is the whole pass of ``oracle.Pass.run`` (COM
centres, P2M, M2M, M2L, L2L, L2P + softened P2P) evaluated on live inputs with
the topology held fixed — the contract of the reference's
``differentiable_accelerations`` (runtime/fmm_evaluate.py:542-731, :1175-1250;
analytic near-field VJP nearfield/grad.py:726-869; analytic L2P VJP
operators/real_p2m_l2p.py:402-491).  Checked against central finite
differences of ``oracle.Pass.run``.

Every linear operator (M2M, M2L, L2L for a displacement) is materialised here
by probing the oracle's own operator with unit vectors, so its transpose is
exact and independent of how the GPU kernels factor it.  Derivatives with
respect to displacements use the ladder identities of the solid harmonics:

  d/dd_a of a local re-expanded about a centre moved by d:   D_a (the L2P gradient ladder)
  d/dd_a of a multipole moved by d:                          D_a^T (its transpose)
  d/dd_a of the order-p triangular M2L:  -D_a applied to the order-(p+1) M2L

where D_a maps degree-n local coefficients to the degree n-1 coefficients of
the a-derivative (the same relations the L2P gradient uses).
"""

from __future__ import annotations

import numpy as np

import oracle as O


def sh(n: int, m: int) -> int:
    return n * n + n + m


def ladder(p: int) -> np.ndarray:
    """D[a] (3, C, C): (D_a F) are the coefficients of d/ddelta_a sum F U(delta)
    in the same basis (degrees <= p-1 filled).  Restates the L2P gradient
    relations dU_n^m/dz = U_{n-1}^m, (d/dx -+ i d/dy) R_n^m = +-R_{n-1}^{m-+1}."""
    C = (p + 1) ** 2
    D = np.zeros((3, C, C))
    X, Y, Z = 0, 1, 2
    for n in range(1, p + 1):
        q = n - 1
        # m = 0
        D[Z, sh(q, 0), sh(n, 0)] += 1.0
        if q >= 1:
            D[X, sh(q, 1), sh(n, 0)] += -1.0
            D[Y, sh(q, -1), sh(n, 0)] += -1.0
        for m in range(1, n + 1):
            fc, fs = sh(n, m), sh(n, -m)
            if m <= q:
                D[Z, sh(q, m), fc] += 1.0
                D[Z, sh(q, -m), fs] += 1.0
            # cos channel: gx += fc * 0.5 (um1 - up1); gy += fc * -0.5 (sp1 + sm1)
            # sin channel: gx += fs * 0.5 (sm1 - sp1); gy += fs * 0.5 (up1 + um1)
            if m - 1 <= q:
                D[X, sh(q, m - 1), fc] += 0.5
                D[Y, sh(q, m - 1), fs] += 0.5
                if m - 1 >= 1:
                    D[Y, sh(q, -(m - 1)), fc] += -0.5
                    D[X, sh(q, -(m - 1)), fs] += 0.5
            if m + 1 <= q:
                D[X, sh(q, m + 1), fc] += -0.5
                D[Y, sh(q, -(m + 1)), fc] += -0.5
                D[X, sh(q, -(m + 1)), fs] += -0.5
                D[Y, sh(q, m + 1), fs] += 0.5
    return D


def _op_matrices(fn, p, deltas, chunk=1024):
    """Dense (P, C, C) matrices of a batched linear operator fn(p, vecs, deltas)."""
    C = (p + 1) ** 2
    P = deltas.shape[0]
    out = np.empty((P, C, C))
    eye = np.eye(C)
    for a in range(0, P, chunk):
        d = deltas[a:a + chunk]
        k = d.shape[0]
        vecs = np.tile(eye, (k, 1))
        dd = np.repeat(d, C, axis=0)
        cols = fn(p, vecs, dd).reshape(k, C, C)  # [pair, input basis j, output i]
        out[a:a + k] = np.transpose(cols, (0, 2, 1))
    return out


def _U(p, deltas):
    return O.p2m(p, deltas, np.ones(deltas.shape[0]))


def _grad_phi(p, F, deltas):
    """grad_delta of sum F U(delta) (rows of F per delta)."""
    _, g = O.l2p(p, F, deltas)
    return g


def fmm_vjp(topo, p, pos, mass, w, G=1.0, eps2=0.0):
    """Gradient of sum(w * acc) w.r.t. sorted positions (N,3) and masses (N,)."""
    t = topo
    pos = np.asarray(pos, np.float64)
    mass = np.asarray(mass, np.float64)
    w = np.asarray(w, np.float64)
    N = pos.shape[0]
    C = (p + 1) ** 2
    ni = t.num_internal
    nodes = t.num_nodes
    L = t.num_leaves
    rg = t.node_ranges
    Dm = ladder(p)

    P = O.Pass(t, np.float64)
    fw = P.run(p, pos, mass, G=G, eps2=eps2)
    cen, M, F = fw["centers"], fw["multipoles"], fw["locals"]
    mu = np.array([mass[a:b + 1].sum() for a, b in rg])
    left, right = t.left_child, t.right_child
    lo = t.level_offsets

    xbar = np.zeros((N, 3))
    mbar = np.zeros(N)
    cbar = np.zeros((nodes, 3))
    Lbar = np.zeros((nodes, C))
    Mbar = np.zeros((nodes, C))

    leaf_of = t.leaf_of_particle
    cl = cen[ni + leaf_of]  # centre of each particle's leaf

    # ---- L2P: a_far = -G grad_delta phi_F(delta), delta = c - x
    delta = cl - pos
    U = _U(p, delta)
    # Fbar_leaf = -G sum_i sum_a w_ia D_a^T U(delta_i)
    contrib = -G * np.einsum("ia,acj,ic->ij", w, Dm, U)
    np.add.at(Lbar, ni + leaf_of, contrib)
    # deltabar_i = -G grad_delta (sum_a w_ia D_a F) . U
    Fl = F[ni + leaf_of]
    Gw = np.einsum("ia,acj,ij->ic", w, Dm, Fl)
    dbar = -G * _grad_phi(p, Gw, delta)
    xbar -= dbar
    np.add.at(cbar, ni + leaf_of, dbar)

    # ---- near field (self leaf + neighbour leaves), softened
    for lf in range(L):
        a0, a1 = rg[ni + lf]
        tg = np.arange(a0, a1 + 1)
        srcs = [np.arange(a0, a1 + 1)]
        for e in range(t.near_offsets[lf], t.near_offsets[lf + 1]):
            s0, s1 = rg[ni + t.near_leaves[e]]
            srcs.append(np.arange(s0, s1 + 1))
        sj = np.concatenate(srcs)
        d = pos[tg][:, None, :] - pos[sj][None, :, :]
        r2 = (d * d).sum(-1) + eps2
        self_mask = tg[:, None] == sj[None, :]
        r2 = np.where(self_mask, 1.0, r2)
        q = 1.0 / np.sqrt(r2)
        q3 = np.where(self_mask, 0.0, q ** 3)
        q5 = np.where(self_mask, 0.0, q ** 5)
        wt = w[tg]
        wd = np.einsum("ia,ija->ij", wt, d)
        # a_i = -G sum_j m_j d q^3 ;  d(w.a_i)/d(d) = -G m_j (w q^3 - 3 q^5 (w.d) d)
        gd = -G * mass[sj][None, :, None] * (wt[:, None, :] * q3[..., None] - 3.0 * (q5 * wd)[..., None] * d)
        xbar[tg] += gd.sum(1)
        np.add.at(xbar, sj, -gd.reshape(-1, 3) if False else -gd.sum(0))
        np.add.at(mbar, sj, (-G * wd * q3).sum(0))

    # ---- L2L reverse, deepest parents first: L_c += T(d) L_p, d = c_p - c_c
    for lev in range(t.num_levels - 1, -1, -1):
        par = np.arange(lo[lev], lo[lev + 1])
        for ch in (left[par], right[par]):
            d = cen[par] - cen[ch]
            T = _op_matrices(O.l2l, p, d)
            X = np.einsum("kij,ki->kj", T, Lbar[ch])  # T^T Lbar_c
            Lbar[par] += X
            DF = np.einsum("acj,kj->akc", Dm, F[par])
            g = np.einsum("kc,akc->ka", X, DF)
            cbar[par] += g
            cbar[ch] -= g

    # ---- M2L reverse: L_t += M2L(d) M_s, d = c_t - c_s
    tgt = np.repeat(np.arange(nodes), np.diff(t.far_offsets))
    src = t.far_sources.astype(np.int64)
    C1 = (p + 2) ** 2
    D1 = ladder(p + 1)
    for a in range(0, src.size, 4096):
        s, tt = src[a:a + 4096], tgt[a:a + 4096]
        d = cen[tt] - cen[s]
        T = _op_matrices(O.m2l, p, d)
        np.add.at(Mbar, s, np.einsum("kij,ki->kj", T, Lbar[tt]))
        Mp = np.zeros((s.size, C1))
        Mp[:, :C] = M[s]
        L1 = O.m2l(p + 1, Mp, d)  # order p+1 triangular M2L
        dL = -np.einsum("acj,kj->akc", D1, L1)[:, :, :C]  # d L_n / d d_a, n <= p
        g = np.einsum("kc,akc->ka", Lbar[tt], dL)
        np.add.at(cbar, tt, g)
        np.add.at(cbar, s, -g)

    # ---- M2M reverse, root first: M_p += T(d) M_c, d = c_c - c_p
    for lev in range(t.num_levels):
        par = np.arange(lo[lev], lo[lev + 1])
        for ch in (left[par], right[par]):
            d = cen[ch] - cen[par]
            T = _op_matrices(O.m2m, p, d)
            Mbar[ch] += np.einsum("kij,ki->kj", T, Mbar[par])
            Mc = np.einsum("kij,kj->ki", T, M[ch])
            g = np.einsum("kc,acj,kj->ka", Mbar[par], np.transpose(Dm, (0, 2, 1)), Mc)
            cbar[ch] += g
            cbar[par] -= g

    # ---- P2M centre term (M_leaf = sum m U(x - c)) before the COM reverse
    y = pos - cl
    gM = _grad_phi(p, Mbar[ni + leaf_of], y)  # grad_y (Mbar . U(y))
    np.add.at(cbar, ni + leaf_of, -(mass[:, None] * gM))

    # ---- COM reverse, root first: c_p = (mu_a c_a + mu_b c_b) / mu_p
    mubar = np.zeros(nodes)
    for lev in range(t.num_levels):
        par = np.arange(lo[lev], lo[lev + 1])
        for ch in (left[par], right[par]):
            f = (mu[ch] / mu[par])[:, None]
            cbar[ch] += f * cbar[par]
            mubar[ch] += mubar[par] + ((cen[ch] - cen[par]) * cbar[par]).sum(1) / mu[par]

    # ---- leaves: P2M + leaf COM
    lid = ni + leaf_of
    Ul = _U(p, y)
    mbar += (Mbar[lid] * Ul).sum(1) + mubar[lid] + (y * cbar[lid]).sum(1) / mu[lid]
    xbar += mass[:, None] * gM + (mass / mu[lid])[:, None] * cbar[lid]
    return xbar, mbar
