"""Error-controlled acceptance with per-pair expansion orders.

The reference's adaptive lane (``adaptive_error_model="dehnen_paper"``,
``adaptive_eps``, ``mac_theta_max``; runtime/_adaptive_policy.py:2216-2376
``adaptive_pair_policy`` with the eq. (15) estimate of :267-376) decides
during the traversal whether a node pair is accepted, and at which of
``p_gears``, from the source's per-degree multipole power and the target's
force scale -- instead of a fixed opening angle.  Here that traversal runs on
the GPU (``jb_dtree_adaptive_walk``), target-centric: each ordered pair
(t <- s) is decided from its own estimate, so a pair may be far for one node
and refined for the other.  (The reference's traversal is mutual and needs
both orientations to agree, which it enforces by taking the stricter one.)

Prepare: the tree and a theta walk (``theta_prepass``), a prepass evaluation
at the top gear on it (its accelerations give the per-node force scale, the
smallest |a| under each node -- the "min" reduction the reference switches to
with dehnen_paper, _adaptive_policy.py:402; its multipoles give Dehnen's
per-degree powers), then the error-controlled walk on the same tree.  The
returned pass runs every far pair at its gear (``Pass.set_gears``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _lib, engine, tree


def _ptr(t):
    return None if t is None else t.data_ptr()


@dataclass
class AdaptivePrepared:
    topology: tree.Topology
    device_topology: engine.DeviceTopology
    pass_: engine.Pass
    orders: tuple
    eps: float
    theta_max: float
    prepass_far_pairs: int
    prepass_near_interactions: int


def node_force_scale(ps: engine.Pass, acc4: torch.Tensor | None = None) -> torch.Tensor:
    """float32 (num_nodes,): the smallest |a| over each node's particles, from
    the pass's sorted acc4 (or `acc4`)."""
    t, dt = ps.dt.topo, ps.dt
    out = torch.empty(t.num_nodes, device=dt.device, dtype=torch.float32)
    lo = np.ascontiguousarray(np.asarray(t.level_offsets, dtype=np.int32))
    a4 = ps.ws.acc4 if acc4 is None else acc4
    _lib.check(_lib.lib().jb_node_force_scale(t.num_nodes, t.num_internal, _ptr(dt.left), _ptr(dt.right),
                                              lo.ctypes.data, t.num_levels, _ptr(dt.node_ranges), _ptr(a4),
                                              _ptr(out), torch.cuda.current_stream(dt.device).cuda_stream),
               "jb_node_force_scale")
    return out


def node_dehnen_power(ps: engine.Pass, p: int | None = None) -> torch.Tensor:
    """float64 (num_nodes, p+1): Dehnen's per-degree power of the multipoles
    in the pass's workspace."""
    p = ps.p if p is None else int(p)
    t = ps.dt.topo
    out = torch.empty((t.num_nodes, p + 1), device=ps.dt.device, dtype=torch.float64)
    _lib.check(_lib.lib().jb_node_dehnen_power(p, t.num_nodes, _ptr(ps.ws.mult), ps.ws.stride, _ptr(out),
                                               torch.cuda.current_stream(ps.dt.device).cuda_stream),
               "jb_node_dehnen_power")
    return out


def prepare(positions, masses, *, leaf_size: int, orders, eps: float, theta_max: float = 1.0,
            theta_prepass: float = 0.6, G: float = 1.0, eps2: float = 0.0, device="cuda",
            m2l_mode: int = _lib.JB_M2L_FP32, p2p_mode: int = _lib.JB_P2P_FP32,
            force_scale: torch.Tensor | None = None, **pass_kw) -> AdaptivePrepared:
    """Tree, force-scale prepass, error-controlled walk and the gear pass.

    orders: ascending expansion orders (the gears); the pass runs at the
    highest.  force_scale: optional per-particle |a| (input order, device)
    from an earlier evaluation, which replaces the prepass's."""
    orders = tuple(int(o) for o in orders)
    if not orders or list(orders) != sorted(set(orders)) or orders[0] < 1 or orders[-1] > _lib.JB_MAX_ORDER:
        raise ValueError(f"gear orders must be ascending in [1, {_lib.JB_MAX_ORDER}], got {orders}")
    if not (eps > 0):
        raise ValueError("eps (the relative force-accuracy target) must be > 0")
    if not (0.0 < theta_max <= 1.0):
        raise ValueError("theta_max must be in (0, 1]")
    dev = torch.device(device)
    pos = torch.as_tensor(positions).to(dev)
    mass = torch.as_tensor(masses).to(dev)
    p_top = orders[-1]
    with tree.DeviceTree(pos, mass, leaf_size=leaf_size, theta=theta_prepass, device=dev) as dtree:
        topo0 = dtree.topology()
        dt0 = engine.DeviceTopology(topo0, dev)
        dt0.validate()
        pre = engine.Pass(dt0, p_top, G=G, eps2=eps2)
        pre.load_particles(pos.float(), mass.float())
        if force_scale is None:
            pre.run()
            acc4 = None
        else:  # an earlier evaluation's |a| (input order) -> sorted slots
            pre.upward()
            a = force_scale.to(device=dev, dtype=torch.float32).reshape(-1)
            acc4 = torch.zeros((topo0.num_particles, 4), device=dev, dtype=torch.float32)
            acc4[:, 0] = a[dt0.perm]
        fscale = node_force_scale(pre, acc4)
        power = node_dehnen_power(pre)
        pre_far, pre_near = topo0.num_far_pairs, topo0.near_pair_interactions()
        del pre, dt0
        dtree.adaptive_walk(power, fscale, G=G, eps=eps, theta_max=theta_max, gear_orders=orders)
        topo = dtree.topology()
    dt = engine.DeviceTopology(topo, dev)
    dt.validate()
    ps = engine.Pass(dt, p_top, G=G, eps2=eps2, m2l_mode=m2l_mode, p2p_mode=p2p_mode, **pass_kw)
    if len(orders) > 1 and topo.num_far_pairs:
        ps.set_gears(torch.from_numpy(topo.far_gears).to(dev), orders)
    return AdaptivePrepared(topology=topo, device_topology=dt, pass_=ps, orders=orders, eps=float(eps),
                            theta_max=float(theta_max), prepass_far_pairs=pre_far,
                            prepass_near_interactions=pre_near)
