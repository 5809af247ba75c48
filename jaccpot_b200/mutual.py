"""Momentum-conserving (mutual) evaluation: the reference's ``jaccpot.mutual``
API (mutual/__init__.py, topology.py:55-612, force.py:82-1093) on this
library's kernels.

The reference restructures its FMM for this lane -- a canonical list that
visits each node pair once, a P2P block that emits +F and -F, a dual M2L --
because its production runtime is target-centric and evaluates the two halves
of a pair independently.  Here the production pass already has the three
properties that make the total force vanish to round-off:

* the dual traversal decides every pair once and emits both directions
  (jb_tree_build / jb_tree_build_device), so A is in B's far list exactly
  when B is in A's, at the same order, and the same holds for leaf pairs;
* expansions are about the centres of mass and the multipoles are the exact
  moments of the particles (M2M loses nothing up to degree p); with the
  triangular truncation n + k <= p of the M2L, the forces on A from B and on
  B from A are the two gradients of one truncated interaction energy, so they
  cancel algebraically (measured: |sum F| / sum |F| = 1e-15 .. 1e-17 with the
  FP64 oracle for p = 2 .. 8);
* a near pair's two terms use the same distance and 1/r^3 (fl(x_j - x_i) =
  -fl(x_i - x_j), and the squared distance and rsqrt are then identical).

What would break it is a per-direction choice of order: the learned gears
pick the order per directed pair, so the mutual lane either runs at one order
or symmetrises the gears (each pair and its reverse at the higher of the two,
``gears.apply_gears(..., symmetric=True)``).  On the GPU (FP32 sums) the
residual is ~1e-9 of sum |F| for the plain and the symmetric-gear forms, and
~1e-6 with per-direction gears.

This module mirrors the reference's entry points: build_mutual_topology(...),
build_mutual_state(...), mutual_accelerations / mutual_weighted_accelerations
(with return_parts -> MutualForceResult), mutual_near_field_forces and
mutual_far_field_forces.  Forces are F = m a of the pass's accelerations; the
accelerations of massless particles are reported as zero, as the reference's
force / mass does.  The block-step form (rung, level_weights;
mutual_level_accelerations and the boundary-weight helpers) scales each pair
by its level's weight inside the kernels (jb_m2l_weighted,
jb_leaf_eval_weighted), the same weight for both directions.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, NamedTuple, Optional, Tuple

import numpy as np
import torch

from . import _lib
from .engine import DeviceTopology, Pass
from .tree import Topology


@dataclass
class MutualTopology:
    """Canonical pair lists (each pair once, ``a < b``) over a symmetric
    topology, mirroring the reference's MutualTopology (topology.py:55)."""

    num_particles: int
    num_nodes: int
    num_internal: int
    num_leaves: int
    max_leaf_size: int
    order: int
    theta: float
    left_child: np.ndarray
    right_child: np.ndarray
    leaf_nodes: np.ndarray  # int32[L], ascending node ids
    far_a: np.ndarray  # int32[num_far / 2] node ids, far_a < far_b
    far_b: np.ndarray
    near_a: np.ndarray  # int32[num_near / 2] leaf indices, near_a < near_b
    near_b: np.ndarray
    self_leaves: np.ndarray  # int32[L] leaf indices (every leaf's self block)
    topology: Topology  # the symmetric lists the pass runs on

    @property
    def forward_permutation(self) -> np.ndarray:
        return self.topology.permutation

    @property
    def inverse_permutation(self) -> np.ndarray:
        return self.topology.inverse_permutation


def build_mutual_topology_from_tree(topology: Topology, *, order: int = 4) -> MutualTopology:
    """Canonical lists of a topology whose far and near lists are symmetric
    (raises ValueError otherwise)."""
    t = topology
    if not t.near_lists_symmetric():
        raise ValueError("the mutual lane needs symmetric neighbour lists")
    tgt = t.far_pair_targets()
    src = t.far_sources
    rev = t.far_reverse_index()  # raises when a far pair has no reverse
    assert rev.shape[0] == src.shape[0]
    keep = tgt < src
    ntg = np.repeat(np.arange(t.num_leaves, dtype=np.int32), np.diff(t.near_offsets))
    nkeep = ntg < t.near_leaves
    return MutualTopology(
        num_particles=t.num_particles, num_nodes=t.num_nodes, num_internal=t.num_internal,
        num_leaves=t.num_leaves, max_leaf_size=t.max_leaf_occupancy, order=int(order), theta=t.theta,
        left_child=t.left_child, right_child=t.right_child,
        leaf_nodes=np.arange(t.num_internal, t.num_nodes, dtype=np.int32),
        far_a=tgt[keep].astype(np.int32), far_b=src[keep].astype(np.int32),
        near_a=ntg[nkeep].astype(np.int32), near_b=t.near_leaves[nkeep].astype(np.int32),
        self_leaves=np.arange(t.num_leaves, dtype=np.int32), topology=t)


def build_mutual_topology(positions, masses, *, theta: float = 0.6, order: int = 4, leaf_size: int = 16,
                          solver: Any = None) -> Tuple[MutualTopology, Any]:
    """Tree and lists from the solver's prepare (on the GPU when it runs
    there), then the canonical lists; returns (topology, prepared_state) as the
    reference's build_mutual_topology (topology.py:556) does."""
    from .solver import FastMultipoleMethod

    if solver is None:
        solver = FastMultipoleMethod(preset="balanced", basis="real", theta=theta, softening=0.0)
    state = solver.prepare_state(positions, masses, leaf_size=int(leaf_size), max_order=int(order),
                                 theta=float(theta))
    return build_mutual_topology_from_tree(state.topology, order=order), state


@dataclass
class MutualFMMState:
    """Device-resident state of one mutual evaluation (force.py:282 there)."""

    topology: MutualTopology
    device_topology: DeviceTopology
    pass_: Pass
    softening: float
    G: float

    @property
    def forward_permutation(self) -> np.ndarray:
        return self.topology.forward_permutation

    @property
    def inverse_permutation(self) -> np.ndarray:
        return self.topology.inverse_permutation


def build_mutual_state(topology: MutualTopology, *, softening: float, G: float = 1.0, use_pallas: bool = False,
                       near_chunk_size: Optional[int] = None, pallas_interpret: bool = False,
                       index_dtype: Any = None, caps: Any = None, device="cuda",
                       nearfield_compensated: bool = True) -> MutualFMMState:
    """Moves the topology to the device and sets up the pass at the
    topology's order (force.py:450 there).  use_pallas / pallas_interpret /
    near_chunk_size / index_dtype / caps concern the reference's JAX lanes;
    use_pallas=True is refused, the others are accepted and ignored."""
    if use_pallas:
        raise ValueError("use_pallas is not available: the kernels are native sm_100a CUDA")
    dt = DeviceTopology(topology.topology, device)
    dt.validate()
    ps = Pass(dt, topology.order, G=float(G), eps2=float(softening) ** 2, m2l_mode=_lib.JB_M2L_FP32,
              p2p_mode=_lib.JB_P2P_KAHAN if nearfield_compensated else _lib.JB_P2P_FP32)
    return MutualFMMState(topology, dt, ps, float(softening), float(G))


class MutualForceResult(NamedTuple):
    """Accelerations plus the near / far force split (force.py:82 there)."""

    accelerations: Any
    near_forces: Any
    far_forces: Any


def _unsort(sorted_rows: torch.Tensor, perm: torch.Tensor) -> torch.Tensor:
    out = torch.empty_like(sorted_rows)
    out[perm] = sorted_rows
    return out


def _node_rungs(dt: DeviceTopology, rung_sorted: torch.Tensor) -> torch.Tensor:
    """Rung of every node: the finest (largest) rung of its particles, leaves
    first, then up the levels (force.py:885 _cell_rungs there)."""
    t = dt.topo
    node = torch.full((t.num_nodes,), -1, dtype=torch.int32, device=rung_sorted.device)
    leaf = torch.full((t.num_leaves,), -1, dtype=torch.int32, device=rung_sorted.device)
    leaf = leaf.scatter_reduce(0, dt.leaf_of.long(), rung_sorted, reduce="amax", include_self=True)
    node[t.num_internal:] = leaf
    left, right, lo = dt.left.long(), dt.right.long(), dt.level_offsets
    for lev in range(t.num_levels - 1, -1, -1):
        a, b = lo[lev], lo[lev + 1]
        if b > a:
            node[a:b] = torch.maximum(node[left[a:b]], node[right[a:b]])
    return node


def _far_pair_weights(dt: DeviceTopology, node_rung: torch.Tensor, lw: torch.Tensor) -> torch.Tensor:
    """Weight of every directed far entry: lw[max(rung_a, rung_b)], the same
    for both directions of a pair (force.py:920 there)."""
    t = dt.topo
    counts = (dt.far_off[1:] - dt.far_off[:-1]).long()
    tgt = torch.repeat_interleave(torch.arange(t.num_nodes, device=lw.device), counts)
    src = dt.far_src[: t.num_far_pairs].long()
    lev = torch.maximum(node_rung[tgt], node_rung[src]).clamp(0, lw.numel() - 1).long()
    return lw[lev]


def mutual_weighted_accelerations(state: MutualFMMState, positions, masses, *, rung=None, level_weights=None,
                                  return_parts: bool = False):
    """sum_k level_weights[k] * a_k in one traversal (force.py:985 there):
    a pair belongs to the level of its finer endpoint -- max(rung_i, rung_j)
    for particles, the nodes' finest rungs for a far pair -- and is scaled by
    that level's weight, the same for both directions, so momentum stays
    conserved for any weights.  Without rung / level_weights this is the full
    acceleration.  return_parts adds the near and far forces.  Arrays come
    back as the inputs' kind (numpy in, numpy out)."""
    if (rung is None) != (level_weights is None):
        raise ValueError("rung and level_weights go together")
    ps = state.pass_
    dt = state.device_topology
    dev = dt.device
    want_np = not isinstance(positions, torch.Tensor)
    pos = torch.as_tensor(positions).to(device=dev, dtype=torch.float32)
    mass = torch.as_tensor(masses).to(device=dev, dtype=torch.float32)
    perm = dt.perm
    ps.load_particles(pos, mass)
    ps.upward()
    if rung is None:
        ps.m2l()
        ps.l2l()
        ev = lambda part=None: ps.evaluate(part=part)
    else:
        lw = torch.as_tensor(np.asarray(level_weights, dtype=np.float32) if not isinstance(level_weights, torch.Tensor)
                             else level_weights).to(device=dev, dtype=torch.float32).reshape(-1)
        if not 1 <= lw.numel() <= 32:
            raise ValueError("between 1 and 32 level weights")
        r_sorted = torch.as_tensor(rung).to(device=dev, dtype=torch.int32).reshape(-1)[perm].contiguous()
        ps.m2l_weighted(_far_pair_weights(dt, _node_rungs(dt, r_sorted), lw))
        ps.l2l()
        ev = lambda part=None: ps.evaluate_weighted(r_sorted, lw, part=part)
    m_sorted = mass[perm]
    if return_parts:
        near_a = ev("near")[:, :3].clone()
        far_a = ev("far")[:, :3].clone()
        acc = near_a + far_a
    else:
        acc = ev()[:, :3].clone()
    acc = torch.where(m_sorted[:, None] > 0, acc, torch.zeros_like(acc))
    out = _unsort(acc, perm)
    if not return_parts:
        return out.cpu().numpy() if want_np else out
    near_f = _unsort(m_sorted[:, None] * near_a, perm)
    far_f = _unsort(m_sorted[:, None] * far_a, perm)
    if want_np:
        return MutualForceResult(out.cpu().numpy(), near_f.cpu().numpy(), far_f.cpu().numpy())
    return MutualForceResult(out, near_f, far_f)


def mutual_accelerations(state: MutualFMMState, positions, masses, **kwargs):
    """mutual_weighted_accelerations with unit weights (force.py:1071 there)."""
    return mutual_weighted_accelerations(state, positions, masses, **kwargs)


def mutual_level_accelerations(state: MutualFMMState, positions, masses, *, rung, level: int, k_max: int):
    """The accelerations of the level-``level`` interactions alone
    (force.py:1096 there); summed over levels 0 .. k_max they give the full
    acceleration."""
    w = np.zeros(int(k_max) + 1, dtype=np.float32)
    w[int(level)] = 1.0
    return mutual_weighted_accelerations(state, positions, masses, rung=rung, level_weights=w)


# Block-step bookkeeping (force.py:685-883 there): 2**k_max sub-steps per base
# step; boundary s kicks the levels at or above its floor.
def n_sub(k_max: int) -> int:
    return 1 << int(k_max)


def is_sync_boundary(s: int, k_max: int) -> bool:
    return int(s) == 0 or int(s) == (1 << int(k_max))


def active_level_floor(s: int, k_max: int) -> int:
    s, k_max = int(s), int(k_max)
    if is_sync_boundary(s, k_max):
        return 0
    return k_max - ((s & -s).bit_length() - 1)


def level_weights_from_floor(active_floor: int, k_max: int, dt_max: float, *, half: float = 1.0,
                             dtype=np.float64) -> np.ndarray:
    """Level k is kicked with half * dt_max / 2**k; levels below the floor get 0."""
    return np.asarray([(float(half) * float(dt_max) / float(1 << k)) if k >= int(active_floor) else 0.0
                       for k in range(int(k_max) + 1)], dtype=dtype)


def boundary_level_weights(s: int, k_max: int, dt_max: float, *, dtype=np.float64) -> np.ndarray:
    """The kick weights at boundary s: half = 0.5 at the synchronised ends."""
    return level_weights_from_floor(active_level_floor(s, k_max), k_max, dt_max,
                                    half=0.5 if is_sync_boundary(s, k_max) else 1.0, dtype=dtype)


def boundary_weight_table(k_max: int, dt_max: float, *, dtype=np.float64) -> np.ndarray:
    """Row s = boundary_level_weights(s, ...), s = 0 .. 2**k_max."""
    return np.stack([boundary_level_weights(s, k_max, dt_max, dtype=dtype) for s in range(n_sub(k_max) + 1)])


def mutual_near_field_forces(state: MutualFMMState, positions, masses):
    """The P2P part of the mutual force, F = m a_near, caller's order."""
    return mutual_weighted_accelerations(state, positions, masses, return_parts=True).near_forces


def mutual_far_field_forces(state: MutualFMMState, positions, masses):
    """The multipole part of the mutual force, F = m a_far, caller's order."""
    return mutual_weighted_accelerations(state, positions, masses, return_parts=True).far_forces


def momentum_residual(forces) -> float:
    """max over axes of |sum_i F_i| / sum_i |F_i| (float64 sums)."""
    f = forces.double().cpu().numpy() if isinstance(forces, torch.Tensor) else np.asarray(forces, np.float64)
    return float((np.abs(f.sum(0)) / np.maximum(np.abs(f).sum(0), 1e-300)).max())
