"""Multi-GPU form of the pass: target-sharded, sources replicated.

One process per GPU.  The sources (positions + masses, 16 B per particle) are
replicated with one broadcast; every rank runs the cheap upward sweep on all
of them and evaluates only the target leaves of its own Morton range (M2L
restricted to the target nodes that overlap the range, L2P + P2P for its
leaves), so there is no collective inside the pass.  The sharded outputs are
combined, when the caller wants them in one place, by one all_gather of the
sorted (ax, ay, az, phi) slices.  The reference's own multi-GPU design
(spatial domain decomposition with an LET halo) is not this path.
"""

from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from .tree import Topology


def leaf_ranges(num_leaves: int, world: int) -> list[tuple[int, int]]:
    """Contiguous Morton ranges of target leaves, one per rank."""
    return [((num_leaves * r) // world, (num_leaves * (r + 1)) // world) for r in range(world)]


def particle_range(topo: Topology, leaf_lo: int, leaf_hi: int) -> tuple[int, int]:
    """[first, end) of the sorted particle slots owned by leaves [leaf_lo, leaf_hi)."""
    if leaf_hi <= leaf_lo:
        return (0, 0)
    ni = topo.num_internal
    return int(topo.node_ranges[ni + leaf_lo, 0]), int(topo.node_ranges[ni + leaf_hi - 1, 1]) + 1


def replicate_sources(positions: torch.Tensor, masses: torch.Tensor, src: int = 0, group=None) -> None:
    """Broadcasts rank `src`'s (N,3) positions and (N,) masses in place."""
    dist.broadcast(positions, src=src, group=group)
    dist.broadcast(masses, src=src, group=group)


def gather_sorted(local: torch.Tensor, topo: Topology, group=None) -> torch.Tensor:
    """All ranks' sorted output slices -> the full sorted (N, k) array on every rank.

    `local` holds this rank's rows [first, end) of its particle range (in
    sorted order); ranges come from `leaf_ranges`, so they tile [0, N)."""
    world = dist.get_world_size(group)
    ranges = [particle_range(topo, lo, hi) for lo, hi in leaf_ranges(topo.num_leaves, world)]
    width = max(e - b for b, e in ranges)
    k = local.shape[1]
    padded = torch.zeros((width, k), dtype=local.dtype, device=local.device)
    padded[: local.shape[0]] = local
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    out = torch.empty((topo.num_particles, k), dtype=local.dtype, device=local.device)
    for (b, e), part in zip(ranges, parts):
        out[b:e] = part[: e - b]
    return out
