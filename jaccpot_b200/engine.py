"""Device-side evaluation pass: uploads a topology once, then runs
P2M -> M2M (by level) -> M2L -> L2L (by level) -> L2P + P2P on one stream.

This is the B200 replacement for the reference engine's sweep/evaluate seam
(jaccpot/runtime/fmm_sweeps.py:221 prepare_upward_sweep, :442
prepare_downward_sweep, runtime/kernels/_evaluate.py:769
_evaluate_tree_compiled_impl).  Torch provides device memory and streams
only; every arithmetic step is a kernel of libjaccpot_b200.so.
"""

from __future__ import annotations

import copy
import ctypes
import dataclasses

from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .schedule import (MixedGearM2LSchedule, gear_m2l_mixed_schedule, gear_m2l_mixed_schedule_device,
                       gear_m2l_schedule, gear_m2l_schedule_device, leaf_schedule, leaf_schedule_device,
                       m2l_schedule, m2l_schedule_device, mixed_ladder, tc_m2l_schedule)
from .tree import Topology


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def _zero(t: torch.Tensor, stream: torch.cuda.Stream | None) -> None:
    """t.zero_() on `stream` (default: torch's current stream), in order with
    the kernels a stage enqueues there."""
    if stream is None:
        t.zero_()
    else:
        with torch.cuda.stream(stream):
            t.zero_()


def _stream_handle(stream: torch.cuda.Stream | None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


class DeviceTopology:
    """The topology arrays resident in HBM (int32 ids, int64 CSR offsets)."""

    def __init__(self, topo: Topology, device: torch.device | str = "cuda"):
        dev = torch.device(device)
        if dev.type != "cuda":
            raise ValueError("DeviceTopology needs a CUDA device (there is no CPU path)")
        self.topo = topo
        self.device = dev
        up = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(device=dev, dtype=dt)
        self.node_ranges = up(topo.node_ranges.reshape(-1), torch.int32)
        self.left = up(topo.left_child if topo.num_internal else np.zeros(1, np.int32), torch.int32)
        self.right = up(topo.right_child if topo.num_internal else np.zeros(1, np.int32), torch.int32)
        self.far_off = up(topo.far_offsets, torch.int64)
        self.far_src = up(topo.far_sources if topo.num_far_pairs else np.zeros(1, np.int32), torch.int32)
        # per-far-pair gear tags of an error-controlled walk (None: one order)
        self.far_gear = None
        self.near_off = up(topo.near_offsets, torch.int64)
        self.near_src = up(topo.near_leaves if topo.num_near_pairs else np.zeros(1, np.int32), torch.int32)
        self.leaf_of = up(topo.leaf_of_particle, torch.int32)
        self.perm = up(topo.permutation, torch.int64)
        self.inv_perm = up(topo.inverse_permutation, torch.int64)
        self.m2l_targets = up(topo.m2l_targets if topo.m2l_targets.size else np.zeros(1, np.int32), torch.int32)
        self.num_m2l_targets = int(topo.m2l_targets.size)
        self.level_offsets = [int(x) for x in topo.level_offsets]
        # the L2L levels above the shallowest internal far target move zeros
        # (every local there is zero): the sweep starts at that level
        ni = topo.num_internal
        tgt = np.nonzero(np.diff(np.asarray(topo.far_offsets))[:ni] > 0)[0]
        self.l2l_first_level = int(np.asarray(topo.node_level)[tgt].min()) if tgt.size else int(topo.num_levels)

    def far_reverse_index(self) -> torch.Tensor:
        """int32[num_far] on the device: the reverse pair (s <- t) of every far
        pair (t <- s) (jb_far_reverse_index; computed once)."""
        rev = getattr(self, "_far_rev", None)
        if rev is None:
            n = self.topo.num_far_pairs
            rev = torch.empty(max(n, 1), dtype=torch.int32, device=self.device)
            _lib.check(_lib.lib().jb_far_reverse_index(self.topo.num_nodes, self.far_off.data_ptr(),
                                                       self.far_src.data_ptr(), rev.data_ptr(),
                                                       torch.cuda.current_stream(self.device).cuda_stream),
                       "jb_far_reverse_index")
            rev = rev[:n]
            self._far_rev = rev
        return rev

    def validate(self) -> None:
        """Device-side range check of every list entry (jb_validate_lists)."""
        t = self.topo
        bad = torch.zeros(1, dtype=torch.int32, device=self.device)
        _lib.check(_lib.lib().jb_validate_lists(
            t.num_nodes, t.num_internal, _ptr(self.left), _ptr(self.right), _ptr(self.far_off),
            _ptr(self.far_src), t.num_far_pairs, _ptr(self.near_off), _ptr(self.near_src),
            t.num_near_pairs, _ptr(bad), _stream_handle(None)), "jb_validate_lists")
        nbad = int(bad.item())
        if nbad:
            raise _lib.JBError(f"topology has {nbad} out-of-range list entries")
        _lib.check(_lib.lib().jb_validate_leaves(t.num_nodes, t.num_internal, _ptr(self.node_ranges),
                                                 _lib.JB_MAX_LEAF_OCCUPANCY, _ptr(bad), _stream_handle(None)),
                   "jb_validate_leaves")
        nbad = int(bad.item())
        if nbad:
            raise _lib.JBError(f"{nbad} leaves hold more than {_lib.JB_MAX_LEAF_OCCUPANCY} particles "
                               f"(or none): the leaf kernels take leaf_size <= {_lib.JB_MAX_LEAF_OCCUPANCY}")


@dataclass
class Workspace:
    p: int
    stride: int
    pos4: torch.Tensor  # (N, 4) sorted particles
    centers: torch.Tensor  # (nodes, 4)
    mult: torch.Tensor  # (nodes, stride)
    locals: torch.Tensor  # (nodes, stride)
    acc4: torch.Tensor  # (N, 4)

    @staticmethod
    def allocate(dt: DeviceTopology, p: int) -> "Workspace":
        t = dt.topo
        cs = _lib.coeff_stride(p)
        kw = dict(device=dt.device, dtype=torch.float32)
        return Workspace(
            p=p,
            stride=cs,
            pos4=torch.empty((t.num_particles, 4), **kw),
            centers=torch.empty((t.num_nodes, 4), **kw),
            mult=torch.empty((t.num_nodes, cs), **kw),
            locals=torch.empty((t.num_nodes, cs), **kw),
            acc4=torch.empty((t.num_particles, 4), **kw),
        )


def _up(a, dev) -> torch.Tensor:
    """Schedule array on the device (a dummy row when empty, so the pointer
    handed to the library is never null)."""
    if torch.is_tensor(a):
        return a if a.numel() else torch.zeros(4, dtype=torch.int32, device=dev)
    return torch.from_numpy(a if a.size else np.zeros(4, np.int32)).to(dev)


def _on_gpu(dt) -> bool:
    return torch.device(dt.device).type == "cuda"


def l2l_leaf_schedule(topo: Topology, leaf_range: tuple[int, int]):
    """Work units of jb_l2l_leaves for the leaves [lo, hi): (units int32[U,4]
    = (leaf node, first, end, -1), anc int32[...]) where anc[first:end] are the
    leaf's ancestors that received far pairs, nearest first; leaves without
    any are left out; units ordered by their length, longest first (a warp's
    lanes step through their lists together)."""
    ni = topo.num_internal
    lo, hi = leaf_range
    leaves = np.arange(ni + lo, ni + hi, dtype=np.int64)
    has_far = np.diff(np.asarray(topo.far_offsets)) > 0
    parent = np.asarray(topo.parent).astype(np.int64)
    rows, cols = [], []
    idx = np.arange(leaves.size, dtype=np.int64)
    cur = parent[leaves] if leaves.size else leaves
    while cur.size:
        ok = cur >= 0
        idx, cur = idx[ok], cur[ok]
        m = has_far[cur]
        rows.append(idx[m])
        cols.append(cur[m])
        cur = parent[cur]
    rows = np.concatenate(rows) if rows else np.zeros(0, np.int64)
    cols = np.concatenate(cols) if cols else np.zeros(0, np.int64)
    order = np.argsort(rows, kind="stable")  # nearest ancestor first within a leaf
    rows, cols = rows[order], cols[order]
    cnt = np.bincount(rows, minlength=leaves.size)
    off = np.concatenate([[0], np.cumsum(cnt)])
    have = np.nonzero(cnt)[0]
    have = have[np.argsort(-cnt[have], kind="stable")]
    units = np.stack([leaves[have], off[have], off[have + 1], np.full(have.size, -1)], axis=1).astype(np.int32)
    anc = cols.astype(np.int32) if cols.size else np.zeros(1, np.int32)
    return np.ascontiguousarray(units.reshape(-1, 4)), np.ascontiguousarray(anc)


def l2l_leaf_schedule_device(dt: "DeviceTopology", leaf_range: tuple[int, int]):
    """l2l_leaf_schedule on the device (torch operations over the resident
    far offsets and the uploaded parents): the same arrays, as device
    tensors."""
    t, dev = dt.topo, dt.device
    ni = t.num_internal
    lo, hi = leaf_range
    parent = torch.from_numpy(np.asarray(t.parent).astype(np.int64)).to(dev)
    has_far = (dt.far_off[1:] - dt.far_off[:-1]) > 0
    leaves = torch.arange(ni + lo, ni + hi, device=dev, dtype=torch.int64)
    idx = torch.arange(leaves.numel(), device=dev, dtype=torch.int64)
    cur = parent[leaves]
    rows, cols = [], []
    while cur.numel():
        ok = cur >= 0
        idx, cur = idx[ok], cur[ok]
        m = has_far[cur]
        rows.append(idx[m])
        cols.append(cur[m])
        cur = parent[cur]
    z = torch.zeros(0, dtype=torch.int64, device=dev)
    rows = torch.cat(rows) if rows else z
    cols = torch.cat(cols) if cols else z
    order = torch.sort(rows, stable=True).indices  # nearest ancestor first within a leaf
    rows, cols = rows[order], cols[order]
    cnt = torch.bincount(rows, minlength=leaves.numel())
    off = torch.cat([torch.zeros(1, dtype=torch.int64, device=dev), torch.cumsum(cnt, 0)])
    have = torch.nonzero(cnt).flatten()
    have = have[torch.sort(-cnt[have], stable=True).indices]
    units = torch.stack([leaves[have], off[have], off[have + 1], torch.full_like(have, -1)], dim=1)
    return units.to(torch.int32).contiguous(), cols.to(torch.int32).contiguous()


def _restrict_gears(gs, targets, num_nodes: int, dev):
    """The gear schedule's units and split entries of the given target nodes
    only (a leaf range's M2L), the per-gear unit ranges recounted.  Units keep
    their order and slots, so every kept target gets exactly the rows it has
    in the full schedule."""
    from .schedule import GearM2LSchedule

    units = torch.as_tensor(gs.units).to(dev)
    split = torch.as_tensor(gs.split).to(dev)
    offs = torch.as_tensor(np.asarray(gs.gear_offsets, dtype=np.int64)).to(dev)
    keep = torch.zeros(num_nodes, dtype=torch.bool, device=dev)
    keep[torch.as_tensor(np.asarray(targets, dtype=np.int64)).to(dev)] = True
    ng = int(offs.numel()) - 1
    if units.shape[0]:
        gear_of = torch.bucketize(torch.arange(units.shape[0], device=dev), offs[1:], right=True)
        mask = keep[units[:, 0].long()]
        units = units[mask].contiguous()
        counts = torch.bincount(gear_of[mask], minlength=ng)
    else:
        counts = torch.zeros(ng, dtype=torch.int64, device=dev)
    new_offs = torch.zeros(ng + 1, dtype=torch.int64)
    new_offs[1:] = torch.cumsum(counts.cpu(), 0)
    if split.shape[0]:
        split = split[keep[split[:, 0].long()]].contiguous()
    return GearM2LSchedule(units, split, gs.num_slots, gs.far_src, new_offs.numpy(), gs.orders, gs.pairs_per_gear)


def _restrict_mixed(gs, targets, num_nodes: int, dev):
    """The mixed gear schedule's units (with their bounds) and split entries
    of the given target nodes only; units keep their order and slots."""
    units = torch.as_tensor(gs.units).to(dev)
    bounds = torch.as_tensor(gs.bounds).to(dev)
    split = torch.as_tensor(gs.split).to(dev)
    keep = torch.zeros(num_nodes, dtype=torch.bool, device=dev)
    keep[torch.as_tensor(np.asarray(targets, dtype=np.int64)).to(dev)] = True
    if units.shape[0]:
        mask = keep[units[:, 0].long()]
        units, bounds = units[mask].contiguous(), bounds[mask].contiguous()
    if split.shape[0]:
        split = split[keep[split[:, 0].long()]].contiguous()
    return dataclasses.replace(gs, units=units, bounds=bounds, split=split)


class PassGraph:
    """A captured pass instantiated by the library with per-node priorities
    (jb_graph_instantiate), so the far-field chain captured on a
    high-priority stream keeps its priority on replay.  replay() launches it
    on torch's current stream, as torch.cuda.CUDAGraph.replay does; the torch
    graph is kept for its memory pool and captured graph."""

    def __init__(self, graph: torch.cuda.CUDAGraph, lib):
        self.graph, self.lib = graph, lib
        ex = ctypes.c_void_p()
        _lib.check(lib.jb_graph_instantiate(ctypes.c_void_p(graph.raw_cuda_graph()), 1, ctypes.byref(ex)),
                   "jb_graph_instantiate")
        self.exec = ex

    def replay(self) -> None:
        _lib.check(self.lib.jb_graph_launch(self.exec, _stream_handle(None)), "jb_graph_launch")

    def reset(self) -> None:
        if self.exec:
            _lib.check(self.lib.jb_graph_exec_destroy(self.exec), "jb_graph_exec_destroy")
            self.exec = ctypes.c_void_p()
        self.graph.reset()

    def __del__(self):
        try:
            if self.exec:
                self.lib.jb_graph_exec_destroy(self.exec)
        except Exception:
            pass


class Pass:
    """One evaluation pass over a resident topology; every method enqueues
    kernels on `stream` (default: torch's current stream) and returns."""

    def __init__(self, dt: DeviceTopology, p: int, *, G: float = 1.0, eps2: float = 0.0,
                 m2l_mode: int = _lib.JB_M2L_FP32, p2p_mode: int = _lib.JB_P2P_FP32,
                 leaf_range: tuple[int, int] | None = None, m2l_unit_pairs: int | None = None,
                 leaf_unit_sources: int = 4096, gear_unit_pairs: int = 128, gear_form: str = "mixed"):
        if not (1 <= int(p) <= _lib.JB_MAX_ORDER):
            raise ValueError(f"max_order must be in [1, {_lib.JB_MAX_ORDER}], got {p}")
        if dt.topo.max_leaf_occupancy > _lib.JB_MAX_LEAF_OCCUPANCY:
            raise ValueError(f"the leaf kernels take at most {_lib.JB_MAX_LEAF_OCCUPANCY} particles per leaf "
                             f"(use leaf_size <= {_lib.JB_MAX_LEAF_OCCUPANCY})")
        self.dt = dt
        self.p = int(p)
        self.G = float(G)
        self.eps2 = float(eps2)
        self.m2l_mode = int(m2l_mode)
        # split-BF16 M2L layout: "units" (thread per work unit, K on the tensor
        # cores), or "tiles" (128 consecutive pairs per tile) with tc_products
        # 1 (K on the tensor cores) or 3 (B, K and B^T)
        self.tc_layout = "units"
        self.tc_products = 1
        self.p2p_mode = int(p2p_mode)
        # work-unit sizes (pairs per M2L unit, per gear unit; sources per leaf
        # unit), measured at clustered N=4M, p=8
        self.gear_unit_pairs = int(gear_unit_pairs)
        # per-pair gears: "mixed" (one launch, jb_m2l_mixed) when the orders lie
        # on mixed_ladder(p), else (or "per_gear") one launch per gear
        if gear_form not in ("mixed", "per_gear"):
            raise ValueError(f"gear_form must be 'mixed' or 'per_gear', got {gear_form!r}")
        self.gear_form = gear_form
        if m2l_unit_pairs is None:  # the tensor-core form steps a group's units together: shorter units
            m2l_unit_pairs = 64 if self.m2l_mode == _lib.JB_M2L_SPLIT_BF16 else 512
        self.m2l_unit_pairs = int(m2l_unit_pairs)
        self.leaf_unit_sources = int(leaf_unit_sources)
        self.ws = Workspace.allocate(dt, self.p)
        self.lib = _lib.lib()
        t = dt.topo
        self.leaf_range = (0, t.num_leaves) if leaf_range is None else (int(leaf_range[0]), int(leaf_range[1]))
        targets = None
        if self.leaf_range != (0, t.num_leaves):
            # only nodes whose particle span meets this leaf range need locals
            lo = int(t.node_ranges[t.num_internal + self.leaf_range[0], 0])
            hi = int(t.node_ranges[t.num_internal + self.leaf_range[1] - 1, 1])
            tg = t.m2l_targets
            targets = tg[(t.node_ranges[tg, 1] >= lo) & (t.node_ranges[tg, 0] <= hi)]
        self._range_targets = targets
        # work-unit schedules: built on the GPU from the resident lists when
        # the pass runs there (the host builders give the same arrays)
        if _on_gpu(dt):
            self.m2l_sched = m2l_schedule_device(dt, max_pairs=self.m2l_unit_pairs, targets=targets)
            self.leaf_sched = leaf_schedule_device(dt, max_sources=leaf_unit_sources, leaf_range=self.leaf_range)
        else:
            self.m2l_sched = m2l_schedule(t, max_pairs=self.m2l_unit_pairs, targets=targets)
            self.leaf_sched = leaf_schedule(t, max_sources=leaf_unit_sources, leaf_range=self.leaf_range)
        dev = dt.device
        up = lambda a: _up(a, dev)
        self.d_m2l_units = up(self.m2l_sched.units)
        self.d_m2l_split = up(self.m2l_sched.split)
        self.m2l_partials = torch.empty((max(self.m2l_sched.num_slots, 1), self.ws.stride), device=dev,
                                        dtype=torch.float32)
        self.d_leaf_units = up(self.leaf_sched.units)
        self.d_leaf_aux = up(self.leaf_sched.aux)
        self.d_leaf_runs = up(self.leaf_sched.runs)
        self.d_leaf_split = up(self.leaf_sched.split)
        self.leaf_partials = torch.empty((max(self.leaf_sched.num_slots, 1) * _lib.JB_MAX_LEAF_OCCUPANCY, 4), device=dev, dtype=torch.float32)
        # the downward sweep straight to this pass's leaves (jb_l2l_leaves) at
        # orders <= 8; l2l(cascade=True), and orders 9-10 (where the direct
        # chain measured slower: 1.07 against 0.88 ms at 4M), run it level by level
        self.l2l_direct = self.p <= 8
        if _on_gpu(dt):
            units, anc = l2l_leaf_schedule_device(dt, self.leaf_range)
        else:
            units, anc = l2l_leaf_schedule(t, self.leaf_range)
        self.num_l2l_units = int(units.shape[0])
        self.d_l2l_units = up(units)
        self.d_l2l_anc = up(anc)
        # run(): the near field on the caller's stream while the upward sweep,
        # M2L and L2L run on a high-priority stream of the pass (same bits)
        self.overlap = True

    def fork(self) -> "Pass":
        """A pass over the same topology and work-unit schedules (shared,
        read-only) with its own workspace and scratch rows, so the two can run
        side by side; lazily built tensor-core and adjoint state is rebuilt on
        first use."""
        q = copy.copy(self)
        q.ws = Workspace.allocate(self.dt, self.p)
        q.m2l_partials = torch.empty_like(self.m2l_partials)
        q.leaf_partials = torch.empty_like(self.leaf_partials)
        if getattr(self, "gear_sched", None) is not None:
            q.gear_partials = torch.empty_like(self.gear_partials)
        for name in ("_tc", "_tc_status", "_adj", "_adj_sched", "_adj_m2l", "_far_stream"):
            q.__dict__.pop(name, None)
        return q

    # -- stages -------------------------------------------------------------
    def load_particles(self, positions: torch.Tensor, masses: torch.Tensor, stream=None) -> None:
        """Morton-order gather of (N,3) positions and (N,) masses (device)."""
        n = self.dt.topo.num_particles
        pos = positions.to(device=self.dt.device, dtype=torch.float32).contiguous()
        mass = masses.to(device=self.dt.device, dtype=torch.float32).contiguous()
        if pos.shape != (n, 3) or mass.shape != (n,):
            raise ValueError("positions must be (N,3) and masses (N,) matching the prepared topology")
        _lib.check(self.lib.jb_gather_sorted(n, _ptr(pos), _ptr(mass), _ptr(self.dt.perm),
                                             _ptr(self.ws.pos4), _stream_handle(stream)), "jb_gather_sorted")

    def upward(self, stream=None) -> None:
        t, dt, ws, s = self.dt.topo, self.dt, self.ws, _stream_handle(stream)
        _lib.check(self.lib.jb_p2m(self.p, _ptr(ws.pos4), t.num_nodes, t.num_internal, _ptr(dt.node_ranges),
                                   _ptr(ws.centers), _ptr(ws.mult), s), "jb_p2m")
        lo = dt.level_offsets
        for lev in range(t.num_levels - 1, -1, -1):
            _lib.check(self.lib.jb_m2m_level(self.p, lo[lev], lo[lev + 1], _ptr(dt.left), _ptr(dt.right),
                                             _ptr(dt.node_ranges), _ptr(ws.centers), _ptr(ws.mult), s),
                       "jb_m2m_level")

    def set_gears(self, gears, orders) -> None:
        """Per-far-pair expansion orders: gears[e] indexes `orders` for pair e
        of the CSR far list (None restores the single maximum order)."""
        if gears is None:
            self.gear_sched = None
            return
        orders = tuple(int(o) for o in orders)
        if max(orders) > self.p or min(orders) < 1:
            raise ValueError(f"gear orders must lie in [1, {self.p}]")
        dev = self.dt.device
        up = lambda a: _up(a, dev)
        if (self.gear_form == "mixed" and self.m2l_mode == _lib.JB_M2L_FP32
                and all(o in mixed_ladder(self.p) for o in orders)):
            if _on_gpu(self.dt):
                gs = gear_m2l_mixed_schedule_device(self.dt, gears, orders, self.p, max_pairs=self.gear_unit_pairs)
            else:
                gs = gear_m2l_mixed_schedule(self.dt.topo, np.asarray(gears), orders, self.p,
                                             max_pairs=self.gear_unit_pairs)
            if getattr(self, "_range_targets", None) is not None:
                gs = _restrict_mixed(gs, self._range_targets, self.dt.topo.num_nodes, dev)
            self.gear_sched = gs
            self.d_gear_units = up(gs.units)
            self.d_gear_bounds = up(gs.bounds)
            self.d_gear_split = up(gs.split)
            self.d_gear_src = up(gs.far_src)
            self.gear_partials = torch.empty((max(gs.num_slots, 1), self.ws.stride), device=dev, dtype=torch.float32)
            return
        if _on_gpu(self.dt):
            gs = gear_m2l_schedule_device(self.dt, gears, orders, max_pairs=self.gear_unit_pairs)
        else:
            gs = gear_m2l_schedule(self.dt.topo, np.asarray(gears), orders, max_pairs=self.gear_unit_pairs)
        if getattr(self, "_range_targets", None) is not None:
            gs = _restrict_gears(gs, self._range_targets, self.dt.topo.num_nodes, self.dt.device)
        self.gear_sched = gs
        self.d_gear_units = up(gs.units)
        self.d_gear_split = up(gs.split)
        self.d_gear_src = up(gs.far_src)
        self.h_gear_orders = np.ascontiguousarray(np.array(orders, dtype=np.int32))
        self.h_gear_offsets = np.ascontiguousarray(gs.gear_offsets.astype(np.int64))
        self.gear_partials = torch.empty((max(gs.num_slots, 1), self.ws.stride), device=dev, dtype=torch.float32)

    def m2l(self, stream=None) -> None:
        ws, s, sc = self.ws, _stream_handle(stream), self.m2l_sched
        _zero(ws.locals, stream)
        if self.m2l_mode == _lib.JB_M2L_SPLIT_BF16:
            self._m2l_split(s, stream)
            return
        gs = getattr(self, "gear_sched", None)
        if isinstance(gs, MixedGearM2LSchedule):
            _lib.check(self.lib.jb_m2l_mixed(
                self.p, int(gs.units.shape[0]), _ptr(self.d_gear_units), _ptr(self.d_gear_bounds), _ptr(ws.mult),
                _ptr(ws.centers), _ptr(self.d_gear_src), _ptr(ws.locals), _ptr(self.gear_partials),
                int(gs.split.shape[0]), _ptr(self.d_gear_split), s), "jb_m2l_mixed")
            return
        if gs is not None:
            _lib.check(self.lib.jb_m2l_gears(
                self.p, self.m2l_mode, len(gs.orders), self.h_gear_orders.ctypes.data,
                self.h_gear_offsets.ctypes.data, _ptr(self.d_gear_units), _ptr(ws.mult), _ptr(ws.centers),
                _ptr(self.d_gear_src), _ptr(ws.locals), _ptr(self.gear_partials), int(gs.split.shape[0]),
                _ptr(self.d_gear_split), s), "jb_m2l_gears")
            return
        _lib.check(self.lib.jb_m2l(self.p, self.m2l_mode, int(sc.units.shape[0]), _ptr(self.d_m2l_units),
                                   _ptr(ws.mult), _ptr(ws.centers), _ptr(self.dt.far_src), _ptr(ws.locals),
                                   _ptr(self.m2l_partials), int(sc.split.shape[0]), _ptr(self.d_m2l_split), s),
                   "jb_m2l")

    def m2l_weighted(self, far_w: torch.Tensor, stream=None) -> None:
        """FP32 M2L at the pass order with far pair e scaled by far_w[e]
        (float32 per CSR far entry, on the device)."""
        ws, s, sc = self.ws, _stream_handle(stream), self.m2l_sched
        w = far_w.to(device=self.dt.device, dtype=torch.float32).contiguous()
        if w.numel() != self.dt.topo.num_far_pairs:
            raise ValueError("one weight per far pair is required")
        _zero(ws.locals, stream)
        _lib.check(self.lib.jb_m2l_weighted(self.p, int(sc.units.shape[0]), _ptr(self.d_m2l_units), _ptr(ws.mult),
                                            _ptr(ws.centers), _ptr(self.dt.far_src), _ptr(w) if w.numel() else None,
                                            _ptr(ws.locals), _ptr(self.m2l_partials), int(sc.split.shape[0]),
                                            _ptr(self.d_m2l_split), s), "jb_m2l_weighted")

    def evaluate_weighted(self, rung_sorted: torch.Tensor, level_weights: torch.Tensor, stream=None,
                          part: str | None = None) -> torch.Tensor:
        """evaluate() with every near pair scaled by
        level_weights[max(rung_i, rung_j)] (rung per sorted particle)."""
        t, dt, ws, sc = self.dt.topo, self.dt, self.ws, self.leaf_sched
        r = rung_sorted.to(device=dt.device, dtype=torch.int32).contiguous()
        lw = level_weights.to(device=dt.device, dtype=torch.float32).contiguous()
        mode = self.p2p_mode
        if part is not None:
            mode |= {"near": _lib.JB_P2P_NEAR_ONLY, "far": _lib.JB_P2P_FAR_ONLY}[part]
        _lib.check(self.lib.jb_leaf_eval_weighted(self.p, mode, _ptr(ws.pos4), _ptr(r), int(lw.numel()), _ptr(lw),
                                                  t.num_internal, int(sc.units.shape[0]), _ptr(self.d_leaf_units),
                                                  _ptr(self.d_leaf_aux), _ptr(self.d_leaf_runs),
                                                  _ptr(dt.node_ranges), _ptr(ws.centers), _ptr(ws.locals), self.G,
                                                  self.eps2, _ptr(ws.acc4), _ptr(self.leaf_partials),
                                                  int(sc.split.shape[0]), _ptr(self.d_leaf_split),
                                                  _stream_handle(stream)), "jb_leaf_eval_weighted")
        return ws.acc4

    def _m2l_split(self, s, stream=None) -> None:
        """Split-BF16 M2L on the tensor cores."""
        if self.tc_layout == "units":
            if getattr(self, "_tc_status", None) is None:
                self._tc_status = torch.zeros(1, device=self.dt.device, dtype=torch.int32)
            _zero(self._tc_status, stream)  # the word reports this launch only
            ws, sc = self.ws, self.m2l_sched
            _lib.check(self.lib.jb_m2l_split_units(self.p, int(sc.units.shape[0]), _ptr(self.d_m2l_units),
                                                   _ptr(ws.mult), _ptr(ws.centers), _ptr(self.dt.far_src),
                                                   _ptr(ws.locals), _ptr(self.m2l_partials),
                                                   int(sc.split.shape[0]), _ptr(self.d_m2l_split),
                                                   _ptr(self._tc_status), s), "jb_m2l_split_units")
            return
        if getattr(self, "_tc", None) is None:
            t, dev = self.dt.topo, self.dt.device
            if self.leaf_range != (0, t.num_leaves):
                raise ValueError("the tensor-core M2L covers the whole far list")
            sc = tc_m2l_schedule(t)
            up = lambda a: torch.from_numpy(a if a.size else np.zeros(4, np.int32)).to(dev)
            self._tc = {
                "sched": sc,
                "seg_off": up(sc.seg_off),
                "segs": up(sc.segs),
                "split": up(sc.split),
                "pair_tgt": up(t.far_pair_targets()),
                "partials": torch.empty((max(sc.num_slots, 1), self.ws.stride), device=dev, dtype=torch.float32),
                "status": torch.zeros(1, device=dev, dtype=torch.int32),
            }
        T, t, ws = self._tc, self.dt.topo, self.ws
        sc = T["sched"]
        _zero(T["status"], stream)
        _lib.check(self.lib.jb_m2l_split(self.p, self.tc_products, sc.num_tiles, t.num_far_pairs, _ptr(T["pair_tgt"]),
                                         _ptr(self.dt.far_src), _ptr(T["seg_off"]), _ptr(T["segs"]), _ptr(ws.mult),
                                         _ptr(ws.centers), _ptr(ws.locals), _ptr(T["partials"]),
                                         int(sc.split.shape[0]), _ptr(T["split"]), _ptr(T["status"]), s),
                   "jb_m2l_split")

    def tc_status(self) -> int:
        """Status word of the last tensor-core M2L (0 = ok, 1 = a barrier wait
        timed out and the locals are incomplete, 2 = the drain after it timed
        out too: the CUDA context is not to be used further).  Reading it
        synchronises the device."""
        T = getattr(self, "_tc", None)
        st = 0 if T is None else int(T["status"].item())
        U = getattr(self, "_tc_status", None)
        return max(st, 0 if U is None else int(U.item()))

    def check_tc_status(self) -> None:
        """Raises JBError when the last tensor-core M2L reported a timeout
        (see tc_status); a no-op for the FP32 M2L."""
        if self.m2l_mode != _lib.JB_M2L_SPLIT_BF16:
            return
        st = self.tc_status()
        if st == 1:
            raise _lib.JBError("tensor-core M2L: an MMA barrier wait timed out; the locals of this pass are "
                               "incomplete")
        if st >= 2:
            raise _lib.JBError("tensor-core M2L: an MMA barrier wait and its drain timed out; the CUDA context "
                               "must not be used further")

    def l2l(self, stream=None, cascade: bool = False) -> None:
        """Downward sweep after the M2L.  By default straight to the leaves:
        each leaf adds L2L(a -> leaf) of every ancestor a with far pairs
        (jb_l2l_leaves, one launch; the internal nodes keep their own M2L
        sums).  cascade=True: level by level (jb_l2l_level), every node's
        local complete -- what the adjoint reads."""
        t, dt, ws, s = self.dt.topo, self.dt, self.ws, _stream_handle(stream)
        if self.l2l_direct and not cascade:
            _lib.check(self.lib.jb_l2l_leaves(self.p, self.num_l2l_units, _ptr(self.d_l2l_units), _ptr(self.d_l2l_anc),
                                              _ptr(ws.centers), _ptr(ws.locals), s), "jb_l2l_leaves")
            return
        lo = dt.level_offsets
        for lev in range(dt.l2l_first_level, t.num_levels):
            _lib.check(self.lib.jb_l2l_level(self.p, lo[lev], lo[lev + 1], _ptr(dt.left), _ptr(dt.right),
                                             _ptr(ws.centers), _ptr(ws.locals), s), "jb_l2l_level")

    _PARTS = {"near": _lib.JB_P2P_NEAR_ONLY, "far": _lib.JB_P2P_FAR_ONLY,
              "near_first": _lib.JB_P2P_NEAR_FIRST, "far_after": _lib.JB_P2P_FAR_AFTER}

    def evaluate(self, stream=None, potential: bool = False, part: str | None = None,
                 out: torch.Tensor | None = None) -> torch.Tensor:
        """L2P + P2P into ws.acc4 (sorted order); part="near" / "far" keeps
        only the P2P / only the L2P contribution.  part="near_first" then
        part="far_after" is the same evaluation in two halves: the first needs
        only ws.pos4 (it can run while upward/downward fill the locals), the
        second adds the L2P and sums split leaves; together they give the
        bits of one call.  out: an (N,4) float32 buffer written instead of
        ws.acc4."""
        t, dt, ws, sc = self.dt.topo, self.dt, self.ws, self.leaf_sched
        acc4 = ws.acc4 if out is None else out
        mode = self.p2p_mode | (_lib.JB_P2P_POTENTIAL if potential else 0)
        if part is not None:
            mode |= self._PARTS[part]
        _lib.check(self.lib.jb_leaf_eval(self.p, mode, _ptr(ws.pos4), t.num_internal, int(sc.units.shape[0]),
                                         _ptr(self.d_leaf_units), _ptr(self.d_leaf_aux), _ptr(self.d_leaf_runs),
                                         _ptr(dt.node_ranges), _ptr(ws.centers), _ptr(ws.locals), self.G,
                                         self.eps2, _ptr(acc4), _ptr(self.leaf_partials),
                                         int(sc.split.shape[0]), _ptr(self.d_leaf_split),
                                         _stream_handle(stream)), "jb_leaf_eval")
        return acc4

    def evaluate_targets(self, targets_sorted: torch.Tensor, out: torch.Tensor | None = None,
                         stream=None) -> torch.Tensor:
        t, dt, ws = self.dt.topo, self.dt, self.ws
        ts = targets_sorted.to(device=dt.device, dtype=torch.int32).contiguous()
        nt = int(ts.shape[0])
        if out is None:
            out = torch.empty((nt, 4), device=dt.device, dtype=torch.float32)
        _lib.check(self.lib.jb_eval_targets(self.p, _ptr(ws.pos4), t.num_internal, _ptr(dt.node_ranges),
                                            _ptr(ws.centers), _ptr(ws.locals), _ptr(dt.near_off),
                                            _ptr(dt.near_src), _ptr(dt.leaf_of), nt, _ptr(ts), self.G, self.eps2,
                                            _ptr(out), _stream_handle(stream)), "jb_eval_targets")
        return out

    def unsort(self, acc: torch.Tensor, pot: torch.Tensor | None, stream=None) -> None:
        n = self.dt.topo.num_particles
        _lib.check(self.lib.jb_gather_unsorted(n, _ptr(self.ws.acc4), _ptr(self.dt.inv_perm), _ptr(acc),
                                               _ptr(pot), _stream_handle(stream)), "jb_gather_unsorted")

    def downward(self, stream=None, cascade: bool = False) -> None:
        self.m2l(stream)
        self.l2l(stream, cascade=cascade)

    def far_stream(self) -> torch.cuda.Stream:
        """The high-priority stream run(overlap=True) puts the far-field chain
        on: its short level launches then take SMs ahead of the near field's
        waiting blocks instead of queueing behind them."""
        if getattr(self, "_far_stream", None) is None:
            hi = torch.cuda.Stream.priority_range()[1] if hasattr(torch.cuda.Stream, "priority_range") else -1
            self._far_stream = torch.cuda.Stream(device=self.dt.device, priority=min(-1, int(hi)))
        return self._far_stream

    def run(self, stream=None, cascade: bool = False, potential: bool = False,
            overlap: bool | None = None) -> torch.Tensor:
        """Whole pass on the particles already in ws.pos4; returns sorted acc4
        (cascade: the level-by-level downward sweep, see l2l).  overlap
        (default self.overlap): the near field runs on `stream` while the
        upward sweep, M2L and L2L run on far_stream(), joined before the L2P
        and the sum of split leaves; the result has the same bits as the
        one-stream order (at 4M, p = 8: 7.89 -> 7.64 ms a step)."""
        if not (self.overlap if overlap is None else overlap):
            self.upward(stream)
            self.downward(stream, cascade=cascade)
            return self.evaluate(stream, potential=potential)
        main = stream if stream is not None else torch.cuda.current_stream(self.dt.device)
        far = self.far_stream()
        far.wait_stream(main)  # the particles are loaded
        self.evaluate(main, potential=potential, part="near_first")
        self.upward(far)
        self.downward(far, cascade=cascade)
        main.wait_stream(far)
        return self.evaluate(main, potential=potential, part="far_after")

    def capture(self, positions: torch.Tensor, masses: torch.Tensor, acc: torch.Tensor,
                potential: torch.Tensor | None = None, warmup: int = 2, overlap: bool | None = None,
                node_priority: bool = False):
        """A CUDA graph of the whole step on this pass's topology: gather of
        `positions` (N,3) / `masses` (N,) into Morton order, the pass, and the
        un-permute into `acc` (N,3) (and `potential` (N,), evaluated then).
        Replaying it (``graph.replay()``, on the current stream) re-evaluates
        the pass on whatever those buffers hold at that moment: the graph
        fixes their addresses, so later inputs are copied into them.  The
        launches are this object's (the same kernels, order and arguments as
        the eager calls), so a replay gives the eager step's bits; the workspace
        is shared with eager use of the same pass.  overlap (default
        self.overlap): the graph forks the far-field chain onto far_stream()
        as run(overlap=True) does; with node_priority its launches keep that
        stream's priority in the graph (a PassGraph, instantiated by the
        library), else the graph is torch's own (the two measured the same at
        4M, p = 8: 7.64 ms a step)."""
        pot = potential is not None
        ov = self.overlap if overlap is None else bool(overlap)

        def step():
            self.load_particles(positions, masses)
            self.run(potential=pot, overlap=ov)
            self.unsort(acc, potential)

        side = torch.cuda.Stream(device=self.dt.device)
        side.wait_stream(torch.cuda.current_stream(self.dt.device))
        with torch.cuda.stream(side):  # the first launches of each kind, outside the capture
            for _ in range(max(1, int(warmup))):
                step()
        torch.cuda.current_stream(self.dt.device).wait_stream(side)
        prio = ov and node_priority
        graph = torch.cuda.CUDAGraph(keep_graph=True) if prio else torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            step()
        return PassGraph(graph, self.lib) if prio else graph

    # -- adjoint --------------------------------------------------------------
    def _adj_buffers(self):
        if getattr(self, "_adj", None) is None:
            t, dev, cs = self.dt.topo, self.dt.device, self.ws.stride
            f32 = dict(device=dev, dtype=torch.float32)
            self._adj = {
                "w4": torch.empty((t.num_particles, 4), **f32),
                "zeros": torch.zeros((t.num_particles,), **f32),
                "xm4": torch.empty((t.num_particles, 4), **f32),
                "lbar": torch.empty((t.num_nodes, cs), **f32),
                "mbar": torch.empty((t.num_nodes, cs), **f32),
                "cbar4": torch.empty((t.num_nodes, 4), **f32),
                "g4": torch.empty((max(t.num_far_pairs, 1), 4), **f32),
                "pair_tgt": torch.from_numpy(t.far_pair_targets() if t.num_far_pairs else np.zeros(1, np.int32)).to(dev),
                "rev": (self.dt.far_reverse_index() if _on_gpu(self.dt) and t.num_far_pairs else
                        torch.from_numpy(t.far_reverse_index() if t.num_far_pairs else np.zeros(1, np.int32)).to(dev)),
            }
            if not t.near_lists_symmetric():
                raise ValueError("the near-field adjoint needs symmetric neighbour lists")
            # full near list of every leaf (the forward schedule may be a leaf range)
            self._adj_sched = (leaf_schedule_device(self.dt, max_sources=4096) if _on_gpu(self.dt)
                               else leaf_schedule(t, max_sources=4096))
            up = lambda a: _up(a, dev)
            self._adj["units"] = up(self._adj_sched.units)
            self._adj["aux"] = up(self._adj_sched.aux)
            self._adj["runs"] = up(self._adj_sched.runs)
            self._adj["split"] = up(self._adj_sched.split)
            self._adj["partials"] = torch.empty((max(self._adj_sched.num_slots, 1) * _lib.JB_MAX_LEAF_OCCUPANCY, 4), **f32)
        return self._adj

    def vjp(self, w: torch.Tensor, grad_pos: torch.Tensor, grad_mass: torch.Tensor, stream=None,
            recompute: bool = True) -> None:
        """Gradient of sum(w * acc) w.r.t. the input-order positions and masses
        currently loaded (acc = the pass's accelerations, input order), written
        into grad_pos (N,3) and grad_mass (N,).  recompute=True reruns the
        upward and downward sweeps first (multipoles / locals are not kept from
        the forward call); False reuses the coefficients already in the
        workspace."""
        if self.p > 9:
            raise ValueError("the adjoint is built for expansion orders <= 9")
        if self.leaf_range != (0, self.dt.topo.num_leaves):
            raise ValueError("the adjoint runs on the whole leaf range")
        t, dt, ws, lb, s = self.dt.topo, self.dt, self.ws, self.lib, _stream_handle(stream)
        A = self._adj_buffers()
        sc = self._adj_sched
        if recompute:  # the reverse sweeps read every node's complete local
            self.upward(stream)
            self.downward(stream, cascade=True)
        w = w.to(device=dt.device, dtype=torch.float32).contiguous()
        _lib.check(lb.jb_gather_sorted(t.num_particles, _ptr(w), _ptr(A["zeros"]), _ptr(dt.perm), _ptr(A["w4"]), s),
                   "jb_gather_sorted(w)")
        _zero(A["cbar4"], stream)
        _zero(A["mbar"], stream)
        _lib.check(lb.jb_adj_near(_ptr(ws.pos4), _ptr(A["w4"]), t.num_internal, int(sc.units.shape[0]),
                                  _ptr(A["units"]), _ptr(A["aux"]), _ptr(A["runs"]), _ptr(dt.node_ranges), self.G,
                                  self.eps2, _ptr(A["xm4"]), _ptr(A["partials"]), int(sc.split.shape[0]),
                                  _ptr(A["split"]), s), "jb_adj_near")
        _lib.check(lb.jb_adj_leaf_far(self.p, _ptr(ws.pos4), _ptr(A["w4"]), t.num_nodes, t.num_internal,
                                      _ptr(dt.node_ranges), _ptr(ws.centers), _ptr(ws.locals), self.G,
                                      _ptr(A["xm4"]), _ptr(A["lbar"]), _ptr(A["cbar4"]), s), "jb_adj_leaf_far")
        lo = dt.level_offsets
        for lev in range(t.num_levels - 1, -1, -1):
            _lib.check(lb.jb_adj_l2l_level(self.p, lo[lev], lo[lev + 1], _ptr(dt.left), _ptr(dt.right),
                                           _ptr(ws.centers), _ptr(ws.locals), _ptr(A["lbar"]), _ptr(A["cbar4"]), s),
                       "jb_adj_l2l_level")
        if hasattr(self, "_adj_m2l"):
            msc = self._adj_m2l
        else:
            msc = m2l_schedule_device(dt, max_pairs=512) if _on_gpu(dt) else m2l_schedule(t, max_pairs=512)
            self._adj_m2l = msc
            up = lambda a: _up(a, dt.device)
            A["m2l_units"], A["m2l_split"] = up(msc.units), up(msc.split)
            A["m2l_partials"] = torch.empty((max(msc.num_slots, 1), ws.stride), device=dt.device,
                                            dtype=torch.float32)
        _lib.check(lb.jb_adj_m2l(self.p, int(msc.units.shape[0]), _ptr(A["m2l_units"]), _ptr(A["lbar"]),
                                 _ptr(ws.centers), _ptr(dt.far_src), _ptr(A["mbar"]), _ptr(A["m2l_partials"]),
                                 int(msc.split.shape[0]), _ptr(A["m2l_split"]), s), "jb_adj_m2l")
        _lib.check(lb.jb_adj_m2l_centers(self.p, t.num_nodes, t.num_far_pairs, _ptr(A["pair_tgt"]),
                                         _ptr(dt.far_src), _ptr(dt.far_off), _ptr(A["rev"]), _ptr(ws.mult),
                                         _ptr(A["lbar"]), _ptr(ws.centers), _ptr(A["g4"]), _ptr(A["cbar4"]), s),
                   "jb_adj_m2l_centers")
        for lev in range(t.num_levels):
            _lib.check(lb.jb_adj_m2m_level(self.p, lo[lev], lo[lev + 1], _ptr(dt.left), _ptr(dt.right),
                                           _ptr(ws.centers), _ptr(ws.mult), _ptr(A["mbar"]), _ptr(A["cbar4"]), s),
                       "jb_adj_m2m_level")
        _lib.check(lb.jb_adj_p2m(self.p, _ptr(ws.pos4), t.num_nodes, t.num_internal, _ptr(dt.node_ranges),
                                 _ptr(ws.centers), _ptr(A["mbar"]), _ptr(A["cbar4"]), _ptr(A["xm4"]), s),
                   "jb_adj_p2m")
        _lib.check(lb.jb_gather_unsorted(t.num_particles, _ptr(A["xm4"]), _ptr(dt.inv_perm), _ptr(grad_pos),
                                         _ptr(grad_mass), s), "jb_gather_unsorted(grad)")

    def launches_per_run(self) -> int:
        """This library's kernel launches in one run(): P2M, one M2M per level,
        the M2L (one launch per non-empty gear with gears) and its split
        reduce, one L2L per level from the first with a non-zero local, the
        leaf L2P + P2P and their split reduce."""
        t = self.dt.topo
        gs = getattr(self, "gear_sched", None)
        if isinstance(gs, MixedGearM2LSchedule):
            m2l = int(gs.units.shape[0] > 0) + int(gs.split.shape[0] > 0)
        elif gs is not None and self.m2l_mode == _lib.JB_M2L_FP32:
            m2l = int((np.diff(np.asarray(gs.gear_offsets)) > 0).sum()) + int(gs.split.shape[0] > 0)
        else:
            m2l = 1 + int(self.m2l_sched.split.shape[0] > 0)
        l2l = t.num_levels - self.dt.l2l_first_level
        return (1 + t.num_levels + m2l + l2l + 2 + int(self.leaf_sched.split.shape[0] > 0))
