"""Work-unit schedules for the far-field (M2L) and leaf-evaluation kernels.

Built once per topology on the host (prepare time, like the reference's
near-field schedules in nearfield/_schedules.py:271 and the M2L chunking of
runtime/kernels/_m2l.py:1667).  Both bound the work of one GPU thread / warp
so that no single long interaction list sets the kernel's duration:

* M2L units: at most ``max_pairs`` consecutive pairs of one target's CSR list;
* leaf units: one target leaf and a slice of its neighbour list holding at
  most ``max_sources`` source particles, stored as runs of consecutive
  neighbour leaves (contiguous particle ranges).

Targets (leaves) split over several units get consecutive scratch slots and an
entry in the split list; the reduce kernels sum those slots in order, so the
result does not depend on scheduling.  Units are ordered by decreasing work.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .tree import Topology


@dataclass
class M2LSchedule:
    units: np.ndarray  # int32[U, 4] (target, first pair, end pair, slot)
    split: np.ndarray  # int32[S, 4] (target, first slot, slot count, 0)
    num_slots: int


@dataclass
class LeafSchedule:
    units: np.ndarray  # int32[U, 4] (leaf, first run, end run, source count)
    aux: np.ndarray  # int32[U, 2] (slot, flags)
    runs: np.ndarray  # int32[R, 2] (first particle, count)
    split: np.ndarray  # int32[S, 4] (leaf, first slot, slot count, 0)
    num_slots: int


def _slots(n_per: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Slot of every unit (-1 for singletons) and each split owner's first slot."""
    multi = np.repeat(n_per > 1, n_per)
    slot = np.where(multi, np.cumsum(multi) - 1, -1).astype(np.int32)
    first = np.cumsum(n_per) - n_per
    return slot, slot[first]


def m2l_schedule(topo: Topology, max_pairs: int = 64, targets: np.ndarray | None = None) -> M2LSchedule:
    off = topo.far_offsets
    counts = np.diff(off)
    tg = topo.m2l_targets if targets is None else np.asarray(targets, dtype=np.int64)
    tg = tg[counts[tg] > 0].astype(np.int64)
    c = counts[tg]
    nu = (c + max_pairs - 1) // max_pairs
    if tg.size == 0:
        return M2LSchedule(np.zeros((0, 4), np.int32), np.zeros((0, 4), np.int32), 0)
    rep = np.repeat(tg, nu)
    k = np.arange(int(nu.sum())) - np.repeat(np.cumsum(nu) - nu, nu)
    start = off[rep] + k * max_pairs
    end = np.minimum(start + max_pairs, off[rep + 1])
    slot, first_slot = _slots(nu)
    units = np.stack([rep, start, end, slot], axis=1).astype(np.int32)
    order = np.argsort(-(end - start), kind="stable")
    units = np.ascontiguousarray(units[order])
    sp = nu > 1
    split = np.stack([tg[sp], first_slot[sp], nu[sp], np.zeros(int(sp.sum()), np.int64)], axis=1).astype(np.int32)
    return M2LSchedule(units, np.ascontiguousarray(split), int((slot >= 0).sum()))


@dataclass
class GearM2LSchedule:
    """M2L units when every far pair carries its own expansion order (gear).

    ``far_src`` is the CSR source list with each target's pairs regrouped by
    gear (stable); ``units`` (target, first, end, slot) index it and never mix
    gears; ``gear_offsets[g]:gear_offsets[g+1]`` are the units of gear g (one
    launch each, at that gear's order).  Targets covered by more than one unit
    write scratch slots that ``split`` sums in slot order."""

    units: np.ndarray  # int32[U, 4]
    split: np.ndarray  # int32[S, 4]
    num_slots: int
    far_src: np.ndarray  # int32[num_far] regrouped sources
    gear_offsets: np.ndarray  # int64[G + 1]
    orders: tuple
    pairs_per_gear: np.ndarray  # int64[G]


def gear_m2l_schedule(topo: Topology, gears: np.ndarray, orders, max_pairs: int = 64) -> GearM2LSchedule:
    gears = np.asarray(gears, dtype=np.int64).reshape(-1)
    if gears.shape[0] != topo.num_far_pairs:
        raise ValueError("one gear per far pair is required")
    ng = len(orders)
    if gears.size and (gears.min() < 0 or gears.max() >= ng):
        raise ValueError("gear index out of range")
    off = topo.far_offsets
    tgt = np.repeat(np.arange(topo.num_nodes, dtype=np.int64), np.diff(off))
    order = np.lexsort((gears, tgt))  # by target, then gear (stable inside)
    far_src = topo.far_sources[order].astype(np.int32)
    g_sorted = gears[order]
    t_sorted = tgt[order]
    if order.size == 0:
        z4 = np.zeros((0, 4), np.int32)
        return GearM2LSchedule(z4, z4, 0, far_src, np.zeros(ng + 1, np.int64), tuple(orders), np.zeros(ng, np.int64))
    brk = np.ones(order.size, dtype=bool)
    brk[1:] = (t_sorted[1:] != t_sorted[:-1]) | (g_sorted[1:] != g_sorted[:-1])
    seg_start = np.nonzero(brk)[0]
    seg_end = np.concatenate([seg_start[1:], [order.size]])
    seg_t, seg_g = t_sorted[seg_start], g_sorted[seg_start]
    cnt = seg_end - seg_start
    nu = (cnt + max_pairs - 1) // max_pairs
    rep = np.repeat(np.arange(seg_start.size), nu)
    k = np.arange(int(nu.sum())) - np.repeat(np.cumsum(nu) - nu, nu)
    u_start = seg_start[rep] + k * max_pairs
    u_end = np.minimum(u_start + max_pairs, seg_end[rep])
    u_t, u_g = seg_t[rep], seg_g[rep]
    # units are target-major here: number of units per target -> slots
    tb = np.ones(u_t.size, dtype=bool)
    tb[1:] = u_t[1:] != u_t[:-1]
    t_first = np.nonzero(tb)[0]
    n_per = np.diff(np.concatenate([t_first, [u_t.size]]))
    slot, first_slot = _slots(n_per)
    units = np.stack([u_t, u_start, u_end, slot], axis=1).astype(np.int32)
    srt = np.lexsort((-(u_end - u_start), u_g))
    units = np.ascontiguousarray(units[srt])
    ug = u_g[srt]
    gear_offsets = np.searchsorted(ug, np.arange(ng + 1)).astype(np.int64)
    sp = n_per > 1
    split = np.stack([u_t[t_first][sp], first_slot[sp], n_per[sp], np.zeros(int(sp.sum()), np.int64)],
                     axis=1).astype(np.int32)
    ppg = np.bincount(gears, minlength=ng).astype(np.int64)
    return GearM2LSchedule(units, np.ascontiguousarray(split), int((slot >= 0).sum()), far_src, gear_offsets,
                           tuple(int(o) for o in orders), ppg)


MIXED_SEGMENTS = 4


def mixed_ladder(p_max: int) -> tuple:
    """Orders the one-launch gear M2L (jb_m2l_mixed) evaluates: p_max,
    p_max-2, p_max-4, p_max-6, those >= 1."""
    return tuple(o for o in range(p_max, p_max - 2 * MIXED_SEGMENTS, -2) if o >= 1)


@dataclass
class MixedGearM2LSchedule:
    """M2L units for per-pair gears whose orders lie on ``mixed_ladder(p_max)``,
    run in one launch (jb_m2l_mixed).

    ``far_src`` is the CSR source list with each target's pairs sorted by
    order, highest first (stable inside); ``units`` (target, first, end, slot)
    are slices of at most ``max_pairs`` of one target's list and ``bounds``
    (b1, b2, b3, end) cut a unit into the segments [b_j, b_j+1) (b_0 = first)
    of order p_max - 2j.  Units are sorted by decreasing segment lengths,
    highest order first (stable), so neighbouring units have similar ones.
    Targets covered by more than one unit write scratch slots that ``split``
    sums in slot order."""

    units: np.ndarray  # int32[U, 4]
    bounds: np.ndarray  # int32[U, 4]
    split: np.ndarray  # int32[S, 4]
    num_slots: int
    far_src: np.ndarray  # int32[num_far] sorted by order inside each target
    orders: tuple
    pairs_per_gear: np.ndarray  # int64[G]
    p_max: int


def _mixed_segments(orders, p_max: int) -> np.ndarray:
    ladder = mixed_ladder(p_max)
    if any(int(o) not in ladder for o in orders):
        raise ValueError(f"gear orders {tuple(orders)} are not on the ladder {ladder}")
    return np.array([(p_max - int(o)) // 2 for o in orders], dtype=np.int64)


def gear_m2l_mixed_schedule(topo: Topology, gears: np.ndarray, orders, p_max: int,
                            max_pairs: int = 128) -> MixedGearM2LSchedule:
    gears = np.asarray(gears, dtype=np.int64).reshape(-1)
    if gears.shape[0] != topo.num_far_pairs:
        raise ValueError("one gear per far pair is required")
    ng = len(orders)
    if gears.size and (gears.min() < 0 or gears.max() >= ng):
        raise ValueError("gear index out of range")
    seg_of = _mixed_segments(orders, p_max)
    off = topo.far_offsets.astype(np.int64)
    nodes = topo.num_nodes
    tgt = np.repeat(np.arange(nodes, dtype=np.int64), np.diff(off))
    seg = seg_of[gears] if gears.size else np.zeros(0, np.int64)
    order = np.lexsort((seg, tgt))  # by target, then segment (stable inside)
    far_src = topo.far_sources[order].astype(np.int32)
    ppg = np.bincount(gears, minlength=ng).astype(np.int64)
    z4 = np.zeros((0, 4), np.int32)
    if order.size == 0:
        return MixedGearM2LSchedule(z4, z4, z4, 0, far_src, tuple(orders), ppg, int(p_max))
    # segment starts of every target: off + counts of the higher segments
    cnt = np.zeros((nodes, MIXED_SEGMENTS), np.int64)
    np.add.at(cnt, (tgt, seg), 1)
    starts = off[:-1, None] + np.concatenate([np.zeros((nodes, 1), np.int64), np.cumsum(cnt, axis=1)], axis=1)
    n_t = np.diff(off)
    nu = (n_t + max_pairs - 1) // max_pairs
    u_t = np.repeat(np.arange(nodes, dtype=np.int64), nu)
    k = np.arange(int(nu.sum())) - np.repeat(np.cumsum(nu) - nu, nu)
    u_s = off[u_t] + k * max_pairs
    u_e = np.minimum(u_s + max_pairs, off[u_t + 1])
    bd = np.clip(starts[u_t], u_s[:, None], u_e[:, None])  # [U, 5]: b_0 = first .. b_4 = end
    slot, first_slot = _slots(nu[nu > 0])
    units = np.stack([u_t, u_s, u_e, slot], axis=1).astype(np.int32)
    bounds = np.stack([bd[:, 1], bd[:, 2], bd[:, 3], u_e], axis=1).astype(np.int32)
    c = np.diff(bd, axis=1)  # segment lengths
    srt = np.lexsort(tuple(-c[:, j] for j in range(MIXED_SEGMENTS - 1, -1, -1)))
    t_nonempty = np.nonzero(nu > 0)[0]
    sp = nu[t_nonempty] > 1
    split = np.stack([t_nonempty[sp], first_slot[sp], nu[t_nonempty][sp], np.zeros(int(sp.sum()), np.int64)],
                     axis=1).astype(np.int32)
    return MixedGearM2LSchedule(np.ascontiguousarray(units[srt]), np.ascontiguousarray(bounds[srt]),
                                np.ascontiguousarray(split), int((slot >= 0).sum()), far_src,
                                tuple(int(o) for o in orders), ppg, int(p_max))


@dataclass
class TcM2LSchedule:
    """Tiles of 128 consecutive far pairs (CSR order, sorted by target) for the
    tensor-core M2L.  seg_off[t]:seg_off[t+1] index the target runs of tile t,
    segs[i] = (target, first row, end row, slot): slot -1 when the target's
    whole list lies in the tile (the run writes the local row), else a scratch
    row that ``split`` sums in slot order."""

    num_tiles: int
    seg_off: np.ndarray  # int32[num_tiles + 1]
    segs: np.ndarray  # int32[S, 4]
    split: np.ndarray  # int32[T, 4]
    num_slots: int


def tc_m2l_schedule(topo: Topology, tile: int = 128) -> TcM2LSchedule:
    npairs = topo.num_far_pairs
    nt = (npairs + tile - 1) // tile
    if npairs == 0:
        z = np.zeros((0, 4), np.int32)
        return TcM2LSchedule(0, np.zeros(1, np.int32), z, z, 0)
    tgt = np.repeat(np.arange(topo.num_nodes, dtype=np.int64), np.diff(topo.far_offsets))
    e = np.arange(npairs, dtype=np.int64)
    brk = np.ones(npairs, dtype=bool)
    brk[1:] = (tgt[1:] != tgt[:-1]) | (e[1:] % tile == 0)
    st = np.nonzero(brk)[0]
    en = np.concatenate([st[1:], [npairs]])
    seg_t = tgt[st]
    seg_tile = st // tile
    # segments per target: whole list in one segment -> no slot
    tb = np.ones(st.size, dtype=bool)
    tb[1:] = seg_t[1:] != seg_t[:-1]
    first = np.nonzero(tb)[0]
    n_per = np.diff(np.concatenate([first, [st.size]]))
    slot, first_slot = _slots(n_per)
    segs = np.stack([seg_t, st - seg_tile * tile, en - seg_tile * tile, slot], axis=1).astype(np.int32)
    seg_off = np.searchsorted(seg_tile, np.arange(nt + 1)).astype(np.int32)
    sp = n_per > 1
    split = np.stack([seg_t[first][sp], first_slot[sp], n_per[sp], np.zeros(int(sp.sum()), np.int64)],
                     axis=1).astype(np.int32)
    return TcM2LSchedule(int(nt), seg_off, np.ascontiguousarray(segs), np.ascontiguousarray(split),
                         int((slot >= 0).sum()))


def leaf_schedule(topo: Topology, max_sources: int = 4096, leaf_range: tuple[int, int] | None = None) -> LeafSchedule:
    lo, hi = (0, topo.num_leaves) if leaf_range is None else leaf_range
    ni = topo.num_internal
    cnt_leaf = (topo.node_ranges[ni:, 1] - topo.node_ranges[ni:, 0] + 1).astype(np.int64)
    start_leaf = topo.node_ranges[ni:, 0].astype(np.int64)
    noff = topo.near_offsets
    e0, e1 = int(noff[lo]), int(noff[hi])
    src = topo.near_leaves[e0:e1].astype(np.int64)
    tgt = np.repeat(np.arange(lo, hi, dtype=np.int64), np.diff(noff[lo:hi + 1]))
    w = cnt_leaf[src]
    # exclusive cumulative source count within each target leaf
    cs = np.cumsum(w)
    leaf_base = np.concatenate([[0], cs])[noff[lo:hi + 1][:-1] - e0]
    cum_excl = cs - w - np.repeat(leaf_base, np.diff(noff[lo:hi + 1]))
    uil = cum_excl // max_sources  # unit index within its leaf
    if src.size:
        brk = np.ones(src.size, dtype=bool)
        brk[1:] = (tgt[1:] != tgt[:-1]) | (uil[1:] != uil[:-1]) | (src[1:] != src[:-1] + 1)
        rid = np.cumsum(brk) - 1
        rfirst = np.nonzero(brk)[0]
        run_start = start_leaf[src[rfirst]]
        run_cnt = np.add.reduceat(w, rfirst)
        runs = np.stack([run_start, run_cnt], axis=1).astype(np.int32)
        run_tgt, run_uil = tgt[rfirst], uil[rfirst]
        ubrk = np.ones(rfirst.size, dtype=bool)
        ubrk[1:] = (run_tgt[1:] != run_tgt[:-1]) | (run_uil[1:] != run_uil[:-1])
        ufirst = np.nonzero(ubrk)[0]
        u_leaf = run_tgt[ufirst]
        u_rb = ufirst
        u_re = np.concatenate([ufirst[1:], [rfirst.size]])
        u_ns = np.add.reduceat(run_cnt, ufirst)
        u_first = run_uil[ufirst] == 0
        del rid
    else:
        runs = np.zeros((0, 2), np.int32)
        u_leaf = u_rb = u_re = u_ns = np.zeros(0, np.int64)
        u_first = np.zeros(0, bool)
    # leaves without neighbours still need their self block + far field
    all_leaves = np.arange(lo, hi, dtype=np.int64)
    has = np.zeros(hi - lo, dtype=bool)
    has[u_leaf - lo] = True
    lone = all_leaves[~has]
    u_leaf = np.concatenate([u_leaf, lone])
    u_rb = np.concatenate([u_rb, np.zeros(lone.size, np.int64)])
    u_re = np.concatenate([u_re, np.zeros(lone.size, np.int64)])
    u_ns = np.concatenate([u_ns, np.zeros(lone.size, np.int64)])
    u_first = np.concatenate([u_first, np.ones(lone.size, bool)])
    # group units of a leaf together (leaf order, first unit first) to assign slots
    order = np.lexsort((~u_first, u_leaf))
    u_leaf, u_rb, u_re, u_ns, u_first = u_leaf[order], u_rb[order], u_re[order], u_ns[order], u_first[order]
    leaves_u, n_per = np.unique(u_leaf, return_counts=True)
    slot, first_slot = _slots(n_per)
    work = u_ns + np.where(u_first, cnt_leaf[u_leaf], 0)
    units = np.stack([u_leaf, u_rb, u_re, u_ns], axis=1).astype(np.int32)
    aux = np.stack([slot, u_first.astype(np.int64)], axis=1).astype(np.int32)
    srt = np.argsort(-work, kind="stable")
    sp = n_per > 1
    split = np.stack([leaves_u[sp], first_slot[sp], n_per[sp], np.zeros(int(sp.sum()), np.int64)],
                     axis=1).astype(np.int32)
    return LeafSchedule(np.ascontiguousarray(units[srt]), np.ascontiguousarray(aux[srt]),
                        np.ascontiguousarray(runs), np.ascontiguousarray(split), int((slot >= 0).sum()))


# ---------------------------------------------------------------------------
# The same schedules built on the GPU (csrc/schedule_gpu.cu).  They take the
# device-resident lists of an engine.DeviceTopology and return the same
# dataclasses with torch tensors (on the device) in place of the index arrays;
# gear_offsets and pairs_per_gear stay on the host (kernel launch bounds).
# ---------------------------------------------------------------------------
def _sched_info_cls():
    import ctypes

    class SchedInfo(ctypes.Structure):
        _fields_ = [("num_units", ctypes.c_int64), ("num_split", ctypes.c_int64), ("num_slots", ctypes.c_int64),
                    ("num_runs", ctypes.c_int64), ("num_targets", ctypes.c_int64)]

    return SchedInfo


_SchedInfo = None


def _run_device(fn_name: str, args: list, device):
    """Calls one jb_*_schedule_device builder; returns (info, field getter, free)."""
    import ctypes

    import torch

    from . import _lib
    from .tree import device_view

    global _SchedInfo
    if _SchedInfo is None:
        _SchedInfo = _sched_info_cls()
    lb = _lib.lib()
    h = ctypes.c_void_p()
    stream = torch.cuda.current_stream(device).cuda_stream
    _lib.check(getattr(lb, fn_name)(*args, stream, ctypes.byref(h)), fn_name)
    info = _SchedInfo()
    _lib.check(lb.jb_dsched_info(h, ctypes.byref(info)), "jb_dsched_info")

    def field(fid: int, shape, dtype):
        return device_view(lb.jb_dsched_field(h, fid), shape, dtype, device).clone()

    return info, field, (lambda: lb.jb_dsched_free(h))


def _ptr(t) -> int:
    return int(t.data_ptr())


def m2l_schedule_device(dt, max_pairs: int = 64, targets=None) -> M2LSchedule:
    """GPU twin of :func:`m2l_schedule` over ``dt`` (engine.DeviceTopology)."""
    import torch

    from . import _lib

    t = dt.topo
    tg = None
    if targets is not None:
        tg = torch.as_tensor(np.asarray(targets, dtype=np.int32)).to(dt.device)
    info, field, free = _run_device("jb_m2l_schedule_device",
                                    [t.num_nodes, _ptr(dt.far_off), int(max_pairs),
                                     -1 if tg is None else int(tg.numel()), None if tg is None else _ptr(tg)],
                                    dt.device)
    try:
        units = field(_lib.JB_SCHED_UNITS, (info.num_units, 4), np.int32)
        split = field(_lib.JB_SCHED_SPLIT, (info.num_split, 4), np.int32)
    finally:
        free()
    return M2LSchedule(units, split, int(info.num_slots))


def leaf_schedule_device(dt, max_sources: int = 4096, leaf_range: tuple[int, int] | None = None) -> LeafSchedule:
    """GPU twin of :func:`leaf_schedule` over ``dt`` (engine.DeviceTopology)."""
    from . import _lib

    t = dt.topo
    lo, hi = (0, t.num_leaves) if leaf_range is None else (int(leaf_range[0]), int(leaf_range[1]))
    info, field, free = _run_device("jb_leaf_schedule_device",
                                    [t.num_internal, t.num_leaves, _ptr(dt.node_ranges), _ptr(dt.near_off),
                                     _ptr(dt.near_src), lo, hi, int(max_sources)], dt.device)
    try:
        units = field(_lib.JB_SCHED_UNITS, (info.num_units, 4), np.int32)
        aux = field(_lib.JB_SCHED_AUX, (info.num_units, 2), np.int32)
        runs = field(_lib.JB_SCHED_RUNS, (info.num_runs, 2), np.int32)
        split = field(_lib.JB_SCHED_SPLIT, (info.num_split, 4), np.int32)
    finally:
        free()
    return LeafSchedule(units, aux, runs, split, int(info.num_slots))


def gear_m2l_mixed_schedule_device(dt, gears, orders, p_max: int, max_pairs: int = 128) -> MixedGearM2LSchedule:
    """GPU twin of :func:`gear_m2l_mixed_schedule`."""
    import torch

    from . import _lib

    _mixed_segments(orders, p_max)  # the library checks the same; this gives the message
    t = dt.topo
    g = torch.as_tensor(gears).to(device=dt.device, dtype=torch.int32).reshape(-1).contiguous()
    if g.numel() != t.num_far_pairs:
        raise ValueError("one gear per far pair is required")
    ng = len(orders)
    ho = np.ascontiguousarray(np.array(orders, dtype=np.int32))
    info, field, free = _run_device("jb_gear_mixed_schedule_device",
                                    [t.num_nodes, _ptr(dt.far_off), _ptr(dt.far_src), _ptr(g), ng, ho.ctypes.data,
                                     int(p_max), int(max_pairs)], dt.device)
    try:
        units = field(_lib.JB_SCHED_UNITS, (info.num_units, 4), np.int32)
        bounds = field(_lib.JB_SCHED_AUX, (info.num_units, 4), np.int32)
        split = field(_lib.JB_SCHED_SPLIT, (info.num_split, 4), np.int32)
        far_src = field(_lib.JB_SCHED_FAR_SOURCES, (t.num_far_pairs,), np.int32)
        ppg = field(_lib.JB_SCHED_PAIRS_PER_GEAR, (ng,), np.int64).cpu().numpy()
    finally:
        free()
    return MixedGearM2LSchedule(units, bounds, split, int(info.num_slots), far_src, tuple(int(o) for o in orders),
                                ppg, int(p_max))


def gear_m2l_schedule_device(dt, gears, orders, max_pairs: int = 64) -> GearM2LSchedule:
    """GPU twin of :func:`gear_m2l_schedule`; ``gears`` is one int per far pair
    (numpy or torch)."""
    import torch

    from . import _lib

    t = dt.topo
    g = torch.as_tensor(gears).to(device=dt.device, dtype=torch.int32).reshape(-1).contiguous()
    if g.numel() != t.num_far_pairs:
        raise ValueError("one gear per far pair is required")
    ng = len(orders)
    info, field, free = _run_device("jb_gear_schedule_device",
                                    [t.num_nodes, _ptr(dt.far_off), _ptr(dt.far_src), _ptr(g), ng, int(max_pairs)],
                                    dt.device)
    try:
        units = field(_lib.JB_SCHED_UNITS, (info.num_units, 4), np.int32)
        split = field(_lib.JB_SCHED_SPLIT, (info.num_split, 4), np.int32)
        far_src = field(_lib.JB_SCHED_FAR_SOURCES, (t.num_far_pairs,), np.int32)
        gear_offsets = field(_lib.JB_SCHED_GEAR_OFFSETS, (ng + 1,), np.int64).cpu().numpy()
        ppg = field(_lib.JB_SCHED_PAIRS_PER_GEAR, (ng,), np.int64).cpu().numpy()
    finally:
        free()
    return GearM2LSchedule(units, split, int(info.num_slots), far_src, gear_offsets, tuple(int(o) for o in orders),
                           ppg)
