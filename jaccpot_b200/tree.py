"""Host prepare: tree topology and interaction lists (yggdrax stand-in).

``build_topology`` calls ``jb_tree_build`` (csrc/tree_build.cpp) and returns a
:class:`Topology` of numpy arrays in the layout the reference's kernels read
from yggdrax artefacts (``Tree.node_ranges/left_child/right_child``,
``NodeInteractionList``, ``NodeNeighborList``, the Morton permutation), see
jaccpot/runtime/fmm_state.py:870-897 for the state that carries them.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib


@dataclass
class Topology:
    num_particles: int
    num_nodes: int
    num_internal: int
    num_leaves: int
    num_levels: int
    max_leaf_occupancy: int
    leaf_size: int
    theta: float
    permutation: np.ndarray  # int64[N] sorted slot -> input index
    inverse_permutation: np.ndarray  # int64[N] input index -> sorted slot
    node_ranges: np.ndarray  # int32[num_nodes, 2] inclusive
    left_child: np.ndarray  # int32[num_internal]
    right_child: np.ndarray  # int32[num_internal]
    parent: np.ndarray  # int32[num_nodes]
    node_level: np.ndarray  # int32[num_nodes]
    level_offsets: np.ndarray  # int32[num_levels + 1]
    leaf_of_particle: np.ndarray  # int32[N]
    far_offsets: np.ndarray  # int64[num_nodes + 1]
    far_sources: np.ndarray  # int32[num_far]
    near_offsets: np.ndarray  # int64[num_leaves + 1]
    near_leaves: np.ndarray  # int32[num_near]
    centers_f64: np.ndarray  # float64[num_nodes, 3] (host COM used by the MAC)
    radii_f64: np.ndarray  # float64[num_nodes]
    m2l_targets: np.ndarray = field(default=None)  # int32, nodes with >= 1 far pair, longest list first
    # error-controlled walk only: gear index of every far pair and the gears' orders
    far_gears: np.ndarray = field(default=None)  # int32[num_far]
    gear_orders: tuple = field(default=None)

    @property
    def num_far_pairs(self) -> int:
        return int(self.far_sources.shape[0])

    @property
    def num_near_pairs(self) -> int:
        return int(self.near_leaves.shape[0])

    def far_pair_targets(self) -> np.ndarray:
        """int32[num_far]: the target node of every far pair (CSR row of each entry)."""
        return np.repeat(np.arange(self.num_nodes, dtype=np.int32), np.diff(self.far_offsets)).astype(np.int32)

    def far_reverse_index(self) -> np.ndarray:
        """int32[num_far]: index of the pair (s <- t) for every pair (t <- s).

        The dual traversal emits every accepted pair in both directions, so the
        reverse always exists; raises if it does not (the adjoint relies on it)."""
        tgt = self.far_pair_targets().astype(np.int64)
        src = self.far_sources.astype(np.int64)
        key = tgt * self.num_nodes + src
        order = np.argsort(key, kind="stable")
        rkey = src * self.num_nodes + tgt
        pos = np.searchsorted(key[order], rkey)
        pos = np.minimum(pos, max(key.size - 1, 0))
        rev = order[pos] if key.size else np.zeros(0, np.int64)
        if key.size and not np.array_equal(key[rev], rkey):
            raise ValueError("far lists are not symmetric")
        return rev.astype(np.int32)

    def near_lists_symmetric(self) -> bool:
        """True when leaf B is in A's neighbour list exactly when A is in B's."""
        tgt = np.repeat(np.arange(self.num_leaves, dtype=np.int64), np.diff(self.near_offsets))
        src = self.near_leaves.astype(np.int64)
        a = np.sort(tgt * self.num_leaves + src)
        b = np.sort(src * self.num_leaves + tgt)
        return bool(np.array_equal(a, b))

    def near_pair_interactions(self) -> int:
        """Particle-particle interactions of the near field (self blocks included)."""
        cnt = (self.node_ranges[:, 1] - self.node_ranges[:, 0] + 1).astype(np.int64)
        leaf_cnt = cnt[self.num_internal:]
        src_cnt = leaf_cnt[self.near_leaves]
        per_edge_t = np.repeat(leaf_cnt, np.diff(self.near_offsets))
        return int((per_edge_t * src_cnt).sum() + (leaf_cnt * (leaf_cnt - 1)).sum())


def _field_sizes(n: int, info) -> dict:
    return {
        "permutation": n,
        "node_ranges": 2 * info.num_nodes,
        "left_child": info.num_internal,
        "right_child": info.num_internal,
        "parent": info.num_nodes,
        "node_level": info.num_nodes,
        "level_offsets": info.num_levels + 1,
        "leaf_of_particle": n,
        "far_offsets": info.num_nodes + 1,
        "far_sources": info.num_far_pairs,
        "near_offsets": info.num_leaves + 1,
        "near_leaves": info.num_near_pairs,
        "centers_f64": 3 * info.num_nodes,
        "radii_f64": info.num_nodes,
        "far_gears": info.num_far_pairs,
    }


def _copy_fields(copy_fn, handle, n: int, info, with_gears: bool = False) -> dict:
    sizes = _field_sizes(n, info)
    arrs = {}
    for name, (fid, dt) in _lib.TREE_FIELDS.items():
        if name == "far_gears" and not with_gears:
            continue
        a = np.empty(max(sizes[name], 1), dtype=dt)
        _lib.check(copy_fn(handle, fid, a.ctypes.data), f"tree field copy ({name})")
        arrs[name] = a[: sizes[name]]
    return arrs


def _topology(n: int, info, arrs: dict, leaf_size: int, theta: float, gear_orders=None) -> Topology:
    perm = arrs["permutation"]
    inv = np.empty_like(perm)
    inv[perm] = np.arange(n, dtype=np.int64)
    counts = np.diff(arrs["far_offsets"])
    tg = np.nonzero(counts)[0]
    order = np.argsort(-counts[tg], kind="stable")
    return Topology(
        num_particles=n,
        num_nodes=info.num_nodes,
        num_internal=info.num_internal,
        num_leaves=info.num_leaves,
        num_levels=info.num_levels,
        max_leaf_occupancy=info.max_leaf_occupancy,
        leaf_size=int(leaf_size),
        theta=float(theta),
        permutation=perm,
        inverse_permutation=inv,
        node_ranges=arrs["node_ranges"].reshape(-1, 2),
        left_child=arrs["left_child"],
        right_child=arrs["right_child"],
        parent=arrs["parent"],
        node_level=arrs["node_level"],
        level_offsets=arrs["level_offsets"],
        leaf_of_particle=arrs["leaf_of_particle"],
        far_offsets=arrs["far_offsets"],
        far_sources=arrs["far_sources"],
        near_offsets=arrs["near_offsets"],
        near_leaves=arrs["near_leaves"],
        centers_f64=arrs["centers_f64"].reshape(-1, 3),
        radii_f64=arrs["radii_f64"],
        m2l_targets=tg[order].astype(np.int32),
        far_gears=arrs.get("far_gears"),
        gear_orders=None if gear_orders is None else tuple(int(o) for o in gear_orders),
    )


def build_topology(positions, masses, *, leaf_size: int = 16, theta: float = 0.6, device=None) -> Topology:
    """Tree + lists on the host (``jb_tree_build``), or on the GPU
    (``jb_tree_build_device``, the same arrays bit for bit) when ``device`` is
    a CUDA device."""
    if device is not None and str(device).startswith("cuda"):
        return build_topology_device(positions, masses, leaf_size=leaf_size, theta=theta, device=device)
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3))
    mass = np.ascontiguousarray(np.asarray(masses, dtype=np.float64).reshape(-1))
    n = pos.shape[0]
    if mass.shape[0] != n:
        raise ValueError("positions and masses disagree in length")
    lb = _lib.lib()
    h = ctypes.c_void_p()
    _lib.check(lb.jb_tree_build(n, pos.ctypes.data, mass.ctypes.data, int(leaf_size), float(theta),
                                ctypes.byref(h)), "jb_tree_build")
    try:
        info = _lib.TreeInfo()
        _lib.check(lb.jb_tree_info(h, ctypes.byref(info)), "jb_tree_info")
        arrs = _copy_fields(lb.jb_tree_copy, h, n, info)
    finally:
        lb.jb_tree_free(h)
    return _topology(n, info, arrs, leaf_size, theta)


def device_view(ptr, shape, dtype, device):
    """Zero-copy torch view (``__cuda_array_interface__`` v3) of device memory
    owned by a library handle; valid while the handle lives."""
    import torch

    dtype = np.dtype(dtype)
    shape = tuple(int(x) for x in shape)
    if int(np.prod(shape)) == 0:
        return torch.zeros(shape, dtype=torch.from_numpy(np.zeros(0, dtype)).dtype, device=device)

    class _View:
        __cuda_array_interface__ = {"shape": shape, "typestr": dtype.str, "data": (int(ptr), False), "version": 3,
                                    "strides": None}

    return torch.as_tensor(_View(), device=device)


class DeviceTree:
    """Owner of a ``jb_tree_build_device`` handle: the tree and lists of a
    particle set, resident on the GPU.  ``field(name)`` is a zero-copy torch
    view of one array (valid while the handle lives); ``topology()`` copies
    everything back into a :class:`Topology`.  Use as a context manager or
    call ``free()``."""

    def __init__(self, positions, masses, *, leaf_size: int = 16, theta: float = 0.6, device="cuda"):
        import torch

        self._torch = torch
        pos = torch.as_tensor(positions).to(device=device, dtype=torch.float64).reshape(-1, 3).contiguous()
        mass = torch.as_tensor(masses).to(device=device, dtype=torch.float64).reshape(-1).contiguous()
        n = pos.shape[0]
        if mass.shape[0] != n:
            raise ValueError("positions and masses disagree in length")
        self.n, self.leaf_size, self.theta, self.device = int(n), int(leaf_size), float(theta), pos.device
        self._lb = _lib.lib()
        self._h = ctypes.c_void_p()
        stream = torch.cuda.current_stream(pos.device).cuda_stream
        _lib.check(self._lb.jb_tree_build_device(n, pos.data_ptr(), mass.data_ptr(), self.leaf_size, self.theta,
                                                 stream, ctypes.byref(self._h)), "jb_tree_build_device")
        self.info = _lib.TreeInfo()
        _lib.check(self._lb.jb_dtree_info(self._h, ctypes.byref(self.info)), "jb_dtree_info")
        self.sizes = _field_sizes(self.n, self.info)
        self.gear_orders = None  # set by adaptive_walk

    def adaptive_walk(self, power, force_scale, *, G: float, eps: float, theta_max: float = 1.0,
                      gear_orders=(8,)) -> None:
        """Replaces the lists by those of the error-controlled walk
        (jb_dtree_adaptive_walk: Dehnen eq. (15)/(16a) acceptance, target-
        centric, per-pair gears).  power: float64 (num_nodes, P+1) Dehnen
        source powers; force_scale: float32 (num_nodes,) -- both on this
        tree's device, in its node order."""
        torch = self._torch
        orders = np.ascontiguousarray(np.asarray(gear_orders, dtype=np.int32))
        pw = power.to(device=self.device, dtype=torch.float64).contiguous()
        fs = force_scale.to(device=self.device, dtype=torch.float32).contiguous()
        if pw.dim() != 2 or pw.shape[0] != self.info.num_nodes or fs.shape != (self.info.num_nodes,):
            raise ValueError("power must be (num_nodes, P+1) and force_scale (num_nodes,)")
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._lb.jb_dtree_adaptive_walk(self._h, int(pw.shape[1]), pw.data_ptr(), fs.data_ptr(),
                                                   float(G), float(eps), float(theta_max), int(orders.size),
                                                   orders.ctypes.data, stream), "jb_dtree_adaptive_walk")
        _lib.check(self._lb.jb_dtree_info(self._h, ctypes.byref(self.info)), "jb_dtree_info")
        self.sizes = _field_sizes(self.n, self.info)
        self.gear_orders = tuple(int(o) for o in orders)

    def field(self, name: str):
        fid, dt = _lib.TREE_FIELDS[name]
        return device_view(self._lb.jb_dtree_field(self._h, fid), (self.sizes[name],), dt, self.device)

    def topology(self) -> Topology:
        arrs = _copy_fields(self._lb.jb_dtree_copy, self._h, self.n, self.info, with_gears=self.gear_orders is not None)
        return _topology(self.n, self.info, arrs, self.leaf_size, self.theta, self.gear_orders)

    def free(self) -> None:
        if self._h:
            self._lb.jb_dtree_free(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()

    def __del__(self):
        try:
            self.free()
        except Exception:  # interpreter shutdown
            pass


def build_topology_device(positions, masses, *, leaf_size: int = 16, theta: float = 0.6, device="cuda") -> Topology:
    """The tree and lists built on the GPU by ``jb_tree_build_device``
    (csrc/tree_gpu.cu) from float64 copies of the inputs on ``device``; the
    arrays are copied back into the same :class:`Topology` the host build
    returns."""
    with DeviceTree(positions, masses, leaf_size=leaf_size, theta=theta, device=device) as dtree:
        return dtree.topology()
