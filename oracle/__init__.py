"""CPU oracle for the FMM evaluation pass — TEST INFRASTRUCTURE ONLY.

A ctypes front end to ``oracle/fmm_oracle.cpp``, the C++ restatement of
jaccpot's real-basis (Dehnen, no-sqrt2) operators and evaluation pass.  Only
``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` may
import this package; the product (``jaccpot_b200``) never does.

Parity status: pinned.  The operators are checked against the reference's own
known-answer identities (``tests/unit/operators/test_real_harmonics.py``) and
the pass against the reference's committed golden accelerations
(``tests/characterization/golden/*.npz``), regenerated inputs included; see
``tests/test_oracle_golden.py``.

All arrays are numpy, C-contiguous; ``dtype`` is float64 or float32 and selects
the ``_f64`` / ``_f32`` instantiation.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "_build" / "libjaccpot_oracle.so"
_lib = None


def build(force: bool = False) -> Path:
    """Compile the oracle library with ``make`` (g++ -O3 -fopenmp)."""
    srcs = [_HERE / "fmm_oracle.cpp", _HERE / "tree_oracle.cpp"]
    if force or not _LIB_PATH.exists() or any(_LIB_PATH.stat().st_mtime < s.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(_LIB_PATH))
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _sfx(dtype) -> str:
    dt = np.dtype(dtype)
    if dt == np.float64:
        return "f64"
    if dt == np.float32:
        return "f32"
    raise TypeError(f"oracle supports float32/float64, got {dt}")


def _c(a, dtype) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=dtype)


def sh_size(p: int) -> int:
    return (p + 1) * (p + 1)


def set_threads(n: int) -> int:
    f = lib().oracle_set_threads
    f.restype = ctypes.c_int
    return int(f(ctypes.c_int(n)))


def bu_matrix(ell: int) -> np.ndarray:
    """B_U for degree ``ell`` (real_dehnen_q.py:300-380), float64."""
    w = 2 * ell + 1
    out = np.zeros((w, w), dtype=np.float64)
    lib().oracle_bu(ctypes.c_int(ell), _p(out))
    return out


def _batched(name, p, a, d, dtype, out_cols):
    dtype = np.dtype(dtype)
    a = _c(a, dtype)
    d = _c(d, dtype).reshape(-1, 3)
    n = d.shape[0]
    out = np.zeros((n, out_cols), dtype=dtype)
    getattr(lib(), f"oracle_{name}_{_sfx(dtype)}")(
        ctypes.c_int(p), ctypes.c_int64(n), _p(a), _p(d), _p(out)
    )
    return out


def p2m(p, deltas, masses, dtype=np.float64):
    """M_n^m = m U_n^m(delta), delta = x - centre (real_p2m_l2p.py:51)."""
    dtype = np.dtype(dtype)
    d = _c(deltas, dtype).reshape(-1, 3)
    m = _c(masses, dtype).reshape(-1)
    out = np.zeros((d.shape[0], sh_size(p)), dtype=dtype)
    getattr(lib(), f"oracle_p2m_{_sfx(dtype)}")(
        ctypes.c_int(p), ctypes.c_int64(d.shape[0]), _p(d), _p(m), _p(out)
    )
    return out


def l2p(p, locals_, deltas, dtype=np.float64):
    """(potential, grad_delta) of sum F U(delta), delta = centre - x."""
    dtype = np.dtype(dtype)
    F = _c(locals_, dtype).reshape(-1, sh_size(p))
    d = _c(deltas, dtype).reshape(-1, 3)
    n = d.shape[0]
    pot = np.zeros(n, dtype=dtype)
    grad = np.zeros((n, 3), dtype=dtype)
    getattr(lib(), f"oracle_l2p_{_sfx(dtype)}")(
        ctypes.c_int(p), ctypes.c_int64(n), _p(F), _p(d), _p(pot), _p(grad)
    )
    return pot, grad


def m2m(p, mult, deltas, dtype=np.float64):
    """delta = source - destination (child - parent)."""
    return _batched("m2m", p, mult, deltas, dtype, sh_size(p))


def l2l(p, loc, deltas, dtype=np.float64):
    """delta = old - new centre (parent - child)."""
    return _batched("l2l", p, loc, deltas, dtype, sh_size(p))


def m2l(p, mult, deltas, dtype=np.float64):
    """delta = target - source centre."""
    return _batched("m2l", p, mult, deltas, dtype, sh_size(p))


class Pass:
    """Runs the whole evaluation pass on a topology (see jaccpot_b200.tree)."""

    def __init__(self, topo, dtype=np.float64):
        self.t = topo
        self.dtype = np.dtype(dtype)
        self.sfx = _sfx(self.dtype)
        i32 = lambda a: _c(a, np.int32)
        i64 = lambda a: _c(a, np.int64)
        self.ranges = i32(topo.node_ranges)
        self.left = i32(topo.left_child)
        self.right = i32(topo.right_child)
        self.level_off = i32(topo.level_offsets)
        self.far_off = i64(topo.far_offsets)
        self.far_src = i32(topo.far_sources)
        self.near_off = i64(topo.near_offsets)
        self.near_leaf = i32(topo.near_leaves)
        self.leaf_of = i32(topo.leaf_of_particle)

    def com(self, pos, mass):
        pos = _c(pos, self.dtype)
        mass = _c(mass, self.dtype)
        out = np.zeros((self.t.num_nodes, 3), dtype=self.dtype)
        getattr(lib(), f"oracle_com_{self.sfx}")(
            ctypes.c_int64(pos.shape[0]), _p(pos), _p(mass), ctypes.c_int(self.t.num_nodes),
            _p(self.ranges), _p(out))
        return out

    def upward(self, p, pos, mass, centers):
        pos = _c(pos, self.dtype)
        mass = _c(mass, self.dtype)
        centers = _c(centers, self.dtype)
        mult = np.zeros((self.t.num_nodes, sh_size(p)), dtype=self.dtype)
        getattr(lib(), f"oracle_upward_{self.sfx}")(
            ctypes.c_int(p), _p(pos), _p(mass), ctypes.c_int(self.t.num_nodes),
            ctypes.c_int(self.t.num_internal), _p(self.ranges), _p(self.left), _p(self.right),
            _p(self.level_off), ctypes.c_int(self.t.num_levels), _p(centers), _p(mult))
        return mult

    def m2l_accumulate(self, p, mult, centers, loc=None):
        mult = _c(mult, self.dtype)
        centers = _c(centers, self.dtype)
        if loc is None:
            loc = np.zeros((self.t.num_nodes, sh_size(p)), dtype=self.dtype)
        loc = _c(loc, self.dtype)
        getattr(lib(), f"oracle_m2l_accumulate_{self.sfx}")(
            ctypes.c_int(p), ctypes.c_int(self.t.num_nodes), _p(mult), _p(centers),
            _p(self.far_off), _p(self.far_src), _p(loc))
        return loc

    def l2l_cascade(self, p, centers, loc):
        loc = np.array(loc, dtype=self.dtype, order="C", copy=True)
        centers = _c(centers, self.dtype)
        getattr(lib(), f"oracle_l2l_cascade_{self.sfx}")(
            ctypes.c_int(p), _p(self.left), _p(self.right), _p(self.level_off),
            ctypes.c_int(self.t.num_levels), _p(centers), _p(loc))
        return loc

    def evaluate(self, p, pos, mass, centers, loc, G, eps2, want_pot=True):
        pos = _c(pos, self.dtype)
        mass = _c(mass, self.dtype)
        centers = _c(centers, self.dtype)
        loc = _c(loc, self.dtype)
        acc = np.zeros((pos.shape[0], 3), dtype=self.dtype)
        pot = np.zeros(pos.shape[0], dtype=self.dtype) if want_pot else None
        dt = ctypes.c_double if self.dtype == np.float64 else ctypes.c_float
        getattr(lib(), f"oracle_evaluate_{self.sfx}")(
            ctypes.c_int(p), _p(pos), _p(mass), ctypes.c_int(self.t.num_nodes),
            ctypes.c_int(self.t.num_internal), _p(self.ranges), _p(centers), _p(loc),
            _p(self.near_off), _p(self.near_leaf), dt(G), dt(eps2), _p(acc),
            _p(pot) if pot is not None else None)
        return acc, pot

    def evaluate_targets(self, p, pos, mass, centers, loc, targets_sorted, G, eps2):
        pos = _c(pos, self.dtype)
        mass = _c(mass, self.dtype)
        centers = _c(centers, self.dtype)
        loc = _c(loc, self.dtype)
        ts = _c(targets_sorted, np.int32)
        nt = ts.shape[0]
        acc = np.zeros((nt, 3), dtype=self.dtype)
        pot = np.zeros(nt, dtype=self.dtype)
        dt = ctypes.c_double if self.dtype == np.float64 else ctypes.c_float
        getattr(lib(), f"oracle_evaluate_targets_{self.sfx}")(
            ctypes.c_int(p), _p(pos), _p(mass), ctypes.c_int(self.t.num_internal),
            _p(self.ranges), _p(centers), _p(loc), _p(self.near_off), _p(self.near_leaf),
            _p(self.leaf_of), ctypes.c_int64(nt), _p(ts), dt(G), dt(eps2), _p(acc), _p(pot))
        return acc, pot

    def evaluate_range(self, p, pos, mass, centers, loc, leaf_lo, leaf_hi, G, eps2):
        """evaluate() for the leaves [leaf_lo, leaf_hi) only; the other rows of
        the returned (N, 3) array are zero."""
        pos = _c(pos, self.dtype)
        mass = _c(mass, self.dtype)
        centers = _c(centers, self.dtype)
        loc = _c(loc, self.dtype)
        acc = np.zeros((pos.shape[0], 3), dtype=self.dtype)
        dt = ctypes.c_double if self.dtype == np.float64 else ctypes.c_float
        getattr(lib(), f"oracle_evaluate_range_{self.sfx}")(
            ctypes.c_int(p), _p(pos), _p(mass), ctypes.c_int(self.t.num_nodes),
            ctypes.c_int(self.t.num_internal), _p(self.ranges), _p(centers), _p(loc),
            _p(self.near_off), _p(self.near_leaf), dt(G), dt(eps2), ctypes.c_int(leaf_lo),
            ctypes.c_int(leaf_hi), _p(acc), None)
        return acc

    def run(self, p, pos_sorted, mass_sorted, G=1.0, eps2=0.0):
        """Whole pass on sorted particles; returns a dict of every stage."""
        centers = self.com(pos_sorted, mass_sorted)
        mult = self.upward(p, pos_sorted, mass_sorted, centers)
        loc = self.m2l_accumulate(p, mult, centers)
        loc = self.l2l_cascade(p, centers, loc)
        acc, pot = self.evaluate(p, pos_sorted, mass_sorted, centers, loc, G, eps2)
        return {"centers": centers, "multipoles": mult, "locals": loc, "acc": acc, "pot": pot}


_TREE_FIELDS = (("permutation", np.int64, "n"), ("node_ranges", np.int32, "2nodes"),
                ("left_child", np.int32, "internal"), ("right_child", np.int32, "internal"),
                ("parent", np.int32, "nodes"), ("node_level", np.int32, "nodes"),
                ("level_offsets", np.int32, "levels+1"), ("leaf_of_particle", np.int32, "n"),
                ("far_offsets", np.int64, "nodes+1"), ("far_sources", np.int32, "far"),
                ("near_offsets", np.int64, "leaves+1"), ("near_leaves", np.int32, "near"),
                ("centers_f64", np.float64, "3nodes"), ("radii_f64", np.float64, "nodes"))


def tree_build(pos, mass, leaf_size, theta):
    """The oracle's own tree + lists (oracle/tree_oracle.cpp, a transcription
    of oracle/tree.py): a namespace with the Topology fields that Pass reads."""
    from types import SimpleNamespace

    pos = _c(pos, np.float64).reshape(-1, 3)
    mass = _c(mass, np.float64).reshape(-1)
    n = pos.shape[0]
    sizes = np.zeros(6, np.int64)
    f = lib().oracle_tree_build
    f.restype = ctypes.c_void_p
    h = f(ctypes.c_int64(n), _p(pos), _p(mass), ctypes.c_int(int(leaf_size)), ctypes.c_double(float(theta)),
          _p(sizes))
    if not h:
        raise ValueError("oracle_tree_build: bad arguments")
    nodes, internal, leaves, levels, far, near = (int(v) for v in sizes)
    dims = {"n": n, "2nodes": 2 * nodes, "internal": internal, "nodes": nodes, "levels+1": levels + 1,
            "nodes+1": nodes + 1, "far": far, "leaves+1": leaves + 1, "near": near, "3nodes": 3 * nodes}
    out = SimpleNamespace(num_particles=n, num_nodes=nodes, num_internal=internal, num_leaves=leaves,
                          num_levels=levels, leaf_size=int(leaf_size), theta=float(theta))
    try:
        for fid, (name, dt, dim) in enumerate(_TREE_FIELDS):
            a = np.empty(max(dims[dim], 1), dtype=dt)
            if lib().oracle_tree_copy(ctypes.c_void_p(h), ctypes.c_int(fid), _p(a)) != 0:
                raise RuntimeError(f"oracle_tree_copy({name})")
            setattr(out, name, a[:dims[dim]])
    finally:
        lib().oracle_tree_free(ctypes.c_void_p(h))
    out.node_ranges = out.node_ranges.reshape(-1, 2)
    out.centers_f64 = out.centers_f64.reshape(-1, 3)
    out.inverse_permutation = np.empty_like(out.permutation)
    out.inverse_permutation[out.permutation] = np.arange(n, dtype=np.int64)
    return out


def direct_sum(pos, mass, targets=None, G=1.0, eps2=0.0):
    """FP64 O(N*T) direct sum (runtime/reference.py:292); returns (acc, pot)."""
    pos = _c(pos, np.float64)
    mass = _c(mass, np.float64)
    n = pos.shape[0]
    tg = np.arange(n, dtype=np.int64) if targets is None else _c(targets, np.int64)
    acc = np.zeros((tg.shape[0], 3), dtype=np.float64)
    pot = np.zeros(tg.shape[0], dtype=np.float64)
    lib().oracle_direct_f64(
        ctypes.c_int64(n), _p(pos), _p(mass), ctypes.c_int64(tg.shape[0]), _p(tg),
        ctypes.c_double(G), ctypes.c_double(eps2), _p(acc), _p(pot))
    return acc, pot
