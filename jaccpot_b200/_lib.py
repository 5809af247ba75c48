"""ctypes binding of ``libjaccpot_b200.so`` (the C ABI in include/jaccpot_b200.h).

The library is built in-tree by :mod:`jaccpot_b200.build`.  There is no
fallback: if it is missing, or a CUDA entry point reports an error, the call
raises.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "_lib" / "libjaccpot_b200.so"

JB_OK = 0
ERRORS = {
    1: "invalid argument",
    2: "unsupported expansion order",
    3: "CUDA error",
    4: "list index out of range",
    5: "workspace too small",
    6: "host allocation failed",
    7: "non-finite input",
    8: "mode not supported for this order",
}
JB_MAX_ORDER = 10
JB_M2L_FP32, JB_M2L_SPLIT_BF16 = 0, 1
JB_P2P_FP32, JB_P2P_KAHAN, JB_P2P_POTENTIAL, JB_P2P_FAR_ONLY, JB_P2P_NEAR_ONLY = 0, 1, 2, 4, 8
JB_P2P_NEAR_FIRST, JB_P2P_FAR_AFTER = 16, 32
JB_LEAF_EVAL_NOALLOC_MAX_SLOTS = 16384
JB_MAX_LEAF_OCCUPANCY = 64
JB_MIXED_GEAR_SEGMENTS = 4
JB_LEAF_ERR_OCCUPANCY, JB_LEAF_ERR_SLOT = 1, 2
(JB_SCHED_UNITS, JB_SCHED_AUX, JB_SCHED_RUNS, JB_SCHED_SPLIT, JB_SCHED_FAR_SOURCES, JB_SCHED_GEAR_OFFSETS,
 JB_SCHED_TARGETS, JB_SCHED_PAIRS_PER_GEAR) = range(8)

# jb_tree_copy field ids
TREE_FIELDS = {
    "permutation": (0, "int64"),
    "node_ranges": (1, "int32"),
    "left_child": (2, "int32"),
    "right_child": (3, "int32"),
    "parent": (4, "int32"),
    "node_level": (5, "int32"),
    "level_offsets": (6, "int32"),
    "leaf_of_particle": (7, "int32"),
    "far_offsets": (8, "int64"),
    "far_sources": (9, "int32"),
    "near_offsets": (10, "int64"),
    "near_leaves": (11, "int32"),
    "centers_f64": (12, "float64"),
    "radii_f64": (13, "float64"),
    "far_gears": (14, "int32"),
}


class JBError(RuntimeError):
    pass


class TreeInfo(ctypes.Structure):
    _fields_ = [
        ("num_particles", ctypes.c_int64),
        ("num_nodes", ctypes.c_int32),
        ("num_internal", ctypes.c_int32),
        ("num_leaves", ctypes.c_int32),
        ("num_levels", ctypes.c_int32),
        ("num_far_pairs", ctypes.c_int64),
        ("num_near_pairs", ctypes.c_int64),
        ("max_leaf_occupancy", ctypes.c_int32),
    ]


_lib = None

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_F = ctypes.c_float
_D = ctypes.c_double

_SIGNATURES = {
    "jb_tree_build": [_I64, _P, _P, _I, _D, ctypes.POINTER(_P)],
    "jb_tree_info": [_P, ctypes.POINTER(TreeInfo)],
    "jb_tree_copy": [_P, _I, _P],
    "jb_tree_free": [_P],
    "jb_tree_build_device": [_I64, _P, _P, _I, _D, _P, ctypes.POINTER(_P)],
    "jb_dtree_info": [_P, ctypes.POINTER(TreeInfo)],
    "jb_dtree_field": [_P, _I],
    "jb_dtree_copy": [_P, _I, _P],
    "jb_dtree_free": [_P],
    "jb_dtree_adaptive_walk": [_P, _I, _P, _P, _D, _D, _D, _I, _P, _P],
    "jb_node_dehnen_power": [_I, _I, _P, _I, _P, _P],
    "jb_far_dehnen_gears": [_I64, _P, _P, _P, _P, _I, _P, _P, _D, _D, _I, _P, _P, _P],
    "jb_node_force_scale": [_I, _I, _P, _P, _P, _I, _P, _P, _P, _P],
    "jb_set_level_split": [_I, _I],
    "jb_set_leaf_form": [_I],
    "jb_set_m2l_fetch": [_I],
    "jb_graph_instantiate": [_P, _I, ctypes.POINTER(_P)],
    "jb_graph_launch": [_P, _P],
    "jb_graph_exec_destroy": [_P],
    "jb_far_reverse_index": [_I, _P, _P, _P, _P],
    "jb_m2l_weighted": [_I, _I, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P],
    "jb_leaf_eval_weighted": [_I, _I, _P, _P, _I, _P, _I, _I, _P, _P, _P, _P, _P, _P, _F, _F, _P, _P, _I, _P, _P],
    "jb_m2l_schedule_device": [_I, _P, _I, _I, _P, _P, ctypes.POINTER(_P)],
    "jb_leaf_schedule_device": [_I, _I, _P, _P, _P, _I, _I, _I, _P, ctypes.POINTER(_P)],
    "jb_gear_schedule_device": [_I, _P, _P, _P, _I, _I, _P, ctypes.POINTER(_P)],
    "jb_gear_mixed_schedule_device": [_I, _P, _P, _P, _I, _P, _I, _I, _P, ctypes.POINTER(_P)],
    "jb_dsched_info": [_P, _P],
    "jb_dsched_field": [_P, _I],
    "jb_dsched_free": [_P],
    "jb_coeff_stride": [_I],
    "jb_last_cuda_error": [],
    "jb_gather_sorted": [_I64, _P, _P, _P, _P, _P],
    "jb_validate_lists": [_I, _I, _P, _P, _P, _P, _I64, _P, _P, _I64, _P, _P],
    "jb_validate_leaves": [_I, _I, _P, _I, _P, _P],
    "jb_leaf_eval_errors": [ctypes.POINTER(_I), _I, _P],
    "jb_p2m": [_I, _P, _I, _I, _P, _P, _P, _P],
    "jb_m2m_level": [_I, _I, _I, _P, _P, _P, _P, _P, _P],
    "jb_m2l": [_I, _I, _I, _P, _P, _P, _P, _P, _P, _I, _P, _P],
    "jb_m2l_gears": [_I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P],
    "jb_m2l_mixed": [_I, _I, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P],
    "jb_m2l_split": [_I, _I, _I, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P],
    "jb_m2l_split_units": [_I, _I, _P, _P, _P, _P, _P, _P, _I, _P, _P, _P],
    "jb_l2l_leaves": [_I, _I, _P, _P, _P, _P, _P],
    "jb_l2l_level": [_I, _I, _I, _P, _P, _P, _P, _P],
    "jb_leaf_eval": [_I, _I, _P, _I, _I, _P, _P, _P, _P, _P, _P, _F, _F, _P, _P, _I, _P, _P],
    "jb_leaf_eval_noalloc": [_I, _I, _P, _I, _I, _P, _P, _P, _P, _P, _P, _F, _F, _P, _I, _I, _P, _P],
    "jb_eval_targets": [_I, _P, _I, _P, _P, _P, _P, _P, _P, _I64, _P, _F, _F, _P, _P],
    "jb_adj_near": [_P, _P, _I, _I, _P, _P, _P, _P, _F, _F, _P, _P, _I, _P, _P],
    "jb_adj_leaf_far": [_I, _P, _P, _I, _I, _P, _P, _P, _F, _P, _P, _P, _P],
    "jb_adj_l2l_level": [_I, _I, _I, _P, _P, _P, _P, _P, _P, _P],
    "jb_adj_m2l": [_I, _I, _P, _P, _P, _P, _P, _P, _I, _P, _P],
    "jb_adj_m2l_centers": [_I, _I, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    "jb_adj_m2m_level": [_I, _I, _I, _P, _P, _P, _P, _P, _P, _P],
    "jb_adj_p2m": [_I, _P, _I, _I, _P, _P, _P, _P, _P, _P],
    "jb_gear_param_count": [],
    "jb_gear_node_features": [_I, _I, _I, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P],
    "jb_gear_pair_features": [_I64, _P, _P, _P, _P, _P, _P, _P, _F, _P, _P],
    "jb_gear_errors": [_I64, _P, _P, _P, _P, _P, _P, _P, _F, _P, _P],
    "jb_gear_train_grad": [_I, _P, _P, _P, _P, _P, _P],
    "jb_gear_adam": [_I, _P, _F, _F, _F, _F, _F, _I, _P, _P, _P, _P, _P],
    "jb_gear_select": [_I64, _P, _P, _P, _P, _P, _P, _F, _P, _P, _F, _F, _P, _P],
    "jb_scatter_unsorted": [_I64, _P, _P, _P, _P, _P],
    "jb_gather_unsorted": [_I64, _P, _P, _P, _P, _P],
    "jb_direct_f64": [_I64, _P, _I64, _P, _D, _D, _P, _P],
    "jb_probe_throughput": [_I, _I, _I, _P, _P],
}

EXPORTED = tuple(_SIGNATURES)


def lib() -> ctypes.CDLL:
    """Loads the library (once); raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise JBError(
                f"{LIB_PATH} is missing: build it with `python -m jaccpot_b200.build` "
                "(there is no CPU fallback)"
            )
        lb = ctypes.CDLL(str(LIB_PATH))
        for name, args in _SIGNATURES.items():
            fn = getattr(lb, name)
            fn.argtypes = args
            fn.restype = ctypes.c_char_p if name == "jb_last_cuda_error" else (
                None if name in ("jb_tree_free", "jb_dtree_free", "jb_dsched_free") else (
                    ctypes.c_void_p if name in ("jb_dtree_field", "jb_dsched_field") else ctypes.c_int))
        _lib = lb
    return _lib


def check(status: int, what: str) -> None:
    if status != JB_OK:
        msg = ERRORS.get(status, f"status {status}")
        if status == 3:
            msg += ": " + (lib().jb_last_cuda_error() or b"").decode()
        raise JBError(f"{what} failed: {msg}")


def coeff_stride(p: int) -> int:
    s = lib().jb_coeff_stride(int(p))
    if s <= 0:
        raise JBError(f"expansion order {p} is outside [1, {JB_MAX_ORDER}]")
    return s
