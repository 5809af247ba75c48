"""The C-ABI library loads without a GPU and exports every entry point that
include/*.h declares; argument validation answers without touching the
device."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

from jaccpot_b200 import _lib

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        names += re.findall(r"JB_API\s+[\w\s\*]+?\b(jb_\w+)\s*\(", h.read_text())
    return sorted(set(names))


def test_header_declares_the_pass():
    names = declared_symbols()
    for required in ("jb_tree_build", "jb_p2m", "jb_m2m_level", "jb_m2l", "jb_l2l_level", "jb_leaf_eval",
                     "jb_eval_targets", "jb_gather_sorted", "jb_scatter_unsorted", "jb_validate_lists"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert set(declared_symbols()) <= set(_lib.EXPORTED)


def test_argument_errors_without_a_device():
    lib = _lib.lib()
    assert lib.jb_coeff_stride(8) == 84
    assert lib.jb_coeff_stride(0) == 0 and lib.jb_coeff_stride(11) == 0
    assert lib.jb_p2m(8, None, 1, 0, None, None, None, None) == 1
    assert lib.jb_m2l(8, 0, -1, None, None, None, None, None, None, 0, None, None) == 1
    assert lib.jb_m2l(8, 9, 1, 1, 1, 1, 1, 1, 1, 0, None, None) == 8
    assert lib.jb_leaf_eval(8, 64, 1, 0, 1, 1, 1, 1, 1, 1, 1, 1.0, 0.0, 1, 1, 0, None, None) == 1
    # at most one of the part flags (near / far alone, or one half of the two-stream form)
    for a, b in ((_lib.JB_P2P_NEAR_FIRST, _lib.JB_P2P_FAR_AFTER), (_lib.JB_P2P_NEAR_ONLY, _lib.JB_P2P_FAR_AFTER),
                 (_lib.JB_P2P_FAR_ONLY, _lib.JB_P2P_NEAR_FIRST), (_lib.JB_P2P_FAR_ONLY, _lib.JB_P2P_NEAR_ONLY)):
        assert lib.jb_leaf_eval(8, a | b, 1, 0, 1, 1, 1, 1, 1, 1, 1, 1.0, 0.0, 1, 1, 0, None, None) == 1
    assert lib.jb_graph_instantiate(None, 1, ctypes.byref(ctypes.c_void_p())) == 1
    assert lib.jb_graph_instantiate(1, 2, ctypes.byref(ctypes.c_void_p())) == 1
    assert lib.jb_graph_launch(None, None) == 1 and lib.jb_graph_exec_destroy(None) == 1
    assert lib.jb_m2m_level(8, 5, 4, None, None, None, None, None, None) == 1
    assert lib.jb_gather_sorted(-1, None, None, None, None, None) == 1
    assert lib.jb_direct_f64(0, None, 0, None, 1.0, 0.0, None, None) == 1
    info = _lib.TreeInfo()
    assert lib.jb_tree_info(None, ctypes.byref(info)) == 1


def test_leaf_checks_refuse_bad_arguments_without_a_device():
    lib = _lib.lib()
    # max_occupancy outside [1, JB_MAX_LEAF_OCCUPANCY], null arrays
    assert lib.jb_validate_leaves(3, 1, 1, 65, 1, None) == 1
    assert lib.jb_validate_leaves(3, 1, 1, 0, 1, None) == 1
    assert lib.jb_validate_leaves(3, 1, None, 32, 1, None) == 1
    assert lib.jb_leaf_eval_errors(None, 0, None) == 1


def test_tensor_core_status_raises_on_the_host():
    """The split-BF16 M2L's status word: 1 (a barrier wait timed out) and 2
    (its drain timed out too) raise; 0 and the FP32 M2L do not."""
    torch = pytest.importorskip("torch")
    from jaccpot_b200 import engine

    ps = engine.Pass.__new__(engine.Pass)  # host logic only: no device pass is built
    ps.m2l_mode = _lib.JB_M2L_SPLIT_BF16
    ps._tc = None
    for word, msg in ((1, "incomplete"), (2, "must not be used")):
        ps._tc_status = torch.tensor([word], dtype=torch.int32)
        with pytest.raises(_lib.JBError, match=msg):
            ps.check_tc_status()
    ps._tc_status = torch.tensor([0], dtype=torch.int32)
    ps.check_tc_status()
    ps.m2l_mode = _lib.JB_M2L_FP32
    ps._tc_status = torch.tensor([1], dtype=torch.int32)
    ps.check_tc_status()  # the FP32 M2L has no status word
