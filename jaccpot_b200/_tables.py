"""Constant tables for the CUDA kernels, generated at build time.

The only non-trivial constants of the real-basis operators are the per-degree
x<->z swap matrices ``B_U`` (multipole side; the local side uses the
transpose).  They follow Dehnen (2014) eq. 63 for the complex basis and the
no-sqrt2 real conversion ``B_U = Q B_complex^T Q^-1`` exactly as
jaccpot/operators/real_dehnen_q.py:49-143 and :300-380 define them; this module
restates that construction in numpy (float64) and writes
``csrc/generated/bu_tables.h`` as a static ``__constant__`` initialiser, so the
kernels need no run-time upload.

``bu_nonzero`` is the sparsity rule the unrolled kernels rely on to skip the
zero entries at compile time: ``B_U`` keeps the cos class (m >= 0) and the sin
class (m < 0) apart (it preserves parity in y) and inside each class only the
entries whose z-parity matches the source's x-parity survive.  ``generate``
asserts that every entry outside that pattern is exactly zero.
"""

from __future__ import annotations

from pathlib import Path

import numpy as np

MAX_ORDER = 10


def _complex_b(ell: int) -> np.ndarray:
    prev = np.ones((1, 1))
    for n in range(ell):
        nn = n + 1
        w = 2 * nn + 1

        def get(m, l):
            if abs(m) > n or abs(l) > n:
                return 0.0
            return prev[m + n, l + n]

        nxt = np.zeros((w, w))
        for mt in range(-nn, nn + 1):
            for lt in range(-nn, nn + 1):
                if abs(mt) <= n:
                    v = 0.5 * (get(mt, lt - 1) - get(mt, lt + 1))
                elif mt == n + 1:
                    v = 0.5 * (get(n, lt - 1) + get(n, lt + 1) + 2.0 * get(n, lt))
                else:
                    v = 0.5 * (get(-n, lt - 1) + get(-n, lt + 1) - 2.0 * get(-n, lt))
                nxt[mt + nn, lt + nn] = v
        prev = nxt
    return prev


def _q(ell: int) -> np.ndarray:
    w = 2 * ell + 1
    q = np.zeros((w, w), dtype=np.complex128)
    q[ell, ell] = 1.0
    for m in range(1, ell + 1):
        ph = (-1.0) ** m
        q[ell + m, ell + m] = 0.5
        q[ell + m, ell - m] = 0.5 * ph
        q[ell - m, ell + m] = -0.5j
        q[ell - m, ell - m] = 0.5j * ph
    return q


def bu_matrix(ell: int) -> np.ndarray:
    """Real multipole-side swap matrix for degree ``ell`` (float64)."""
    q = _q(ell)
    b = _complex_b(ell)
    return np.real(q @ b.T @ np.linalg.inv(q))


def bu_nonzero(ell: int, i: int, j: int) -> bool:
    """Compile-time sparsity rule of ``B_U`` (row i, column j of degree ell)."""
    mi, mj = i - ell, j - ell
    if (mi >= 0) != (mj >= 0):
        return False
    if mi >= 0:
        return (ell + mi + mj) % 2 == 0
    return (ell + abs(mi) + abs(mj)) % 2 == 1


def bu_offset(ell: int) -> int:
    return sum((2 * l + 1) ** 2 for l in range(ell))


def generate(out_path: Path, max_order: int = MAX_ORDER) -> Path:
    vals = []
    for ell in range(max_order + 1):
        b = bu_matrix(ell)
        w = 2 * ell + 1
        for i in range(w):
            for j in range(w):
                if not bu_nonzero(ell, i, j):
                    if b[i, j] != 0.0 and abs(b[i, j]) > 1e-12:
                        raise AssertionError(f"B_U sparsity rule broken at l={ell} ({i},{j})")
                    b[i, j] = 0.0
        vals.extend(b.reshape(-1).tolist())
    lines = [
        "// Generated by jaccpot_b200/_tables.py -- do not edit.",
        "// B_U per degree l (row-major (2l+1)^2), offset sum_{k<l} (2k+1)^2.",
        "#pragma once",
        f"#define JB_BU_MAX_ORDER {max_order}",
        f"static __constant__ float c_BU[{len(vals)}] = {{",
    ]
    for k in range(0, len(vals), 6):
        lines.append("  " + ", ".join(f"{float(np.float32(v))!r}f" for v in vals[k : k + 6]) + ",")
    lines.append("};")
    text = "\n".join(lines) + "\n"
    out_path.parent.mkdir(parents=True, exist_ok=True)
    if not out_path.exists() or out_path.read_text() != text:
        out_path.write_text(text)
    return out_path


if __name__ == "__main__":
    generate(Path(__file__).resolve().parent / "csrc" / "generated" / "bu_tables.h")
