"""Extracts the reference's golden outputs used by tests/test_oracle_golden.py.

The reference (jaccpot) commits outputs of its public API for seeded inputs:
  tests/characterization/golden/uni_real_n{256,1024}_p{2,4,6}.npz   accel (N,3) f64
  tests/characterization/golden/clu_real_n256_p4.npz                accel (N,3) f64 (clustered)
  tests/characterization/golden_modes/bkt_uni_real_n256_p4.npz      accel, potential
  tests/characterization/golden_grad/uni_real_n{128,256}_p{2,4}.npz grad_positions, grad_masses
They were produced with preset="accurate", theta 0.5, softening 1e-2, G 1
(leaf 8 for the forward cases, leaf 4 for the gradient cases) on inputs drawn
from jax.random.PRNGKey(0xC0FFEE), which tests/golden/jax_prng.py regenerates.

Usage: python tests/golden/make_fixtures.py REFERENCE_ROOT
(REFERENCE_ROOT: the jaccpot checkout holding tests/characterization/.)
Writes tests/golden/reference_goldens.npz (real-basis cases only).
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

FORWARD = ["uni_real_n256_p2", "uni_real_n256_p4", "uni_real_n256_p6", "uni_real_n1024_p4",
           "clu_real_n256_p4"]
MODES = ["bkt_uni_real_n256_p4"]
GRAD = ["uni_real_n128_p2", "uni_real_n128_p4", "uni_real_n256_p4"]


def main(ref_root: str) -> Path:
    base = Path(ref_root) / "tests" / "characterization"
    out = {}
    for c in FORWARD:
        out[f"{c}/accel"] = np.load(base / "golden" / f"{c}.npz")["accel"]
    for c in MODES:
        d = np.load(base / "golden_modes" / f"{c}.npz")
        out[f"{c}/accel"] = d["accel"]
        out[f"{c}/potential"] = d["potential"]
    for c in GRAD:
        d = np.load(base / "golden_grad" / f"{c}.npz")
        out[f"grad_{c}/grad_positions"] = d["grad_positions"]
        out[f"grad_{c}/grad_masses"] = d["grad_masses"]
    dst = Path(__file__).resolve().parent / "reference_goldens.npz"
    np.savez_compressed(dst, **out)
    return dst


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit(__doc__)
    print(main(sys.argv[1]))
