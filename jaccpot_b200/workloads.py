"""Seeded synthetic particle sets with the shapes and distributions of the
benchmark configurations (uniform cube, Plummer sphere, 64-clump Plummer
mixture).  The Plummer sampler follows the inverse-CDF radius of
jaccpot/bench/validation/mac_error_distribution.py:79-94 (truncated at 20
scale radii, isotropic directions)."""

from __future__ import annotations

import numpy as np


def uniform_cube(n: int, seed: int = 0, dtype=np.float32):
    """Positions i.i.d. U[-1,1]^3, masses U[0.5,1.5]."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1.0, 1.0, size=(n, 3))
    mass = rng.uniform(0.5, 1.5, size=n)
    return pos.astype(dtype), mass.astype(dtype)


def _plummer_positions(rng, n: int, scale: float = 1.0) -> np.ndarray:
    u = rng.uniform(size=n)
    radius = scale * u ** (1.0 / 3.0) / np.sqrt(np.maximum(1.0 - u ** (2.0 / 3.0), 1e-12))
    radius = np.minimum(radius, 20.0 * scale)
    cos_t = rng.uniform(-1.0, 1.0, size=n)
    sin_t = np.sqrt(np.maximum(1.0 - cos_t ** 2, 0.0))
    phi = rng.uniform(0.0, 2.0 * np.pi, size=n)
    return np.stack([radius * sin_t * np.cos(phi), radius * sin_t * np.sin(phi), radius * cos_t], axis=1)


def plummer(n: int, seed: int = 0, dtype=np.float32):
    """Plummer sphere (scale 1, truncated at r = 20), equal masses 1/N."""
    rng = np.random.default_rng(seed)
    pos = _plummer_positions(rng, n, 1.0)
    mass = np.full(n, 1.0 / n)
    return pos.astype(dtype), mass.astype(dtype)


def clustered(n: int, seed: int = 0, dtype=np.float32, clumps: int = 64):
    """Mixture of `clumps` Plummer spheres: centres U[-50,50]^3, scale radii
    log-uniform in [0.1, 2], membership weights ~ Dirichlet(1), masses
    lognormal(0, 0.5) normalised to sum 1."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-50.0, 50.0, size=(clumps, 3))
    scales = np.exp(rng.uniform(np.log(0.1), np.log(2.0), size=clumps))
    weights = rng.dirichlet(np.ones(clumps))
    counts = rng.multinomial(n, weights)
    parts = []
    for c in range(clumps):
        if counts[c]:
            parts.append(centres[c] + _plummer_positions(rng, int(counts[c]), float(scales[c])))
    pos = np.concatenate(parts, axis=0)
    pos = pos[rng.permutation(n)]
    mass = rng.lognormal(0.0, 0.5, size=n)
    mass = mass / mass.sum()
    return pos.astype(dtype), mass.astype(dtype)


GENERATORS = {"uniform": uniform_cube, "plummer": plummer, "clustered": clustered}


def relative_errors(est: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """Per-particle |a - a_ref| / |a_ref| (mac_error_distribution.py:192-200)."""
    est = np.asarray(est, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    return np.linalg.norm(est - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-300)
