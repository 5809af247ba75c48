"""Numpy restatement of JAX's default PRNG (threefry2x32), used only to
regenerate the inputs of the reference's golden fixtures, which store outputs
but not inputs (jaccpot tests/characterization/test_fmm_golden.py:166-187 draws
them from jax.random.PRNGKey(0xC0FFEE)).

Algorithm: Threefry-2x32 with 20 rounds (Salmon et al., "Parallel random
numbers: as easy as 1, 2, 3", SC'11), keyed and counted the way JAX's
``threefry_partitionable`` mode does it (the default since JAX 0.5): a key is
two uint32 words; ``split(key, n)`` and ``random_bits(key, shape)`` hash the
(hi, lo) words of the flat element index; 64-bit draws concatenate the two
output words; floats take the top mantissa bits (``uniform``), ``normal`` is
sqrt(2) * erfinv(u) with u uniform on (nextafter(-1, 0), 1).  ``randint``
(int64, the default integer type with 64-bit mode on) draws two 64-bit words
from the two halves of ``split(key)`` and folds them modulo the span, the
higher word weighted by 2**64 mod span (JAX's documented construction that
keeps the modulo bias at 2**-64 for any span).
"""

from __future__ import annotations

import numpy as np
from scipy.special import erfinv

_ROT = ((13, 15, 26, 6), (17, 29, 16, 24))
_M32 = np.uint64(0xFFFFFFFF)


def _rotl(x, r):
    return ((x << np.uint32(r)) | (x >> np.uint32(32 - r))).astype(np.uint32)


def threefry2x32(k0, k1, x0, x1):
    k0, k1 = np.uint32(k0), np.uint32(k1)
    ks = [k0, k1, np.uint32(k0 ^ k1 ^ np.uint32(0x1BD11BDA))]
    x0 = (np.asarray(x0, np.uint32) + ks[0]).astype(np.uint32)
    x1 = (np.asarray(x1, np.uint32) + ks[1]).astype(np.uint32)
    for blk in range(5):
        for r in _ROT[blk % 2]:
            x0 = (x0 + x1).astype(np.uint32)
            x1 = _rotl(x1, r)
            x1 = (x1 ^ x0).astype(np.uint32)
        x0 = (x0 + ks[(blk + 1) % 3]).astype(np.uint32)
        x1 = (x1 + ks[(blk + 2) % 3] + np.uint32(blk + 1)).astype(np.uint32)
    return x0, x1


def key(seed: int):
    s = int(seed)
    return (np.uint32((s >> 32) & 0xFFFFFFFF), np.uint32(s & 0xFFFFFFFF))


def _iota_hi_lo(n: int):
    idx = np.arange(n, dtype=np.uint64)
    return (idx >> np.uint64(32)).astype(np.uint32), (idx & _M32).astype(np.uint32)


def split(k, num: int = 2):
    hi, lo = _iota_hi_lo(num)
    a, b = threefry2x32(k[0], k[1], hi, lo)
    return [(a[i], b[i]) for i in range(num)]


def random_bits(k, shape, width: int):
    n = int(np.prod(shape))
    hi, lo = _iota_hi_lo(n)
    a, b = threefry2x32(k[0], k[1], hi, lo)
    if width == 64:
        bits = (a.astype(np.uint64) << np.uint64(32)) | b.astype(np.uint64)
    elif width == 32:
        bits = a ^ b
    else:
        raise ValueError(width)
    return bits.reshape(shape)


def uniform(k, shape, minval=0.0, maxval=1.0):
    """float64 uniform on [minval, maxval) (jax.random.uniform with dtype=float64)."""
    bits = random_bits(k, shape, 64)
    fb = (bits >> np.uint64(64 - 52)) | np.float64(1.0).view(np.uint64)
    f = fb.view(np.float64) - 1.0
    return np.maximum(minval, f * (maxval - minval) + minval)


def normal(k, shape):
    lo = np.nextafter(-1.0, 0.0)
    u = uniform(k, shape, lo, 1.0)
    return np.sqrt(2.0) * erfinv(u)


def randint(k, shape, minval: int, maxval: int):
    """int64 integers on [minval, maxval) (jax.random.randint, 64-bit mode)."""
    k1, k2 = split(k, 2)
    higher = random_bits(k1, shape, 64)
    lower = random_bits(k2, shape, 64)
    span = int(maxval) - int(minval)
    if span <= 0:
        raise ValueError("empty range")
    mult = (pow(2, 32, span) ** 2) % span  # 2**64 mod span, squared in halves
    hi = np.array([int(h) % span for h in higher.ravel()], dtype=object)
    lo = np.array([int(v) % span for v in lower.ravel()], dtype=object)
    off = (hi * mult + lo) % span
    return (int(minval) + off.astype(np.int64)).reshape(shape)


def golden_inputs(distribution: str, n: int):
    """Positions and masses of the reference's golden cases, drawn from
    PRNGKey(0xC0FFEE) the way tests/characterization/test_fmm_golden.py:171-193
    draws them ("uniform": uniform in [-1, 1)^3; "clustered": four Gaussian
    blobs of width 0.08 around centres uniform in [-0.8, 0.8)^3, clipped to
    [-1, 1])."""
    k = key(0xC0FFEE)
    k_pos, k_mass, k_blob = split(k, 3)
    if distribution == "uniform":
        pos = uniform(k_pos, (n, 3), -1.0, 1.0)
    elif distribution == "clustered":
        n_blobs = 4
        centers = uniform(k_blob, (n_blobs, 3), -0.8, 0.8)
        assign = randint(k_pos, (n,), 0, n_blobs)
        jitter = 0.08 * normal(k_mass, (n, 3))
        pos = np.clip(centers[assign] + jitter, -1.0, 1.0)
    else:
        raise ValueError(f"unknown distribution {distribution!r}")
    mass = np.abs(normal(k_mass, (n,))) + 0.5
    return pos, mass
