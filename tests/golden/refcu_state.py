"""Seeded input states for the reference-kernel golden vectors.

TEST INFRASTRUCTURE ONLY.  The values are a fixed function of the seed and
the grid shape, computed with integer hashing and NumPy's sin (no random
generator whose stream could change between NumPy versions), so the tests
can rebuild an input that is too large to store (128 x 128 x 256) and feed
the same values to the oracle and to the CUDA kernels.
"""
from __future__ import annotations

import numpy as np


def _noise(shape, seed: int, field: int) -> np.ndarray:
    """Uniform values in [-1, 1) from a 64-bit integer hash of the cell index."""
    n = int(np.prod(shape))
    offset = (0x9E3779B97F4A7C15 * (seed * 8 + field + 1)) % (1 << 64)
    x = np.arange(n, dtype=np.uint64) + np.uint64(offset)
    # splitmix64 finaliser (Steele, Lea, Flood 2014)
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    x = x ^ (x >> np.uint64(31))
    u = (x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return (2.0 * u - 1.0).reshape(shape)


def primitives(shape, seed: int) -> list[np.ndarray]:
    """rho, vx, vy, vz, p over the whole ghosted grid (float64): smooth
    waves of a few wavelengths plus 5 % cell noise; rho and p stay in
    [0.55, 1.45]."""
    nx, ny, nz = (int(s) for s in shape)
    x = (np.arange(nx) / nx)[:, None, None]
    y = (np.arange(ny) / ny)[None, :, None]
    z = (np.arange(nz) / nz)[None, None, :]
    out = []
    for f, amp in enumerate((0.3, 0.5, 0.5, 0.5, 0.3)):
        k = 1 + (seed + 3 * f) % 3
        ph = 0.7 * f + 0.3 * seed
        wave = np.sin(2 * np.pi * k * x + ph) * np.cos(2 * np.pi * (k % 2 + 1) * y + ph) \
            * np.sin(2 * np.pi * (4 - k) * z + 2 * ph)
        v = amp * wave + 0.05 * _noise(shape, seed, f)
        if f in (0, 4):
            v = 1.0 + v
        out.append(np.ascontiguousarray(v, dtype=np.float64))
    return out
