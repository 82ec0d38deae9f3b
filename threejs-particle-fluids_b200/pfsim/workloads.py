"""Seeded synthetic workloads with the shapes of the benchmark configurations.

The reference publishes no benchmark data; these generators stand in for it
with the sizes and value distributions the configurations name. Every
generator takes an explicit seed and uses numpy's PCG64.
"""

from __future__ import annotations

import numpy as np


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


# ----------------------------------------------------------------- sort ----

def sort_uniform(n: int, seed: int = 1) -> np.ndarray:
    """n float4 positions uniform in the unit cube, w = 0."""
    r = rng(seed)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = r.random((n, 3), dtype=np.float32)
    return pos


def sort_blobs(n: int, seed: int = 2, blobs: int = 64, sigma: float = 0.02) -> np.ndarray:
    """n float4 positions from `blobs` Gaussian blobs (sigma) with uniform
    centres, clamped into [0, 1 - 2^-24]; each point picks a blob uniformly."""
    r = rng(seed)
    centres = r.random((blobs, 3))
    which = r.integers(0, blobs, n)
    pts = centres[which] + r.normal(0.0, sigma, (n, 3))
    pts = np.clip(pts, 0.0, 1.0 - 2.0**-24)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = pts.astype(np.float32)
    return pos


SORT_GRID_DIMS = (128, 128, 128)
SORT_CELL = 1.0 / 128.0
