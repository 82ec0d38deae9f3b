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


# ---------------------------------------------------------------- scenes ----

def fill_box(lo, hi, spacing: float) -> np.ndarray:
    """Lattice points filling a box, offset half a spacing from its corner,
    x fastest inside z inside y (src/simulation/layout.ts:7-14). The loop
    accumulates coordinates in double precision as the reference does."""
    pts = []
    y = lo[1] + spacing / 2
    while y < hi[1]:
        z = lo[2] + spacing / 2
        while z < hi[2]:
            x = lo[0] + spacing / 2
            while x < hi[0]:
                pts.append((x, y, z))
                x += spacing
            z += spacing
        y += spacing
    return np.array(pts, np.float64).reshape(-1, 3)


def lattice_rest_density(spacing: float, h: float, mass: float) -> float:
    """SPH density at an interior point of an unjittered cubic lattice."""
    r = int(np.ceil(h / spacing))
    ax = np.arange(-r, r + 1)
    g = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3) * spacing
    rsq = (g * g).sum(1)
    rsq = rsq[rsq < h * h]
    poly6 = 315.0 / (64.0 * np.pi * h**9)
    return float(mass * poly6 * ((h * h - rsq) ** 3).sum())


def dam_break(n_budget: int = 5000, seed: int = 0, scale: float = 1.0, jitter: float = 0.05,
              substeps: int = 2, iterations: int = 4, xsph: float = 0.01, gravity=(0.0, -9.81, 0.0),
              offset=(0.0, 0.0, 0.0)):
    """A PBF dam break: container [-0.5,0,-0.3]-[0.5,0.8,0.3], fluid filling
    [-0.5,0,-0.3]-[-0.1,0.5,0.3], both scaled by `scale` and shifted by
    `offset`, lattice spacing from the particle budget, each point jittered
    by +-jitter*spacing, h = 2 spacing, grid cell h, rest density from the
    unjittered lattice, XSPH viscosity only; walls on five sides (open top)."""
    from . import recipe as R

    off = np.asarray(offset, np.float64)
    c_lo = np.array([-0.5, 0.0, -0.3]) * scale + off
    c_hi = np.array([0.5, 0.8, 0.3]) * scale + off
    f_lo = np.array([-0.5, 0.0, -0.3]) * scale + off
    f_hi = np.array([-0.1, 0.5, 0.3]) * scale + off
    vol = float(np.prod(f_hi - f_lo))
    s = (vol / n_budget) ** (1.0 / 3.0)
    pts = fill_box(f_lo, f_hi, s)
    r = rng(seed)
    pts = pts + r.uniform(-jitter * s, jitter * s, pts.shape)
    n = pts.shape[0]
    h = 2.0 * s
    mass = 1000.0 * s**3
    rho0 = lattice_rest_density(s, h, mass)
    spacing = (mass / rho0) ** (1.0 / 3.0)  # so that restDensity * spacing^3 = mass
    fluid = R.FluidOpts(range=(0, n), rest_density=rho0, particle_spacing=spacing, smoothing_radius=h,
                        compliance=1e-4, viscosity=xsph)
    height = c_hi[1] - c_lo[1]
    loop = R.LoopOpts(substeps=substeps, iterations=iterations, gravity=tuple(gravity),
                      grid_min=tuple(c_lo - 2 * h), grid_max=tuple(c_hi + np.array([2 * h, height, 2 * h])))
    return R.Recipe(
        capacity=n,
        radius=s / 2.0,
        uploads=[R.Upload(0, pts.astype(np.float32))],
        materials=[("fluid", fluid)],
        prims=R.container_walls(tuple(c_lo), tuple(c_hi)),
        loop=loop,
        name=f"dam_break_{n}",
    )
