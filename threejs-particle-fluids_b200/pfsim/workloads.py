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

def _axis(lo: float, hi: float, spacing: float) -> np.ndarray:
    """lo + spacing/2, then repeated `+= spacing` while below hi, accumulated
    sequentially in double precision exactly as the reference's loop."""
    n = max(0, int(np.ceil((hi - lo) / spacing)) + 2)
    steps = np.full(n, spacing)
    steps[0] = lo + spacing / 2
    vals = np.add.accumulate(steps)
    return vals[vals < hi]


def fill_box(lo, hi, spacing: float) -> np.ndarray:
    """Lattice points filling a box, offset half a spacing from its corner,
    x fastest inside z inside y (src/simulation/layout.ts:7-14)."""
    xs, ys, zs = (_axis(lo[a], hi[a], spacing) for a in range(3))
    Y, Z, X = np.meshgrid(ys, zs, xs, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], -1)


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


def cloth_sheet(side: int = 64, seed: int = 0, scale: float = 1.0, compliance: float = 1e-6,
                substeps: int = 2, iterations: int = 4, offset=(0.0, 0.0, 0.0), bend_compliance: float | None = None,
                tethers: bool = False, tether_compliance: float = 0.0, stretch_tolerance: float = 0.0,
                wind=None, drag: float = 0.6125, lift: float = 0.3, damping: float | None = None):
    """A hanging cloth sheet of side x side particles (PlaneGeometry with
    side-1 segments per axis, structural + shear distance constraints, the
    top row pinned) inside the dam-break container scaled by `scale`; the
    sheet hangs in the x-y plane from just below the container top, tilted
    by a seeded small angle so it swings."""
    from . import recipe as R
    from . import shapes

    off = np.asarray(offset, np.float64)
    c_lo = np.array([-0.5, 0.0, -0.3]) * scale + off
    c_hi = np.array([0.5, 0.8, 0.3]) * scale + off
    width = 0.8 * (c_hi[0] - c_lo[0])
    height = 0.7 * (c_hi[1] - c_lo[1])
    pos, index = shapes.plane_geometry(width, height, side - 1, side - 1)
    r = rng(seed)
    tilt = r.uniform(-0.4, 0.4)
    ct, st = np.cos(tilt), np.sin(tilt)
    # tilt about the x axis (the pinned top edge), then place below the lid
    y, z = pos[:, 1].copy(), pos[:, 2].copy()
    pos[:, 1] = ct * y - st * z
    pos[:, 2] = st * y + ct * z
    top = c_hi[1] - 0.05 * (c_hi[1] - c_lo[1])
    pos += np.array([0.5 * (c_lo[0] + c_hi[0]), top - pos[:, 1].max(), 0.5 * (c_lo[2] + c_hi[2])])
    graph = shapes.create_cloth_graph(pos, index, 0.2, pinned=range(side))
    n = pos.shape[0]
    edge = width / (side - 1)
    cloth = R.ClothOpts(offset=0, positions=graph.positions.astype(np.float32), inv_mass=graph.inv_mass,
                        pairs=graph.pairs, rest_lengths=graph.rest_lengths, stretch_compliance=compliance)
    if bend_compliance is not None:  # dihedral bending as well (the batch configuration has stretch only)
        cloth.bending, cloth.bending_rest = graph.bending, graph.bending_rest.astype(np.float32)
        cloth.bend_compliance = bend_compliance
    if tethers:  # long-range attachments to the pinned top row
        cloth.tether_particle, cloth.tether_anchor, cloth.tether_rest = shapes.build_tethers(
            graph.inv_mass, graph.pairs, graph.rest_lengths, stretch_tolerance=stretch_tolerance)
        cloth.tether_compliance = tether_compliance
    if wind is not None:  # drag and lift on the sheet's triangles
        cloth.triangles, cloth.wind, cloth.drag, cloth.lift = graph.triangles, tuple(wind), drag, lift
    cloth.damping = damping
    loop = R.LoopOpts(substeps=substeps, iterations=iterations)
    return R.Recipe(capacity=n, radius=0.5 * edge, materials=[("cloth", cloth)],
                    prims=R.container_walls(tuple(c_lo), tuple(c_hi)), loop=loop, name=f"cloth_{side}x{side}")


def softbody_compliance(softness: float, count: int) -> float:
    """Simulation.addSoftbody's softness mapping (src/simulation/handles.ts:246-248)."""
    return 10 ** (-6 + softness * 3) * (count / 200)


def _softbody_set(r, n_bodies: int, spacing: float, per_body: int, region_lo, region_hi, density: float):
    """n_bodies voxelised spheres/boxes of about per_body particles at lattice
    spacing `spacing`, 26-neighbour clusters, softness log-uniform on
    [0.05, 1], laid out on a grid inside the region."""
    from . import shapes

    rad = 0.5 * spacing
    R_sphere = spacing * (3 * per_body / (4 * np.pi)) ** (1 / 3)
    half_box = 0.5 * spacing * per_body ** (1 / 3)
    size = 2.2 * max(R_sphere, half_box)
    lo, hi = np.asarray(region_lo, float), np.asarray(region_hi, float)
    nxz = max(1, int((hi[0] - lo[0]) // size)), max(1, int((hi[2] - lo[2]) // size))
    bodies = []
    for b in range(n_bodies):
        gx, gz, gy = b % nxz[0], (b // nxz[0]) % nxz[1], b // (nxz[0] * nxz[1])
        c = lo + np.array([(gx + 0.5) * size, (gy + 0.5) * size, (gz + 0.5) * size])
        if r.random() < 0.5:
            vox = shapes.voxel_sphere(c, R_sphere, rad, neighborhood=26)
        else:
            vox = shapes.voxel_box(c, (half_box, half_box, half_box), rad, neighborhood=26)
        softness = float(np.exp(r.uniform(np.log(0.05), np.log(1.0))))
        bodies.append((vox, softbody_compliance(softness, vox.count)))
    return bodies


def mixed_scene(n_budget: int = 50_000, n_fluid: int = 30_000, n_bodies: int = 20, seed: int = 0,
                substeps: int = 3, iterations: int = 4, scale: float = 1.0, offset=(0.0, 0.0, 0.0)):
    """Fluid block (as the dam break, spacing from the fluid's share of the
    budget) plus soft bodies of about (budget - fluid)/n_bodies particles each
    at the same spacing and the fluid's density, their surfaces acting as
    dynamic fluid boundaries, and one sphere collider (radius 0.1) moving on a
    circle (PrimitiveSet.setSphere every step)."""
    from . import recipe as R

    off = np.asarray(offset, np.float64)
    c_lo = np.array([-0.5, 0.0, -0.3]) * scale + off
    c_hi = np.array([0.5, 0.8, 0.3]) * scale + off
    f_lo, f_hi = c_lo.copy(), np.array([-0.1, 0.5, 0.3]) * scale + off
    vol = float(np.prod(f_hi - f_lo))
    s = (vol / n_fluid) ** (1.0 / 3.0)
    r = rng(seed)
    fpts = fill_box(f_lo, f_hi, s)
    fpts = fpts + r.uniform(-0.05 * s, 0.05 * s, fpts.shape)
    nf = fpts.shape[0]
    h = 2.0 * s
    mass = 1000.0 * s**3
    rho0 = lattice_rest_density(s, h, mass)
    spacing = (mass / rho0) ** (1.0 / 3.0)
    per_body = max(27, (n_budget - n_fluid) // max(n_bodies, 1))
    region_lo = np.array([-0.08, 0.02, -0.28]) * scale + off
    region_hi = np.array([0.48, 0.78, 0.28]) * scale + off
    bodies = _softbody_set(r, n_bodies, s, per_body, region_lo, region_hi, 1000.0)
    # particle layout: soft bodies first (surface first within each), then fluid
    uploads, defs, bounds = [], [], []
    start = 0
    inv_m = np.float32(1.0 / mass)
    for vox, comp in bodies:
        uploads.append(R.Upload(start, vox.positions, None, np.full(vox.count, inv_m, np.float32)))
        defs.append(R.BodyDef(range=(start, vox.count), surface_count=vox.surface_count, compliance=comp,
                              edges=vox.edges))
        bounds.append((start, vox.surface_count))
        start += vox.count
    uploads.append(R.Upload(start, fpts.astype(np.float32)))
    fluid = R.FluidOpts(range=(start, nf), rest_density=rho0, particle_spacing=spacing, smoothing_radius=h,
                        compliance=1e-4, viscosity=0.01, boundaries=bounds)
    cap = start + nf
    sphere_r = 0.1 * scale
    centre = np.array([0.2, 0.25, 0.0]) * scale + off
    orbit, period = 0.15 * scale, 2.0
    prims = R.container_walls(tuple(c_lo), tuple(c_hi)) + [R.sphere(tuple(centre + [orbit, 0, 0]), sphere_r)]
    slot = len(prims) - 1

    def motion(step: int, dt: float):
        w = 2 * np.pi / period
        t = (step + 1) * dt
        c = centre + orbit * np.array([np.cos(w * t), 0.0, np.sin(w * t)])
        v = orbit * w * np.array([-np.sin(w * t), 0.0, np.cos(w * t)])
        p = R.sphere(tuple(c), sphere_r, velocity=tuple(v))
        p.flags |= 2  # PrimitiveSet.setSphere marks the sphere as swept
        return {slot: p}

    height = c_hi[1] - c_lo[1]
    loop = R.LoopOpts(substeps=substeps, iterations=iterations, grid_min=tuple(c_lo - 2 * h),
                      grid_max=tuple(c_hi + np.array([2 * h, height, 2 * h])))
    return R.Recipe(capacity=cap, radius=s / 2.0, uploads=uploads,
                    materials=[("soft", R.SoftbodyOpts(defs, "local")), ("fluid", fluid)],
                    prims=prims, loop=loop, name=f"mixed_{cap}", motion=motion)


def softbody_pile(n_budget: int, seed: int = 0, per_body: int = 1000, scale: float = 1.0,
                  substeps: int = 3, iterations: int = 4, offset=(0.0, 0.0, 0.0)):
    """Soft bodies only: about n_budget/per_body voxelised spheres and boxes
    (26-neighbour clusters) dropping into the container."""
    from . import recipe as R

    off = np.asarray(offset, np.float64)
    c_lo = np.array([-0.5, 0.0, -0.3]) * scale + off
    c_hi = np.array([0.5, 0.8, 0.3]) * scale + off
    n_bodies = max(1, n_budget // per_body)
    vol = float(np.prod(c_hi - c_lo)) * 0.5
    s = (vol / max(n_budget, 1)) ** (1.0 / 3.0)
    r = rng(seed)
    bodies = _softbody_set(r, n_bodies, s, per_body, c_lo + 0.02 * scale, c_hi - 0.02 * scale, 1000.0)
    uploads, defs = [], []
    start = 0
    inv_m = np.float32(1.0 / (1000.0 * s**3))
    for vox, comp in bodies:
        uploads.append(R.Upload(start, vox.positions, None, np.full(vox.count, inv_m, np.float32)))
        defs.append(R.BodyDef(range=(start, vox.count), surface_count=vox.surface_count, compliance=comp,
                              edges=vox.edges))
        start += vox.count
    loop = R.LoopOpts(substeps=substeps, iterations=iterations)
    return R.Recipe(capacity=start, radius=s / 2.0, uploads=uploads, materials=[("soft", R.SoftbodyOpts(defs, "local"))],
                    prims=R.container_walls(tuple(c_lo), tuple(c_hi)), loop=loop, name=f"softbodies_{start}")


def log_uniform(r, lo: float, hi: float) -> float:
    return float(np.exp(r.uniform(np.log(lo), np.log(hi))))


def batch_stream(n_scenes: int = 256, seed: int = 0, n_lo: int = 5_000, n_hi: int = 200_000,
                 fluid_share: float = 0.7):
    """Uneven scenes for batching: particle counts log-uniform on
    [n_lo, n_hi]; fluid_share of them dam breaks (container scale U[0.5, 2]),
    the rest cloth sheets of 64^2-256^2 particles (compliance 1e-6, pinned
    top row). All step with 2 substeps and 4 iterations."""
    r = rng(seed)
    out = []
    for i in range(n_scenes):
        n = int(round(log_uniform(r, n_lo, n_hi)))
        scale = float(r.uniform(0.5, 2.0))
        if r.random() < fluid_share:
            out.append(dam_break(n, seed=seed * 100003 + i, scale=scale))
        else:
            side = int(np.clip(round(np.sqrt(n)), 64, 256))
            out.append(cloth_sheet(side, seed=seed * 100003 + i, scale=scale))
    return out


def serve_request(r, index: int, seed: int, n_lo: int = 5_000, n_hi: int = 500_000):
    """One serving request: a scene spec with N log-uniform on [n_lo, n_hi],
    material fluid/soft/cloth at 60/20/20 and a lifetime U[60, 600] steps."""
    n = int(round(log_uniform(r, n_lo, n_hi)))
    u = r.random()
    scale = float(r.uniform(0.5, 2.0))
    s = seed * 1000003 + index
    if u < 0.6:
        rec = dam_break(n, seed=s, scale=scale)
    elif u < 0.8:
        rec = softbody_pile(n, seed=s, scale=scale, substeps=2)
    else:
        side = int(np.clip(round(np.sqrt(n)), 64, 256))
        rec = cloth_sheet(side, seed=s, scale=scale)
    lifetime = int(r.integers(60, 601))
    return rec, lifetime
