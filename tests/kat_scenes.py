"""Scenes of the reference's analytical known-answer tests, as recipes that
either backend (the CUDA path through the C ABI, or the oracle) replays.

Each builder names the reference test it restates; the expected values and
tolerances live in the tests that use these scenes.
"""

from __future__ import annotations

import math

import numpy as np

from pfsim import recipe as R

DT = 1.0 / 60.0
G = 9.81


def free_fall() -> R.Recipe:
    """tests/analytical/integrate/integrate-free-fall.gpu.test.ts:8-24: one
    particle at the origin, no material, no collider, one substep."""
    return R.Recipe(
        capacity=1,
        radius=0.05,
        uploads=[R.Upload(0, np.zeros((1, 3), np.float32), np.zeros((1, 3), np.float32), np.ones(1, np.float32))],
        loop=R.LoopOpts(substeps=1),
        name="free-fall",
    )


def free_fall_reference(steps: int) -> float:
    """The test's own CPU reference (integrate-free-fall.gpu.test.ts:26-32):
    semi-implicit Euler in double precision."""
    v = y = 0.0
    for _ in range(steps):
        v -= G * DT
        y += v * DT
    return y


def distance_pair(compliance: float, substeps: int, iterations: int, constrained: bool = True) -> R.Recipe:
    """tests/analytical/xpbd/xpbd-limits.gpu.test.ts:44-56 and 80-106: particle 0
    pinned at the origin, particle 1 at (0, -1, 0), joined by one distance
    constraint of rest length 1 (a one-edge cloth graph carries it)."""
    pos = np.array([[0.0, 0.0, 0.0], [0.0, -1.0, 0.0]], np.float32)
    w = np.array([0.0, 1.0], np.float32)
    r = R.Recipe(capacity=2, radius=0.02, loop=R.LoopOpts(substeps=substeps, iterations=iterations),
                 name=f"distance-pair-{compliance:g}")
    if constrained:
        r.materials.append(("cloth", R.ClothOpts(offset=0, positions=pos, inv_mass=w,
                                                 pairs=np.array([[0, 1]], np.uint32),
                                                 rest_lengths=np.array([1.0], np.float32),
                                                 stretch_compliance=compliance)))
    else:
        r.uploads.append(R.Upload(0, pos, np.zeros_like(pos), w))
    return r


LATTICE, SPACING, H, REST = 5, 0.025, 0.04, 1000.0


def density_lattice() -> R.Recipe:
    """tests/analytical/fluids/density-pair-list-cpu-parity.gpu.test.ts:33-86:
    a 5x5x5 lattice at spacing 0.025, h = 0.04, rest density 1000, mass
    rho0 * spacing^3; no gravity, so the first lambda pass sees the lattice."""
    idx = np.arange(LATTICE ** 3)
    x, y, z = idx % LATTICE, (idx // LATTICE) % LATTICE, idx // (LATTICE * LATTICE)
    pos = (np.stack([x, y, z], -1) * SPACING).astype(np.float32)
    m = REST * SPACING ** 3
    w = np.full(pos.shape[0], np.float32(1.0 / m), np.float32)
    r = R.Recipe(capacity=pos.shape[0], radius=SPACING * 0.5,
                 uploads=[R.Upload(0, pos, np.zeros_like(pos), w)],
                 loop=R.LoopOpts(substeps=1, iterations=1, gravity=(0.0, 0.0, 0.0)),
                 name="density-lattice")
    r.materials.append(("fluid", R.FluidOpts(range=(0, pos.shape[0]), rest_density=REST, particle_spacing=SPACING,
                                             smoothing_radius=H, compliance=1e-6)))
    return r


def density_brute_force() -> np.ndarray:
    """The test's CPU ground truth (density-pair-list-cpu-parity.gpu.test.ts:94-118):
    rho_i = sum_j m W_poly6(|x_i - x_j|, h), double precision."""
    idx = np.arange(LATTICE ** 3)
    p = np.stack([idx % LATTICE, (idx // LATTICE) % LATTICE, idx // (LATTICE * LATTICE)], -1) * SPACING
    p = p.astype(np.float32).astype(np.float64)
    poly6 = 315.0 / (64.0 * math.pi * H ** 9)
    m = REST * SPACING ** 3
    d = ((p[:, None, :] - p[None, :, :]) ** 2).sum(-1)
    t = np.where(d < H * H, (H * H - d) ** 3, 0.0)
    return m * poly6 * t.sum(1)


def plane_rest() -> R.Recipe:
    """tests/analytical/collider/collider-plane-rest.gpu.test.ts:16-34: one
    particle of radius 0.05 dropped from y = 0.5 onto the plane y = 0
    (muS 0.5, muK 0.4), 4 substeps, 4 iterations."""
    pos = np.array([[0.0, 0.5, 0.0]], np.float32)
    return R.Recipe(capacity=1, radius=0.05,
                    uploads=[R.Upload(0, pos, np.zeros_like(pos), np.ones(1, np.float32))],
                    prims=[R.plane((0, 1, 0), (0, 0, 0), 0.5, 0.4)],
                    loop=R.LoopOpts(substeps=4, iterations=4),
                    name="plane-rest")


def run_trace(scene, frames: int, every: int = 1, field=None):
    """Step a built scene, reading positions (and velocities) every `every`
    frames and on the last one."""
    from pfsim import _native as N

    out = []
    for n in range(frames):
        scene.step(DT)
        if n % every == 0 or n == frames - 1:
            out.append((scene.readback(N.PF_FIELD_POSITIONS).copy(), scene.readback(N.PF_FIELD_VELOCITIES).copy()))
    return out


# ---- the colouring test's graphs (xpbd-group-partition.test.ts:48-166) ----
def chain_pairs(n: int = 10) -> np.ndarray:
    return np.array([[i, i + 1] for i in range(n - 1)], np.uint32)


def star_pairs(n: int = 8) -> np.ndarray:
    return np.array([[0, leaf] for leaf in range(1, n + 1)], np.uint32)


def random_graphs(trials: int = 10):
    """The test's LCG (multiplier 1664525, increment 1013904223, seed
    0xdeadc0de) drawing 10 random simple graphs (xpbd-group-partition.test.ts:102-127)."""
    state = [0xDEADC0DE]

    def nxt():
        state[0] = (state[0] * 1664525 + 1013904223) & 0xFFFFFFFF
        return state[0] / 0x100000000

    graphs = []
    for _ in range(trials):
        n_particles = 20 + int(math.floor(nxt() * 30))
        n_edges = 30 + int(math.floor(nxt() * 50))
        seen = set()
        pairs = []
        attempts = 0
        while len(pairs) < n_edges and attempts < n_edges * 10:
            attempts += 1
            i = int(math.floor(nxt() * n_particles))
            j = int(math.floor(nxt() * n_particles))
            if i == j:
                continue
            key = (min(i, j), max(i, j))
            if key in seen:
                continue
            seen.add(key)
            pairs.append((i, j))
        graphs.append(np.array(pairs, np.uint32).reshape(-1, 2))
    return graphs


def rot_x(t):
    c, s = math.cos(t), math.sin(t)
    return np.array([[1, 0, 0], [0, c, -s], [0, s, c]])


def rot_y(t):
    c, s = math.cos(t), math.sin(t)
    return np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])


def rot_z(t):
    c, s = math.cos(t), math.sin(t)
    return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])


def polar_cases():
    """(A, expected R, tolerance) of softbody-polar-decomp.gpu.test.ts:119-200."""
    I = np.eye(3)
    Rk = rot_x(0.4) @ rot_z(-0.3)
    S = np.array([[1.5, 0.2, 0.0], [0.2, 1.2, 0.0], [0.0, 0.0, 1.0]])
    return [
        ("identity", I, I, 1e-4),
        ("rot-z", rot_z(math.pi / 4), rot_z(math.pi / 4), 1e-4),
        ("rot-y", rot_y(math.pi / 3), rot_y(math.pi / 3), 1e-4),
        ("rot-x", rot_x(-math.pi / 6), rot_x(-math.pi / 6), 1e-4),
        ("composed", rot_z(0.3) @ rot_y(-0.7) @ rot_x(0.5), rot_z(0.3) @ rot_y(-0.7) @ rot_x(0.5), 1e-4),
        ("uniform-stretch", np.diag([2.5, 2.5, 2.5]), I, 1e-4),
        ("diag-stretch", np.diag([3.0, 1.5, 0.8]), I, 1e-4),
        ("rot-stretch", rot_z(math.pi / 6) @ np.diag([2.0, 1.0, 0.5]), rot_z(math.pi / 6), 1e-4),
        ("rot-shear", Rk @ S, Rk, 1e-4),
        ("near-identity", rot_z(1e-3), rot_z(1e-3), 1e-5),
    ]


# ---- SDF collider (tests/analytical/sdf/*) ----
def sdf_sphere_grid(res: int = 64, radius: float = 0.5, pad: float = 0.1):
    """An exact sphere SDF baked at voxel centres (the reference bakes a UV
    sphere mesh; the analytic field stands in for the bake)."""
    from pfsim import recipe as R

    return R.sphere_sdf((0.0, 0.0, 0.0), radius, res=res, pad=pad)


def lcg_js(seed: int):
    """The tests' `seed = (Math.imul(seed, 1664525) + 1013904223) | 0` and
    `(seed >>> 0) / 2^32`."""
    state = [seed & 0xFFFFFFFF]

    def nxt():
        state[0] = (state[0] * 1664525 + 1013904223) & 0xFFFFFFFF
        return state[0] / 0x100000000

    return nxt


def sdf_rotated_scaled():
    """sdf-rotated-scaled.gpu.test.ts:41-110: 100 particles (r = 0.04) inside a
    sphere of mesh radius 0.5 placed at (0.3, 0, -0.2), scaled 2x and rotated
    pi/3 about (1, 1, 0); one step of 1 substep x 4 iterations, no gravity."""
    rand = lcg_js(0xC0FFEE42)
    center = np.array([0.3, 0.0, -0.2])
    scale, r = 2.0, 0.04
    inner = scale * 0.5 - 2 * r
    pts = []
    while len(pts) < 100:
        u = np.array([rand() * 2 - 1, rand() * 2 - 1, rand() * 2 - 1])
        if (u * u).sum() > 1:
            continue
        pts.append(center + u * inner)
    pos = np.array(pts, np.float32)
    axis = np.array([1.0, 1.0, 0.0]) / np.sqrt(2.0)
    q = (*(axis * np.sin(np.pi / 6)), np.cos(np.pi / 6))
    g = sdf_sphere_grid()
    g.position, g.rotation, g.scale = tuple(center), q, scale
    from pfsim import recipe as R

    rec = R.Recipe(capacity=100, radius=r, uploads=[R.Upload(0, pos, np.zeros_like(pos), np.ones(100, np.float32))],
                   sdfs=[g], loop=R.LoopOpts(substeps=1, iterations=4, gravity=(0.0, 0.0, 0.0)),
                   name="sdf-rotated-scaled")
    return rec, center, scale * 0.5


# ---- cloth bending (tests/analytical/cloth/bending-rest.gpu.test.ts) ----
def folded_quad(dihedral: float):
    """bending-rest.gpu.test.ts:33-54: two triangles sharing the edge
    (0,0,0)-(1,0,0), the second rotated about it so that the dihedral is
    `dihedral`; edge endpoints pinned; stretch 1e-7, bend 1e-5, radius 0.05,
    8 substeps x 1 iteration, no gravity."""
    from pfsim import shapes

    c, s = np.cos(np.pi - dihedral), np.sin(np.pi - dihedral)
    pos = np.array([[0, 0, 0], [1, 0, 0], [0.5, 1, 0], [0.5, c, s]], np.float64)
    g = shapes.create_cloth_graph(pos, np.array([0, 1, 2, 0, 3, 1]), 0.2, pinned=[0, 1])
    cloth = R.ClothOpts(offset=0, positions=g.positions.astype(np.float32), inv_mass=g.inv_mass, pairs=g.pairs,
                        rest_lengths=g.rest_lengths, stretch_compliance=1e-7, bending=g.bending,
                        bending_rest=g.bending_rest.astype(np.float32), bend_compliance=1e-5)
    rec = R.Recipe(capacity=4, radius=0.05, materials=[("cloth", cloth)],
                   loop=R.LoopOpts(substeps=8, iterations=1, gravity=(0.0, 0.0, 0.0)), name="folded-quad")
    return rec, g


def signed_dihedral(pos: np.ndarray) -> float:
    from pfsim import shapes

    return float(shapes.dihedral_angles(np.asarray(pos, np.float64)[:, :3], np.array([[0, 1, 2, 3]]))[0])


def grid_sheet(m: int, x0: float = 0.0):
    """The m x m sheets of tests/analytical/cloth/tether-stretch.gpu.test.ts:
    39-70, tether-unilateral.gpu.test.ts:40-66 (x0 = 0) and
    wind-deflection.gpu.test.ts:55-83 (x0 = -0.5): vertex (i, j) at
    (x0 + i/(m-1), -j/(m-1), 0) as float32, triangles (a, c, d), (a, d, b)
    per quad, the top row pinned. Returns (positions, index, pinned)."""
    j, i = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    pos = np.stack([x0 + i / (m - 1), -(j / (m - 1)), np.zeros((m, m))], -1).reshape(-1, 3)
    pos = pos.astype(np.float32).astype(np.float64)
    idx = []
    for jj in range(m - 1):
        for ii in range(m - 1):
            a, b = jj * m + ii, jj * m + ii + 1
            c, d = (jj + 1) * m + ii, (jj + 1) * m + ii + 1
            idx += [a, c, d, a, d, b]
    return pos, np.array(idx, np.int64), list(range(m))


def cloth_system(graph, substeps: int, iterations: int, gravity=(0.0, -G, 0.0), stretch: float = 1e-7,
                 bend: float = 1e-5, tether_compliance: float = 0.0, wind=(0.0, 0.0, 0.0), drag: float = 0.6125,
                 lift: float = 0.3, radius: float = 0.05, positions=None, name: str = "cloth"):
    """new ClothSystem(particles, {graph, stretchCompliance, bendCompliance,
    tetherCompliance, wind, drag, lift}) in a SimLoop of its own
    (ClothSystem.ts:102-141, 190-245): stretch, bending and tether colours,
    drag and lift on the graph's triangles. `positions` replaces the
    uploaded positions after the cloth wrote its own (as the tests'
    uploadParticles calls do). Returns (recipe, tethers)."""
    from pfsim import shapes

    tp, ta, tr = shapes.build_tethers(graph.inv_mass, graph.pairs, graph.rest_lengths)
    n = graph.positions.shape[0]
    cloth = R.ClothOpts(offset=0, positions=graph.positions.astype(np.float32),
                        inv_mass=np.asarray(graph.inv_mass, np.float32), pairs=graph.pairs,
                        rest_lengths=np.asarray(graph.rest_lengths, np.float32), stretch_compliance=stretch,
                        bending=graph.bending, bending_rest=graph.bending_rest.astype(np.float32),
                        bend_compliance=bend, tether_particle=tp, tether_anchor=ta, tether_rest=tr,
                        tether_compliance=tether_compliance, triangles=graph.triangles, wind=tuple(wind),
                        drag=drag, lift=lift)
    r = R.Recipe(capacity=n, radius=radius, materials=[("cloth", cloth)],
                 loop=R.LoopOpts(substeps=substeps, iterations=iterations, gravity=tuple(gravity)), name=name)
    if positions is not None:
        cloth.positions = np.asarray(positions, np.float32)
    return r, (tp, ta, tr)


def run_damped(scene, frames: int, damp: float) -> None:
    """The tests' frame loop: step, then scale every velocity by `damp`
    (read the buffer, multiply, write it back)."""
    from pfsim import _native as N

    for _ in range(frames):
        scene.step(DT)
        scene.write(N.PF_FIELD_VELOCITIES, scene.readback(N.PF_FIELD_VELOCITIES) * np.float32(damp))


def wind_deflection_analytic(surface_density: float, g: float, v: float, drag: float, lift: float) -> float:
    """wind-deflection.gpu.test.ts:85-121: Newton iteration on
    rho_s g sin(t) = v^2 (drag cos^2(t) - lift sin^2(t))."""
    rsg, vsq = surface_density * g, v * v
    f = lambda t: rsg * math.sin(t) - vsq * (drag * math.cos(t) ** 2 - lift * math.sin(t) ** 2)
    df = lambda t: rsg * math.cos(t) + vsq * (2 * drag * math.cos(t) * math.sin(t)
                                              + 2 * lift * math.sin(t) * math.cos(t))
    t = math.atan(vsq * drag / max(rsg, 1e-9))
    for _ in range(12):
        d = df(t)
        if abs(d) < 1e-12:
            break
        nt = t - f(t) / d
        if abs(nt - t) < 1e-9:
            t = nt
            break
        t = nt
    return t


def wind_deflection_angle(pos4: np.ndarray, inv_mass: np.ndarray, top: list) -> tuple:
    """wind-deflection.gpu.test.ts:177-212: the pivot (mean of the top row)
    to the free particles' centre of mass, as (angle from vertical, dy, dz)."""
    py = float(np.mean(pos4[top, 1]))
    pz = float(np.mean(pos4[top, 2]))
    free = inv_mass != 0
    dy = float(np.mean(pos4[free, 1])) - py
    dz = float(np.mean(pos4[free, 2])) - pz
    return math.atan2(dz, abs(dy)), dy, dz


def particles(pos, radius: float, substeps: int, iterations: int, gravity=(0.0, -G, 0.0), vel=None,
              inv_mass=None, group=None, contact=None, prims=(), quiet=(), name: str = "particles") -> R.Recipe:
    """new ParticleSystem(capacity, r) + uploadParticles + SimLoop({substeps,
    iterations, gravity, contact: {maxContacts, muS, muK}, colliders}) of the
    contact tests (tests/analytical/contact/*.gpu.test.ts). `contact` is
    (max_contacts, mu_s, mu_k) or None; `quiet` lists noSelfContacts ranges
    of materials with no other kernels."""
    p = np.asarray(pos, np.float32).reshape(-1, 3)
    n = len(p)
    up = R.Upload(0, p, None if vel is None else np.asarray(vel, np.float32).reshape(-1, 3),
                  None if inv_mass is None else np.asarray(inv_mass, np.float32),
                  None if group is None else np.asarray(group, np.uint32))
    loop = R.LoopOpts(substeps=substeps, iterations=iterations, gravity=tuple(gravity))
    if contact is not None:
        loop.contact = True
        loop.max_contacts, loop.contact_mu_s, loop.contact_mu_k = contact
    return R.Recipe(capacity=n, radius=radius, uploads=[up], prims=list(prims), loop=loop, quiet=list(quiet),
                    name=name)


def lattice(side: int, spacing: float, origin=(0.0, 0.0, 0.0), centred_xz: bool = True) -> np.ndarray:
    """side^3 points, x outermost then y then z (the tests' ix, iy, iz loops)."""
    c = (side - 1) / 2 if centred_xz else 0.0
    pts = [((ix - c) * spacing + origin[0], iy * spacing + origin[1], (iz - c) * spacing + origin[2])
           for ix in range(side) for iy in range(side) for iz in range(side)]
    return np.array(pts, np.float64)


def column_on_slab(r: float = 0.025, columns: int = 200, slab: int = 60):
    """contact-generate-emitters.gpu.test.ts:35-76: a column of particles in
    collision group 1 resting on a pinned slab in group 2. Returns
    (positions, inverse masses, groups)."""
    sp = 2 * r
    side = math.ceil(columns ** (1 / 3))
    pos, w, g = [], [], []
    for i in range(columns):
        x, y, z = i % side, (i // side) % side, i // (side * side)
        pos.append((-side * sp * 0.5 + (x + 0.5) * sp, (y + 0.5) * sp, -side * sp * 0.5 + (z + 0.5) * sp))
        w.append(1.0)
        g.append(1)
    ss = math.ceil(math.sqrt(slab))
    for i in range(slab):
        x, z = i % ss, i // ss
        pos.append((-ss * sp * 0.5 + (x + 0.5) * sp, -sp * 0.5, -ss * sp * 0.5 + (z + 0.5) * sp))
        w.append(0.0)
        g.append(2)
    return np.array(pos), np.array(w, np.float32), np.array(g, np.uint32)


def pair_overlap(pos4: np.ndarray, two_r: float) -> float:
    """Largest 2r - |x_a - x_b| over all pairs (contact-non-interpenetration)."""
    p = pos4[:, :3].astype(np.float64)
    d = np.linalg.norm(p[:, None, :] - p[None, :, :], axis=-1)
    iu = np.triu_indices(len(p), 1)
    return float((two_r - d[iu]).max())


def unit_cube_mesh(half=(0.5, 0.5, 0.5)):
    """softbody-voxelize.test.ts:20-62: the box mesh of pfsim.mesh.box_mesh."""
    from pfsim import mesh as M

    return M.box_mesh(half)


def uv_sphere(radius: float, stacks: int, slices: int):
    """The tests' UV sphere (tests/_helpers/sdf-test-meshes.ts:23-87)."""
    from pfsim import mesh as M

    return M.uv_sphere(radius, stacks, slices)


def torus(ring_radius: float, tube_radius: float, ring_segs: int, tube_segs: int):
    """The tests' torus (sdf-test-meshes.ts:102-141)."""
    from pfsim import mesh as M

    return M.torus(ring_radius, tube_radius, ring_segs, tube_segs)


def sample_field(data: np.ndarray, origin, voxel, p) -> float:
    """src/sdf/sample.ts:12-47 in doubles (data indexed [z, y, x])."""
    rz, ry, rx = data.shape
    res = (rx, ry, rz)
    i, t = [], []
    for a in range(3):
        g = (p[a] - origin[a]) / voxel[a] - 0.5
        f = min(max(math.floor(g), 0), res[a] - 2)
        i.append(f)
        t.append(min(max(g - f, 0.0), 1.0))
    c = lambda dx, dy, dz: float(data[i[2] + dz, i[1] + dy, i[0] + dx])
    L = lambda a, b, w: a + (b - a) * w
    c0 = L(L(c(0, 0, 0), c(1, 0, 0), t[0]), L(c(0, 1, 0), c(1, 1, 0), t[0]), t[1])
    c1 = L(L(c(0, 0, 1), c(1, 0, 1), t[0]), L(c(0, 1, 1), c(1, 1, 1), t[0]), t[1])
    return L(c0, c1, t[2])


# ---------------------------------------------------------------- soft bodies
SM_DT = 1.0 / 240.0  # softbody-pass3-apply.gpu.test.ts:34


def unit_cube_rest() -> np.ndarray:
    """softbody-pass3-apply.gpu.test.ts:51-62: the eight corners of a unit cube
    about the origin (rest centre of mass 0)."""
    return np.array([[x, y, z] for z in (-0.5, 0.5) for y in (-0.5, 0.5) for x in (-0.5, 0.5)], np.float32)


def shape_match_body(rest: np.ndarray, start: np.ndarray, compliance: float, iterations: int,
                     inv_mass=1.0) -> R.Recipe:
    """softbody-pass3-apply.gpu.test.ts:115-161 at the scene level: one body
    with global shape matching over `rest`, its particles at `start` with no
    velocity and no gravity, one substep of `iterations` iterations. The
    predicted positions are then `start`, and the step's positions are the
    predicted positions after the shape-matching iterations (what the test
    reads back)."""
    n = rest.shape[0]
    body = R.BodyDef(range=(0, n), compliance=compliance, rest_positions=np.asarray(rest, np.float32))
    return R.Recipe(
        capacity=n,
        radius=0.05,
        uploads=[R.Upload(0, np.asarray(start, np.float32), np.zeros((n, 3), np.float32),
                          np.broadcast_to(np.asarray(inv_mass, np.float32), (n,)).copy())],
        materials=[("soft", R.SoftbodyOpts([body], "global"))],
        loop=R.LoopOpts(substeps=1, iterations=iterations, gravity=(0.0, 0.0, 0.0)),
        name="shape-match-cube",
    )


def shape_match_weights(inv_mass: np.ndarray) -> np.ndarray:
    """SoftbodySystem.ts:366-372: each dynamic particle weighs its mass over the
    body's mean mass (all 1 when the masses are equal), a kinematic one 1."""
    inv_mass = np.asarray(inv_mass, np.float64)
    m = np.where(inv_mass > 0, 1.0 / np.where(inv_mass > 0, inv_mass, 1.0), 0.0)
    dyn = m[m > 0]
    if dyn.size == 0 or np.all(dyn == dyn[0]):
        return np.ones_like(m)
    return np.where(m > 0, m / dyn.mean(), 1.0)


def shape_match_goal(rest: np.ndarray, x: np.ndarray, weights=None) -> np.ndarray:
    """goal_i = R r_i + c for the frame fitted to positions x: c the weighted
    mean of x, r_i the rest positions less their weighted centre, R the
    rotation of the polar decomposition of sum w_i (x_i - c) r_i^T
    (shapeMatch.ts:49-135, SoftbodySystem.ts:181-189, the test's CPU check)."""
    x = np.asarray(x, np.float64)
    r = np.asarray(rest, np.float64)
    w = np.ones(len(x)) if weights is None else np.asarray(weights, np.float64)
    c, rc = (w[:, None] * x).sum(0) / w.sum(), (w[:, None] * r).sum(0) / w.sum()
    a = (w[:, None] * (x - c)).T @ (r - rc)
    u, _, vt = np.linalg.svd(a)
    d = np.sign(np.linalg.det(u @ vt))
    rot = u @ np.diag([1.0, 1.0, d]) @ vt
    return (r - rc) @ rot.T + c


# ------------------------------------------------------------- non-penetration
def non_penetration() -> R.Recipe:
    """tests/analytical/collider/collider-non-penetration.gpu.test.ts:46-81:
    three particles (r = 0.05) and one PrimitiveSet of a plane at y = 0, a
    solid sphere below it and an inverted box (a container) around (1, 0, 0),
    each with muS 0.3 and muK 0.2; 4 substeps, 4 iterations, gravity -9.81."""
    pos = np.array([[-1.0, 0.5, 0.0], [0.0, 0.0, 0.0], [1.0, 0.0, 0.0]], np.float32)
    prims = [R.plane((0, 1, 0), (-1.0, 0.0, 0.0), 0.3, 0.2),
             R.sphere((0.0, -0.5, 0.0), 0.3, mu_s=0.3, mu_k=0.2),
             R.box((1.0, 0.0, 0.0), (0.3, 0.3, 0.3), invert=True, mu_s=0.3, mu_k=0.2)]
    return R.Recipe(capacity=3, radius=0.05,
                    uploads=[R.Upload(0, pos, np.zeros_like(pos), np.ones(3, np.float32))],
                    prims=prims, loop=R.LoopOpts(substeps=4, iterations=4), name="non-penetration")


def non_penetration_phis(x: np.ndarray) -> np.ndarray:
    """The test's CPU SDFs (collider-non-penetration.gpu.test.ts:23-44) of
    each particle against the plane, the sphere and the inverted box."""
    x = np.asarray(x, np.float64)[:, :3]
    plane = x[:, 1] - 0.0
    sphere = np.linalg.norm(x - np.array([0.0, -0.5, 0.0]), axis=1) - 0.3
    q = np.abs(x - np.array([1.0, 0.0, 0.0])) - 0.3
    box = np.linalg.norm(np.maximum(q, 0.0), axis=1) + np.minimum(q.max(1), 0.0)
    return np.stack([plane, sphere, -box], axis=1)


def axis_angle_quat(axis, angle: float) -> tuple:
    """(x, y, z, w) of a rotation by `angle` about the unit `axis`."""
    s = math.sin(angle / 2.0)
    return (axis[0] * s, axis[1] * s, axis[2] * s, math.cos(angle / 2.0))


ROTATED_BOXES = [  # collider-rotated-box-non-penetration.gpu.test.ts:67-95: centre, half extents, rotation, invert
    ((-1.0, 0.0, 0.0), (0.4, 0.05, 0.4), axis_angle_quat((0, 0, 1), math.pi / 6), False),
    ((0.0, 0.0, 0.0), (0.4, 0.05, 0.4), axis_angle_quat((1, 0, 0), math.pi / 4), False),
    ((1.0, 0.0, 0.0), (0.3, 0.3, 0.3), axis_angle_quat((0, 1, 0), math.pi / 5), True),
]


def rotated_boxes() -> R.Recipe:
    """collider-rotated-box-non-penetration.gpu.test.ts:52-104: three
    particles (r = 0.05) above two tilted slabs and inside a rotated
    container, muS 0.3 and muK 0.2; 4 substeps, 4 iterations, gravity -9.81."""
    pos = np.array([[-1.0, 0.8, 0.0], [0.0, 0.8, 0.0], [1.0, 0.0, 0.0]], np.float32)
    prims = [R.box(c, h, rotation=q, invert=inv, mu_s=0.3, mu_k=0.2) for c, h, q, inv in ROTATED_BOXES]
    return R.Recipe(capacity=3, radius=0.05,
                    uploads=[R.Upload(0, pos, np.zeros_like(pos), np.ones(3, np.float32))],
                    prims=prims, loop=R.LoopOpts(substeps=4, iterations=4), name="rotated-boxes")


def rotated_box_phis(x: np.ndarray) -> np.ndarray:
    """The test's CPU oriented-box SDF (lines 30-49): the point in the box's
    frame by the inverse rotation, then the axis-aligned box distance."""
    x = np.asarray(x, np.float64)[:, :3]
    out = []
    for c, h, q, inv in ROTATED_BOXES:
        qx, qy, qz, qw = q
        rot = np.array([[1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qz * qw), 2 * (qx * qz + qy * qw)],
                        [2 * (qx * qy + qz * qw), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qx * qw)],
                        [2 * (qx * qz - qy * qw), 2 * (qy * qz + qx * qw), 1 - 2 * (qx * qx + qy * qy)]])
        local = (x - np.asarray(c)) @ rot  # rows: rot^T (x - c)
        d = np.abs(local) - np.asarray(h)
        dist = np.linalg.norm(np.maximum(d, 0.0), axis=1) + np.minimum(d.max(1), 0.0)
        out.append(-dist if inv else dist)
    return np.stack(out, axis=1)


def sphere_bowl(n: int = 100) -> R.Recipe:
    """collider-sphere-bowl-rest.gpu.test.ts:34-88: 100 particles (r = 0.05)
    in a cloud above the centre of an inverted unit sphere (muS 0.5, muK 0.4),
    placed by the test's LCG from seed 0xc0ffee; particle contacts on
    (maxContacts 8N, muS 0.5, muK 0.4); 4 substeps, 4 iterations."""
    rand = lcg_js(0xC0FFEE)
    pos = []
    for _ in range(n):
        x = 0.3 * (rand() * 2 - 1)
        y = 0.3 + 0.3 * abs(rand() * 2 - 1)
        z = 0.3 * (rand() * 2 - 1)
        pos.append((x, y, z))
    return particles(pos, 0.05, 4, 4, vel=np.zeros((n, 3), np.float32), inv_mass=np.ones(n, np.float32),
                     contact=(8 * n, 0.5, 0.4), prims=[R.sphere((0.0, 0.0, 0.0), 1.0, invert=True, mu_s=0.5, mu_k=0.4)],
                     name="sphere-bowl")


def spring_pair(compliance: float, substeps: int, iterations: int, offset: float = 0.05) -> R.Recipe:
    """xpbd-frequency.gpu.test.ts:66-106: particle 0 pinned at the origin,
    particle 1 (mass 1) released at (0, -(1 + offset), 0), one distance
    constraint of rest length 1 and compliance alpha, no gravity."""
    pos = np.array([[0.0, 0.0, 0.0], [0.0, -(1.0 + offset), 0.0]], np.float32)
    w = np.array([0.0, 1.0], np.float32)
    r = R.Recipe(capacity=2, radius=0.02,
                 loop=R.LoopOpts(substeps=substeps, iterations=iterations, gravity=(0.0, 0.0, 0.0)),
                 name=f"spring-{compliance:g}")
    r.materials.append(("cloth", R.ClothOpts(offset=0, positions=pos, inv_mass=w,
                                             pairs=np.array([[0, 1]], np.uint32),
                                             rest_lengths=np.array([1.0], np.float32),
                                             stretch_compliance=compliance)))
    return r


def spring_period(scene, frame_dt: float, frames: int) -> float:
    """The test's period estimate (lines 126-157): upward zero crossings of
    y + 1, interpolated within the frame, averaged gap."""
    from pfsim import _native as N

    disp = []
    for _ in range(frames):
        scene.step(frame_dt)
        disp.append(float(scene.readback(N.PF_FIELD_POSITIONS)[1, 1]) + 1.0)
    t = [(i - 1 + (0.0 if disp[i - 1] == disp[i] else -disp[i - 1] / (disp[i] - disp[i - 1]))) * frame_dt
         for i in range(1, frames) if disp[i - 1] <= 0 < disp[i]]
    assert len(t) >= 3, t
    return float(np.mean(np.diff(t)))


def energy_drift_cloud(n: int = 1000):
    """integrate-energy-drift.gpu.test.ts:26-48: 1000 particles from the
    test's LCG (seed 0xc0ffee), positions in [-5, 5] x [10, 50] x [-5, 5] and
    velocities in [-2, 2]^3 drawn particle by particle; no material, no
    collider, one substep. Returns the recipe and the initial state."""
    rand = lcg_js(0xC0FFEE)
    pos, vel = [], []
    for _ in range(n):
        pos.append([-5 + 10 * rand(), 10 + 40 * rand(), -5 + 10 * rand()])
        vel.append([-2 + 4 * rand(), -2 + 4 * rand(), -2 + 4 * rand()])
    pos, vel = np.array(pos, np.float32), np.array(vel, np.float32)
    rec = particles(pos, 0.05, 1, 2, vel=vel, inv_mass=np.ones(n, np.float32), name="energy-drift")
    return rec, pos, vel


def mean_energy(pos, vel) -> float:
    """The test's mean energy per particle, 1/2 |v|^2 + g y."""
    pos, vel = np.asarray(pos, np.float64), np.asarray(vel, np.float64)
    return float((0.5 * (vel[:, :3] ** 2).sum(1) + G * pos[:, 1]).mean())


def sealed_tank():
    """mass-conservation.gpu.test.ts:24-77: 8 x 12 x 8 = 768 fluid particles
    at spacing 0.025 (r = spacing / 2, h = 0.05, rest density 1000,
    compliance 1e-4, mass rest density x spacing^3) in an open-top tank of
    five planes at +-0.15 in x and z; 4 substeps, 2 iterations."""
    s, nx, ny, nz = 0.025, 8, 12, 8
    pos = [[-(nx * s) / 2 + s * 0.5 + i * s, s * 0.5 + j * s, -(nz * s) / 2 + s * 0.5 + k * s]
           for j in range(ny) for k in range(nz) for i in range(nx)]
    pos = np.array(pos, np.float32)
    n = len(pos)
    w = np.full(n, np.float32(1.0 / (1000.0 * s ** 3)), np.float32)
    half = 0.15
    prims = [R.plane((0, 1, 0), (0.0, 0.0, 0.0)), R.plane((1, 0, 0), (-half, 0.0, 0.0)),
             R.plane((-1, 0, 0), (half, 0.0, 0.0)), R.plane((0, 0, 1), (0.0, 0.0, -half)),
             R.plane((0, 0, -1), (0.0, 0.0, half))]
    r = R.Recipe(capacity=n, radius=s * 0.5, uploads=[R.Upload(0, pos, np.zeros_like(pos), w)], prims=prims,
                 loop=R.LoopOpts(substeps=4, iterations=2), name="sealed-tank")
    r.materials.append(("fluid", R.FluidOpts(range=(0, n), rest_density=1000.0, particle_spacing=s,
                                             smoothing_radius=0.05, compliance=1e-4)))
    return r


def box_container(n: int = 1000) -> R.Recipe:
    """collider-box-container.gpu.test.ts:24-73: 1000 particles (r = 0.02)
    from the test's LCG (seed 0xdecafbad) in x, z in [-0.4, 0.4], y in [0.2,
    0.45], dropped in an inverted unit box (muS 0.5, muK 0.4); particle
    contacts on (maxContacts 8N, default friction); 4 substeps, 4 iterations."""
    rand = lcg_js(0xDECAFBAD)
    pos = []
    for _ in range(n):
        x = (rand() * 2 - 1) * 0.4
        y = 0.2 + rand() * 0.25
        z = (rand() * 2 - 1) * 0.4
        pos.append((x, y, z))
    return particles(pos, 0.02, 4, 4, vel=np.zeros((n, 3), np.float32), inv_mass=np.ones(n, np.float32),
                     contact=(8 * n, -1.0, -1.0),
                     prims=[R.box((0.0, 0.0, 0.0), (0.5, 0.5, 0.5), invert=True, mu_s=0.5, mu_k=0.4)],
                     name="box-container")
