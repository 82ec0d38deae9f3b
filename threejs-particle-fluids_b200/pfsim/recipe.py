"""Backend-neutral scene descriptions and the native (CUDA) backend.

A ``Recipe`` is a plain description of one scene in the reference's terms: a
ParticleSystem (capacity, radius, uploaded particles), materials in SimLoop
order (FluidSystem, SoftbodySystem, ClothSystem), PrimitiveSet primitives and
the SimLoop options. ``NativeBackend.build(recipe)`` replays it through the C
ABI in the order the reference's constructors would run, and returns a
``Scene`` handle. Any other object with the same methods (the CPU oracle in
the test suite) can replay the same recipe.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from . import _native as N

# ---------------------------------------------------------------- recipe ----


@dataclass
class Upload:
    start: int
    pos: np.ndarray  # (n, 3) or (n, 4) float32
    vel: np.ndarray | None = None
    inv_mass: np.ndarray | None = None
    group: np.ndarray | None = None  # collision groups (uint32)


@dataclass
class FluidOpts:
    """FluidSystemOptions (src/fluids/FluidSystem.ts:31-54)."""

    range: tuple[int, int] = (0, 0)  # (start, count); count 0 = every particle
    rest_density: float = 0.0
    particle_spacing: float = 0.0
    smoothing_radius: float = 0.0
    compliance: float = -1.0
    viscosity: float | None = None
    vorticity: float | None = None
    surface_tension: float | None = None
    adhesion: float | None = None
    boundaries: list[tuple[int, int]] = field(default_factory=list)
    boundary_static: list[bool] = field(default_factory=list)


@dataclass
class BodyDef:
    """SoftbodyDef (src/softbody/SoftbodySystem.ts:29-60)."""

    range: tuple[int, int]
    surface_count: int | None = None
    compliance: float = 0.0
    rest_positions: np.ndarray | None = None
    edges: np.ndarray | None = None  # (m, 2) body-local pairs


@dataclass
class SoftbodyOpts:
    bodies: list[BodyDef]
    shape_matching: str = "global"
    self_collision: bool = False


@dataclass
class ClothOpts:
    """ClothSystemOptions with a ClothGraph (src/cloth/ClothSystem.ts:37-70)."""

    offset: int
    positions: np.ndarray  # (n, 3)
    inv_mass: np.ndarray  # (n,)
    pairs: np.ndarray  # (m, 2) cloth-local
    rest_lengths: np.ndarray  # (m,)
    stretch_compliance: float = -1.0
    bending: np.ndarray | None = None  # (b, 4) cloth-local (p1, p2, p3, p4)
    bending_rest: np.ndarray | None = None  # (b,) signed rest angles
    bend_compliance: float = -1.0
    tether_particle: np.ndarray | None = None  # (t,) cloth-local free particles
    tether_anchor: np.ndarray | None = None  # (t,) cloth-local pinned anchors
    tether_rest: np.ndarray | None = None  # (t,) rest radii
    tether_compliance: float = -1.0
    triangles: np.ndarray | None = None  # (k, 3) cloth-local: drag and lift (aero.ts)
    wind: tuple = (0.0, 0.0, 0.0)
    drag: float = -1.0
    lift: float = -1.0
    damping: float | None = None  # None: no velocity smoothing pass


def cloth_params(wind=(0.0, 0.0, 0.0), drag: float = 0.6125, lift: float = 0.3, damping: float = 0.0,
                 bend_compliance: float = 1e-5) -> N.ClothParams:
    """The ClothSystem setters' values as the C-ABI's pf_cloth_params."""
    p = N.ClothParams()
    p.wind[:] = [float(w) for w in wind]
    p.drag, p.lift, p.damping, p.bend_compliance = drag, lift, damping, bend_compliance
    return p


@dataclass
class Prim:
    kind: int
    flags: int = 0
    data0: tuple = (0.0, 0.0, 0.0, 0.0)
    data1: tuple = (0.0, 0.0, 0.0, 0.0)
    velocity: tuple = (0.0, 0.0, 0.0, 0.0)
    rotation: tuple = (0.0, 0.0, 0.0, 1.0)
    spin: tuple = (0.0, 0.0, 0.0, 0.0)

    def cstruct(self) -> N.Primitive:
        p = N.Primitive()
        p.kind, p.flags = int(self.kind), int(self.flags)
        p.data0[:] = [float(v) for v in self.data0]
        p.data1[:] = [float(v) for v in self.data1]
        p.velocity[:] = [float(v) for v in self.velocity]
        p.rotation[:] = [float(v) for v in self.rotation]
        p.spin[:] = [float(v) for v in self.spin]
        return p


@dataclass
class Sdf:
    """SDFData + SDFColliderOptions (src/core/collision/SDFCollider.ts:32-58)."""

    data: np.ndarray  # (nz, ny, nx) float32 distances, x fastest in memory
    origin: tuple
    voxel_size: tuple
    position: tuple = (0.0, 0.0, 0.0)
    rotation: tuple = (0.0, 0.0, 0.0, 1.0)
    scale: float = 1.0
    thickness: float = 0.0
    mu_s: float = 0.5
    mu_k: float = 0.4

    def cstruct(self, keep) -> N.SdfDesc:
        d = N.SdfDesc()
        arr = np.ascontiguousarray(self.data, np.float32)
        nz, ny, nx = arr.shape
        d.res[:] = [nx, ny, nz]
        d.data = keep.f32(arr.reshape(-1))
        d.origin[:] = [float(v) for v in self.origin]
        d.voxel_size[:] = [float(v) for v in self.voxel_size]
        d.position[:] = [float(v) for v in self.position]
        d.rotation[:] = [float(v) for v in self.rotation]
        d.scale, d.thickness, d.mu_s, d.mu_k = float(self.scale), float(self.thickness), float(self.mu_s), float(self.mu_k)
        return d


def sphere_sdf(center, radius, res: int = 32, pad: float = 0.25, invert: bool = False, **kw) -> Sdf:
    """A baked sphere: distances at voxel centres of a res^3 grid around it
    (negated for a bowl that holds particles inside)."""
    c = np.asarray(center, np.float64)
    ext = radius * (1.0 + pad)
    vs = 2.0 * ext / res
    idx = (np.arange(res) + 0.5) * vs - ext
    z, y, x = np.meshgrid(idx, idx, idx, indexing="ij")
    d = np.sqrt(x * x + y * y + z * z) - radius
    if invert:
        d = -d
    return Sdf(d.astype(np.float32), tuple(c - ext), (vs, vs, vs), **kw)


def plane(normal, point, mu_s: float = 0.5, mu_k: float = 0.4) -> Prim:
    """PrimitiveSet.addPlane (PrimitiveSet.ts:166-170): the normal is normalised."""
    n = np.asarray(normal, np.float64)
    n = n / np.linalg.norm(n)
    return Prim(N.PF_PRIM_PLANE, 0, (*n, 0.0), (*point, mu_s), (0.0, 0.0, 0.0, mu_k))


def sphere(center, radius, invert=False, mu_s=0.5, mu_k=0.4, velocity=(0.0, 0.0, 0.0)) -> Prim:
    return Prim(N.PF_PRIM_SPHERE, N.PF_PRIM_INVERT if invert else 0, (*center, radius), (0.0, 0.0, 0.0, mu_s),
                (*velocity, mu_k))


def box(center, half, rotation=(0.0, 0.0, 0.0, 1.0), invert=False, mu_s=0.5, mu_k=0.4) -> Prim:
    return Prim(N.PF_PRIM_BOX, N.PF_PRIM_INVERT if invert else 0, (*center, 0.0), (*half, mu_s), (0.0, 0.0, 0.0, mu_k),
                tuple(rotation))


def capsule(a, b, radius, mu_s=0.5, mu_k=0.4) -> Prim:
    return Prim(N.PF_PRIM_CAPSULE, 0, (*a, radius), (*b, mu_s), (0.0, 0.0, 0.0, mu_k))


def container_walls(lo, hi, closed: bool = False) -> list[Prim]:
    """The Simulation façade's container planes (Simulation.ts:779-787)."""
    walls = [
        plane((0, 1, 0), lo),
        plane((1, 0, 0), lo),
        plane((-1, 0, 0), hi),
        plane((0, 0, 1), lo),
        plane((0, 0, -1), hi),
    ]
    if closed:
        walls.append(plane((0, -1, 0), hi))
    return walls


@dataclass
class LoopOpts:
    """SimLoopOptions (src/core/loop.ts:33-57) plus the grid bounds."""

    substeps: int = 4
    iterations: int = 2
    gravity: tuple = (0.0, -9.81, 0.0)
    hash_origin: tuple = (0.0, 0.0, 0.0)
    grid_min: tuple = (0.0, 0.0, 0.0)
    grid_max: tuple = (0.0, 0.0, 0.0)
    contact: bool = False  # SimLoopOptions.contact
    contact_mu_s: float = -1.0
    contact_mu_k: float = -1.0
    max_contacts: int = 0


@dataclass
class Recipe:
    capacity: int
    radius: float
    uploads: list[Upload] = field(default_factory=list)
    materials: list[tuple[str, Any]] = field(default_factory=list)
    prims: list[Prim] = field(default_factory=list)
    sdfs: list[Sdf] = field(default_factory=list)
    loop: LoopOpts = field(default_factory=LoopOpts)
    quiet: list = field(default_factory=list)  # noSelfContacts ranges (start, count) of no material
    name: str = ""
    # optional per-step primitive motion: fn(step_index, dt) -> {slot: Prim}
    motion: Any = None

    @property
    def particle_substeps(self) -> int:
        return self.capacity * self.loop.substeps


# --------------------------------------------------- C struct conversion ----
class _Keep:
    """Keeps numpy buffers alive while a C call reads them."""

    def __init__(self):
        self.refs = []

    def f32(self, a, shape_last=None):
        arr = np.ascontiguousarray(a, dtype=np.float32)
        self.refs.append(arr)
        return arr.ctypes.data_as(C.POINTER(C.c_float))

    def u32(self, a):
        arr = np.ascontiguousarray(a, dtype=np.uint32)
        self.refs.append(arr)
        return arr.ctypes.data_as(C.POINTER(C.c_uint32))


def pos4(a: np.ndarray) -> np.ndarray:
    a = np.asarray(a, np.float32)
    if a.shape[1] == 4:
        return np.ascontiguousarray(a)
    out = np.zeros((a.shape[0], 4), np.float32)
    out[:, :3] = a
    return out


def fluid_desc(o: FluidOpts, keep: _Keep) -> N.FluidDesc:
    d = N.FluidDesc()
    d.range.start, d.range.count = o.range
    d.rest_density = o.rest_density
    d.particle_spacing = o.particle_spacing
    d.smoothing_radius = o.smoothing_radius
    d.compliance = o.compliance
    if o.viscosity is not None:
        d.viscosity = o.viscosity
        d.flags |= N.PF_FLUID_VISCOSITY
    if o.vorticity is not None:
        d.vorticity = o.vorticity
        d.flags |= N.PF_FLUID_VORTICITY
    if o.surface_tension is not None:
        d.surface_tension = o.surface_tension
        d.flags |= N.PF_FLUID_SURFACE_TENSION
    if o.adhesion is not None:
        d.adhesion = o.adhesion
        d.flags |= N.PF_FLUID_ADHESION
    if o.boundaries:
        arr = (N.Range * len(o.boundaries))(*[N.Range(s, c) for s, c in o.boundaries])
        keep.refs.append(arr)
        d.n_boundaries = len(o.boundaries)
        d.boundaries = C.cast(arr, C.POINTER(N.Range))
        st = np.array([1 if (i < len(o.boundary_static) and o.boundary_static[i]) else 0 for i in range(len(o.boundaries))], np.uint8)
        keep.refs.append(st)
        d.boundary_static = st.ctypes.data_as(C.POINTER(C.c_uint8))
    return d


def softbody_desc(o: SoftbodyOpts, keep: _Keep) -> N.SoftbodyDesc:
    defs = (N.SoftbodyDef * len(o.bodies))()
    for i, b in enumerate(o.bodies):
        defs[i].range.start, defs[i].range.count = b.range
        defs[i].surface_count = 0xFFFFFFFF if b.surface_count is None else int(b.surface_count)
        defs[i].compliance = b.compliance
        if b.rest_positions is not None:
            defs[i].rest_positions = keep.f32(np.asarray(b.rest_positions, np.float32).reshape(-1))
        if b.edges is not None and len(b.edges):
            e = np.asarray(b.edges, np.uint32).reshape(-1)
            defs[i].edges = keep.u32(e)
            defs[i].n_edges = e.size // 2
    keep.refs.append(defs)
    d = N.SoftbodyDesc()
    d.n_bodies = len(o.bodies)
    d.bodies = C.cast(defs, C.POINTER(N.SoftbodyDef))
    d.shape_matching = N.PF_SHAPE_MATCH_LOCAL if o.shape_matching == "local" else N.PF_SHAPE_MATCH_GLOBAL
    d.self_collision = 1 if o.self_collision else 0
    return d


def cloth_desc(o: ClothOpts, keep: _Keep) -> N.ClothDesc:
    d = N.ClothDesc()
    d.offset = o.offset
    d.n_particles = len(o.positions)
    d.positions = keep.f32(np.asarray(o.positions, np.float32).reshape(-1))
    d.inv_mass = keep.f32(o.inv_mass)
    pr = np.asarray(o.pairs, np.uint32).reshape(-1)
    d.n_pairs = pr.size // 2
    d.pairs = keep.u32(pr)
    d.rest_lengths = keep.f32(o.rest_lengths)
    d.stretch_compliance = o.stretch_compliance
    if o.bending is not None and len(o.bending):
        b = np.asarray(o.bending, np.uint32).reshape(-1)
        d.n_bending = b.size // 4
        d.bending = keep.u32(b)
        d.bending_rest = keep.f32(np.asarray(o.bending_rest, np.float32))
    d.bend_compliance = o.bend_compliance
    if o.tether_particle is not None and len(o.tether_particle):
        d.n_tethers = len(o.tether_particle)
        d.tether_particle = keep.u32(np.asarray(o.tether_particle, np.uint32))
        d.tether_anchor = keep.u32(np.asarray(o.tether_anchor, np.uint32))
        d.tether_rest = keep.f32(np.asarray(o.tether_rest, np.float32))
    d.tether_compliance = o.tether_compliance
    if o.triangles is not None and len(o.triangles):
        t = np.asarray(o.triangles, np.uint32).reshape(-1)
        d.n_triangles = t.size // 3
        d.triangles = keep.u32(t)
    d.wind[:] = [float(w) for w in o.wind]
    d.drag, d.lift = o.drag, o.lift
    if o.damping is not None:
        d.has_damping, d.damping = 1, o.damping
    return d


def loop_desc(o: LoopOpts) -> N.LoopDesc:
    d = N.LoopDesc()
    d.substeps, d.iterations = o.substeps, o.iterations
    d.gravity[:] = list(o.gravity)
    d.hash_origin[:] = list(o.hash_origin)
    d.grid_min[:] = list(o.grid_min)
    d.grid_max[:] = list(o.grid_max)
    d.contact = 1 if o.contact else 0
    d.contact_mu_s, d.contact_mu_k, d.max_contacts = o.contact_mu_s, o.contact_mu_k, o.max_contacts
    return d


def read_contacts(fn, handle, capacity: int) -> tuple[int, np.ndarray]:
    cap = max(1, 32 * capacity)
    out = np.empty(2 * cap, np.uint32)
    count, stored = C.c_uint32(0), C.c_uint32(0)
    N.check(fn(handle, out.ctypes.data_as(C.POINTER(C.c_uint32)), cap, C.byref(count), C.byref(stored)))
    m = min(stored.value, cap)
    return int(count.value), out[: 2 * m].reshape(-1, 2).copy()


# --------------------------------------------------------- native backend ----
FIELD_SHAPES = {
    N.PF_FIELD_POSITIONS: (np.float32, 4),
    N.PF_FIELD_PREDICTED: (np.float32, 4),
    N.PF_FIELD_VELOCITIES: (np.float32, 4),
    N.PF_FIELD_INV_MASS: (np.float32, 1),
    N.PF_FIELD_BOUNDARY_VOLUME: (np.float32, 1),
    N.PF_FIELD_DENSITY: (np.float32, 1),
    N.PF_FIELD_ROTATION: (np.float32, 4),
    N.PF_FIELD_PREDICTED_ROTATION: (np.float32, 4),
    N.PF_FIELD_ANGULAR_VELOCITY: (np.float32, 4),
    N.PF_FIELD_LAMBDA: (np.float32, 1),
    N.PF_FIELD_NEIGHBOR_COUNT: (np.uint32, 1),
    N.PF_FIELD_NEIGHBORS: (np.uint32, N.MAX_NEIGHBORS),
    N.PF_FIELD_CELL_PERM: (np.uint32, 1),
}


def alloc_field(field_id: int, capacity: int) -> np.ndarray:
    dt, width = FIELD_SHAPES[field_id]
    return np.empty((capacity, width) if width > 1 else (capacity,), dt)


class Scene:
    """A built scene on the native backend (pf_scene handle)."""

    def __init__(self, handle, recipe: Recipe):
        self.h = handle
        self.recipe = recipe
        self.capacity = recipe.capacity
        self.steps = 0

    def step(self, dt: float) -> None:
        L = N.lib()
        if self.recipe.motion is not None:
            for slot, prim in self.recipe.motion(self.steps, dt).items():
                p = prim.cstruct()
                N.check(L.pf_set_primitive(self.h, slot, C.byref(p)))
        N.check(L.pf_step(self.h, float(dt)))
        self.steps += 1

    def set_primitive(self, slot: int, prim: Prim) -> None:
        p = prim.cstruct()
        N.check(N.lib().pf_set_primitive(self.h, slot, C.byref(p)))

    def contacts(self) -> tuple[int, np.ndarray]:
        """pf_contacts_read: (pairs found in the last substep, dropped ones
        included; the stored pairs as an (m, 2) array, each pair ascending,
        sorted)."""
        return read_contacts(N.lib().pf_contacts_read, self.h, self.capacity)

    def write(self, field_id: int, data: np.ndarray) -> None:
        """pf_write: a whole field (positions, predicted, velocities: float4 x
        capacity; inverse mass: float x capacity) in particle order."""
        a = np.ascontiguousarray(data, np.float32)
        N.check(N.lib().pf_write(self.h, field_id, a.ctypes.data_as(C.c_void_p), a.nbytes))

    def set_cloth_params(self, material: int, params: N.ClothParams) -> None:
        """pf_cloth_set_params: the ClothSystem setters of material `material`."""
        N.check(N.lib().pf_cloth_set_params(self.h, material, C.byref(params)))

    def readback(self, field_id: int) -> np.ndarray:
        out = alloc_field(field_id, self.capacity)
        N.check(N.lib().pf_readback(self.h, field_id, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def overflow(self) -> dict:
        o = N.Overflow()
        N.check(N.lib().pf_overflow_read(self.h, C.byref(o)))
        return {k: bool(getattr(o, k)) for k, _ in N.Overflow._fields_}

    def last_step_ms(self) -> float:
        ms = C.c_float(0)
        N.check(N.lib().pf_last_step_ms(self.h, C.byref(ms)))
        return ms.value

    def close(self) -> None:
        if self.h:
            N.lib().pf_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NativeBackend:
    """Replays recipes through libpfsim (the CUDA path)."""

    name = "cuda"

    def build(self, r: Recipe, build_loop: bool = True) -> Scene:
        L = N.lib()
        desc = N.SceneDesc(r.capacity, r.radius)
        h = C.c_void_p()
        N.check(L.pf_scene_create(C.byref(desc), C.byref(h)))
        scene = Scene(h, r)
        keep = _Keep()
        for u in r.uploads:
            p = pos4(u.pos)
            v = None if u.vel is None else keep.f32(pos4(u.vel))
            w = None if u.inv_mass is None else keep.f32(u.inv_mass)
            g = None if u.group is None else keep.u32(np.asarray(u.group, np.uint32))
            N.check(L.pf_upload_particles(h, keep.f32(p), v, w, g, u.start, p.shape[0]))
        for kind, opts in r.materials:
            if kind == "fluid":
                N.check(L.pf_add_fluid(h, C.byref(fluid_desc(opts, keep)), None))
            elif kind == "soft":
                N.check(L.pf_add_softbodies(h, C.byref(softbody_desc(opts, keep)), None))
            elif kind == "cloth":
                N.check(L.pf_add_cloth(h, C.byref(cloth_desc(opts, keep)), None))
            else:
                raise ValueError(kind)
        for q in r.quiet:
            N.check(L.pf_add_no_self_contacts(h, N.Range(*q)))
        for p in r.prims:
            cs = p.cstruct()
            N.check(L.pf_add_primitive(h, C.byref(cs), None))
        for g in r.sdfs:
            N.check(L.pf_add_sdf_collider(h, C.byref(g.cstruct(keep)), None))
        if build_loop:
            ld = loop_desc(r.loop)
            N.check(L.pf_loop_build(h, C.byref(ld)))
        return scene


class Batch:
    """Many built scenes stepped as one world (pf_batch): one launch per stage,
    one CUDA graph per tick."""

    def __init__(self, scenes: list[Scene], use_graph: bool = True):
        L = N.lib()
        arr = (C.c_void_p * len(scenes))(*[s.h for s in scenes])
        opts = N.BatchOpts(1 if use_graph else 0, 0)
        h = C.c_void_p()
        N.check(L.pf_batch_create(arr, len(scenes), C.byref(opts), C.byref(h)))
        self.h = h
        self.recipes = [s.recipe for s in scenes]
        self.capacities = [s.capacity for s in scenes]
        self.steps = 0

    def step(self, dt: float) -> None:
        L = N.lib()
        for i, r in enumerate(self.recipes):
            if r.motion is not None:
                for slot, prim in r.motion(self.steps, dt).items():
                    p = prim.cstruct()
                    N.check(L.pf_batch_set_primitive(self.h, i, slot, C.byref(p)))
        N.check(L.pf_batch_step(self.h, float(dt)))
        self.steps += 1

    def readback(self, index: int, field_id: int) -> np.ndarray:
        out = alloc_field(field_id, self.capacities[index])
        N.check(N.lib().pf_batch_readback(self.h, index, field_id, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def write(self, index: int, field_id: int, data: np.ndarray) -> None:
        a = np.ascontiguousarray(data, np.float32)
        N.check(N.lib().pf_batch_write(self.h, index, field_id, a.ctypes.data_as(C.c_void_p), a.nbytes))

    def set_cloth_params(self, index: int, material: int, params: N.ClothParams) -> None:
        N.check(N.lib().pf_batch_cloth_set_params(self.h, index, material, C.byref(params)))

    def overflow(self, index: int) -> dict:
        o = N.Overflow()
        N.check(N.lib().pf_batch_overflow_read(self.h, index, C.byref(o)))
        return {k: bool(getattr(o, k)) for k, _ in N.Overflow._fields_}

    def last_step_ms(self) -> float:
        ms = C.c_float(0)
        N.check(N.lib().pf_batch_last_step_ms(self.h, C.byref(ms)))
        return ms.value

    def particle_substeps(self) -> int:
        return int(N.lib().pf_batch_particle_substeps(self.h))

    def close(self) -> None:
        if self.h:
            N.lib().pf_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous batching (pf_server): scenes are admitted in FIFO order as
    the HBM budget allows, every live scene is stepped once per tick, and a
    scene retires after its lifetime. Primitive motion callbacks of recipes
    are not applied to served scenes."""

    def __init__(self, budget_bytes: int = 0, max_scenes: int = 0, use_graph: bool = True, max_cohorts: int = 0,
                 plain: bool = False, async_build: bool = True):
        opts = N.ServerOpts(int(budget_bytes), int(max_scenes), 1 if use_graph else 0, int(max_cohorts),
                            N.PF_SERVER_PLAIN if plain else N.PF_SERVER_BATCHED, 1 if async_build else 0)
        h = C.c_void_p()
        N.check(N.lib().pf_server_create(C.byref(opts), C.byref(h)))
        self.h = h
        self.capacity: dict[int, int] = {}

    @staticmethod
    def estimate_bytes(r: Recipe) -> int:
        scene = NativeBackend().build(r, build_loop=False)
        out = C.c_uint64(0)
        ld = loop_desc(r.loop)
        N.check(N.lib().pf_server_estimate_bytes(scene.h, C.byref(ld), C.byref(out)))
        scene.close()
        return int(out.value)

    def submit(self, r: Recipe, lifetime: int) -> int:
        scene = NativeBackend().build(r, build_loop=False)
        ld = loop_desc(r.loop)
        t = C.c_uint64(0)
        try:
            N.check(N.lib().pf_server_submit(self.h, scene.h, C.byref(ld), int(lifetime), C.byref(t)))
        finally:
            scene.close()
        self.capacity[t.value] = r.capacity
        return int(t.value)

    def tick(self, dt: float) -> None:
        N.check(N.lib().pf_server_tick(self.h, float(dt)))

    def drain(self) -> None:
        N.check(N.lib().pf_server_drain_build(self.h))

    def state(self, ticket: int) -> tuple[int, int]:
        st, done = C.c_uint32(0), C.c_uint32(0)
        N.check(N.lib().pf_server_request_state(self.h, ticket, C.byref(st), C.byref(done)))
        return int(st.value), int(done.value)

    def readback(self, ticket: int, field_id: int) -> np.ndarray:
        out = alloc_field(field_id, self.capacity[ticket])
        N.check(N.lib().pf_server_readback(self.h, ticket, field_id, out.ctypes.data_as(C.c_void_p), out.nbytes))
        return out

    def stats(self) -> dict:
        o = N.ServerStats()
        N.check(N.lib().pf_server_stats_read(self.h, C.byref(o)))
        return {k: getattr(o, k) for k, _ in N.ServerStats._fields_ if k != "reserved0"}

    def close(self) -> None:
        if self.h:
            N.lib().pf_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
