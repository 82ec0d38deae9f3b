"""The reference's solver API, by the reference's names, on the CUDA path.

Low level (src/core, src/fluids, src/softbody, src/cloth):

    particles = ParticleSystem(capacity, particle_radius)
    particles.upload_particles([{"position": ..., "velocity": ..., "inv_mass": ...}, ...])
    fluid = FluidSystem(particles, range=(0, n), rest_density=..., particle_spacing=..., ...)
    colliders = PrimitiveSet(particles); colliders.add_plane((0, 1, 0), (0, 0, 0))
    loop = SimLoop(particles, substeps=4, iterations=2, materials=[fluid], colliders=[colliders])
    loop.step(1 / 60); snap = particles.readback(); loop.dispose()

The classes record what the reference's constructors record and build one
scene through the C ABI when the SimLoop is constructed (the point at which
the reference compiles its kernels). Errors are PfError with the reference's
"<Class>: <reason>" text. `Simulation` is the façade
(src/simulation/Simulation.ts:301-634) for containers, fluid boxes, soft
spheres and boxes, cloth sheets and primitive colliders, with the reference's
fluid defaults (viscosity, surface tension, vorticity, adhesion).
"""

from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass, field
from typing import Sequence

import numpy as np

from . import _native as N
from . import recipe as R
from . import shapes


def _err(cls: str, msg: str) -> N.PfError:
    return N.PfError(N.PF_ERR_INVALID, f"{cls}: {msg}")


@dataclass
class Snapshot:
    """ParticleSnapshot (src/core/particles.ts:200-227): float4 rows."""

    positions: np.ndarray
    velocities: np.ndarray


class ParticleSystem:
    """src/core/particles.ts:52-316."""

    def __init__(self, capacity: int, particle_radius: float):
        if not (isinstance(capacity, (int, np.integer)) and capacity > 0):
            raise _err("ParticleSystem", f"capacity must be a positive integer, got {capacity}")
        if not (particle_radius > 0 and math.isfinite(particle_radius)):
            raise _err("ParticleSystem", f"particleRadius must be positive, got {particle_radius}")
        self.capacity = int(capacity)
        self.particle_radius = float(particle_radius)
        self.uploads: list[R.Upload] = []
        self.loop: SimLoop | None = None
        self.disposed = False

    def upload_particles(self, particles, start: int = 0) -> None:
        """A list of {"position", "velocity"?, "inv_mass"?} or a (n, 3|4) array."""
        self._live()
        if isinstance(particles, np.ndarray):
            pos, vel, w = particles, None, None
        else:
            pos = np.array([p["position"] for p in particles], np.float32)
            vel = np.array([p.get("velocity", (0.0, 0.0, 0.0)) for p in particles], np.float32)
            w = np.array([p.get("inv_mass", 1.0) for p in particles], np.float32)
        if start + len(pos) > self.capacity:
            raise _err("ParticleSystem", f"upload of {len(pos)} particles at {start} exceeds capacity {self.capacity}")
        if self.loop is not None:
            raise N.PfError(N.PF_ERR_STATE, "ParticleSystem: upload before the SimLoop is built")
        self.uploads.append(R.Upload(start, np.asarray(pos, np.float32), vel, w))

    def readback(self) -> Snapshot:
        self._live()
        if self.loop is None or self.loop.scene is None:
            raise N.PfError(N.PF_ERR_STATE, "ParticleSystem: readback needs a built SimLoop")
        s = self.loop.scene
        return Snapshot(s.readback(N.PF_FIELD_POSITIONS), s.readback(N.PF_FIELD_VELOCITIES))

    def dispose(self) -> None:
        self.disposed = True

    def _live(self):
        if self.disposed:
            raise N.PfError(N.PF_ERR_STATE, "ParticleSystem: has been disposed")


class FluidSystem:
    """src/fluids/FluidSystem.ts:31-127 (options as FluidSystemOptions)."""

    def __init__(self, particles: ParticleSystem, range: tuple[int, int] | None = None, rest_density: float = 1000.0,
                 particle_spacing: float | None = None, smoothing_radius: float | None = None,
                 compliance: float = 1e-4, viscosity: float | None = None, vorticity: float | None = None,
                 surface_tension: float | None = None, adhesion: float | None = None,
                 boundaries: Sequence[tuple[int, int]] = (), boundary_static: Sequence[bool] = ()):
        spacing = particle_spacing if particle_spacing is not None else 2.0 * particles.particle_radius
        h = smoothing_radius if smoothing_radius is not None else 2.0 * spacing
        self.particles = particles
        self.opts = R.FluidOpts(range=tuple(range) if range else (0, particles.capacity), rest_density=rest_density,
                                particle_spacing=spacing, smoothing_radius=h, compliance=compliance,
                                viscosity=viscosity, vorticity=vorticity, surface_tension=surface_tension,
                                adhesion=adhesion, boundaries=list(boundaries),
                                boundary_static=list(boundary_static))
    kind = "fluid"


class SoftbodySystem:
    """src/softbody/SoftbodySystem.ts:29-199: bodies of {range, surface_count,
    compliance, rest_positions?, edges?}; shape_matching 'local' or 'global'."""

    def __init__(self, particles: ParticleSystem, bodies: list[dict], shape_matching: str = "local",
                 self_collision: bool = False):
        if shape_matching not in ("local", "global"):
            raise _err("SoftbodySystem", f"shapeMatching must be 'local' or 'global', got {shape_matching}")
        self.particles = particles
        self.opts = R.SoftbodyOpts([R.BodyDef(range=tuple(b["range"]), surface_count=b.get("surface_count"),
                                              compliance=b.get("compliance", 0.0),
                                              rest_positions=b.get("rest_positions"), edges=b.get("edges"))
                                    for b in bodies], shape_matching, bool(self_collision))
    kind = "soft"


class ClothSystem:
    """src/cloth/ClothSystem.ts:37-304 with a ClothGraph (pfsim.shapes):
    stretch, dihedral bending and long-range tether constraints (tethers
    built from the graph's pins by buildTethers), aerodynamic drag and lift
    on the graph's triangles, and the optional velocity smoothing pass. The
    wind, drag, lift, damping and bend_compliance setters take effect from
    the next step."""

    kind = "cloth"

    def __init__(self, particles: ParticleSystem, graph, offset: int = 0, stretch_compliance: float = 1e-7,
                 bend_compliance: float = 1e-5, tether_compliance: float = 0.0, stretch_tolerance: float = 0.0,
                 wind=(0.0, 0.0, 0.0), drag: float = 0.6125, lift: float = 0.3, damping: float | None = None):
        for name, v in (("stretchCompliance", stretch_compliance), ("bendCompliance", bend_compliance),
                        ("tetherCompliance", tether_compliance), ("stretchTolerance", stretch_tolerance),
                        ("drag", drag), ("lift", lift)):
            _non_negative(name, v)
        if damping is not None:
            _unit_interval("damping", damping)
        self.particles = particles
        self.graph = graph
        self.offset = offset
        self._wind = tuple(float(w) for w in wind)
        self._drag, self._lift = float(drag), float(lift)
        self._damping = damping
        self._bend = float(bend_compliance)
        self.tethers = shapes.build_tethers(graph.inv_mass, graph.pairs, graph.rest_lengths,
                                            stretch_tolerance=stretch_tolerance)
        tp, ta, tr = self.tethers
        self.opts = R.ClothOpts(offset=offset, positions=np.asarray(graph.positions, np.float32),
                                inv_mass=np.asarray(graph.inv_mass, np.float32), pairs=graph.pairs,
                                rest_lengths=np.asarray(graph.rest_lengths, np.float32),
                                stretch_compliance=stretch_compliance,
                                bending=graph.bending, bending_rest=np.asarray(graph.bending_rest, np.float32),
                                bend_compliance=bend_compliance,
                                tether_particle=tp, tether_anchor=ta, tether_rest=tr,
                                tether_compliance=tether_compliance, triangles=graph.triangles,
                                wind=self._wind, drag=drag, lift=lift, damping=damping)

    def _push(self) -> None:
        loop = self.particles.loop
        if loop is None or loop.scene is None or self not in loop.materials:
            return
        loop.scene.set_cloth_params(loop.materials.index(self), self.params())

    def params(self):
        return R.cloth_params(self._wind, self._drag, self._lift, self._damping or 0.0, self._bend)

    @property
    def wind(self) -> tuple:
        return self._wind

    @wind.setter
    def wind(self, value) -> None:
        w = tuple(float(x) for x in value)
        if len(w) != 3 or not all(math.isfinite(x) for x in w):
            raise _err("ClothSystem", f"wind must be three finite numbers, got {value}")
        self._wind = w
        self._push()

    @property
    def drag(self) -> float:
        return self._drag

    @drag.setter
    def drag(self, value: float) -> None:
        self._drag = _non_negative("drag", value)
        self._push()

    @property
    def lift(self) -> float:
        return self._lift

    @lift.setter
    def lift(self, value: float) -> None:
        self._lift = _non_negative("lift", value)
        self._push()

    @property
    def damping(self) -> float:
        return self._damping or 0.0

    @damping.setter
    def damping(self, value: float) -> None:
        _unit_interval("damping", value)
        if self._damping is None:
            raise _err("ClothSystem", "damping was not given at creation, so there is no smoothing pass to change")
        self._damping = float(value)
        self._push()

    @property
    def bend_compliance(self) -> float:
        return self._bend

    @bend_compliance.setter
    def bend_compliance(self, value: float) -> None:
        self._bend = _non_negative("bendCompliance", value)
        self._push()


def _non_negative(name: str, value: float) -> float:
    """ClothSystem.ts:290-295."""
    if not (value >= 0) or not math.isfinite(value):
        raise _err("ClothSystem", f"{name} must be ≥ 0, got {value}")
    return float(value)


def _unit_interval(name: str, value: float) -> float:
    """ClothSystem.ts:297-302."""
    if not (0 <= value <= 1):
        raise _err("ClothSystem", f"{name} must be between 0 and 1, got {value}")
    return float(value)


class PrimitiveSet:
    """src/core/collision/PrimitiveSet.ts:121-553."""

    def __init__(self, particles: ParticleSystem):
        self.particles = particles
        self.prims: list[R.Prim] = []
        self.loop: SimLoop | None = None

    def _add(self, p: R.Prim) -> int:
        if p.data1[3] < 0 or p.velocity[3] < 0:
            raise _err("PrimitiveSet", "friction coefficients must be non-negative")
        self.prims.append(p)
        return len(self.prims) - 1

    def add_plane(self, normal, point, mu_s: float = 0.5, mu_k: float = 0.4) -> int:
        return self._add(R.plane(normal, point, mu_s, mu_k))

    def add_sphere(self, center, radius: float, invert: bool = False, mu_s: float = 0.5, mu_k: float = 0.4) -> int:
        return self._add(R.sphere(center, radius, invert, mu_s, mu_k))

    def add_box(self, center, half, rotation=(0.0, 0.0, 0.0, 1.0), invert: bool = False, mu_s: float = 0.5,
                mu_k: float = 0.4) -> int:
        return self._add(R.box(center, half, rotation, invert, mu_s, mu_k))

    def add_capsule(self, a, b, radius: float, mu_s: float = 0.5, mu_k: float = 0.4) -> int:
        return self._add(R.capsule(a, b, radius, mu_s, mu_k))

    def set_sphere(self, slot: int, center, radius: float, velocity=(0.0, 0.0, 0.0)) -> None:
        """PrimitiveSet.setSphere: moves a sphere; with a velocity its contact
        sweeps (FLAG_SWEEP)."""
        p = self.prims[slot]
        q = R.Prim(p.kind, p.flags | (N.PF_PRIM_SWEEP if any(velocity) else 0), (*center, radius), p.data1,
                   (*velocity, p.velocity[3]), p.rotation, p.spin)
        self.prims[slot] = q
        if self.loop is not None and self.loop.scene is not None:
            self.loop.scene.set_primitive(self.loop.prim_base(self) + slot, q)


class SDFCollider:
    """src/core/collision/SDFCollider.ts:62-317."""

    def __init__(self, particles: ParticleSystem, data: np.ndarray, origin, voxel_size, mu_s: float = 0.5,
                 mu_k: float = 0.4, thickness: float = 0.0, position=(0.0, 0.0, 0.0),
                 rotation=(0.0, 0.0, 0.0, 1.0), scale: float = 1.0):
        arr = np.asarray(data, np.float32)
        if arr.ndim != 3 or min(arr.shape) < 4:
            raise _err("SDFCollider", f"resolution must be integers >= 4, got {list(arr.shape[::-1])}")
        if not thickness >= 0:
            raise _err("SDFCollider", f"thickness must be non-negative, got {thickness}")
        self.particles = particles
        self.sdf = R.Sdf(arr, tuple(origin), tuple(voxel_size), tuple(position), tuple(rotation), float(scale),
                         float(thickness), float(mu_s), float(mu_k))
        self.loop: SimLoop | None = None


class SimLoop:
    """src/core/loop.ts:33-57, 92-417: builds the scene (one world on the
    GPU) from the particle system, its materials in order and its colliders."""

    def __init__(self, particles: ParticleSystem, substeps: int = 4, iterations: int = 2,
                 gravity=(0.0, -9.81, 0.0), materials: Sequence = (), colliders: Sequence = (),
                 hash_origin=(0.0, 0.0, 0.0), grid_min=(0.0, 0.0, 0.0), grid_max=(0.0, 0.0, 0.0),
                 contact: bool | dict = False):
        if not (isinstance(substeps, int) and substeps >= 1):
            raise _err("SimLoop", f"substeps must be an integer >= 1, got {substeps}")
        if not (isinstance(iterations, int) and iterations >= 0):
            raise _err("SimLoop", f"iterations must be a non-negative integer, got {iterations}")
        for m in materials:
            if m.particles is not particles:
                raise _err("SimLoop", "a material belongs to another ParticleSystem")
        self.particles = particles
        self.materials = list(materials)
        self.colliders = list(colliders)
        rec = R.Recipe(capacity=particles.capacity, radius=particles.particle_radius, uploads=list(particles.uploads),
                       loop=R.LoopOpts(substeps=substeps, iterations=iterations, gravity=tuple(gravity),
                                       hash_origin=tuple(hash_origin), grid_min=tuple(grid_min),
                                       grid_max=tuple(grid_max)))
        if contact:
            # SimLoopOptions.contact: true or {muS, muK, maxContacts} (loop.ts:20-30)
            c = contact if isinstance(contact, dict) else {}
            mus, muk = c.get("mu_s", 0.5), c.get("mu_k", 0.4)
            if not (mus >= 0) or not (muk >= 0):
                raise _err("SimLoop", f"friction coefficients must be non-negative (got muS={mus}, muK={muk})")
            mc = c.get("max_contacts", 8 * particles.capacity)
            if not (isinstance(mc, int) and mc > 0):
                raise N.PfError(N.PF_ERR_INVALID, f"ContactBuffer: maxContacts must be a positive integer, got {mc}")
            rec.loop.contact, rec.loop.contact_mu_s, rec.loop.contact_mu_k, rec.loop.max_contacts = True, mus, muk, mc
        for m in self.materials:
            rec.materials.append((m.kind, m.opts))
        for c in self.colliders:
            if isinstance(c, PrimitiveSet):
                rec.prims.extend(c.prims)
            elif isinstance(c, SDFCollider):
                rec.sdfs.append(c.sdf)
            else:
                raise _err("SimLoop", f"unknown collider {type(c).__name__}")
            c.loop = self
        self.recipe = rec
        self.scene = R.NativeBackend().build(rec)
        particles.loop = self
        self.disposed = False

    def prim_base(self, prims: PrimitiveSet) -> int:
        base = 0
        for c in self.colliders:
            if c is prims:
                return base
            if isinstance(c, PrimitiveSet):
                base += len(c.prims)
        raise _err("SimLoop", "collider is not part of this loop")

    def step(self, dt: float) -> None:
        if self.disposed:
            raise N.PfError(N.PF_ERR_STATE, "SimLoop: has been disposed")
        self.scene.step(dt)

    def readback_overflow(self) -> dict:
        return self.scene.overflow()

    def contacts(self) -> tuple[int, np.ndarray]:
        """loop.contacts.readbackCount() and readbackPairs() (ContactBuffer.ts:75-97)."""
        return self.scene.contacts()

    def dispose(self) -> None:
        if not self.disposed:
            self.scene.close()
            self.disposed = True


# -------------------------------------------------------- frame pacing ----
STEP_TOLERANCE = 1e-6  # a millionth of a step still counts as a whole step (frameStepper.ts:2)


class FrameStepper:
    """src/core/frameStepper.ts:35-88: a fixed-timestep accumulator. Each
    pump adds the wall-clock time since the previous pump and takes whole
    steps of `fixed_dt` from it, at most `max_steps_per_frame`; time past
    that cap is dropped (the simulation runs slower than real time instead
    of falling behind). The first pump only starts the clock."""

    def __init__(self, fixed_dt: float, max_steps_per_frame: int = 4):
        if not (isinstance(fixed_dt, (int, float)) and math.isfinite(fixed_dt) and fixed_dt > 0):
            raise _err("FrameStepper", f"fixedDt must be positive, got {fixed_dt}")
        if not (isinstance(max_steps_per_frame, int) and max_steps_per_frame > 0):
            raise _err("FrameStepper", f"maxStepsPerFrame must be a positive integer, got {max_steps_per_frame}")
        self.fixed_dt = float(fixed_dt)
        self.max_steps_per_frame = max_steps_per_frame
        self.accumulator = 0.0
        self.last_ms: float | None = None

    def pump(self, now_ms: float, step) -> dict:
        """Runs step(fixed_dt) as many times as the elapsed time allows;
        returns {steps, truncated, remainder_seconds}."""
        if self.last_ms is None:
            self.last_ms = now_ms
            return {"steps": 0, "truncated": False, "remainder_seconds": 0.0}
        self.accumulator += max(0.0, (now_ms - self.last_ms) / 1000.0)
        self.last_ms = now_ms
        # whole steps counted, not subtracted one by one, so rounding cannot
        # leave a step's worth of time behind
        available = self.accumulator / self.fixed_dt
        truncated = available > self.max_steps_per_frame + STEP_TOLERANCE
        steps = self.max_steps_per_frame if truncated else min(math.floor(available + STEP_TOLERANCE),
                                                               self.max_steps_per_frame)
        self.accumulator = 0.0 if truncated else max(0.0, self.accumulator - steps * self.fixed_dt)
        for _ in range(steps):
            step(self.fixed_dt)
        return {"steps": steps, "truncated": truncated, "remainder_seconds": self.accumulator}

    def reset(self) -> None:
        """Forget elapsed time (after a pause), so the next pump does not catch up."""
        self.accumulator = 0.0
        self.last_ms = None


# ------------------------------------------------------------- façade ----
@dataclass
class _FluidReq:
    box: tuple
    viscosity: float
    vorticity: float
    surface_tension: float
    adhesion: float


@dataclass
class _SoftReq:
    shape: str
    center: tuple
    size: float
    softness: float
    density: float


@dataclass
class _ClothReq:
    width: float
    height: float
    position: tuple
    softness: float
    pin: str
    weight: float
    wind: tuple


class Simulation:
    """The façade (src/simulation/Simulation.ts:62-107, 301-634) for the
    hot-path materials: `container` (lo, hi) with walls and an open top
    (Simulation.ts:779-787), a particle budget or a particle radius, fluids
    filling boxes, soft spheres and boxes, cloth sheets pinned along the top
    edge, and primitive colliders. Built at the first step."""

    def __init__(self, container=None, particles: int | None = None, particle_radius: float | None = None,
                 gravity=(0.0, -9.81, 0.0), substeps: int | None = None, closed: bool = False):
        if (particles is None) == (particle_radius is None):
            raise _err("Simulation", "give exactly one of `particles` or `particleRadius`")
        if particles is not None and not (isinstance(particles, int) and particles > 0):
            raise _err("Simulation", f"particles must be a positive integer, got {particles}")
        if particle_radius is not None and not (particle_radius > 0 and math.isfinite(particle_radius)):
            raise _err("Simulation", f"particleRadius must be a positive number of metres, got {particle_radius}")
        self.container = None if container is None else (tuple(container[0]), tuple(container[1]))
        self.budget = particles
        self.radius = particle_radius
        self.gravity = tuple(gravity)
        self.substeps = substeps
        self.closed = closed
        self.fluids: list[_FluidReq] = []
        self.softs: list[_SoftReq] = []
        self.cloths: list[_ClothReq] = []
        self.prims: list[R.Prim] = []
        self.loop: SimLoop | None = None
        self.particles: ParticleSystem | None = None
        # Simulation.ts:313-318: 60 steps per second of wall clock when
        # step() gets no dt; a pause of over 250 ms restarts the clock
        self.stepper = FrameStepper(1.0 / 60.0)
        self._last_step_ms = -math.inf
        self._clock = lambda: time.perf_counter() * 1000.0
        # Simulation.ts:542-546: a step() while another runs (another thread
        # here) waits for that one and does not step again
        self._step_lock = threading.Lock()
        self._stepping: threading.Event | None = None

    def _not_started(self, what: str):
        if self.loop is not None:
            raise N.PfError(N.PF_ERR_STATE, f"{what}: the simulation has started")

    def add_fluid(self, box, viscosity: float = 0.01, vorticity: float = 0.02, surface_tension: float = 0.1,
                  adhesion: float = 0.1) -> None:
        """Simulation.addFluid (Simulation.ts:342-368) with its defaults:
        viscosity 0.01, surface tension 0.1, vorticity 0.02, adhesion 0.1."""
        self._not_started("addFluid")
        self.fluids.append(_FluidReq((tuple(box[0]), tuple(box[1])), viscosity, vorticity, surface_tension,
                                     adhesion))

    def add_softbody(self, shape: str, center, size: float, softness: float = 0.5, density: float = 1000.0) -> None:
        self._not_started("addSoftbody")
        if shape not in ("sphere", "box"):
            raise _err("addSoftbody", f"shape must be 'sphere' or 'box', got {shape}")
        self.softs.append(_SoftReq(shape, tuple(center), float(size), float(softness), float(density)))

    def add_cloth(self, width: float, height: float, position=(0.0, 0.5, 0.0), softness: float = 0.75,
                  pin: str = "top", weight: float = 0.1, wind=(0.0, 0.0, 0.0)) -> int:
        """Simulation.addCloth (Simulation.ts:416-426) with its defaults:
        softness 0.75, weight 0.1 kg/m^2, no wind. Returns the cloth's index
        for set_cloth_wind."""
        self._not_started("addCloth")
        if pin not in ("top", "none"):
            raise _err("addCloth", f"pin must be 'top' or 'none', got {pin}")
        self.cloths.append(_ClothReq(width, height, tuple(position), softness, pin, float(weight),
                                     tuple(float(w) for w in wind)))
        return len(self.cloths) - 1

    def set_cloth_wind(self, index: int, wind) -> None:
        """Cloth.wind (the façade copies it into its ClothSystem before each
        step, Simulation.ts:632)."""
        c = self.cloths[index]
        c.wind = tuple(float(w) for w in wind)
        if self.loop is not None:
            self._cloth_systems[index].wind = c.wind

    def add_floor(self, y: float = 0.0) -> None:
        self.prims.append(R.plane((0, 1, 0), (0.0, y, 0.0)))

    def add_sphere(self, radius: float, center) -> None:
        self.prims.append(R.sphere(center, radius))

    def add_box(self, center, half) -> None:
        self.prims.append(R.box(center, half))

    def add_capsule(self, a, b, radius: float) -> None:
        self.prims.append(R.capsule(a, b, radius))

    # layout: one particle size for everything (Simulation.ts:640-700)
    def _volumes(self):
        v = [float(np.prod(np.subtract(f.box[1], f.box[0]))) for f in self.fluids]
        v += [(4.0 / 3.0) * math.pi * (s.size ** 3) if s.shape == "sphere" else (2 * s.size) ** 3 for s in self.softs]
        return v

    def _radius(self) -> float:
        if self.radius is not None:
            return self.radius
        vol = sum(self._volumes())
        area = sum(c.width * c.height for c in self.cloths)
        # particles = vol / (2r)^3 + area / (2r)^2, solved for r by bisection
        lo, hi = 1e-5, 1.0
        for _ in range(80):
            r = 0.5 * (lo + hi)
            n = vol / (2 * r) ** 3 + area / (2 * r) ** 2
            lo, hi = (r, hi) if n > self.budget else (lo, r)
        return hi

    def _build(self) -> None:
        from . import shapes
        from . import workloads as W

        r = self._radius()
        s = 2.0 * r
        chunks, mats = [], []
        n = 0
        h = 2.0 * s
        for f in self.fluids:
            pts = W.fill_box(np.array(f.box[0]), np.array(f.box[1]), s)
            mass = 1000.0 * s ** 3
            rho0 = W.lattice_rest_density(s, h, mass)
            chunks.append((n, pts))
            mats.append(("fluid", R.FluidOpts(range=(n, len(pts)), rest_density=rho0,
                                              particle_spacing=(mass / rho0) ** (1 / 3), smoothing_radius=h,
                                              compliance=1e-4, viscosity=f.viscosity,
                                              vorticity=f.vorticity or None,
                                              surface_tension=f.surface_tension or None,
                                              adhesion=f.adhesion or None)))
            n += len(pts)
        bodies = []
        for b in self.softs:
            if b.shape == "sphere":
                vox = shapes.voxel_sphere(b.center, b.size, r, neighborhood=26)
            else:
                vox = shapes.voxel_box(b.center, (b.size, b.size, b.size), r, neighborhood=26)
            chunks.append((n, vox.positions))
            m = b.density * s ** 3
            bodies.append(R.BodyDef(range=(n, vox.count), surface_count=vox.surface_count,
                                    compliance=W.softbody_compliance(b.softness, vox.count), edges=vox.edges))
            chunks[-1] = (n, vox.positions, np.full(vox.count, 1.0 / m, np.float32))
            n += vox.count
        if bodies:
            mats.append(("soft", R.SoftbodyOpts(bodies, "local")))
        for c in self.cloths:
            seg_w = max(1, int(round(c.width / s)))
            seg_h = max(1, int(round(c.height / s)))
            pos, idx = shapes.plane_geometry(c.width, c.height, seg_w, seg_h)
            pos = pos + np.asarray(c.position)
            pinned = range(seg_w + 1) if c.pin == "top" else ()
            g = shapes.create_cloth_graph(pos, idx, c.weight, pinned=pinned)
            # Simulation.ts:703-718, handles.ts:298-300
            bend = 10 ** (-1 + c.softness * 5) * (seg_w / 30) ** 4 * (0.35 / c.weight)
            mats.append(("cloth", (g, n, dict(bend_compliance=bend, stretch_tolerance=0.06, wind=c.wind,
                                              drag=0.18, lift=0.02, damping=0.1))))
            n += len(pos)
        if n == 0:
            raise N.PfError(N.PF_ERR_STATE, "Simulation: nothing to simulate; add a fluid, soft body or cloth")
        # Simulation.ts:722-737: every fluid treats the soft bodies' surfaces
        # and the cloths as dynamic boundaries
        solids = [(b.range[0], b.surface_count) for b in bodies]
        solids += [(opts[1], len(opts[0].positions)) for kind, opts in mats if kind == "cloth"]
        for kind, opts in mats:
            if kind == "fluid":
                opts.boundaries = list(solids)
                opts.boundary_static = [False] * len(solids)
        ps = ParticleSystem(n, r)
        for ch in chunks:
            start, pts = ch[0], ch[1]
            w = ch[2] if len(ch) > 2 else None
            ps.uploads.append(R.Upload(start, np.asarray(pts, np.float32), None, w))
        prims = list(self.prims)
        if self.container is not None:
            prims += R.container_walls(self.container[0], self.container[1], self.closed)
        # Simulation.ts:820-836: substeps from the stiffest material at this
        # particle size; contacts when soft bodies or cloth are present
        base = max(4 if self.fluids else 0, 6 if bodies else 0, 8 if self.cloths else 0)
        substeps = self.substeps or min(24, math.ceil(base * max(1.0, 0.018 / r)))
        rec_loop = dict(substeps=int(substeps), iterations=2, gravity=self.gravity)
        if bodies or self.cloths:
            rec_loop["contact"] = {"mu_s": 0.3, "mu_k": 0.2}
        # the neighbour grid window: the container (open top: twice as
        # high) plus two smoothing radii, so the fluid never outgrows it
        grid = {}
        if self.container is not None:
            lo, hi = np.asarray(self.container[0], float), np.asarray(self.container[1], float)
            pad = 2.0 * 2.0 * s
            top = hi.copy()
            if not self.closed:
                top[1] += hi[1] - lo[1]
            grid = dict(grid_min=tuple(lo - pad), grid_max=tuple(top + pad))
        self.particles = ps
        matobjs = []
        self._cloth_systems = []
        for kind, opts in mats:
            if kind == "cloth":
                g, off, kw = opts
                o = ClothSystem(ps, g, offset=off, **kw)
                self._cloth_systems.append(o)
            else:
                o = object.__new__({"fluid": FluidSystem, "soft": SoftbodySystem}[kind])
                o.particles, o.opts = ps, opts
            matobjs.append(o)
        pset = PrimitiveSet(ps)
        pset.prims = prims
        self.loop = SimLoop(ps, materials=matobjs, colliders=[pset] if prims else [], **rec_loop, **grid)

    def start(self) -> None:
        """Simulation.start (Simulation.ts:549-560): build now instead of at
        the first step."""
        if self.loop is None:
            self._build()

    def step(self, dt: float | None = None) -> None:
        """Simulation.step (Simulation.ts:542-584). With dt, advance by dt;
        without it, keep pace with the wall clock at 60 fixed steps per
        second (at most 4 per call; a pause of over 250 ms starts the clock
        again instead of catching up). A call made while another thread's
        step runs waits for that step and returns: it covers this frame."""
        with self._step_lock:
            running = self._stepping
            if running is None:
                self._stepping = threading.Event()
        if running is not None:
            running.wait()
            return
        try:
            self.start()
            if dt is None:
                now = self._clock()
                if now - self._last_step_ms > 250.0:
                    self.stepper.reset()
                self._last_step_ms = now
                self.stepper.pump(now, self._advance)
            else:
                self._advance(dt)
        finally:
            with self._step_lock:
                self._stepping.set()
                self._stepping = None

    def _advance(self, dt: float) -> None:
        """Simulation.advance (Simulation.ts:611-634): the cloths take their
        current wind, then the loop steps."""
        for c, system in zip(self.cloths, self._cloth_systems):
            if system.wind != c.wind:
                system.wind = c.wind
        self.loop.step(dt)

    def readback(self) -> Snapshot:
        if self.particles is None:
            raise N.PfError(N.PF_ERR_STATE, "Simulation: step before reading back")
        return self.particles.readback()

    def dispose(self) -> None:
        if self.loop is not None:
            self.loop.dispose()


def trim_device_memory() -> None:
    """Hand back the device memory the library keeps from destroyed
    simulations (pf_trim_device_memory). No reference counterpart."""
    N.check(N.lib().pf_trim_device_memory())
