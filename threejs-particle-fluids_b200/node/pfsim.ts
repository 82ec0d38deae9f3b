/**
 * pfsim.ts — the reference's solver classes on top of libpfsim.so.
 *
 * A drop-in for the hot path of threejs-particle-fluids: ParticleSystem,
 * FluidSystem, SoftbodySystem, ClothSystem, PrimitiveSet, SDFCollider,
 * SimLoop, FrameStepper and a Simulation facade with the reference's names,
 * option objects, defaults, constructor checks and error texts
 * (src/core/particles.ts, src/fluids/FluidSystem.ts, src/softbody/
 * SoftbodySystem.ts, src/cloth/ClothSystem.ts, src/core/collision/*.ts,
 * src/core/loop.ts, src/core/frameStepper.ts, src/simulation/Simulation.ts).
 * Instead of TSL compute nodes, each class records its options and SimLoop
 * hands them to the native addon (pfsim_napi.c) in material order, then
 * steps the scene on the GPU through it. Rendering stays with the caller:
 * readback() returns the positions and velocities a renderer draws.
 *
 * Not built or run on the machine this repository was developed on: it has
 * no Node.js or TypeScript. The Python mirror (pfsim/api.py) implements the
 * same classes over the same C entry points and is what the tests exercise.
 */

// eslint-disable-next-line @typescript-eslint/no-require-imports
const addon = require('./build/Release/pfsim_napi.node');

export type Vec3 = readonly [number, number, number];
export interface ParticleRange {
  readonly start: number;
  readonly count: number;
}

/** Field ids of pf_readback / pf_write (include/pfsim.h pf_field). */
export const Field = {
  positions: 0,
  predicted: 1,
  velocities: 2,
  invMass: 3,
  boundaryVolume: 4,
  density: 5,
  rotation: 6,
  predictedRotation: 7,
  angularVelocity: 8,
  lambda: 9,
  neighborCount: 10,
  neighbors: 11,
  cellPerm: 12,
} as const;

function fail(cls: string, reason: string): never {
  throw new Error(`${cls}: ${reason}`);
}
function nonNegative(value: number, name: string, cls = 'ClothSystem'): void {
  if (!Number.isFinite(value) || value < 0) fail(cls, `${name} must be a non-negative number, got ${value}`);
}
function assertRange(particles: ParticleSystem, range: ParticleRange, cls: string): void {
  const { start, count } = range;
  if (!Number.isInteger(start) || !Number.isInteger(count) || start < 0 || count < 0 ||
      start + count > particles.capacity) {
    fail(cls, `invalid particle range [${start}, ${start + count}) for capacity ${particles.capacity}`);
  }
}

// ----------------------------------------------------------- particles ---

export interface ParticleInit {
  readonly position: Vec3;
  readonly velocity?: Vec3;
  readonly invMass?: number;
  readonly collisionGroup?: number;
}

/** src/core/particles.ts:52-316: the particle state, owned by a native scene. */
export class ParticleSystem {
  readonly capacity: number;
  readonly particleRadius: number;
  /** The native scene (pf_scene); created here, built into a loop by SimLoop. */
  readonly scene: unknown;
  loop: SimLoop | undefined;
  private disposed = false;

  constructor(capacity: number, particleRadius: number) {
    if (!Number.isInteger(capacity) || capacity <= 0) {
      fail('ParticleSystem', `capacity must be a positive integer, got ${capacity}`);
    }
    if (!Number.isFinite(particleRadius) || particleRadius <= 0) {
      fail('ParticleSystem', `particleRadius must be a positive number, got ${particleRadius}`);
    }
    this.capacity = capacity;
    this.particleRadius = particleRadius;
    this.scene = addon.createScene(capacity, particleRadius);
  }

  /** particles.ts:131-190: write particles starting at slot `start`. */
  uploadParticles(init: readonly ParticleInit[], start = 0): void {
    this.assertLive();
    if (!Number.isInteger(start) || start < 0 || start + init.length > this.capacity) {
      fail('ParticleSystem.uploadParticles', 'invalid particle range');
    }
    const n = init.length;
    const pos = new Float32Array(4 * n);
    const vel = new Float32Array(4 * n);
    const w = new Float32Array(n);
    const g = new Uint32Array(n);
    init.forEach((p, i) => {
      const invMass = p.invMass ?? 1;
      if (!Number.isFinite(invMass) || invMass < 0) fail('ParticleSystem.uploadParticles', `invMass ${invMass}`);
      const group = p.collisionGroup ?? 0;
      if (!Number.isInteger(group) || group < 0 || group >= 2 ** 32) {
        fail('ParticleSystem.uploadParticles', `collisionGroup ${group}`);
      }
      pos.set([p.position[0], p.position[1], p.position[2], 0], 4 * i);
      if (p.velocity) vel.set([p.velocity[0], p.velocity[1], p.velocity[2], 0], 4 * i);
      w[i] = invMass;
      g[i] = group;
    });
    addon.uploadParticles(this.scene, pos, vel, w, g, start);
  }

  /** particles.ts:163-173. */
  setInvMass(range: ParticleRange, invMass: number): void {
    this.assertLive();
    if (!Number.isFinite(invMass) || invMass < 0) fail('ParticleSystem.setInvMass', `invMass must be >= 0, got ${invMass}`);
    assertRange(this, range, 'ParticleSystem.setInvMass');
    addon.setInvMass(this.scene, range.start, range.count, invMass);
  }

  /** particles.ts:192-227: positions and velocities, xyzw per particle. */
  async readback(): Promise<{ positions: Float32Array; velocities: Float32Array }> {
    this.assertLive();
    await this.loop?.pending;
    const positions = new Float32Array(4 * this.capacity);
    const velocities = new Float32Array(4 * this.capacity);
    addon.readback(this.scene, Field.positions, positions);
    addon.readback(this.scene, Field.velocities, velocities);
    return { positions, velocities };
  }

  /** Any other field of include/pfsim.h (density, lambda, neighbour lists ...). */
  async readField(field: number, out: Float32Array | Uint32Array): Promise<void> {
    this.assertLive();
    await this.loop?.pending;
    addon.readback(this.scene, field, out);
  }

  /** Whole-field write in particle order (a caller setting a buffer and flagging needsUpdate). */
  async writeField(field: number, data: Float32Array): Promise<void> {
    this.assertLive();
    await this.loop?.pending;
    addon.write(this.scene, field, data);
  }

  dispose(): void {
    if (this.disposed) return;
    this.disposed = true;
    addon.destroyScene(this.scene);
  }

  assertLive(): void {
    if (this.disposed) fail('ParticleSystem', 'has been disposed');
  }
}

// ----------------------------------------------------------- materials ---

/** A material of SimLoop: adds itself to the native scene in loop order. */
export interface Material {
  readonly particles: ParticleSystem;
  /** Called by SimLoop's constructor, in materials order. */
  attach(scene: unknown): number;
}

export interface FluidBoundary {
  readonly range: ParticleRange;
  readonly dynamic?: boolean;
}
export interface FluidSystemOptions {
  readonly range?: ParticleRange;
  readonly restDensity?: number;
  readonly particleSpacing?: number;
  readonly smoothingRadius?: number;
  readonly compliance?: number;
  readonly viscosity?: number;
  readonly vorticity?: number;
  readonly surfaceTension?: number;
  readonly adhesion?: number;
}

/** src/fluids/FluidSystem.ts:31-255: PBF fluid with its optional effects. */
export class FluidSystem implements Material {
  readonly particles: ParticleSystem;
  readonly options: FluidSystemOptions;
  private readonly boundaries: FluidBoundary[] = [];

  constructor(particles: ParticleSystem, options: FluidSystemOptions = {}) {
    const range = options.range ?? { start: 0, count: particles.capacity };
    assertRange(particles, range, 'FluidSystem');
    for (const key of ['restDensity', 'particleSpacing', 'smoothingRadius'] as const) {
      const v = options[key];
      if (v !== undefined && (!Number.isFinite(v) || v <= 0)) fail('FluidSystem', `${key} must be positive, got ${v}`);
    }
    for (const key of ['compliance', 'viscosity', 'vorticity', 'surfaceTension', 'adhesion'] as const) {
      const v = options[key];
      if (v !== undefined) nonNegative(v, key, 'FluidSystem');
    }
    this.particles = particles;
    this.options = { ...options, range };
  }

  /** FluidSystem.addBoundary (FluidSystem.ts:171-183): before the loop is built. */
  addBoundary(range: ParticleRange, options: { dynamic?: boolean } = {}): void {
    assertRange(this.particles, range, 'FluidSystem.addBoundary');
    this.boundaries.push({ range, dynamic: options.dynamic ?? true });
  }

  attach(scene: unknown): number {
    const o = this.options;
    return addon.addFluid(scene, {
      start: o.range!.start, count: o.range!.count, restDensity: o.restDensity, particleSpacing: o.particleSpacing,
      smoothingRadius: o.smoothingRadius, compliance: o.compliance, viscosity: o.viscosity,
      vorticity: o.vorticity, surfaceTension: o.surfaceTension, adhesion: o.adhesion,
      boundaries: this.boundaries.map((b) => ({ start: b.range.start, count: b.range.count, dynamic: b.dynamic })),
    });
  }
}

export interface SoftbodyDef {
  readonly range: ParticleRange;
  readonly surfaceCount?: number;
  readonly compliance?: number;
  readonly restPositions?: Float32Array;
  readonly edges?: Uint32Array;
}
export interface SoftbodySystemOptions {
  readonly bodies: readonly SoftbodyDef[];
  readonly shapeMatching?: 'global' | 'local';
  readonly selfCollision?: boolean;
}

/** src/softbody/SoftbodySystem.ts:29-234: shape matching over bodies or clusters. */
export class SoftbodySystem implements Material {
  readonly particles: ParticleSystem;
  readonly options: SoftbodySystemOptions;

  constructor(particles: ParticleSystem, options: SoftbodySystemOptions) {
    if (!options.bodies?.length) fail('SoftbodySystem', 'needs at least one body');
    for (const b of options.bodies) {
      assertRange(particles, b.range, 'SoftbodySystem');
      if (b.compliance !== undefined) nonNegative(b.compliance, 'compliance', 'SoftbodySystem');
    }
    this.particles = particles;
    this.options = options;
  }

  attach(scene: unknown): number {
    return addon.addSoftbodies(scene, {
      bodies: this.options.bodies.map((b) => ({
        start: b.range.start, count: b.range.count, surfaceCount: b.surfaceCount, compliance: b.compliance ?? 0,
        restPositions: b.restPositions, edges: b.edges,
      })),
      shapeMatching: this.options.shapeMatching ?? 'global',
      selfCollision: this.options.selfCollision ?? false,
    });
  }
}

/** The arrays of createClothGraph (src/cloth/graph.ts:130-342). */
export interface ClothGraph {
  readonly positions: readonly Vec3[];
  readonly invMass: readonly number[];
  readonly distancePairs: Uint32Array;
  readonly distanceRestLengths: readonly number[];
  readonly bendingTuples?: Uint32Array;
  readonly bendingRestAngles?: readonly number[];
  readonly triangles?: Uint32Array;
}
export interface ClothSystemOptions {
  readonly graph: ClothGraph;
  readonly offset?: number;
  readonly stretchCompliance?: number;
  readonly bendCompliance?: number;
  readonly tetherCompliance?: number;
  readonly stretchTolerance?: number;
  readonly wind?: Vec3;
  readonly drag?: number;
  readonly lift?: number;
  readonly damping?: number;
}

/** src/cloth/ClothSystem.ts:37-287: stretch, bending, tethers, drag and lift, smoothing. */
export class ClothSystem implements Material {
  readonly particles: ParticleSystem;
  readonly range: ParticleRange;
  readonly tethers: { particle: Uint32Array; anchor: Uint32Array; rest: Float32Array };
  private readonly options: ClothSystemOptions;
  private scene: unknown;
  private material = -1;
  private params: { wind: Vec3; drag: number; lift: number; damping: number; bendCompliance: number };

  constructor(particles: ParticleSystem, options: ClothSystemOptions) {
    const { graph } = options;
    this.range = { start: options.offset ?? 0, count: graph.positions.length };
    assertRange(particles, this.range, 'ClothSystem');
    for (const key of ['stretchCompliance', 'bendCompliance', 'tetherCompliance', 'stretchTolerance', 'drag',
                       'lift'] as const) {
      const v = options[key];
      if (v !== undefined) nonNegative(v, key);
    }
    if (options.damping !== undefined && !(options.damping >= 0 && options.damping <= 1)) {
      fail('ClothSystem', `damping must be in [0, 1], got ${options.damping}`);
    }
    this.particles = particles;
    this.options = options;
    this.params = { wind: options.wind ?? [0, 0, 0], drag: options.drag ?? 0.6125, lift: options.lift ?? 0.3,
                    damping: options.damping ?? 0, bendCompliance: options.bendCompliance ?? 1e-5 };
    // ClothSystem.ts:125-128: tethers from the pins
    this.tethers = addon.buildTethers({
      invMass: Float32Array.from(graph.invMass), pairs: graph.distancePairs,
      restLengths: Float64Array.from(graph.distanceRestLengths), maxAttachments: 4,
      stretchTolerance: options.stretchTolerance ?? 0,
    });
  }

  attach(scene: unknown): number {
    const { graph, options: o } = { graph: this.options.graph, options: this.options };
    const hasTethers = this.tethers.particle.length > 0;
    this.scene = scene;
    this.material = addon.addCloth(scene, {
      offset: this.range.start,
      positions: Float32Array.from(graph.positions.flat()),
      invMass: Float32Array.from(graph.invMass),
      pairs: graph.distancePairs,
      restLengths: Float32Array.from(graph.distanceRestLengths),
      stretchCompliance: o.stretchCompliance,
      bending: graph.bendingTuples,
      bendingRest: graph.bendingRestAngles ? Float32Array.from(graph.bendingRestAngles) : undefined,
      bendCompliance: this.params.bendCompliance,
      tetherParticle: hasTethers ? this.tethers.particle : undefined,
      tetherAnchor: hasTethers ? this.tethers.anchor : undefined,
      tetherRest: hasTethers ? this.tethers.rest : undefined,
      tetherCompliance: o.tetherCompliance,
      triangles: graph.triangles,
      wind: this.params.wind, drag: this.params.drag, lift: this.params.lift,
      damping: o.damping,
    });
    return this.material;
  }

  /** ClothSystem.ts:143-188 setters: take effect at the next step. */
  get wind(): Vec3 { return this.params.wind; }
  set wind(v: Vec3) { this.params.wind = v; this.push(); }
  get drag(): number { return this.params.drag; }
  set drag(v: number) { nonNegative(v, 'drag'); this.params.drag = v; this.push(); }
  get lift(): number { return this.params.lift; }
  set lift(v: number) { nonNegative(v, 'lift'); this.params.lift = v; this.push(); }
  get damping(): number { return this.params.damping; }
  set damping(v: number) {
    if (this.options.damping === undefined) fail('ClothSystem', 'damping was not enabled at construction');
    if (!(v >= 0 && v <= 1)) fail('ClothSystem', `damping must be in [0, 1], got ${v}`);
    this.params.damping = v;
    this.push();
  }
  get bendCompliance(): number { return this.params.bendCompliance; }
  set bendCompliance(v: number) { nonNegative(v, 'bendCompliance'); this.params.bendCompliance = v; this.push(); }

  private push(): void {
    if (this.material >= 0) addon.clothSetParams(this.scene, this.material, this.params);
  }
}

// ----------------------------------------------------------- colliders ---

export interface PrimitiveRecord {
  readonly kind: 'plane' | 'sphere' | 'box' | 'capsule';
  readonly invert?: boolean;
  readonly sweep?: boolean;
  readonly data0?: readonly number[];
  readonly data1?: readonly number[];
  readonly velocity?: readonly number[];
  readonly rotation?: readonly number[];
  readonly spin?: readonly number[];
}
export interface Collider {
  attach(scene: unknown): void;
}

/** src/core/collision/PrimitiveSet.ts:166-257 (records of primitives.ts:125-186). */
export class PrimitiveSet implements Collider {
  private readonly prims: PrimitiveRecord[] = [];
  private scene: unknown;
  private base = 0;

  addPlane(normal: Vec3, point: Vec3, muS = 0.5, muK = 0.3): number {
    return this.add({ kind: 'plane', data0: [...normal, 0], data1: [...point, muS], velocity: [0, 0, 0, muK] });
  }
  addSphere(center: Vec3, radius: number, muS = 0.5, muK = 0.3, invert = false): number {
    return this.add({ kind: 'sphere', invert, data0: [...center, radius], data1: [0, 0, 0, muS], velocity: [0, 0, 0, muK] });
  }
  addBox(center: Vec3, half: Vec3, rotation: readonly number[] = [0, 0, 0, 1], invert = false, muS = 0.5, muK = 0.3): number {
    return this.add({ kind: 'box', invert, data0: [...center, 0], data1: [...half, muS], velocity: [0, 0, 0, muK], rotation });
  }
  addCapsule(a: Vec3, b: Vec3, radius: number, muS = 0.5, muK = 0.3): number {
    return this.add({ kind: 'capsule', data0: [...a, radius], data1: [...b, muS], velocity: [0, 0, 0, muK] });
  }
  /** PrimitiveSet.setSphere: a moving sphere sweeps its path within a step. */
  setSphere(slot: number, center: Vec3, radius: number, velocity: Vec3 = [0, 0, 0]): void {
    const p = this.prims[slot];
    if (!p || p.kind !== 'sphere') fail('PrimitiveSet', `slot ${slot} is not a sphere`);
    const next: PrimitiveRecord = { ...p, sweep: true, data0: [...center, radius],
                                    velocity: [...velocity, p.velocity?.[3] ?? 0.3] };
    this.prims[slot] = next;
    if (this.scene !== undefined) addon.setPrimitive(this.scene, this.base + slot, next);
  }
  attach(scene: unknown): void {
    this.scene = scene;
    this.prims.forEach((p, i) => {
      const slot = addon.addPrimitive(scene, p);
      if (i === 0) this.base = slot;
    });
  }
  private add(p: PrimitiveRecord): number {
    if (this.scene !== undefined) fail('PrimitiveSet', 'primitives must be added before the SimLoop is built');
    this.prims.push(p);
    return this.prims.length - 1;
  }
}

export interface SDFColliderOptions {
  readonly muS?: number;
  readonly muK?: number;
  readonly thickness?: number;
  readonly position?: Vec3;
  readonly rotation?: readonly [number, number, number, number];
  readonly scale?: number;
}

/** src/core/collision/SDFCollider.ts:68-317 over a baked distance grid. */
export class SDFCollider implements Collider {
  private scene: unknown;
  private slot = -1;

  constructor(
    readonly sdf: { res: Vec3; data: Float32Array; origin: Vec3; voxelSize: Vec3 },
    readonly options: SDFColliderOptions = {},
  ) {
    for (const key of ['muS', 'muK', 'thickness'] as const) {
      const v = options[key];
      if (v !== undefined) nonNegative(v, key, 'SDFCollider');
    }
  }
  attach(scene: unknown): void {
    this.scene = scene;
    const o = this.options;
    this.slot = addon.addSdfCollider(scene, { ...this.sdf, position: o.position ?? [0, 0, 0],
      rotation: o.rotation ?? [0, 0, 0, 1], scale: o.scale ?? 1, thickness: o.thickness ?? 0,
      muS: o.muS ?? 0.5, muK: o.muK ?? 0.3 });
  }
  /** SDFCollider.setPosition / setRotation / setScale in one call. */
  setTransform(position: Vec3, rotation: readonly [number, number, number, number], scale: number): void {
    if (this.slot < 0) fail('SDFCollider', 'not attached to a SimLoop yet');
    addon.setSdfTransform(this.scene, this.slot, position, rotation, scale);
  }
}

// ---------------------------------------------------------------- loop ---

export interface ContactOptions {
  readonly muS?: number;
  readonly muK?: number;
  readonly maxContacts?: number;
}
export interface SimLoopOptions {
  readonly substeps?: number;
  readonly iterations?: number;
  readonly gravity?: Vec3;
  readonly materials?: readonly Material[];
  readonly colliders?: readonly Collider[];
  readonly contact?: boolean | ContactOptions;
  readonly hashOrigin?: Vec3;
  /** Size and first placement of the neighbour grid window (no reference counterpart; see pfsim.h). */
  readonly gridMin?: Vec3;
  readonly gridMax?: Vec3;
}
export interface SimLoopOverflow {
  readonly positions: boolean;
  readonly velocities: boolean;
  readonly grid: boolean;
  readonly contacts: boolean;
  readonly neighbors: boolean;
  readonly deviceError: boolean;
  readonly gridClamped: boolean;
}

/** src/core/loop.ts:92-417: the substep pipeline, run by the native scene. */
export class SimLoop {
  readonly particles: ParticleSystem;
  /** The step in flight; readbacks wait for it. */
  pending: Promise<void> | undefined;
  private disposed = false;

  constructor(particles: ParticleSystem, options: SimLoopOptions = {}) {
    const substeps = options.substeps ?? 4;
    const iterations = options.iterations ?? 2;
    if (!Number.isInteger(substeps) || substeps < 1) fail('SimLoop', `substeps must be an integer >= 1, got ${substeps}`);
    if (!Number.isInteger(iterations) || iterations < 0) {
      fail('SimLoop', `iterations must be a non-negative integer, got ${iterations}`);
    }
    for (const m of options.materials ?? []) {
      if (m.particles !== particles) fail('SimLoop', 'a material belongs to another ParticleSystem');
    }
    particles.assertLive();
    this.particles = particles;
    for (const m of options.materials ?? []) m.attach(particles.scene);
    for (const c of options.colliders ?? []) c.attach(particles.scene);
    const contact = options.contact;
    addon.buildLoop(particles.scene, {
      substeps, iterations, gravity: options.gravity ?? [0, -9.81, 0], hashOrigin: options.hashOrigin ?? [0, 0, 0],
      gridMin: options.gridMin, gridMax: options.gridMax,
      contact: contact === true ? {} : contact || undefined,
    });
    particles.loop = this;
  }

  /** loop.ts:267-279: one frame of `substeps` substeps, on the GPU. */
  step(dt: number): Promise<void> {
    if (this.disposed) return Promise.reject(new Error('SimLoop: has been disposed'));
    if (!(dt > 0) || !Number.isFinite(dt)) {
      return Promise.reject(new Error(`SimLoop: step dt must be a positive finite number, got ${dt}`));
    }
    const run = (this.pending ?? Promise.resolve()).then(() => addon.step(this.particles.scene, dt));
    this.pending = run.finally(() => {
      if (this.pending === guarded) this.pending = undefined;
    });
    const guarded = this.pending;
    return run;
  }

  /** loop.ts:286-295. */
  async readbackOverflow(): Promise<SimLoopOverflow> {
    await this.pending;
    return addon.readbackOverflow(this.particles.scene);
  }

  /** loop.contacts.readbackCount() / readbackPairs() (ContactBuffer.ts:75-97). */
  async contacts(capacity: number): Promise<{ count: number; pairs: Uint32Array }> {
    await this.pending;
    return addon.contacts(this.particles.scene, capacity);
  }

  dispose(): void {
    this.disposed = true;
  }
}

// ---------------------------------------------------------- frame pacing ---

const STEP_TOLERANCE = 1e-6;

/** src/core/frameStepper.ts:35-88: fixed steps at wall-clock speed. */
export class FrameStepper {
  readonly fixedDt: number;
  readonly maxStepsPerFrame: number;
  private accumulator = 0;
  private lastMs: number | null = null;

  constructor(options: { fixedDt: number; maxStepsPerFrame?: number }) {
    if (!Number.isFinite(options.fixedDt) || options.fixedDt <= 0) {
      fail('FrameStepper', `fixedDt must be positive, got ${options.fixedDt}`);
    }
    const cap = options.maxStepsPerFrame ?? 4;
    if (!Number.isInteger(cap) || cap <= 0) fail('FrameStepper', `maxStepsPerFrame must be a positive integer, got ${cap}`);
    this.fixedDt = options.fixedDt;
    this.maxStepsPerFrame = cap;
  }

  async pump(nowMs: number, step: (dt: number) => Promise<void>):
      Promise<{ steps: number; truncated: boolean; remainderSeconds: number }> {
    if (this.lastMs === null) {
      this.lastMs = nowMs;
      return { steps: 0, truncated: false, remainderSeconds: 0 };
    }
    this.accumulator += Math.max(0, (nowMs - this.lastMs) / 1000);
    this.lastMs = nowMs;
    const available = this.accumulator / this.fixedDt;
    const truncated = available > this.maxStepsPerFrame + STEP_TOLERANCE;
    const steps = truncated ? this.maxStepsPerFrame
                            : Math.min(Math.floor(available + STEP_TOLERANCE), this.maxStepsPerFrame);
    this.accumulator = truncated ? 0 : Math.max(0, this.accumulator - steps * this.fixedDt);
    for (let i = 0; i < steps; i++) await step(this.fixedDt);
    return { steps, truncated, remainderSeconds: this.accumulator };
  }

  reset(): void {
    this.accumulator = 0;
    this.lastMs = null;
  }
}

// --------------------------------------------------------------- facade ---

/**
 * The part of src/simulation/Simulation.ts the hot path needs: a built
 * SimLoop stepped by `step(dt?)`. Without dt it keeps pace with the clock
 * at 60 steps per second (at most 4 per call, the clock restarted after a
 * pause of over 250 ms); a call while a step runs returns that step's
 * promise (Simulation.ts:542-584). Scene construction (addFluid,
 * addSoftbody, addCloth, colliders) is the caller's: build the materials
 * with the classes above and hand them to `start`.
 */
export class Simulation {
  private readonly stepper = new FrameStepper({ fixedDt: 1 / 60 });
  private lastStepMs = -Infinity;
  private stepping: Promise<void> | undefined;
  private loop: SimLoop | undefined;

  constructor(private readonly build: () => SimLoop) {}

  start(): void {
    this.loop ??= this.build();
  }

  step(dt?: number): Promise<void> {
    this.stepping ??= this.runStep(dt).finally(() => (this.stepping = undefined));
    return this.stepping;
  }

  private async runStep(dt: number | undefined): Promise<void> {
    this.start();
    const loop = this.loop!;
    if (dt === undefined) {
      const now = performance.now();
      if (now - this.lastStepMs > 250) this.stepper.reset();
      this.lastStepMs = now;
      await this.stepper.pump(now, (fixed) => loop.step(fixed));
    } else {
      await loop.step(dt);
    }
  }

  dispose(): void {
    this.loop?.dispose();
    this.loop?.particles.dispose();
  }
}

/**
 * Hands back the device memory the library keeps from destroyed simulations
 * (pf_trim_device_memory). No reference counterpart: the reference's buffers
 * belong to the WebGPU device.
 */
export function trimDeviceMemory(): void {
  addon.trimDeviceMemory();
}
