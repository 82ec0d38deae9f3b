/*
 * pfsim.h — C ABI of the B200 particle solver (libpfsim.so).
 *
 * The library replaces the WebGPU compute path of threejs-particle-fluids for
 * one hot path: the neighbour-grid counting sort (src/core/hashGrid/) and the
 * XPBD solver substep that uses it (src/core/loop.ts with the fluid, soft-body,
 * cloth and collider materials). Every entry point below names the reference
 * interface it stands in for. The signatures use plain C types, pointers and
 * sizes only, so a Node N-API shim, Python ctypes or a C++ host can bind them.
 *
 * Conventions
 *  - Every call returns pf_status. On failure pf_last_error() returns a
 *    thread-local message prefixed like the reference's errors
 *    ("<Class>: <reason>", e.g. src/core/loop.ts:270-272).
 *  - Handles own their device memory; pf_*_destroy frees it, and any later use
 *    of a destroyed handle is the caller's bug (the reference throws
 *    "... has been disposed", src/core/particles.ts:255-257).
 *  - Pointers documented as "host" are ordinary CPU memory copied in or out;
 *    pointers documented as "device" are CUDA device pointers.
 *  - Calls on one handle are not re-entrant (the reference's step() is
 *    serialised by its promise, src/simulation/Simulation.ts:542-546).
 *  - Vectors are xyzw float4 (16 bytes), as the reference's vec4 buffers.
 */
#ifndef PFSIM_H
#define PFSIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PFSIM_ABI_VERSION 3

#if defined(__GNUC__)
#define PF_API __attribute__((visibility("default")))
#else
#define PF_API
#endif

typedef enum pf_status {
  PF_OK = 0,
  PF_ERR_INVALID = 1,   /* bad argument (the reference throws Error) */
  PF_ERR_CUDA = 2,      /* a CUDA runtime call failed */
  PF_ERR_STATE = 3,     /* call out of order (e.g. step before loop build) */
  PF_ERR_OOM = 4,       /* device allocation failed */
  PF_ERR_DEVICE = 5,    /* a kernel reported an error status (bounded wait expired) */
  PF_ERR_BUDGET = 6     /* serving admission refused: HBM budget exhausted */
} pf_status;

/* Thread-local text of the last error on this thread ("" when none). */
PF_API const char* pf_last_error(void);
/* PFSIM_ABI_VERSION of the loaded library. */
PF_API int pf_abi_version(void);
/* Worlds (SimLoops, batches, server cohorts) take their device memory from
 * a pool of the current device that keeps what destroyed worlds and grown
 * grids free, for the next world of the process. This waits for the device
 * and hands the pool's unused memory back (for other allocators of the
 * process, or other processes). No reference counterpart. */
PF_API pf_status pf_trim_device_memory(void);

/* ------------------------------------------------------------------------ */
/* Neighbour grid: standalone stable counting sort                          */
/* ------------------------------------------------------------------------ */

typedef enum pf_key_kind {
  /* cell = clamp(floor((x - origin) / cell_size), 0, dims-1) per axis,
   * key = ix + dims[0] * (iy + dims[1] * iz). */
  PF_KEY_LINEAR = 0,
  /* The reference bucket: Morton(cell + 512) & (table_size - 1) with the
   * cell coordinate clamped to [-2^30, 2^30-1]
   * (src/core/hashGrid/cellIndex.ts:113-170, mortonHash.ts:39-79). */
  PF_KEY_MORTON = 1
} pf_key_kind;

typedef struct pf_grid_desc {
  uint32_t key_kind;   /* pf_key_kind */
  float origin[3];     /* HashGridOptions.hashOrigin (HashGrid.ts:47) */
  float cell_size;     /* HashGridOptions.cellSize (HashGrid.ts:34) */
  uint32_t dims[3];    /* PF_KEY_LINEAR: cells per axis */
  uint32_t table_size; /* PF_KEY_MORTON: power-of-two bucket count (HashGrid.ts:40) */
} pf_grid_desc;

/* Number of cells (keys) the descriptor defines, or 0 if it is invalid. */
PF_API uint64_t pf_grid_cells(const pf_grid_desc* grid);

/*
 * Stable counting sort of n particles by cell key.
 * Replaces HashGrid.rebuild() (src/core/hashGrid/HashGrid.ts:219-222): the
 * reset / cellIndexAndHistogram / blockScan / blockSumScan /
 * finalizeCellRanges / scatter kernels (cellIndex.ts:101-170, sort.ts:72-192).
 * Unlike the reference's atomic scatter the output is stable: particles of one
 * cell appear in ascending index order.
 *   d_pos4    device, n x float4 positions (w ignored)
 *   d_perm    device, n entries: particle index at each sorted slot
 *             (HashGridSnapshot.sortedIndices)
 *   d_start   device, C entries: first slot of each cell (cellStart)
 *   d_count   device, C entries: particles per cell (counts; cellEnd = start+count)
 *   d_keys    device, n entries or NULL: each particle's key (cellIndex)
 *   d_overflow device, 1 entry or NULL: 1 if a cell coordinate left the
 *             Morton range or was clamped (HashGrid.overflowFlag)
 *   stream    cudaStream_t or NULL for the legacy default stream
 * d_pos4 must be 16-byte aligned (float4 elements); the other buffers need
 * 4-byte alignment. Missing or misaligned buffers return PF_ERR_INVALID
 * before any device work.
 * Scratch memory comes from a per-device workspace owned by the library.
 */
PF_API pf_status pf_sort(const float* d_pos4, uint32_t n, const pf_grid_desc* grid,
                  uint32_t* d_perm, uint32_t* d_start, uint32_t* d_count,
                  uint32_t* d_keys, uint32_t* d_overflow, void* stream);

/* pf_sort that allocates no device memory (no counterpart in the reference;
 * added for callers that cannot allocate, such as hosts whose own pool owns
 * the device memory or loops where an allocation would stall the frame).
 * Same arguments and results as pf_sort. Its scratch is one fixed 23 MiB
 * block compiled into the library, so n <= 1,048,576 particles and at most
 * 2,097,152 cells per call; larger sizes return PF_ERR_INVALID. The runtime
 * loads that block lazily: the first call on a device reserves it there
 * (until the process exits) and looks up its address, so make that call
 * before the host's pool claims the device's memory and before any stream
 * capture. A call with n = 0 and NULL start and count does only this
 * set-up. Calls share the block: calls whose GPU work overlaps race, so
 * serialise them. pf_sort_device_errors on the same stream reads the
 * block's device error word. */
PF_API pf_status pf_sort_noalloc(const float* d_pos4, uint32_t n, const pf_grid_desc* grid,
                                 uint32_t* d_perm, uint32_t* d_start, uint32_t* d_count,
                                 uint32_t* d_keys, uint32_t* d_overflow, void* stream);

/* Synchronises `stream` and returns, then clears, the device error word of
 * the most recent pf_sort or pf_sort_noalloc on that stream (0 = no error;
 * bit 0 = a bounded look-back wait expired and the outputs are not to be
 * trusted). */
PF_API pf_status pf_sort_device_errors(void* stream, uint32_t* bits);

/* pf_sort with host buffers: copies the positions in, sorts, copies the
 * outputs back (any output pointer may be NULL). Synchronous. */
PF_API pf_status pf_sort_host(const float* h_pos4, uint32_t n, const pf_grid_desc* grid,
                       uint32_t* h_perm, uint32_t* h_start, uint32_t* h_count,
                       uint32_t* h_keys, uint32_t* h_overflow);

/* ------------------------------------------------------------------------ */
/* Scene: ParticleSystem + materials + colliders + SimLoop                   */
/* ------------------------------------------------------------------------ */

typedef struct pf_scene pf_scene;

typedef struct pf_range {
  uint32_t start;
  uint32_t count;
} pf_range;

/* new ParticleSystem(renderer, capacity, particleRadius)
 * (src/core/particles.ts:81-113). */
typedef struct pf_scene_desc {
  uint32_t capacity;
  float particle_radius;
} pf_scene_desc;

PF_API pf_status pf_scene_create(const pf_scene_desc* desc, pf_scene** out);
PF_API void pf_scene_destroy(pf_scene* scene);


/* ParticleSystem.uploadParticles(data, start) (particles.ts:121-160).
 * Host arrays of n entries starting at slot `start`; vel4/inv_mass/group may
 * be NULL for the reference defaults (0 velocity, invMass 1, group 0). */
PF_API pf_status pf_upload_particles(pf_scene* scene, const float* pos4, const float* vel4,
                                     const float* inv_mass, const uint32_t* group,
                                     uint32_t start, uint32_t n);

/* ParticleSystem.setInvMass(range, invMass) (particles.ts:163-173). */
PF_API pf_status pf_set_inv_mass(pf_scene* scene, pf_range range, float inv_mass);

/* new FluidSystem(particles, options) and FluidSystem.addBoundary
 * (src/fluids/FluidSystem.ts:31-54, 90-127, 171-183). Zero fields take the
 * reference defaults: rest_density 1000, particle_spacing 2r,
 * smoothing_radius 2*spacing. compliance < 0 selects the default 1e-4.
 * XSPH viscosity runs only when PF_FLUID_VISCOSITY is set, as optional effects
 * only compile in when given (FluidSystem.ts:111-115). */
#define PF_FLUID_VISCOSITY 1u
/* Vorticity confinement with strength `vorticity` (FluidSystemOptions.vorticity,
 * FluidSystem.ts:48; velocity.ts:13-120): the curl is gathered in the XSPH
 * walk, then eta = grad|omega| over fluid neighbours and
 * v += vorticity * dt * (eta/|eta| x omega). */
#define PF_FLUID_VORTICITY 2u
/* Surface tension (FluidSystemOptions.surfaceTension; Akinci et al. 2013
 * cohesion + curvature, cohesion.ts:33-120) and adhesion to boundary
 * particles (FluidSystemOptions.adhesion, adhesion.ts:33-76): velocity
 * changes gathered in a fixed-point accumulator (maxMag 50) once per
 * substep after the neighbour list, applied to v and to x* (times dt)
 * before the pressure solve (FluidSystem.ts:233-255). */
#define PF_FLUID_SURFACE_TENSION 4u
#define PF_FLUID_ADHESION 8u
typedef struct pf_fluid_desc {
  pf_range range;               /* count 0 = every particle */
  float rest_density;
  float particle_spacing;
  float smoothing_radius;
  float compliance;
  float viscosity;
  uint32_t flags;
  uint32_t n_boundaries;
  const pf_range* boundaries;   /* host, n_boundaries entries */
  const uint8_t* boundary_static; /* host or NULL: 1 = static boundary (addBoundary dynamic:false) */
  float vorticity;              /* used when PF_FLUID_VORTICITY is set */
  float surface_tension;        /* gamma, used when PF_FLUID_SURFACE_TENSION is set */
  float adhesion;               /* beta, used when PF_FLUID_ADHESION is set */
} pf_fluid_desc;
PF_API pf_status pf_add_fluid(pf_scene* scene, const pf_fluid_desc* desc, uint32_t* material_index);

/* new SoftbodySystem(particles, {bodies, shapeMatching})
 * (src/softbody/SoftbodySystem.ts:29-73, 132-199). */
typedef struct pf_softbody_def {
  pf_range range;
  uint32_t surface_count;       /* UINT32_MAX = every particle */
  float compliance;
  const float* rest_positions;  /* host xyz x count, or NULL = uploaded positions */
  const uint32_t* edges;        /* host pairs of body-local indices */
  uint32_t n_edges;             /* number of pairs */
} pf_softbody_def;
enum { PF_SHAPE_MATCH_GLOBAL = 0, PF_SHAPE_MATCH_LOCAL = 1 };
typedef struct pf_softbody_desc {
  uint32_t n_bodies;
  const pf_softbody_def* bodies;
  uint32_t shape_matching;      /* PF_SHAPE_MATCH_* */
  /* SoftbodySystemOptions.selfCollision (SoftbodySystem.ts:72, 218-234):
   * 0 = at pf_loop_build every body whose particles share no non-zero
   * collision group gets a fresh one (above every uploaded group), so its
   * particles never contact each other. */
  uint32_t self_collision;
} pf_softbody_desc;
PF_API pf_status pf_add_softbodies(pf_scene* scene, const pf_softbody_desc* desc,
                                   uint32_t* material_index);

/* new ClothSystem(particles, {graph, offset, stretchCompliance, bendCompliance,
 * tetherCompliance, wind, drag, lift, damping})
 * (src/cloth/ClothSystem.ts:37-141, 190-245) with the graph produced by
 * createClothGraph (src/cloth/graph.ts:130-342). Each iteration solves the
 * distance (stretch) colours, then the dihedral bending colours when the graph
 * has bending tuples (src/cloth/bending.ts), then the long-range tether
 * colours when tethers are given (src/cloth/tether.ts; build them from the
 * pins with pf_cloth_build_tethers). With triangles, aerodynamic drag and
 * lift move the predicted positions once per substep before the solve
 * (src/cloth/aero.ts); with has_damping, each particle's velocity is blended
 * toward the mean of its edge neighbours' after the substep
 * (ClothSystem.buildDamping, ClothSystem.ts:249-287). The cloth's particles
 * are uploaded from the graph. */
typedef struct pf_cloth_desc {
  uint32_t offset;
  uint32_t n_particles;
  const float* positions;       /* host xyz x n_particles (graph.positions) */
  const float* inv_mass;        /* host n_particles (graph.invMass) */
  uint32_t n_pairs;
  const uint32_t* pairs;        /* host cloth-local pairs (graph.distancePairs) */
  const float* rest_lengths;    /* host n_pairs (graph.distanceRestLengths) */
  float stretch_compliance;     /* < 0 selects the default 1e-7 */
  uint32_t n_bending;           /* 0: no bending constraints */
  const uint32_t* bending;      /* host cloth-local (p1, p2, p3, p4) x n_bending (graph.bendingTuples) */
  const float* bending_rest;    /* host n_bending signed rest angles (graph.bendingRestAngles) */
  float bend_compliance;        /* < 0 selects the default 1e-5 */
  uint32_t n_tethers;           /* 0: no tethers */
  const uint32_t* tether_particle; /* host cloth-local free particle per tether */
  const uint32_t* tether_anchor;   /* host cloth-local pinned anchor per tether */
  const float* tether_rest;        /* host rest radius per tether (metres) */
  float tether_compliance;      /* < 0 selects the default 0 */
  uint32_t n_triangles;         /* 0: no drag or lift */
  const uint32_t* triangles;    /* host cloth-local (i1, i2, i3) x n_triangles (graph.triangles) */
  float wind[3];                /* m/s */
  float drag;                   /* 1/2 C_D rho_air; < 0 selects the default 0.6125 */
  float lift;                   /* 1/2 C_L rho_air; < 0 selects the default 0.3 */
  uint32_t has_damping;         /* 0: no velocity smoothing pass (damping undefined) */
  float damping;                /* in [0, 1] */
} pf_cloth_desc;
PF_API pf_status pf_add_cloth(pf_scene* scene, const pf_cloth_desc* desc, uint32_t* material_index);

/* ClothSystem.wind / drag / lift / damping / bendCompliance setters
 * (ClothSystem.ts:143-188) for the cloth added as `material_index`: they
 * take effect from the next step. drag, lift and bend_compliance must be
 * >= 0 and finite, damping in [0, 1] (it needs has_damping at creation).
 * On a scene inside a batch, use the pf_batch_ form with the scene's index. */
typedef struct pf_cloth_params {
  float wind[3];
  float drag;
  float lift;
  float damping;
  float bend_compliance;
} pf_cloth_params;
PF_API pf_status pf_cloth_get_params(pf_scene* scene, uint32_t material_index, pf_cloth_params* out);
PF_API pf_status pf_cloth_set_params(pf_scene* scene, uint32_t material_index, const pf_cloth_params* params);

/* buildTethers (src/cloth/tetherBuild.ts:84-219): long-range attachments of
 * every free particle (inv_mass > 0) to the nearest pinned particle of each
 * of its `max_attachments` geodesically closest pinned islands, with rest
 * radius = geodesic distance x (1 + stretch_tolerance). Islands are the
 * connected components of the pinned particles over pinned-only edges; the
 * geodesic distances come from a multi-source Dijkstra per island over the
 * edge graph weighted by rest length, whose binary-heap order settles ties
 * as the reference's does. Outputs are cloth-local, particle-major, each
 * particle's islands nearest first; `capacity` entries are available in
 * each output array (n_particles x max_attachments always suffices) and
 * `count` receives the number written. max_attachments 0 selects 4. */
typedef struct pf_tether_build_desc {
  uint32_t n_particles;
  const float* inv_mass;        /* host n_particles (graph.invMass) */
  uint32_t n_pairs;
  const uint32_t* pairs;        /* host cloth-local pairs (graph.distancePairs) */
  const double* rest_lengths;   /* host n_pairs (graph.distanceRestLengths, doubles) */
  uint32_t max_attachments;
  double stretch_tolerance;     /* >= 0 */
} pf_tether_build_desc;
PF_API pf_status pf_cloth_build_tethers(const pf_tether_build_desc* desc, uint32_t* particle,
                                        uint32_t* anchor, float* rest, uint32_t capacity,
                                        uint32_t* count);

/* PrimitiveSet.addPlane/addSphere/addBox/addCapsule and setSphere
 * (src/core/collision/PrimitiveSet.ts:166-257), using the packed GPU record
 * of the reference (primitives.ts:125-186, PrimitiveSet.ts:64-76). */
enum { PF_PRIM_PLANE = 0, PF_PRIM_SPHERE = 1, PF_PRIM_BOX = 2, PF_PRIM_CAPSULE = 3 };
enum { PF_PRIM_INVERT = 1, PF_PRIM_SWEEP = 2 };
typedef struct pf_primitive {
  uint32_t kind;
  uint32_t flags;
  float data0[4];     /* plane: normal; sphere/box: centre (w radius); capsule: a (w radius) */
  float data1[4];     /* plane: point; box: half extents; capsule: b; w = muS */
  float velocity[4];  /* w = muK */
  float rotation[4];  /* unit quaternion xyzw (boxes) */
  float spin[4];      /* angular velocity about the pivot, rad/s */
} pf_primitive;
PF_API pf_status pf_add_primitive(pf_scene* scene, const pf_primitive* prim, uint32_t* slot);
PF_API pf_status pf_set_primitive(pf_scene* scene, uint32_t slot, const pf_primitive* prim);

/* new SDFCollider(particles, sdf, {muS, muK, thickness, position, rotation,
 * scale}) (src/core/collision/SDFCollider.ts:88-137): a signed-distance grid
 * (one distance per voxel, x fastest; voxel (i, j, k) centred at
 * origin + (i + 0.5, j + 0.5, k + 0.5) * voxel_size in the collider's local
 * frame) stored as half floats (converted round-to-nearest-even), sampled
 * trilinearly with clamp-to-edge, its gradient by central differences one
 * voxel apart (sdf.ts:107-147). A particle touches it where
 * phi < radius + thickness; contact and friction are those of the
 * primitives (collider.ts:53-118) against a static surface. Colliders run
 * in the order added: the primitives of the scene, then its SDF colliders. */
typedef struct pf_sdf_desc {
  uint32_t res[3];      /* >= 4 each */
  const float* data;    /* res[0] * res[1] * res[2] distances */
  float origin[3];      /* local-frame corner of voxel (0, 0, 0) */
  float voxel_size[3];  /* > 0 */
  float position[3];    /* world position of the local origin */
  float rotation[4];    /* unit quaternion (x, y, z, w) */
  float scale;          /* uniform, > 0 */
  float thickness;      /* >= 0 */
  float mu_s, mu_k;     /* >= 0 */
} pf_sdf_desc;

PF_API pf_status pf_add_sdf_collider(pf_scene* scene, const pf_sdf_desc* sdf, uint32_t* slot);
/* SDFCollider.setPosition / setRotation / setScale (SDFCollider.ts:170-201):
 * takes effect from the next step. */
PF_API pf_status pf_set_sdf_transform(pf_scene* scene, uint32_t slot, const float position[3],
                                      const float rotation[4], float scale);

/* new SimLoop(particles, {substeps, iterations, gravity, hashOrigin})
 * (src/core/loop.ts:33-57, 117-243). Builds the substep pipeline for the
 * materials and colliders added so far and allocates the device state. */
typedef struct pf_loop_desc {
  uint32_t substeps;
  uint32_t iterations;
  float gravity[3];
  float hash_origin[3];
  /* First size and placement of the neighbour grid window in metres. The
   * grid is a window over the reference's cell lattice (cell = the widest
   * query radius, aligned to hash_origin) that moves with the particles
   * each substep, and grows between steps (to twice their spread on an
   * axis, up to 2^27 cells) when they come close to its size. Particles
   * spread wider than the window before it has grown (on the first step,
   * or past that limit) are clamped into its border cells
   * (pf_overflow.grid_clamped). min >= max on any axis selects a window
   * four times the extent of the uploaded particles (at least 16 cells
   * more), centred on them. */
  float grid_min[3];
  float grid_max[3];
  /* SimLoopOptions.contact (loop.ts:20-30, 347-417; src/core/contact/):
   * particle-particle contacts between every pair of particles within 2r
   * (candidates within 2r x 1.1) outside a common non-zero collision group,
   * found from the particles outside the noSelfContacts ranges (the fluids'
   * and pf_add_no_self_contacts'), with static friction in the solve and
   * kinetic friction after it. */
  uint32_t contact;             /* 0 = off */
  float contact_mu_s;           /* < 0 selects the default 0.5 */
  float contact_mu_k;           /* < 0 selects the default 0.4 */
  uint32_t max_contacts;        /* pairs kept per substep; 0 selects 8 x capacity */
} pf_loop_desc;
PF_API pf_status pf_loop_build(pf_scene* scene, const pf_loop_desc* desc);

/* A material that only declares MaterialKernels.noSelfContacts
 * (materials.ts:45): particles of `range` search for no contacts, so pairs
 * of two of them are never generated (pairs with another particle are found
 * from the other side). Fluids declare their own range this way. */
PF_API pf_status pf_add_no_self_contacts(pf_scene* scene, pf_range range);

/* ContactBuffer.readbackCount / readbackPairs (ContactBuffer.ts:75-97): the
 * pairs the last substep generated, dropped ones included in `count`;
 * `pairs` receives up to `capacity` (i, j) particle-index pairs, each pair
 * ordered i < j and the list sorted. Synchronous. */
PF_API pf_status pf_contacts_read(pf_scene* scene, uint32_t* pairs, uint32_t capacity, uint32_t* count,
                                  uint32_t* stored);

/* SimLoop.step(dt) (loop.ts:267-279): one frame of `substeps` substeps, dt in
 * seconds (a double, as the reference's JavaScript number). Asynchronous. */
PF_API pf_status pf_step(pf_scene* scene, double dt);


/* ParticleSystem.readback() (particles.ts:192-227) and material outputs. */
typedef enum pf_field {
  PF_FIELD_POSITIONS = 0,          /* float4 x capacity, w = 0 */
  PF_FIELD_PREDICTED = 1,          /* float4 x capacity, w = 0 */
  PF_FIELD_VELOCITIES = 2,         /* float4 x capacity */
  PF_FIELD_INV_MASS = 3,           /* float x capacity */
  PF_FIELD_BOUNDARY_VOLUME = 4,    /* float x capacity */
  PF_FIELD_DENSITY = 5,            /* float x capacity (FluidSystem.density) */
  PF_FIELD_ROTATION = 6,           /* float4 x capacity */
  PF_FIELD_PREDICTED_ROTATION = 7, /* float4 x capacity */
  PF_FIELD_ANGULAR_VELOCITY = 8,   /* float4 x capacity */
  PF_FIELD_LAMBDA = 9,             /* float x capacity (fluid lambda) */
  PF_FIELD_NEIGHBOR_COUNT = 10,    /* uint32 x capacity (NeighborList.counts) */
  PF_FIELD_NEIGHBORS = 11,         /* uint32 x capacity x 64, row i = particle i's neighbours */
  PF_FIELD_CELL_PERM = 12          /* uint32 x capacity: particle index per sorted slot */
} pf_field;
PF_API pf_status pf_readback(pf_scene* scene, uint32_t field, void* dst_host, size_t bytes);
/* Whole-field write of POSITIONS, PREDICTED, VELOCITIES (float4 x capacity,
 * w ignored) or INV_MASS (float x capacity) in particle order, as the
 * reference's callers set a buffer's array and flag needsUpdate (for
 * example a test damping velocities between frames, or moving pinned
 * particles; particles.ts:81-113). Synchronous; takes effect from the next
 * step. PREDICTED needs a built scene. */
PF_API pf_status pf_write(pf_scene* scene, uint32_t field, const void* src_host, size_t bytes);

/* SimLoop.readbackOverflow() (loop.ts:59-69, 286-295) plus the neighbour-list
 * flag of FluidSystem.readbackOverflow().
 *   grid          a cell coordinate left the reference's Morton range
 *                 (|cell| >= 512 cells from hashOrigin; cellIndex.ts:145-169),
 *                 exactly where the reference raises its flag
 *   grid_clamped  (no reference counterpart) the scene's particles spread
 *                 wider than its grid window, so some were clamped into the
 *                 window's border cells: neighbour sets stay complete, but
 *                 their order can depart from the reference's walk. The window
 *                 follows the particles each substep and grows between steps
 *                 (see pf_loop_desc.grid_min/max), so this fires only when a
 *                 step outruns it. */
typedef struct pf_overflow {
  uint32_t positions;
  uint32_t velocities;
  uint32_t grid;
  uint32_t contacts;
  uint32_t neighbors;
  uint32_t device_error;
  uint32_t grid_clamped;
} pf_overflow;
PF_API pf_status pf_overflow_read(pf_scene* scene, pf_overflow* out);

/* Device milliseconds of the last pf_step (CUDA events on the scene stream). */
PF_API pf_status pf_last_step_ms(pf_scene* scene, float* ms);

/* ------------------------------------------------------------------------ */
/* Batching: many scenes, one launch per stage, one CUDA graph per tick       */
/* ------------------------------------------------------------------------ */

typedef struct pf_batch pf_batch;

typedef struct pf_batch_opts {
  uint32_t use_graph;        /* capture each tick as a CUDA graph */
  uint32_t block_size;       /* 0 = autotuned */
} pf_batch_opts;

/* Pack the current state of `n` built scenes into one batch. The scenes stay
 * valid and independent; the batch owns copies of their state. */
PF_API pf_status pf_batch_create(pf_scene* const* scenes, uint32_t n, const pf_batch_opts* opts,
                                 pf_batch** out);
PF_API void pf_batch_destroy(pf_batch* batch);
/* One step of every scene; dt applies to all. Asynchronous. */
PF_API pf_status pf_batch_step(pf_batch* batch, double dt);
/* Move scene `index`'s primitive `slot` (PrimitiveSet.setSphere etc.). */
PF_API pf_status pf_batch_set_primitive(pf_batch* batch, uint32_t index, uint32_t slot,
                                        const pf_primitive* prim);
/* Scene `index`'s cloth parameters (pf_cloth_set_params). */
PF_API pf_status pf_batch_cloth_set_params(pf_batch* batch, uint32_t index, uint32_t material_index,
                                           const pf_cloth_params* params);
PF_API pf_status pf_batch_readback(pf_batch* batch, uint32_t index, uint32_t field, void* dst_host,
                                   size_t bytes);
PF_API pf_status pf_batch_write(pf_batch* batch, uint32_t index, uint32_t field, const void* src_host,
                                size_t bytes);
PF_API pf_status pf_batch_overflow_read(pf_batch* batch, uint32_t index, pf_overflow* out);
PF_API pf_status pf_batch_last_step_ms(pf_batch* batch, float* ms);
/* Particle-substeps one pf_batch_step advances (sum over scenes of N * substeps). */
PF_API uint64_t pf_batch_particle_substeps(pf_batch* batch);
/* Kernel launches of the batch's last step (counted when it was issued or
 * captured), and the bytes of per-step parameters copied host-to-device. */
PF_API uint64_t pf_batch_launches_per_step(pf_batch* batch);
PF_API uint64_t pf_batch_step_upload_bytes(pf_batch* batch);
/* The cudaStream_t the batch (or a built scene) runs on, for callers that
 * order their own work after it or time it with events. */
PF_API void* pf_batch_stream(pf_batch* batch);
PF_API void* pf_scene_stream(pf_scene* scene);
/* Positions of every scene of the batch, each scene's particles in particle
 * order (w = 0), scenes concatenated in batch order: one device gather and
 * one device-to-host copy (pinned host memory makes it fastest). Synchronous. */
PF_API pf_status pf_batch_read_positions(pf_batch* batch, float* dst_host, size_t bytes);
/* pf_batch_read_positions without the wait, as the reference's readback
 * returns a promise (particles.ts:200-227): the gather is queued on the
 * batch's stream behind its work so far, and the copy to dst_host runs on a
 * second stream, beside the steps that follow. dst_host holds the positions
 * once pf_batch_wait_reads returns; until then leave it alone and keep it
 * alive. Use pinned host memory (a pageable destination makes the copy
 * synchronous). Two reads can be in flight; a third first waits for the
 * oldest. */
PF_API pf_status pf_batch_read_positions_async(pf_batch* batch, float* dst_host, size_t bytes);
/* Waits until every pf_batch_read_positions_async of the batch has landed. */
PF_API pf_status pf_batch_wait_reads(pf_batch* batch);
/* Average device milliseconds of one solver stage launched `reps` times on the
 * batch's current state: 0 neighbour lists, 1 density + lambda, 2 position
 * correction, 3 XSPH, 4 predict. `items` receives the particles the stage
 * covers (fluid particles for 0-3). For measurement; it changes no state
 * that the next pf_batch_step reads. */
PF_API pf_status pf_batch_profile_stage(pf_batch* batch, uint32_t stage, uint32_t reps, float* ms,
                                        uint64_t* items);
/* The fluid neighbour-pass configuration the autotuner chose on the batch's
 * first step: path 0 = one thread per slot (block threads per block, list
 * entries fetched `unroll` at a time), 1 = warp tiles. `group` (may be NULL)
 * receives the fluid particles per group of the scenes that hold only one
 * fluid of one mass, stepped group by group so that a group's lists stay in
 * L2 across its passes (0: one launch per pass over all of them).
 * `entry_bits` (may be NULL) receives the width of the list entries: 16
 * (offsets from a per-warp base where a warp's rows allow it) or 32 (whole
 * slots in every warp). */
PF_API pf_status pf_batch_tuning(pf_batch* batch, uint32_t* path, uint32_t* block, uint32_t* unroll,
                                 uint32_t* group, uint32_t* entry_bits);

/* ------------------------------------------------------------------------ */
/* Mesh -> particle setup on the GPU                                          */
/* ------------------------------------------------------------------------ */

/* A triangle mesh as toTriangleMesh reads a BufferGeometry (src/core/mesh.ts:
 * 16-56): xyz float vertices and three indices per triangle. */
typedef struct pf_mesh {
  const float* vertices;        /* host xyz x n_vertices */
  uint32_t n_vertices;
  const uint32_t* indices;      /* host, n_indices entries (a multiple of 3) */
  uint32_t n_indices;
} pf_mesh;

/* Output of the voxeliser (VoxelizeResult, voxelize.ts:23-36). `count`,
 * `surface_count` and `edge_count` are always set; `positions` (xyz x count,
 * surface particles first) is written when `capacity` >= count, `edges`
 * (pairs i < j) up to `edge_capacity` pairs, so a first call with NULL
 * buffers sizes the second. */
typedef struct pf_voxels {
  float* positions;
  uint32_t capacity;
  uint32_t* edges;
  uint32_t edge_capacity;
  uint32_t count, surface_count, edge_count;
} pf_voxels;

/* voxelize(mesh, {particleRadius, largestPiece}) (src/softbody/voxelize.ts:
 * 50-161): grid points at spacing 2r over the mesh's box, inside by
 * ray-cast parity (every point against every triangle on the GPU, in
 * doubles as the reference computes), then the largest face-connected
 * piece when asked, surface particles first, face-adjacent pairs. */
PF_API pf_status pf_voxelize_mesh(const pf_mesh* mesh, double particle_radius, uint32_t largest_piece,
                                  pf_voxels* out);
/* voxelize(SDFData, {particleRadius, dilation, largestPiece}): inside where
 * the trilinear field (sample.ts:12-47) is below `dilation`. `data` is the
 * float field, x fastest. */
PF_API pf_status pf_voxelize_sdf(const float* data, const uint32_t res[3], const double origin[3],
                                 const double voxel_size[3], double particle_radius, double dilation,
                                 uint32_t largest_piece, pf_voxels* out);
/* bakeMeshToSdf(mesh, {resolution, padding}) (src/sdf/bake.ts:84-139): a
 * resolution^3 cubic grid around the mesh (padding < 0 selects two voxels,
 * one below resolution 8), per voxel centre the distance to the closest
 * triangle and the sign of the three jittered axis-ray parities' majority,
 * on the GPU in doubles. `data` receives resolution^3 floats (x fastest),
 * `origin` and `voxel_size` the grid, `inconsistent` the voxels whose
 * votes split; more than 1% of them fails as the reference throws (the
 * field is written first). */
PF_API pf_status pf_bake_sdf(const pf_mesh* mesh, uint32_t resolution, double padding, float* data,
                             double origin[3], double* voxel_size, uint64_t* inconsistent);

/* ------------------------------------------------------------------------ */
/* Serving: continuous batching under an HBM budget                           */
/* ------------------------------------------------------------------------ */

typedef struct pf_server pf_server;

/* Scheduling modes. BATCHED packs admitted scenes into cohorts (one world,
 * one launch per solver stage, one CUDA graph per tick each); PLAIN gives
 * every scene its own world stepped on its own stream without graphs, the
 * per-scene loop of the reference's Simulation.step (Simulation.ts:542-634). */
enum { PF_SERVER_BATCHED = 0, PF_SERVER_PLAIN = 1 };

typedef struct pf_server_opts {
  uint64_t hbm_budget_bytes;  /* device bytes live cohorts may hold (0: 150 GB) */
  uint32_t max_scenes;        /* live + building scenes at most (0: 65536) */
  uint32_t use_graph;         /* BATCHED: capture each cohort's tick as a CUDA graph */
  uint32_t max_cohorts;       /* BATCHED: cohorts before the smallest is folded into the next (0: 4) */
  uint32_t mode;              /* PF_SERVER_BATCHED or PF_SERVER_PLAIN */
  uint32_t async_build;       /* build admitted cohorts on a host worker thread while ticks go on */
} pf_server_opts;

typedef struct pf_server_stats {
  uint32_t live;              /* scenes stepped each tick */
  uint32_t queued;            /* submitted, waiting for memory or a slot */
  uint32_t building;          /* admitted, their cohort is being built */
  uint32_t finished;
  uint32_t cohorts;
  uint32_t reserved0;
  uint64_t ticks;
  uint64_t particle_substeps; /* sum over ticks of the live scenes' particles x substeps */
  uint64_t state_bytes;       /* device bytes held by cohorts and the build in flight */
  uint64_t rebuilds;          /* cohorts built (admission waves and folds) */
  double busy_ms;             /* sum of tick wall times */
  float last_tick_ms;
  float p50_tick_ms;
  float p99_tick_ms;
  float max_tick_ms;
  float max_swap_ms;          /* longest swap-in of a built cohort (imports, frees) */
  float max_admit_ms;         /* longest admission (synchronous builds included) */
  float last_admit_ms;        /* admission inside the last tick (PLAIN: its world builds);
                                 last_tick_ms minus this is that tick's stepping */
  float max_step_ms;          /* longest stepping inside a tick: every cohort's launches and
                                 the wait for them (a fresh cohort's graph capture included) */
  float max_free_ms;          /* longest release of emptied cohorts inside a tick */
} pf_server_stats;

/* Request states reported by pf_server_request_state. */
enum { PF_REQ_QUEUED = 0, PF_REQ_BUILDING = 1, PF_REQ_LIVE = 2, PF_REQ_DONE = 3 };

PF_API pf_status pf_server_create(const pf_server_opts* opts, pf_server** out);
PF_API void pf_server_destroy(pf_server* server);
/* Queue a scene for admission: materials and primitives added, and either a
 * built SimLoop (loop == NULL: its current state is taken) or an unbuilt one
 * with `loop` giving the SimLoop options. The server copies the scene; the
 * caller keeps ownership of `scene`. The request retires after
 * `lifetime_steps` ticks of stepping. */
PF_API pf_status pf_server_submit(pf_server* server, pf_scene* scene, const pf_loop_desc* loop,
                                  uint32_t lifetime_steps, uint64_t* ticket);
/* Swap in a finished cohort build, admit what fits the budget (FIFO), step
 * every live scene once by dt, retire scenes whose lifetime is over. */
PF_API pf_status pf_server_tick(pf_server* server, double dt);
/* Wait for a cohort build in flight (if any) and swap it in. */
PF_API pf_status pf_server_drain_build(pf_server* server);
PF_API pf_status pf_server_request_state(pf_server* server, uint64_t ticket, uint32_t* state,
                                         uint32_t* steps_done);
/* A live request's field (any pf_field), or a finished request's final state
 * (positions, velocities, inverse mass, boundary volume, rotation, angular
 * velocity). */
PF_API pf_status pf_server_readback(pf_server* server, uint64_t ticket, uint32_t field, void* dst, size_t bytes);
/* Device bytes a scene would hold alone in a cohort (the admission estimate). */
PF_API pf_status pf_server_estimate_bytes(pf_scene* scene, const pf_loop_desc* loop, uint64_t* bytes);
PF_API pf_status pf_server_stats_read(pf_server* server, pf_server_stats* out);

#ifdef __cplusplus
}
#endif

#endif /* PFSIM_H */
