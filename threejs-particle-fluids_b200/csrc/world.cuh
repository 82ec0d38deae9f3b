// world.cuh — the solver engine: one "world" packs one or more independent
// scenes (ParticleSystem + materials + colliders + SimLoop each) into shared
// device arrays and steps all of them with one launch per solver stage.
//
// Layout (B200-first):
//  * Each scene owns a segment of slots [seg_start, seg_end), 256-aligned, so
//    every 256-thread block belongs to exactly one scene and reads its
//    parameters uniformly. Particle ids equal slots at creation; after every
//    grid rebuild the per-slot state is physically permuted into cell order
//    (stable: ascending id inside a cell), so neighbour gathers and per-slot
//    passes are coalesced float4 loads. ids[slot] and inv[id] map between the
//    two orders; materials with topology (cloth pairs, shape-matching groups)
//    address particles by id through inv[].
//  * Scenes with a fluid get a bounded linear grid (cell = smoothing radius)
//    at a private key offset; one stable counting sort covers every scene.
//  * Per-slot state (x, x*, v, boundary volume, material tag) is
//    double-buffered; the permutation gathers from one buffer into the other.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "grid_sort.cuh"
#include "pfsim.h"

namespace pf {

constexpr uint32_t kSegAlign = 256;
constexpr uint32_t kMaxNbr = 64;  // NeighborList MAX_NEIGHBORS (neighborList.ts:14)
// The slot path's neighbour list is blocked by warp: each warp of slots owns
// an 8 KB block. Entries are 16-bit offsets from a per-warp base slot
// (nbr_base[k / 32]) when every slot the warp's 27-cell rows reach lies
// within 65,536 slots of the lowest, which is the common case. Then the
// entries go in groups of kNbrGroup (16 bytes) per slot: group g of the
// warp's 32 slots is 512 contiguous bytes, slot k's 16 bytes at lane k % 32
// (nbr16_at), so a warp reads a group as one coalesced 16-byte load per
// lane. Otherwise the warp's base is kNbrWide and its entries are whole
// slots, word nbr_col(k) + m * kNbrStride (a warp's m-th entries one line).
// The 16-bit groups fill half the block; the list build stores hits past
// the kMaxNbr-th in group kMaxNbr / kNbrGroup, which no reader reads.
constexpr uint32_t kNbrStride = 32;
constexpr uint32_t kNbrGroup = 8;
constexpr uint32_t kNbrWide = 0x80000000u;
static_assert(kSegAlign % kNbrStride == 0, "a scene's segment starts on a list block");
static_assert(kMaxNbr % kNbrGroup == 0, "whole groups");
__host__ __device__ __forceinline__ size_t nbr_col(size_t k) {
  return (k >> 5) * (size_t)kMaxNbr * kNbrStride + (k & 31);
}
// halfword index of slot k's 16-bit entry m
__host__ __device__ __forceinline__ size_t nbr16_at(size_t k, uint32_t m) {
  return (k >> 5) * (size_t)kMaxNbr * kNbrStride * 2 + (size_t)(m / kNbrGroup) * (kNbrStride * kNbrGroup) +
         (k & 31) * kNbrGroup + (m % kNbrGroup);
}
__host__ __device__ __forceinline__ size_t nbr16_col(size_t k) { return nbr16_at(k, 0); }
constexpr uint32_t kBlock = 256;
constexpr uint64_t kSortCellCap = 0x7fffffffull;  // keys of a world's sort stay below this
constexpr uint32_t kMaxContacts = 32;  // contact pairs kept per emitting particle per substep

// ------------------------------------------------------------- host spec ----
struct RangeU {
  uint32_t start = 0, count = 0;
  bool contains(uint32_t i) const { return i >= start && i < start + count; }
};

struct FluidSpec {
  RangeU range;
  double rho0, spacing, h, compliance, viscosity, vorticity = 0, surface_tension = 0, adhesion = 0;
  bool has_visc, has_vort = false, has_st = false, has_ad = false;
  std::vector<RangeU> bnd;
  std::vector<uint8_t> bnd_static;
};

struct BodySpec {
  RangeU range;
  uint32_t surface;
  double compliance;
};

struct SoftSpec {
  bool local = true;
  bool self_collision = false;
  std::vector<BodySpec> bodies;
  RangeU span;
  std::vector<float> rest4;        // float4 per particle of the scene (cap)
  std::vector<float> weights;      // per particle (cap)
  std::vector<uint32_t> offsets;   // CSR by particle (cap + 1), local mode
  std::vector<uint32_t> indices;   // CSR members (particle indices)
  std::vector<float> rest_centers4;  // float4 per particle, local mode
};

struct ClothSpec {
  uint32_t offset = 0, n = 0;
  std::vector<uint32_t> pairs;  // absolute particle indices
  std::vector<float> rest;
  float compliance = 1e-7f;
  std::vector<std::vector<uint32_t>> colors;  // constraint indices per colour
  // bending (bending.ts): (p1, p2, p3, p4) absolute indices per constraint
  std::vector<uint32_t> bend;
  std::vector<float> bend_rest;
  float bend_compliance = 1e-5f;
  std::vector<std::vector<uint32_t>> bend_colors;
  // tethers (tether.ts): (free particle, pinned anchor) absolute indices
  std::vector<uint32_t> tether;
  std::vector<float> tether_rest;
  float tether_compliance = 0.0f;
  std::vector<std::vector<uint32_t>> tether_colors;
  // aerodynamics (aero.ts): absolute triangle indices
  std::vector<uint32_t> tris;
  float wind[3] = {0.0f, 0.0f, 0.0f};
  float drag = 0.6125f, lift = 0.3f;
  // velocity smoothing (ClothSystem.buildDamping)
  bool has_damping = false;
  float damping = 0.0f;
};

// SDFCollider state (SDFCollider.ts:88-137): the grid as half floats plus
// the transform and contact parameters.
struct SdfSpec {
  uint32_t res[3] = {0, 0, 0};
  std::vector<uint16_t> half;  // res[0] * res[1] * res[2], x fastest
  float origin[3], voxel[3], position[3];
  double rot_q[4];             // unit quaternion (x, y, z, w)
  float scale, thickness, mu_s, mu_k;
};

enum MatKind : uint32_t { MAT_FLUID = 0, MAT_SOFT = 1, MAT_CLOTH = 2 };

struct SceneSpec {
  uint32_t cap = 0;
  double radius = 0;
  std::vector<float> pos4, vel4, inv_mass, bvol;
  std::vector<float> rot4, angv4;  // orientation state (identity / zero)
  std::vector<uint32_t> group;
  std::vector<std::pair<MatKind, uint32_t>> materials;
  std::vector<FluidSpec> fluids;
  std::vector<SoftSpec> softs;
  std::vector<ClothSpec> cloths;
  std::vector<pf_primitive> prims;
  std::vector<SdfSpec> sdfs;
  std::vector<RangeU> quiet;  // pf_add_no_self_contacts ranges (fluids' ranges are implied)
  pf_loop_desc loop{};
  bool built = false;
  bool initialized = false;  // the one-time init pass (static boundaries) ran
  // Grid bounds resolved from the initial positions at the first build; a
  // scene rebuilt later (into a batch or a serving cohort) keeps its grid.
  bool bounds_resolved = false;
  double grid_lo[3] = {0, 0, 0}, grid_hi[3] = {0, 0, 0};
};

// ----------------------------------------------------------- device data ----
struct DevScene {
  uint32_t seg_start, seg_end, cap;
  uint32_t substeps, iterations;
  float gx, gy, gz;
  float dt;        // substep length (per step)
  float substeps_f;
  float radius;    // particle radius as an f32 literal
  uint32_t has_grid;
  uint32_t cell_base, cells;  // dead cell = cell_base + cells
  float ox, oy, oz, cell;
  // The grid is a window of dims cells over the reference's unbounded cell
  // lattice: cell (i, j, k) = floor((x - origin) / cell) lies at local cell
  // (i, j, k) - lo. lo0 is the window placed at build; each substep the
  // window moves the least that covers every particle of the scene
  // (k_grid_fit writes lo), so a window at least as large as the scene's
  // extent never clamps.
  int32_t lo[3];
  int32_t lo0[3];
  uint32_t dims[3];
  uint32_t prim_base, prim_count;
  uint32_t planes_fast;  // every primitive is a plane that neither sweeps nor spins (plane4 holds it)
  float pos_scale, pos_inv, vel_scale, vel_inv;
  float sb_scale, sb_inv;
  uint32_t fluid_first, fluid_count;  // this scene's fluids in the fluid table
  uint32_t soft_local_ranks;          // bit r: a local shape-matching system at material rank r
  uint32_t init_pending;              // the one-time init pass has not run for this scene
  uint32_t sdf_base, sdf_count;       // this scene's SDF colliders in the SDF table
  uint32_t collide_rank1;             // r + 1: colliders run inside the apply of fluid rank r (its last material)
  uint32_t contact;                   // particle-particle contacts on
  uint32_t max_contacts;              // pairs solved per substep (the first in slot order)
  float c_mus, c_muk;                 // contact friction
  float c_dist, c_cand2;              // 2r and (2r * 1.1)^2 as f32 literals
  float prune_slack;                  // metres the neighbour walk's cell boxes are widened by when pruning
  // one fluid over every particle, no boundaries, one inverse mass: every
  // neighbour has mass homog_mass, and the position pass gathers (x*, lambda)
  // from xl in one load
  uint32_t homog;
  float homog_mass;
  // a single-fluid scene of one mass with nothing else but fused colliders,
  // stepped by the L2-sized groups of World::run_groups (the world's other
  // passes leave it alone)
  uint32_t grouped;
};

// One SDF collider as the kernels read it (sdf.ts:17-80 fields).
struct DevSdf {
  uint32_t res[3];
  uint32_t data_off;  // first voxel in the half-float pool
  float origin[3], inv_voxel[3], voxel[3];
  float position[3];
  float rot[9], inv_rot[9];  // row-major R and R^T
  float scale, inv_scale, thickness, mu_s, mu_k;
};

struct DevFluid {
  uint32_t scene, rank;
  float rho0, inv_rho0, volume, h, hsq, poly6, spiky, compliance, c_xsph;
  uint32_t has_visc;
  uint32_t has_vort;
  float vort_eps;  // vorticity confinement strength
  uint32_t has_st, has_ad;  // surface tension, adhesion
  float gamma, beta, mass;
  float coh_coef, coh_h6_64;   // cohesion spline: 32/(pi h^9), h^6/64
  float adh_coef, adh_m4h, adh_2h;  // adhesion spline: 0.007/h^3.25, -4/h, 2h
  uint32_t range_end;          // first id past the fluid's range
  float imp_scale, imp_inv;    // impulse accumulator (maxMag 50)
  uint32_t bnd_first, bnd_count;
  uint32_t react_lo, react_hi;  // covering id range of the boundaries (lo == hi: no reaction)
  float react_scale, react_inv;
};

// Mutable parameters of one cloth (ClothSystem.ts:143-188 setters).
struct DevCloth {
  float wind[3];
  float drag, lift, damping, bend_compliance, pad;
};

struct DevBoundary {
  uint32_t start, count;  // absolute ids
  uint32_t fluid;
  uint32_t is_static;
};

struct DevSoft {
  uint32_t scene, rank, local;
  float ai, maxc2;
};

struct DevBody {
  uint32_t scene, soft;  // soft = index into DevSoft
  uint32_t start, count; // absolute ids
  float compliance;
};

// Per-scene overflow words (SimLoopOverflow + neighbour-list flag).
enum FlagIdx : uint32_t {
  FLAG_POS = 0,
  FLAG_VEL = 1,
  FLAG_GRID = 2,
  FLAG_CONTACTS = 3,
  FLAG_NBR = 4,
  FLAG_SOFT = 5,
  FLAG_REACT = 6,
  FLAG_DEVICE = 7,
  FLAG_CLAMP = 8,  // a particle lay outside its scene's grid window and was clamped into it
  kNumFlags = 9
};

// Per-slot tag: low 16 bits fluid index + 1, high 16 bits boundary index + 1.
__host__ __device__ inline uint32_t tag_fluid(uint32_t t) { return t & 0xffffu; }
__host__ __device__ inline uint32_t tag_bnd(uint32_t t) { return t >> 16; }

// A tile of the fluid neighbour passes: own particles [p0, p1) of one grid
// row segment, and its halo (the nine neighbouring row segments) as slot
// ranges rs[r] .. rs[r] + (roff[r + 1] - roff[r]), concatenated in (dz, dy)
// order starting at halo index roff[r].
struct Tile {
  uint32_t scene, p0, p1, halo;
  uint32_t rs[9];
  uint32_t roff[10];
};

struct StateBuf {
  float4* x = nullptr;   // committed positions, w = inverse mass
  float4* xs = nullptr;  // predicted positions, w = inverse mass
  float4* v = nullptr;   // velocities
  float* bv = nullptr;   // boundary volume
  uint32_t* tag = nullptr;
  float* dens = nullptr;  // fluid density of the last density pass (read by surface tension)
};

// Everything a stage kernel needs, passed by value.
struct WorldView {
  uint32_t n;            // total slots
  uint32_t prim_stride;  // colliders (primitives + SDFs) per slot in the collider lambda array
  const DevScene* scenes;
  const uint32_t* chunk_scene;  // scene of each 256-slot chunk
  // the 256-slot chunks (ascending) of the scenes with a fluid, and of the
  // scenes whose colliders run in their own pass: those passes' slot kernels
  // are launched over their chunks only
  const uint32_t* fchunk;
  const uint32_t* cchunk;
  uint32_t n_fchunk, n_cchunk;
  DevScene* scenes_rw;
  uint32_t* flags;              // kNumFlags per scene
  int32_t* bbox;                // per scene: lowest and highest cell of the predicted positions (6 words)
  int32_t* bbox_last;           // per scene: the bounds the last window fit used (6 words; read between steps)
  float* clocks;                // collider sweep clock per scene (PrimitiveSet.motionClock)
  const DevFluid* fluids;
  const DevBoundary* bnds;
  const pf_primitive* prims;
  const float4* plane4;  // 2 per primitive: (normal, inverted), (point, 0); read in scenes with planes_fast
  const DevSdf* sdfs;
  const uint16_t* sdf_half;  // half-float voxels of every SDF collider
  StateBuf cur, nxt;
  uint32_t* ids;
  uint32_t* inv;
  uint32_t* keys;     // by id
  uint32_t* perm;     // new slot -> id (sort output)
  uint32_t* cstart;
  uint32_t* ccount;
  uint32_t* nbr;      // kMaxNbr * n, blocked by warp: 16- or 32-bit entries (slot path)
  uint32_t* nbr_base; // per warp of slots: base slot of its 16-bit entries, or kNbrWide
  uint32_t nbr_wide_only;  // the list build stores whole 32-bit slots for every warp (a tuned choice)
  uint16_t* nbr16;    // the same storage, kMaxNbr * n halfwords: halo index of each neighbour (tile path)
  uint32_t* ncount;
  uint32_t* slot_tile;  // tile of each slot (this substep)
  Tile* tiles;
  uint32_t* tile_count;
  uint32_t max_tiles;
  const uint32_t* row_base;    // first global grid row of each fluid scene (n_grid_scenes + 1)
  const uint32_t* grid_scene;  // scene of each fluid scene index
  uint32_t n_grid_scenes;
  uint32_t n_rows;
  float* lambda;
  // per slot (lambda, q): the slot path's lambda, and the neighbour mass code
  // q = bv > 0 ? bv : -(own mass), so a neighbour pass reads both the
  // multiplier and the SPH mass (shared.ts:52-62) in one 8-byte gather
  float2* lm;
  float4* xl;  // (x*, lambda) per fluid slot of homogeneous scenes, written by the density pass
  float4* dx;
  float4* dv;
  float4* vort;       // curl of the velocity per slot, w = its length (vorticity confinement)
  float4* normal;     // scaled colour-field normal per slot (surface tension)
  int4* acc_imp;      // fixed-point velocity changes of surface tension and adhesion
  float2* plam;       // (lambda_n, lambda_t) per slot x primitive
  uint32_t* cmask;    // per slot: bit p set once collider p < 32 touched it this substep (plam entry valid)
  int4* acc_react;    // fixed-point reaction sums per slot
  // soft bodies (by id unless noted)
  const DevSoft* softs;
  const DevBody* bodies;
  const uint32_t* grp;       // group ids (local shape matching)
  const uint32_t* grp_soft;  // soft index per group
  uint32_t n_grp;
  const uint32_t* csr_off;   // by id, n + 1
  const uint32_t* csr_idx;
  const float4* rest;        // rest offsets, w = compliance
  const float4* rest_c;      // neighbourhood rest centres
  const float* weights;
  // 4 rows per cluster id: the rotation's rows with the cluster centre's
  // x, y, z in w, then (rest centre, compliance); the record the
  // shape-matching gather reads per (member, cluster) pair, 64 aligned bytes
  float4* rot4;
  float4* q;                 // orientation
  float4* qp;                // predicted orientation
  float4* omega;             // angular velocity
  float4* pair_lambda;       // per CSR entry
  // the clusters that hold each particle (by id): entries [mem_off[j],
  // mem_off[j + 1]) of mem are (cluster centre id, CSR position), mem_soft[j]
  // the particle's soft system
  const uint32_t* mem_off;
  const uint2* mem;
  const uint32_t* mem_soft;
  const uint32_t* mem_ids;   // the ids held by at least one cluster, ascending
  uint32_t n_mem_ids;
  float4* lambda_g;          // global matching multipliers per id
  float4* body_c;            // per body
  float4* body_r;            // 3 rows per body
  uint32_t n_bodies;
  // cloth
  const uint32_t* c_i;
  const uint32_t* c_j;
  const float* c_rest;
  const float* c_comp;
  const uint32_t* c_scene;
  float* c_lambda;
  uint32_t n_cons;
  // cloth bending (bending.ts), by (rank, colour)
  const uint4* b_idx;  // particle ids (p1, p2, p3, p4)
  const float* b_rest;
  const uint32_t* b_cloth;  // cloth parameter index (bending compliance)
  const uint32_t* b_scene;
  float* b_lambda;
  uint32_t n_bend;
  // cloth tethers (tether.ts), by (rank, colour)
  const uint4* t_rec;  // (particle id, anchor id, rest bits, compliance bits)
  const uint32_t* t_scene;
  float* t_lambda;
  uint32_t n_teth;
  // cloth aerodynamics (aero.ts): one record per cloth particle, its
  // incident triangles as a CSR over a_tri
  const uint2* a_vtx;   // (particle id, cloth parameter index)
  const uint32_t* a_off;
  const uint4* a_tri;   // (i1, i2, i3) particle ids
  // cloth velocity smoothing (ClothSystem.buildDamping): one record per
  // cloth particle, its edge neighbours as a CSR over d_nbr
  const uint2* d_vtx;   // (particle id, cloth parameter index)
  const uint32_t* d_off;
  const uint32_t* d_nbr;  // particle ids
  float4* d_smooth;     // blended velocity per record
  const DevCloth* cloth_par;
  // particle contacts (src/core/contact/): per emitting slot, up to
  // kMaxContacts partner slots in column-major lists (entry m of slot k at
  // m * n + k) with their multipliers and last normal
  const uint32_t* cgroup;   // collision group by id
  const uint8_t* cquiet;    // 1: inside a noSelfContacts range, by id
  uint32_t* con_nbr;
  uint32_t* con_cnt;        // pairs found per slot (uncapped)
  uint32_t* con_pre;        // exclusive prefix of con_cnt inside the slot's 256-slot chunk
  uint32_t* chunk_sum;      // per chunk: pairs found, and pairs past the per-slot cap
  uint32_t* chunk_drop;
  uint32_t* chunk_off;      // per chunk: first pair index inside its scene
  int2* con_lam;            // (lambda_n, lambda_t) ticks of 2^-20 kg m
  float4* con_nrm;
  int4* acc_con;            // fixed-point position (then velocity) sums per slot
  uint2* con_stat;          // per scene: pairs found in the last substep, pairs past the per-slot cap
};

class World {
 public:
  World() = default;
  ~World();
  World(const World&) = delete;
  World& operator=(const World&) = delete;

  // Pack `specs` (their current host state) into device arrays. With
  // `plan_only` nothing touches the GPU: the layout is computed and
  // device_bytes() reports what the build would allocate.
  // `skip_state[s]` set: scene s's dynamic state is not uploaded (it is
  // imported with import_scene before the first step).
  pf_status build(const std::vector<SceneSpec*>& specs, bool use_graph, bool plan_only = false,
                  const std::vector<uint8_t>* skip_state = nullptr);
  // Overwrite scene `s`'s dynamic state (positions with inverse mass,
  // velocities, boundary volumes, orientations, angular velocities) with
  // scene `src_s` of `src`, device to device. Both worlds hold the same
  // scene spec; `src` must be idle.
  pf_status import_scene(uint32_t s, const World& src, uint32_t src_s);
  // Stop stepping scene `s` (its slots keep their last state).
  void retire(uint32_t s);
  bool retired(uint32_t s) const { return h_scenes_[s].substeps == 0; }
  pf_status step(double dt);
  pf_status set_primitive(uint32_t scene, uint32_t slot, const pf_primitive& p);
  pf_status set_sdf_transform(uint32_t scene, uint32_t slot, const float pos[3], const double q[4], float scale);
  pf_status set_cloth_params(uint32_t scene, uint32_t material, const pf_cloth_params& p);
  pf_status write(uint32_t scene, uint32_t field, const void* src, size_t bytes);
  pf_status readback(uint32_t scene, uint32_t field, void* dst, size_t bytes);
  // Copies the scene's state (by particle index) back into its spec.
  pf_status pull_state(uint32_t scene, SceneSpec* spec);
  pf_status overflow(uint32_t scene, pf_overflow* out);
  pf_status contacts(uint32_t scene, uint32_t* pairs, uint32_t capacity, uint32_t* count, uint32_t* stored);
  // Device milliseconds between the start and end events of the last step.
  pf_status elapsed_ms(float* ms);
  cudaStream_t stream() const { return stream_; }
  uint32_t scene_count() const { return (uint32_t)specs_.size(); }
  uint64_t particle_substeps_per_step() const;
  // Positions of every scene, each in particle order, w = 0, concatenated in
  // scene order, into host memory (one gather kernel + one copy).
  pf_status read_positions(float* dst_host, size_t bytes);
  // read_positions queued behind the work so far: the gather on the world's
  // stream, the copy on a second stream beside the next steps (two staging
  // buffers, so at most two reads in flight); dst_host is written once
  // wait_reads returns.
  pf_status read_positions_async(float* dst_host, size_t bytes);
  pf_status wait_reads();
  uint64_t total_particles() const;
  uint64_t launches_per_step() const { return launches_per_step_; }
  size_t step_upload_bytes() const { return sizeof(DevScene) * h_scenes_.size(); }
  // Average device milliseconds of one solver stage run `reps` times on the
  // current state (substep 0, iteration 0, material rank 0).
  pf_status profile_stage(uint32_t stage, uint32_t reps, float* ms, uint64_t* items);
  // Neighbour-pass configuration the autotuner chose (path 0: one thread
  // per slot, `block` threads per block, list entries fetched `unroll` at a
  // time; path 1: warp tiles).
  // The slot path tunes each of its kernels on its own: kSlotNbr (list
  // build), kSlotLambda (density + lambda), kSlotDelta (position
  // correction), kSlotVel (XSPH and the other velocity-stage passes).
  struct Tuning {
    uint32_t path = 0;
    uint32_t block[4] = {256, 256, 256, 256};
    uint32_t unroll[4] = {4, 4, 4, 4};
    // fluid particles per group of run_groups (0: no groups): the scenes
    // that only hold one fluid of one mass run their whole substep group by
    // group, so a group's lists and records stay in L2 across its passes
    uint32_t group = 0;
    // the list build walks its nine rows as one sequence (k_s_neighbors kFlat)
    uint32_t nbr_flat = 0;
    // list entries as whole 32-bit slots in every warp instead of 16-bit
    // offsets where they fit: fewer bytes against fewer decode instructions
    uint32_t nbr_wide = 0;
  };
  void tuning(uint32_t* path, uint32_t* block, uint32_t* unroll = nullptr) const {
    *path = tune_.path;
    *block = tune_.block[kSlotLambda];
    if (unroll) *unroll = tune_.unroll[kSlotLambda];
  }
  const Tuning& tuning_all() const { return tune_; }
  bool tuned() const { return tuned_; }
  bool has_fluid() const { return any_fluid_; }
  // Use a configuration tuned elsewhere (another world of the same kind of
  // scenes) instead of timing candidates on the first step.
  void set_tuning(const Tuning& t) {
    tune_ = t;
    tuned_ = true;
    apply_grouping();  // this world's own groups of that size
    drop_graphs();     // captured launches depend on the path
  }
  size_t device_bytes() const { return bytes_; }

 private:
  pf_status alloc_all();
  void run_substep(uint32_t s, uint32_t parity);
  // bbox_ready: the predict pass of this substep gathered the cell bounds
  // the grid window follows (otherwise a separate pass gathers them)
  void run_sort_and_permute(uint32_t parity, bool bbox_ready);
  void run_init_pass();
  void launch_tiles_build(const WorldView& V, uint32_t s);
  template <typename K, typename... A>
  void launch_fluid(uint32_t block, K kernel, const WorldView& V, A... args);
  uint32_t mem_lanes_ = 32;  // lanes per cluster member in the shape-matching gather
  void run_fluid_neighbors(const WorldView& V, uint32_t s);
  void run_fluid_lambda_delta(const WorldView& V, uint32_t r, uint32_t s, uint32_t it);
  void run_fluid_xsph(const WorldView& V, uint32_t r, uint32_t s);
  // L2-sized groups of the single-fluid scenes (their chunks lead fchunk):
  // each group's substep (list build, iterations, advect, XSPH) in turn
  void run_groups(const WorldView& V, uint32_t s, bool apply);
  WorldView group_view(const WorldView& V, size_t g) const;
  WorldView rest_view(const WorldView& V) const;  // the other fluid scenes' chunks
  void apply_grouping();  // groups_ and the scenes' grouped flags from tune_.group
  bool grouping() const { return tune_.path == 0 && !groups_.empty(); }
  pf_status tune();
  pf_status tune_trials();  // time the candidates on this world's state
  // tuning cache file (PFSIM_TUNE_CACHE): the key of this world on this GPU,
  // and the lookup (true: tune_ holds a valid cached choice) and append
  std::string tune_key() const;
  bool load_tuning(const char* file, const std::string& key);
  void store_tuning(const char* file, const std::string& key) const;
  template <typename K, typename... A>
  void launch_tiled(K kernel, size_t smem, const WorldView& V, A... args);
  void launch_frame_start_at(uint32_t parity);
  pf_status upload_params(double dt);
  WorldView view(uint32_t parity) const;

  std::vector<SceneSpec*> specs_;
  std::vector<DevScene> h_scenes_;
  std::vector<DevFluid> h_fluids_;
  std::vector<DevBoundary> h_bnds_;
  std::vector<DevSoft> h_softs_;
  std::vector<DevBody> h_bodies_;
  std::vector<pf_primitive> h_prims_;
  std::vector<DevSdf> h_sdfs_;
  bool sdfs_dirty_ = false;
  // stage plan
  uint32_t max_rank_ = 0, max_sub_ = 0, max_iter_ = 0;
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> cloth_ranges_;  // [rank] -> per colour [begin,end)
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> bend_ranges_;   // [rank] -> per colour [begin,end)
  std::vector<std::vector<std::pair<uint32_t, uint32_t>>> teth_ranges_;   // [rank] -> per colour [begin,end)
  std::pair<uint32_t, uint32_t> aero_ranges_[2] = {{0, 0}, {0, 0}};      // before / after the fluid preSolve
  std::vector<std::pair<uint32_t, uint32_t>> damp_ranges_;               // [rank] -> [begin,end)
  std::vector<DevCloth> h_cloth_par_;
  std::vector<std::vector<int32_t>> cloth_par_of_;  // [scene][material] -> parameter index (-1: not a cloth)
  bool cloth_par_dirty_ = false;
  DevCloth* cloth_par_dev_ = nullptr;
  void launch_cloth_rank(const WorldView& V, uint32_t r, uint32_t s, uint32_t it, cudaStream_t st);
  void launch_aero(const WorldView& V, uint32_t stage, uint32_t s);
  bool any_grid_ = false, any_prims_ = false, any_fluid_ = false, any_visc_ = false, any_vort_ = false;
  bool any_imp_ = false;  // surface tension or adhesion somewhere
  bool any_soft_local_ = false, any_soft_global_ = false, any_static_bnd_ = false, any_dyn_bnd_ = false;
  bool any_react_ = false;
  bool any_unfused_prims_ = false;  // a scene whose colliders run in their own pass
  bool any_contact_ = false;        // a scene with particle contacts
  bool any_multi_fluid_ = false;    // a scene with two or more fluids (slot path only)
  bool fuse_dens_ = false;          // the slot list build forms the first density and lambda
  // single-fluid scenes (DevScene::grouped candidates): their chunks are
  // fchunk[0, n_pure_chunks_), scene by scene; per scene its end chunk and
  // its fluid particles
  uint32_t n_pure_chunks_ = 0;
  std::vector<uint32_t> pure_end_;
  std::vector<uint64_t> pure_parts_;
  std::vector<uint32_t> pure_scene_;
  std::vector<std::pair<uint32_t, uint32_t>> groups_;  // chunk ranges [begin, end) of fchunk
  uint32_t n_ = 0, cells_ = 0, prim_stride_ = 0;
  // device memory: one arena
  void* arena_ = nullptr;
  size_t bytes_ = 0;
  WorldView base_{};
  StateBuf buf_[2];
  SortScratch sort_{};
  RadixPlan radix_{};
  uint32_t parity_ = 0;
  bool inited_ = false;
  // neighbour passes: autotuned once per world, before the first graph capture
  static constexpr int kSlotNbr = 0, kSlotLambda = 1, kSlotDelta = 2, kSlotVel = 3;
  Tuning tune_{};
  bool tuned_ = false;
  // graph
  bool use_graph_ = false;
  cudaGraphExec_t graph_[2] = {nullptr, nullptr};
  void drop_graphs();
  double graph_dt_ = -1;
  cudaStream_t stream_ = nullptr;
  // second stream for cloth-only scenes (fork/join inside each substep)
  bool side_ok_ = false;
  cudaStream_t side_stream_ = nullptr;
  cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  float last_ms_ = 0;
  // pinned staging for per-step parameters
  DevScene* h_pinned_scenes_ = nullptr;
  pf_primitive* h_pinned_prims_ = nullptr;
  std::vector<float4> h_plane4_;
  float4* h_pinned_plane4_ = nullptr;
  void refresh_planes(int only_scene);
  std::vector<bool> lam_in_xl_;  // per scene: the last step kept lambda in xl (homogeneous scene)
  DevSdf* h_pinned_sdfs_ = nullptr;
  DevCloth* h_pinned_cloth_ = nullptr;
  bool prims_dirty_ = true;
  size_t pair_entries_ = 0;
  float4* stage_pos_ = nullptr;  // gather buffer of read_positions
  float4* stage_pos2_ = nullptr;  // the second one of read_positions_async
  cudaStream_t read_stream_ = nullptr;  // copies of read_positions_async (made on first use)
  cudaEvent_t ev_gathered_[2] = {nullptr, nullptr}, ev_read_[2] = {nullptr, nullptr};
  bool read_pending_[2] = {false, false};
  uint32_t read_next_ = 0;
  uint64_t* prefix_dev_ = nullptr;
  uint64_t launches_per_step_ = 0;
  std::vector<uint64_t> prefix_;   // particle offset of each scene in read_positions
  // Grid windows grow with their particles: after each step the last window
  // fit's cell bounds come back to pinned memory (a ring of kBoundsRing
  // buffers, each with an event), and before a later step any window they
  // have nearly outgrown is widened and the cell arrays laid out again
  // (outside any graph), from the newest bounds that have arrived.
  static constexpr uint32_t kBoundsRing = 4;
  int32_t* h_pinned_bbox_ = nullptr;  // kBoundsRing buffers of 6 words per scene
  cudaEvent_t ev_bounds_[kBoundsRing] = {};
  uint64_t steps_done_ = 0;
  uint64_t bounds_seen_ = 0;  // steps_done_ of the last bounds looked at, plus one (0: none yet)
  // Per-step parameters go through a ring of kParamRing pinned staging
  // buffers, so the host can queue that many steps ahead; a buffer is
  // written again once the event of its last upload has passed.
  static constexpr uint32_t kParamRing = 3;
  cudaEvent_t ev_params_[kParamRing] = {};
  bool params_pending_[kParamRing] = {};
  uint64_t uploads_ = 0;
  pf_status wait_uploads();  // every upload queued so far (before rewriting the single-buffer tables)
  void* grid_arena_ = nullptr;  // cell arrays once the windows outgrow the arena's
  void* sort_arena_ = nullptr;  // sort scratch once the windows pass the cells it was carved for
  uint64_t cells_cap_ = 0;      // cells the current cell arrays and sort scratch hold
  std::vector<int32_t> grow_prev_ext_;  // per scene and axis: the spread in cells at the last look
  uint32_t regrowths_ = 0;
  bool graphs_stale_ = false;  // the windows grew: capture the graphs again before launching one
  pf_status maybe_grow_windows();
  pf_status relayout_grid();

 public:
  uint32_t window_regrowths() const { return regrowths_; }
};

}  // namespace pf
