// world.cu — stage kernels of the solver substep and the World host engine.
//
// One substep follows the reference's stage order (src/core/loop.ts:175-242):
//   predict -> [grid rebuild: keys+histogram, stable sort, permute state]
//   -> preSolve (collider lambda reset, boundary volumes, neighbour lists,
//      multiplier resets) -> iterations x [materials in order, colliders +
//      position apply] -> advect -> postSolve (XSPH, orientations)
//   -> friction + velocity apply -> clock tick.
// Every kernel covers all scenes of the world; a 256-slot block belongs to
// one scene. Colliders add to their own particle only, so the reference's
// fixed-point accumulate-then-apply is done in registers (same integer sums).

#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <set>

#include "devmem.cuh"
#include "world.cuh"
#include "world_kernels.cuh"
#include "world_slots.cuh"
#include "world_tiles.cuh"
#include "world_contacts.cuh"

namespace pf {

namespace {

// ---------------------------------------------------------- frame start ----
__global__ void k_frame_start(WorldView V, uint32_t nscenes) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nscenes) return;
  const DevScene& S = V.scenes[s];
  for (uint32_t f = 0; f < kNumFlags; ++f) V.flags[s * kNumFlags + f] = 0;
  // PrimitiveSet.ts:400-402: clock = dt * (substeps - 1)
  V.clocks[s] = S.dt * (S.substeps_f - 1.0f);
}

// PrimitiveSet.ts:403-405, once per substep after friction.
__global__ void k_tick(WorldView V, uint32_t nscenes, uint32_t sub) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nscenes) return;
  const DevScene& S = V.scenes[s];
  if (sub >= S.substeps || S.prim_count == 0) return;
  V.clocks[s] = fmaxf(V.clocks[s] - S.dt, 0.0f);
}

// ------------------------------------------------------------ integrate ----
// integrate.ts:25-34, and the cell bounds of every scene's predicted
// positions (the grid window follows them; scenes past their substeps give
// their unchanged ones). A 256-slot block belongs to one scene.
__global__ void __launch_bounds__(kBlock) k_predict(WorldView V, uint32_t sub) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t s = scene_index(V, k);
  const DevScene& S = V.scenes[s];
  const float4 x = V.cur.x[k];
  f3 p = mk(0.0f, 0.0f, 0.0f);
  if (sub < S.substeps && x.w > 0.0f) {
    const float4 v = V.cur.v[k];
    const float dt = S.dt;
    const f3 vel = xyz(v) + mk(S.gx, S.gy, S.gz) * dt;
    V.cur.v[k] = with_w(vel, 0.0f);
    p = xyz(x) + vel * dt;
    V.cur.xs[k] = with_w(p, x.w);
  } else if (S.has_grid) {
    p = xyz(V.cur.xs[k]);
  }
  if (S.has_grid) bbox_block_add(V, S, s, k < S.seg_start + S.cap, p);
}

// The cell bounds of every scene's predicted positions, where no predict
// pass gathered them (the one-time init pass and the autotuner's sort).
__global__ void __launch_bounds__(kBlock) k_bbox(WorldView V) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t s = scene_index(V, k);
  const DevScene& S = V.scenes[s];
  if (S.has_grid) bbox_block_add(V, S, s, k < S.seg_start + S.cap, xyz(V.cur.xs[k]));
}

// Places each grid scene's window for this substep: the least move of the
// build-time window (lo0) that covers the scene's cell bounds, or lo0 where
// the bounds are wider than the window (the keys then clamp and flag). The
// bounds are kept in bbox_last (the host widens windows between steps from
// them) and reset for the next substep.
__global__ void k_grid_fit(WorldView V, uint32_t nscenes) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nscenes) return;
  DevScene& S = V.scenes_rw[s];
  if (!S.has_grid) return;
  int32_t* b = V.bbox + 6 * s;
  float big = 0.0f;
  const float org[3] = {S.ox, S.oy, S.oz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int64_t mn = b[a], mx = b[a + 3], d = S.dims[a];
    if (mn <= mx) {  // scenes past their substeps keep their last bounds
      V.bbox_last[6 * s + a] = b[a];
      V.bbox_last[6 * s + a + 3] = b[a + 3];
    }
    int64_t lo = S.lo0[a];
    if (mn <= mx && mx - mn + 1 <= d) {
      if (lo > mn) lo = mn;
      if (lo + d - 1 < mx) lo = mx - d + 1;
    }
    S.lo[a] = (int32_t)lo;
    b[a] = INT32_MAX;
    b[a + 3] = INT32_MIN;
    big = fmaxf(big, fabsf(org[a]) + fmaxf(fabsf((float)lo), fabsf((float)(lo + d))) * S.cell);
  }
  // the neighbour walk prunes a cell only when its box, widened by this
  // slack (far above the f32 rounding of cell_of and of the box edges), is
  // out of reach
  S.prune_slack = big * (1.0f / 65536.0f) + 1e-9f;
}

// integrate.ts:36-44 (scenes stepped by groups advect there)
__device__ __forceinline__ void advect_slot(const WorldView& V, const DevScene& S, uint32_t k) {
  const float4 x = V.cur.x[k];
  if (!(x.w > 0.0f)) return;
  const float4 xs = V.cur.xs[k];
  V.cur.v[k] = with_w((xyz(xs) - xyz(x)) / S.dt, 0.0f);
  V.cur.x[k] = xs;
}
__global__ void __launch_bounds__(kBlock) k_advect(WorldView V, uint32_t sub) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= V.n) return;
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps || S.grouped) return;
  advect_slot(V, S, k);
}
// The advect of one group of run_groups, over its chunks.
__global__ void __launch_bounds__(kBlock) k_advect_chunks(WorldView V, uint32_t sub) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_fchunk * kSegAlign) return;
  const uint32_t k = chunk_slot(V.fchunk, g);
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps) return;
  advect_slot(V, S, k);
}

// ---------------------------------------------------------------- grid ----
// Keys by particle id (cell of the predicted position in the scene's grid
// window, offset by the scene's key base; dead padding goes to the scene's
// last key), with the radix digit counts of the sort in a block histogram
// (grid-stride loop, one flush per block).
__global__ void __launch_bounds__(kBlock) k_keys(WorldView V, DigitHist h) {
  extern __shared__ uint32_t sh[];
  digit_hist_zero(sh, h);
  __syncthreads();
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < V.n; k += gridDim.x * blockDim.x) {
    const uint32_t s = scene_index(V, k);
    const DevScene& S = V.scenes[s];
    const uint32_t id = V.ids[k];
    uint32_t key;
    bool clamped = false, ref_over = false;
    if (id >= S.seg_start + S.cap) {
      key = S.cell_base + S.cells;
    } else if (S.has_grid) {
      int32_t cx, cy, cz;
      local_cell(S, xyz(V.cur.xs[k]), &cx, &cy, &cz, &clamped, &ref_over);
      key = S.cell_base + (uint32_t)cx + S.dims[0] * ((uint32_t)cy + S.dims[1] * (uint32_t)cz);
    } else {
      key = S.cell_base + (id - S.seg_start);
    }
    V.keys[id] = key;
    digit_hist_add(sh, h, key);
    if (clamped) atomicOr(V.flags + s * kNumFlags + FLAG_CLAMP, 1u);
    if (ref_over) atomicOr(V.flags + s * kNumFlags + FLAG_GRID, 1u);
  }
  __syncthreads();
  digit_hist_flush(sh, h);
}

// Gather the per-slot state into cell order: new slot k takes particle
// perm[k] from its old slot inv[perm[k]]; per-substep sums start at zero.
__global__ void __launch_bounds__(kBlock) k_permute(WorldView V) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= V.n) return;
  const uint32_t id = V.perm[k];
  const uint32_t o = V.inv[id];
  const float4 xo = V.cur.x[o];
  const float bvo = V.cur.bv[o];
  V.nxt.x[k] = xo;
  V.nxt.xs[k] = V.cur.xs[o];
  V.nxt.v[k] = V.cur.v[o];
  V.nxt.bv[k] = bvo;
  if (V.lm) V.lm[k] = make_float2(0.0f, mass_code(bvo, xo.w));
  V.nxt.tag[k] = V.cur.tag[o];
  V.nxt.dens[k] = V.cur.dens[o];
  V.ids[k] = id;
  V.inv[id] = k;
  // lambda is read for every neighbour, fluid or not (positionDelta.ts:193),
  // and is zero for particles no fluid solves; slots change owners here.
  V.lambda[k] = 0.0f;
  // the first 32 collider multipliers start at zero through the mask
  V.cmask[k] = 0u;
  for (uint32_t p = 32; p < V.prim_stride; ++p) V.plam[(size_t)k * V.prim_stride + p] = make_float2(0.0f, 0.0f);
  if (V.acc_react) V.acc_react[k] = make_int4(0, 0, 0, 0);
  if (V.acc_imp) V.acc_imp[k] = make_int4(0, 0, 0, 0);
}

// Without a grid the slots never move; only the per-substep sums reset.
__global__ void __launch_bounds__(kBlock) k_reset_sums(WorldView V) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= V.n) return;
  V.cmask[k] = 0u;
  for (uint32_t p = 32; p < V.prim_stride; ++p) V.plam[(size_t)k * V.prim_stride + p] = make_float2(0.0f, 0.0f);
  if (V.acc_react) V.acc_react[k] = make_int4(0, 0, 0, 0);
}

// ---------------------------------------------------------------- fluid ----
// boundaryVolume.ts:36-52: V_i = 1 / max(sum_j W(x_i - x_j), 1e-12) over the
// particle's own boundary range, walking the grid (not the neighbour list).
__global__ void __launch_bounds__(kBlock) k_boundary_volume(WorldView V, uint32_t want_static, uint32_t sub) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= V.n) return;
  const uint32_t b = tag_bnd(V.cur.tag[k]);
  if (!b) return;
  const DevBoundary B = V.bnds[b - 1];
  if (B.is_static != want_static) return;
  const DevScene& S = scene_at(V, k);
  if (want_static ? !S.init_pending : sub >= S.substeps) return;
  const DevFluid& F = V.fluids[B.fluid];
  const float4* pos = want_static ? V.cur.x : V.cur.xs;
  const f3 xi = xyz(pos[k]);
  float sum = 0.0f;
  walk27(S, V.cstart, V.ccount, xi, [&](uint32_t j) {
    const uint32_t idj = V.ids[j];
    if (idj < B.start || idj >= B.start + B.count) return true;
    const f3 off = xi - xyz(pos[j]);
    const float rsq = dot(off, off);
    if (rsq >= F.hsq) return true;
    sum += poly6(rsq, F);
    return true;
  });
  const float bv = 1.0f / fmaxf(sum, 1e-12f);
  V.cur.bv[k] = bv;
  if (V.lm) V.lm[k].y = bv;
}

// A 256-thread block covers one 256-slot chunk, hence one scene: its
// primitives are staged in shared memory once per block (all threads,
// before any returns), and read from there by every particle.
constexpr uint32_t kSmemPrims = 16;
struct PrimStage {
  pf_primitive p[kSmemPrims];
};
__device__ __forceinline__ const pf_primitive* stage_prims(const WorldView& V, PrimStage& st,
                                                           uint32_t first = blockIdx.x * blockDim.x) {
  const uint32_t sb = first < V.n ? scene_index(V, first) : 0u;
  const DevScene& S = V.scenes[sb];
  const pf_primitive* src = V.prims + S.prim_base;
  if (S.prim_count > kSmemPrims) return src;  // uniform over the block
  constexpr uint32_t kWords = sizeof(pf_primitive) / 4;
  const uint32_t* w = reinterpret_cast<const uint32_t*>(src);
  uint32_t* d = reinterpret_cast<uint32_t*>(st.p);
  for (uint32_t t = threadIdx.x; t < S.prim_count * kWords; t += blockDim.x) d[t] = __ldg(w + t);
  __syncthreads();
  return st.p;
}

// positionDelta.ts:217-226, then the reaction accumulator's apply over the
// covering range of the fluid's boundaries (FluidSystem.ts:280-287).
// With skip_homog the slots of single-fluid scenes of one mass are left to
// the position pass, which applies them itself (k_s_delta).
__global__ void __launch_bounds__(kBlock, 4) k_fluid_apply(WorldView V, uint32_t rank, uint32_t sub, uint32_t it,
                                                        uint32_t skip_homog) {
  // launched over the chunks of the scenes with a fluid (a block is one chunk)
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = g < V.n_fchunk * kSegAlign;
  const uint32_t k = live ? chunk_slot(V.fchunk, g) : 0u;
  // the slot's own loads go out first, so their latency overlaps the
  // primitive staging and the scene lookup
  uint32_t tg = 0;
  float4 x = make_float4(0, 0, 0, 0), d = make_float4(0, 0, 0, 0);
  if (live) {
    tg = __ldg(V.cur.tag + k);
    x = V.cur.xs[k];
    d = V.dx[k];
  }
  __shared__ PrimStage st;
  const pf_primitive* prims = stage_prims(V, st, chunk_slot(V.fchunk, blockIdx.x * blockDim.x));
  if (!live) return;
  const uint32_t s = scene_index(V, k);
  const DevScene& S = V.scenes[s];
  if (sub >= S.substeps || it >= S.iterations || S.fluid_count == 0 || (skip_homog && S.homog)) return;
  const uint32_t f = tag_fluid(tg);
  bool changed = false;
  if (f && V.fluids[f - 1].rank == rank) {
    x.x += d.x;
    x.y += d.y;
    x.z += d.z;
    changed = true;
  }
  if (V.acc_react) {
    const uint32_t id = V.ids[k];
    for (uint32_t q = 0; q < S.fluid_count; ++q) {
      const DevFluid& F = V.fluids[S.fluid_first + q];
      if (F.rank != rank || F.react_lo == F.react_hi) continue;
      if (id < F.react_lo || id >= F.react_hi) continue;
      int4 t = V.acc_react[k];
      bool sat = false;
      const f3 c = ticks_change(t.x, t.y, t.z, F.react_inv, &sat);
      V.acc_react[k] = make_int4(0, 0, 0, 0);
      x.x += c.x;
      x.y += c.y;
      x.z += c.z;
      changed = true;
      if (sat) atomicOr(V.flags + s * kNumFlags + FLAG_REACT, 1u);
    }
  }
  // the scene's colliders follow its last material in the same pass
  if (S.collide_rank1 == rank + 1 && collide_particle(V, S, s, k, x, prims)) changed = true;
  if (changed) V.cur.xs[k] = x;
}

// velocity.ts:99-120: the vorticity confinement force eps (N x omega) dt with
// N = eta / |eta| (eta from k_s_vort_grad, in dx), then the XSPH change.
__global__ void __launch_bounds__(kBlock) k_xsph_apply(WorldView V, uint32_t rank, uint32_t sub) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_fchunk * kSegAlign) return;
  const uint32_t k = chunk_slot(V.fchunk, g);  // slots of the scenes with a fluid
  const uint32_t f = tag_fluid(V.cur.tag[k]);
  if (!f) return;
  const DevFluid& F = V.fluids[f - 1];
  if (F.rank != rank || !(F.has_visc || F.has_vort)) return;
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps) return;
  f3 change = mk(0.0f, 0.0f, 0.0f);
  if (F.has_vort) {
    const f3 eta = xyz(V.dx[k]);
    const float el = len(eta);
    if (el >= 1e-12f) change = change + cross(eta / el, xyz(V.vort[k])) * F.vort_eps * S.dt;
  }
  if (F.has_visc) change = change + xyz(V.dv[k]);
  float4 v = V.cur.v[k];
  v.x += change.x;
  v.y += change.y;
  v.z += change.z;
  V.cur.v[k] = v;
}

// ------------------------------------------------------------ colliders ----

// PrimitiveSet.ts:339-365 + SDFCollider.ts:256-281 with collider.ts:53-89,
// fused with the position accumulator's apply (loop.ts:225): a contact only
// adds to its own particle, so the sum of rounded ticks is formed in
// registers. Scenes whose last material is a fluid run this inside the
// fluid's apply instead (collide_rank1).
__global__ void __launch_bounds__(kBlock, 4) k_collide(WorldView V, uint32_t sub, uint32_t it) {
  // launched over the chunks of the scenes that need this pass (a block is
  // one chunk)
  static_assert(kBlock == kSegAlign, "one block per chunk");
  __shared__ PrimStage st;
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  const pf_primitive* prims = stage_prims(V, st, chunk_slot(V.cchunk, blockIdx.x * blockDim.x));
  if (g >= V.n_cchunk * kSegAlign) return;
  const uint32_t k = chunk_slot(V.cchunk, g);
  const uint32_t s = scene_index(V, k);
  const DevScene& S = V.scenes[s];
  if ((S.prim_count + S.sdf_count == 0 && !S.contact) || S.collide_rank1 || sub >= S.substeps || it >= S.iterations)
    return;
  float4 xs4 = V.cur.xs[k];
  int4 start = make_int4(0, 0, 0, 0);
  if (S.contact) {
    start = V.acc_con[k];
    if (start.x | start.y | start.z) V.acc_con[k] = make_int4(0, 0, 0, 0);
  }
  if (collide_particle(V, S, s, k, xs4, prims, start)) V.cur.xs[k] = xs4;
}

// PrimitiveSet.ts:367-398 with collider.ts:96-118, fused with the velocity
// accumulator's apply (loop.ts:226-230).
__global__ void __launch_bounds__(kBlock) k_friction(WorldView V, uint32_t sub) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  // A slot has work when a collider touched it this substep (the others'
  // multipliers are zero and add nothing) or contact friction
  // (k_con_friction) scattered velocity ticks for it first. A block without
  // any leaves before staging its scene's primitives.
  bool work = false;
  uint32_t s = 0, mask = 0;
  int4 start = make_int4(0, 0, 0, 0);
  if (k < V.n) {
    // the slot's contact mask goes out with the scene lookup, not after it
    const uint32_t m = V.cmask[k];
    s = scene_index(V, k);
    const DevScene& S0 = V.scenes[s];
    if ((S0.prim_count + S0.sdf_count > 0 || S0.contact) && sub < S0.substeps) {
      if (S0.contact) {
        start = V.acc_con[k];
        if (start.x | start.y | start.z) V.acc_con[k] = make_int4(0, 0, 0, 0);
      }
      mask = m;
      work = mask || S0.prim_count + S0.sdf_count > 32 || (start.x | start.y | start.z);
    }
  }
  if (!__syncthreads_or(work)) return;
  __shared__ PrimStage st;
  const pf_primitive* prims = stage_prims(V, st);
  if (!work) return;
  const DevScene& S = V.scenes[s];
  auto ln_at = [&](uint32_t i) {
    return (i < 32 && !((mask >> i) & 1u)) ? 0.0f : V.plam[(size_t)k * V.prim_stride + i].x;
  };
  const float4 xs4 = V.cur.xs[k];
  const float w = xs4.w;
  const bool moves = w > 0.0f;
  const uint32_t n_prim = moves ? S.prim_count : 0u, n_sdf = moves ? S.sdf_count : 0u;
  const f3 xstar = xyz(xs4);
  const f3 vel = xyz(V.cur.v[k]);
  const float clock = V.clocks[s];
  uint32_t tx = (uint32_t)start.x, ty = (uint32_t)start.y, tz = (uint32_t)start.z;
  bool any = (start.x | start.y | start.z) != 0;
  for (uint32_t p = 0; p < n_prim; ++p) {
    const float ln = ln_at(p);
    if (!(ln > 0.0f)) continue;
    const pf_primitive& P = prims[p];
    float phi;
    f3 g;
    prim_sdf(P, xstar, clock, &phi, &g);
    const float gl = len(g);
    if (!(gl > 1e-6f)) continue;
    const f3 nrm = g / gl;
    const f3 rel = vel - prim_surface_velocity(P, xstar, clock);
    const f3 vt = rel - nrm * dot(nrm, rel);
    const float vtl = len(vt);
    if (vtl > 1e-6f) {
      const float change = fminf(P.velocity[3] * ln * w / S.dt, vtl);
      const f3 c = neg((vt / vtl) * change);
      tx += (uint32_t)to_ticks(c.x, S.vel_scale);
      ty += (uint32_t)to_ticks(c.y, S.vel_scale);
      tz += (uint32_t)to_ticks(c.z, S.vel_scale);
      any = true;
    }
  }
  // SDFCollider.ts:283-299 against a static surface
  for (uint32_t q = 0; q < n_sdf; ++q) {
    const float ln = ln_at(S.prim_count + q);
    if (!(ln > 0.0f)) continue;
    const DevSdf& G = V.sdfs[S.sdf_base + q];
    float phi;
    f3 g;
    sdf_sample(V.sdf_half, G, xstar, &phi, &g);
    const float gl = len(g);
    if (!(gl > 1e-6f)) continue;
    const f3 nrm = g / gl;
    const f3 vt = vel - nrm * dot(nrm, vel);
    const float vtl = len(vt);
    if (vtl > 1e-6f) {
      const float change = fminf(G.mu_k * ln * w / S.dt, vtl);
      const f3 c = neg((vt / vtl) * change);
      tx += (uint32_t)to_ticks(c.x, S.vel_scale);
      ty += (uint32_t)to_ticks(c.y, S.vel_scale);
      tz += (uint32_t)to_ticks(c.z, S.vel_scale);
      any = true;
    }
  }
  if (!any) return;
  bool sat = false;
  const f3 c = ticks_change((int)tx, (int)ty, (int)tz, S.vel_inv, &sat);
  V.cur.v[k] = with_w(vel + c, 0.0f);
  if (sat) atomicOr(V.flags + s * kNumFlags + FLAG_VEL, 1u);
}

// ---------------------------------------------------------------- cloth ----
// distance.ts:264-288 for one colour of constraints (no two share a particle).
__global__ void __launch_bounds__(kBlock) k_cloth(WorldView V, uint32_t begin, uint32_t end, uint32_t sub,
                                                  uint32_t it) {
  const uint32_t q = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= end) return;
  const DevScene& S = V.scenes[V.c_scene[q]];
  if (sub >= S.substeps || it >= S.iterations) return;
  const uint32_t i = V.inv[V.c_i[q]], j = V.inv[V.c_j[q]];
  const float4 xi = V.cur.xs[i], xj = V.cur.xs[j];
  const float wi = xi.w, wj = xj.w;
  const float ws = wi + wj;
  const f3 off = xyz(xi) - xyz(xj);
  const float l = len(off);
  if (ws <= 0.0f || l < 1e-12f) return;
  const f3 nrm = off / l;
  const float lc = V.c_lambda[q];
  const float at = V.c_comp[q] / (S.dt * S.dt);
  const float dl = (-(l - V.c_rest[q]) - at * lc) / (ws + at);
  V.cur.xs[i] = with_w(xyz(xi) + nrm * (wi * dl), wi);
  V.cur.xs[j] = with_w(xyz(xj) - nrm * (wj * dl), wj);
  V.c_lambda[q] = lc + dl;
}

// bending.ts:130-235: one colour of dihedral bending constraints (no two
// share a particle); the closed-form gradients of the signed angle
// theta = atan2((N1 x N2).E, (N1.N2)|E|) with E = p2 - p1,
// N1 = (p3 - p1) x (p3 - p2), N2 = (p4 - p2) x (p4 - p1), and the XPBD
// multiplier update (xpbd.ts:26-36).
__global__ void __launch_bounds__(kBlock) k_bend(WorldView V, uint32_t begin, uint32_t end, uint32_t sub, uint32_t it) {
  const uint32_t q = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= end) return;
  const DevScene& S = V.scenes[V.b_scene[q]];
  if (sub >= S.substeps || it >= S.iterations) return;
  const uint4 id = V.b_idx[q];
  const uint32_t i1 = V.inv[id.x], i2 = V.inv[id.y], i3 = V.inv[id.z], i4 = V.inv[id.w];
  const float4 p1 = V.cur.xs[i1], p2 = V.cur.xs[i2], p3 = V.cur.xs[i3], p4 = V.cur.xs[i4];
  const f3 x1 = xyz(p1), x2 = xyz(p2), x3 = xyz(p3), x4 = xyz(p4);
  const f3 E = x2 - x1;
  const float e2 = dot(E, E);
  if (e2 < 1e-24f) return;
  const float el = sqrtf(e2);
  const f3 a3 = x3 - x1, b3 = x3 - x2;
  const f3 n1 = cross(a3, b3);
  const f3 a4 = x4 - x2, b4 = x4 - x1;
  const f3 n2 = cross(a4, b4);
  const float n1s = dot(n1, n1), n2s = dot(n2, n2);
  if (n1s < 1e-24f || n2s < 1e-24f) return;
  const float st = dot(cross(n1, n2), E);
  const float ct = dot(n1, n2) * el;
  const float C = atan2f(st, ct) - V.b_rest[q];
  const f3 N1 = n1 / n1s, N2 = n2 / n2s;
  const f3 g3 = neg(N1 * el), g4 = neg(N2 * el);
  const float c31 = dot(b3, E) / el, c32 = dot(a4, E) / el;
  const float c41 = dot(a3, E) / el, c42 = dot(b4, E) / el;
  const f3 g1 = neg(N1 * c31 + N2 * c32);
  const f3 g2 = N1 * c41 + N2 * c42;
  const float w1 = p1.w, w2 = p2.w, w3 = p3.w, w4 = p4.w;
  const float sg = dot(g1, g1) * w1 + dot(g2, g2) * w2 + dot(g3, g3) * w3 + dot(g4, g4) * w4;
  if (sg <= 1e-30f) return;
  const float lc = V.b_lambda[q];
  const float at = V.cloth_par[V.b_cloth[q]].bend_compliance / (S.dt * S.dt);
  const float dl = (-C - at * lc) / (sg + at);
  V.cur.xs[i1] = with_w(x1 + g1 * (w1 * dl), w1);
  V.cur.xs[i2] = with_w(x2 + g2 * (w2 * dl), w2);
  V.cur.xs[i3] = with_w(x3 + g3 * (w3 * dl), w3);
  V.cur.xs[i4] = with_w(x4 + g4 * (w4 * dl), w4);
  V.b_lambda[q] = lc + dl;
}

// tether.ts:117-154: one colour of long-range attachments (no two share a
// free particle). Unilateral: slack inside the rest radius (lambda reset),
// otherwise the XPBD projection of the free particle onto the sphere about
// its pinned anchor, read at its predicted position.
__global__ void __launch_bounds__(kBlock) k_tether(WorldView V, uint32_t begin, uint32_t end, uint32_t sub,
                                                   uint32_t it) {
  const uint32_t q = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= end) return;
  const DevScene& S = V.scenes[V.t_scene[q]];
  if (sub >= S.substeps || it >= S.iterations) return;
  const uint4 r = V.t_rec[q];
  const uint32_t i = V.inv[r.x];
  const float4 xi = V.cur.xs[i];
  const float w = xi.w;
  if (w <= 0.0f) return;
  const f3 d = xyz(xi) - xyz(V.cur.xs[V.inv[r.y]]);
  const float l = len(d);
  const float rest = __uint_as_float(r.z);
  if (l <= rest) {
    V.t_lambda[q] = 0.0f;
    return;
  }
  if (l < 1e-12f) return;
  const float lc = V.t_lambda[q];
  const float at = __uint_as_float(r.w) / (S.dt * S.dt);
  const float dl = (-(l - rest) - at * lc) / (w + at);
  V.cur.xs[i] = with_w(xyz(xi) + (d / l) * (w * dl), w);
  V.t_lambda[q] = lc + dl;
}

// aero.ts:203-283: drag and lift of each incident triangle (Keckeisen et al.
// 2004), a third of each triangle's force per vertex, gathered per cloth
// particle (no scatter) from the committed positions and the velocities after
// the prediction; the sum moves the predicted position by dt^2 w F.
__global__ void __launch_bounds__(kBlock) k_aero(WorldView V, uint32_t begin, uint32_t end, uint32_t sub) {
  const uint32_t q = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= end) return;
  const uint2 rec = V.a_vtx[q];
  const uint32_t k = V.inv[rec.x];
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps) return;
  const float4 xs = V.cur.xs[k];
  const float w = xs.w;
  if (w <= 0.0f) return;
  const DevCloth& P = V.cloth_par[rec.y];
  const f3 wind = mk(P.wind[0], P.wind[1], P.wind[2]);
  const float drag = P.drag, lift = P.lift;
  f3 fsum = mk(0.0f, 0.0f, 0.0f);
  const uint32_t m1 = V.a_off[q + 1];
  for (uint32_t m = V.a_off[q]; m < m1; ++m) {
    const uint4 t = V.a_tri[m];
    const uint32_t s1 = V.inv[t.x], s2 = V.inv[t.y], s3 = V.inv[t.z];
    const f3 vrel = (xyz(V.cur.v[s1]) + xyz(V.cur.v[s2]) + xyz(V.cur.v[s3])) / 3.0f - wind;
    const float vrs = dot(vrel, vrel);
    if (!(vrs > 1e-12f)) continue;
    const f3 x1 = xyz(V.cur.x[s1]);
    const f3 nraw = cross(xyz(V.cur.x[s2]) - x1, xyz(V.cur.x[s3]) - x1);
    const float nms = dot(nraw, nraw);
    if (!(nms > 1e-12f)) continue;
    const float nm = sqrtf(nms);
    const float area = nm * 0.5f;
    const f3 nunit = nraw / nm;
    const f3 nbar = nunit * (dot(nunit, vrel) < 0.0f ? -1.0f : 1.0f);
    const f3 vhat = vrel / sqrtf(vrs);
    const f3 fdrag = neg(vhat * (drag * vrs * area * dot(nbar, vhat)));
    const f3 flift = cross(cross(nbar, vhat), vhat) * (lift * vrs * area);
    fsum = fsum + (fdrag + flift) / 3.0f;
  }
  V.cur.xs[k] = with_w(xyz(xs) + fsum * (S.dt * S.dt * w), w);
}

// ClothSystem.ts:264-277: the mean velocity of each cloth particle's edge
// neighbours, blended with its own (mix(v, mean, damping)).
__global__ void __launch_bounds__(kBlock) k_damp_mean(WorldView V, uint32_t begin, uint32_t end, uint32_t sub) {
  const uint32_t q = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= end) return;
  const uint2 rec = V.d_vtx[q];
  const uint32_t k = V.inv[rec.x];
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps) return;
  const float4 v = V.cur.v[k];
  const uint32_t m0 = V.d_off[q], m1 = V.d_off[q + 1];
  f3 sum = mk(0.0f, 0.0f, 0.0f);
  for (uint32_t m = m0; m < m1; ++m) sum = sum + xyz(V.cur.v[V.inv[V.d_nbr[m]]]);
  const f3 mean = sum / (float)max(m1 - m0, 1u);
  const float t = V.cloth_par[rec.y].damping;
  V.d_smooth[q] = with_w(xyz(v) * (1.0f - t) + mean * t, v.w);
}

// ClothSystem.ts:278-284: particles with inverse mass > 0 take the blend.
__global__ void __launch_bounds__(kBlock) k_damp_apply(WorldView V, uint32_t begin, uint32_t end, uint32_t sub) {
  const uint32_t q = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= end) return;
  const uint32_t k = V.inv[V.d_vtx[q].x];
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps || !(V.cur.x[k].w > 0.0f)) return;
  V.cur.v[k] = V.d_smooth[q];
}

// ---------------------------------------------------------- soft bodies ----
__device__ __forceinline__ bool group_active(const WorldView& V, uint32_t g, uint32_t rank, uint32_t sub,
                                             uint32_t it, const DevSoft** D, const DevScene** S) {
  *D = &V.softs[V.grp_soft[g]];
  *S = &V.scenes[(*D)->scene];
  return (*D)->rank == rank && sub < (*S)->substeps && it < (*S)->iterations;
}

// rotation.ts:297-314
__global__ void __launch_bounds__(kBlock) k_rot_predict(WorldView V, uint32_t sub) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_grp) return;
  const DevSoft& D = V.softs[V.grp_soft[g]];
  const DevScene& S = V.scenes[D.scene];
  if (sub >= S.substeps) return;
  const uint32_t i = V.grp[g];
  const float4 q = V.q[i];
  const f3 om = xyz(V.omega[i]);
  const float mag = len(om);
  if (mag < 1e-8f) {
    V.qp[i] = q;
    return;
  }
  const float half = mag * S.dt * 0.5f;
  float sh, ch;
  sincosf(half, &sh, &ch);
  const f3 sx = om * (sh / mag);
  const f3 qx = xyz(q);
  const f3 nx = qx * ch + sx * q.w + cross(sx, qx);
  V.qp[i] = with_w(nx, ch * q.w - dot(sx, qx));
}

// rotation.ts:316-343
__global__ void __launch_bounds__(kBlock) k_rot_advect(WorldView V, uint32_t sub) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_grp) return;
  const DevSoft& D = V.softs[V.grp_soft[g]];
  const DevScene& S = V.scenes[D.scene];
  if (sub >= S.substeps) return;
  const uint32_t i = V.grp[g];
  const float4 q = V.q[i];
  float4 qp = V.qp[i];
  const float dd = qp.x * qp.x + qp.y * qp.y + qp.z * qp.z + qp.w * qp.w;
  const float nrm = sqrtf(fmaxf(dd, 1e-12f));
  qp = make_float4(qp.x / nrm, qp.y / nrm, qp.z / nrm, qp.w / nrm);
  const f3 qi = mk(-q.x, -q.y, -q.z);
  const f3 qpx = xyz(qp);
  const f3 rpre = qpx * q.w + qi * qp.w + cross(qpx, qi);
  const float rwpre = qp.w * q.w - dot(qpx, qi);
  const float flip = rwpre < 0.0f ? -1.0f : 1.0f;
  const f3 rx = rpre * flip;
  const float rw = rwpre * flip;
  const float hs = len(rx);
  if (hs < 1e-8f) {
    V.omega[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  } else {
    const float angle = atan2f(hs, rw) * 2.0f;
    const f3 om = rx * ((angle / hs) / S.dt);
    const float sc = sqrtf(1.0e4f / fmaxf(dot(om, om), 1.0e4f));
    V.omega[i] = with_w(om * sc, 0.0f);
  }
  V.q[i] = qp;
}

// shapeMatchImplicit.ts:46-71 (the cluster's centre) and 100-217 (its moment
// matrix and rotation), one thread per cluster. The moment of a cluster reads
// only its own centre, so the thread forms the centre first, in CSR order as
// the reference's centre pass does, and keeps it in registers; the members'
// positions come back from cache for the moment.
__global__ void __launch_bounds__(kBlock) k_sm_moment(WorldView V, uint32_t rank, uint32_t sub, uint32_t it) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_grp) return;
  const DevSoft* D;
  const DevScene* S;
  if (!group_active(V, g, rank, sub, it, &D, &S)) return;
  const uint32_t i = V.grp[g];
  const uint32_t s = V.csr_off[i], e = V.csr_off[i + 1];
  f3 sum = mk(0.0f, 0.0f, 0.0f);
  for (uint32_t m = s; m < e; ++m) sum = sum + xyz(V.cur.xs[V.inv[V.csr_idx[m]]]);
  const float inv_cnt = 1.0f / (float)max(e - s, 1u);
  const f3 c = e == s ? mk(0.0f, 0.0f, 0.0f) : sum * inv_cnt;
  float a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const f3 cb = xyz(V.rest_c[i]);
  const float ai = D->ai;
  for (uint32_t m = s; m < e; ++m) {
    const uint32_t j = V.csr_idx[m];
    const float4 qj = V.qp[j];
    const float xx = qj.x * qj.x, yy = qj.y * qj.y, zz = qj.z * qj.z, xy = qj.x * qj.y, xz = qj.x * qj.z,
                yz = qj.y * qj.z, wx = qj.w * qj.x, wy = qj.w * qj.y, wz = qj.w * qj.z;
    a[0] += ai * (1.0f - (yy + zz) * 2.0f);
    a[1] += ai * ((xy - wz) * 2.0f);
    a[2] += ai * ((xz + wy) * 2.0f);
    a[3] += ai * ((xy + wz) * 2.0f);
    a[4] += ai * (1.0f - (xx + zz) * 2.0f);
    a[5] += ai * ((yz - wx) * 2.0f);
    a[6] += ai * ((xz - wy) * 2.0f);
    a[7] += ai * ((yz + wx) * 2.0f);
    a[8] += ai * (1.0f - (xx + yy) * 2.0f);
    const f3 xj = xyz(V.cur.xs[V.inv[j]]) - c;
    const f3 xt = xyz(V.rest[j]) - cb;
    a[0] += xj.x * xt.x;
    a[1] += xj.x * xt.y;
    a[2] += xj.x * xt.z;
    a[3] += xj.y * xt.x;
    a[4] += xj.y * xt.y;
    a[5] += xj.y * xt.z;
    a[6] += xj.z * xt.x;
    a[7] += xj.z * xt.y;
    a[8] += xj.z * xt.z;
  }
  float r[9];
  polar3(a, r);
  if (e == s) {
    r[0] = 1; r[1] = 0; r[2] = 0; r[3] = 0; r[4] = 1; r[5] = 0; r[6] = 0; r[7] = 0; r[8] = 1;
  }
  V.rot4[4 * (size_t)i + 0] = make_float4(r[0], r[1], r[2], c.x);
  V.rot4[4 * (size_t)i + 1] = make_float4(r[3], r[4], r[5], c.y);
  V.rot4[4 * (size_t)i + 2] = make_float4(r[6], r[7], r[8], c.z);
  V.rot4[4 * (size_t)i + 3] = make_float4(cb.x, cb.y, cb.z, V.rest[i].w);
}

// shapeMatchImplicit.ts:248-308 taken by member, with the accumulator's
// apply (accumulator.ts:148-178) for the particle. The reference scatters
// each cluster's corrections to its members as fixed-point ticks, integer
// sums whose order does not matter. Here a group of L lanes takes one
// particle (by id, from the list of cluster members; 32 / L particles per
// warp, L chosen per world from how many clusters hold a particle): each lane
// forms the corrections of clusters that hold it, term for term as the
// cluster would, and updates those pairs' multipliers (each pair belongs to
// one member); the lanes' tick sums are added across the group, and its first
// lane applies them to the particle's predicted position. No other group
// reads that position in this pass: the clusters' centres and rotations come
// from the passes before. Every lane of a warp reaches the shuffles: a lane
// past the last member, or whose member's body skips this pass, adds zero.
template <uint32_t L>
__global__ void __launch_bounds__(kBlock, 5) k_sm_gather(WorldView V, uint32_t rank, uint32_t sub, uint32_t it) {
  static_assert(L == 1 || L == 2 || L == 4 || L == 8 || L == 16 || L == 32,
                "lanes per member: a power of two dividing the warp");
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x % L;
  bool act = t / L < V.n_mem_ids;
  const DevSoft* D = nullptr;
  const DevScene* S = nullptr;
  uint32_t tx = 0, ty = 0, tz = 0, sj = 0;
  float4 xj = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  uint32_t j = 0, b = 0, e = 0, c0 = 0, c1 = 0;
  float4 rest4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (act) {
    // the member's own records are loaded beside its body and scene (they
    // do not depend on them), so the chains of dependent loads overlap
    j = __ldg(V.mem_ids + t / L);
    const uint32_t soft = V.mem_soft[j];
    b = V.mem_off[j];
    e = V.mem_off[j + 1];
    sj = V.inv[j];
    rest4 = V.rest[j];
    c0 = V.csr_off[j];
    c1 = V.csr_off[j + 1];
    D = &V.softs[soft];
    xj = V.cur.xs[sj];
    S = &V.scenes[D->scene];
    act = D->rank == rank && sub < S->substeps && it < S->iterations;
  }
  if (act) {
    const f3 rj = xyz(rest4);
    const float wj = xj.w;
    const float mj = fmaxf((float)(c1 - c0), 1.0f);
    const float dt2 = S->dt * S->dt;
    const float maxc2 = D->maxc2, scale = S->sb_scale;
    for (uint32_t q = b + lane; q < e; q += L) {
      const uint2 im = __ldg(V.mem + q);
      const uint32_t i = im.x, m = im.y;
      // the cluster's record: rotation rows with the centre, then the rest
      // centre and compliance (written by k_sm_moment this iteration)
      const float4 a0 = V.rot4[4 * (size_t)i], a1 = V.rot4[4 * (size_t)i + 1], a2 = V.rot4[4 * (size_t)i + 2],
                   a3 = V.rot4[4 * (size_t)i + 3];
      const f3 R0 = xyz(a0), R1 = xyz(a1), R2 = xyz(a2);
      const f3 c = mk(a0.w, a1.w, a2.w);
      const f3 cb = xyz(a3);
      const float at = a3.w / dt2;
      const f3 lo = xyz(V.pair_lambda[m]);
      const f3 rr = rj - cb;
      const f3 goal = mk(dot(R0, rr), dot(R1, rr), dot(R2, rr)) + c;
      const f3 C = xyz(xj) - goal;
      const float denom = wj + at;
      const f3 dl = (neg(C) - lo * at) / denom;
      V.pair_lambda[m] = with_w(lo + dl, 0.0f);
      const f3 dx = (dl * wj) / mj;
      const float sc = sqrtf(maxc2 / fmaxf(dot(dx, dx), maxc2));
      const f3 v = dx * sc;
      tx += (uint32_t)to_ticks(v.x, scale);
      ty += (uint32_t)to_ticks(v.y, scale);
      tz += (uint32_t)to_ticks(v.z, scale);
    }
  }
#pragma unroll
  for (uint32_t o = L / 2; o > 0; o >>= 1) {
    tx += __shfl_xor_sync(0xffffffffu, tx, o);
    ty += __shfl_xor_sync(0xffffffffu, ty, o);
    tz += __shfl_xor_sync(0xffffffffu, tz, o);
  }
  if (!act || lane != 0 || !(tx | ty | tz)) return;
  bool sat = false;
  const f3 ch = ticks_change((int)tx, (int)ty, (int)tz, S->sb_inv, &sat);
  V.cur.xs[sj] = with_w(xyz(xj) + ch, xj.w);
  if (sat) atomicOr(V.flags + D->scene * kNumFlags + FLAG_SOFT, 1u);
}

// shapeMatchImplicit.ts:325-401
__global__ void __launch_bounds__(kBlock) k_sm_qp(WorldView V, uint32_t rank, uint32_t sub, uint32_t it) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_grp) return;
  const DevSoft* D;
  const DevScene* S;
  if (!group_active(V, g, rank, sub, it, &D, &S)) return;
  const uint32_t i = V.grp[g];
  if (V.csr_off[i + 1] <= V.csr_off[i]) return;
  const float4 r0 = V.rot4[4 * (size_t)i], r1 = V.rot4[4 * (size_t)i + 1], r2 = V.rot4[4 * (size_t)i + 2];
  const float m00 = r0.x, m01 = r0.y, m02 = r0.z, m10 = r1.x, m11 = r1.y, m12 = r1.z, m20 = r2.x, m21 = r2.y,
              m22 = r2.z;
  const float tr = m00 + m11 + m22;
  float qx, qy, qz, qw;
  if (tr > 0.0f) {
    const float sq = 0.5f / sqrtf(tr + 1.0f);
    qw = 0.25f / sq;
    qx = (m21 - m12) * sq;
    qy = (m02 - m20) * sq;
    qz = (m10 - m01) * sq;
  } else if (m00 > m11 && m00 > m22) {
    const float sq = 2.0f * sqrtf(1.0f + m00 - m11 - m22);
    qw = (m21 - m12) / sq;
    qx = 0.25f * sq;
    qy = (m01 + m10) / sq;
    qz = (m02 + m20) / sq;
  } else if (m11 > m22) {
    const float sq = 2.0f * sqrtf(1.0f + m11 - m00 - m22);
    qw = (m02 - m20) / sq;
    qx = (m01 + m10) / sq;
    qy = 0.25f * sq;
    qz = (m12 + m21) / sq;
  } else {
    const float sq = 2.0f * sqrtf(1.0f + m22 - m00 - m11);
    qw = (m10 - m01) / sq;
    qx = (m02 + m20) / sq;
    qy = (m12 + m21) / sq;
    qz = 0.25f * sq;
  }
  const float4 q0 = V.q[i];
  const float d = q0.x * qx + q0.y * qy + q0.z * qz + q0.w * qw;
  const float fl = d < 0.0f ? -1.0f : 1.0f;
  V.qp[i] = make_float4(qx * fl, qy * fl, qz * fl, qw * fl);
}

// shapeMatch.ts:53-229: one 256-thread block per body reduces the centre of
// mass and A = sum m x r^T (strided partial sums, then a tree), and thread 0
// takes the polar decomposition.
__global__ void __launch_bounds__(256) k_body_frame(WorldView V, uint32_t rank, uint32_t sub, uint32_t it,
                                                    uint32_t require_global) {
  const uint32_t b = blockIdx.x;
  if (b >= V.n_bodies) return;
  const DevBody B = V.bodies[b];
  const DevSoft& D = V.softs[B.soft];
  const DevScene& S = V.scenes[B.scene];
  if (D.rank != rank || sub >= S.substeps || it >= S.iterations) return;
  if (require_global && D.local) return;
  __shared__ float4 s4[256];
  __shared__ float sr[9][256];
  const uint32_t t = threadIdx.x;
  float4 acc = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  float r[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (uint32_t li = t; li < B.count; li += 256) {
    const uint32_t id = B.start + li;
    const float mi = V.weights[id];
    const f3 xi = xyz(V.cur.xs[V.inv[id]]);
    acc.x += xi.x * mi;
    acc.y += xi.y * mi;
    acc.z += xi.z * mi;
    acc.w += mi;
    const f3 xw = xi * mi;
    const f3 ri = xyz(V.rest[id]);
    r[0] += ri.x * xw.x; r[1] += ri.y * xw.x; r[2] += ri.z * xw.x;
    r[3] += ri.x * xw.y; r[4] += ri.y * xw.y; r[5] += ri.z * xw.y;
    r[6] += ri.x * xw.z; r[7] += ri.y * xw.z; r[8] += ri.z * xw.z;
  }
  s4[t] = acc;
  for (int m = 0; m < 9; ++m) sr[m][t] = r[m];
  __syncthreads();
  for (uint32_t st = 128; st > 0; st >>= 1) {
    if (t < st) {
      const float4 o = s4[t + st];
      s4[t] = make_float4(s4[t].x + o.x, s4[t].y + o.y, s4[t].z + o.z, s4[t].w + o.w);
      for (int m = 0; m < 9; ++m) sr[m][t] += sr[m][t + st];
    }
    __syncthreads();
  }
  if (t == 0) {
    const float4 tot = s4[0];
    V.body_c[b] = make_float4(tot.x / tot.w, tot.y / tot.w, tot.z / tot.w, 0.0f);
    float a[9], rr[9];
    for (int m = 0; m < 9; ++m) a[m] = sr[m][0];
    polar3(a, rr);
    V.body_r[3 * b + 0] = make_float4(rr[0], rr[1], rr[2], 0.0f);
    V.body_r[3 * b + 1] = make_float4(rr[3], rr[4], rr[5], 0.0f);
    V.body_r[3 * b + 2] = make_float4(rr[6], rr[7], rr[8], 0.0f);
  }
}

// shapeMatch.ts:277-351
__global__ void __launch_bounds__(256) k_global_apply(WorldView V, uint32_t rank, uint32_t sub, uint32_t it) {
  const uint32_t b = blockIdx.x;
  if (b >= V.n_bodies) return;
  const DevBody B = V.bodies[b];
  const DevSoft& D = V.softs[B.soft];
  const DevScene& S = V.scenes[B.scene];
  if (D.local || D.rank != rank || sub >= S.substeps || it >= S.iterations) return;
  const f3 R0 = xyz(V.body_r[3 * b]), R1 = xyz(V.body_r[3 * b + 1]), R2 = xyz(V.body_r[3 * b + 2]);
  const f3 c = xyz(V.body_c[b]);
  const float at = B.compliance / (S.dt * S.dt);
  for (uint32_t li = threadIdx.x; li < B.count; li += 256) {
    const uint32_t id = B.start + li;
    const uint32_t sl = V.inv[id];
    const f3 ri = xyz(V.rest[id]);
    const f3 goal = mk(dot(R0, ri), dot(R1, ri), dot(R2, ri)) + c;
    const float4 xs = V.cur.xs[sl];
    const f3 C = xyz(xs) - goal;
    const f3 lo = xyz(V.lambda_g[id]);
    const f3 dl = (neg(C) - lo * at) / (xs.w + at);
    V.lambda_g[id] = with_w(lo + dl, 0.0f);
    V.cur.xs[sl] = with_w(xyz(xs) + dl * xs.w, xs.w);
  }
}

// Positions by particle index for read-back: one thread per id.
__global__ void __launch_bounds__(kBlock) k_gather_positions(WorldView V, const uint64_t* __restrict__ prefix,
                                                             float4* __restrict__ out) {
  const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= V.n) return;
  const uint32_t s = V.chunk_scene[id >> 8];
  const DevScene& S = V.scenes[s];
  const uint32_t local = id - S.seg_start;
  if (local >= S.cap) return;
  const float4 x = V.cur.x[V.inv[id]];
  out[prefix[s] + local] = make_float4(x.x, x.y, x.z, 0.0f);
}

// FluidSystem.ts:248-253: the impulse accumulator's apply over the fluid's
// range, into the velocity and (times dt) the predicted position.
__global__ void __launch_bounds__(kBlock) k_imp_apply(WorldView V, uint32_t rank, uint32_t sub) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_fchunk * kSegAlign) return;
  const uint32_t k = chunk_slot(V.fchunk, g);  // slots of the scenes with a fluid
  const uint32_t f = tag_fluid(V.cur.tag[k]);
  if (!f) return;
  const DevFluid& F = V.fluids[f - 1];
  if (F.rank != rank || !(F.has_st || F.has_ad)) return;
  const uint32_t s = scene_index(V, k);
  const DevScene& S = V.scenes[s];
  if (sub >= S.substeps) return;
  const int4 t = V.acc_imp[k];
  V.acc_imp[k] = make_int4(0, 0, 0, 0);
  bool sat = false;
  const f3 c = ticks_change(t.x, t.y, t.z, F.imp_inv, &sat);
  const float4 v = V.cur.v[k];
  V.cur.v[k] = make_float4(v.x + c.x, v.y + c.y, v.z + c.z, v.w);
  const float4 x = V.cur.xs[k];
  const f3 d = c * S.dt;
  V.cur.xs[k] = make_float4(x.x + d.x, x.y + d.y, x.z + d.z, x.w);
  if (sat) atomicOr(V.flags + s * kNumFlags + FLAG_VEL, 1u);
}

// Fresh slot maps (ids = inv = identity) and identity orientations.
__global__ void __launch_bounds__(kBlock) k_init_slots(uint32_t* __restrict__ ids, uint32_t* __restrict__ inv,
                                                       float4* __restrict__ q, float4* __restrict__ qp, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  ids[i] = i;
  inv[i] = i;
  if (q) {
    q[i] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    qp[i] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
  }
}

// Dynamic state of one scene from another world, by particle index, written
// the way build() writes a spec's state (x* = x, q* = q, zero w lanes).
__global__ void __launch_bounds__(kBlock) k_import_scene(WorldView V, uint32_t seg, uint32_t cap,
                                                         const float4* __restrict__ sx, const float4* __restrict__ sv,
                                                         const float* __restrict__ sbv, const uint32_t* __restrict__ sinv,
                                                         uint32_t sseg, const float4* __restrict__ sq,
                                                         const float4* __restrict__ som) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cap) return;
  const uint32_t from = sinv[sseg + i];
  const float4 x = sx[from];
  const float4 v = sv[from];
  V.cur.x[seg + i] = x;
  V.cur.xs[seg + i] = x;
  V.cur.v[seg + i] = make_float4(v.x, v.y, v.z, 0.0f);
  V.cur.bv[seg + i] = sbv[from];
  if (V.q) {
    const float4 q = sq ? sq[sseg + i] : make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    const float4 w = som ? som[sseg + i] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    V.q[seg + i] = q;
    V.qp[seg + i] = q;
    V.omega[seg + i] = make_float4(w.x, w.y, w.z, 0.0f);
  }
}

// Kernel launches issued since the counter was last reset (per step).
thread_local uint64_t t_launches = 0;

template <typename K, typename... A>
void launch_slots(K kernel, uint32_t n, cudaStream_t st, A... args) {
  if (n == 0) return;
  kernel<<<div_up(n, kBlock), kBlock, 0, st>>>(args...);
  ++t_launches;
}

size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

// The slot neighbour passes use no shared memory and gather their
// neighbours' records through L1: each asks for the largest L1 (a hint the
// runtime may round), once per device, outside any stream capture.
template <typename K>
cudaError_t prefer_l1(K kernel) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxL1);
}
template <uint32_t U>
cudaError_t prefer_l1_depth() {
  cudaError_t e = cudaSuccess;
  auto on = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
  on(prefer_l1(k_s_neighbors<U, false, false>));
  on(prefer_l1(k_s_neighbors<U, true, false>));
  on(prefer_l1(k_s_neighbors<U, false, true>));
  on(prefer_l1(k_s_neighbors<U, true, true>));
  on(prefer_l1(k_s_lambda<U>));
  on(prefer_l1(k_s_delta<U, false>));
  on(prefer_l1(k_s_delta<U, true>));
  on(prefer_l1(k_s_xsph<U, false>));
  on(prefer_l1(k_s_xsph<U, true>));
  return e;
}
cudaError_t slot_kernels_prepare() {
  static std::mutex m;
  static std::set<int> ready;
  int dev = 0;
  if (cudaError_t e = cudaGetDevice(&dev); e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(m);
  if (ready.count(dev)) return cudaSuccess;
  for (cudaError_t e : {prefer_l1_depth<2>(), prefer_l1_depth<4>(), prefer_l1_depth<8>()})
    if (e != cudaSuccess) return e;
  ready.insert(dev);
  return cudaSuccess;
}

}  // namespace

// ================================================================ World ====

void World::drop_graphs() {
  for (auto& g : graph_)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
}

World::~World() {
  drop_graphs();
  if (read_stream_) {
    cudaStreamSynchronize(read_stream_);
    cudaStreamDestroy(read_stream_);
  }
  for (int b = 0; b < 2; ++b) {
    if (ev_gathered_[b]) cudaEventDestroy(ev_gathered_[b]);
    if (ev_read_[b]) cudaEventDestroy(ev_read_[b]);
  }
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  for (auto& e : ev_params_)
    if (e) cudaEventDestroy(e);
  for (auto& e : ev_bounds_)
    if (e) cudaEventDestroy(e);
  if (h_pinned_bbox_) cudaFreeHost(h_pinned_bbox_);
  // the device memory goes back to the pool in stream order, once this
  // world's streams are idle: no other stream touches it after that
  if (side_stream_) cudaStreamSynchronize(side_stream_);
  if (stream_) cudaStreamSynchronize(stream_);
  dev_free(grid_arena_, stream_);
  dev_free(sort_arena_, stream_);
  dev_free(arena_, stream_);
  if (ev_fork_) cudaEventDestroy(ev_fork_);
  if (ev_join_) cudaEventDestroy(ev_join_);
  if (side_stream_) cudaStreamDestroy(side_stream_);
  if (stream_) cudaStreamDestroy(stream_);
  if (h_pinned_scenes_) cudaFreeHost(h_pinned_scenes_);
  if (h_pinned_prims_) cudaFreeHost(h_pinned_prims_);
  if (h_pinned_plane4_) cudaFreeHost(h_pinned_plane4_);
  if (h_pinned_sdfs_) cudaFreeHost(h_pinned_sdfs_);
  if (h_pinned_cloth_) cudaFreeHost(h_pinned_cloth_);
}

WorldView World::view(uint32_t parity) const {
  WorldView v = base_;
  v.nbr_wide_only = tune_.nbr_wide;
  v.cur = buf_[parity & 1];
  v.nxt = buf_[(parity & 1) ^ 1];
  return v;
}

uint64_t World::particle_substeps_per_step() const {
  uint64_t t = 0;
  for (auto* s : specs_) t += (uint64_t)s->cap * s->loop.substeps;
  return t;
}

namespace {
struct Carver {
  char* base;
  size_t off = 0;
  template <typename T>
  T* take(size_t count) {
    T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += al256(sizeof(T) * std::max<size_t>(count, 1));
    return p;
  }
};

float f32(double v) { return static_cast<float>(v); }

uint32_t bits_of(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}
}  // namespace

// Kernel-side view of an SDF collider: R from the unit quaternion (the
// rotation part of three's Matrix4.makeRotationFromQuaternion, computed in
// double and rounded to f32 as a mat3 uniform would be), its transpose, and
// the reciprocals SDFCollider.ts:115-128 precomputes.
DevSdf make_dev_sdf(const SdfSpec& g, uint32_t data_off) {
  DevSdf d{};
  for (int a = 0; a < 3; ++a) {
    d.res[a] = g.res[a];
    d.origin[a] = g.origin[a];
    d.voxel[a] = g.voxel[a];
    d.inv_voxel[a] = (float)(1.0 / (double)g.voxel[a]);
    d.position[a] = g.position[a];
  }
  d.data_off = data_off;
  const double x = g.rot_q[0], y = g.rot_q[1], z = g.rot_q[2], w = g.rot_q[3];
  const double R[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w * z),     2 * (x * z + w * y),
                       2 * (x * y + w * z),     1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                       2 * (x * z - w * y),     2 * (y * z + w * x),     1 - 2 * (x * x + y * y)};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      d.rot[3 * r + c] = (float)R[3 * r + c];
      d.inv_rot[3 * r + c] = (float)R[3 * c + r];
    }
  d.scale = g.scale;
  d.inv_scale = (float)(1.0 / (double)g.scale);
  d.thickness = g.thickness;
  d.mu_s = g.mu_s;
  d.mu_k = g.mu_k;
  return d;
}

pf_status World::build(const std::vector<SceneSpec*>& specs, bool use_graph, bool plan_only,
                       const std::vector<uint8_t>* skip_state) {
  specs_ = specs;
  use_graph_ = use_graph;
  const uint32_t K = (uint32_t)specs.size();
  if (K == 0) return fail(PF_ERR_INVALID, "SimLoop: no scenes to build");
  // ---- segments, grids, materials -----------------------------------
  uint64_t slot = 0, cell = 0;
  h_scenes_.assign(K, DevScene{});
  h_fluids_.clear();
  h_bnds_.clear();
  h_softs_.clear();
  h_bodies_.clear();
  h_prims_.clear();
  h_sdfs_.clear();
  uint64_t sdf_voxels = 0;
  max_rank_ = max_sub_ = max_iter_ = 0;
  prim_stride_ = 1;
  for (uint32_t s = 0; s < K; ++s) {
    const SceneSpec& sp = *specs[s];
    DevScene& S = h_scenes_[s];
    S.seg_start = (uint32_t)slot;
    S.cap = sp.cap;
    S.seg_end = (uint32_t)(slot + ((sp.cap + kSegAlign - 1) / kSegAlign) * kSegAlign);
    slot = S.seg_end;
    S.substeps = sp.loop.substeps ? sp.loop.substeps : 4;
    S.iterations = sp.loop.iterations;
    S.substeps_f = (float)S.substeps;
    S.init_pending = sp.initialized ? 0u : 1u;
    S.gx = sp.loop.gravity[0];
    S.gy = sp.loop.gravity[1];
    S.gz = sp.loop.gravity[2];
    S.radius = f32(sp.radius);
    S.pos_scale = f32(std::floor(1073741824.0 / 10.0));
    S.pos_inv = f32(1.0 / std::floor(1073741824.0 / 10.0));
    S.vel_scale = f32(std::floor(1073741824.0 / 50.0));
    S.vel_inv = f32(1.0 / std::floor(1073741824.0 / 50.0));
    S.sb_scale = S.pos_scale;
    S.sb_inv = S.pos_inv;
    max_sub_ = std::max(max_sub_, S.substeps);
    max_iter_ = std::max(max_iter_, S.iterations);
    max_rank_ = std::max(max_rank_, (uint32_t)sp.materials.size());
    // particle contacts (loop.ts:148-160, 388-417)
    S.contact = sp.loop.contact ? 1u : 0u;
    S.max_contacts = sp.loop.max_contacts ? sp.loop.max_contacts : (uint32_t)std::min<uint64_t>(8ull * sp.cap, 0xffffffffull);
    S.c_mus = sp.loop.contact_mu_s >= 0 ? sp.loop.contact_mu_s : 0.5f;
    S.c_muk = sp.loop.contact_mu_k >= 0 ? sp.loop.contact_mu_k : 0.4f;
    S.c_dist = f32(2.0 * sp.radius);
    {
      const double cr = 2.0 * sp.radius * kContactRadiusExpansion;
      S.c_cand2 = f32(cr * cr);
    }
    any_contact_ = any_contact_ || S.contact;
    any_multi_fluid_ = any_multi_fluid_ || sp.fluids.size() > 1;
    S.homog = 0;
    S.homog_mass = 0.0f;
    if (sp.fluids.size() == 1 && sp.fluids[0].range.start == 0 && sp.fluids[0].range.count == sp.cap &&
        sp.fluids[0].bnd.empty() && sp.cap > 0) {
      const float w0 = sp.inv_mass[0];
      bool same = w0 > 0.0f;
      for (uint32_t i = 1; i < sp.cap && same; ++i) same = sp.inv_mass[i] == w0;
      if (same) {
        S.homog = 1;
        S.homog_mass = 1.0f / w0;  // the mass code_mass gives every neighbour
      }
    }
    // grid: one grid for every neighbour query, sized for the widest
    double h = S.contact ? 2.0 * sp.radius * kContactRadiusExpansion : 0.0;
    for (auto& f : sp.fluids) h = std::max(h, f.h);
    S.has_grid = h > 0;
    if (S.has_grid) {
      const float cs = f32(h);
      S.cell = cs;
      S.ox = sp.loop.hash_origin[0];
      S.oy = sp.loop.hash_origin[1];
      S.oz = sp.loop.hash_origin[2];
      double mn[3], mx[3];
      bool auto_bounds = false;
      for (int a = 0; a < 3; ++a) {
        mn[a] = sp.loop.grid_min[a];
        mx[a] = sp.loop.grid_max[a];
        auto_bounds = auto_bounds || !(mx[a] > mn[a]);
      }
      if (auto_bounds && sp.bounds_resolved) {
        for (int a = 0; a < 3; ++a) {
          mn[a] = sp.grid_lo[a];
          mx[a] = sp.grid_hi[a];
        }
      } else if (auto_bounds) {
        for (int a = 0; a < 3; ++a) {
          mn[a] = 1e30;
          mx[a] = -1e30;
        }
        for (uint32_t i = 0; i < sp.cap; ++i)
          for (int a = 0; a < 3; ++a) {
            mn[a] = std::min(mn[a], (double)sp.pos4[4 * i + a]);
            mx[a] = std::max(mx[a], (double)sp.pos4[4 * i + a]);
          }
        // a window four times the initial extent per axis (at least 16
        // cells more), centred on the particles: it moves with them each
        // substep, so it clamps only once the particles spread wider than it
        double ext[3], cells_w = 1.0;
        for (int a = 0; a < 3; ++a) {
          ext[a] = std::max(4.0 * (mx[a] - mn[a]), (mx[a] - mn[a]) + 16.0 * h);
          cells_w *= ext[a] / h + 5.0;
        }
        // at most 2^24 cells of window: shrink it evenly past that
        const double shrink = cells_w > double(1u << 24) ? std::cbrt(double(1u << 24) / cells_w) : 1.0;
        for (int a = 0; a < 3; ++a) {
          const double c = 0.5 * (mn[a] + mx[a]), half = 0.5 * std::max(ext[a] * shrink, mx[a] - mn[a]);
          mn[a] = c - half;
          mx[a] = c + half;
        }
        if (!plan_only) {
          SceneSpec& w = *specs[s];
          w.bounds_resolved = true;
          for (int a = 0; a < 3; ++a) {
            w.grid_lo[a] = mn[a];
            w.grid_hi[a] = mx[a];
          }
        }
      }
      const double org[3] = {S.ox, S.oy, S.oz};
      uint64_t cells = 1;
      for (int a = 0; a < 3; ++a) {
        const int64_t lo = (int64_t)std::floor((mn[a] - org[a]) / cs) - 2;
        const int64_t hi = (int64_t)std::floor((mx[a] - org[a]) / cs) + 2;
        S.lo[a] = (int32_t)lo;
        S.lo0[a] = (int32_t)lo;
        S.dims[a] = (uint32_t)(hi - lo + 1);
        cells *= S.dims[a];
      }
      if (cells > (1ull << 27))
        return fail(PF_ERR_INVALID, "SimLoop: neighbour grid over " + std::to_string(cells) +
                                        " cells; give tighter grid bounds");
      S.cells = (uint32_t)cells;
      // the neighbour walk prunes a cell only when its box, widened by this
      // slack (far above the f32 rounding of cell_of and of the box edges),
      // is out of reach
      double big = 0;
      for (int a = 0; a < 3; ++a)
        big = std::max(big, std::fabs(org[a]) + std::max(std::fabs((double)S.lo[a]),
                                                         std::fabs((double)S.lo[a] + S.dims[a])) * cs);
      S.prune_slack = f32(big * (1.0 / 65536.0) + 1e-9);
    } else {
      S.cells = sp.cap;
    }
    S.cell_base = (uint32_t)cell;
    cell += (uint64_t)S.cells + 1;
    // primitives
    S.prim_base = (uint32_t)h_prims_.size();
    S.prim_count = (uint32_t)sp.prims.size();
    for (auto& p : sp.prims) h_prims_.push_back(p);
    S.sdf_base = (uint32_t)h_sdfs_.size();
    S.sdf_count = (uint32_t)sp.sdfs.size();
    for (auto& g : sp.sdfs) {
      h_sdfs_.push_back(make_dev_sdf(g, (uint32_t)sdf_voxels));
      sdf_voxels += g.half.size();
    }
    prim_stride_ = std::max(prim_stride_, S.prim_count + S.sdf_count);
    // fluids
    S.fluid_first = (uint32_t)h_fluids_.size();
    S.fluid_count = (uint32_t)sp.fluids.size();
    S.soft_local_ranks = 0;
    for (uint32_t r = 0; r < sp.materials.size(); ++r) {
      const MatKind kind = sp.materials[r].first;
      const uint32_t idx = sp.materials[r].second;
      if (kind == MAT_FLUID) {
        const FluidSpec& fs = sp.fluids[idx];
        DevFluid F{};
        F.scene = s;
        F.rank = r;
        F.rho0 = f32(fs.rho0);
        F.inv_rho0 = 1.0f / F.rho0;
        F.volume = f32(fs.spacing * fs.spacing * fs.spacing);
        F.h = f32(fs.h);
        F.hsq = f32(fs.h * fs.h);
        F.poly6 = f32(315.0 / (64.0 * M_PI * std::pow(fs.h, 9)));
        F.spiky = f32(45.0 / (M_PI * std::pow(fs.h, 6)));
        F.compliance = f32(fs.compliance);
        F.c_xsph = f32(fs.viscosity);
        F.has_visc = fs.has_visc ? 1u : 0u;
        F.has_vort = fs.has_vort ? 1u : 0u;
        F.vort_eps = f32(fs.vorticity);
        F.has_st = fs.has_st ? 1u : 0u;
        F.has_ad = fs.has_ad ? 1u : 0u;
        F.gamma = f32(fs.surface_tension);
        F.beta = f32(fs.adhesion);
        F.mass = f32(fs.rho0 * fs.spacing * fs.spacing * fs.spacing);
        F.coh_coef = f32(32.0 / (M_PI * std::pow(fs.h, 9)));
        F.coh_h6_64 = f32(std::pow(fs.h, 6) / 64.0);
        F.adh_coef = f32(0.007 / std::pow(fs.h, 3.25));
        F.adh_m4h = f32(-4.0 / fs.h);
        F.adh_2h = f32(2.0 * fs.h);
        F.range_end = S.seg_start + fs.range.start + fs.range.count;
        F.imp_scale = S.vel_scale;
        F.imp_inv = S.vel_inv;
        F.bnd_first = (uint32_t)h_bnds_.size();
        F.bnd_count = (uint32_t)fs.bnd.size();
        uint32_t lo = UINT32_MAX, hi = 0;
        for (size_t b = 0; b < fs.bnd.size(); ++b) {
          DevBoundary B{};
          B.start = S.seg_start + fs.bnd[b].start;
          B.count = fs.bnd[b].count;
          B.fluid = (uint32_t)h_fluids_.size();
          B.is_static = fs.bnd_static[b];
          lo = std::min(lo, B.start);
          hi = std::max(hi, B.start + B.count);
          h_bnds_.push_back(B);
          any_static_bnd_ = any_static_bnd_ || B.is_static;
          any_dyn_bnd_ = any_dyn_bnd_ || !B.is_static;
        }
        F.react_lo = fs.bnd.empty() ? 0 : lo;
        F.react_hi = fs.bnd.empty() ? 0 : hi;
        any_react_ = any_react_ || !fs.bnd.empty();
        F.react_scale = S.pos_scale;
        F.react_inv = S.pos_inv;
        any_fluid_ = true;
        any_visc_ = any_visc_ || fs.has_visc;
        any_vort_ = any_vort_ || fs.has_vort;
        any_imp_ = any_imp_ || fs.has_st || fs.has_ad;
        h_fluids_.push_back(F);
      } else if (kind == MAT_SOFT) {
        const SoftSpec& ss = sp.softs[idx];
        DevSoft D{};
        D.scene = s;
        D.rank = r;
        D.local = ss.local ? 1u : 0u;
        D.ai = f32(sp.radius * sp.radius / 5.0);
        const double maxc = 5.0 * sp.radius;
        D.maxc2 = f32(maxc * maxc);
        const uint32_t di = (uint32_t)h_softs_.size();
        h_softs_.push_back(D);
        for (auto& b : ss.bodies) {
          DevBody Bd{};
          Bd.scene = s;
          Bd.soft = di;
          Bd.start = S.seg_start + b.range.start;
          Bd.count = b.range.count;
          Bd.compliance = f32(b.compliance);
          h_bodies_.push_back(Bd);
        }
        if (ss.local) {
          S.soft_local_ranks |= 1u << r;
          any_soft_local_ = true;
        } else {
          any_soft_global_ = true;
        }
      }
    }
    any_grid_ = any_grid_ || S.has_grid;
    any_prims_ = any_prims_ || S.prim_count > 0 || S.sdf_count > 0;
    // colliders fuse into the last material's pass when that is a fluid
    S.collide_rank1 = 0;
    if (S.prim_count + S.sdf_count > 0 || S.contact) {
      // contact pairs are solved after every material and before the
      // colliders, so a scene with contacts keeps its collider pass apart
      if (!S.contact && !sp.materials.empty() && sp.materials.back().first == MAT_FLUID)
        S.collide_rank1 = (uint32_t)sp.materials.size();
      else
        any_unfused_prims_ = true;
    }
  }
  if (max_rank_ > 32) return fail(PF_ERR_INVALID, "SimLoop: at most 32 materials per scene");
  refresh_planes(-1);
  // The side stream applies when every scene that holds cloth, or whose
  // colliders run in their own pass, has cloth materials only.
  {
    bool any_side = false, ok = true;
    for (uint32_t s = 0; s < K; ++s) {
      const SceneSpec& sp = *specs[s];
      bool cloth_only = true, has_cloth = false;
      for (auto& m : sp.materials) {
        cloth_only = cloth_only && m.first == MAT_CLOTH;
        has_cloth = has_cloth || m.first == MAT_CLOTH;
      }
      const bool unfused = (h_scenes_[s].prim_count + h_scenes_[s].sdf_count > 0 || h_scenes_[s].contact) &&
                           h_scenes_[s].collide_rank1 == 0;
      if (has_cloth || unfused) {
        ok = ok && cloth_only;
        any_side = true;
      }
    }
    // only worth a second stream when other scenes run alongside
    side_ok_ = ok && any_side && (any_fluid_ || !h_softs_.empty());
  }
  n_ = (uint32_t)slot;
  cells_ = (uint32_t)cell;
  // ---- cloth parameters, one record per cloth material -------------------
  h_cloth_par_.clear();
  cloth_par_of_.assign(K, {});
  for (uint32_t s = 0; s < K; ++s) {
    const SceneSpec& sp = *specs[s];
    cloth_par_of_[s].assign(sp.materials.size(), -1);
    for (uint32_t r = 0; r < sp.materials.size(); ++r) {
      if (sp.materials[r].first != MAT_CLOTH) continue;
      const ClothSpec& cl = sp.cloths[sp.materials[r].second];
      DevCloth P{};
      for (int a = 0; a < 3; ++a) P.wind[a] = cl.wind[a];
      P.drag = cl.drag;
      P.lift = cl.lift;
      P.damping = cl.damping;
      P.bend_compliance = cl.bend_compliance;
      cloth_par_of_[s][r] = (int32_t)h_cloth_par_.size();
      h_cloth_par_.push_back(P);
    }
  }
  cloth_par_dirty_ = false;
  // ---- cloth constraints by (rank, colour) ----------------------------
  std::vector<uint32_t> ci, cj, csc;
  std::vector<float> crest, ccomp;
  cloth_ranges_.assign(max_rank_, {});
  for (uint32_t r = 0; r < max_rank_; ++r) {
    uint32_t ncol = 0;
    for (uint32_t s = 0; s < K; ++s) {
      const SceneSpec& sp = *specs[s];
      if (r < sp.materials.size() && sp.materials[r].first == MAT_CLOTH)
        ncol = std::max(ncol, (uint32_t)sp.cloths[sp.materials[r].second].colors.size());
    }
    for (uint32_t c = 0; c < ncol; ++c) {
      const uint32_t begin = (uint32_t)ci.size();
      for (uint32_t s = 0; s < K; ++s) {
        const SceneSpec& sp = *specs[s];
        if (!(r < sp.materials.size() && sp.materials[r].first == MAT_CLOTH)) continue;
        const ClothSpec& cl = sp.cloths[sp.materials[r].second];
        if (c >= cl.colors.size()) continue;
        const uint32_t base = h_scenes_[s].seg_start;
        for (uint32_t q : cl.colors[c]) {
          ci.push_back(base + cl.pairs[2 * q]);
          cj.push_back(base + cl.pairs[2 * q + 1]);
          crest.push_back(cl.rest[q]);
          ccomp.push_back(cl.compliance);
          csc.push_back(s);
        }
      }
      cloth_ranges_[r].push_back({begin, (uint32_t)ci.size()});
    }
  }
  // ---- cloth bending constraints by (rank, colour) ---------------------
  std::vector<uint4> bidx;
  std::vector<float> brest;
  std::vector<uint32_t> bsc, bcl;
  bend_ranges_.assign(max_rank_, {});
  for (uint32_t r = 0; r < max_rank_; ++r) {
    uint32_t ncol = 0;
    for (uint32_t s = 0; s < K; ++s) {
      const SceneSpec& sp = *specs[s];
      if (r < sp.materials.size() && sp.materials[r].first == MAT_CLOTH)
        ncol = std::max(ncol, (uint32_t)sp.cloths[sp.materials[r].second].bend_colors.size());
    }
    for (uint32_t c = 0; c < ncol; ++c) {
      const uint32_t begin = (uint32_t)bidx.size();
      for (uint32_t s = 0; s < K; ++s) {
        const SceneSpec& sp = *specs[s];
        if (!(r < sp.materials.size() && sp.materials[r].first == MAT_CLOTH)) continue;
        const ClothSpec& cl = sp.cloths[sp.materials[r].second];
        if (c >= cl.bend_colors.size()) continue;
        const uint32_t base = h_scenes_[s].seg_start;
        for (uint32_t q : cl.bend_colors[c]) {
          const uint32_t* t = cl.bend.data() + 4ull * q;
          bidx.push_back(make_uint4(base + t[0], base + t[1], base + t[2], base + t[3]));
          brest.push_back(cl.bend_rest[q]);
          bcl.push_back((uint32_t)cloth_par_of_[s][r]);
          bsc.push_back(s);
        }
      }
      bend_ranges_[r].push_back({begin, (uint32_t)bidx.size()});
    }
  }
  // ---- cloth tethers by (rank, colour) -----------------------------------
  std::vector<uint4> trec;
  std::vector<uint32_t> tsc;
  teth_ranges_.assign(max_rank_, {});
  for (uint32_t r = 0; r < max_rank_; ++r) {
    uint32_t ncol = 0;
    for (uint32_t s = 0; s < K; ++s) {
      const SceneSpec& sp = *specs[s];
      if (r < sp.materials.size() && sp.materials[r].first == MAT_CLOTH)
        ncol = std::max(ncol, (uint32_t)sp.cloths[sp.materials[r].second].tether_colors.size());
    }
    for (uint32_t c = 0; c < ncol; ++c) {
      const uint32_t begin = (uint32_t)trec.size();
      for (uint32_t s = 0; s < K; ++s) {
        const SceneSpec& sp = *specs[s];
        if (!(r < sp.materials.size() && sp.materials[r].first == MAT_CLOTH)) continue;
        const ClothSpec& cl = sp.cloths[sp.materials[r].second];
        if (c >= cl.tether_colors.size()) continue;
        const uint32_t base = h_scenes_[s].seg_start;
        for (uint32_t q : cl.tether_colors[c]) {
          trec.push_back(make_uint4(base + cl.tether[2 * q], base + cl.tether[2 * q + 1], bits_of(cl.tether_rest[q]),
                                    bits_of(cl.tether_compliance)));
          tsc.push_back(s);
        }
      }
      teth_ranges_[r].push_back({begin, (uint32_t)trec.size()});
    }
  }
  // ---- cloth aerodynamics: per particle, its incident triangles ----------
  // A cloth's drag and lift run before the fluids' preSolve (stage 0) when no
  // fluid precedes it in its scene's materials, else after it (stage 1): the
  // fluid neighbour lists see the cloth's predicted positions as the
  // reference's material order leaves them.
  std::vector<uint2> avtx;
  std::vector<uint32_t> aoff(1, 0);
  std::vector<uint4> atri;
  for (uint32_t stage = 0; stage < 2; ++stage) {
    const uint32_t begin = (uint32_t)avtx.size();
    for (uint32_t s = 0; s < K; ++s) {
      const SceneSpec& sp = *specs[s];
      const uint32_t base = h_scenes_[s].seg_start;
      bool fluid_before = false;
      for (uint32_t r = 0; r < sp.materials.size(); ++r) {
        if (sp.materials[r].first == MAT_FLUID) fluid_before = true;
        if (sp.materials[r].first != MAT_CLOTH) continue;
        const ClothSpec& cl = sp.cloths[sp.materials[r].second];
        if (cl.tris.empty() || (fluid_before ? 1u : 0u) != stage) continue;
        // aero.ts:160-183: CSR of incident triangles in triangle order
        const size_t nt = cl.tris.size() / 3;
        std::vector<uint32_t> off(cl.n + 1, 0);
        for (uint32_t v : cl.tris) ++off[v - cl.offset + 1];
        for (uint32_t v = 0; v < cl.n; ++v) off[v + 1] += off[v];
        std::vector<uint32_t> inc(off.back()), cur(off.begin(), off.end() - 1);
        for (size_t t = 0; t < nt; ++t)
          for (int c = 0; c < 3; ++c) inc[cur[cl.tris[3 * t + c] - cl.offset]++] = (uint32_t)t;
        const uint32_t par = (uint32_t)cloth_par_of_[s][r];
        for (uint32_t v = 0; v < cl.n; ++v) {
          avtx.push_back(make_uint2(base + cl.offset + v, par));
          for (uint32_t m = off[v]; m < off[v + 1]; ++m) {
            const uint32_t* t = cl.tris.data() + 3ull * inc[m];
            atri.push_back(make_uint4(base + t[0], base + t[1], base + t[2], 0u));
          }
          aoff.push_back((uint32_t)atri.size());
        }
      }
    }
    aero_ranges_[stage] = {begin, (uint32_t)avtx.size()};
  }
  // the list build forms the first iteration's density when nothing moves
  // particles between the two passes
  fuse_dens_ = !any_imp_ && aero_ranges_[1].second == aero_ranges_[1].first;
  // ---- cloth velocity smoothing by rank: per particle, its edge neighbours -
  std::vector<uint2> dvtx;
  std::vector<uint32_t> doff(1, 0), dnbr;
  damp_ranges_.assign(max_rank_, {0, 0});
  for (uint32_t r = 0; r < max_rank_; ++r) {
    const uint32_t begin = (uint32_t)dvtx.size();
    for (uint32_t s = 0; s < K; ++s) {
      const SceneSpec& sp = *specs[s];
      if (!(r < sp.materials.size() && sp.materials[r].first == MAT_CLOTH)) continue;
      const ClothSpec& cl = sp.cloths[sp.materials[r].second];
      if (!cl.has_damping) continue;
      const uint32_t base = h_scenes_[s].seg_start;
      // ClothSystem.ts:252-263: neighbours in pair order, both directions
      const size_t np = cl.pairs.size() / 2;
      std::vector<uint32_t> off(cl.n + 1, 0);
      for (uint32_t v : cl.pairs) ++off[v - cl.offset + 1];
      for (uint32_t v = 0; v < cl.n; ++v) off[v + 1] += off[v];
      std::vector<uint32_t> nb(off.back()), cur(off.begin(), off.end() - 1);
      for (size_t q = 0; q < np; ++q) {
        const uint32_t i = cl.pairs[2 * q], j = cl.pairs[2 * q + 1];
        nb[cur[i - cl.offset]++] = j;
        nb[cur[j - cl.offset]++] = i;
      }
      const uint32_t par = (uint32_t)cloth_par_of_[s][r];
      for (uint32_t v = 0; v < cl.n; ++v) {
        dvtx.push_back(make_uint2(base + cl.offset + v, par));
        for (uint32_t m = off[v]; m < off[v + 1]; ++m) dnbr.push_back(base + nb[m]);
        doff.push_back((uint32_t)dnbr.size());
      }
    }
    damp_ranges_[r] = {begin, (uint32_t)dvtx.size()};
  }
  // ---- soft-body tables (global by id) ----------------------------------
  std::vector<uint32_t> grp, grp_soft, csr_off(n_ + 1, 0), csr_idx;
  std::vector<float> rest4(4ull * n_, 0.0f), restc4(4ull * n_, 0.0f), weights(n_, 0.0f);
  {
    uint32_t di = 0;
    std::vector<uint32_t> deg(n_, 0);
    std::vector<std::pair<uint32_t, const SoftSpec*>> locals;  // (scene, spec)
    for (uint32_t s = 0; s < K; ++s) {
      const SceneSpec& sp = *specs[s];
      const uint32_t base = h_scenes_[s].seg_start;
      for (uint32_t r = 0; r < sp.materials.size(); ++r) {
        if (sp.materials[r].first != MAT_SOFT) continue;
        const SoftSpec& ss = sp.softs[sp.materials[r].second];
        for (uint32_t i = 0; i < sp.cap; ++i) {
          if (ss.weights[i] != 0.0f || ss.rest4[4 * i + 3] != 0.0f || ss.rest4[4 * i] != 0.0f ||
              ss.rest4[4 * i + 1] != 0.0f || ss.rest4[4 * i + 2] != 0.0f) {
            for (int c = 0; c < 4; ++c) rest4[4ull * (base + i) + c] = ss.rest4[4 * i + c];
            weights[base + i] = ss.weights[i];
          }
        }
        if (ss.local) {
          for (uint32_t i = ss.span.start; i < ss.span.start + ss.span.count; ++i) {
            grp.push_back(base + i);
            grp_soft.push_back(di);
            deg[base + i] = ss.offsets[i + 1] - ss.offsets[i];
            for (int c = 0; c < 4; ++c) restc4[4ull * (base + i) + c] = ss.rest_centers4[4 * i + c];
          }
          locals.push_back({s, &ss});
        }
        ++di;
      }
    }
    for (uint32_t i = 0; i < n_; ++i) csr_off[i + 1] = csr_off[i] + deg[i];
    csr_idx.assign(std::max<uint32_t>(1, csr_off[n_]), 0);
    for (auto& [s, ss] : locals) {
      const uint32_t base = h_scenes_[s].seg_start;
      for (uint32_t i = ss->span.start; i < ss->span.start + ss->span.count; ++i) {
        const uint32_t from = ss->offsets[i], to = ss->offsets[i + 1];
        for (uint32_t k = from; k < to; ++k) csr_idx[csr_off[base + i] + (k - from)] = base + ss->indices[k];
      }
    }
  }
  // the clusters that hold each particle: (centre id, CSR position) by member
  std::vector<uint32_t> mem_off(n_ + 1, 0), mem_soft(n_, 0), mem_ids;
  std::vector<uint2> mem;
  {
    for (uint32_t g = 0; g < grp.size(); ++g)
      for (uint32_t m = csr_off[grp[g]]; m < csr_off[grp[g] + 1]; ++m) {
        ++mem_off[csr_idx[m] + 1];
        mem_soft[csr_idx[m]] = grp_soft[g];
      }
    std::vector<uint32_t> held;  // clusters holding each member
    for (uint32_t i = 0; i < n_; ++i) {
      if (mem_off[i + 1]) {
        mem_ids.push_back(i);
        held.push_back(mem_off[i + 1]);
      }
      mem_off[i + 1] += mem_off[i];
    }
    // lanes per member in k_sm_gather: the smallest power of two that takes
    // the clusters of nine members in ten in at most sixteen rounds. Each
    // member starts with a chain of dependent loads (its id, body, scene,
    // slot and position), so more members per warp keep more of those chains
    // in flight; some rounds per member cost less than idle chains. On the
    // serving stream's soft bodies (27 clusters per member) one served tick
    // took 15.8, 13.2, 11.8, 10.7, 10.4 and 10.9 ms with 32, 16, 8, 4, 2 and
    // 1 lanes.
    mem_lanes_ = 1;
    if (!held.empty()) {
      const size_t at = (held.size() * 9) / 10;
      std::nth_element(held.begin(), held.begin() + at, held.end());
      const uint32_t p90 = held[at];
      while (mem_lanes_ < 32 && mem_lanes_ * 16 < p90) mem_lanes_ *= 2;
    }
    if (const char* e = std::getenv("PFSIM_MEMBER_LANES")) {  // fixed choice for measurements and tests
      const uint32_t l = (uint32_t)std::atoi(e);
      if (l == 1 || l == 2 || l == 4 || l == 8 || l == 16 || l == 32) mem_lanes_ = l;
    }
    mem.assign(std::max<uint32_t>(1, mem_off[n_]), make_uint2(0, 0));
    std::vector<uint32_t> at(mem_off.begin(), mem_off.end() - 1);
    for (uint32_t g = 0; g < grp.size(); ++g)
      for (uint32_t m = csr_off[grp[g]]; m < csr_off[grp[g] + 1]; ++m) mem[at[csr_idx[m]]++] = make_uint2(grp[g], m);
  }
  // ---- chunk table and per-slot state ----------------------------------
  std::vector<uint32_t> chunk(n_ / kSegAlign, 0);
  for (uint32_t s = 0; s < K; ++s)
    for (uint32_t c = h_scenes_[s].seg_start / kSegAlign; c < h_scenes_[s].seg_end / kSegAlign; ++c) chunk[c] = s;
  // scenes that hold one fluid of one mass and nothing else but colliders
  // fused into its apply: candidates for the L2-sized groups of run_groups.
  // Their chunks lead the fluid chunk list, scene by scene.
  std::vector<uint8_t> pure(K, 0);
  pure_end_.clear();
  pure_parts_.clear();
  pure_scene_.clear();
  for (uint32_t s = 0; s < K; ++s) {
    const DevScene& S = h_scenes_[s];
    if (S.fluid_count != 1 || !S.homog || S.contact || specs[s]->materials.size() != 1) continue;
    if (S.prim_count + S.sdf_count > 0 && S.collide_rank1 != 1) continue;
    const DevFluid& F = h_fluids_[S.fluid_first];
    if (F.has_vort || F.has_st || F.has_ad || F.bnd_count) continue;
    pure[s] = 1;
  }
  std::vector<uint32_t> fchunk, cchunk;
  for (uint32_t s = 0; s < K; ++s) {
    if (!pure[s]) continue;
    for (uint32_t c = h_scenes_[s].seg_start / kSegAlign; c < h_scenes_[s].seg_end / kSegAlign; ++c) fchunk.push_back(c);
    pure_end_.push_back((uint32_t)fchunk.size());
    pure_parts_.push_back(h_scenes_[s].cap);
    pure_scene_.push_back(s);
  }
  n_pure_chunks_ = (uint32_t)fchunk.size();
  for (uint32_t c = 0; c < chunk.size(); ++c) {
    const DevScene& S = h_scenes_[chunk[c]];
    if (S.fluid_count && !pure[chunk[c]]) fchunk.push_back(c);
    if ((S.prim_count + S.sdf_count > 0 || S.contact) && S.collide_rank1 == 0) cchunk.push_back(c);
  }
  groups_.clear();
  std::vector<float> dens(n_, 0.0f);
  std::vector<uint32_t> tag(n_, 0);
  for (uint32_t s = 0; s < K; ++s) {
    const SceneSpec& sp = *specs[s];
    const uint32_t base = h_scenes_[s].seg_start;
    for (uint32_t f = 0; f < h_scenes_[s].fluid_count; ++f) {
      const FluidSpec& fs = sp.fluids[f];
      for (uint32_t i = fs.range.start; i < fs.range.start + fs.range.count; ++i) {
        tag[base + i] = (tag[base + i] & 0xffff0000u) | (h_scenes_[s].fluid_first + f + 1);
        dens[base + i] = f32(fs.rho0);
      }
    }
  }
  for (uint32_t b = 0; b < h_bnds_.size(); ++b) {
    const DevBoundary& B = h_bnds_[b];
    for (uint32_t i = B.start; i < B.start + B.count; ++i) tag[i] = (tag[i] & 0xffffu) | ((b + 1) << 16);
  }
  // ---- fluid grid rows and the tile budget ------------------------------
  std::vector<uint32_t> row_base(1, 0), grid_scene;
  uint64_t max_tiles = 1;
  for (uint32_t s = 0; s < K; ++s) {
    const DevScene& S = h_scenes_[s];
    if (!S.has_grid || S.fluid_count == 0) continue;
    grid_scene.push_back(s);
    row_base.push_back(row_base.back() + S.dims[1] * S.dims[2]);
    // every tile holds at least one particle (and one cell, whatever the
    // window's size once it has grown)
    max_tiles += S.cap;
  }
  max_tiles = std::min<uint64_t>(max_tiles, 0xffffffffull);
  // ---- allocate one arena ----------------------------------------------
  const size_t N = n_;
  const size_t P = prim_stride_;
  const bool need_soft = !grp.empty() || !h_bodies_.empty();
  uint64_t total_real = 0;
  prefix_.assign(K, 0);
  for (uint32_t s = 0; s < K; ++s) {
    prefix_[s] = total_real;
    total_real += h_scenes_[s].cap;
  }
  const uint64_t cell_room = std::min<uint64_t>(kSortCellCap, 2ull * cells_);
  auto layout = [&](Carver& cv) {
    base_.scenes_rw = cv.take<DevScene>(K);
    base_.chunk_scene = cv.take<uint32_t>(chunk.size());
    base_.fchunk = cv.take<uint32_t>(fchunk.size());
    base_.cchunk = cv.take<uint32_t>(cchunk.size());
    base_.n_fchunk = (uint32_t)fchunk.size();
    base_.n_cchunk = (uint32_t)cchunk.size();
    base_.flags = cv.take<uint32_t>(K * kNumFlags);
    base_.bbox = cv.take<int32_t>(6 * K);
    base_.bbox_last = cv.take<int32_t>(6 * K);
    base_.clocks = cv.take<float>(K);
    base_.fluids = cv.take<DevFluid>(h_fluids_.size());
    base_.bnds = cv.take<DevBoundary>(h_bnds_.size());
    base_.prims = cv.take<pf_primitive>(h_prims_.size());
    base_.plane4 = cv.take<float4>(2 * h_prims_.size());
    base_.sdfs = cv.take<DevSdf>(h_sdfs_.size());
    base_.sdf_half = cv.take<uint16_t>(sdf_voxels);
    for (int b = 0; b < 2; ++b) {
      buf_[b].x = cv.take<float4>(N);
      buf_[b].xs = cv.take<float4>(N);
      buf_[b].v = cv.take<float4>(N);
      buf_[b].bv = cv.take<float>(N);
      buf_[b].tag = cv.take<uint32_t>(N);
      buf_[b].dens = cv.take<float>(N);
    }
    base_.ids = cv.take<uint32_t>(N);
    base_.inv = cv.take<uint32_t>(N);
    base_.keys = cv.take<uint32_t>(N);
    base_.perm = cv.take<uint32_t>(N);
    // room for the windows to double before the cell arrays move
    base_.cstart = cv.take<uint32_t>(cell_room);
    base_.ccount = cv.take<uint32_t>(cell_room);
    base_.nbr = any_fluid_ ? cv.take<uint32_t>(N * kMaxNbr) : nullptr;
    base_.nbr_base = any_fluid_ ? cv.take<uint32_t>(N / 32) : nullptr;
    base_.nbr16 = reinterpret_cast<uint16_t*>(base_.nbr);
    base_.ncount = cv.take<uint32_t>(N);
    base_.slot_tile = cv.take<uint32_t>(N);
    base_.tiles = cv.take<Tile>(max_tiles);
    base_.tile_count = cv.take<uint32_t>(1);
    base_.row_base = cv.take<uint32_t>(row_base.size());
    base_.grid_scene = cv.take<uint32_t>(grid_scene.size());
    base_.lambda = cv.take<float>(N);
    base_.lm = any_fluid_ ? cv.take<float2>(N) : nullptr;
    base_.xl = any_fluid_ ? cv.take<float4>(N) : nullptr;
    base_.dx = cv.take<float4>(N);
    base_.dv = cv.take<float4>(N);
    base_.vort = any_vort_ ? cv.take<float4>(N) : nullptr;
    base_.normal = any_imp_ ? cv.take<float4>(N) : nullptr;
    base_.acc_imp = any_imp_ ? cv.take<int4>(N) : nullptr;
    base_.plam = cv.take<float2>(N * P);
    base_.cmask = cv.take<uint32_t>(N);
    base_.acc_react = any_react_ ? cv.take<int4>(N) : nullptr;
    base_.softs = cv.take<DevSoft>(h_softs_.size());
    base_.bodies = cv.take<DevBody>(h_bodies_.size());
    base_.grp = cv.take<uint32_t>(grp.size());
    base_.grp_soft = cv.take<uint32_t>(grp_soft.size());
    base_.csr_off = need_soft ? cv.take<uint32_t>(N + 1) : nullptr;
    base_.csr_idx = cv.take<uint32_t>(csr_idx.size());
    base_.rest = need_soft ? cv.take<float4>(N) : nullptr;
    base_.rest_c = need_soft ? cv.take<float4>(N) : nullptr;
    base_.weights = need_soft ? cv.take<float>(N) : nullptr;
    base_.rot4 = need_soft ? cv.take<float4>(4 * N) : nullptr;
    base_.q = need_soft ? cv.take<float4>(N) : nullptr;
    base_.qp = need_soft ? cv.take<float4>(N) : nullptr;
    base_.omega = need_soft ? cv.take<float4>(N) : nullptr;
    base_.pair_lambda = cv.take<float4>(csr_idx.size());
    base_.mem_off = any_soft_local_ ? cv.take<uint32_t>(N + 1) : nullptr;
    base_.mem = any_soft_local_ ? cv.take<uint2>(mem.size()) : nullptr;
    base_.mem_soft = any_soft_local_ ? cv.take<uint32_t>(N) : nullptr;
    base_.mem_ids = any_soft_local_ ? cv.take<uint32_t>(mem_ids.size()) : nullptr;
    base_.n_mem_ids = any_soft_local_ ? (uint32_t)mem_ids.size() : 0u;
    base_.lambda_g = need_soft ? cv.take<float4>(N) : nullptr;
    base_.body_c = cv.take<float4>(h_bodies_.size());
    base_.body_r = cv.take<float4>(3 * h_bodies_.size());
    base_.c_i = cv.take<uint32_t>(ci.size());
    base_.c_j = cv.take<uint32_t>(cj.size());
    base_.c_rest = cv.take<float>(crest.size());
    base_.c_comp = cv.take<float>(ccomp.size());
    base_.c_scene = cv.take<uint32_t>(csc.size());
    base_.c_lambda = cv.take<float>(ci.size());
    base_.b_idx = cv.take<uint4>(bidx.size());
    base_.b_rest = cv.take<float>(brest.size());
    base_.b_cloth = cv.take<uint32_t>(bcl.size());
    base_.b_scene = cv.take<uint32_t>(bsc.size());
    base_.b_lambda = cv.take<float>(bidx.size());
    base_.t_rec = cv.take<uint4>(trec.size());
    base_.t_scene = cv.take<uint32_t>(tsc.size());
    base_.t_lambda = cv.take<float>(trec.size());
    base_.a_vtx = cv.take<uint2>(avtx.size());
    base_.a_off = cv.take<uint32_t>(aoff.size());
    base_.a_tri = cv.take<uint4>(atri.size());
    base_.d_vtx = cv.take<uint2>(dvtx.size());
    base_.d_off = cv.take<uint32_t>(doff.size());
    base_.d_nbr = cv.take<uint32_t>(dnbr.size());
    base_.d_smooth = cv.take<float4>(dvtx.size());
    cloth_par_dev_ = cv.take<DevCloth>(h_cloth_par_.size());
    base_.cloth_par = cloth_par_dev_;
    // particle contacts
    const size_t CH = N / kSegAlign;
    base_.cgroup = any_contact_ ? cv.take<uint32_t>(N) : nullptr;
    base_.cquiet = any_contact_ ? cv.take<uint8_t>(N) : nullptr;
    base_.con_nbr = any_contact_ ? cv.take<uint32_t>(kMaxContacts * N) : nullptr;
    base_.con_cnt = any_contact_ ? cv.take<uint32_t>(N) : nullptr;
    base_.con_pre = any_contact_ ? cv.take<uint32_t>(N) : nullptr;
    base_.chunk_sum = any_contact_ ? cv.take<uint32_t>(CH) : nullptr;
    base_.chunk_drop = any_contact_ ? cv.take<uint32_t>(CH) : nullptr;
    base_.chunk_off = any_contact_ ? cv.take<uint32_t>(CH) : nullptr;
    base_.con_lam = any_contact_ ? cv.take<int2>(kMaxContacts * N) : nullptr;
    base_.con_nrm = any_contact_ ? cv.take<float4>(kMaxContacts * N) : nullptr;
    base_.acc_con = any_contact_ ? cv.take<int4>(N) : nullptr;
    base_.con_stat = any_contact_ ? cv.take<uint2>(K) : nullptr;
    stage_pos_ = cv.take<float4>(total_real);
    stage_pos2_ = cv.take<float4>(total_real);
    prefix_dev_ = cv.take<uint64_t>(K);
  };
  Carver probe{nullptr};
  layout(probe);
  // the sort scratch is carved for 64 times the cells (its cell-sized part
  // is 1/512 byte per cell), so growing windows seldom re-allocate it
  const uint64_t sort_cells = std::min<uint64_t>(kSortCellCap, std::max<uint64_t>(64ull * cells_, 1ull << 20));
  const size_t sort_bytes = sort_scratch_bytes(n_, sort_cells);
  bytes_ = probe.off + al256(sort_bytes);
  if (plan_only) return PF_OK;
  (void)sm_count();  // cache the SM count outside any stream capture
  PF_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  if (const cudaError_t e = dev_alloc(&arena_, bytes_, stream_); e != cudaSuccess) {
    arena_ = nullptr;
    if (e == cudaErrorMemoryAllocation)
      return fail(PF_ERR_OOM, "SimLoop: out of device memory (" + std::to_string(bytes_) + " bytes)");
    return fail(PF_ERR_CUDA, std::string("SimLoop: device allocation failed: ") + cudaGetErrorString(e));
  }
  // the pool's allocation is ordered on stream_: wait for it, so copies on
  // any stream may use the arena
  PF_CUDA(cudaStreamSynchronize(stream_));
  Carver cv{static_cast<char*>(arena_)};
  layout(cv);
  sort_scratch_carve(static_cast<char*>(arena_) + probe.off, n_, sort_cells, &sort_);
  radix_ = radix_plan(cells_);
  cells_cap_ = cell_room;
  grow_prev_ext_.assign(3 * K, 0);
  base_.scenes = base_.scenes_rw;
  base_.n = n_;
  base_.prim_stride = prim_stride_;
  base_.n_grp = (uint32_t)grp.size();
  base_.n_bodies = (uint32_t)h_bodies_.size();
  base_.n_cons = (uint32_t)ci.size();
  base_.n_bend = (uint32_t)bidx.size();
  base_.n_teth = (uint32_t)trec.size();
  base_.max_tiles = (uint32_t)max_tiles;
  base_.n_grid_scenes = (uint32_t)grid_scene.size();
  base_.n_rows = row_base.back();
  pair_entries_ = any_soft_local_ ? csr_idx.size() : 0;
  if (side_ok_) {
    PF_CUDA(cudaStreamCreateWithFlags(&side_stream_, cudaStreamNonBlocking));
    PF_CUDA(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
    PF_CUDA(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
  }
  PF_CUDA(cudaEventCreate(&ev0_));
  PF_CUDA(cudaEventCreate(&ev1_));
  for (uint32_t q = 0; q < kParamRing; ++q) PF_CUDA(cudaEventCreateWithFlags(&ev_params_[q], cudaEventDisableTiming));
  for (uint32_t q = 0; q < kBoundsRing; ++q) PF_CUDA(cudaEventCreateWithFlags(&ev_bounds_[q], cudaEventDisableTiming));
  PF_CUDA(cudaMallocHost(&h_pinned_bbox_, sizeof(int32_t) * 6 * kBoundsRing * std::max<size_t>(1, K)));
  PF_CUDA(cudaMallocHost(&h_pinned_scenes_, sizeof(DevScene) * kParamRing * std::max<size_t>(1, K)));
  PF_CUDA(cudaMallocHost(&h_pinned_prims_, sizeof(pf_primitive) * std::max<size_t>(1, h_prims_.size())));
  PF_CUDA(cudaMallocHost(&h_pinned_plane4_, sizeof(float4) * 2 * std::max<size_t>(1, h_prims_.size())));
  PF_CUDA(cudaMallocHost(&h_pinned_sdfs_, sizeof(DevSdf) * std::max<size_t>(1, h_sdfs_.size())));
  PF_CUDA(cudaMallocHost(&h_pinned_cloth_, sizeof(DevCloth) * std::max<size_t>(1, h_cloth_par_.size())));
  // ---- upload ----------------------------------------------------------
  auto up = [&](const void* dst, const void* src, size_t bytes) -> pf_status {
    if (bytes == 0) return PF_OK;
    PF_CUDA(cudaMemcpyAsync(const_cast<void*>(dst), src, bytes, cudaMemcpyHostToDevice, stream_));
    return PF_OK;
  };
  PF_CUDA(cudaMemsetAsync(arena_, 0, probe.off, stream_));
  PF_CUDA(sort_scratch_zero(sort_, stream_));
  PF_CUDA(radix_prepare());  // before any graph capture
  PF_CUDA(slot_kernels_prepare());
  PF_TRY(up(base_.scenes_rw, h_scenes_.data(), sizeof(DevScene) * K));
  {
    // empty cell bounds: the predict pass narrows them (a pageable source:
    // the copy has read it when the call returns)
    std::vector<int32_t> empty(6 * K, 0);
    for (uint32_t s = 0; s < K; ++s)
      for (int a = 0; a < 3; ++a) {
        empty[6 * s + a] = INT32_MAX;
        empty[6 * s + a + 3] = INT32_MIN;
      }
    PF_TRY(up(base_.bbox, empty.data(), 4ull * empty.size()));
  }
  PF_TRY(up(base_.chunk_scene, chunk.data(), 4 * chunk.size()));
  PF_TRY(up(const_cast<uint32_t*>(base_.fchunk), fchunk.data(), 4 * fchunk.size()));
  PF_TRY(up(const_cast<uint32_t*>(base_.cchunk), cchunk.data(), 4 * cchunk.size()));
  PF_TRY(up(base_.fluids, h_fluids_.data(), sizeof(DevFluid) * h_fluids_.size()));
  PF_TRY(up(base_.bnds, h_bnds_.data(), sizeof(DevBoundary) * h_bnds_.size()));
  PF_TRY(up(base_.prims, h_prims_.data(), sizeof(pf_primitive) * h_prims_.size()));
  PF_TRY(up(const_cast<float4*>(base_.plane4), h_plane4_.data(), sizeof(float4) * 2 * h_prims_.size()));
  PF_TRY(up(base_.sdfs, h_sdfs_.data(), sizeof(DevSdf) * h_sdfs_.size()));
  {
    uint64_t off = 0;
    for (uint32_t s = 0; s < K; ++s)
      for (auto& g : specs[s]->sdfs) {
        PF_TRY(up(base_.sdf_half + off, g.half.data(), 2 * g.half.size()));
        off += g.half.size();
      }
  }
  // identity slot maps and orientations on the device; the scenes' own state
  // goes to their segments (scenes whose state is imported afterwards skip it)
  k_init_slots<<<div_up(n_, kBlock), kBlock, 0, stream_>>>(base_.ids, base_.inv, base_.q, base_.qp, n_);
  PF_CUDA(cudaGetLastError());
  {
    // pageable copies: the call returns once the source has been consumed,
    // so the staging vectors can be refilled for the next scene
    std::vector<float4> sx, sv, so;
    for (uint32_t s = 0; s < K; ++s) {
      if (skip_state && (*skip_state)[s]) continue;
      const SceneSpec& sp = *specs[s];
      const uint32_t base = h_scenes_[s].seg_start, cap = sp.cap;
      sx.resize(cap);
      sv.resize(cap);
      for (uint32_t i = 0; i < cap; ++i) {
        sx[i] = make_float4(sp.pos4[4 * i], sp.pos4[4 * i + 1], sp.pos4[4 * i + 2], sp.inv_mass[i]);
        sv[i] = make_float4(sp.vel4[4 * i], sp.vel4[4 * i + 1], sp.vel4[4 * i + 2], 0.0f);
      }
      PF_TRY(up(buf_[0].x + base, sx.data(), 16ull * cap));
      PF_TRY(up(buf_[0].xs + base, sx.data(), 16ull * cap));
      PF_TRY(up(buf_[0].v + base, sv.data(), 16ull * cap));
      PF_TRY(up(buf_[0].bv + base, sp.bvol.data(), 4ull * cap));
      if (base_.q && !sp.rot4.empty()) {
        PF_TRY(up(base_.q + base, sp.rot4.data(), 16ull * cap));
        PF_TRY(up(base_.qp + base, sp.rot4.data(), 16ull * cap));
      }
      if (base_.omega && !sp.angv4.empty()) {
        so.resize(cap);
        for (uint32_t i = 0; i < cap; ++i)
          so[i] = make_float4(sp.angv4[4 * i], sp.angv4[4 * i + 1], sp.angv4[4 * i + 2], 0.0f);
        PF_TRY(up(base_.omega + base, so.data(), 16ull * cap));
      }
    }
  }
  PF_TRY(up(buf_[0].tag, tag.data(), 4 * N));
  PF_TRY(up(buf_[0].dens, dens.data(), 4 * N));
  PF_TRY(up(base_.softs, h_softs_.data(), sizeof(DevSoft) * h_softs_.size()));
  PF_TRY(up(base_.bodies, h_bodies_.data(), sizeof(DevBody) * h_bodies_.size()));
  PF_TRY(up(base_.grp, grp.data(), 4 * grp.size()));
  PF_TRY(up(base_.grp_soft, grp_soft.data(), 4 * grp_soft.size()));
  if (need_soft) {
    PF_TRY(up(base_.csr_off, csr_off.data(), 4 * csr_off.size()));
    PF_TRY(up(base_.csr_idx, csr_idx.data(), 4 * csr_idx.size()));
    if (any_soft_local_) {
      PF_TRY(up(const_cast<uint32_t*>(base_.mem_off), mem_off.data(), 4 * mem_off.size()));
      PF_TRY(up(const_cast<uint2*>(base_.mem), mem.data(), sizeof(uint2) * mem.size()));
      PF_TRY(up(const_cast<uint32_t*>(base_.mem_soft), mem_soft.data(), 4 * mem_soft.size()));
      PF_TRY(up(const_cast<uint32_t*>(base_.mem_ids), mem_ids.data(), 4 * mem_ids.size()));
    }
    PF_TRY(up(base_.rest, rest4.data(), 16 * N));
    PF_TRY(up(base_.rest_c, restc4.data(), 16 * N));
    PF_TRY(up(base_.weights, weights.data(), 4 * N));
    std::vector<float4> ident(3 * h_bodies_.size());
    for (size_t b = 0; b < h_bodies_.size(); ++b) {
      ident[3 * b] = make_float4(1, 0, 0, 0);
      ident[3 * b + 1] = make_float4(0, 1, 0, 0);
      ident[3 * b + 2] = make_float4(0, 0, 1, 0);
    }
    PF_TRY(up(base_.body_r, ident.data(), 16 * ident.size()));
  }
  PF_TRY(up(base_.c_i, ci.data(), 4 * ci.size()));
  PF_TRY(up(base_.c_j, cj.data(), 4 * cj.size()));
  PF_TRY(up(base_.c_rest, crest.data(), 4 * crest.size()));
  PF_TRY(up(base_.c_comp, ccomp.data(), 4 * ccomp.size()));
  PF_TRY(up(base_.c_scene, csc.data(), 4 * csc.size()));
  PF_TRY(up(base_.b_idx, bidx.data(), sizeof(uint4) * bidx.size()));
  PF_TRY(up(base_.b_rest, brest.data(), 4 * brest.size()));
  PF_TRY(up(base_.b_cloth, bcl.data(), 4 * bcl.size()));
  PF_TRY(up(base_.t_rec, trec.data(), sizeof(uint4) * trec.size()));
  PF_TRY(up(base_.t_scene, tsc.data(), 4 * tsc.size()));
  PF_TRY(up(base_.a_vtx, avtx.data(), sizeof(uint2) * avtx.size()));
  PF_TRY(up(base_.a_off, aoff.data(), 4 * aoff.size()));
  PF_TRY(up(base_.a_tri, atri.data(), sizeof(uint4) * atri.size()));
  PF_TRY(up(base_.d_vtx, dvtx.data(), sizeof(uint2) * dvtx.size()));
  PF_TRY(up(base_.d_off, doff.data(), 4 * doff.size()));
  PF_TRY(up(base_.d_nbr, dnbr.data(), 4 * dnbr.size()));
  PF_TRY(up(cloth_par_dev_, h_cloth_par_.data(), sizeof(DevCloth) * h_cloth_par_.size()));
  if (any_contact_) {
    // collision groups and noSelfContacts membership by id
    std::vector<uint32_t> cg(n_, 0);
    std::vector<uint8_t> cq(n_, 1);
    for (uint32_t s = 0; s < K; ++s) {
      const SceneSpec& sp = *specs[s];
      const uint32_t base = h_scenes_[s].seg_start;
      for (uint32_t i = 0; i < sp.cap; ++i) {
        cg[base + i] = sp.group[i];
        cq[base + i] = 0;
      }
      for (auto& f : sp.fluids)
        for (uint32_t i = f.range.start; i < f.range.start + f.range.count; ++i) cq[base + i] = 1;
      for (auto& q : sp.quiet)
        for (uint32_t i = q.start; i < q.start + q.count; ++i) cq[base + i] = 1;
    }
    PF_TRY(up(base_.cgroup, cg.data(), 4ull * n_));
    PF_TRY(up(base_.cquiet, cq.data(), n_));
    PF_CUDA(cudaMemsetAsync(base_.acc_con, 0, 16ull * n_, stream_));
    PF_CUDA(cudaMemsetAsync(base_.con_cnt, 0, 4ull * n_, stream_));
    PF_CUDA(cudaMemsetAsync(base_.con_stat, 0, 8ull * K, stream_));
  }
  PF_TRY(up(base_.b_scene, bsc.data(), 4 * bsc.size()));
  PF_TRY(up(prefix_dev_, prefix_.data(), 8 * prefix_.size()));
  PF_TRY(up(base_.row_base, row_base.data(), 4 * row_base.size()));
  PF_TRY(up(base_.grid_scene, grid_scene.data(), 4 * grid_scene.size()));
  PF_CUDA(cudaFuncSetAttribute(k_t_neighbors, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemNbr));
  PF_CUDA(cudaFuncSetAttribute(k_t_lambda, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemLambda));
  PF_CUDA(cudaFuncSetAttribute(k_t_delta, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemDelta));
  PF_CUDA(cudaFuncSetAttribute(k_t_xsph, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemXsph));
  PF_CUDA(cudaStreamSynchronize(stream_));
  parity_ = 0;
  inited_ = true;
  for (auto* sp : specs_)
    if (!sp->initialized) inited_ = false;
  prims_dirty_ = false;
  return PF_OK;
}

// The compact form of each primitive for the collider passes' plane test,
// and per scene whether every primitive takes it: a plane that neither
// sweeps nor spins, with a finite velocity (prim_sdf's unswept plane; its
// x_w + v * 0 is x_w but for the sign of a zero, which d1 + (x - d1) does
// not keep).
void World::refresh_planes(int only_scene) {
  if (only_scene < 0) h_plane4_.assign(2 * std::max<size_t>(1, h_prims_.size()), make_float4(0.0f, 0.0f, 0.0f, 0.0f));
  for (size_t s = 0; s < h_scenes_.size(); ++s) {
    if (only_scene >= 0 && s != (size_t)only_scene) continue;
    DevScene& S = h_scenes_[s];
    bool fast = true;
    for (uint32_t q = 0; q < S.prim_count; ++q) {
      const pf_primitive& p = h_prims_[S.prim_base + q];
      h_plane4_[2 * (S.prim_base + q)] =
          make_float4(p.data0[0], p.data0[1], p.data0[2], (p.flags & PF_PRIM_INVERT) ? 1.0f : 0.0f);
      h_plane4_[2 * (S.prim_base + q) + 1] = make_float4(p.data1[0], p.data1[1], p.data1[2], 0.0f);
      fast = fast && p.kind == PF_PRIM_PLANE && !(p.flags & PF_PRIM_SWEEP) && p.spin[0] == 0.0f &&
             p.spin[1] == 0.0f && p.spin[2] == 0.0f && std::isfinite(p.velocity[0]) &&
             std::isfinite(p.velocity[1]) && std::isfinite(p.velocity[2]);
    }
    S.planes_fast = fast ? 1u : 0u;
  }
}

pf_status World::set_primitive(uint32_t scene, uint32_t slot, const pf_primitive& p) {
  if (scene >= specs_.size()) return fail(PF_ERR_INVALID, "PrimitiveSet: no such scene");
  const DevScene& S = h_scenes_[scene];
  if (slot >= S.prim_count) return fail(PF_ERR_INVALID, "PrimitiveSet: no primitive in slot " + std::to_string(slot));
  h_prims_[S.prim_base + slot] = p;
  specs_[scene]->prims[slot] = p;
  refresh_planes((int)scene);
  prims_dirty_ = true;
  return PF_OK;
}

pf_status World::set_sdf_transform(uint32_t scene, uint32_t slot, const float pos[3], const double q[4], float scale) {
  if (scene >= specs_.size()) return fail(PF_ERR_INVALID, "SDFCollider: no such scene");
  const DevScene& S = h_scenes_[scene];
  if (slot >= S.sdf_count) return fail(PF_ERR_INVALID, "SDFCollider: no collider in slot " + std::to_string(slot));
  SdfSpec& g = specs_[scene]->sdfs[slot];
  for (int a = 0; a < 3; ++a) g.position[a] = pos[a];
  for (int a = 0; a < 4; ++a) g.rot_q[a] = q[a];
  g.scale = scale;
  h_sdfs_[S.sdf_base + slot] = make_dev_sdf(g, h_sdfs_[S.sdf_base + slot].data_off);
  sdfs_dirty_ = true;
  return PF_OK;
}

pf_status World::set_cloth_params(uint32_t scene, uint32_t material, const pf_cloth_params& p) {
  if (scene >= specs_.size()) return fail(PF_ERR_INVALID, "ClothSystem: no such scene");
  if (material >= cloth_par_of_[scene].size() || cloth_par_of_[scene][material] < 0)
    return fail(PF_ERR_INVALID, "ClothSystem: material " + std::to_string(material) + " is not a cloth");
  ClothSpec& cl = specs_[scene]->cloths[specs_[scene]->materials[material].second];
  DevCloth& P = h_cloth_par_[(size_t)cloth_par_of_[scene][material]];
  for (int a = 0; a < 3; ++a) P.wind[a] = cl.wind[a] = p.wind[a];
  P.drag = cl.drag = p.drag;
  P.lift = cl.lift = p.lift;
  P.damping = cl.damping = p.damping;
  P.bend_compliance = cl.bend_compliance = p.bend_compliance;
  cloth_par_dirty_ = true;
  return PF_OK;
}

pf_status World::upload_params(double dt) {
  const uint32_t K = (uint32_t)h_scenes_.size();
  for (uint32_t s = 0; s < K; ++s) h_scenes_[s].dt = h_scenes_[s].substeps ? f32(dt / h_scenes_[s].substeps) : 0.0f;
  // where this step's density passes leave lambda (read back by PF_FIELD_LAMBDA)
  lam_in_xl_.resize(K);
  for (uint32_t s = 0; s < K; ++s) lam_in_xl_[s] = h_scenes_[s].homog != 0;
  // Earlier steps' copies may still wait behind earlier work: a ring slot's
  // pinned source is written only once its last copy has run, and the
  // single-buffer tables (rewritten only after a setter) once every copy has.
  const uint32_t slot = (uint32_t)(uploads_ % kParamRing);
  if (params_pending_[slot]) {
    PF_CUDA(cudaEventSynchronize(ev_params_[slot]));
    params_pending_[slot] = false;
  }
  if ((sdfs_dirty_ && !h_sdfs_.empty()) || (cloth_par_dirty_ && !h_cloth_par_.empty()) ||
      (prims_dirty_ && !h_prims_.empty()))
    PF_TRY(wait_uploads());
  DevScene* staged = h_pinned_scenes_ + (size_t)slot * K;
  std::memcpy(staged, h_scenes_.data(), sizeof(DevScene) * K);
  PF_CUDA(cudaMemcpyAsync(base_.scenes_rw, staged, sizeof(DevScene) * K, cudaMemcpyHostToDevice, stream_));
  if (sdfs_dirty_ && !h_sdfs_.empty()) {
    std::memcpy(h_pinned_sdfs_, h_sdfs_.data(), sizeof(DevSdf) * h_sdfs_.size());
    PF_CUDA(cudaMemcpyAsync(const_cast<DevSdf*>(base_.sdfs), h_pinned_sdfs_, sizeof(DevSdf) * h_sdfs_.size(),
                            cudaMemcpyHostToDevice, stream_));
    sdfs_dirty_ = false;
  }
  if (cloth_par_dirty_ && !h_cloth_par_.empty()) {
    std::memcpy(h_pinned_cloth_, h_cloth_par_.data(), sizeof(DevCloth) * h_cloth_par_.size());
    PF_CUDA(cudaMemcpyAsync(cloth_par_dev_, h_pinned_cloth_, sizeof(DevCloth) * h_cloth_par_.size(),
                            cudaMemcpyHostToDevice, stream_));
    cloth_par_dirty_ = false;
  }
  if (prims_dirty_ && !h_prims_.empty()) {
    std::memcpy(h_pinned_prims_, h_prims_.data(), sizeof(pf_primitive) * h_prims_.size());
    std::memcpy(h_pinned_plane4_, h_plane4_.data(), sizeof(float4) * 2 * h_prims_.size());
    PF_CUDA(cudaMemcpyAsync(const_cast<float4*>(base_.plane4), h_pinned_plane4_, sizeof(float4) * 2 * h_prims_.size(),
                            cudaMemcpyHostToDevice, stream_));
    PF_CUDA(cudaMemcpyAsync(const_cast<pf_primitive*>(base_.prims), h_pinned_prims_,
                            sizeof(pf_primitive) * h_prims_.size(), cudaMemcpyHostToDevice, stream_));
    prims_dirty_ = false;
  }
  PF_CUDA(cudaEventRecord(ev_params_[slot], stream_));
  params_pending_[slot] = true;
  ++uploads_;
  return PF_OK;
}

pf_status World::wait_uploads() {
  for (uint32_t q = 0; q < kParamRing; ++q)
    if (params_pending_[q]) {
      PF_CUDA(cudaEventSynchronize(ev_params_[q]));
      params_pending_[q] = false;
    }
  return PF_OK;
}

void World::launch_frame_start_at(uint32_t parity) {
  const uint32_t K = (uint32_t)h_scenes_.size();
  k_frame_start<<<div_up(K, 128), 128, 0, stream_>>>(view(parity), K);
  ++t_launches;
}

// Cut the fluid scenes' grid rows into tiles and build the neighbour lists.
void World::launch_tiles_build(const WorldView& V, uint32_t s) {
  cudaMemsetAsync(base_.tile_count, 0, 4, stream_);
  launch_slots(k_build_tiles, base_.n_rows, stream_, V, s);
  launch_tiled(k_t_neighbors, kSmemNbr, V, s);
}

// One-thread-per-slot fluid kernels at a tuned block size.
template <typename K, typename... A>
void World::launch_fluid(uint32_t block, K kernel, const WorldView& V, A... args) {
  const uint32_t slots = V.n_fchunk * kSegAlign;  // the view's chunks of scenes with a fluid
  if (!slots) return;
  kernel<<<div_up(slots, block), block, 0, stream_>>>(V, args...);
  ++t_launches;
}

// A slot kernel of kind KIND at that kind's tuned block size and fetch depth.
#define PF_BY_UNROLL(KIND, K, ...)                                                      \
  do {                                                                                  \
    const uint32_t b_ = tune_.block[KIND], u_ = tune_.unroll[KIND];                     \
    if (u_ == 2) launch_fluid(b_, K<2>, __VA_ARGS__);                                   \
    else if (u_ == 8) launch_fluid(b_, K<8>, __VA_ARGS__);                              \
    else launch_fluid(b_, K<4>, __VA_ARGS__);                                           \
  } while (0)
// The list build, forming the first iteration's density and lambda of
// first-material fluids when nothing moves between the two (fuse_dens_).
#define PF_NBR_FLAT(FLAT, ...)                                                          \
  do {                                                                                  \
    const uint32_t b_ = tune_.block[kSlotNbr], u_ = tune_.unroll[kSlotNbr];             \
    if (fuse_dens_) {                                                                   \
      if (u_ == 2) launch_fluid(b_, k_s_neighbors<2, true, FLAT>, __VA_ARGS__);         \
      else if (u_ == 8) launch_fluid(b_, k_s_neighbors<8, true, FLAT>, __VA_ARGS__);    \
      else launch_fluid(b_, k_s_neighbors<4, true, FLAT>, __VA_ARGS__);                 \
    } else {                                                                            \
      if (u_ == 2) launch_fluid(b_, k_s_neighbors<2, false, FLAT>, __VA_ARGS__);        \
      else if (u_ == 8) launch_fluid(b_, k_s_neighbors<8, false, FLAT>, __VA_ARGS__);   \
      else launch_fluid(b_, k_s_neighbors<4, false, FLAT>, __VA_ARGS__);                \
    }                                                                                   \
  } while (0)
#define PF_NBR(...)                                                                     \
  do {                                                                                  \
    if (tune_.nbr_flat) PF_NBR_FLAT(true, __VA_ARGS__);                                 \
    else PF_NBR_FLAT(false, __VA_ARGS__);                                               \
  } while (0)
// XSPH, without the boundary-volume gather when the world has no boundaries.
#define PF_XSPH(...)                                                                    \
  do {                                                                                  \
    const uint32_t b_ = tune_.block[kSlotVel], u_ = tune_.unroll[kSlotVel];             \
    if (any_static_bnd_ || any_dyn_bnd_) {                                              \
      if (u_ == 2) launch_fluid(b_, k_s_xsph<2, true>, __VA_ARGS__);                    \
      else if (u_ == 8) launch_fluid(b_, k_s_xsph<8, true>, __VA_ARGS__);               \
      else launch_fluid(b_, k_s_xsph<4, true>, __VA_ARGS__);                            \
    } else {                                                                            \
      if (u_ == 2) launch_fluid(b_, k_s_xsph<2, false>, __VA_ARGS__);                   \
      else if (u_ == 8) launch_fluid(b_, k_s_xsph<8, false>, __VA_ARGS__);              \
      else launch_fluid(b_, k_s_xsph<4, false>, __VA_ARGS__);                           \
    }                                                                                   \
  } while (0)
// The position pass, without the boundary-reaction code when no fluid has
// boundaries.
#define PF_DELTA(...)                                                                   \
  do {                                                                                  \
    const uint32_t b_ = tune_.block[kSlotDelta], u_ = tune_.unroll[kSlotDelta];         \
    if (any_react_) {                                                                   \
      if (u_ == 2) launch_fluid(b_, k_s_delta<2, true>, __VA_ARGS__);                   \
      else if (u_ == 8) launch_fluid(b_, k_s_delta<8, true>, __VA_ARGS__);              \
      else launch_fluid(b_, k_s_delta<4, true>, __VA_ARGS__);                           \
    } else {                                                                            \
      if (u_ == 2) launch_fluid(b_, k_s_delta<2, false>, __VA_ARGS__);                  \
      else if (u_ == 8) launch_fluid(b_, k_s_delta<8, false>, __VA_ARGS__);             \
      else launch_fluid(b_, k_s_delta<4, false>, __VA_ARGS__);                          \
    }                                                                                   \
  } while (0)

void World::run_fluid_neighbors(const WorldView& V, uint32_t s) {
  if (tune_.path == 1) {
    launch_tiles_build(V, s);
  } else {
    PF_NBR(V, s);
  }
}

void World::run_fluid_lambda_delta(const WorldView& V, uint32_t r, uint32_t s, uint32_t it) {
  if (tune_.path == 1) {
    launch_tiled(k_t_lambda, kSmemLambda, V, r, s, it);
    launch_tiled(k_t_delta, kSmemDelta, V, r, s, it);
  } else {
    // the list build formed rank 0's first density and lambda
    if (!(fuse_dens_ && r == 0 && it == 0)) PF_BY_UNROLL(kSlotLambda, k_s_lambda, V, r, s, it);
    PF_DELTA(V, r, s, it, 1u);
  }
}

void World::run_fluid_xsph(const WorldView& V, uint32_t r, uint32_t s) {
  if (tune_.path == 1) {
    launch_tiled(k_t_xsph, kSmemXsph, V, r, s);
  } else {
    PF_XSPH(V, r, s);
  }
}

WorldView World::group_view(const WorldView& V, size_t g) const {
  WorldView W = V;
  W.fchunk = base_.fchunk + groups_[g].first;
  W.n_fchunk = groups_[g].second - groups_[g].first;
  return W;
}

WorldView World::rest_view(const WorldView& V) const {
  if (!grouping()) return V;
  WorldView W = V;
  W.fchunk = base_.fchunk + n_pure_chunks_;
  W.n_fchunk = base_.n_fchunk - n_pure_chunks_;
  return W;
}

// Groups of consecutive single-fluid scenes of about tune_.group fluid
// particles (whole scenes), and each scene's grouped flag.
void World::apply_grouping() {
  groups_.clear();
  for (auto& S : h_scenes_) S.grouped = 0;
  if (tune_.path != 0 || tune_.group == 0 || pure_end_.empty()) return;
  uint32_t c0 = 0;
  uint64_t parts = 0;
  for (size_t i = 0; i < pure_end_.size(); ++i) {
    parts += pure_parts_[i];
    h_scenes_[pure_scene_[i]].grouped = 1;
    if (parts >= tune_.group || i + 1 == pure_end_.size()) {
      groups_.push_back({c0, pure_end_[i]});
      c0 = pure_end_[i];
      parts = 0;
    }
  }
}

// The substep of the grouped scenes, group by group: the list build, the
// solver iterations (density + lambda, position correction with its fused
// apply and colliders), advect, XSPH and its apply. A group's lists and
// records stay in L2 across these passes. `apply` = 0 leaves x* and the
// velocities alone (the autotuner's timing).
void World::run_groups(const WorldView& V, uint32_t s, bool apply) {
  for (size_t g = 0; g < groups_.size(); ++g) {
    const WorldView G = group_view(V, g);
    PF_NBR(G, s);
    for (uint32_t it = 0; it < max_iter_; ++it) {
      if (!(fuse_dens_ && it == 0)) PF_BY_UNROLL(kSlotLambda, k_s_lambda, G, 0u, s, it);
      PF_DELTA(G, 0u, s, it, apply ? 1u : 0u);
    }
    if (apply) launch_fluid(kBlock, k_advect_chunks, G, s);
    if (any_visc_) {
      PF_XSPH(G, 0u, s);
      if (apply) launch_slots(k_xsph_apply, G.n_fchunk * kSegAlign, stream_, G, 0u, s);
    }
  }
}

// Tuning cache. With PFSIM_TUNE_CACHE naming a file, the tuner first looks
// there for a line
//   pfsim-tune-1 <gpu> <sms> <config> <n> <path> <block x4> <unroll x4> <group> <flat> <wide>
// keyed by the GPU (its name, blanks as '_', and its SM count), the world's
// configuration (a 64-bit FNV-1a hash, in hex, of its scenes' capacities,
// substeps, iterations, build-time grid windows, fluids and contacts, and
// of the world's feature flags) and its particle count. A world whose key
// is there takes the last such line's choices and times nothing; a world
// that times its candidates appends its line. A line that does not parse,
// or whose choices this world cannot run, is passed over. The choices set
// the speed: both paths build the same neighbour lists, and on the slot
// path every block size, fetch depth, group size and entry width steps to
// the same bits.
std::string World::tune_key() const {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](uint64_t v) {
    for (int b = 0; b < 8; ++b) {
      h ^= (v >> (8 * b)) & 0xffu;
      h *= 1099511628211ull;
    }
  };
  mix(h_scenes_.size());
  for (const DevScene& S : h_scenes_) {
    mix(S.cap);
    mix(S.seg_end - S.seg_start);
    mix(S.substeps);
    mix(S.iterations);
    mix(S.has_grid);
    for (int a = 0; a < 3; ++a) mix(S.dims[a]);
    mix(S.fluid_count);
    mix(S.contact);
  }
  mix(h_fluids_.size());
  for (const DevFluid& F : h_fluids_) mix(F.rank);
  mix((uint64_t)any_visc_ | (uint64_t)any_vort_ << 1 | (uint64_t)any_imp_ << 2 | (uint64_t)any_multi_fluid_ << 3 |
      (uint64_t)fuse_dens_ << 4 | (uint64_t)any_contact_ << 5);
  mix(pure_parts_.size());
  for (uint64_t p : pure_parts_) mix(p);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop{};
  std::string gpu = "unknown";
  if (cudaGetDeviceProperties(&prop, dev) == cudaSuccess) {
    gpu.assign(prop.name, strnlen(prop.name, sizeof(prop.name)));
    for (char& c : gpu)
      if (c == ' ' || c == '\t') c = '_';
    if (gpu.empty()) gpu = "unknown";
  }
  char buf[320];
  std::snprintf(buf, sizeof buf, "%s %d %016llx %u", gpu.c_str(), sm_count(), (unsigned long long)h, n_);
  return buf;
}

bool World::load_tuning(const char* file, const std::string& key) {
  FILE* f = std::fopen(file, "r");
  if (!f) return false;
  uint64_t pure_total = 0;
  for (uint64_t p : pure_parts_) pure_total += p;
  auto valid = [&](const Tuning& t) {
    if (t.path > 1 || t.nbr_flat > 1 || t.nbr_wide > 1) return false;
    if (t.path == 1 && (any_vort_ || any_imp_ || any_multi_fluid_)) return false;
    for (int q = 0; q < 4; ++q) {
      const uint32_t b = t.block[q], u = t.unroll[q];
      if (b != 128 && b != 256 && b != 512) return false;
      if (u != 2 && u != 4 && u != 8) return false;
      if (u == 8 && b == 512) return false;  // never a candidate
    }
    return t.group == 0 || (!pure_end_.empty() && t.group < pure_total);
  };
  bool found = false;
  Tuning hit;
  char line[512];
  while (std::fgets(line, sizeof line, f)) {
    char tag[32], gpu[256], cfg[32];
    int sms = 0;
    unsigned n = 0;
    Tuning t;
    const int got = std::sscanf(line, "%31s %255s %d %31s %u %u %u %u %u %u %u %u %u %u %u %u %u", tag, gpu, &sms, cfg, &n,
                                &t.path, &t.block[0], &t.block[1], &t.block[2], &t.block[3], &t.unroll[0], &t.unroll[1],
                                &t.unroll[2], &t.unroll[3], &t.group, &t.nbr_flat, &t.nbr_wide);
    if (got != 17 || std::strcmp(tag, "pfsim-tune-1") != 0) continue;
    char k[320];
    std::snprintf(k, sizeof k, "%s %d %s %u", gpu, sms, cfg, n);
    if (key != k || !valid(t)) continue;
    hit = t;
    found = true;
  }
  std::fclose(f);
  if (found) tune_ = hit;
  return found;
}

void World::store_tuning(const char* file, const std::string& key) const {
  char line[512];
  const Tuning& t = tune_;
  const int len = std::snprintf(line, sizeof line, "pfsim-tune-1 %s %u %u %u %u %u %u %u %u %u %u %u %u\n", key.c_str(),
                                t.path, t.block[0], t.block[1], t.block[2], t.block[3], t.unroll[0], t.unroll[1],
                                t.unroll[2], t.unroll[3], t.group, t.nbr_flat, t.nbr_wide);
  if (len <= 0 || len >= (int)sizeof line) return;
  // one short line written at once in append mode: lines of worlds tuned at
  // the same time by other processes do not interleave
  FILE* f = std::fopen(file, "a");
  if (!f) {
    if (verbose()) std::fprintf(stderr, "pfsim: tuning cache %s not writable\n", file);
    return;
  }
  std::fwrite(line, 1, (size_t)len, f);
  std::fclose(f);
}

// Autotuner: on the world's own state (one grid rebuild, as the next
// substep would do; the permutation is canonical, so no result changes),
// time each slot kernel (list build, density + lambda, position correction,
// XSPH) at every block size and fetch depth and keep each kernel's fastest;
// then one substep's slot passes with 16-bit and with 32-bit list entries,
// and keep the faster; then time one substep's worth of the warp-tile path
// against the tuned slot path and keep the faster. The passes write only
// per-substep scratch (lists, lambda, density, deltas), which every substep
// rebuilds; none moves a predicted position (the warp-tile trial needs them
// where the sort saw them).
pf_status World::tune() {
  tuned_ = true;
  if (!any_fluid_ || n_ == 0) return PF_OK;
  if (const char* e = std::getenv("PFSIM_NBR_PATH")) {  // fixed choice for measurements
    tune_.path = ((uint32_t)std::atoi(e) == 1 && !any_vort_ && !any_imp_ && !any_multi_fluid_) ? 1u : 0u;
    uint32_t blk = 256, unr = 4;
    if (const char* b = std::getenv("PFSIM_SLOT_BLOCK")) blk = (uint32_t)std::atoi(b);
    if (blk != 128 && blk != 256 && blk != 512) blk = 256;
    if (const char* u = std::getenv("PFSIM_SLOT_UNROLL")) unr = (uint32_t)std::atoi(u);
    if (unr != 2 && unr != 8) unr = 4;
    for (int q = 0; q < 4; ++q) {
      tune_.block[q] = blk;
      tune_.unroll[q] = unr;
    }
    tune_.group = 0;
    if (const char* g = std::getenv("PFSIM_GROUP")) tune_.group = (uint32_t)std::atoi(g);
    tune_.nbr_flat = 0;
    if (const char* fl = std::getenv("PFSIM_NBR_FLAT")) tune_.nbr_flat = std::atoi(fl) ? 1u : 0u;
    tune_.nbr_wide = 0;
    if (const char* nw = std::getenv("PFSIM_NBR_WIDE")) tune_.nbr_wide = std::atoi(nw) ? 1u : 0u;
    apply_grouping();
    return PF_OK;
  }
  const char* cache = std::getenv("PFSIM_TUNE_CACHE");
  if (cache && !*cache) cache = nullptr;
  const std::string key = cache ? tune_key() : std::string();
  if (cache && load_tuning(cache, key)) {
    apply_grouping();
    if (verbose()) std::fprintf(stderr, "pfsim: tuning of %s from %s\n", key.c_str(), cache);
    return PF_OK;
  }
  PF_TRY(tune_trials());
  if (cache) store_tuning(cache, key);
  return PF_OK;
}

pf_status World::tune_trials() {
  run_sort_and_permute(parity_, false);
  parity_ ^= 1;
  const WorldView V = view(parity_);
  const uint32_t rank = h_fluids_[0].rank;
  // the density passes below overwrite the densities the first substep's
  // surface tension reads: keep them in the sort-key buffer (free until the
  // next sort)
  float* keep = reinterpret_cast<float*>(base_.keys);
  PF_CUDA(cudaMemcpyAsync(keep, V.cur.dens, 4ull * n_, cudaMemcpyDeviceToDevice, stream_));
  auto timed = [&](auto&& body, float* out) -> pf_status {
    float t = 0;
    for (int rep = 0; rep < 2; ++rep) {
      PF_CUDA(cudaEventRecord(ev0_, stream_));
      body();
      PF_CUDA(cudaEventRecord(ev1_, stream_));
      PF_CUDA(cudaEventSynchronize(ev1_));
      float ms = 0;
      PF_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
      t = rep == 0 ? ms : std::min(t, ms);
    }
    PF_CUDA(cudaGetLastError());
    *out = t;
    return PF_OK;
  };
  const uint32_t iters = std::max(max_iter_, 1u);
  const bool vel = any_visc_ || any_vort_;
  // the slot path, kernel by kernel (the list first: the others read it)
  tune_.path = 0;
  const uint32_t blocks[3] = {128, 256, 512}, unrolls[3] = {2, 4, 8};
  float slot_total = 0;
  for (int kind = 0; kind < 4; ++kind) {
    if (kind == kSlotVel && !vel) continue;
    float best = 1e30f;
    uint32_t bb = 256, bu = 4, bf = 0;
    for (uint32_t flat = 0; flat < (kind == kSlotNbr ? 2u : 1u); ++flat)
    for (uint32_t b : blocks)
      for (uint32_t u : unrolls) {
        if (u == 8 && b == 512) continue;
        tune_.block[kind] = b;
        tune_.unroll[kind] = u;
        if (kind == kSlotNbr) tune_.nbr_flat = flat;
        float t = 0;
        PF_TRY(timed(
            [&] {
              if (kind == kSlotNbr) PF_NBR(V, 0u);
              else if (kind == kSlotLambda) PF_BY_UNROLL(kSlotLambda, k_s_lambda, V, rank, 0u, 0u);
              else if (kind == kSlotDelta) PF_DELTA(V, rank, 0u, 0u, 0u);
              else PF_XSPH(V, rank, 0u);
            },
            &t));
        if (t < best) {
          best = t;
          bb = b;
          bu = u;
          bf = kind == kSlotNbr ? tune_.nbr_flat : 0u;
        }
      }
    tune_.block[kind] = bb;
    tune_.unroll[kind] = bu;
    if (kind == kSlotNbr) tune_.nbr_flat = bf;
    const uint32_t reps = kind == kSlotDelta ? iters : (kind == kSlotLambda ? iters - (fuse_dens_ ? 1u : 0u) : 1u);
    slot_total += best * reps;
  }
  // L2-sized groups of the single-fluid scenes: time their neighbour passes
  // group by group against one launch per pass over all of them
  tune_.group = 0;
  uint64_t pure_total = 0;
  for (uint64_t p : pure_parts_) pure_total += p;
  if (!pure_end_.empty() && !std::getenv("PFSIM_NO_GROUPS")) {
    float best = 1e30f;
    uint32_t best_g = 0;
    const uint32_t cands[4] = {0u, 393216u, 786432u, 1572864u};
    for (uint32_t gsz : cands) {
      if (gsz && gsz >= pure_total) continue;  // one group is no grouping
      tune_.group = gsz ? gsz : 0xffffffffu;   // 0 here: all pure scenes as one launch
      apply_grouping();
      float t = 0;
      PF_TRY(timed([&] { run_groups(V, 0u, false); }, &t));
      if (t < best) {
        best = t;
        best_g = gsz;
      }
    }
    tune_.group = best_g;
    apply_grouping();
  }
  // the list's entry width: one substep's slot passes timed with 16-bit
  // offsets (where a warp's rows allow them) and with 32-bit slots. As in
  // the trials above, the position pass only forms its corrections (no
  // apply): the tuner leaves the predicted positions as the sort saw them,
  // which the warp-tile trial below relies on (its halo rows come from the
  // sorted cells).
  {
    auto substep = [&] {
      const WorldView W = view(parity_);
      PF_NBR(W, 0u);
      for (uint32_t it = 0; it < iters; ++it) {
        if (!(fuse_dens_ && it == 0)) PF_BY_UNROLL(kSlotLambda, k_s_lambda, W, rank, 0u, 0u);
        PF_DELTA(W, rank, 0u, 0u, 0u);
      }
      if (vel) PF_XSPH(W, rank, 0u);
    };
    float t16 = 0, t32 = 0;
    tune_.nbr_wide = 0;
    PF_TRY(timed(substep, &t16));
    tune_.nbr_wide = 1;
    PF_TRY(timed(substep, &t32));
    // 32-bit entries move half again as many bytes, so they must win
    // clearly (a few per cent can be the noise of two timings)
    tune_.nbr_wide = t32 < 0.97f * t16 ? 1u : 0u;
    slot_total = tune_.nbr_wide ? t32 : t16;
  }
  // the warp-tile path has no vorticity or surface pass and reads one shared
  // lambda buffer: worlds with those, or with a scene of several fluids,
  // stay on slots
  if (!(any_vort_ || any_imp_ || any_multi_fluid_)) {
    tune_.path = 1;
    float t = 0;
    PF_TRY(timed(
        [&] {
          run_fluid_neighbors(V, 0);
          for (uint32_t it = 0; it < iters; ++it) run_fluid_lambda_delta(V, rank, 0, 0);
          if (vel) run_fluid_xsph(V, rank, 0);
        },
        &t));
    tune_.path = t < slot_total ? 1u : 0u;
    apply_grouping();  // groups are a slot-path schedule
  }
  PF_CUDA(cudaMemcpyAsync(V.cur.dens, keep, 4ull * n_, cudaMemcpyDeviceToDevice, stream_));
  return PF_OK;
}

template <typename K, typename... A>
void World::launch_tiled(K kernel, size_t smem, const WorldView& V, A... args) {
  const uint32_t grid = std::max<uint32_t>(
      1, std::min<uint32_t>(div_up(base_.max_tiles, kTileWarps), (uint32_t)sm_count() * 16));
  kernel<<<grid, kTileThreads, smem, stream_>>>(V, args...);
  ++t_launches;
}

// Keys of the current predicted positions, stable sort, permute into the
// other buffer; `parity` names the current buffer.
void World::run_sort_and_permute(uint32_t parity, bool bbox_ready) {
  const WorldView V = view(parity);
  const uint32_t K = (uint32_t)h_scenes_.size();
  if (!bbox_ready) launch_slots(k_bbox, n_, stream_, V);
  k_grid_fit<<<div_up(K, 128), 128, 0, stream_>>>(V, K);
  ++t_launches;
  cudaMemsetAsync(sort_.counters, 0, 4ull * kNumCounters, stream_);
  cudaMemsetAsync(sort_.digit_count, 0, 4ull * kRadixMaxPasses * kRadixMaxDigits, stream_);
  k_keys<<<keys_grid(n_, kBlock), kBlock, 4ull * radix_.passes * radix_.digits, stream_>>>(V, digit_hist(radix_, sort_));
  launch_grid_sort(V.keys, n_, cells_, radix_, V.ccount, V.cstart, V.perm, sort_, stream_);
  t_launches += 1 + grid_sort_launches(radix_, n_);  // the keys, then the sort
  launch_slots(k_permute, n_, stream_, V);
}

void World::run_init_pass() {
  // FluidSystem.ts:228-231 + loop.ts:237: static boundaries get their volume
  // once, from committed positions, after a grid rebuild.
  if (!any_static_bnd_) return;
  run_sort_and_permute(parity_, false);
  parity_ ^= 1;
  launch_slots(k_boundary_volume, n_, stream_, view(parity_), 1u, 0u);
}

// ClothSystem.ts:193-212: the stretch colours, then the bending colours.
void World::launch_cloth_rank(const WorldView& V, uint32_t r, uint32_t s, uint32_t it, cudaStream_t st) {
  for (auto& rg : cloth_ranges_[r])
    if (rg.second > rg.first) {
      k_cloth<<<div_up(rg.second - rg.first, kBlock), kBlock, 0, st>>>(V, rg.first, rg.second, s, it);
      ++t_launches;
    }
  if (r < bend_ranges_.size())
    for (auto& rg : bend_ranges_[r])
      if (rg.second > rg.first) {
        k_bend<<<div_up(rg.second - rg.first, kBlock), kBlock, 0, st>>>(V, rg.first, rg.second, s, it);
        ++t_launches;
      }
  if (r < teth_ranges_.size())
    for (auto& rg : teth_ranges_[r])
      if (rg.second > rg.first) {
        k_tether<<<div_up(rg.second - rg.first, kBlock), kBlock, 0, st>>>(V, rg.first, rg.second, s, it);
        ++t_launches;
      }
}

void World::launch_aero(const WorldView& V, uint32_t stage, uint32_t s) {
  const auto& rg = aero_ranges_[stage];
  if (rg.second <= rg.first) return;
  k_aero<<<div_up(rg.second - rg.first, kBlock), kBlock, 0, stream_>>>(V, rg.first, rg.second, s);
  ++t_launches;
}

void World::run_substep(uint32_t s, uint32_t parity) {
  WorldView V = view(parity);
  launch_slots(k_predict, n_, stream_, V, s);
  if (any_soft_local_) launch_slots(k_rot_predict, base_.n_grp, stream_, V, s);
  if (any_grid_) {
    run_sort_and_permute(parity, true);
    V = view(parity ^ 1);
  } else {
    launch_slots(k_reset_sums, n_, stream_, V);
  }
  // the other fluid scenes' passes run over their chunks (all fluid chunks
  // without groups); the grouped scenes run after the cloth fork below
  const WorldView VF = rest_view(V);
  // preSolve: contacts first (loop.ts:196-223), then the materials'
  if (any_contact_) {
    const uint32_t K = (uint32_t)h_scenes_.size();
    k_con_gen<<<n_ / kBlock, kBlock, 0, stream_>>>(V, s);
    k_con_scan<<<K, 1024, 0, stream_>>>(V, s);
    launch_slots(k_con_stab, n_, stream_, V, s);
    launch_slots(k_con_apply2, n_, stream_, V, s);
    t_launches += 2;
  }
  launch_aero(V, 0, s);
  if (any_dyn_bnd_) launch_slots(k_boundary_volume, n_, stream_, V, 0u, s);
  if (any_fluid_) run_fluid_neighbors(VF, s);
  // FluidSystem.ts:233-255: surface tension and adhesion, once per substep
  if (any_imp_)
    for (uint32_t r = 0; r < max_rank_; ++r) {
      bool st = false, imp = false;
      for (auto& F : h_fluids_) {
        st = st || (F.rank == r && F.has_st);
        imp = imp || (F.rank == r && (F.has_st || F.has_ad));
      }
      if (!imp) continue;
      if (st) PF_BY_UNROLL(kSlotVel, k_s_color_normal, VF, r, s);
      PF_BY_UNROLL(kSlotVel, k_s_impulses, VF, r, s);
      launch_slots(k_imp_apply, VF.n_fchunk * kSegAlign, stream_, VF, r, s);
    }
  launch_aero(V, 1, s);
  // pair multipliers reset every substep (buildImplicitResetPairLambdaKernel)
  if (any_soft_local_ && pair_entries_) cudaMemsetAsync(base_.pair_lambda, 0, 16ull * pair_entries_, stream_);
  if (any_soft_global_) cudaMemsetAsync(base_.lambda_g, 0, 16ull * n_, stream_);
  if (base_.n_cons) cudaMemsetAsync(base_.c_lambda, 0, 4ull * base_.n_cons, stream_);
  if (base_.n_bend) cudaMemsetAsync(base_.b_lambda, 0, 4ull * base_.n_bend, stream_);
  if (base_.n_teth) cudaMemsetAsync(base_.t_lambda, 0, 4ull * base_.n_teth, stream_);
  // iterations
  // Cloth-only scenes (and material-free scenes with colliders) share no
  // slot with the others: their colour sweeps and collider passes run on a
  // second stream, overlapping the fluid and soft-body iterations.
  const bool fork = side_ok_ && side_stream_;
  if (fork) {
    cudaEventRecord(ev_fork_, stream_);
    cudaStreamWaitEvent(side_stream_, ev_fork_, 0);
    for (uint32_t it = 0; it < max_iter_; ++it) {
      for (uint32_t r = 0; r < cloth_ranges_.size(); ++r) launch_cloth_rank(V, r, s, it, side_stream_);
      if (any_contact_) launch_slots(k_con_solve, n_, side_stream_, V, s, it);
      if (any_unfused_prims_) launch_slots(k_collide, base_.n_cchunk * kSegAlign, side_stream_, V, s, it);
    }
  }
  // the grouped single-fluid scenes' whole substep, beside the cloth sweeps
  if (grouping()) run_groups(V, s, true);
  for (uint32_t it = 0; it < max_iter_; ++it) {
    for (uint32_t r = 0; r < max_rank_; ++r) {
      bool has_fluid = false, has_local = false, has_global = false;
      for (auto& F : h_fluids_) has_fluid = has_fluid || F.rank == r;
      for (auto& D : h_softs_) {
        has_local = has_local || (D.rank == r && D.local);
        has_global = has_global || (D.rank == r && !D.local);
      }
      if (has_fluid && VF.n_fchunk) {
        run_fluid_lambda_delta(VF, r, s, it);
        // on the slot path the position pass applies homogeneous scenes itself
        const bool slot = tune_.path == 0;
        bool rest = !slot;
        for (auto& S : h_scenes_) rest = rest || (S.fluid_count && !S.homog);
        if (rest) launch_slots(k_fluid_apply, VF.n_fchunk * kSegAlign, stream_, VF, r, s, it, slot ? 1u : 0u);
      }
      if (has_local) {
        launch_slots(k_sm_moment, base_.n_grp, stream_, V, r, s, it);
        if (base_.n_mem_ids) {  // mem_lanes_ lanes per cluster member
          const uint32_t grid = (uint32_t)(((uint64_t)mem_lanes_ * base_.n_mem_ids + kBlock - 1) / kBlock);
          if (mem_lanes_ == 1) k_sm_gather<1><<<grid, kBlock, 0, stream_>>>(V, r, s, it);
          else if (mem_lanes_ == 2) k_sm_gather<2><<<grid, kBlock, 0, stream_>>>(V, r, s, it);
          else if (mem_lanes_ == 4) k_sm_gather<4><<<grid, kBlock, 0, stream_>>>(V, r, s, it);
          else if (mem_lanes_ == 8) k_sm_gather<8><<<grid, kBlock, 0, stream_>>>(V, r, s, it);
          else if (mem_lanes_ == 16) k_sm_gather<16><<<grid, kBlock, 0, stream_>>>(V, r, s, it);
          else k_sm_gather<32><<<grid, kBlock, 0, stream_>>>(V, r, s, it);
          ++t_launches;
        }
        launch_slots(k_sm_qp, base_.n_grp, stream_, V, r, s, it);
      }
      if (has_global && base_.n_bodies) {
        k_body_frame<<<base_.n_bodies, 256, 0, stream_>>>(V, r, s, it, 1u);
        k_global_apply<<<base_.n_bodies, 256, 0, stream_>>>(V, r, s, it);
        t_launches += 2;
      }
      if (!fork && r < cloth_ranges_.size()) launch_cloth_rank(V, r, s, it, stream_);
    }
    if (!fork && any_contact_) launch_slots(k_con_solve, n_, stream_, V, s, it);
    if (!fork && any_unfused_prims_) launch_slots(k_collide, base_.n_cchunk * kSegAlign, stream_, V, s, it);
  }
  if (fork) {
    cudaEventRecord(ev_join_, side_stream_);
    cudaStreamWaitEvent(stream_, ev_join_, 0);
  }
  launch_slots(k_advect, n_, stream_, V, s);
  for (uint32_t r = 0; r < max_rank_; ++r) {
    bool has_velocity = false, has_vort = false, has_local = false;
    for (auto& F : h_fluids_) {
      has_velocity = has_velocity || (F.rank == r && (F.has_visc || F.has_vort));
      has_vort = has_vort || (F.rank == r && F.has_vort);
    }
    for (auto& D : h_softs_) has_local = has_local || (D.rank == r && D.local);
    if (has_velocity && VF.n_fchunk) {
      run_fluid_xsph(VF, r, s);
      if (has_vort) PF_BY_UNROLL(kSlotVel, k_s_vort_grad, VF, r, s);
      launch_slots(k_xsph_apply, VF.n_fchunk * kSegAlign, stream_, VF, r, s);
    }
    if (has_local) {
      launch_slots(k_rot_advect, base_.n_grp, stream_, V, s);
      if (base_.n_bodies) {
        k_body_frame<<<base_.n_bodies, 256, 0, stream_>>>(V, r, s, 0u, 0u);
        ++t_launches;
      }
    }
    if (r < damp_ranges_.size() && damp_ranges_[r].second > damp_ranges_[r].first) {
      const auto& rg = damp_ranges_[r];
      const uint32_t g = div_up(rg.second - rg.first, kBlock);
      k_damp_mean<<<g, kBlock, 0, stream_>>>(V, rg.first, rg.second, s);
      k_damp_apply<<<g, kBlock, 0, stream_>>>(V, rg.first, rg.second, s);
      t_launches += 2;
    }
  }
  // friction: the velocity sums reset, contact friction, collider friction,
  // applied (loop.ts:226-230)
  if (any_contact_) launch_slots(k_con_friction, n_, stream_, V, s);
  if (any_prims_ || any_contact_) launch_slots(k_friction, n_, stream_, V, s);
  if (any_prims_) {
    const uint32_t K = (uint32_t)h_scenes_.size();
    k_tick<<<div_up(K, 128), 128, 0, stream_>>>(V, K, s);
    ++t_launches;
  }
}

pf_status World::step(double dt) {
  if (!(dt > 0) || !std::isfinite(dt))
    return fail(PF_ERR_INVALID, "SimLoop: step dt must be a positive finite number, got " + std::to_string(dt));
  PF_TRY(maybe_grow_windows());
  PF_TRY(upload_params(dt));
  PF_CUDA(cudaEventRecord(ev0_, stream_));
  if (!tuned_) {
    PF_TRY(tune());
    PF_TRY(upload_params(dt));  // the scenes' grouped flags the tuner set
  }
  if (!inited_) {
    run_init_pass();
    inited_ = true;
    for (auto* sp : specs_) sp->initialized = true;
    for (auto& S : h_scenes_) S.init_pending = 0;
  }
  const uint32_t flips = any_grid_ ? (max_sub_ & 1u) : 0u;
  auto body = [&](uint32_t p0) {
    t_launches = 0;
    launch_frame_start_at(p0);
    uint32_t p = p0;
    for (uint32_t s = 0; s < max_sub_; ++s) {
      run_substep(s, p);
      if (any_grid_) p ^= 1;
    }
  };
  if (use_graph_) {
    // Both start parities are captured on the first step, so later steps
    // only launch (no capture runs while a host thread builds another world).
    // After the grid windows grew, the captured steps are captured again
    // and, where the launches keep their shape, updated in place (cheaper
    // than a new instantiation).
    const uint32_t parities[2] = {parity_, parity_ ^ flips};
    for (uint32_t i = 0; i < (flips ? 2u : 1u); ++i) {
      const uint32_t p = parities[i];
      cudaGraphExec_t& g = graph_[p];
      if (g && !graphs_stale_) continue;
      const auto t_cap = std::chrono::steady_clock::now();
      const bool updating = g != nullptr;
      cudaGraph_t graph;
      PF_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      body(p);
      launches_per_step_ = t_launches;
      PF_CUDA(cudaStreamEndCapture(stream_, &graph));
      if (g) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(g, graph, &info) != cudaSuccess) {
          cudaGetLastError();
          cudaGraphExecDestroy(g);
          g = nullptr;
        }
      }
      const bool updated = updating && g;
      cudaError_t e = cudaSuccess;
      if (!g) e = cudaGraphInstantiate(&g, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) return fail(PF_ERR_CUDA, std::string("SimLoop: graph instantiate: ") + cudaGetErrorString(e));
      if (verbose())
        std::fprintf(stderr, "pfsim: step graph %s: %.2f ms\n",
                     updated ? "updated" : (updating ? "instantiated again (update refused)" : "instantiated"),
                     std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_cap).count());
    }
    graphs_stale_ = false;
    PF_CUDA(cudaGraphLaunch(graph_[parity_], stream_));
  } else {
    body(parity_);
    launches_per_step_ = t_launches;
  }
  parity_ ^= flips;
  PF_CUDA(cudaEventRecord(ev1_, stream_));
  if (any_grid_) {
    // this step's bounds, into its ring buffer, with an event a later step
    // queries (the host reads a buffer only once its copy has landed, and
    // only before queueing the copy that reuses it)
    const size_t K6 = 6 * h_scenes_.size();
    const uint32_t q = (uint32_t)(steps_done_ % kBoundsRing);
    PF_CUDA(cudaMemcpyAsync(h_pinned_bbox_ + K6 * q, base_.bbox_last, sizeof(int32_t) * K6, cudaMemcpyDeviceToHost,
                            stream_));
    PF_CUDA(cudaEventRecord(ev_bounds_[q], stream_));
  }
  ++steps_done_;
  PF_CUDA(cudaGetLastError());
  return PF_OK;
}

// Before a step: a grid scene whose particles' cell bounds (as the window
// fit of the newest step whose bounds have arrived saw them) come within a
// margin of its window's size on some axis gets a window twice their spread
// there, centred on them, so it never has to clamp (the reference's hash
// grid is unbounded). The margin covers the spread's growth over the steps
// from those bounds to the end of the one about to be queued, and one more.
// Windows past 2^27 cells stay as they are (their keys clamp and flag).
pf_status World::maybe_grow_windows() {
  if (!any_grid_ || steps_done_ == 0) return PF_OK;
  // the newest step whose bounds have landed (the ring holds the last
  // kBoundsRing steps; one that is still queued is skipped, not waited for)
  uint64_t seen_step = 0;
  bool found = false;
  const uint64_t oldest = steps_done_ > kBoundsRing ? steps_done_ - kBoundsRing : 0;
  for (uint64_t t = steps_done_; t-- > oldest;) {
    if (t + 1 <= bounds_seen_) break;  // looked at already
    const cudaError_t e = cudaEventQuery(ev_bounds_[t % kBoundsRing]);
    if (e == cudaSuccess) {
      seen_step = t;
      found = true;
      break;
    }
    if (e != cudaErrorNotReady) PF_CUDA(e);
  }
  if (!found) return PF_OK;
  // steps from those bounds to the end of the step about to be queued
  const uint64_t ahead = steps_done_ - seen_step;
  const uint64_t since = bounds_seen_ ? seen_step + 1 - bounds_seen_ : 1;  // steps since the last look
  bounds_seen_ = seen_step + 1;
  const int32_t* seen = h_pinned_bbox_ + 6 * h_scenes_.size() * (seen_step % kBoundsRing);
  bool any = false;
  for (uint32_t s = 0; s < h_scenes_.size(); ++s) {
    DevScene& S = h_scenes_[s];
    if (!S.has_grid) continue;
    const int32_t* b = seen + 6 * s;
    int64_t lo[3], dims[3];
    bool grow = false;
    for (int a = 0; a < 3; ++a) {
      const int64_t mn = b[a], mx = b[a + 3], d = S.dims[a];
      lo[a] = S.lo0[a];
      dims[a] = d;
      if (mn > mx) continue;  // no particle
      // within two cells of clamping, plus the spread's growth per step
      // over the steps from these bounds to the end of the next one, and
      // one step more; a fluid that walls hold stops growing there
      const int64_t ext = mx - mn + 1;
      int32_t& prev = grow_prev_ext_[3 * s + a];
      const int64_t rate = prev > 0 ? (std::max<int64_t>(0, ext - prev) + (int64_t)since - 1) / (int64_t)since : 0;
      prev = (int32_t)ext;
      if (ext + (int64_t)(ahead + 1) * rate + 4 <= d) continue;
      dims[a] = std::max<int64_t>(d, 2 * ext + 8);
      lo[a] = ((mn + mx) >> 1) - dims[a] / 2;
      grow = true;
    }
    if (!grow) continue;
    const uint64_t cells = (uint64_t)dims[0] * dims[1] * dims[2];
    if (cells > (1ull << 27)) continue;
    for (int a = 0; a < 3; ++a) grow_prev_ext_[3 * s + a] = 0;
    bool fits = true;
    for (int a = 0; a < 3; ++a) fits = fits && lo[a] > INT32_MIN / 2 && lo[a] + dims[a] < INT32_MAX / 2;
    if (!fits) continue;
    const float org[3] = {S.ox, S.oy, S.oz};
    double big = 0;
    for (int a = 0; a < 3; ++a) {
      S.lo0[a] = S.lo[a] = (int32_t)lo[a];
      S.dims[a] = (uint32_t)dims[a];
      big = std::max(big, std::fabs((double)org[a]) + std::max(std::fabs((double)lo[a]),
                                                               std::fabs((double)(lo[a] + dims[a]))) * S.cell);
    }
    S.cells = (uint32_t)cells;
    S.prune_slack = f32(big * (1.0 / 65536.0) + 1e-9);
    any = true;
  }
  if (!any) return PF_OK;
  return relayout_grid();
}

// The cell layout after windows changed size: key bases, the fluid grid
// rows, the cell arrays and sort scratch (a new block when the arena's are
// too small), the radix plan; graphs are captured again on the next step.
pf_status World::relayout_grid() {
  const auto t_start = std::chrono::steady_clock::now();
  const uint32_t cells_before = cells_;
  PF_CUDA(cudaStreamSynchronize(stream_));
  if (side_stream_) PF_CUDA(cudaStreamSynchronize(side_stream_));
  uint64_t cell = 0;
  for (auto& S : h_scenes_) {
    S.cell_base = (uint32_t)cell;
    cell += (uint64_t)S.cells + 1;
  }
  if (cell > kSortCellCap) return fail(PF_ERR_INVALID, "SimLoop: grid windows over 2^31 - 1 cells");
  cells_ = (uint32_t)cell;
  std::vector<uint32_t> row_base(1, 0);
  for (auto& S : h_scenes_)
    if (S.has_grid && S.fluid_count) row_base.push_back(row_base.back() + S.dims[1] * S.dims[2]);
  PF_CUDA(cudaMemcpy(const_cast<uint32_t*>(base_.row_base), row_base.data(), 4 * row_base.size(),
                     cudaMemcpyHostToDevice));
  base_.n_rows = row_base.back();
  if (cells_ > cells_cap_) {
    // new cell arrays with twice the room
    const uint64_t cap = std::min<uint64_t>(kSortCellCap, 2ull * cells_);
    const size_t cell_bytes = al256(4ull * cap);
    void* g = nullptr;
    if (const cudaError_t e = dev_alloc(&g, 2 * cell_bytes, stream_); e != cudaSuccess) {
      return fail(e == cudaErrorMemoryAllocation ? PF_ERR_OOM : PF_ERR_CUDA,
                  "SimLoop: growing the grid windows needs " + std::to_string(2 * cell_bytes) + " more bytes");
    }
    char* p = static_cast<char*>(g);
    base_.cstart = reinterpret_cast<uint32_t*>(p);
    base_.ccount = reinterpret_cast<uint32_t*>(p + cell_bytes);
    dev_free(grid_arena_, stream_);  // the streams are idle (synchronized above)
    grid_arena_ = g;
    bytes_ += 2 * cell_bytes;
    cells_cap_ = cap;
  }
  if (cells_ > sort_.c_cap) {
    // new sort scratch only once the windows pass the 64 times the cells the
    // old one was carved for
    const uint64_t sort_cells = std::min<uint64_t>(kSortCellCap, 64ull * cells_);
    const size_t bytes = sort_scratch_bytes(n_, sort_cells);
    void* g = nullptr;
    if (const cudaError_t e = dev_alloc(&g, bytes, stream_); e != cudaSuccess) {
      return fail(e == cudaErrorMemoryAllocation ? PF_ERR_OOM : PF_ERR_CUDA,
                  "SimLoop: growing the grid windows needs " + std::to_string(bytes) + " more bytes");
    }
    sort_scratch_carve(g, n_, sort_cells, &sort_);
    PF_CUDA(sort_scratch_zero(sort_, stream_));
    dev_free(sort_arena_, stream_);
    sort_arena_ = g;
    bytes_ += bytes;
  }
  PF_CUDA(cudaStreamSynchronize(stream_));  // new blocks usable from every stream
  radix_ = radix_plan(cells_);
  ++regrowths_;
  graphs_stale_ = true;
  if (verbose())
    std::fprintf(stderr, "pfsim: grid windows grew: %u -> %u cells, %.2f ms\n", cells_before, cells_,
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count());
  return PF_OK;
}


// Whole-field host write in particle order, the inverse of readback for the
// writable fields: the slot array of the current parity is read, its
// particles' entries patched through the id map, and written back (the w
// lane of positions holds the inverse mass and is kept).
pf_status World::write(uint32_t scene, uint32_t field, const void* src, size_t bytes) {
  if (scene >= specs_.size()) return fail(PF_ERR_INVALID, "write: no such scene");
  if (field > PF_FIELD_INV_MASS)
    return fail(PF_ERR_INVALID, "write: field " + std::to_string(field) + " cannot be written");
  const DevScene& S = h_scenes_[scene];
  const uint32_t cap = S.cap, seg = S.seg_end - S.seg_start;
  const bool w_only = field == PF_FIELD_INV_MASS;
  const size_t need = (w_only ? 4ull : 16ull) * cap;
  if (!src || bytes < need)
    return fail(PF_ERR_INVALID, "write: source holds " + std::to_string(bytes) + " bytes, need " + std::to_string(need));
  const float* f = static_cast<const float*>(src);
  for (size_t i = 0; i < need / 4; ++i) {
    if (!std::isfinite(f[i])) return fail(PF_ERR_INVALID, "write: values must be finite");
    if (w_only && !(f[i] >= 0)) return fail(PF_ERR_INVALID, "write: invMass must be a finite number >= 0");
  }
  PF_CUDA(cudaStreamSynchronize(stream_));
  std::vector<uint32_t> ids(seg);
  PF_CUDA(cudaMemcpy(ids.data(), base_.ids + S.seg_start, 4ull * seg, cudaMemcpyDeviceToHost));
  const StateBuf& B = buf_[parity_];
  if (w_only && h_scenes_[scene].homog) {
    // masses may differ from now on; the captured steps launch the separate
    // apply only for inhomogeneous scenes, so they are captured again
    h_scenes_[scene].homog = 0;
    drop_graphs();
  }
  auto patch = [&](float4* dev) -> pf_status {
    std::vector<float4> tmp(seg);
    PF_CUDA(cudaMemcpy(tmp.data(), dev + S.seg_start, 16ull * seg, cudaMemcpyDeviceToHost));
    for (uint32_t k = 0; k < seg; ++k) {
      const uint32_t id = ids[k] - S.seg_start;
      if (id >= cap) continue;
      if (w_only) {
        tmp[k].w = f[id];
      } else {
        tmp[k].x = f[4ull * id];
        tmp[k].y = f[4ull * id + 1];
        tmp[k].z = f[4ull * id + 2];
      }
    }
    PF_CUDA(cudaMemcpy(dev + S.seg_start, tmp.data(), 16ull * seg, cudaMemcpyHostToDevice));
    return PF_OK;
  };
  switch (field) {
    case PF_FIELD_POSITIONS: return patch(B.x);
    case PF_FIELD_PREDICTED: return patch(B.xs);
    case PF_FIELD_VELOCITIES: return patch(B.v);
    default:
      PF_TRY(patch(B.x));
      return patch(B.xs);
  }
}

pf_status World::readback(uint32_t scene, uint32_t field, void* dst, size_t bytes) {
  if (scene >= specs_.size()) return fail(PF_ERR_INVALID, "readback: no such scene");
  PF_CUDA(cudaStreamSynchronize(stream_));
  const DevScene& S = h_scenes_[scene];
  const uint32_t cap = S.cap, seg = S.seg_end - S.seg_start;
  const StateBuf& B = buf_[parity_];
  std::vector<uint32_t> ids(seg);
  PF_CUDA(cudaMemcpy(ids.data(), base_.ids + S.seg_start, 4ull * seg, cudaMemcpyDeviceToHost));
  auto need = [&](size_t b) -> pf_status {
    if (bytes < b) return fail(PF_ERR_INVALID, "readback: destination holds " + std::to_string(bytes) +
                                                   " bytes, need " + std::to_string(b));
    return PF_OK;
  };
  auto by_slot4 = [&](const float4* src, bool zero_w, bool w_only) -> pf_status {
    std::vector<float4> tmp(seg);
    PF_CUDA(cudaMemcpy(tmp.data(), src + S.seg_start, 16ull * seg, cudaMemcpyDeviceToHost));
    if (w_only) {
      PF_TRY(need(4ull * cap));
      float* o = static_cast<float*>(dst);
      for (uint32_t k = 0; k < seg; ++k) {
        const uint32_t id = ids[k] - S.seg_start;
        if (id < cap) o[id] = tmp[k].w;
      }
      return PF_OK;
    }
    PF_TRY(need(16ull * cap));
    float4* o = static_cast<float4*>(dst);
    for (uint32_t k = 0; k < seg; ++k) {
      const uint32_t id = ids[k] - S.seg_start;
      if (id < cap) o[id] = zero_w ? make_float4(tmp[k].x, tmp[k].y, tmp[k].z, 0.0f) : tmp[k];
    }
    return PF_OK;
  };
  // one float per slot of the segment (host copy), out by particle id
  auto by_host1 = [&](const float* tmp, bool fluid_only) -> pf_status {
    PF_TRY(need(4ull * cap));
    std::vector<uint32_t> tag(seg);
    PF_CUDA(cudaMemcpy(tag.data(), B.tag + S.seg_start, 4ull * seg, cudaMemcpyDeviceToHost));
    float* o = static_cast<float*>(dst);
    for (uint32_t k = 0; k < seg; ++k) {
      const uint32_t id = ids[k] - S.seg_start;
      if (id < cap) o[id] = (fluid_only && !tag_fluid(tag[k])) ? 0.0f : tmp[k];
    }
    return PF_OK;
  };
  auto by_slot1 = [&](const float* src, bool fluid_only) -> pf_status {
    std::vector<float> tmp(seg);
    PF_CUDA(cudaMemcpy(tmp.data(), src + S.seg_start, 4ull * seg, cudaMemcpyDeviceToHost));
    return by_host1(tmp.data(), fluid_only);
  };
  auto by_id4 = [&](const float4* src) -> pf_status {
    PF_TRY(need(16ull * cap));
    if (!src) {
      float4* o = static_cast<float4*>(dst);
      for (uint32_t i = 0; i < cap; ++i) o[i] = make_float4(0, 0, 0, field == PF_FIELD_ANGULAR_VELOCITY ? 0.0f : 1.0f);
      return PF_OK;
    }
    PF_CUDA(cudaMemcpy(dst, src + S.seg_start, 16ull * cap, cudaMemcpyDeviceToHost));
    return PF_OK;
  };
  switch (field) {
    case PF_FIELD_POSITIONS: return by_slot4(B.x, true, false);
    case PF_FIELD_PREDICTED: return by_slot4(B.xs, true, false);
    case PF_FIELD_VELOCITIES: return by_slot4(B.v, true, false);
    case PF_FIELD_INV_MASS: return by_slot4(B.x, false, true);
    case PF_FIELD_BOUNDARY_VOLUME: return by_slot1(B.bv, false);
    case PF_FIELD_DENSITY: return by_slot1(B.dens, true);
    case PF_FIELD_LAMBDA: {
      // the slot path keeps lambda beside x* (xl) in single-fluid scenes of
      // one mass and in lm otherwise; the warp-tile path in lambda
      if (tune_.path == 1 || !base_.lm) return by_slot1(base_.lambda, true);
      const bool in_xl = scene < lam_in_xl_.size() && lam_in_xl_[scene];
      const size_t words = in_xl ? 4 : 2;
      std::vector<float> raw(words * seg);
      PF_CUDA(cudaMemcpy(raw.data(), in_xl ? (const float*)(base_.xl + S.seg_start) : (const float*)(base_.lm + S.seg_start),
                         4ull * words * seg, cudaMemcpyDeviceToHost));
      std::vector<float> lam(seg);
      for (uint32_t k = 0; k < seg; ++k) lam[k] = raw[words * k + (in_xl ? 3 : 0)];
      return by_host1(lam.data(), true);
    }
    case PF_FIELD_ROTATION: return by_id4(base_.q);
    case PF_FIELD_PREDICTED_ROTATION: return by_id4(base_.qp);
    case PF_FIELD_ANGULAR_VELOCITY: return by_id4(base_.omega);
    case PF_FIELD_CELL_PERM: {
      PF_TRY(need(4ull * cap));
      uint32_t* o = static_cast<uint32_t*>(dst);
      uint32_t w = 0;
      for (uint32_t k = 0; k < seg && w < cap; ++k) {
        const uint32_t id = ids[k] - S.seg_start;
        if (id < cap) o[w++] = id;
      }
      return PF_OK;
    }
    case PF_FIELD_NEIGHBOR_COUNT:
    case PF_FIELD_NEIGHBORS: {
      const bool lists = field == PF_FIELD_NEIGHBORS;
      PF_TRY(need(4ull * cap * (lists ? kMaxNbr : 1)));
      std::vector<uint32_t> cnt(seg), tag(seg);
      PF_CUDA(cudaMemcpy(cnt.data(), base_.ncount + S.seg_start, 4ull * seg, cudaMemcpyDeviceToHost));
      PF_CUDA(cudaMemcpy(tag.data(), B.tag + S.seg_start, 4ull * seg, cudaMemcpyDeviceToHost));
      uint32_t* o = static_cast<uint32_t*>(dst);
      if (!lists) {
        for (uint32_t k = 0; k < seg; ++k) {
          const uint32_t id = ids[k] - S.seg_start;
          if (id < cap) o[id] = tag_fluid(tag[k]) ? cnt[k] : 0u;
        }
        return PF_OK;
      }
      std::fill(o, o + (size_t)cap * kMaxNbr, 0xffffffffu);
      if (!base_.nbr16) return PF_OK;
      if (tune_.path == 0) {
        // segments start on a warp boundary, so their list blocks are one range
        std::vector<uint32_t> all((size_t)seg * kMaxNbr), seg_ids(seg), wbase(seg / 32);
        PF_CUDA(cudaMemcpy(seg_ids.data(), base_.ids + S.seg_start, 4ull * seg, cudaMemcpyDeviceToHost));
        PF_CUDA(cudaMemcpy(all.data(), base_.nbr + nbr_col(S.seg_start), 4ull * seg * kMaxNbr, cudaMemcpyDeviceToHost));
        PF_CUDA(cudaMemcpy(wbase.data(), base_.nbr_base + S.seg_start / 32, 4ull * (seg / 32), cudaMemcpyDeviceToHost));
        const uint16_t* all16 = reinterpret_cast<const uint16_t*>(all.data());
        for (uint32_t m = 0; m < kMaxNbr; ++m) {
          for (uint32_t k = 0; k < seg; ++k) {
            const uint32_t id = ids[k] - S.seg_start;
            if (id >= cap || !tag_fluid(tag[k]) || m >= cnt[k]) continue;
            const uint32_t wb = wbase[k / 32];
            // a slot of the same scene's segment
            const uint32_t j = (wb & kNbrWide) ? all[nbr_col(k) + (size_t)m * kNbrStride]
                                               : wb + all16[nbr16_at(k, m)];
            o[(size_t)id * kMaxNbr + m] = (j >= S.seg_start && j < S.seg_end) ? seg_ids[j - S.seg_start] - S.seg_start
                                                                               : 0xfffffffeu;
          }
        }
        return PF_OK;
      }
      uint32_t nt = 0;
      PF_CUDA(cudaMemcpy(&nt, base_.tile_count, 4, cudaMemcpyDeviceToHost));
      nt = std::min(nt, base_.max_tiles);
      std::vector<Tile> tiles(nt);
      PF_CUDA(cudaMemcpy(tiles.data(), base_.tiles, sizeof(Tile) * nt, cudaMemcpyDeviceToHost));
      std::vector<uint32_t> st(seg), all_ids(n_);
      std::vector<uint16_t> col(seg);
      PF_CUDA(cudaMemcpy(st.data(), base_.slot_tile + S.seg_start, 4ull * seg, cudaMemcpyDeviceToHost));
      PF_CUDA(cudaMemcpy(all_ids.data(), base_.ids, 4ull * n_, cudaMemcpyDeviceToHost));
      for (uint32_t m = 0; m < kMaxNbr; ++m) {
        PF_CUDA(cudaMemcpy(col.data(), base_.nbr16 + (size_t)m * n_ + S.seg_start, 2ull * seg, cudaMemcpyDeviceToHost));
        for (uint32_t k = 0; k < seg; ++k) {
          const uint32_t id = ids[k] - S.seg_start;
          if (id >= cap || !tag_fluid(tag[k]) || m >= cnt[k] || st[k] >= nt) continue;
          const Tile& T = tiles[st[k]];
          const uint32_t h = col[k];
          int r = 0;
          while (r < 8 && h >= T.roff[r + 1]) ++r;
          const uint32_t j = T.rs[r] + (h - T.roff[r]);
          o[(size_t)id * kMaxNbr + m] = all_ids[j] - S.seg_start;
        }
      }
      return PF_OK;
    }
    default:
      return fail(PF_ERR_INVALID, "readback: unknown field " + std::to_string(field));
  }
}

pf_status World::import_scene(uint32_t s, const World& src, uint32_t src_s) {
  if (s >= h_scenes_.size() || src_s >= src.h_scenes_.size()) return fail(PF_ERR_INVALID, "import: no such scene");
  const DevScene& S = h_scenes_[s];
  const DevScene& T = src.h_scenes_[src_s];
  if (S.cap != T.cap) return fail(PF_ERR_INVALID, "import: scenes differ in capacity");
  if (S.cap == 0) return PF_OK;
  const StateBuf& B = src.buf_[src.parity_];
  const WorldView V = view(parity_);
  k_import_scene<<<div_up(S.cap, kBlock), kBlock, 0, stream_>>>(V, S.seg_start, S.cap, B.x, B.v, B.bv, src.base_.inv,
                                                                 T.seg_start, src.base_.q, src.base_.omega);
  PF_CUDA(cudaGetLastError());
  return PF_OK;
}

void World::retire(uint32_t s) {
  if (s >= h_scenes_.size()) return;
  h_scenes_[s].substeps = 0;
  h_scenes_[s].iterations = 0;
}

pf_status World::pull_state(uint32_t scene, SceneSpec* sp) {
  const uint32_t cap = h_scenes_[scene].cap;
  std::vector<float4> t(cap);
  PF_TRY(readback(scene, PF_FIELD_POSITIONS, t.data(), 16ull * cap));
  for (uint32_t i = 0; i < cap; ++i) {
    sp->pos4[4 * i] = t[i].x;
    sp->pos4[4 * i + 1] = t[i].y;
    sp->pos4[4 * i + 2] = t[i].z;
  }
  PF_TRY(readback(scene, PF_FIELD_VELOCITIES, t.data(), 16ull * cap));
  for (uint32_t i = 0; i < cap; ++i) {
    sp->vel4[4 * i] = t[i].x;
    sp->vel4[4 * i + 1] = t[i].y;
    sp->vel4[4 * i + 2] = t[i].z;
  }
  PF_TRY(readback(scene, PF_FIELD_INV_MASS, sp->inv_mass.data(), 4ull * cap));
  PF_TRY(readback(scene, PF_FIELD_BOUNDARY_VOLUME, sp->bvol.data(), 4ull * cap));
  sp->rot4.resize(4ull * cap);
  sp->angv4.resize(4ull * cap);
  PF_TRY(readback(scene, PF_FIELD_ROTATION, sp->rot4.data(), 16ull * cap));
  PF_TRY(readback(scene, PF_FIELD_ANGULAR_VELOCITY, sp->angv4.data(), 16ull * cap));
  return PF_OK;
}

pf_status World::overflow(uint32_t scene, pf_overflow* out) {
  if (scene >= specs_.size()) return fail(PF_ERR_INVALID, "readbackOverflow: no such scene");
  PF_CUDA(cudaStreamSynchronize(stream_));
  uint32_t f[kNumFlags];
  PF_CUDA(cudaMemcpy(f, base_.flags + scene * kNumFlags, sizeof(f), cudaMemcpyDeviceToHost));
  uint32_t err = 0;
  PF_CUDA(cudaMemcpy(&err, sort_.counters + kCounterError, 4, cudaMemcpyDeviceToHost));
  out->positions = f[FLAG_POS] | f[FLAG_SOFT] | f[FLAG_REACT];
  out->velocities = f[FLAG_VEL];
  out->grid = f[FLAG_GRID];
  out->grid_clamped = f[FLAG_CLAMP];
  out->contacts = f[FLAG_CONTACTS];
  if (h_scenes_[scene].contact) {
    // loop.ts:290-301: the last substep's pair count against maxContacts
    uint2 st;
    PF_CUDA(cudaMemcpy(&st, base_.con_stat + scene, sizeof(uint2), cudaMemcpyDeviceToHost));
    out->contacts |= (st.x > h_scenes_[scene].max_contacts || st.y > 0) ? 1u : 0u;
  }
  out->neighbors = f[FLAG_NBR];
  out->device_error = err | f[FLAG_DEVICE];
  return PF_OK;
}

// ContactBuffer.readbackCount / readbackPairs for one scene: the pairs of
// the last substep as particle indices, each pair ascending, sorted.
pf_status World::contacts(uint32_t scene, uint32_t* pairs, uint32_t capacity, uint32_t* count, uint32_t* stored) {
  if (scene >= specs_.size()) return fail(PF_ERR_INVALID, "contacts: no such scene");
  const DevScene& S = h_scenes_[scene];
  if (!S.contact) return fail(PF_ERR_STATE, "contacts: the SimLoop was built without contact");
  PF_CUDA(cudaStreamSynchronize(stream_));
  const uint32_t seg = S.seg_end - S.seg_start;
  uint2 st;
  PF_CUDA(cudaMemcpy(&st, base_.con_stat + scene, sizeof(uint2), cudaMemcpyDeviceToHost));
  std::vector<uint32_t> ids(seg), cnt(seg), pre(seg), off(seg / kSegAlign), nb((size_t)kMaxContacts * seg);
  PF_CUDA(cudaMemcpy(ids.data(), base_.ids + S.seg_start, 4ull * seg, cudaMemcpyDeviceToHost));
  PF_CUDA(cudaMemcpy(cnt.data(), base_.con_cnt + S.seg_start, 4ull * seg, cudaMemcpyDeviceToHost));
  PF_CUDA(cudaMemcpy(pre.data(), base_.con_pre + S.seg_start, 4ull * seg, cudaMemcpyDeviceToHost));
  PF_CUDA(cudaMemcpy(off.data(), base_.chunk_off + S.seg_start / kSegAlign, 4ull * off.size(), cudaMemcpyDeviceToHost));
  for (uint32_t m = 0; m < kMaxContacts; ++m)
    PF_CUDA(cudaMemcpy(nb.data() + (size_t)m * seg, base_.con_nbr + (size_t)m * n_ + S.seg_start, 4ull * seg,
                       cudaMemcpyDeviceToHost));
  std::vector<std::pair<uint32_t, uint32_t>> out;
  for (uint32_t k = 0; k < seg; ++k) {
    const uint32_t c = std::min(cnt[k], kMaxContacts);
    const uint32_t first = off[k / kSegAlign] + pre[k];
    for (uint32_t m = 0; m < c && first + m < S.max_contacts; ++m) {
      const uint32_t a = ids[k] - S.seg_start, b = ids[nb[(size_t)m * seg + k] - S.seg_start] - S.seg_start;
      out.push_back({std::min(a, b), std::max(a, b)});
    }
  }
  std::sort(out.begin(), out.end());
  if (count) *count = st.x;
  if (stored) *stored = (uint32_t)out.size();
  for (size_t q = 0; pairs && q < out.size() && q < capacity; ++q) {
    pairs[2 * q] = out[q].first;
    pairs[2 * q + 1] = out[q].second;
  }
  return PF_OK;
}

pf_status World::elapsed_ms(float* ms) {
  PF_CUDA(cudaEventSynchronize(ev1_));
  PF_CUDA(cudaEventElapsedTime(ms, ev0_, ev1_));
  last_ms_ = *ms;
  return PF_OK;
}

uint64_t World::total_particles() const {
  uint64_t t = 0;
  for (auto& S : h_scenes_) t += S.cap;
  return t;
}

pf_status World::read_positions(float* dst, size_t bytes) {
  const uint64_t total = total_particles();
  if (bytes < 16ull * total) return fail(PF_ERR_INVALID, "readback: destination too small");
  PF_TRY(wait_reads());  // an async read may still copy out of stage_pos_
  launch_slots(k_gather_positions, n_, stream_, view(parity_), (const uint64_t*)prefix_dev_, stage_pos_);
  PF_CUDA(cudaMemcpyAsync(dst, stage_pos_, 16ull * total, cudaMemcpyDeviceToHost, stream_));
  PF_CUDA(cudaStreamSynchronize(stream_));
  return PF_OK;
}

pf_status World::read_positions_async(float* dst, size_t bytes) {
  const uint64_t total = total_particles();
  if (bytes < 16ull * total) return fail(PF_ERR_INVALID, "readback: destination too small");
  if (!read_stream_) {
    PF_CUDA(cudaStreamCreateWithFlags(&read_stream_, cudaStreamNonBlocking));
    for (int b = 0; b < 2; ++b) {
      PF_CUDA(cudaEventCreateWithFlags(&ev_gathered_[b], cudaEventDisableTiming));
      PF_CUDA(cudaEventCreateWithFlags(&ev_read_[b], cudaEventDisableTiming));
    }
  }
  const uint32_t b = read_next_;
  read_next_ ^= 1u;
  if (read_pending_[b]) {  // the read two calls back still copies out of this staging buffer
    PF_CUDA(cudaEventSynchronize(ev_read_[b]));
    read_pending_[b] = false;
  }
  float4* stage = b ? stage_pos2_ : stage_pos_;
  launch_slots(k_gather_positions, n_, stream_, view(parity_), (const uint64_t*)prefix_dev_, stage);
  PF_CUDA(cudaEventRecord(ev_gathered_[b], stream_));
  PF_CUDA(cudaStreamWaitEvent(read_stream_, ev_gathered_[b], 0));
  PF_CUDA(cudaMemcpyAsync(dst, stage, 16ull * total, cudaMemcpyDeviceToHost, read_stream_));
  PF_CUDA(cudaEventRecord(ev_read_[b], read_stream_));
  read_pending_[b] = true;
  return PF_OK;
}

pf_status World::wait_reads() {
  for (int b = 0; b < 2; ++b)
    if (read_pending_[b]) {
      PF_CUDA(cudaEventSynchronize(ev_read_[b]));
      read_pending_[b] = false;
    }
  return PF_OK;
}

pf_status World::profile_stage(uint32_t stage, uint32_t reps, float* ms, uint64_t* items) {
  const WorldView V = view(parity_);
  const uint32_t rank = h_fluids_.empty() ? 0u : h_fluids_[0].rank;
  uint64_t fluid = 0;
  for (uint32_t s = 0; s < specs_.size(); ++s)
    for (auto& f : specs_[s]->fluids) fluid += f.range.count;
  auto run_on = [&](const WorldView& W) {
    switch (stage) {
      case 0:
        if (tune_.path == 1) launch_tiled(k_t_neighbors, kSmemNbr, W, 0u);
        else PF_NBR(W, 0u);
        break;
      case 1:
        if (tune_.path == 1) launch_tiled(k_t_lambda, kSmemLambda, W, rank, 0u, 0u);
        else PF_BY_UNROLL(kSlotLambda, k_s_lambda, W, rank, 0u, 0u);
        break;
      case 2:  // with the apply the step fuses in (it rewrites x*, which the next predict replaces)
        if (tune_.path == 1) launch_tiled(k_t_delta, kSmemDelta, W, rank, 0u, 0u);
        else PF_DELTA(W, rank, 0u, 0u, 1u);
        break;
      case 3:
        if (tune_.path == 1) launch_tiled(k_t_xsph, kSmemXsph, W, rank, 0u);
        else PF_XSPH(W, rank, 0u);
        break;
      case 4: launch_slots(k_predict, n_, stream_, W, 0u); break;
      default: break;
    }
  };
  // as the step launches it: group by group, then the other fluid scenes
  auto run = [&]() {
    if (stage < 4 && grouping()) {
      for (size_t g = 0; g < groups_.size(); ++g) run_on(group_view(V, g));
      const WorldView R = rest_view(V);
      if (R.n_fchunk) run_on(R);
    } else {
      run_on(V);
    }
  };
  if (stage > 4) return fail(PF_ERR_INVALID, "profile: unknown stage");
  if (items) *items = stage == 4 ? total_particles() : fluid;
  run();
  PF_CUDA(cudaEventRecord(ev0_, stream_));
  for (uint32_t r = 0; r < reps; ++r) run();
  PF_CUDA(cudaEventRecord(ev1_, stream_));
  PF_CUDA(cudaEventSynchronize(ev1_));
  float t = 0;
  PF_CUDA(cudaEventElapsedTime(&t, ev0_, ev1_));
  *ms = t / (float)std::max(reps, 1u);
  return PF_OK;
}

}  // namespace pf
