// capi_scene.cu — C ABI of scenes (ParticleSystem + materials + colliders +
// SimLoop) and of batches of scenes.
//
// The host-side set-up follows the reference constructors so that a scene
// built through this ABI holds the same initial state the reference would:
// FluidSystem sets its particles' inverse mass (FluidSystem.ts:90-127),
// SoftbodySystem derives rest offsets, mass weights, the neighbour CSR and
// rest centres from the uploaded particles (SoftbodySystem.ts:132-199,
// 277-340, 366-514), ClothSystem uploads its graph and colours its distance
// constraints greedily (ClothSystem.ts:102-141, types.ts:95-150).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "world.cuh"
#include "capi_handles.cuh"


namespace pf {
namespace {

bool range_ok(const SceneSpec& s, RangeU r) { return r.count > 0 && (uint64_t)r.start + r.count <= s.cap; }
bool overlaps(RangeU a, RangeU b) { return a.start < b.start + b.count && b.start < a.start + a.count; }

// f32 -> IEEE half, round to nearest even, after clamping to +-65504 as the
// SDFCollider's half-float upload does (SDFCollider.ts:101-103).
uint16_t half_rn(float f) {
  if (f > 65504.0f) f = 65504.0f;
  if (f < -65504.0f) f = -65504.0f;
  uint32_t x;
  std::memcpy(&x, &f, 4);
  const uint32_t sign = (x >> 16) & 0x8000u;
  const uint32_t ax = x & 0x7fffffffu;
  if (ax > 0x7f800000u) return (uint16_t)(sign | 0x7e00u);  // NaN
  if (ax < 0x38800000u) {                                    // below 2^-14: a half subnormal
    float af;
    std::memcpy(&af, &ax, 4);
    return (uint16_t)(sign | (uint32_t)std::nearbyint(af * 16777216.0f));
  }
  uint32_t h = ((ax >> 23) - 112u) << 10 | ((ax & 0x7fffffu) >> 13);
  const uint32_t rem = ax & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) ++h;
  return (uint16_t)(sign | h);
}

// SDFCollider.setPosition / setRotation / setScale checks (SDFCollider.ts:170-201).
pf_status sdf_transform(const float pos[3], const float rot[4], float scale, SdfSpec* g) {
  double q[4], n = 0;
  for (int a = 0; a < 4; ++a) {
    q[a] = rot[a];
    n += q[a] * q[a];
  }
  n = std::sqrt(n);
  if (!(n > 1e-12) || !std::isfinite(n)) return fail(PF_ERR_INVALID, "SDFCollider.setRotation: rotation must be a non-zero quaternion");
  if (!(scale > 0) || !std::isfinite(scale))
    return fail(PF_ERR_INVALID, "SDFCollider.setScale: scale must be positive, got " + std::to_string(scale));
  for (int a = 0; a < 3; ++a) g->position[a] = pos[a];
  for (int a = 0; a < 4; ++a) g->rot_q[a] = q[a] / n;
  g->scale = scale;
  return PF_OK;
}

pf_status not_built(const pf_scene* s, const char* what) {
  if (!s) return fail(PF_ERR_INVALID, std::string(what) + ": scene is NULL");
  if (s->spec.built)
    return fail(PF_ERR_STATE, std::string(what) + ": add materials and colliders before building the SimLoop");
  return PF_OK;
}

// Smallest eigenvalue of a symmetric 3x3 (xx, xy, xz, yy, yz, zz) by Jacobi
// rotations on the largest off-diagonal entry (SoftbodySystem.ts:424-470).
double smallest_eigenvalue(double a00, double a01, double a02, double a11, double a12, double a22) {
  for (int sweep = 0; sweep < 30; ++sweep) {
    const double off = std::fabs(a01) + std::fabs(a02) + std::fabs(a12);
    if (off < 1e-14) break;
    const int pivot = (std::fabs(a01) >= std::fabs(a02) && std::fabs(a01) >= std::fabs(a12)) ? 0
                      : (std::fabs(a02) >= std::fabs(a12))                                    ? 1
                                                                                              : 2;
    double apq, app, aqq;
    if (pivot == 0) { apq = a01; app = a00; aqq = a11; }
    else if (pivot == 1) { apq = a02; app = a00; aqq = a22; }
    else { apq = a12; app = a11; aqq = a22; }
    if (std::fabs(apq) < 1e-20) break;
    const double theta = (aqq - app) / (2 * apq);
    const double sgn = theta > 0 ? 1.0 : (theta < 0 ? -1.0 : 1.0);
    const double t = sgn / (std::fabs(theta) + std::sqrt(1 + theta * theta));
    const double c = 1 / std::sqrt(1 + t * t), s = t * c;
    if (pivot == 0) {
      const double n02 = c * a02 - s * a12, n12 = s * a02 + c * a12;
      a00 = app - t * apq; a11 = aqq + t * apq; a01 = 0; a02 = n02; a12 = n12;
    } else if (pivot == 1) {
      const double n01 = c * a01 - s * a12, n12 = s * a01 + c * a12;
      a00 = app - t * apq; a22 = aqq + t * apq; a02 = 0; a01 = n01; a12 = n12;
    } else {
      const double n01 = c * a01 - s * a02, n02 = s * a01 + c * a02;
      a11 = app - t * apq; a22 = aqq + t * apq; a12 = 0; a01 = n01; a02 = n02;
    }
  }
  return std::min(a00, std::min(a11, a22));
}

// Greedy colouring in constraint order: each constraint takes the lowest
// colour none of its particles has yet (types.ts:95-150).
// types.ts:59-114: greedy colouring in constraint order; each constraint of
// `arity` particles takes the lowest group none of its particles owns yet.
std::vector<std::vector<uint32_t>> color_groups(const std::vector<uint32_t>& parts, uint32_t arity, uint32_t n,
                                                uint32_t cap) {
  std::vector<std::vector<uint32_t>> owned(cap);
  std::vector<std::vector<uint32_t>> colors;
  for (uint32_t c = 0; c < n; ++c) {
    uint32_t g = 0;
    for (;;) {
      bool clash = false;
      for (uint32_t k = 0; k < arity && !clash; ++k) {
        const auto& o = owned[parts[(size_t)arity * c + k]];
        clash = std::find(o.begin(), o.end(), g) != o.end();
      }
      if (!clash) break;
      ++g;
    }
    if (g >= colors.size()) colors.resize(g + 1);
    colors[g].push_back(c);
    for (uint32_t k = 0; k < arity; ++k) owned[parts[(size_t)arity * c + k]].push_back(g);
  }
  return colors;
}

std::vector<std::vector<uint32_t>> color_pairs(const std::vector<uint32_t>& pairs, uint32_t n, uint32_t cap) {
  return color_groups(pairs, 2, n, cap);
}

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" {

pf_status pf_scene_create(const pf_scene_desc* d, pf_scene** out) {
  if (!d || !out) return fail(PF_ERR_INVALID, "ParticleSystem: NULL argument");
  if (d->capacity == 0) return fail(PF_ERR_INVALID, "ParticleSystem: capacity must be a positive integer, got 0");
  if (!(d->particle_radius > 0) || !std::isfinite(d->particle_radius))
    return fail(PF_ERR_INVALID, "ParticleSystem: particleRadius must be a positive finite number, got " +
                                    std::to_string(d->particle_radius));
  auto* s = new pf_scene;
  SceneSpec& sp = s->spec;
  sp.cap = d->capacity;
  sp.radius = d->particle_radius;
  sp.pos4.assign(4ull * sp.cap, 0.0f);
  sp.vel4.assign(4ull * sp.cap, 0.0f);
  sp.inv_mass.assign(sp.cap, 0.0f);
  sp.bvol.assign(sp.cap, 0.0f);
  sp.group.assign(sp.cap, 0u);
  sp.rot4.assign(4ull * sp.cap, 0.0f);
  sp.angv4.assign(4ull * sp.cap, 0.0f);
  for (uint32_t i = 0; i < sp.cap; ++i) sp.rot4[4 * i + 3] = 1.0f;
  *out = s;
  return PF_OK;
}

void pf_scene_destroy(pf_scene* s) { delete s; }

pf_status pf_upload_particles(pf_scene* s, const float* pos4, const float* vel4, const float* inv_mass,
                              const uint32_t* group, uint32_t start, uint32_t n) {
  if (!s) return fail(PF_ERR_INVALID, "ParticleSystem.uploadParticles: scene is NULL");
  SceneSpec& sp = s->spec;
  if ((uint64_t)start + n > sp.cap)
    return fail(PF_ERR_INVALID, "ParticleSystem.uploadParticles: invalid particle range start=" + std::to_string(start) +
                                    " count=" + std::to_string(n) + " (capacity " + std::to_string(sp.cap) + ")");
  if (n && !pos4) return fail(PF_ERR_INVALID, "ParticleSystem.uploadParticles: positions are NULL");
  if (s->world) return fail(PF_ERR_STATE, "ParticleSystem.uploadParticles: upload before building the SimLoop");
  for (uint32_t k = 0; k < n; ++k) {
    if (inv_mass && !(inv_mass[k] >= 0 && std::isfinite(inv_mass[k])))
      return fail(PF_ERR_INVALID, "ParticleSystem.uploadParticles: invMass must be a finite number >= 0");
  }
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t i = start + k;
    for (int c = 0; c < 3; ++c) {
      sp.pos4[4 * i + c] = pos4[4 * k + c];
      sp.vel4[4 * i + c] = vel4 ? vel4[4 * k + c] : 0.0f;
    }
    sp.pos4[4 * i + 3] = sp.vel4[4 * i + 3] = 0.0f;
    sp.inv_mass[i] = inv_mass ? inv_mass[k] : 1.0f;
    sp.group[i] = group ? group[k] : 0u;
  }
  return PF_OK;
}

pf_status pf_set_inv_mass(pf_scene* s, pf_range r, float w) {
  if (!s) return fail(PF_ERR_INVALID, "ParticleSystem.setInvMass: scene is NULL");
  if (!range_ok(s->spec, {r.start, r.count}))
    return fail(PF_ERR_INVALID, "ParticleSystem.setInvMass: invalid particle range");
  if (!(w >= 0) || !std::isfinite(w)) return fail(PF_ERR_INVALID, "ParticleSystem.setInvMass: invMass must be >= 0");
  if (s->world) return fail(PF_ERR_STATE, "ParticleSystem.setInvMass: set before building the SimLoop");
  for (uint32_t i = r.start; i < r.start + r.count; ++i) s->spec.inv_mass[i] = w;
  return PF_OK;
}

pf_status pf_add_fluid(pf_scene* s, const pf_fluid_desc* d, uint32_t* mat) {
  PF_TRY(not_built(s, "FluidSystem"));
  if (!d) return fail(PF_ERR_INVALID, "FluidSystem: options are NULL");
  SceneSpec& sp = s->spec;
  FluidSpec f;
  f.range.start = d->range.count ? d->range.start : 0;
  f.range.count = d->range.count ? d->range.count : sp.cap;
  if (!range_ok(sp, f.range))
    return fail(PF_ERR_INVALID, "FluidSystem: invalid particle range start=" + std::to_string(f.range.start) +
                                    " count=" + std::to_string(f.range.count));
  auto positive = [](double v, const char* name, double* out) -> pf_status {
    if (!(v > 0) || !std::isfinite(v))
      return fail(PF_ERR_INVALID, std::string("FluidSystem: ") + name + " must be positive, got " + std::to_string(v));
    *out = v;
    return PF_OK;
  };
  PF_TRY(positive(d->rest_density > 0 ? d->rest_density : 1000.0, "restDensity", &f.rho0));
  PF_TRY(positive(d->particle_spacing > 0 ? (double)d->particle_spacing : 2.0 * sp.radius, "particleSpacing", &f.spacing));
  PF_TRY(positive(d->smoothing_radius > 0 ? (double)d->smoothing_radius : 2.0 * f.spacing, "smoothingRadius", &f.h));
  f.compliance = d->compliance >= 0 ? d->compliance : 1e-4;
  if (!std::isfinite(f.compliance)) return fail(PF_ERR_INVALID, "FluidSystem: compliance must be >= 0");
  f.has_visc = (d->flags & PF_FLUID_VISCOSITY) != 0;
  f.viscosity = d->viscosity;
  if (f.has_visc && !std::isfinite(f.viscosity))
    return fail(PF_ERR_INVALID, "FluidSystem: viscosity must be finite");
  f.has_vort = (d->flags & PF_FLUID_VORTICITY) != 0;
  f.vorticity = f.has_vort ? d->vorticity : 0.0;
  if (f.has_vort && !std::isfinite(f.vorticity))
    return fail(PF_ERR_INVALID, "FluidSystem: vorticity must be finite");
  f.has_st = (d->flags & PF_FLUID_SURFACE_TENSION) != 0;
  f.surface_tension = f.has_st ? d->surface_tension : 0.0;
  if (f.has_st && !std::isfinite(f.surface_tension))
    return fail(PF_ERR_INVALID, "FluidSystem: surfaceTension must be finite");
  f.has_ad = (d->flags & PF_FLUID_ADHESION) != 0;
  f.adhesion = f.has_ad ? d->adhesion : 0.0;
  if (f.has_ad && !std::isfinite(f.adhesion))
    return fail(PF_ERR_INVALID, "FluidSystem: adhesion must be finite");
  for (uint32_t b = 0; b < d->n_boundaries; ++b) {
    RangeU r{d->boundaries[b].start, d->boundaries[b].count};
    if (!range_ok(sp, r)) return fail(PF_ERR_INVALID, "FluidSystem.addBoundary: invalid particle range");
    if (overlaps(r, f.range)) return fail(PF_ERR_INVALID, "FluidSystem.addBoundary: a boundary cannot overlap the fluid");
    for (auto& o : f.bnd)
      if (overlaps(r, o)) return fail(PF_ERR_INVALID, "FluidSystem.addBoundary: boundaries cannot overlap each other");
    f.bnd.push_back(r);
    f.bnd_static.push_back(d->boundary_static ? d->boundary_static[b] : 0);
  }
  // FluidSystem.ts:117-118: the fluid owns its particles' mass.
  const double mass = f.rho0 * f.spacing * f.spacing * f.spacing;
  const float w = (float)(1.0 / mass);
  for (uint32_t i = f.range.start; i < f.range.start + f.range.count; ++i) sp.inv_mass[i] = w;
  sp.fluids.push_back(std::move(f));
  sp.materials.push_back({MAT_FLUID, (uint32_t)sp.fluids.size() - 1});
  if (mat) *mat = (uint32_t)sp.materials.size() - 1;
  return PF_OK;
}

pf_status pf_add_softbodies(pf_scene* s, const pf_softbody_desc* d, uint32_t* mat) {
  PF_TRY(not_built(s, "SoftbodySystem"));
  if (!d || d->n_bodies == 0) return fail(PF_ERR_INVALID, "SoftbodySystem: at least one body is required");
  SceneSpec& sp = s->spec;
  SoftSpec ss;
  ss.local = d->shape_matching == PF_SHAPE_MATCH_LOCAL;
  ss.self_collision = d->self_collision != 0;
  ss.rest4.assign(4ull * sp.cap, 0.0f);
  ss.weights.assign(sp.cap, 0.0f);
  std::vector<uint8_t> used(sp.cap, 0);
  uint32_t span_lo = UINT32_MAX, span_hi = 0;
  for (uint32_t b = 0; b < d->n_bodies; ++b) {
    const pf_softbody_def& def = d->bodies[b];
    const std::string who = "SoftbodySystem: body " + std::to_string(b);
    RangeU r{def.range.start, def.range.count};
    if (r.count == 0) return fail(PF_ERR_INVALID, who + " has no particles");
    if (!range_ok(sp, r)) return fail(PF_ERR_INVALID, who + ": invalid particle range");
    for (uint32_t i = r.start; i < r.start + r.count; ++i) {
      if (used[i]) return fail(PF_ERR_INVALID, "SoftbodySystem: particle " + std::to_string(i) + " belongs to two bodies");
      used[i] = 1;
    }
    std::vector<float> restp(3ull * r.count);
    for (uint32_t k = 0; k < r.count; ++k)
      for (int c = 0; c < 3; ++c)
        restp[3 * k + c] = def.rest_positions ? def.rest_positions[3 * k + c] : sp.pos4[4ull * (r.start + k) + c];
    const uint32_t surface = def.surface_count == UINT32_MAX ? r.count : def.surface_count;
    if (surface > r.count) return fail(PF_ERR_INVALID, who + " surfaceCount is out of range");
    for (uint32_t e = 0; e < def.n_edges; ++e) {
      const uint32_t i = def.edges[2 * e], j = def.edges[2 * e + 1];
      if (!(i < r.count) || !(j < r.count) || i == j) return fail(PF_ERR_INVALID, who + " has an invalid edge");
    }
    if (ss.local && def.n_edges == 0 && r.count > 1)
      return fail(PF_ERR_INVALID, who + " needs edges for local shape matching");
    // massWeights (SoftbodySystem.ts:366-372)
    std::vector<double> masses(r.count);
    std::vector<double> dyn;
    for (uint32_t k = 0; k < r.count; ++k) {
      const double w = sp.inv_mass[r.start + k];
      masses[k] = w > 0 ? 1.0 / w : 0.0;
      if (masses[k] > 0) dyn.push_back(masses[k]);
    }
    bool all_eq = true;
    for (double m : dyn) all_eq = all_eq && m == dyn[0];
    std::vector<float> bw(r.count, 1.0f);
    if (!all_eq) {
      double mean = 0;
      for (double m : dyn) mean += m;
      mean /= (double)dyn.size();
      for (uint32_t k = 0; k < r.count; ++k) bw[k] = (float)(masses[k] > 0 ? masses[k] / mean : 1.0);
    }
    double cx = 0, cy = 0, cz = 0, tot = 0;
    for (uint32_t k = 0; k < r.count; ++k) {
      cx += (double)restp[3 * k] * bw[k];
      cy += (double)restp[3 * k + 1] * bw[k];
      cz += (double)restp[3 * k + 2] * bw[k];
      tot += bw[k];
    }
    cx /= tot;
    cy /= tot;
    cz /= tot;
    // assertVolumetric (SoftbodySystem.ts:392-421)
    double xx = 0, xy = 0, xz = 0, yy = 0, yz = 0, zz = 0;
    for (uint32_t k = 0; k < r.count; ++k) {
      const double x = restp[3 * k] - cx, y = restp[3 * k + 1] - cy, z = restp[3 * k + 2] - cz;
      xx += x * x; xy += x * y; xz += x * z; yy += y * y; yz += y * z; zz += z * z;
    }
    const double smallest = std::sqrt(std::max(0.0, smallest_eigenvalue(xx, xy, xz, yy, yz, zz)));
    if (smallest < sp.radius * 1e-3)
      return fail(PF_ERR_INVALID, who + " is flat; shape matching needs a 3D particle cloud");
    if (!(def.compliance >= 0) || !std::isfinite(def.compliance))
      return fail(PF_ERR_INVALID, "SoftbodySystem: compliance must be >= 0");
    for (uint32_t k = 0; k < r.count; ++k) {
      const uint32_t i = r.start + k;
      ss.weights[i] = bw[k];
      ss.rest4[4 * i] = (float)(restp[3 * k] - cx);
      ss.rest4[4 * i + 1] = (float)(restp[3 * k + 1] - cy);
      ss.rest4[4 * i + 2] = (float)(restp[3 * k + 2] - cz);
      ss.rest4[4 * i + 3] = def.compliance;
    }
    BodySpec body;
    body.range = r;
    body.surface = surface;
    body.compliance = def.compliance;
    ss.bodies.push_back(body);
    span_lo = std::min(span_lo, r.start);
    span_hi = std::max(span_hi, r.start + r.count);
  }
  ss.span = {span_lo, span_hi - span_lo};
  if (ss.local) {
    // buildNeighborGraph (SoftbodySystem.ts:489-514)
    std::vector<uint32_t> degree(sp.cap, 0);
    for (uint32_t b = 0; b < d->n_bodies; ++b) {
      const pf_softbody_def& def = d->bodies[b];
      for (uint32_t k = 0; k < def.range.count; ++k) degree[def.range.start + k] += 1;
      for (uint32_t e = 0; e < def.n_edges; ++e) {
        degree[def.range.start + def.edges[2 * e]] += 1;
        degree[def.range.start + def.edges[2 * e + 1]] += 1;
      }
    }
    ss.offsets.assign(sp.cap + 1ull, 0);
    for (uint32_t i = 0; i < sp.cap; ++i) ss.offsets[i + 1] = ss.offsets[i] + degree[i];
    ss.indices.assign(std::max<uint32_t>(1, ss.offsets[sp.cap]), 0);
    std::vector<uint32_t> cursor(ss.offsets.begin(), ss.offsets.begin() + sp.cap);
    for (uint32_t b = 0; b < d->n_bodies; ++b) {
      const pf_softbody_def& def = d->bodies[b];
      for (uint32_t i = def.range.start; i < def.range.start + def.range.count; ++i) ss.indices[cursor[i]++] = i;
      for (uint32_t e = 0; e < def.n_edges; ++e) {
        const uint32_t i = def.range.start + def.edges[2 * e], j = def.range.start + def.edges[2 * e + 1];
        ss.indices[cursor[i]++] = j;
        ss.indices[cursor[j]++] = i;
      }
    }
    // rest centres accumulated into f32 storage (SoftbodySystem.ts:283-295)
    ss.rest_centers4.assign(4ull * sp.cap, 0.0f);
    for (auto& body : ss.bodies)
      for (uint32_t i = body.range.start; i < body.range.start + body.range.count; ++i) {
        const uint32_t from = ss.offsets[i], to = ss.offsets[i + 1];
        for (uint32_t k = from; k < to; ++k) {
          const uint32_t j = ss.indices[k];
          for (int a = 0; a < 3; ++a)
            ss.rest_centers4[4 * i + a] =
                (float)((double)ss.rest_centers4[4 * i + a] + (double)ss.rest4[4 * j + a] / (double)(to - from));
        }
      }
  }
  sp.softs.push_back(std::move(ss));
  sp.materials.push_back({MAT_SOFT, (uint32_t)sp.softs.size() - 1});
  if (mat) *mat = (uint32_t)sp.materials.size() - 1;
  return PF_OK;
}

pf_status pf_add_cloth(pf_scene* s, const pf_cloth_desc* d, uint32_t* mat) {
  PF_TRY(not_built(s, "ClothSystem"));
  if (!d) return fail(PF_ERR_INVALID, "ClothSystem: options are NULL");
  SceneSpec& sp = s->spec;
  if (!range_ok(sp, {d->offset, d->n_particles}))
    return fail(PF_ERR_INVALID, "ClothSystem: invalid particle range start=" + std::to_string(d->offset) +
                                    " count=" + std::to_string(d->n_particles));
  if (d->n_pairs == 0) return fail(PF_ERR_INVALID, "createDistanceConstraints: pairs is empty");
  const double comp = d->stretch_compliance >= 0 ? d->stretch_compliance : 1e-7;
  if (!std::isfinite(comp)) return fail(PF_ERR_INVALID, "ClothSystem: stretchCompliance must be >= 0");
  for (uint32_t q = 0; q < d->n_pairs; ++q) {
    const uint32_t i = d->pairs[2 * q], j = d->pairs[2 * q + 1];
    if (i >= d->n_particles || j >= d->n_particles)
      return fail(PF_ERR_INVALID, "createDistanceConstraints: pair has out-of-range index");
    if (i == j) return fail(PF_ERR_INVALID, "createDistanceConstraints: pair references the same particle");
  }
  // ClothSystem.ts:131-140: positions and masses from the graph, velocity 0.
  for (uint32_t k = 0; k < d->n_particles; ++k) {
    const uint32_t i = d->offset + k;
    for (int c = 0; c < 3; ++c) {
      sp.pos4[4 * i + c] = d->positions[3 * k + c];
      sp.vel4[4 * i + c] = 0.0f;
    }
    sp.pos4[4 * i + 3] = sp.vel4[4 * i + 3] = 0.0f;
    sp.inv_mass[i] = d->inv_mass[k];
  }
  ClothSpec cl;
  cl.offset = d->offset;
  cl.n = d->n_particles;
  cl.pairs.resize(2ull * d->n_pairs);
  for (size_t q = 0; q < cl.pairs.size(); ++q) cl.pairs[q] = d->offset + d->pairs[q];
  cl.rest.assign(d->rest_lengths, d->rest_lengths + d->n_pairs);
  cl.compliance = (float)comp;
  cl.colors = color_pairs(cl.pairs, d->n_pairs, sp.cap);
  // bending.ts:46-129: tuples of four distinct cloth particles, rest angles,
  // one compliance (ClothSystem default 1e-5), coloured with arity 4
  if (d->n_bending) {
    if (!d->bending || !d->bending_rest)
      return fail(PF_ERR_INVALID, "createClothBendingConstraints: tuples or restAngles missing");
    const double bc = d->bend_compliance >= 0 ? d->bend_compliance : 1e-5;
    if (!std::isfinite(bc)) return fail(PF_ERR_INVALID, "ClothSystem: bendCompliance must be >= 0");
    cl.bend.resize(4ull * d->n_bending);
    for (uint32_t q = 0; q < d->n_bending; ++q) {
      const uint32_t* t = d->bending + 4ull * q;
      for (int k = 0; k < 4; ++k) {
        if (t[k] >= d->n_particles)
          return fail(PF_ERR_INVALID, "createClothBendingConstraints: tuple index exceeds the cloth's particles");
        for (int m = 0; m < k; ++m)
          if (t[m] == t[k]) return fail(PF_ERR_INVALID, "createClothBendingConstraints: tuple has duplicate indices");
        cl.bend[4ull * q + k] = d->offset + t[k];
      }
    }
    cl.bend_rest.assign(d->bending_rest, d->bending_rest + d->n_bending);
    cl.bend_compliance = (float)bc;
    cl.bend_colors = color_groups(cl.bend, 4, d->n_bending, sp.cap);
  }
  // tether.ts:64-110: (free particle, anchor, rest radius) per tether, one
  // compliance (ClothSystem default 0), coloured with arity 1 on the particle
  if (d->n_tethers) {
    if (!d->tether_particle || !d->tether_anchor || !d->tether_rest)
      return fail(PF_ERR_INVALID, "createClothTetherConstraints: tether arrays missing");
    const double tc = d->tether_compliance >= 0 ? d->tether_compliance : 0.0;
    if (!std::isfinite(tc))
      return fail(PF_ERR_INVALID, "createClothTetherConstraints: compliance must be a non-negative finite number");
    cl.tether.resize(2ull * d->n_tethers);
    std::vector<uint32_t> who(d->n_tethers);
    for (uint32_t q = 0; q < d->n_tethers; ++q) {
      const uint32_t p = d->tether_particle[q], a = d->tether_anchor[q];
      if (p >= d->n_particles)
        return fail(PF_ERR_INVALID, "createClothTetherConstraints: tether particle " + std::to_string(p) + " out of range");
      if (a >= d->n_particles)
        return fail(PF_ERR_INVALID, "createClothTetherConstraints: tether anchor " + std::to_string(a) + " out of range");
      if (!(d->tether_rest[q] >= 0) || !std::isfinite(d->tether_rest[q]))
        return fail(PF_ERR_INVALID, "createClothTetherConstraints: tether for particle " + std::to_string(p) +
                                        " has invalid restRadius");
      cl.tether[2 * q] = d->offset + p;
      cl.tether[2 * q + 1] = d->offset + a;
      who[q] = d->offset + p;
    }
    cl.tether_rest.assign(d->tether_rest, d->tether_rest + d->n_tethers);
    cl.tether_compliance = (float)tc;
    cl.tether_colors = color_groups(who, 1, d->n_tethers, sp.cap);
  }
  // aero.ts:118-158: cloth-local triangles; drag 0.6125, lift 0.3 by default
  if (d->n_triangles) {
    if (!d->triangles) return fail(PF_ERR_INVALID, "createClothAeroKernel: triangles missing");
    cl.tris.resize(3ull * d->n_triangles);
    for (size_t q = 0; q < cl.tris.size(); ++q) {
      if (d->triangles[q] >= d->n_particles)
        return fail(PF_ERR_INVALID, "createClothAeroKernel: triangle " + std::to_string(q / 3) +
                                        " has out-of-range vertex " + std::to_string(d->triangles[q]));
      cl.tris[q] = d->offset + d->triangles[q];
    }
  }
  cl.drag = d->drag >= 0 ? d->drag : 0.6125f;
  cl.lift = d->lift >= 0 ? d->lift : 0.3f;
  if (!std::isfinite(cl.drag)) return fail(PF_ERR_INVALID, "ClothSystem: drag must be >= 0");
  if (!std::isfinite(cl.lift)) return fail(PF_ERR_INVALID, "ClothSystem: lift must be >= 0");
  for (int a = 0; a < 3; ++a) {
    if (!std::isfinite(d->wind[a])) return fail(PF_ERR_INVALID, "ClothSystem: wind must be finite");
    cl.wind[a] = d->wind[a];
  }
  cl.has_damping = d->has_damping != 0;
  if (cl.has_damping) {
    if (!(d->damping >= 0 && d->damping <= 1))
      return fail(PF_ERR_INVALID, "ClothSystem: damping must be between 0 and 1, got " + std::to_string(d->damping));
    cl.damping = d->damping;
  }
  sp.cloths.push_back(std::move(cl));
  sp.materials.push_back({MAT_CLOTH, (uint32_t)sp.cloths.size() - 1});
  if (mat) *mat = (uint32_t)sp.materials.size() - 1;
  return PF_OK;
}

static const ClothSpec* cloth_of(const SceneSpec& sp, uint32_t mat) {
  if (mat >= sp.materials.size() || sp.materials[mat].first != MAT_CLOTH) return nullptr;
  return &sp.cloths[sp.materials[mat].second];
}

// ClothSystem.ts:152-188: the setters' checks.
static pf_status check_cloth_params(const ClothSpec& cl, const pf_cloth_params& p) {
  auto nonneg = [](float v, const char* name) -> pf_status {
    if (!(v >= 0) || !std::isfinite(v))
      return fail(PF_ERR_INVALID, std::string("ClothSystem: ") + name + " must be >= 0, got " + std::to_string(v));
    return PF_OK;
  };
  PF_TRY(nonneg(p.drag, "drag"));
  PF_TRY(nonneg(p.lift, "lift"));
  PF_TRY(nonneg(p.bend_compliance, "bendCompliance"));
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(p.wind[a])) return fail(PF_ERR_INVALID, "ClothSystem: wind must be finite");
  if (!(p.damping >= 0 && p.damping <= 1))
    return fail(PF_ERR_INVALID, "ClothSystem: damping must be between 0 and 1, got " + std::to_string(p.damping));
  if (p.damping != cl.damping && !cl.has_damping)
    return fail(PF_ERR_INVALID, "ClothSystem: damping was not given at creation, so there is no smoothing pass to change");
  return PF_OK;
}

pf_status pf_cloth_get_params(pf_scene* s, uint32_t mat, pf_cloth_params* out) {
  if (!s || !out) return fail(PF_ERR_INVALID, "ClothSystem: NULL argument");
  const ClothSpec* cl = cloth_of(s->spec, mat);
  if (!cl) return fail(PF_ERR_INVALID, "ClothSystem: material " + std::to_string(mat) + " is not a cloth");
  for (int a = 0; a < 3; ++a) out->wind[a] = cl->wind[a];
  out->drag = cl->drag;
  out->lift = cl->lift;
  out->damping = cl->damping;
  out->bend_compliance = cl->bend_compliance;
  return PF_OK;
}

pf_status pf_cloth_set_params(pf_scene* s, uint32_t mat, const pf_cloth_params* p) {
  if (!s || !p) return fail(PF_ERR_INVALID, "ClothSystem: NULL argument");
  const ClothSpec* cl = cloth_of(s->spec, mat);
  if (!cl) return fail(PF_ERR_INVALID, "ClothSystem: material " + std::to_string(mat) + " is not a cloth");
  PF_TRY(check_cloth_params(*cl, *p));
  if (s->world) return s->world->set_cloth_params(0, mat, *p);
  ClothSpec& w = s->spec.cloths[s->spec.materials[mat].second];
  for (int a = 0; a < 3; ++a) w.wind[a] = p->wind[a];
  w.drag = p->drag;
  w.lift = p->lift;
  w.damping = p->damping;
  w.bend_compliance = p->bend_compliance;
  return PF_OK;
}

// tetherBuild.ts:226-275: a binary min-heap on the distance alone, with the
// reference's sift rules (strict comparisons), so that equal distances leave
// the heap in the same order and Dijkstra keeps the same nearest anchor.
namespace {
struct DistHeap {
  std::vector<std::pair<double, uint32_t>> d;
  void push(double dist, uint32_t u) {
    d.push_back({dist, u});
    size_t i = d.size() - 1;
    while (i > 0) {
      const size_t p = (i - 1) >> 1;
      if (d[i].first < d[p].first) {
        std::swap(d[i], d[p]);
        i = p;
      } else {
        break;
      }
    }
  }
  std::pair<double, uint32_t> pop() {
    const auto top = d[0];
    const auto last = d.back();
    d.pop_back();
    if (!d.empty()) {
      d[0] = last;
      size_t i = 0;
      const size_t n = d.size();
      for (;;) {
        const size_t l = 2 * i + 1, r = 2 * i + 2;
        size_t m = i;
        if (l < n && d[l].first < d[m].first) m = l;
        if (r < n && d[r].first < d[m].first) m = r;
        if (m == i) break;
        std::swap(d[i], d[m]);
        i = m;
      }
    }
    return top;
  }
};
}  // namespace

pf_status pf_cloth_build_tethers(const pf_tether_build_desc* desc, uint32_t* particle, uint32_t* anchor,
                                 float* rest, uint32_t capacity, uint32_t* count) {
  if (!desc || !count) return fail(PF_ERR_INVALID, "buildTethers: NULL argument");
  *count = 0;
  const uint32_t n = desc->n_particles;
  const uint32_t max_att = desc->max_attachments ? desc->max_attachments : 4u;
  if (!(desc->stretch_tolerance >= 0) || !std::isfinite(desc->stretch_tolerance))
    return fail(PF_ERR_INVALID, "buildTethers: stretchTolerance must be a non-negative finite number, got " +
                                    std::to_string(desc->stretch_tolerance));
  if (n && !desc->inv_mass) return fail(PF_ERR_INVALID, "buildTethers: invMass missing");
  if (desc->n_pairs && (!desc->pairs || !desc->rest_lengths)) return fail(PF_ERR_INVALID, "buildTethers: pairs missing");
  for (uint64_t q = 0; q < 2ull * desc->n_pairs; ++q)
    if (desc->pairs[q] >= n) return fail(PF_ERR_INVALID, "buildTethers: pair has out-of-range index");
  std::vector<uint8_t> pinned(n);
  uint32_t n_pinned = 0;
  for (uint32_t i = 0; i < n; ++i) n_pinned += (pinned[i] = desc->inv_mass[i] == 0.0f);
  if (n_pinned == 0) return PF_OK;
  // adjacency in pair order, both directions (tetherBuild.ts:129-136)
  std::vector<uint32_t> off(n + 1, 0);
  for (uint64_t q = 0; q < 2ull * desc->n_pairs; ++q) ++off[desc->pairs[q] + 1];
  for (uint32_t v = 0; v < n; ++v) off[v + 1] += off[v];
  std::vector<uint32_t> to(off.back()), cur(off.begin(), off.end() - 1);
  std::vector<double> wt(off.back());
  for (uint32_t e = 0; e < desc->n_pairs; ++e) {
    const uint32_t a = desc->pairs[2 * e], b = desc->pairs[2 * e + 1];
    to[cur[a]] = b;
    wt[cur[a]++] = desc->rest_lengths[e];
    to[cur[b]] = a;
    wt[cur[b]++] = desc->rest_lengths[e];
  }
  // islands: connected pinned particles over pinned-only edges (:141-157)
  std::vector<int32_t> island(n, -1);
  int32_t n_islands = 0;
  for (uint32_t s0 = 0; s0 < n; ++s0) {
    if (!pinned[s0] || island[s0] != -1) continue;
    const int32_t id = n_islands++;
    std::vector<uint32_t> stack{s0};
    island[s0] = id;
    while (!stack.empty()) {
      const uint32_t u = stack.back();
      stack.pop_back();
      for (uint32_t m = off[u]; m < off[u + 1]; ++m)
        if (pinned[to[m]] && island[to[m]] == -1) {
          island[to[m]] = id;
          stack.push_back(to[m]);
        }
    }
  }
  // one multi-source Dijkstra per island (:172-207)
  struct Att {
    int32_t island;
    double dist;
    uint32_t anchor;
  };
  std::vector<std::vector<Att>> atts(n);
  std::vector<double> dist(n);
  std::vector<int64_t> nearest(n);
  for (int32_t id = 0; id < n_islands; ++id) {
    std::fill(dist.begin(), dist.end(), std::numeric_limits<double>::infinity());
    std::fill(nearest.begin(), nearest.end(), -1);
    DistHeap heap;
    for (uint32_t i = 0; i < n; ++i)
      if (pinned[i] && island[i] == id) {
        dist[i] = 0;
        nearest[i] = i;
        heap.push(0.0, i);
      }
    while (!heap.d.empty()) {
      const auto [du, u] = heap.pop();
      if (du > dist[u]) continue;
      for (uint32_t m = off[u]; m < off[u + 1]; ++m) {
        const double nd = du + wt[m];
        if (nd < dist[to[m]]) {
          dist[to[m]] = nd;
          nearest[to[m]] = nearest[u];
          heap.push(nd, to[m]);
        }
      }
    }
    for (uint32_t v = 0; v < n; ++v)
      if (!pinned[v] && std::isfinite(dist[v])) atts[v].push_back({id, dist[v], (uint32_t)nearest[v]});
  }
  // the closest max_attachments islands of each free particle (:211-219)
  const double scale = 1.0 + desc->stretch_tolerance;
  uint32_t k = 0;
  for (uint32_t v = 0; v < n; ++v) {
    if (pinned[v]) continue;
    auto& list = atts[v];
    std::stable_sort(list.begin(), list.end(), [](const Att& a, const Att& b) {
      return a.dist < b.dist || (a.dist == b.dist && a.island < b.island);
    });
    const size_t take = std::min<size_t>(max_att, list.size());
    for (size_t q = 0; q < take; ++q) {
      if (k >= capacity) return fail(PF_ERR_INVALID, "buildTethers: output capacity " + std::to_string(capacity) + " too small");
      if (particle) particle[k] = v;
      if (anchor) anchor[k] = list[q].anchor;
      if (rest) rest[k] = (float)(list[q].dist * scale);
      ++k;
    }
  }
  *count = k;
  return PF_OK;
}

pf_status pf_add_primitive(pf_scene* s, const pf_primitive* p, uint32_t* slot) {
  PF_TRY(not_built(s, "PrimitiveSet"));
  if (!p || p->kind > PF_PRIM_CAPSULE) return fail(PF_ERR_INVALID, "PrimitiveSet: unknown primitive kind");
  if (!(p->data1[3] >= 0) || !(p->velocity[3] >= 0))
    return fail(PF_ERR_INVALID, "PrimitiveSet: friction coefficients must be non-negative");
  s->spec.prims.push_back(*p);
  if (slot) *slot = (uint32_t)s->spec.prims.size() - 1;
  return PF_OK;
}

pf_status pf_set_primitive(pf_scene* s, uint32_t slot, const pf_primitive* p) {
  if (!s || !p) return fail(PF_ERR_INVALID, "PrimitiveSet: NULL argument");
  if (slot >= s->spec.prims.size()) return fail(PF_ERR_INVALID, "PrimitiveSet: no primitive in slot " + std::to_string(slot));
  if (s->world) return s->world->set_primitive(0, slot, *p);
  s->spec.prims[slot] = *p;
  return PF_OK;
}

pf_status pf_add_sdf_collider(pf_scene* s, const pf_sdf_desc* d, uint32_t* slot) {
  PF_TRY(not_built(s, "SDFCollider"));
  if (!d || !d->data) return fail(PF_ERR_INVALID, "SDFCollider: no distance data");
  for (int a = 0; a < 3; ++a)
    if (d->res[a] < 4)
      return fail(PF_ERR_INVALID, "SDFCollider: resolution must be integers >= 4, got [" + std::to_string(d->res[0]) +
                                      ", " + std::to_string(d->res[1]) + ", " + std::to_string(d->res[2]) + "]");
  const uint64_t n = (uint64_t)d->res[0] * d->res[1] * d->res[2];
  if (n > (1ull << 31)) return fail(PF_ERR_INVALID, "SDFCollider: grid too large");
  for (int a = 0; a < 3; ++a)
    if (!(d->voxel_size[a] > 0) || !std::isfinite(d->voxel_size[a]))
      return fail(PF_ERR_INVALID, "SDFCollider: voxel size must be positive");
  if (!(d->thickness >= 0) || !std::isfinite(d->thickness))
    return fail(PF_ERR_INVALID, "SDFCollider: thickness must be non-negative, got " + std::to_string(d->thickness));
  if (!(d->mu_s >= 0) || !(d->mu_k >= 0))
    return fail(PF_ERR_INVALID, "SDFCollider: friction coefficients must be non-negative");
  SdfSpec g;
  PF_TRY(sdf_transform(d->position, d->rotation, d->scale, &g));
  for (int a = 0; a < 3; ++a) {
    g.res[a] = d->res[a];
    g.origin[a] = d->origin[a];
    g.voxel[a] = d->voxel_size[a];
  }
  g.thickness = d->thickness;
  g.mu_s = d->mu_s;
  g.mu_k = d->mu_k;
  g.half.resize(n);
  for (uint64_t i = 0; i < n; ++i) g.half[i] = half_rn(d->data[i]);
  s->spec.sdfs.push_back(std::move(g));
  if (slot) *slot = (uint32_t)s->spec.sdfs.size() - 1;
  return PF_OK;
}

pf_status pf_set_sdf_transform(pf_scene* s, uint32_t slot, const float position[3], const float rotation[4],
                               float scale) {
  if (!s || !position || !rotation) return fail(PF_ERR_INVALID, "SDFCollider: NULL argument");
  if (slot >= s->spec.sdfs.size())
    return fail(PF_ERR_INVALID, "SDFCollider: no collider in slot " + std::to_string(slot));
  SdfSpec t;
  PF_TRY(sdf_transform(position, rotation, scale, &t));
  if (s->world) return s->world->set_sdf_transform(0, slot, t.position, t.rot_q, t.scale);
  SdfSpec& g = s->spec.sdfs[slot];
  for (int a = 0; a < 3; ++a) g.position[a] = t.position[a];
  for (int a = 0; a < 4; ++a) g.rot_q[a] = t.rot_q[a];
  g.scale = t.scale;
  return PF_OK;
}

pf_status pf_add_no_self_contacts(pf_scene* s, pf_range r) {
  PF_TRY(not_built(s, "Material"));
  if (!range_ok(s->spec, {r.start, r.count}))
    return fail(PF_ERR_INVALID, "Material: invalid noSelfContacts range start=" + std::to_string(r.start) +
                                    " count=" + std::to_string(r.count));
  s->spec.quiet.push_back({r.start, r.count});
  return PF_OK;
}

pf_status pf_contacts_read(pf_scene* s, uint32_t* pairs, uint32_t capacity, uint32_t* count, uint32_t* stored) {
  if (!s) return fail(PF_ERR_INVALID, "contacts: scene is NULL");
  if (!s->world) return fail(PF_ERR_STATE, "contacts: build the SimLoop first");
  return s->world->contacts(0, pairs, capacity, count, stored);
}

pf_status pf_loop_build(pf_scene* s, const pf_loop_desc* d) {
  PF_TRY(not_built(s, "SimLoop"));
  if (!d) return fail(PF_ERR_INVALID, "SimLoop: options are NULL");
  if (d->substeps < 1) return fail(PF_ERR_INVALID, "SimLoop: substeps must be an integer >= 1, got 0");
  if (d->contact) {
    const float ms = d->contact_mu_s >= 0 ? d->contact_mu_s : 0.5f, mk = d->contact_mu_k >= 0 ? d->contact_mu_k : 0.4f;
    if (!std::isfinite(ms) || !std::isfinite(mk))
      return fail(PF_ERR_INVALID, "SimLoop: friction coefficients must be non-negative");
  }
  PF_TRY(allocate_collision_groups(s->spec));
  s->spec.loop = *d;
  s->spec.built = true;
  auto w = std::make_unique<World>();
  const pf_status st = w->build({&s->spec}, false);
  if (st != PF_OK) {
    s->spec.built = false;
    return st;
  }
  s->world = std::move(w);
  return PF_OK;
}

pf_status pf_step(pf_scene* s, double dt) {
  if (!s) return fail(PF_ERR_INVALID, "SimLoop: scene is NULL");
  if (!s->world) return fail(PF_ERR_STATE, "SimLoop: build the loop before stepping");
  return s->world->step(dt);
}

pf_status pf_write(pf_scene* s, uint32_t field, const void* src, size_t bytes) {
  if (!s || !src) return fail(PF_ERR_INVALID, "write: NULL argument");
  if (s->world) return s->world->write(0, field, src, bytes);
  SceneSpec& sp = s->spec;
  const float* f = static_cast<const float*>(src);
  const size_t n4 = 16ull * sp.cap, n1 = 4ull * sp.cap;
  switch (field) {
    case PF_FIELD_POSITIONS:
    case PF_FIELD_VELOCITIES: {
      if (bytes < n4) return fail(PF_ERR_INVALID, "write: source too small");
      std::vector<float>& dst = field == PF_FIELD_POSITIONS ? sp.pos4 : sp.vel4;
      for (size_t i = 0; i < 4ull * sp.cap; ++i)
        if (!std::isfinite(f[i])) return fail(PF_ERR_INVALID, "write: values must be finite");
      for (size_t i = 0; i < sp.cap; ++i)
        for (int c = 0; c < 3; ++c) dst[4 * i + c] = f[4 * i + c];
      return PF_OK;
    }
    case PF_FIELD_INV_MASS:
      if (bytes < n1) return fail(PF_ERR_INVALID, "write: source too small");
      for (size_t i = 0; i < sp.cap; ++i)
        if (!(f[i] >= 0) || !std::isfinite(f[i])) return fail(PF_ERR_INVALID, "write: invMass must be a finite number >= 0");
      std::copy(f, f + sp.cap, sp.inv_mass.begin());
      return PF_OK;
    case PF_FIELD_PREDICTED:
      return fail(PF_ERR_STATE, "write: predicted positions exist once the SimLoop is built");
    default:
      return fail(PF_ERR_INVALID, "write: field " + std::to_string(field) + " cannot be written");
  }
}

pf_status pf_readback(pf_scene* s, uint32_t field, void* dst, size_t bytes) {
  if (!s || !dst) return fail(PF_ERR_INVALID, "readback: NULL argument");
  if (s->world) return s->world->readback(0, field, dst, bytes);
  return pf::spec_readback(s->spec, field, dst, bytes);
}

}  // extern "C"

// loop.ts:163-166 with SoftbodySystem.ts:218-234: collision groups above
// every uploaded one, one per soft body that has none of its own, in
// material then body order (unless the system collides with itself).
pf_status pf::allocate_collision_groups(SceneSpec& sp) {
  uint32_t next = 1;
  for (uint32_t g : sp.group) next = std::max(next, g + 1);
  for (auto& m : sp.materials) {
    if (m.first != MAT_SOFT) continue;
    const SoftSpec& ss = sp.softs[m.second];
    if (ss.self_collision) continue;
    for (size_t b = 0; b < ss.bodies.size(); ++b) {
      const RangeU r = ss.bodies[b].range;
      if (!r.count) continue;
      const uint32_t g0 = sp.group[r.start];
      bool shared = true;
      for (uint32_t i = r.start; i < r.start + r.count; ++i) shared = shared && sp.group[i] == g0;
      if (shared && g0 != 0) continue;
      if (!shared)
        return fail(PF_ERR_INVALID, "SoftbodySystem: body " + std::to_string(b) +
                                        " has mixed collision groups; give all its particles one group, or none");
      for (uint32_t i = r.start; i < r.start + r.count; ++i) sp.group[i] = next;
      ++next;
    }
  }
  return PF_OK;
}

pf_status pf::spec_readback(const SceneSpec& sp, uint32_t field, void* dst, size_t bytes) {
  auto copy = [&](const void* src, size_t b) -> pf_status {
    if (bytes < b) return fail(PF_ERR_INVALID, "readback: destination too small");
    std::memcpy(dst, src, b);
    return PF_OK;
  };
  switch (field) {
    case PF_FIELD_POSITIONS:
    case PF_FIELD_PREDICTED: return copy(sp.pos4.data(), 16ull * sp.cap);
    case PF_FIELD_VELOCITIES: return copy(sp.vel4.data(), 16ull * sp.cap);
    case PF_FIELD_INV_MASS: return copy(sp.inv_mass.data(), 4ull * sp.cap);
    case PF_FIELD_BOUNDARY_VOLUME: return copy(sp.bvol.data(), 4ull * sp.cap);
    case PF_FIELD_ROTATION:
    case PF_FIELD_PREDICTED_ROTATION: return copy(sp.rot4.data(), 16ull * sp.cap);
    case PF_FIELD_ANGULAR_VELOCITY: return copy(sp.angv4.data(), 16ull * sp.cap);
    default: return fail(PF_ERR_STATE, "readback: field is available once the SimLoop is built");
  }
}

extern "C" {

pf_status pf_overflow_read(pf_scene* s, pf_overflow* out) {
  if (!s || !out) return fail(PF_ERR_INVALID, "readbackOverflow: NULL argument");
  std::memset(out, 0, sizeof(*out));
  if (!s->world) return PF_OK;
  return s->world->overflow(0, out);
}

pf_status pf_last_step_ms(pf_scene* s, float* ms) {
  if (!s || !ms || !s->world) return fail(PF_ERR_STATE, "SimLoop: no step has run");
  return s->world->elapsed_ms(ms);
}

// ----------------------------------------------------------------- batch ----

pf_status pf_batch_create(pf_scene* const* scenes, uint32_t n, const pf_batch_opts* opts, pf_batch** out) {
  if (!scenes || !n || !out) return fail(PF_ERR_INVALID, "batch: no scenes");
  auto b = std::make_unique<pf_batch>();
  std::vector<SceneSpec*> specs;
  for (uint32_t i = 0; i < n; ++i) {
    pf_scene* s = scenes[i];
    if (!s || !s->world) return fail(PF_ERR_STATE, "batch: scene " + std::to_string(i) + " has no built SimLoop");
    auto copy = std::make_unique<SceneSpec>(s->spec);
    PF_TRY(s->world->pull_state(0, copy.get()));
    specs.push_back(copy.get());
    b->specs.push_back(std::move(copy));
  }
  b->world = std::make_unique<World>();
  PF_TRY(b->world->build(specs, opts ? opts->use_graph != 0 : true));
  *out = b.release();
  return PF_OK;
}

void pf_batch_destroy(pf_batch* b) { delete b; }

pf_status pf_batch_step(pf_batch* b, double dt) {
  if (!b) return fail(PF_ERR_INVALID, "batch: NULL");
  return b->world->step(dt);
}

pf_status pf_batch_set_primitive(pf_batch* b, uint32_t index, uint32_t slot, const pf_primitive* p) {
  if (!b || !p) return fail(PF_ERR_INVALID, "batch: NULL");
  return b->world->set_primitive(index, slot, *p);
}

pf_status pf_batch_cloth_set_params(pf_batch* b, uint32_t index, uint32_t mat, const pf_cloth_params* p) {
  if (!b || !p) return fail(PF_ERR_INVALID, "batch: NULL");
  if (index >= b->specs.size()) return fail(PF_ERR_INVALID, "batch: no scene " + std::to_string(index));
  const ClothSpec* cl = cloth_of(*b->specs[index], mat);
  if (!cl) return fail(PF_ERR_INVALID, "ClothSystem: material " + std::to_string(mat) + " is not a cloth");
  PF_TRY(check_cloth_params(*cl, *p));
  return b->world->set_cloth_params(index, mat, *p);
}

pf_status pf_batch_write(pf_batch* b, uint32_t index, uint32_t field, const void* src, size_t bytes) {
  if (!b || !src) return fail(PF_ERR_INVALID, "batch: NULL");
  return b->world->write(index, field, src, bytes);
}

pf_status pf_batch_readback(pf_batch* b, uint32_t index, uint32_t field, void* dst, size_t bytes) {
  if (!b || !dst) return fail(PF_ERR_INVALID, "batch: NULL");
  return b->world->readback(index, field, dst, bytes);
}

pf_status pf_batch_overflow_read(pf_batch* b, uint32_t index, pf_overflow* out) {
  if (!b || !out) return fail(PF_ERR_INVALID, "batch: NULL");
  return b->world->overflow(index, out);
}

pf_status pf_batch_last_step_ms(pf_batch* b, float* ms) {
  if (!b || !ms) return fail(PF_ERR_INVALID, "batch: NULL");
  return b->world->elapsed_ms(ms);
}

uint64_t pf_batch_particle_substeps(pf_batch* b) { return b ? b->world->particle_substeps_per_step() : 0; }

uint64_t pf_batch_launches_per_step(pf_batch* b) { return b ? b->world->launches_per_step() : 0; }
uint64_t pf_batch_step_upload_bytes(pf_batch* b) { return b ? b->world->step_upload_bytes() : 0; }

void* pf_batch_stream(pf_batch* b) { return b ? (void*)b->world->stream() : nullptr; }
void* pf_scene_stream(pf_scene* s) { return (s && s->world) ? (void*)s->world->stream() : nullptr; }

pf_status pf_batch_read_positions(pf_batch* b, float* dst_host, size_t bytes) {
  if (!b || !dst_host) return fail(PF_ERR_INVALID, "batch: NULL");
  return b->world->read_positions(dst_host, bytes);
}

pf_status pf_batch_read_positions_async(pf_batch* b, float* dst_host, size_t bytes) {
  if (!b || !dst_host) return fail(PF_ERR_INVALID, "batch: NULL");
  return b->world->read_positions_async(dst_host, bytes);
}

pf_status pf_batch_wait_reads(pf_batch* b) {
  if (!b) return fail(PF_ERR_INVALID, "batch: NULL");
  return b->world->wait_reads();
}

pf_status pf_batch_tuning(pf_batch* b, uint32_t* path, uint32_t* block, uint32_t* unroll, uint32_t* group,
                          uint32_t* entry_bits) {
  if (!b || !path || !block || !unroll) return fail(PF_ERR_INVALID, "batch: NULL");
  b->world->tuning(path, block, unroll);
  if (group) *group = b->world->tuning_all().group;
  if (entry_bits) *entry_bits = b->world->tuning_all().nbr_wide ? 32u : 16u;
  return PF_OK;
}

pf_status pf_batch_profile_stage(pf_batch* b, uint32_t stage, uint32_t reps, float* ms, uint64_t* items) {
  if (!b || !ms) return fail(PF_ERR_INVALID, "batch: NULL");
  return b->world->profile_stage(stage, reps, ms, items);
}

}  // extern "C"
