/*
 * pfsim_napi.c — Node-API addon over libpfsim.so (include/pfsim.h).
 *
 * The reference keeps its host in TypeScript on Node.js; a maintainer who
 * moves its solver step onto this library builds this addon with node-gyp
 * (binding.gyp beside this file) and uses pfsim.ts, which mirrors the
 * reference's SimLoop / ParticleSystem / material / collider classes on top
 * of it. Every export is a thin marshalling layer: JavaScript objects and
 * typed arrays become the plain structs and pointers of pfsim.h, a non-OK
 * status becomes a thrown Error carrying pf_last_error() (the reference's
 * "<Class>: <reason>" text), and step() runs on libuv's thread pool and
 * returns a Promise, as the reference's SimLoop.step does.
 *
 * Not built or run on the machine this repository was developed on: it has
 * no Node.js. The Python binding (pfsim/_native.py) calls the same entry
 * points in the same order and is what the tests exercise.
 *
 * Typed arrays are checked for their element type and length before their
 * memory is handed to the library, so a Float64Array where a Float32Array is
 * expected throws instead of being read with the wrong stride.
 */
#include <node_api.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "pfsim.h"

/* ------------------------------------------------------------ helpers --- */

#define CHECK_NAPI(call)                                                      \
  do {                                                                        \
    if ((call) != napi_ok) {                                                  \
      napi_throw_error(env, NULL, "pfsim: N-API call failed: " #call);        \
      return NULL;                                                            \
    }                                                                         \
  } while (0)

static napi_value throw_msg(napi_env env, const char* msg) {
  napi_throw_error(env, NULL, msg);
  return NULL;
}

static napi_value throw_last(napi_env env) { return throw_msg(env, pf_last_error()); }

static napi_value undefined(napi_env env) {
  napi_value v;
  napi_get_undefined(env, &v);
  return v;
}

static napi_value make_u32(napi_env env, uint32_t x) {
  napi_value v;
  napi_create_uint32(env, x, &v);
  return v;
}

static napi_value make_f64(napi_env env, double x) {
  napi_value v;
  napi_create_double(env, x, &v);
  return v;
}

static int has(napi_env env, napi_value obj, const char* name) {
  bool b = false;
  napi_value v;
  napi_valuetype t;
  if (napi_has_named_property(env, obj, name, &b) != napi_ok || !b) return 0;
  if (napi_get_named_property(env, obj, name, &v) != napi_ok) return 0;
  napi_typeof(env, v, &t);
  return t != napi_undefined && t != napi_null;
}

static double get_f64(napi_env env, napi_value obj, const char* name, double dflt) {
  napi_value v;
  double x = dflt;
  if (!has(env, obj, name)) return dflt;
  napi_get_named_property(env, obj, name, &v);
  if (napi_get_value_double(env, v, &x) != napi_ok) return dflt;
  return x;
}

static uint32_t get_u32(napi_env env, napi_value obj, const char* name, uint32_t dflt) {
  napi_value v;
  uint32_t x = dflt;
  if (!has(env, obj, name)) return dflt;
  napi_get_named_property(env, obj, name, &v);
  if (napi_get_value_uint32(env, v, &x) != napi_ok) return dflt;
  return x;
}

static int get_bool(napi_env env, napi_value obj, const char* name, int dflt) {
  napi_value v;
  bool b = dflt != 0;
  if (!has(env, obj, name)) return dflt;
  napi_get_named_property(env, obj, name, &v);
  if (napi_get_value_bool(env, v, &b) != napi_ok) return dflt;
  return b ? 1 : 0;
}

/* obj[name] as an array of n numbers (a JS array or any typed array). */
static int get_vec(napi_env env, napi_value obj, const char* name, uint32_t n, double* out) {
  napi_value arr, e;
  if (!has(env, obj, name)) return 0;
  napi_get_named_property(env, obj, name, &arr);
  for (uint32_t i = 0; i < n; ++i) {
    if (napi_get_element(env, arr, i, &e) != napi_ok || napi_get_value_double(env, e, &out[i]) != napi_ok)
      return 0;
  }
  return 1;
}

/* A typed array of element type `want` (or null/undefined when `optional`):
 * its data pointer and element count. Returns 0 after throwing on a wrong
 * type. */
static int typed(napi_env env, napi_value v, napi_typedarray_type want, int optional, void** data, size_t* len) {
  napi_valuetype t;
  bool is_typed = false;
  napi_typedarray_type ty;
  *data = NULL;
  *len = 0;
  napi_typeof(env, v, &t);
  if (t == napi_undefined || t == napi_null) {
    if (optional) return 1;
    napi_throw_type_error(env, NULL, "pfsim: a typed array is required");
    return 0;
  }
  napi_is_typedarray(env, v, &is_typed);
  if (!is_typed || napi_get_typedarray_info(env, v, &ty, len, data, NULL, NULL) != napi_ok || ty != want) {
    napi_throw_type_error(env, NULL,
                          want == napi_float32_array   ? "pfsim: expected a Float32Array"
                          : want == napi_uint32_array  ? "pfsim: expected a Uint32Array"
                          : want == napi_float64_array ? "pfsim: expected a Float64Array"
                          : want == napi_uint8_array   ? "pfsim: expected a Uint8Array"
                                                       : "pfsim: wrong typed array type");
    return 0;
  }
  return 1;
}

static int typed_prop(napi_env env, napi_value obj, const char* name, napi_typedarray_type want, int optional,
                      void** data, size_t* len) {
  napi_value v;
  if (!has(env, obj, name)) {
    *data = NULL;
    *len = 0;
    if (optional) return 1;
    napi_throw_type_error(env, NULL, "pfsim: a required typed array field is missing");
    return 0;
  }
  napi_get_named_property(env, obj, name, &v);
  return typed(env, v, want, optional, data, len);
}

/* Bytes per element of a typed array type (for readback/write sizes). */
static size_t elem_bytes(napi_typedarray_type t) {
  switch (t) {
    case napi_int8_array:
    case napi_uint8_array:
    case napi_uint8_clamped_array: return 1;
    case napi_int16_array:
    case napi_uint16_array: return 2;
    case napi_int32_array:
    case napi_uint32_array:
    case napi_float32_array: return 4;
    default: return 8;
  }
}

/* A scene handle as a JS External: the wrapper lets dispose() and the
 * garbage collector agree on who frees it. */
typedef struct {
  pf_scene* scene;
  int busy; /* a step is running on the thread pool */
} SceneBox;

static void scene_finalize(napi_env env, void* data, void* hint) {
  SceneBox* b = (SceneBox*)data;
  (void)env;
  (void)hint;
  if (b->scene && !b->busy) pf_scene_destroy(b->scene);
  free(b);
}

static SceneBox* scene_of(napi_env env, napi_value v) {
  SceneBox* b = NULL;
  if (napi_get_value_external(env, v, (void**)&b) != napi_ok || !b) {
    napi_throw_type_error(env, NULL, "pfsim: expected a scene handle");
    return NULL;
  }
  if (!b->scene) {
    napi_throw_error(env, NULL, "ParticleSystem: has been disposed");
    return NULL;
  }
  if (b->busy) {
    napi_throw_error(env, NULL, "SimLoop: a step is running on this scene; await it first");
    return NULL;
  }
  return b;
}

#define ARGS(n)                                                        \
  size_t argc = (n);                                                   \
  napi_value argv[(n) > 0 ? (n) : 1];                                  \
  CHECK_NAPI(napi_get_cb_info(env, info, &argc, argv, NULL, NULL));    \
  if (argc < (n)) return throw_msg(env, "pfsim: too few arguments")

/* ------------------------------------------------------------- scene --- */

/* createScene(capacity, particleRadius) -> scene (new ParticleSystem) */
static napi_value create_scene(napi_env env, napi_callback_info info) {
  ARGS(2);
  uint32_t cap;
  double radius;
  CHECK_NAPI(napi_get_value_uint32(env, argv[0], &cap));
  CHECK_NAPI(napi_get_value_double(env, argv[1], &radius));
  pf_scene_desc d = {cap, (float)radius};
  pf_scene* s = NULL;
  if (pf_scene_create(&d, &s) != PF_OK) return throw_last(env);
  SceneBox* b = (SceneBox*)calloc(1, sizeof *b);
  if (!b) {
    pf_scene_destroy(s);
    return throw_msg(env, "pfsim: out of host memory");
  }
  b->scene = s;
  napi_value out;
  CHECK_NAPI(napi_create_external(env, b, scene_finalize, NULL, &out));
  return out;
}

/* destroyScene(scene): dispose(); later calls throw "has been disposed" */
static napi_value destroy_scene(napi_env env, napi_callback_info info) {
  ARGS(1);
  SceneBox* b = NULL;
  CHECK_NAPI(napi_get_value_external(env, argv[0], (void**)&b));
  if (b && b->busy) return throw_msg(env, "SimLoop: dispose while a step is running; await it first");
  if (b && b->scene) {
    pf_scene_destroy(b->scene);
    b->scene = NULL;
  }
  return undefined(env);
}

/* uploadParticles(scene, pos4: Float32Array, vel4|null, invMass|null, group: Uint32Array|null, start) */
static napi_value upload(napi_env env, napi_callback_info info) {
  ARGS(6);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  void *pos, *vel, *w, *g;
  size_t np, nv, nw, ng;
  if (!typed(env, argv[1], napi_float32_array, 0, &pos, &np)) return NULL;
  if (!typed(env, argv[2], napi_float32_array, 1, &vel, &nv)) return NULL;
  if (!typed(env, argv[3], napi_float32_array, 1, &w, &nw)) return NULL;
  if (!typed(env, argv[4], napi_uint32_array, 1, &g, &ng)) return NULL;
  uint32_t start;
  CHECK_NAPI(napi_get_value_uint32(env, argv[5], &start));
  const uint32_t n = (uint32_t)(np / 4);
  if (np % 4 || (vel && nv != np) || (w && nw != n) || (g && ng != n))
    return throw_msg(env, "ParticleSystem.uploadParticles: array lengths disagree (4 floats per position)");
  if (pf_upload_particles(b->scene, (const float*)pos, (const float*)vel, (const float*)w, (const uint32_t*)g, start,
                          n) != PF_OK)
    return throw_last(env);
  return undefined(env);
}

/* setInvMass(scene, start, count, invMass) */
static napi_value set_inv_mass(napi_env env, napi_callback_info info) {
  ARGS(4);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  pf_range r;
  double w;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &r.start));
  CHECK_NAPI(napi_get_value_uint32(env, argv[2], &r.count));
  CHECK_NAPI(napi_get_value_double(env, argv[3], &w));
  if (pf_set_inv_mass(b->scene, r, (float)w) != PF_OK) return throw_last(env);
  return undefined(env);
}

/* --------------------------------------------------------- materials --- */

/* addFluid(scene, {start, count, restDensity, particleSpacing, smoothingRadius,
 *   compliance, viscosity, vorticity, surfaceTension, adhesion,
 *   boundaries: [{start, count, dynamic}]}) -> material index */
static napi_value add_fluid(napi_env env, napi_callback_info info) {
  ARGS(2);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  napi_value o = argv[1];
  pf_fluid_desc d;
  memset(&d, 0, sizeof d);
  d.range.start = get_u32(env, o, "start", 0);
  d.range.count = get_u32(env, o, "count", 0);
  d.rest_density = (float)get_f64(env, o, "restDensity", 0.0);
  d.particle_spacing = (float)get_f64(env, o, "particleSpacing", 0.0);
  d.smoothing_radius = (float)get_f64(env, o, "smoothingRadius", 0.0);
  d.compliance = (float)get_f64(env, o, "compliance", -1.0);
  if (has(env, o, "viscosity")) {
    d.flags |= PF_FLUID_VISCOSITY;
    d.viscosity = (float)get_f64(env, o, "viscosity", 0.0);
  }
  if (has(env, o, "vorticity")) {
    d.flags |= PF_FLUID_VORTICITY;
    d.vorticity = (float)get_f64(env, o, "vorticity", 0.0);
  }
  if (has(env, o, "surfaceTension")) {
    d.flags |= PF_FLUID_SURFACE_TENSION;
    d.surface_tension = (float)get_f64(env, o, "surfaceTension", 0.0);
  }
  if (has(env, o, "adhesion")) {
    d.flags |= PF_FLUID_ADHESION;
    d.adhesion = (float)get_f64(env, o, "adhesion", 0.0);
  }
  pf_range* ranges = NULL;
  uint8_t* stat = NULL;
  if (has(env, o, "boundaries")) {
    napi_value arr, e;
    uint32_t n = 0;
    napi_get_named_property(env, o, "boundaries", &arr);
    napi_get_array_length(env, arr, &n);
    ranges = (pf_range*)calloc(n ? n : 1, sizeof *ranges);
    stat = (uint8_t*)calloc(n ? n : 1, 1);
    if (!ranges || !stat) {
      free(ranges);
      free(stat);
      return throw_msg(env, "pfsim: out of host memory");
    }
    for (uint32_t i = 0; i < n; ++i) {
      napi_get_element(env, arr, i, &e);
      ranges[i].start = get_u32(env, e, "start", 0);
      ranges[i].count = get_u32(env, e, "count", 0);
      stat[i] = get_bool(env, e, "dynamic", 1) ? 0 : 1;
    }
    d.n_boundaries = n;
    d.boundaries = ranges;
    d.boundary_static = stat;
  }
  uint32_t mat = 0;
  const pf_status st = pf_add_fluid(b->scene, &d, &mat);
  free(ranges);
  free(stat);
  if (st != PF_OK) return throw_last(env);
  return make_u32(env, mat);
}

/* addSoftbodies(scene, {bodies: [{start, count, surfaceCount, compliance,
 *   restPositions?: Float32Array (xyz), edges?: Uint32Array (pairs)}],
 *   shapeMatching: 'global' | 'local', selfCollision}) -> material index */
static napi_value add_softbodies(napi_env env, napi_callback_info info) {
  ARGS(2);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  napi_value o = argv[1], arr, e, sm;
  uint32_t n = 0;
  if (!has(env, o, "bodies")) return throw_msg(env, "SoftbodySystem: bodies is required");
  napi_get_named_property(env, o, "bodies", &arr);
  napi_get_array_length(env, arr, &n);
  pf_softbody_def* defs = (pf_softbody_def*)calloc(n ? n : 1, sizeof *defs);
  if (!defs) return throw_msg(env, "pfsim: out of host memory");
  for (uint32_t i = 0; i < n; ++i) {
    void *rest, *edges;
    size_t nr, ne;
    napi_get_element(env, arr, i, &e);
    defs[i].range.start = get_u32(env, e, "start", 0);
    defs[i].range.count = get_u32(env, e, "count", 0);
    defs[i].surface_count = get_u32(env, e, "surfaceCount", UINT32_MAX);
    defs[i].compliance = (float)get_f64(env, e, "compliance", 0.0);
    if (!typed_prop(env, e, "restPositions", napi_float32_array, 1, &rest, &nr) ||
        !typed_prop(env, e, "edges", napi_uint32_array, 1, &edges, &ne)) {
      free(defs);
      return NULL;
    }
    if ((rest && nr != 3ull * defs[i].range.count) || ne % 2) {
      free(defs);
      return throw_msg(env, "SoftbodySystem: restPositions or edges have the wrong length");
    }
    defs[i].rest_positions = (const float*)rest;
    defs[i].edges = (const uint32_t*)edges;
    defs[i].n_edges = (uint32_t)(ne / 2);
  }
  pf_softbody_desc d;
  memset(&d, 0, sizeof d);
  d.n_bodies = n;
  d.bodies = defs;
  d.shape_matching = PF_SHAPE_MATCH_GLOBAL;
  if (has(env, o, "shapeMatching")) {
    char mode[16] = {0};
    size_t len = 0;
    napi_get_named_property(env, o, "shapeMatching", &sm);
    napi_get_value_string_utf8(env, sm, mode, sizeof mode, &len);
    d.shape_matching = strcmp(mode, "local") == 0 ? PF_SHAPE_MATCH_LOCAL : PF_SHAPE_MATCH_GLOBAL;
  }
  d.self_collision = (uint32_t)get_bool(env, o, "selfCollision", 0);
  uint32_t mat = 0;
  const pf_status st = pf_add_softbodies(b->scene, &d, &mat);
  free(defs);
  if (st != PF_OK) return throw_last(env);
  return make_u32(env, mat);
}

/* addCloth(scene, {offset, positions: Float32Array (xyz), invMass: Float32Array,
 *   pairs: Uint32Array, restLengths: Float32Array, stretchCompliance,
 *   bending?: Uint32Array (4 per), bendingRest?: Float32Array, bendCompliance,
 *   tetherParticle?, tetherAnchor?: Uint32Array, tetherRest?: Float32Array,
 *   tetherCompliance, triangles?: Uint32Array, wind: [x, y, z], drag, lift,
 *   damping?}) -> material index */
static napi_value add_cloth(napi_env env, napi_callback_info info) {
  ARGS(2);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  napi_value o = argv[1];
  pf_cloth_desc d;
  memset(&d, 0, sizeof d);
  void *pos, *w, *pairs, *rest, *bend = NULL, *bend_rest = NULL, *tp = NULL, *ta = NULL, *tr = NULL, *tri = NULL;
  size_t npos, nw, npairs, nrest, nb = 0, nbr = 0, ntp = 0, nta = 0, ntr = 0, ntri = 0;
  if (!typed_prop(env, o, "positions", napi_float32_array, 0, &pos, &npos) ||
      !typed_prop(env, o, "invMass", napi_float32_array, 0, &w, &nw) ||
      !typed_prop(env, o, "pairs", napi_uint32_array, 0, &pairs, &npairs) ||
      !typed_prop(env, o, "restLengths", napi_float32_array, 0, &rest, &nrest) ||
      !typed_prop(env, o, "bending", napi_uint32_array, 1, &bend, &nb) ||
      !typed_prop(env, o, "bendingRest", napi_float32_array, 1, &bend_rest, &nbr) ||
      !typed_prop(env, o, "tetherParticle", napi_uint32_array, 1, &tp, &ntp) ||
      !typed_prop(env, o, "tetherAnchor", napi_uint32_array, 1, &ta, &nta) ||
      !typed_prop(env, o, "tetherRest", napi_float32_array, 1, &tr, &ntr) ||
      !typed_prop(env, o, "triangles", napi_uint32_array, 1, &tri, &ntri))
    return NULL;
  if (npos % 3 || nw != npos / 3 || npairs % 2 || nrest != npairs / 2 || nb % 4 || nbr != nb / 4 ||
      ntp != nta || ntp != ntr || ntri % 3)
    return throw_msg(env, "ClothSystem: graph arrays have inconsistent lengths");
  d.offset = get_u32(env, o, "offset", 0);
  d.n_particles = (uint32_t)(npos / 3);
  d.positions = (const float*)pos;
  d.inv_mass = (const float*)w;
  d.n_pairs = (uint32_t)(npairs / 2);
  d.pairs = (const uint32_t*)pairs;
  d.rest_lengths = (const float*)rest;
  d.stretch_compliance = (float)get_f64(env, o, "stretchCompliance", -1.0);
  d.n_bending = (uint32_t)(nb / 4);
  d.bending = (const uint32_t*)bend;
  d.bending_rest = (const float*)bend_rest;
  d.bend_compliance = (float)get_f64(env, o, "bendCompliance", -1.0);
  d.n_tethers = (uint32_t)ntp;
  d.tether_particle = (const uint32_t*)tp;
  d.tether_anchor = (const uint32_t*)ta;
  d.tether_rest = (const float*)tr;
  d.tether_compliance = (float)get_f64(env, o, "tetherCompliance", -1.0);
  d.n_triangles = (uint32_t)(ntri / 3);
  d.triangles = (const uint32_t*)tri;
  double wind[3] = {0, 0, 0};
  get_vec(env, o, "wind", 3, wind);
  for (int i = 0; i < 3; ++i) d.wind[i] = (float)wind[i];
  d.drag = (float)get_f64(env, o, "drag", -1.0);
  d.lift = (float)get_f64(env, o, "lift", -1.0);
  d.has_damping = has(env, o, "damping") ? 1u : 0u;
  d.damping = (float)get_f64(env, o, "damping", 0.0);
  uint32_t mat = 0;
  if (pf_add_cloth(b->scene, &d, &mat) != PF_OK) return throw_last(env);
  return make_u32(env, mat);
}

static napi_value cloth_params_obj(napi_env env, const pf_cloth_params* p) {
  napi_value o, wind;
  napi_create_object(env, &o);
  napi_create_array_with_length(env, 3, &wind);
  for (uint32_t i = 0; i < 3; ++i) napi_set_element(env, wind, i, make_f64(env, p->wind[i]));
  napi_set_named_property(env, o, "wind", wind);
  napi_set_named_property(env, o, "drag", make_f64(env, p->drag));
  napi_set_named_property(env, o, "lift", make_f64(env, p->lift));
  napi_set_named_property(env, o, "damping", make_f64(env, p->damping));
  napi_set_named_property(env, o, "bendCompliance", make_f64(env, p->bend_compliance));
  return o;
}

/* clothGetParams(scene, material) -> {wind, drag, lift, damping, bendCompliance} */
static napi_value cloth_get_params(napi_env env, napi_callback_info info) {
  ARGS(2);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  uint32_t mat;
  pf_cloth_params p;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &mat));
  if (pf_cloth_get_params(b->scene, mat, &p) != PF_OK) return throw_last(env);
  return cloth_params_obj(env, &p);
}

/* clothSetParams(scene, material, {wind, drag, lift, damping, bendCompliance})
 * (fields left out keep their values) */
static napi_value cloth_set_params(napi_env env, napi_callback_info info) {
  ARGS(3);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  uint32_t mat;
  pf_cloth_params p;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &mat));
  if (pf_cloth_get_params(b->scene, mat, &p) != PF_OK) return throw_last(env);
  double wind[3] = {p.wind[0], p.wind[1], p.wind[2]};
  get_vec(env, argv[2], "wind", 3, wind);
  for (int i = 0; i < 3; ++i) p.wind[i] = (float)wind[i];
  p.drag = (float)get_f64(env, argv[2], "drag", p.drag);
  p.lift = (float)get_f64(env, argv[2], "lift", p.lift);
  p.damping = (float)get_f64(env, argv[2], "damping", p.damping);
  p.bend_compliance = (float)get_f64(env, argv[2], "bendCompliance", p.bend_compliance);
  if (pf_cloth_set_params(b->scene, mat, &p) != PF_OK) return throw_last(env);
  return undefined(env);
}

/* buildTethers({invMass: Float32Array, pairs: Uint32Array, restLengths:
 *   Float64Array, maxAttachments, stretchTolerance}) -> {particle, anchor, rest} */
static napi_value build_tethers(napi_env env, napi_callback_info info) {
  ARGS(1);
  napi_value o = argv[0];
  void *w, *pairs, *rest;
  size_t nw, np, nr;
  if (!typed_prop(env, o, "invMass", napi_float32_array, 0, &w, &nw) ||
      !typed_prop(env, o, "pairs", napi_uint32_array, 0, &pairs, &np) ||
      !typed_prop(env, o, "restLengths", napi_float64_array, 0, &rest, &nr))
    return NULL;
  if (np % 2 || nr != np / 2) return throw_msg(env, "buildTethers: pairs and restLengths disagree");
  pf_tether_build_desc d;
  memset(&d, 0, sizeof d);
  d.n_particles = (uint32_t)nw;
  d.inv_mass = (const float*)w;
  d.n_pairs = (uint32_t)(np / 2);
  d.pairs = (const uint32_t*)pairs;
  d.rest_lengths = (const double*)rest;
  d.max_attachments = get_u32(env, o, "maxAttachments", 0);
  d.stretch_tolerance = get_f64(env, o, "stretchTolerance", 0.0);
  const uint32_t k = d.max_attachments ? d.max_attachments : 4;
  const size_t cap = (size_t)d.n_particles * k;
  napi_value ab_p, ab_a, ab_r, tp, ta, tr, out;
  void *pp, *pa, *pr;
  CHECK_NAPI(napi_create_arraybuffer(env, 4 * (cap ? cap : 1), &pp, &ab_p));
  CHECK_NAPI(napi_create_arraybuffer(env, 4 * (cap ? cap : 1), &pa, &ab_a));
  CHECK_NAPI(napi_create_arraybuffer(env, 4 * (cap ? cap : 1), &pr, &ab_r));
  uint32_t count = 0;
  if (pf_cloth_build_tethers(&d, (uint32_t*)pp, (uint32_t*)pa, (float*)pr, (uint32_t)cap, &count) != PF_OK)
    return throw_last(env);
  CHECK_NAPI(napi_create_typedarray(env, napi_uint32_array, count, ab_p, 0, &tp));
  CHECK_NAPI(napi_create_typedarray(env, napi_uint32_array, count, ab_a, 0, &ta));
  CHECK_NAPI(napi_create_typedarray(env, napi_float32_array, count, ab_r, 0, &tr));
  napi_create_object(env, &out);
  napi_set_named_property(env, out, "particle", tp);
  napi_set_named_property(env, out, "anchor", ta);
  napi_set_named_property(env, out, "rest", tr);
  return out;
}

/* --------------------------------------------------------- colliders --- */

/* {kind: 'plane'|'sphere'|'box'|'capsule', invert, sweep, data0: [4], data1: [4],
 *  velocity: [4], rotation: [4], spin: [3]} -> pf_primitive (primitives.ts record) */
static int primitive_of(napi_env env, napi_value o, pf_primitive* p) {
  char kind[16] = {0};
  size_t len = 0;
  napi_value k;
  double v[4];
  memset(p, 0, sizeof *p);
  p->rotation[3] = 1.0f;
  if (!has(env, o, "kind")) return 0;
  napi_get_named_property(env, o, "kind", &k);
  napi_get_value_string_utf8(env, k, kind, sizeof kind, &len);
  if (!strcmp(kind, "plane")) p->kind = PF_PRIM_PLANE;
  else if (!strcmp(kind, "sphere")) p->kind = PF_PRIM_SPHERE;
  else if (!strcmp(kind, "box")) p->kind = PF_PRIM_BOX;
  else if (!strcmp(kind, "capsule")) p->kind = PF_PRIM_CAPSULE;
  else return 0;
  p->flags = (get_bool(env, o, "invert", 0) ? PF_PRIM_INVERT : 0u) | (get_bool(env, o, "sweep", 0) ? PF_PRIM_SWEEP : 0u);
#define VEC4(field)                                          \
  if (get_vec(env, o, #field, 4, v))                         \
    for (int i = 0; i < 4; ++i) p->field[i] = (float)v[i];
  VEC4(data0)
  VEC4(data1)
  VEC4(velocity)
  VEC4(rotation)
#undef VEC4
  if (get_vec(env, o, "spin", 3, v))
    for (int i = 0; i < 3; ++i) p->spin[i] = (float)v[i];
  return 1;
}

/* addPrimitive(scene, prim) -> slot */
static napi_value add_primitive(napi_env env, napi_callback_info info) {
  ARGS(2);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  pf_primitive p;
  if (!primitive_of(env, argv[1], &p)) return throw_msg(env, "PrimitiveSet: unknown primitive kind");
  uint32_t slot = 0;
  if (pf_add_primitive(b->scene, &p, &slot) != PF_OK) return throw_last(env);
  return make_u32(env, slot);
}

/* setPrimitive(scene, slot, prim) (PrimitiveSet.setSphere / attach) */
static napi_value set_primitive(napi_env env, napi_callback_info info) {
  ARGS(3);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  uint32_t slot;
  pf_primitive p;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &slot));
  if (!primitive_of(env, argv[2], &p)) return throw_msg(env, "PrimitiveSet: unknown primitive kind");
  if (pf_set_primitive(b->scene, slot, &p) != PF_OK) return throw_last(env);
  return undefined(env);
}

/* addSdfCollider(scene, {res: [3], data: Float32Array, origin: [3], voxelSize: [3],
 *   position: [3], rotation: [4], scale, thickness, muS, muK}) -> slot */
static napi_value add_sdf_collider(napi_env env, napi_callback_info info) {
  ARGS(2);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  napi_value o = argv[1];
  pf_sdf_desc d;
  memset(&d, 0, sizeof d);
  double v[4];
  void* data;
  size_t n;
  if (!typed_prop(env, o, "data", napi_float32_array, 0, &data, &n)) return NULL;
  if (!get_vec(env, o, "res", 3, v)) return throw_msg(env, "SDFCollider: res is required");
  for (int i = 0; i < 3; ++i) d.res[i] = (uint32_t)v[i];
  if ((size_t)d.res[0] * d.res[1] * d.res[2] != n) return throw_msg(env, "SDFCollider: data length differs from res");
  d.data = (const float*)data;
  if (get_vec(env, o, "origin", 3, v))
    for (int i = 0; i < 3; ++i) d.origin[i] = (float)v[i];
  if (get_vec(env, o, "voxelSize", 3, v))
    for (int i = 0; i < 3; ++i) d.voxel_size[i] = (float)v[i];
  if (get_vec(env, o, "position", 3, v))
    for (int i = 0; i < 3; ++i) d.position[i] = (float)v[i];
  d.rotation[3] = 1.0f;
  if (get_vec(env, o, "rotation", 4, v))
    for (int i = 0; i < 4; ++i) d.rotation[i] = (float)v[i];
  d.scale = (float)get_f64(env, o, "scale", 1.0);
  d.thickness = (float)get_f64(env, o, "thickness", 0.0);
  d.mu_s = (float)get_f64(env, o, "muS", 0.5);
  d.mu_k = (float)get_f64(env, o, "muK", 0.3);
  uint32_t slot = 0;
  if (pf_add_sdf_collider(b->scene, &d, &slot) != PF_OK) return throw_last(env);
  return make_u32(env, slot);
}

/* setSdfTransform(scene, slot, position: [3], rotation: [4], scale) */
static napi_value set_sdf_transform(napi_env env, napi_callback_info info) {
  ARGS(5);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  uint32_t slot;
  double scale, p[3], q[4];
  napi_value e;
  float pf[3], qf[4];
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &slot));
  for (uint32_t i = 0; i < 3; ++i) {
    CHECK_NAPI(napi_get_element(env, argv[2], i, &e));
    CHECK_NAPI(napi_get_value_double(env, e, &p[i]));
    pf[i] = (float)p[i];
  }
  for (uint32_t i = 0; i < 4; ++i) {
    CHECK_NAPI(napi_get_element(env, argv[3], i, &e));
    CHECK_NAPI(napi_get_value_double(env, e, &q[i]));
    qf[i] = (float)q[i];
  }
  CHECK_NAPI(napi_get_value_double(env, argv[4], &scale));
  if (pf_set_sdf_transform(b->scene, slot, pf, qf, (float)scale) != PF_OK) return throw_last(env);
  return undefined(env);
}

/* addNoSelfContacts(scene, start, count) */
static napi_value add_no_self_contacts(napi_env env, napi_callback_info info) {
  ARGS(3);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  pf_range r;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &r.start));
  CHECK_NAPI(napi_get_value_uint32(env, argv[2], &r.count));
  if (pf_add_no_self_contacts(b->scene, r) != PF_OK) return throw_last(env);
  return undefined(env);
}

/* -------------------------------------------------------------- loop --- */

/* buildLoop(scene, {substeps, iterations, gravity: [3], hashOrigin: [3],
 *   gridMin?: [3], gridMax?: [3], contact?: {muS, muK, maxContacts}}) */
static napi_value build_loop(napi_env env, napi_callback_info info) {
  ARGS(2);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  napi_value o = argv[1];
  pf_loop_desc d;
  double v[3];
  memset(&d, 0, sizeof d);
  d.substeps = get_u32(env, o, "substeps", 4);
  d.iterations = get_u32(env, o, "iterations", 2);
  d.gravity[1] = -9.81f;
  if (get_vec(env, o, "gravity", 3, v))
    for (int i = 0; i < 3; ++i) d.gravity[i] = (float)v[i];
  if (get_vec(env, o, "hashOrigin", 3, v))
    for (int i = 0; i < 3; ++i) d.hash_origin[i] = (float)v[i];
  if (get_vec(env, o, "gridMin", 3, v))
    for (int i = 0; i < 3; ++i) d.grid_min[i] = (float)v[i];
  if (get_vec(env, o, "gridMax", 3, v))
    for (int i = 0; i < 3; ++i) d.grid_max[i] = (float)v[i];
  d.contact_mu_s = -1.0f;
  d.contact_mu_k = -1.0f;
  if (has(env, o, "contact")) {
    napi_value c;
    napi_valuetype t;
    napi_get_named_property(env, o, "contact", &c);
    napi_typeof(env, c, &t);
    d.contact = t == napi_object ? 1u : (uint32_t)get_bool(env, o, "contact", 0);
    if (t == napi_object) {
      d.contact_mu_s = (float)get_f64(env, c, "muS", -1.0);
      d.contact_mu_k = (float)get_f64(env, c, "muK", -1.0);
      d.max_contacts = get_u32(env, c, "maxContacts", 0);
    }
  }
  if (pf_loop_build(b->scene, &d) != PF_OK) return throw_last(env);
  return undefined(env);
}

/* step(scene, dt) -> Promise<void>: pf_step, then a wait for the step's end
 * event, on the thread pool. The scene is marked busy until it settles, so
 * no other call reaches the handle meanwhile (calls on one handle are not
 * re-entrant). */
typedef struct {
  SceneBox* box;
  napi_ref keep; /* the scene's External stays alive while the step runs */
  double dt;
  pf_status st;
  char err[512];
  napi_deferred deferred;
  napi_async_work work;
} StepJob;

static void step_exec(napi_env env, void* data) {
  StepJob* j = (StepJob*)data;
  float ms = 0.0f;
  (void)env;
  j->st = pf_step(j->box->scene, j->dt);
  if (j->st == PF_OK) j->st = pf_last_step_ms(j->box->scene, &ms);
  if (j->st != PF_OK) strncpy(j->err, pf_last_error(), sizeof j->err - 1);
}

static void step_done(napi_env env, napi_status status, void* data) {
  StepJob* j = (StepJob*)data;
  napi_value v;
  j->box->busy = 0;
  if (status == napi_ok && j->st == PF_OK) {
    napi_get_undefined(env, &v);
    napi_resolve_deferred(env, j->deferred, v);
  } else {
    napi_value msg;
    napi_create_string_utf8(env, j->err[0] ? j->err : "SimLoop: step cancelled", NAPI_AUTO_LENGTH, &msg);
    napi_create_error(env, NULL, msg, &v);
    napi_reject_deferred(env, j->deferred, v);
  }
  napi_delete_reference(env, j->keep);
  napi_delete_async_work(env, j->work);
  free(j);
}

static napi_value step(napi_env env, napi_callback_info info) {
  ARGS(2);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  napi_value promise, name;
  StepJob* j = (StepJob*)calloc(1, sizeof *j);
  if (!j) return throw_msg(env, "pfsim: out of host memory");
  j->box = b;
  CHECK_NAPI(napi_get_value_double(env, argv[1], &j->dt));
  CHECK_NAPI(napi_create_promise(env, &j->deferred, &promise));
  CHECK_NAPI(napi_create_string_utf8(env, "pf_step", NAPI_AUTO_LENGTH, &name));
  CHECK_NAPI(napi_create_async_work(env, NULL, name, step_exec, step_done, j, &j->work));
  CHECK_NAPI(napi_create_reference(env, argv[0], 1, &j->keep));
  b->busy = 1;
  if (napi_queue_async_work(env, j->work) != napi_ok) {
    b->busy = 0;
    napi_delete_reference(env, j->keep);
    napi_delete_async_work(env, j->work);
    free(j);
    return throw_msg(env, "SimLoop: could not queue the step");
  }
  return promise;
}

/* readback(scene, field, out: TypedArray): the field into `out`, whose byte
 * length must be the field's (pfsim.h pf_field). Synchronous. */
static napi_value readback(napi_env env, napi_callback_info info) {
  ARGS(3);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  uint32_t field;
  napi_typedarray_type ty;
  size_t len;
  void* dst;
  bool is_typed = false;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &field));
  napi_is_typedarray(env, argv[2], &is_typed);
  if (!is_typed) return throw_msg(env, "ParticleSystem.readback: expected a typed array");
  CHECK_NAPI(napi_get_typedarray_info(env, argv[2], &ty, &len, &dst, NULL, NULL));
  if (pf_readback(b->scene, field, dst, len * elem_bytes(ty)) != PF_OK) return throw_last(env);
  return undefined(env);
}

/* write(scene, field, src: TypedArray): whole-field write in particle order. */
static napi_value write_field(napi_env env, napi_callback_info info) {
  ARGS(3);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  uint32_t field;
  napi_typedarray_type ty;
  size_t len;
  void* src;
  bool is_typed = false;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &field));
  napi_is_typedarray(env, argv[2], &is_typed);
  if (!is_typed) return throw_msg(env, "ParticleSystem: expected a typed array");
  CHECK_NAPI(napi_get_typedarray_info(env, argv[2], &ty, &len, &src, NULL, NULL));
  if (ty != napi_float32_array) return throw_msg(env, "ParticleSystem: state fields are Float32Array");
  if (pf_write(b->scene, field, src, len * 4) != PF_OK) return throw_last(env);
  return undefined(env);
}

/* readbackOverflow(scene) -> SimLoopOverflow (loop.ts:59-69) */
static napi_value readback_overflow(napi_env env, napi_callback_info info) {
  ARGS(1);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  pf_overflow o;
  napi_value out, t;
  if (pf_overflow_read(b->scene, &o) != PF_OK) return throw_last(env);
  napi_create_object(env, &out);
#define FLAG(js, c)                    \
  napi_get_boolean(env, o.c != 0, &t); \
  napi_set_named_property(env, out, js, t);
  FLAG("positions", positions)
  FLAG("velocities", velocities)
  FLAG("grid", grid)
  FLAG("contacts", contacts)
  FLAG("neighbors", neighbors)
  FLAG("deviceError", device_error)
  FLAG("gridClamped", grid_clamped)
#undef FLAG
  return out;
}

/* contacts(scene, capacity) -> {count, pairs: Uint32Array (2 per pair)} */
static napi_value contacts(napi_env env, napi_callback_info info) {
  ARGS(2);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  uint32_t cap, count = 0, stored = 0;
  void* data;
  napi_value ab, arr, out;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &cap));
  CHECK_NAPI(napi_create_arraybuffer(env, 8ull * (cap ? cap : 1), &data, &ab));
  if (pf_contacts_read(b->scene, (uint32_t*)data, cap, &count, &stored) != PF_OK) return throw_last(env);
  CHECK_NAPI(napi_create_typedarray(env, napi_uint32_array, 2ull * stored, ab, 0, &arr));
  napi_create_object(env, &out);
  napi_set_named_property(env, out, "count", make_u32(env, count));
  napi_set_named_property(env, out, "pairs", arr);
  return out;
}

/* lastStepMs(scene) -> device milliseconds of the last step */
static napi_value last_step_ms(napi_env env, napi_callback_info info) {
  ARGS(1);
  SceneBox* b = scene_of(env, argv[0]);
  if (!b) return NULL;
  float ms = 0.0f;
  if (pf_last_step_ms(b->scene, &ms) != PF_OK) return throw_last(env);
  return make_f64(env, ms);
}

/* ---------------------------------------------------------- hash grid --- */

/* sortHost(pos4: Float32Array, {cellSize, hashOrigin, hashTableSize} or
 *   {cellSize, hashOrigin, dims}) -> {cellIndex, counts, cellStart,
 *   sortedIndices, overflow} (HashGrid.rebuild + readback) */
static napi_value sort_host(napi_env env, napi_callback_info info) {
  ARGS(2);
  void* pos;
  size_t n4;
  if (!typed(env, argv[0], napi_float32_array, 0, &pos, &n4)) return NULL;
  if (n4 % 4) return throw_msg(env, "HashGrid: positions need 4 floats each");
  const uint32_t n = (uint32_t)(n4 / 4);
  napi_value o = argv[1];
  pf_grid_desc g;
  double v[3];
  memset(&g, 0, sizeof g);
  g.cell_size = (float)get_f64(env, o, "cellSize", 0.0);
  if (get_vec(env, o, "hashOrigin", 3, v))
    for (int i = 0; i < 3; ++i) g.origin[i] = (float)v[i];
  if (get_vec(env, o, "dims", 3, v)) {
    g.key_kind = PF_KEY_LINEAR;
    for (int i = 0; i < 3; ++i) g.dims[i] = (uint32_t)v[i];
  } else {
    uint32_t size = get_u32(env, o, "hashTableSize", 0);
    if (!size) { /* HashGrid.ts:122-124 */
      size = 1;
      while (size < 2ull * (n ? n : 1)) size <<= 1;
    }
    g.key_kind = PF_KEY_MORTON;
    g.table_size = size;
  }
  const uint64_t cells = pf_grid_cells(&g);
  if (!cells) return throw_msg(env, "HashGrid: invalid grid options");
  void *keys, *count, *start, *perm;
  napi_value ab_k, ab_c, ab_s, ab_p, tk, tc, ts, tp, out, ovf;
  CHECK_NAPI(napi_create_arraybuffer(env, 4ull * (n ? n : 1), &keys, &ab_k));
  CHECK_NAPI(napi_create_arraybuffer(env, 4ull * cells, &count, &ab_c));
  CHECK_NAPI(napi_create_arraybuffer(env, 4ull * cells, &start, &ab_s));
  CHECK_NAPI(napi_create_arraybuffer(env, 4ull * (n ? n : 1), &perm, &ab_p));
  uint32_t overflow = 0;
  if (pf_sort_host((const float*)pos, n, &g, (uint32_t*)perm, (uint32_t*)start, (uint32_t*)count, (uint32_t*)keys,
                   &overflow) != PF_OK)
    return throw_last(env);
  CHECK_NAPI(napi_create_typedarray(env, napi_uint32_array, n, ab_k, 0, &tk));
  CHECK_NAPI(napi_create_typedarray(env, napi_uint32_array, cells, ab_c, 0, &tc));
  CHECK_NAPI(napi_create_typedarray(env, napi_uint32_array, cells, ab_s, 0, &ts));
  CHECK_NAPI(napi_create_typedarray(env, napi_uint32_array, n, ab_p, 0, &tp));
  napi_create_object(env, &out);
  napi_set_named_property(env, out, "cellIndex", tk);
  napi_set_named_property(env, out, "counts", tc);
  napi_set_named_property(env, out, "cellStart", ts);
  napi_set_named_property(env, out, "sortedIndices", tp);
  napi_get_boolean(env, overflow != 0, &ovf);
  napi_set_named_property(env, out, "overflow", ovf);
  return out;
}

/* ------------------------------------------------------- mesh set-up --- */

static int mesh_of(napi_env env, napi_value o, pf_mesh* m) {
  void *v, *i;
  size_t nv, ni;
  if (!typed_prop(env, o, "vertices", napi_float32_array, 0, &v, &nv) ||
      !typed_prop(env, o, "indices", napi_uint32_array, 0, &i, &ni))
    return 0;
  if (nv % 3 || ni % 3) {
    napi_throw_error(env, NULL, "pfsim: mesh arrays need 3 entries per vertex and per triangle");
    return 0;
  }
  m->vertices = (const float*)v;
  m->n_vertices = (uint32_t)(nv / 3);
  m->indices = (const uint32_t*)i;
  m->n_indices = (uint32_t)ni;
  return 1;
}

/* voxelizeMesh({vertices, indices}, particleRadius, largestPiece) ->
 *   {positions: Float32Array (xyz), surfaceCount, edges: Uint32Array} */
static napi_value voxelize_mesh(napi_env env, napi_callback_info info) {
  ARGS(3);
  pf_mesh m;
  double r;
  bool largest = false;
  if (!mesh_of(env, argv[0], &m)) return NULL;
  CHECK_NAPI(napi_get_value_double(env, argv[1], &r));
  napi_get_value_bool(env, argv[2], &largest);
  pf_voxels out;
  memset(&out, 0, sizeof out);
  if (pf_voxelize_mesh(&m, r, largest ? 1u : 0u, &out) != PF_OK) return throw_last(env); /* sizes */
  void *pos, *edges;
  napi_value ab_p, ab_e, tp, te, res;
  CHECK_NAPI(napi_create_arraybuffer(env, 12ull * (out.count ? out.count : 1), &pos, &ab_p));
  CHECK_NAPI(napi_create_arraybuffer(env, 8ull * (out.edge_count ? out.edge_count : 1), &edges, &ab_e));
  out.positions = (float*)pos;
  out.capacity = out.count;
  out.edges = (uint32_t*)edges;
  out.edge_capacity = out.edge_count;
  if (pf_voxelize_mesh(&m, r, largest ? 1u : 0u, &out) != PF_OK) return throw_last(env);
  CHECK_NAPI(napi_create_typedarray(env, napi_float32_array, 3ull * out.count, ab_p, 0, &tp));
  CHECK_NAPI(napi_create_typedarray(env, napi_uint32_array, 2ull * out.edge_count, ab_e, 0, &te));
  napi_create_object(env, &res);
  napi_set_named_property(env, res, "positions", tp);
  napi_set_named_property(env, res, "surfaceCount", make_u32(env, out.surface_count));
  napi_set_named_property(env, res, "edges", te);
  return res;
}

/* bakeSdf({vertices, indices}, resolution, padding) -> {data, origin, voxelSize, inconsistent} */
static napi_value bake_sdf(napi_env env, napi_callback_info info) {
  ARGS(3);
  pf_mesh m;
  uint32_t res;
  double padding, origin[3], voxel = 0;
  uint64_t bad = 0;
  if (!mesh_of(env, argv[0], &m)) return NULL;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &res));
  CHECK_NAPI(napi_get_value_double(env, argv[2], &padding));
  const uint64_t n = (uint64_t)res * res * res;
  void* data;
  napi_value ab, td, out, org;
  CHECK_NAPI(napi_create_arraybuffer(env, 4ull * (n ? n : 1), &data, &ab));
  if (pf_bake_sdf(&m, res, padding, (float*)data, origin, &voxel, &bad) != PF_OK) return throw_last(env);
  CHECK_NAPI(napi_create_typedarray(env, napi_float32_array, n, ab, 0, &td));
  napi_create_array_with_length(env, 3, &org);
  for (uint32_t i = 0; i < 3; ++i) napi_set_element(env, org, i, make_f64(env, origin[i]));
  napi_create_object(env, &out);
  napi_set_named_property(env, out, "data", td);
  napi_set_named_property(env, out, "origin", org);
  napi_set_named_property(env, out, "voxelSize", make_f64(env, voxel));
  napi_set_named_property(env, out, "inconsistent", make_f64(env, (double)bad));
  return out;
}

static napi_value abi_version(napi_env env, napi_callback_info info) {
  (void)info;
  napi_value v;
  napi_create_int32(env, pf_abi_version(), &v);
  return v;
}

/* trimDeviceMemory(): hand the device memory the library's pool keeps from
 * destroyed worlds back to the device. */
static napi_value trim_device_memory(napi_env env, napi_callback_info info) {
  (void)info;
  if (pf_trim_device_memory() != PF_OK) return throw_last(env);
  return undefined(env);
}

/* ------------------------------------------------------------ module --- */

NAPI_MODULE_INIT() {
  napi_property_descriptor p[] = {
      {"abiVersion", 0, abi_version, 0, 0, 0, napi_default, 0},
      {"trimDeviceMemory", 0, trim_device_memory, 0, 0, 0, napi_default, 0},
      {"createScene", 0, create_scene, 0, 0, 0, napi_default, 0},
      {"destroyScene", 0, destroy_scene, 0, 0, 0, napi_default, 0},
      {"uploadParticles", 0, upload, 0, 0, 0, napi_default, 0},
      {"setInvMass", 0, set_inv_mass, 0, 0, 0, napi_default, 0},
      {"addFluid", 0, add_fluid, 0, 0, 0, napi_default, 0},
      {"addSoftbodies", 0, add_softbodies, 0, 0, 0, napi_default, 0},
      {"addCloth", 0, add_cloth, 0, 0, 0, napi_default, 0},
      {"clothGetParams", 0, cloth_get_params, 0, 0, 0, napi_default, 0},
      {"clothSetParams", 0, cloth_set_params, 0, 0, 0, napi_default, 0},
      {"buildTethers", 0, build_tethers, 0, 0, 0, napi_default, 0},
      {"addPrimitive", 0, add_primitive, 0, 0, 0, napi_default, 0},
      {"setPrimitive", 0, set_primitive, 0, 0, 0, napi_default, 0},
      {"addSdfCollider", 0, add_sdf_collider, 0, 0, 0, napi_default, 0},
      {"setSdfTransform", 0, set_sdf_transform, 0, 0, 0, napi_default, 0},
      {"addNoSelfContacts", 0, add_no_self_contacts, 0, 0, 0, napi_default, 0},
      {"buildLoop", 0, build_loop, 0, 0, 0, napi_default, 0},
      {"step", 0, step, 0, 0, 0, napi_default, 0},
      {"readback", 0, readback, 0, 0, 0, napi_default, 0},
      {"write", 0, write_field, 0, 0, 0, napi_default, 0},
      {"readbackOverflow", 0, readback_overflow, 0, 0, 0, napi_default, 0},
      {"contacts", 0, contacts, 0, 0, 0, napi_default, 0},
      {"lastStepMs", 0, last_step_ms, 0, 0, 0, napi_default, 0},
      {"sortHost", 0, sort_host, 0, 0, 0, napi_default, 0},
      {"voxelizeMesh", 0, voxelize_mesh, 0, 0, 0, napi_default, 0},
      {"bakeSdf", 0, bake_sdf, 0, 0, 0, napi_default, 0},
  };
  napi_define_properties(env, exports, sizeof p / sizeof p[0], p);
  return exports;
}
