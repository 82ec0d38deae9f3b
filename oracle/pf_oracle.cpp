// pf_oracle.cpp — CPU restatement of the threejs-particle-fluids solver path.
//
// TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA path in
// libpfsim.so: only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg may load it. The product never calls it.
//
// It restates, in plain C++, the TSL kernels the reference compiles to WGSL,
// in the reference's own stage order and FP32 operation order, on particle
// state kept in particle-index order exactly as the reference keeps it:
//   - neighbour grid: Morton bucket key + histogram (src/core/hashGrid/
//     cellIndex.ts:113-170, mortonHash.ts:39-79), exclusive scan + scatter
//     (sort.ts:72-192) made stable (ascending particle index within a cell),
//     27-cell walk (query.ts:24-70), neighbour list (neighborList.ts:14-90);
//   - integration (src/core/integrate.ts:25-44), fixed-point accumulator
//     (src/core/accumulator.ts:88-178), SPH kernels (src/core/sph/kernels.ts);
//   - PBF fluid (src/fluids/sim/lambda.ts, positionDelta.ts, velocity.ts,
//     shared.ts, boundaryVolume.ts; FluidSystem.ts:200-309);
//   - primitive colliders (src/core/collision/primitives.ts, collider.ts,
//     PrimitiveSet.ts:314-416);
//   - shape matching (src/softbody/polarDecomp.ts, shapeMatch.ts,
//     shapeMatchImplicit.ts, rotation.ts, SoftbodySystem.ts);
//   - XPBD distance constraints with greedy colouring (src/core/constraints/
//     xpbd.ts, types.ts:95-185, distance.ts:212-295);
//   - the SimLoop stage order (src/core/loop.ts:175-242, 318-323).
// The engine is templated on the scalar type: Engine<float> is the FP32
// oracle, Engine<double> the FP64 re-run of the same step. Uniforms that the
// reference computes in JavaScript doubles are computed in double and then
// stored at the engine's precision, as the reference stores them in f32
// uniforms.
//
// WGSL semantics restated: round() is ties-to-even (std::nearbyint in the
// default rounding mode); f32 -> i32 conversion saturates and maps NaN to 0;
// division and sqrt are IEEE. Build with -ffp-contract=off so that no
// multiply-add is fused.

#include <algorithm>
#include <cfenv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <thread>

#include "pfsim.h"

namespace {

thread_local std::string g_err;

pf_status fail(pf_status s, const std::string& msg) {
  g_err = msg;
  return s;
}

// Threads used by parallel_for (set by or_set_threads; 1 = serial).
int g_threads = 1;

// Static block partition of [lo, hi) over g_threads std::threads. Every loop
// given to it writes only its own index's outputs (or adds to integer
// accumulators atomically), so the result does not depend on the split.
template <typename F>
void parallel_for(int64_t lo, int64_t hi, F&& fn) {
  const int64_t n = hi - lo;
  const int t = g_threads;
  if (t <= 1 || n < 256) {
    for (int64_t i = lo; i < hi; ++i) fn(i);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(t);
  for (int k = 0; k < t; ++k) {
    const int64_t a = lo + n * k / t, b = lo + n * (k + 1) / t;
    pool.emplace_back([a, b, &fn] {
      for (int64_t i = a; i < b; ++i) fn(i);
    });
  }
  for (auto& th : pool) th.join();
}

// ---------------------------------------------------------------- math ----

template <typename T>
struct V3 {
  T x, y, z;
};
template <typename T>
inline V3<T> v3(T x, T y, T z) {
  return {x, y, z};
}
template <typename T>
inline V3<T> operator+(V3<T> a, V3<T> b) {
  return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <typename T>
inline V3<T> operator-(V3<T> a, V3<T> b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <typename T>
inline V3<T> operator*(V3<T> a, T s) {
  return {a.x * s, a.y * s, a.z * s};
}
template <typename T>
inline V3<T> operator/(V3<T> a, T s) {
  return {a.x / s, a.y / s, a.z / s};
}
template <typename T>
inline V3<T> neg(V3<T> a) {
  return {-a.x, -a.y, -a.z};
}
template <typename T>
inline T dot(V3<T> a, V3<T> b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename T>
inline V3<T> cross(V3<T> a, V3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename T>
inline T length(V3<T> a) {
  return std::sqrt(dot(a, a));
}
template <typename T>
inline T tmax(T a, T b) {
  return a > b ? a : b;  // WGSL max for non-NaN inputs
}
template <typename T>
inline T tmin(T a, T b) {
  return a < b ? a : b;
}

struct Q4 {
  double x, y, z, w;
};

// WGSL i32(f32): truncation toward zero, saturating, NaN -> 0.
inline int32_t sat_i32(double v) {
  if (std::isnan(v)) return 0;
  if (v >= 2147483647.0) return 2147483647;
  if (v <= -2147483648.0) return INT32_MIN;
  return static_cast<int32_t>(v);
}

// ------------------------------------------------------------ grid keys ----

constexpr int32_t kMortonBias = 512;          // mortonHash.ts:25
constexpr int32_t kCellCoordMax = 1 << 30;    // cellIndex.ts:114

// mortonHash.ts:39-50
inline uint32_t part1by2(uint32_t n) {
  uint32_t m = n & 0x000003ffu;
  m = (m | (m << 16)) & 0xff0000ffu;
  m = (m | (m << 8)) & 0x0300f00fu;
  m = (m | (m << 4)) & 0x030c30c3u;
  m = (m | (m << 2)) & 0x09249249u;
  return m;
}

// mortonHash.ts:71-79. The bias is added in i32 and reinterpreted as u32.
inline uint32_t morton_unmasked(int32_t cx, int32_t cy, int32_t cz) {
  uint32_t ux = static_cast<uint32_t>(static_cast<uint32_t>(cx) + static_cast<uint32_t>(kMortonBias));
  uint32_t uy = static_cast<uint32_t>(static_cast<uint32_t>(cy) + static_cast<uint32_t>(kMortonBias));
  uint32_t uz = static_cast<uint32_t>(static_cast<uint32_t>(cz) + static_cast<uint32_t>(kMortonBias));
  return part1by2(ux) | (part1by2(uy) << 1) | (part1by2(uz) << 2);
}

uint64_t grid_cells(const pf_grid_desc& g) {
  if (g.key_kind == PF_KEY_LINEAR) {
    if (!g.dims[0] || !g.dims[1] || !g.dims[2]) return 0;
    return static_cast<uint64_t>(g.dims[0]) * g.dims[1] * g.dims[2];
  }
  if (g.key_kind == PF_KEY_MORTON) {
    if (!g.table_size || (g.table_size & (g.table_size - 1))) return 0;
    return g.table_size;
  }
  return 0;
}

// One particle's key (cellIndex.ts:192-248 for Morton; the linear grid of the
// standalone sort clamps each axis into [0, dims-1]). Returns the overflow
// flag through `over`.
template <typename T>
uint32_t cell_key(const pf_grid_desc& g, T px, T py, T pz, uint32_t* over) {
  const T ox = static_cast<T>(g.origin[0]), oy = static_cast<T>(g.origin[1]),
          oz = static_cast<T>(g.origin[2]);
  const T cs = static_cast<T>(g.cell_size);
  const T rx = std::floor((px - ox) / cs), ry = std::floor((py - oy) / cs),
          rz = std::floor((pz - oz) / cs);
  int32_t cxr = sat_i32(rx), cyr = sat_i32(ry), czr = sat_i32(rz);
  if (g.key_kind == PF_KEY_LINEAR) {
    int32_t cx = std::min(std::max(cxr, 0), static_cast<int32_t>(g.dims[0]) - 1);
    int32_t cy = std::min(std::max(cyr, 0), static_cast<int32_t>(g.dims[1]) - 1);
    int32_t cz = std::min(std::max(czr, 0), static_cast<int32_t>(g.dims[2]) - 1);
    *over = (cx != cxr || cy != cyr || cz != czr) ? 1u : 0u;
    return static_cast<uint32_t>(cx) + g.dims[0] * (static_cast<uint32_t>(cy) + g.dims[1] * static_cast<uint32_t>(cz));
  }
  const int32_t lo = -kCellCoordMax, hi = kCellCoordMax - 1;
  int32_t cx = std::min(std::max(cxr, lo), hi);
  int32_t cy = std::min(std::max(cyr, lo), hi);
  int32_t cz = std::min(std::max(czr, lo), hi);
  bool o = cxr != cx || cyr != cy || czr != cz;
  o = o || cx < -kMortonBias || cx >= kMortonBias;
  o = o || cy < -kMortonBias || cy >= kMortonBias;
  o = o || cz < -kMortonBias || cz >= kMortonBias;
  *over = o ? 1u : 0u;
  return morton_unmasked(cx, cy, cz) & (g.table_size - 1u);
}

// sort.ts:55-195 made stable: histogram, exclusive scan, and a scatter that
// visits particles in ascending index so each cell keeps index order.
template <typename T>
void stable_count_sort(const pf_grid_desc& g, uint32_t n, const T* pos4, uint32_t* keys,
                       uint32_t* perm, uint32_t* start, uint32_t* count, uint32_t* overflow) {
  const uint64_t C = grid_cells(g);
  std::fill(count, count + C, 0u);
  uint32_t over_any = 0;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t over = 0;
    uint32_t k = cell_key<T>(g, pos4[4 * i], pos4[4 * i + 1], pos4[4 * i + 2], &over);
    keys[i] = k;
    count[k] += 1;
    over_any |= over;
  }
  uint32_t acc = 0;
  for (uint64_t c = 0; c < C; ++c) {
    start[c] = acc;
    acc += count[c];
  }
  std::vector<uint32_t> cursor(start, start + C);
  for (uint32_t i = 0; i < n; ++i) perm[cursor[keys[i]]++] = i;
  if (overflow) *overflow = over_any;
}

// ------------------------------------------------------------- engine ----

constexpr uint32_t kMaxNeighbors = 64;  // neighborList.ts:14
constexpr int32_t kHeadroom = 1 << 30;  // accumulator.ts:77

template <typename T>
struct Accum {
  // accumulator.ts:88-178: i32 ticks xyz per particle, scale floor(2^30/maxMag).
  std::vector<int32_t> d;
  uint32_t flag = 0;
  T scale = 0, inv = 0;
  void init(uint32_t cap, double maxMag) {
    d.assign(3 * static_cast<size_t>(cap), 0);
    const double s = std::floor(static_cast<double>(kHeadroom) / maxMag);
    scale = static_cast<T>(s);
    inv = static_cast<T>(1.0 / s);
  }
  static int32_t to_ticks(T v, T scale) {
    // value * scale, round half to even, saturating conversion.
    const T p = v * scale;
    return sat_i32(static_cast<double>(std::nearbyint(p)));
  }
  void add(uint32_t i, V3<T> v) {
    const int32_t a = to_ticks(v.x, scale), b = to_ticks(v.y, scale), c = to_ticks(v.z, scale);
    int32_t* p = &d[3 * static_cast<size_t>(i)];
    __atomic_fetch_add(&p[0], a, __ATOMIC_RELAXED);
    __atomic_fetch_add(&p[1], b, __ATOMIC_RELAXED);
    __atomic_fetch_add(&p[2], c, __ATOMIC_RELAXED);
  }
  void reset() { std::fill(d.begin(), d.end(), 0); }
  // Returns the change for particle i and clears it (buildApplyKernel).
  V3<T> take(uint32_t i, uint32_t* sat) {
    int32_t* p = &d[3 * static_cast<size_t>(i)];
    V3<T> t = v3(static_cast<T>(p[0]), static_cast<T>(p[1]), static_cast<T>(p[2]));
    const T m = tmax(tmax(std::fabs(t.x), std::fabs(t.y)), std::fabs(t.z));
    if (m >= static_cast<T>(kHeadroom)) *sat = 1;
    p[0] = p[1] = p[2] = 0;
    return t * inv;
  }
};

struct Range {
  uint32_t start = 0, count = 0;
  bool contains(uint32_t j) const { return j >= start && j < start + count; }
};

template <typename T>
struct Fluid {
  Range range;
  double restDensity, spacing, h, compliance, viscosity, vorticity = 0, surfaceTension = 0, adhesion = 0;
  bool hasViscosity, hasVorticity = false, hasSurfaceTension = false, hasAdhesion = false;
  std::vector<Range> boundaries;
  std::vector<uint8_t> boundaryStatic;
  // uniforms at engine precision
  T uRho0, uVolume, uMass, uH, uHSq, uPoly6, uSpiky, uCompliance, uC, uEps = 0;
  // buffers (capacity sized like the reference)
  std::vector<T> density, lambda;
  std::vector<V3<T>> deltaX, deltaV;
  std::vector<V3<T>> omega, eta;  // vorticity confinement (velocity.ts:13-21)
  std::vector<T> omegaLength;
  // surface tension and adhesion (cohesion.ts, adhesion.ts)
  T uGamma = 0, uBeta = 0;
  std::vector<V3<T>> normal;
  Accum<T> impulses;  // velocity changes, maxMag 50 (FluidSystem.ts:237)
  std::vector<uint32_t> nbrIdx, nbrCount;  // column-major k*count + local
  uint32_t nbrOverflow = 0;
  bool hasReaction = false;
  Accum<T> reaction;
};

template <typename T>
struct Body {
  Range range;
  uint32_t surfaceCount;
  double compliance;
  std::vector<uint32_t> edges;
  std::vector<float> restPositions;
};

template <typename T>
struct Softbodies {
  std::vector<Body<T>> bodies;
  bool local = true;
  bool selfCollision = false;
  Range span;
  std::vector<float> restOffsets;  // float4 per particle (reference Float32Array)
  std::vector<float> weights;
  std::vector<float> bodyCompliance;
  // local shape matching
  std::vector<uint32_t> offsets, indices;
  std::vector<float> restCenters;  // float4 per particle
  std::vector<V3<T>> centers;
  std::vector<T> rot9;             // 9 per particle (particleRotations rows)
  std::vector<V3<T>> pairLambda;
  Accum<T> acc;
  T uAi, uMaxC, uMaxC2;
  // global + frame outputs
  std::vector<V3<T>> bodyCenters;
  std::vector<T> bodyRot9;
  std::vector<V3<T>> lambdaG;
};

template <typename T>
struct Cloth {
  uint32_t offset, n;
  std::vector<uint32_t> pairs;  // absolute indices
  std::vector<T> rest, compliance;
  std::vector<T> lambda;
  std::vector<std::vector<uint32_t>> groups;
  // bending.ts: (p1, p2, p3, p4) absolute indices, rest angles, one compliance
  std::vector<uint32_t> bend;
  std::vector<T> bendRest, bendLambda;
  T bendCompliance = 0;
  std::vector<std::vector<uint32_t>> bendGroups;
  // tether.ts: (free particle, anchor) absolute indices, rest radii
  std::vector<uint32_t> tether;
  std::vector<T> tetherRest, tetherLambda;
  T tetherCompliance = 0;
  std::vector<std::vector<uint32_t>> tetherGroups;
  // aero.ts: absolute triangles and the per-vertex incidence CSR
  std::vector<uint32_t> tris, incOff, incTri;
  float wind[3] = {0, 0, 0};
  float drag = 0.6125f, lift = 0.3f;
  // ClothSystem.buildDamping: edge-neighbour CSR (cloth-local)
  bool hasDamping = false;
  float damping = 0;
  std::vector<uint32_t> dampOff, dampNbr;
};

struct Prim {
  uint32_t kind, flags;
  float data0[4], data1[4], velocity[4], rotation[4], spin[4];
};

// SDFCollider (src/core/collision/SDFCollider.ts:88-137): the grid holds the
// half-float values the collider's texture holds (widened back to float),
// the transform uniforms are f32.
struct SdfGrid {
  uint32_t res[3];
  std::vector<float> phi;
  float origin[3], voxel[3], invVoxel[3], position[3];
  float R[9], invR[9];  // row-major
  float scale, invScale, thickness, muS, muK;
};

// IEEE half rounding (nearest even) of a value clamped to +-65504, returned
// as the float the half represents.
inline float half_round(float f) {
  f = std::min(std::max(f, -65504.0f), 65504.0f);
  if (std::isnan(f)) return f;
  const float a = std::fabs(f);
  if (a < 6.103515625e-05f) {  // 2^-14: subnormal halves are multiples of 2^-24
    return std::copysign(std::nearbyint(a * 16777216.0f) / 16777216.0f, f);
  }
  int e;
  std::frexp(a, &e);                               // a in [2^(e-1), 2^e)
  const float ulp = std::ldexp(1.0f, e - 1 - 10);  // 10 fraction bits
  return std::copysign(std::nearbyint(a / ulp) * ulp, f);
}

inline void sdf_set_transform(SdfGrid& g, const float pos[3], const float rot[4], float scale) {
  double q[4], n = 0;
  for (int a = 0; a < 4; ++a) {
    q[a] = rot[a];
    n += q[a] * q[a];
  }
  n = std::sqrt(n);
  for (int a = 0; a < 4; ++a) q[a] /= n;
  const double x = q[0], y = q[1], z = q[2], w = q[3];
  // rotation matrix of a unit quaternion
  const double R[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                       2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                       2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      g.R[3 * r + c] = static_cast<float>(R[3 * r + c]);
      g.invR[3 * r + c] = static_cast<float>(R[3 * c + r]);
    }
  for (int a = 0; a < 3; ++a) g.position[a] = pos[a];
  g.scale = scale;
  g.invScale = static_cast<float>(1.0 / scale);
}

enum MatKind { MAT_FLUID, MAT_SOFT, MAT_CLOTH };

template <typename T>
struct Engine {
  uint32_t cap = 0;
  double radius = 0;
  // particle state (float4 rows; w kept as the reference keeps it)
  std::vector<T> pos, pred, vel, rot, prot, angv;
  std::vector<T> invMass, bvol;
  std::vector<uint32_t> group;
  // materials in SimLoop order
  std::vector<std::pair<MatKind, int>> materials;
  std::vector<Fluid<T>> fluids;
  std::vector<Softbodies<T>> softs;
  std::vector<Cloth<T>> cloths;
  std::vector<Prim> prims;
  std::vector<SdfGrid> sdfs;
  std::vector<T> sdfLambda;  // 2 * cap * sdfs
  // loop
  bool built = false, initialized = false;
  uint32_t substeps = 4, iterations = 2;
  T gx = 0, gy = 0, gz = 0;
  T dt = 0, uSubsteps = 0;
  // grid
  bool hasGrid = false;
  pf_grid_desc grid{};
  std::vector<uint32_t> cellIndex, counts, cellStart, sorted;
  uint32_t gridOverflow = 0;
  // colliders
  bool hasColliders = false;
  Accum<T> accPos, accVel;
  // particle contacts (loop.ts:347-417, src/core/contact/)
  bool hasContact = false;
  T cMuS = 0, cMuK = 0, cDist = 0, cCand2 = 0;
  uint32_t maxContacts = 0, contactCount = 0;
  std::vector<Range> quietRanges;  // Material.noSelfContacts besides the fluids'
  std::vector<uint8_t> quiet;
  struct Contact {
    uint32_t i, j;
    int32_t ln, lt;  // ticks of 2^-20 kg m (ContactBuffer.ts:16)
    V3<T> n;
  };
  std::vector<Contact> contacts;
  bool hasAcc() const { return hasColliders || hasContact; }
  std::vector<T> primLambda;  // 2 * cap * primCap
  uint32_t primCap = 0;
  T clock = 0;
  int nthreads = 1;

  V3<T> p3(const std::vector<T>& a, uint32_t i) const {
    return v3(a[4 * i], a[4 * i + 1], a[4 * i + 2]);
  }
  void set3(std::vector<T>& a, uint32_t i, V3<T> v, T w) {
    a[4 * i] = v.x;
    a[4 * i + 1] = v.y;
    a[4 * i + 2] = v.z;
    a[4 * i + 3] = w;
  }

  // ------------------------------------------------------------ grid ----
  void rebuild_grid(const std::vector<T>& positions) {
    const uint64_t C = grid_cells(grid);
    cellIndex.resize(cap);
    counts.resize(C);
    cellStart.resize(C);
    sorted.resize(cap);
    stable_count_sort<T>(grid, cap, positions.data(), cellIndex.data(), sorted.data(),
                         cellStart.data(), counts.data(), &gridOverflow);
  }

  // query.ts:24-70: 27 buckets in dz, dy, dx order, buckets already visited
  // skipped; fn(j) for each candidate in bucket order.
  template <typename F>
  void for_each_neighbor(V3<T> p, F&& fn) const {
    const T ox = static_cast<T>(grid.origin[0]), oy = static_cast<T>(grid.origin[1]),
            oz = static_cast<T>(grid.origin[2]), cs = static_cast<T>(grid.cell_size);
    const int32_t qx = sat_i32(std::floor((p.x - ox) / cs));
    const int32_t qy = sat_i32(std::floor((p.y - oy) / cs));
    const int32_t qz = sat_i32(std::floor((p.z - oz) / cs));
    uint32_t visited[27];
    int nv = 0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const uint32_t b =
              morton_unmasked(static_cast<int32_t>(static_cast<uint32_t>(qx) + static_cast<uint32_t>(dx)),
                              static_cast<int32_t>(static_cast<uint32_t>(qy) + static_cast<uint32_t>(dy)),
                              static_cast<int32_t>(static_cast<uint32_t>(qz) + static_cast<uint32_t>(dz))) &
              (grid.table_size - 1u);
          bool seen = false;
          for (int v = 0; v < nv; ++v) seen = seen || visited[v] == b;
          visited[nv++] = b;
          if (seen) continue;
          const uint32_t s = cellStart[b], e = s + counts[b];
          for (uint32_t k = s; k < e; ++k) fn(sorted[k], k);
        }
  }

  // neighborList.ts:48-71 over the grid's sorted predicted positions.
  void build_neighbors(Fluid<T>& f) {
    const uint32_t rc = f.range.count;
    uint32_t ovf = 0;
    parallel_for(0, static_cast<int64_t>(rc), [&](int64_t li) {
      const uint32_t local = static_cast<uint32_t>(li);
      const V3<T> xi = p3(pred, local + f.range.start);
      uint32_t cnt = 0;
      for_each_neighbor(xi, [&](uint32_t j, uint32_t) {
        const V3<T> off = xi - p3(pred, j);  // sortedPredictedPositions[slot] = x*[j]
        if (dot(off, off) < f.uHSq) {
          if (cnt < kMaxNeighbors) {
            f.nbrIdx[static_cast<size_t>(cnt) * rc + local] = j;
            cnt++;
          } else {
            __atomic_store_n(&ovf, 1u, __ATOMIC_RELAXED);
          }
        }
      });
      f.nbrCount[local] = cnt;
    });
    f.nbrOverflow = ovf;
  }

  // ----------------------------------------------------------- sph ----
  static T poly6(T rSq, const Fluid<T>& f) {
    const T d = tmax(f.uHSq - rSq, static_cast<T>(0));
    return d * d * d * f.uPoly6;
  }
  static V3<T> spiky_grad(V3<T> r, const Fluid<T>& f) {
    const T rSq = dot(r, r);
    const T rl = std::sqrt(rSq);
    const T t = tmax(f.uH - rl, static_cast<T>(0));
    const T rSafe = tmax(rl, static_cast<T>(1e-20));
    const V3<T> rHat = r / rSafe;
    const T mag = -(t * t * f.uSpiky);
    return rHat * mag;
  }
  struct NMass {
    T mass, boundaryMass, invMass;
    bool isBoundary;
  };
  NMass neighbor_mass(const Fluid<T>& f, uint32_t j) const {
    const T volume = bvol[j];
    const T w = invMass[j];
    NMass m;
    m.isBoundary = volume > 0;
    m.boundaryMass = f.uRho0 * volume;
    const T own = w > 0 ? static_cast<T>(1) / w : static_cast<T>(0);
    m.mass = m.isBoundary ? m.boundaryMass : own;
    m.invMass = w;
    return m;
  }

  // boundaryVolume.ts:36-52
  void boundary_volume(const Fluid<T>& f, Range r, const std::vector<T>& positions) {
    std::vector<T> out(r.count);
    parallel_for(0, static_cast<int64_t>(r.count), [&](int64_t li) {
      const uint32_t i = r.start + static_cast<uint32_t>(li);
      const V3<T> xi = p3(positions, i);
      T sum = 0;
      for_each_neighbor(xi, [&](uint32_t j, uint32_t) {
        if (!r.contains(j)) return;
        const V3<T> off = xi - p3(positions, j);
        const T rSq = dot(off, off);
        if (rSq >= f.uHSq) return;
        sum += poly6(rSq, f);
      });
      out[li] = static_cast<T>(1) / tmax(sum, static_cast<T>(1e-12));
    });
    for (uint32_t li = 0; li < r.count; ++li) bvol[r.start + li] = out[li];
  }

  // lambda.ts:41-71
  void fluid_lambda(Fluid<T>& f) {
    const uint32_t rc = f.range.count;
    parallel_for(0, static_cast<int64_t>(rc), [&](int64_t li) {
      const uint32_t local = static_cast<uint32_t>(li), i = f.range.start + local;
      const V3<T> xi = p3(pred, i);
      T rho = 0, gradSqSum = 0;
      V3<T> gradSum = v3<T>(0, 0, 0);
      const uint32_t nc = f.nbrCount[local];
      for (uint32_t k = 0; k < nc; ++k) {
        const uint32_t j = f.nbrIdx[static_cast<size_t>(k) * rc + local];
        const V3<T> off = xi - p3(pred, j);
        const NMass nb = neighbor_mass(f, j);
        rho += nb.mass * poly6(dot(off, off), f);
        const V3<T> g = spiky_grad(off, f) * nb.mass;
        gradSum = gradSum + g;
        gradSqSum += dot(g, g) * nb.invMass;
      }
      f.density[i] = rho;
      const T invRho0 = static_cast<T>(1) / f.uRho0;
      const T C = rho * invRho0 - static_cast<T>(1);
      if (C <= 0) {
        f.lambda[i] = 0;
        return;
      }
      const T gradNorm = (dot(gradSum, gradSum) * invMass[i] + gradSqSum) * (invRho0 * invRho0);
      const T alphaTilde = f.uCompliance / (dt * dt);
      f.lambda[i] = -C / tmax(gradNorm + alphaTilde, static_cast<T>(1e-20));
    });
  }

  // positionDelta.ts:41-85
  void fluid_delta(Fluid<T>& f) {
    const uint32_t rc = f.range.count;
    parallel_for(0, static_cast<int64_t>(rc), [&](int64_t li) {
      const uint32_t local = static_cast<uint32_t>(li), i = f.range.start + local;
      const V3<T> xi = p3(pred, i);
      const T lambdaI = f.lambda[i];
      V3<T> sum = v3<T>(0, 0, 0);
      const uint32_t nc = f.nbrCount[local];
      for (uint32_t k = 0; k < nc; ++k) {
        const uint32_t j = f.nbrIdx[static_cast<size_t>(k) * rc + local];
        const NMass nb = neighbor_mass(f, j);
        const V3<T> g = spiky_grad(xi - p3(pred, j), f);
        sum = sum + g * ((lambdaI + f.lambda[j]) * nb.mass);
        if (f.hasReaction && nb.isBoundary && nb.invMass > 0 && lambdaI != 0) {
          bool in = false;
          for (const Range& r : f.boundaries) in = in || r.contains(j);
          if (in) f.reaction.add(j, g * ((-(lambdaI / f.uRho0)) * nb.boundaryMass * nb.invMass));
        }
      }
      f.deltaX[i] = (sum / f.uRho0) * invMass[i];
    });
  }
  void fluid_apply(Fluid<T>& f) {
    for (uint32_t li = 0; li < f.range.count; ++li) {
      const uint32_t i = f.range.start + li;
      set3(pred, i, p3(pred, i) + f.deltaX[i], pred[4 * i + 3]);
    }
  }
  // reaction.accumulator.buildApplyKernel over the covering range of boundaries.
  void fluid_reaction_apply(Fluid<T>& f) {
    uint32_t s = UINT32_MAX, e = 0;
    for (const Range& r : f.boundaries) {
      s = std::min(s, r.start);
      e = std::max(e, r.start + r.count);
    }
    for (uint32_t i = s; i < e; ++i) {
      const V3<T> c = f.reaction.take(i, &f.reaction.flag);
      set3(pred, i, p3(pred, i) + c, pred[4 * i + 3]);
    }
  }

  // velocity.ts:36-120 (XSPH only; vorticity is not part of this path)
  // cohesion.ts:33-48: n_i = h sum_j V_j grad W(x*_i - x*_j)
  void color_normal(Fluid<T>& f) {
    const uint32_t rc = f.range.count;
    parallel_for(0, static_cast<int64_t>(rc), [&](int64_t li) {
      const uint32_t local = static_cast<uint32_t>(li), i = f.range.start + local;
      const V3<T> xi = p3(pred, i);
      V3<T> sum = v3<T>(0, 0, 0);
      const uint32_t nc = f.nbrCount[local];
      for (uint32_t k = 0; k < nc; ++k) {
        const uint32_t j = f.nbrIdx[static_cast<size_t>(k) * rc + local];
        const T volume = bvol[j] > 0 ? bvol[j] : f.uVolume;
        sum = sum + spiky_grad(xi - p3(pred, j), f) * volume;
      }
      f.normal[i] = sum * f.uH;
    });
  }
  // cohesion.ts:54-66: the cohesion spline C(r), constants as f32 literals
  T cohesion_spline(T r, const Fluid<T>& f) const {
    const bool dbl = sizeof(T) == 8;
    auto U = [&](double v) { return dbl ? static_cast<T>(v) : static_cast<T>(static_cast<float>(v)); };
    const T h = U(f.h);
    const T gap = tmax(h - r, static_cast<T>(0));
    const T shared = gap * gap * gap * (r * r * r);
    const T value = r * static_cast<T>(2) > h ? shared : shared * static_cast<T>(2) - U(std::pow(f.h, 6) / 64.0);
    return (r > 0 && r <= h) ? value * U(32.0 / (M_PI * std::pow(f.h, 9))) : static_cast<T>(0);
  }
  // adhesion.ts:33-47: the adhesion spline A(r)
  T adhesion_spline(T r, const Fluid<T>& f) const {
    const bool dbl = sizeof(T) == 8;
    auto U = [&](double v) { return dbl ? static_cast<T>(v) : static_cast<T>(static_cast<float>(v)); };
    const T h = U(f.h);
    const T inner = tmax(r * r * U(-4.0 / f.h) + r * static_cast<T>(6) - U(2.0 * f.h), static_cast<T>(0));
    const T root = std::sqrt(std::sqrt(inner));
    return (r * static_cast<T>(2) > h && r <= h) ? root * U(0.007 / std::pow(f.h, 3.25)) : static_cast<T>(0);
  }
  // cohesion.ts:75-120: each fluid pair once (j > i inside the range)
  void surface_tension(Fluid<T>& f) {
    const uint32_t rc = f.range.count, end = f.range.start + rc;
    parallel_for(0, static_cast<int64_t>(rc), [&](int64_t li) {
      const uint32_t local = static_cast<uint32_t>(li), i = f.range.start + local;
      const V3<T> xi = p3(pred, i);
      const V3<T> ni = f.normal[i];
      const T rhoI = f.density[i];
      const uint32_t nc = f.nbrCount[local];
      for (uint32_t k = 0; k < nc; ++k) {
        const uint32_t j = f.nbrIdx[static_cast<size_t>(k) * rc + local];
        if (j <= i || j >= end) continue;
        const V3<T> off = xi - p3(pred, j);
        const T r = length(off);
        if (r < static_cast<T>(1e-20)) continue;
        const T corr = (f.uRho0 * static_cast<T>(2)) / tmax(rhoI + f.density[j], static_cast<T>(1));
        const V3<T> coh = (off / r) * neg1(f.uGamma * f.uMass * f.uMass * cohesion_spline(r, f));
        const V3<T> curv = (ni - f.normal[j]) * neg1(f.uGamma * f.uMass);
        const V3<T> dv = (coh + curv) * corr / f.uMass * dt;
        f.impulses.add(i, dv);
        f.impulses.add(j, v3<T>(-dv.x, -dv.y, -dv.z));
      }
    });
  }
  // adhesion.ts:55-76: toward boundary neighbours, fluid side only
  void adhesion(Fluid<T>& f) {
    const uint32_t rc = f.range.count;
    parallel_for(0, static_cast<int64_t>(rc), [&](int64_t li) {
      const uint32_t local = static_cast<uint32_t>(li), i = f.range.start + local;
      const V3<T> xi = p3(pred, i);
      const uint32_t nc = f.nbrCount[local];
      for (uint32_t k = 0; k < nc; ++k) {
        const uint32_t j = f.nbrIdx[static_cast<size_t>(k) * rc + local];
        const T volume = bvol[j];
        if (volume <= 0) continue;
        const V3<T> off = xi - p3(pred, j);
        const T r = length(off);
        if (r < static_cast<T>(1e-20)) continue;
        const V3<T> force = (off / r) * neg1(f.uBeta * f.uMass * (f.uRho0 * volume) * adhesion_spline(r, f));
        f.impulses.add(i, force / f.uMass * dt);
      }
    });
  }
  static T neg1(T v) { return -v; }

  // velocity.ts:36-120: one walk for the curl (vorticity) and the XSPH
  // change, the gradient of |omega| over fluid neighbours, then the apply.
  void fluid_velocity(Fluid<T>& f) {
    const uint32_t rc = f.range.count;
    const bool vort = f.hasVorticity, visc = f.hasViscosity;
    parallel_for(0, static_cast<int64_t>(rc), [&](int64_t li) {
      const uint32_t local = static_cast<uint32_t>(li), i = f.range.start + local;
      const V3<T> xi = p3(pos, i), vi = p3(vel, i);
      V3<T> curl = v3<T>(0, 0, 0), smoothing = v3<T>(0, 0, 0);
      const uint32_t nc = f.nbrCount[local];
      for (uint32_t k = 0; k < nc; ++k) {
        const uint32_t j = f.nbrIdx[static_cast<size_t>(k) * rc + local];
        const V3<T> off = xi - p3(pos, j);
        const V3<T> vj = p3(vel, j);
        const T volume = bvol[j] > 0 ? bvol[j] : f.uVolume;
        if (vort) curl = curl + cross(vi - vj, spiky_grad(off, f)) * volume;
        if (visc) smoothing = smoothing + ((vj - vi) * poly6(dot(off, off), f)) * volume;
      }
      if (vort) {
        f.omega[i] = curl;
        f.omegaLength[i] = length(curl);
      }
      if (visc) f.deltaV[i] = smoothing * f.uC;
    });
    if (vort) {
      // velocity.ts:75-92: eta = sum over fluid neighbours of grad W (|w_j| - |w_i|) V
      parallel_for(0, static_cast<int64_t>(rc), [&](int64_t li) {
        const uint32_t local = static_cast<uint32_t>(li), i = f.range.start + local;
        const V3<T> xi = p3(pos, i);
        const T wi = f.omegaLength[i];
        V3<T> e = v3<T>(0, 0, 0);
        const uint32_t nc = f.nbrCount[local];
        for (uint32_t k = 0; k < nc; ++k) {
          const uint32_t j = f.nbrIdx[static_cast<size_t>(k) * rc + local];
          if (bvol[j] > 0) continue;
          e = e + spiky_grad(xi - p3(pos, j), f) * ((f.omegaLength[j] - wi) * f.uVolume);
        }
        f.eta[i] = e;
      });
    }
    // velocity.ts:99-120
    for (uint32_t li = 0; li < rc; ++li) {
      const uint32_t i = f.range.start + li;
      V3<T> change = v3<T>(0, 0, 0);
      if (vort) {
        const V3<T> e = f.eta[i];
        const T el = length(e);
        if (el >= static_cast<T>(1e-12)) change = change + cross(e / el, f.omega[i]) * f.uEps * dt;
      }
      if (visc) change = change + f.deltaV[i];
      set3(vel, i, p3(vel, i) + change, vel[4 * i + 3]);
    }
  }

  // ------------------------------------------------------ integration ----
  void predict() {
    const V3<T> g = v3(gx, gy, gz);
    for (uint32_t i = 0; i < cap; ++i) {
      if (!(invMass[i] > 0)) continue;
      const V3<T> v = p3(vel, i) + g * dt;
      set3(vel, i, v, 0);
      set3(pred, i, p3(pos, i) + v * dt, 0);
    }
  }
  void advect() {
    for (uint32_t i = 0; i < cap; ++i) {
      if (!(invMass[i] > 0)) continue;
      set3(vel, i, (p3(pred, i) - p3(pos, i)) / dt, 0);
      for (int c = 0; c < 4; ++c) pos[4 * i + c] = pred[4 * i + c];
    }
  }

  // -------------------------------------------------------- colliders ----
  static V3<T> qrot(const T q[4], V3<T> v) {
    const V3<T> qv = v3(q[0], q[1], q[2]);
    const V3<T> t = cross(qv, v) * static_cast<T>(2);
    return v + t * q[3] + cross(qv, t);
  }
  V3<T> prim_pivot(const Prim& p) const {
    if (p.kind == PF_PRIM_PLANE) return v3<T>(p.data1[0], p.data1[1], p.data1[2]);
    if (p.kind == PF_PRIM_CAPSULE)
      return (v3<T>(p.data0[0], p.data0[1], p.data0[2]) + v3<T>(p.data1[0], p.data1[1], p.data1[2])) *
             static_cast<T>(0.5);
    return v3<T>(p.data0[0], p.data0[1], p.data0[2]);
  }
  T sweep_time(const Prim& p, T rewind) const {
    return (p.flags & PF_PRIM_SWEEP) ? rewind : static_cast<T>(0);
  }
  // primitives.ts:203-335 with the PrimitiveSet fields (velocity and spin present).
  void prim_sdf(const Prim& p, V3<T> xWorld, T rewind, T* phi, V3<T>* grad) const {
    const T t = sweep_time(p, rewind);
    const V3<T> shifted = xWorld + v3<T>(p.velocity[0], p.velocity[1], p.velocity[2]) * t;
    const V3<T> pivot = prim_pivot(p);
    const V3<T> spin = v3<T>(p.spin[0], p.spin[1], p.spin[2]);
    const T rate = length(spin);
    const T half = rate * t * static_cast<T>(0.5);
    const V3<T> axis = spin / tmax(rate, static_cast<T>(1e-8));
    const V3<T> as = axis * static_cast<T>(std::sin(half));
    const T turn[4] = {as.x, as.y, as.z, static_cast<T>(std::cos(half))};
    const V3<T> x = pivot + qrot(turn, shifted - pivot);
    const T unturn[4] = {-turn[0], -turn[1], -turn[2], turn[3]};
    T ph = 0;
    V3<T> g = v3<T>(0, 0, 0);
    const V3<T> d0 = v3<T>(p.data0[0], p.data0[1], p.data0[2]);
    const V3<T> d1 = v3<T>(p.data1[0], p.data1[1], p.data1[2]);
    if (p.kind == PF_PRIM_PLANE) {
      ph = dot(d0, x - d1);
      g = d0;
    } else if (p.kind == PF_PRIM_SPHERE) {
      const V3<T> diff = x - d0;
      const T len = length(diff);
      ph = len - static_cast<T>(p.data0[3]);
      g = diff / tmax(len, static_cast<T>(1e-8));
    } else if (p.kind == PF_PRIM_BOX) {
      const T rot[4] = {p.rotation[0], p.rotation[1], p.rotation[2], p.rotation[3]};
      const T conj[4] = {-rot[0], -rot[1], -rot[2], rot[3]};
      const V3<T> xl = qrot(conj, x - d0);
      const V3<T> q = v3(std::fabs(xl.x), std::fabs(xl.y), std::fabs(xl.z)) - d1;
      const V3<T> qPos = v3(tmax(q.x, static_cast<T>(0)), tmax(q.y, static_cast<T>(0)), tmax(q.z, static_cast<T>(0)));
      const T outside = length(qPos);
      const T inside = tmin(tmax(tmax(q.x, q.y), q.z), static_cast<T>(0));
      ph = outside + inside;
      const V3<T> sg = v3<T>(xl.x >= 0 ? 1 : -1, xl.y >= 0 ? 1 : -1, xl.z >= 0 ? 1 : -1);
      const T outsideLen = length(qPos);
      const bool isOutside = outsideLen > static_cast<T>(1e-8);
      const bool domX = q.x >= q.y && q.x >= q.z;
      const bool domY = q.y >= q.x && q.y >= q.z;
      const V3<T> insideDir = v3<T>(domX ? sg.x : 0, (!domX && domY) ? sg.y : 0, (!domX && !domY) ? sg.z : 0);
      const V3<T> local = isOutside ? v3(qPos.x * sg.x, qPos.y * sg.y, qPos.z * sg.z) /
                                          tmax(outsideLen, static_cast<T>(1e-8))
                                    : insideDir;
      g = qrot(rot, local);
    } else if (p.kind == PF_PRIM_CAPSULE) {
      const V3<T> ab = d1 - d0;
      const V3<T> ax = x - d0;
      const T abLenSq = tmax(dot(ab, ab), static_cast<T>(1e-8));
      T tt = dot(ax, ab) / abLenSq;
      tt = tmin(tmax(tt, static_cast<T>(0)), static_cast<T>(1));
      const V3<T> closest = d0 + ab * tt;
      const V3<T> diff = x - closest;
      const T len = length(diff);
      ph = len - static_cast<T>(p.data0[3]);
      g = diff / tmax(len, static_cast<T>(1e-8));
    }
    if (p.flags & PF_PRIM_INVERT) {
      ph = -ph;
      g = neg(g);
    }
    g = qrot(unturn, g);
    *phi = ph;
    *grad = g;
  }
  // primitives.ts:342-360
  V3<T> prim_surface_velocity(const Prim& p, V3<T> xWorld, T rewind) const {
    const V3<T> velocity = v3<T>(p.velocity[0], p.velocity[1], p.velocity[2]);
    const V3<T> pivot = prim_pivot(p);
    const T t = sweep_time(p, rewind);
    const V3<T> arm = (xWorld - pivot) + velocity * t;
    return velocity + cross(v3<T>(p.spin[0], p.spin[1], p.spin[2]), arm);
  }

  // PrimitiveSet.ts:339-365 + collider.ts:53-89
  void collider_solve() {
    const T radius = sizeof(T) == 8 ? static_cast<T>(this->radius)
                                    : static_cast<T>(static_cast<float>(this->radius));
    const uint32_t np = static_cast<uint32_t>(prims.size());
    parallel_for(0, static_cast<int64_t>(cap), [&](int64_t pi) {
      const uint32_t p = static_cast<uint32_t>(pi);
      const T w = invMass[p];
      if (!(w > 0)) return;
      const V3<T> xStar = p3(pred, p);
      const V3<T> disp = xStar - p3(pos, p);
      for (uint32_t s = 0; s < np; ++s) {
        T phi;
        V3<T> n;
        prim_sdf(prims[s], xStar, clock, &phi, &n);
        if (!(phi < radius)) continue;
        const V3<T> colDisp = prim_surface_velocity(prims[s], xStar, clock) * dt;
        const T depth = radius - phi;
        const T muS = static_cast<T>(prims[s].data1[3]);
        const size_t li = (static_cast<size_t>(p) * primCap + s) * 2;
        const T lambdaN = primLambda[li] + depth / w;
        primLambda[li] = lambdaN;
        const V3<T> slip = disp - colDisp;
        const V3<T> tang = slip - n * dot(slip, n);
        const T tl = length(tang);
        const T lambdaT = primLambda[li + 1];
        const bool sticks = tl > static_cast<T>(1e-10) && (tl / w <= muS * lambdaN - lambdaT);
        const V3<T> push = n * depth;
        accPos.add(p, sticks ? push - tang : push);
        primLambda[li + 1] = lambdaT + (sticks ? tl / w : static_cast<T>(0));
      }
    });
  }
  // PrimitiveSet.ts:367-398 + collider.ts:96-118
  void collider_friction() {
    const uint32_t np = static_cast<uint32_t>(prims.size());
    parallel_for(0, static_cast<int64_t>(cap), [&](int64_t pi) {
      const uint32_t p = static_cast<uint32_t>(pi);
      const T w = invMass[p];
      if (!(w > 0)) return;
      const V3<T> xStar = p3(pred, p);
      const V3<T> velocity = p3(vel, p);
      for (uint32_t s = 0; s < np; ++s) {
        const T lambdaN = primLambda[(static_cast<size_t>(p) * primCap + s) * 2];
        if (!(lambdaN > 0)) continue;
        T phi;
        V3<T> g;
        prim_sdf(prims[s], xStar, clock, &phi, &g);
        const T len = length(g);
        if (!(len > static_cast<T>(1e-6))) continue;
        const V3<T> n = g / len;
        const V3<T> rel = velocity - prim_surface_velocity(prims[s], xStar, clock);
        const V3<T> vT = rel - n * dot(n, rel);
        const T vTL = length(vT);
        if (vTL > static_cast<T>(1e-6)) {
          const T muK = static_cast<T>(prims[s].velocity[3]);
          const T change = tmin(muK * lambdaN * w / dt, vTL);
          accVel.add(p, neg((vT / vTL) * change));
        }
      }
    });
  }
  // sample.ts:12-53: trilinear filter at continuous grid coordinate g,
  // clamp to the edge voxels.
  static T sdf_trilinear(const SdfGrid& G, T gx, T gy, T gz) {
    gx -= static_cast<T>(0.5);
    gy -= static_cast<T>(0.5);
    gz -= static_cast<T>(0.5);
    const int nx = static_cast<int>(G.res[0]), ny = static_cast<int>(G.res[1]), nz = static_cast<int>(G.res[2]);
    const int i0 = std::min(std::max(static_cast<int>(std::floor(gx)), 0), nx - 2);
    const int j0 = std::min(std::max(static_cast<int>(std::floor(gy)), 0), ny - 2);
    const int k0 = std::min(std::max(static_cast<int>(std::floor(gz)), 0), nz - 2);
    auto c01 = [](T t) { return t < 0 ? static_cast<T>(0) : (t > 1 ? static_cast<T>(1) : t); };
    const T tx = c01(gx - static_cast<T>(i0)), ty = c01(gy - static_cast<T>(j0)), tz = c01(gz - static_cast<T>(k0));
    const size_t sy = static_cast<size_t>(nx), sz = static_cast<size_t>(nx) * ny;
    const size_t b = static_cast<size_t>(i0) + j0 * sy + k0 * sz;
    auto v = [&](size_t o) { return static_cast<T>(G.phi[b + o]); };
    auto lerp = [](T a, T c, T t) { return a + (c - a) * t; };
    const T c00 = lerp(v(0), v(1), tx), c10 = lerp(v(sy), v(sy + 1), tx);
    const T c0z = lerp(v(sz), v(sz + 1), tx), c1z = lerp(v(sz + sy), v(sz + sy + 1), tx);
    return lerp(lerp(c00, c10, ty), lerp(c0z, c1z, ty), tz);
  }
  // sdf.ts:107-147: world -> local, phi, central-difference gradient one
  // voxel apart, back to world.
  static void sdf_sample(const SdfGrid& G, V3<T> x, T* phi, V3<T>* grad) {
    const V3<T> off = v3<T>(x.x - static_cast<T>(G.position[0]), x.y - static_cast<T>(G.position[1]),
                            x.z - static_cast<T>(G.position[2]));
    auto row = [&](const float* M, int r, V3<T> a) {
      return static_cast<T>(M[3 * r]) * a.x + static_cast<T>(M[3 * r + 1]) * a.y + static_cast<T>(M[3 * r + 2]) * a.z;
    };
    const T is = static_cast<T>(G.invScale);
    const V3<T> xl = v3<T>(row(G.invR, 0, off) * is, row(G.invR, 1, off) * is, row(G.invR, 2, off) * is);
    const T gx = (xl.x - static_cast<T>(G.origin[0])) * static_cast<T>(G.invVoxel[0]);
    const T gy = (xl.y - static_cast<T>(G.origin[1])) * static_cast<T>(G.invVoxel[1]);
    const T gz = (xl.z - static_cast<T>(G.origin[2])) * static_cast<T>(G.invVoxel[2]);
    const T one = static_cast<T>(1), two = static_cast<T>(2);
    const T p0 = sdf_trilinear(G, gx, gy, gz);
    const V3<T> gl = v3<T>(
        (sdf_trilinear(G, gx + one, gy, gz) - sdf_trilinear(G, gx - one, gy, gz)) / (two * static_cast<T>(G.voxel[0])),
        (sdf_trilinear(G, gx, gy + one, gz) - sdf_trilinear(G, gx, gy - one, gz)) / (two * static_cast<T>(G.voxel[1])),
        (sdf_trilinear(G, gx, gy, gz + one) - sdf_trilinear(G, gx, gy, gz - one)) / (two * static_cast<T>(G.voxel[2])));
    *phi = p0 * static_cast<T>(G.scale);
    *grad = v3<T>(row(G.R, 0, gl), row(G.R, 1, gl), row(G.R, 2, gl));
  }
  // SDFCollider.ts:256-281 + collider.ts:53-89 (static surface)
  void sdf_solve() {
    const T radius = sizeof(T) == 8 ? static_cast<T>(this->radius)
                                    : static_cast<T>(static_cast<float>(this->radius));
    const uint32_t ns = static_cast<uint32_t>(sdfs.size());
    parallel_for(0, static_cast<int64_t>(cap), [&](int64_t pi) {
      const uint32_t p = static_cast<uint32_t>(pi);
      const T w = invMass[p];
      if (!(w > 0)) return;
      const V3<T> xStar = p3(pred, p);
      const V3<T> disp = xStar - p3(pos, p);
      for (uint32_t q = 0; q < ns; ++q) {
        const SdfGrid& G = sdfs[q];
        T phi;
        V3<T> g;
        sdf_sample(G, xStar, &phi, &g);
        const T gl = length(g);
        if (!(gl > static_cast<T>(1e-6))) continue;
        const T reach = radius + static_cast<T>(G.thickness);
        if (!(phi < reach)) continue;
        const V3<T> n = g / gl;
        const T depth = reach - phi;
        const size_t li = (static_cast<size_t>(p) * ns + q) * 2;
        const T lambdaN = sdfLambda[li] + depth / w;
        sdfLambda[li] = lambdaN;
        const V3<T> tang = disp - n * dot(disp, n);
        const T tl = length(tang);
        const T lambdaT = sdfLambda[li + 1];
        const bool sticks = tl > static_cast<T>(1e-10) && (tl / w <= static_cast<T>(G.muS) * lambdaN - lambdaT);
        const V3<T> push = n * depth;
        accPos.add(p, sticks ? push - tang : push);
        sdfLambda[li + 1] = lambdaT + (sticks ? tl / w : static_cast<T>(0));
      }
    });
  }
  // SDFCollider.ts:283-299 + collider.ts:96-118 (static surface)
  void sdf_friction() {
    const uint32_t ns = static_cast<uint32_t>(sdfs.size());
    parallel_for(0, static_cast<int64_t>(cap), [&](int64_t pi) {
      const uint32_t p = static_cast<uint32_t>(pi);
      const T w = invMass[p];
      if (!(w > 0)) return;
      const V3<T> xStar = p3(pred, p);
      const V3<T> velocity = p3(vel, p);
      for (uint32_t q = 0; q < ns; ++q) {
        const T lambdaN = sdfLambda[(static_cast<size_t>(p) * ns + q) * 2];
        if (!(lambdaN > 0)) continue;
        const SdfGrid& G = sdfs[q];
        T phi;
        V3<T> g;
        sdf_sample(G, xStar, &phi, &g);
        const T len = length(g);
        if (!(len > static_cast<T>(1e-6))) continue;
        const V3<T> n = g / len;
        const V3<T> vT = velocity - n * dot(n, velocity);
        const T vTL = length(vT);
        if (vTL > static_cast<T>(1e-6)) {
          const T change = tmin(static_cast<T>(G.muK) * lambdaN * w / dt, vTL);
          accVel.add(p, neg((vT / vTL) * change));
        }
      }
    });
  }
  void apply_acc(Accum<T>& a, std::vector<T>& target, uint32_t s, uint32_t e) {
    for (uint32_t i = s; i < e; ++i) {
      const V3<T> c = a.take(i, &a.flag);
      set3(target, i, p3(target, i) + c, target[4 * i + 3]);
    }
  }

  // -------------------------------------------------------- soft bodies ----
  // polarDecomp.ts:34-264
  static void polar(const T a[9], T r[9]) {
    T m00 = a[0] * a[0] + a[3] * a[3] + a[6] * a[6];
    T m01 = a[0] * a[1] + a[3] * a[4] + a[6] * a[7];
    T m02 = a[0] * a[2] + a[3] * a[5] + a[6] * a[8];
    T m11 = a[1] * a[1] + a[4] * a[4] + a[7] * a[7];
    T m12 = a[1] * a[2] + a[4] * a[5] + a[7] * a[8];
    T m22 = a[2] * a[2] + a[5] * a[5] + a[8] * a[8];
    T q00 = 1, q01 = 0, q02 = 0, q10 = 0, q11 = 1, q12 = 0, q20 = 0, q21 = 0, q22 = 1;
    const T eps = static_cast<T>(1e-12);
    auto coeffs = [](T app, T aqq, T apq, T* t, T* c, T* s) {
      const T tau = (aqq - app) / (apq * static_cast<T>(2));
      const T sg = tau >= 0 ? static_cast<T>(1) : static_cast<T>(-1);
      const T ta = std::fabs(tau);
      *t = sg / (ta + std::sqrt(ta * ta + static_cast<T>(1)));
      *c = static_cast<T>(1) / std::sqrt(*t * *t + static_cast<T>(1));
      *s = *t * *c;
    };
    for (int sweep = 0; sweep < 8; ++sweep) {
      if (std::fabs(m01) > eps) {
        T t, c, s;
        const T apq = m01, app = m00, aqq = m11;
        coeffs(app, aqq, apq, &t, &c, &s);
        const T o02 = m02, o12 = m12, a0 = q00, a1 = q01, b0 = q10, b1 = q11, c0 = q20, c1 = q21;
        m00 = app - t * apq;
        m11 = aqq + t * apq;
        m01 = 0;
        m02 = c * o02 - s * o12;
        m12 = s * o02 + c * o12;
        q00 = c * a0 - s * a1;
        q01 = s * a0 + c * a1;
        q10 = c * b0 - s * b1;
        q11 = s * b0 + c * b1;
        q20 = c * c0 - s * c1;
        q21 = s * c0 + c * c1;
      }
      if (std::fabs(m02) > eps) {
        T t, c, s;
        const T apq = m02, app = m00, aqq = m22;
        coeffs(app, aqq, apq, &t, &c, &s);
        const T o01 = m01, o12 = m12, a0 = q00, a2 = q02, b0 = q10, b2 = q12, c0 = q20, c2 = q22;
        m00 = app - t * apq;
        m22 = aqq + t * apq;
        m02 = 0;
        m01 = c * o01 - s * o12;
        m12 = s * o01 + c * o12;
        q00 = c * a0 - s * a2;
        q02 = s * a0 + c * a2;
        q10 = c * b0 - s * b2;
        q12 = s * b0 + c * b2;
        q20 = c * c0 - s * c2;
        q22 = s * c0 + c * c2;
      }
      if (std::fabs(m12) > eps) {
        T t, c, s;
        const T apq = m12, app = m11, aqq = m22;
        coeffs(app, aqq, apq, &t, &c, &s);
        const T o01 = m01, o02 = m02, a1 = q01, a2 = q02, b1 = q11, b2 = q12, c1 = q21, c2 = q22;
        m11 = app - t * apq;
        m22 = aqq + t * apq;
        m12 = 0;
        m01 = c * o01 - s * o02;
        m02 = s * o01 + c * o02;
        q01 = c * a1 - s * a2;
        q02 = s * a1 + c * a2;
        q11 = c * b1 - s * b2;
        q12 = s * b1 + c * b2;
        q21 = c * c1 - s * c2;
        q22 = s * c1 + c * c2;
      }
    }
    const T i0 = static_cast<T>(1) / std::sqrt(tmax(m00, static_cast<T>(1e-20)));
    const T i1 = static_cast<T>(1) / std::sqrt(tmax(m11, static_cast<T>(1e-20)));
    const T i2 = static_cast<T>(1) / std::sqrt(tmax(m22, static_cast<T>(1e-20)));
    const T s00 = q00 * q00 * i0 + q01 * q01 * i1 + q02 * q02 * i2;
    const T s01 = q00 * q10 * i0 + q01 * q11 * i1 + q02 * q12 * i2;
    const T s02 = q00 * q20 * i0 + q01 * q21 * i1 + q02 * q22 * i2;
    const T s11 = q10 * q10 * i0 + q11 * q11 * i1 + q12 * q12 * i2;
    const T s12 = q10 * q20 * i0 + q11 * q21 * i1 + q12 * q22 * i2;
    const T s22 = q20 * q20 * i0 + q21 * q21 * i1 + q22 * q22 * i2;
    r[0] = a[0] * s00 + a[1] * s01 + a[2] * s02;
    r[1] = a[0] * s01 + a[1] * s11 + a[2] * s12;
    r[2] = a[0] * s02 + a[1] * s12 + a[2] * s22;
    r[3] = a[3] * s00 + a[4] * s01 + a[5] * s02;
    r[4] = a[3] * s01 + a[4] * s11 + a[5] * s12;
    r[5] = a[3] * s02 + a[4] * s12 + a[5] * s22;
    r[6] = a[6] * s00 + a[7] * s01 + a[8] * s02;
    r[7] = a[6] * s01 + a[7] * s11 + a[8] * s12;
    r[8] = a[6] * s02 + a[7] * s12 + a[8] * s22;
  }

  // rotation.ts:297-314
  void rotation_predict(const Softbodies<T>& sb) {
    for (uint32_t i = sb.span.start; i < sb.span.start + sb.span.count; ++i) {
      const T q[4] = {rot[4 * i], rot[4 * i + 1], rot[4 * i + 2], rot[4 * i + 3]};
      const V3<T> om = p3(angv, i);
      const T mag = length(om);
      if (mag < static_cast<T>(1e-8)) {
        for (int c = 0; c < 4; ++c) prot[4 * i + c] = q[c];
        continue;
      }
      const T half = mag * dt * static_cast<T>(0.5);
      const V3<T> sx = om * (static_cast<T>(std::sin(half)) / mag);
      const T sw = static_cast<T>(std::cos(half));
      const V3<T> qx = v3(q[0], q[1], q[2]);
      const V3<T> nx = qx * sw + sx * q[3] + cross(sx, qx);
      const T nw = sw * q[3] - dot(sx, qx);
      set3(prot, i, nx, nw);
    }
  }
  // rotation.ts:316-343
  void rotation_advect(const Softbodies<T>& sb) {
    for (uint32_t i = sb.span.start; i < sb.span.start + sb.span.count; ++i) {
      const T q[4] = {rot[4 * i], rot[4 * i + 1], rot[4 * i + 2], rot[4 * i + 3]};
      T qp[4] = {prot[4 * i], prot[4 * i + 1], prot[4 * i + 2], prot[4 * i + 3]};
      const T dd = qp[0] * qp[0] + qp[1] * qp[1] + qp[2] * qp[2] + qp[3] * qp[3];
      const T nrm = std::sqrt(tmax(dd, static_cast<T>(1e-12)));
      for (int c = 0; c < 4; ++c) qp[c] = qp[c] / nrm;
      const V3<T> qi = v3(-q[0], -q[1], -q[2]);
      const V3<T> qpx = v3(qp[0], qp[1], qp[2]);
      const V3<T> rpre = qpx * q[3] + qi * qp[3] + cross(qpx, qi);
      const T rwpre = qp[3] * q[3] - dot(qpx, qi);
      const T flip = rwpre < 0 ? static_cast<T>(-1) : static_cast<T>(1);
      const V3<T> rx = rpre * flip;
      const T rw = rwpre * flip;
      const T hs = length(rx);
      if (hs < static_cast<T>(1e-8)) {
        set3(angv, i, v3<T>(0, 0, 0), 0);
      } else {
        const T angle = static_cast<T>(std::atan2(hs, rw)) * static_cast<T>(2);
        const V3<T> om = rx * ((angle / hs) / dt);
        const T sc = std::sqrt(static_cast<T>(1e4) / tmax(dot(om, om), static_cast<T>(1e4)));
        set3(angv, i, om * sc, 0);
      }
      for (int c = 0; c < 4; ++c) rot[4 * i + c] = qp[c];
    }
  }

  // shapeMatchImplicit.ts:46-71
  void sm_center(Softbodies<T>& sb) {
    for (uint32_t i = sb.span.start; i < sb.span.start + sb.span.count; ++i) {
      const uint32_t s = sb.offsets[i], e = sb.offsets[i + 1], n = e - s;
      V3<T> sum = v3<T>(0, 0, 0);
      for (uint32_t k = s; k < e; ++k) sum = sum + p3(pred, sb.indices[k]);
      const T inv = static_cast<T>(1) / static_cast<T>(std::max(n, 1u));
      sb.centers[i] = n == 0 ? v3<T>(0, 0, 0) : sum * inv;
    }
  }
  // shapeMatchImplicit.ts:100-217
  void sm_moment_polar(Softbodies<T>& sb) {
    parallel_for(sb.span.start, static_cast<int64_t>(sb.span.start + sb.span.count), [&](int64_t ii) {
      const uint32_t i = static_cast<uint32_t>(ii);
      const uint32_t s = sb.offsets[i], e = sb.offsets[i + 1];
      T a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      const V3<T> c = sb.centers[i];
      const V3<T> cb = v3<T>(sb.restCenters[4 * i], sb.restCenters[4 * i + 1], sb.restCenters[4 * i + 2]);
      for (uint32_t k = s; k < e; ++k) {
        const uint32_t j = sb.indices[k];
        const T x = prot[4 * j], y = prot[4 * j + 1], z = prot[4 * j + 2], w = prot[4 * j + 3];
        const T xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z, wx = w * x,
                wy = w * y, wz = w * z;
        const T two = 2, one = 1;
        const T rj[9] = {one - (yy + zz) * two, (xy - wz) * two, (xz + wy) * two,
                         (xy + wz) * two, one - (xx + zz) * two, (yz - wx) * two,
                         (xz - wy) * two, (yz + wx) * two, one - (xx + yy) * two};
        for (int m = 0; m < 9; ++m) a[m] += sb.uAi * rj[m];
        const V3<T> xj = p3(pred, j) - c;
        const V3<T> xt = v3<T>(sb.restOffsets[4 * j], sb.restOffsets[4 * j + 1], sb.restOffsets[4 * j + 2]) - cb;
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
      T r[9];
      polar(a, r);
      if (e == s) {
        const T id[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        for (int m = 0; m < 9; ++m) r[m] = id[m];
      }
      for (int m = 0; m < 9; ++m) sb.rot9[9 * static_cast<size_t>(i) + m] = r[m];
    });
  }
  // shapeMatchImplicit.ts:248-308
  void sm_scatter(Softbodies<T>& sb) {
    parallel_for(sb.span.start, static_cast<int64_t>(sb.span.start + sb.span.count), [&](int64_t ii) {
      const uint32_t i = static_cast<uint32_t>(ii);
      const uint32_t s = sb.offsets[i], e = sb.offsets[i + 1];
      const T* R = &sb.rot9[9 * static_cast<size_t>(i)];
      const V3<T> R0 = v3(R[0], R[1], R[2]), R1 = v3(R[3], R[4], R[5]), R2 = v3(R[6], R[7], R[8]);
      const V3<T> c = sb.centers[i];
      const V3<T> cb = v3<T>(sb.restCenters[4 * i], sb.restCenters[4 * i + 1], sb.restCenters[4 * i + 2]);
      const T alphaTilde = static_cast<T>(sb.restOffsets[4 * i + 3]) / (dt * dt);
      for (uint32_t k = s; k < e; ++k) {
        const uint32_t j = sb.indices[k];
        const V3<T> rr = v3<T>(sb.restOffsets[4 * j], sb.restOffsets[4 * j + 1], sb.restOffsets[4 * j + 2]) - cb;
        const V3<T> goal = v3(dot(R0, rr), dot(R1, rr), dot(R2, rr)) + c;
        const V3<T> C = p3(pred, j) - goal;
        const T wj = invMass[j];
        const T denom = wj + alphaTilde;
        const V3<T> lo = sb.pairLambda[k];
        const V3<T> dl = (neg(C) - lo * alphaTilde) / denom;
        sb.pairLambda[k] = lo + dl;
        const T mj = tmax(static_cast<T>(sb.offsets[j + 1] - sb.offsets[j]), static_cast<T>(1));
        const V3<T> dx = (dl * wj) / mj;
        const T sc = std::sqrt(sb.uMaxC2 / tmax(dot(dx, dx), sb.uMaxC2));
        sb.acc.add(j, dx * sc);
      }
    });
  }
  // shapeMatchImplicit.ts:325-401
  void sm_qp_write(Softbodies<T>& sb) {
    for (uint32_t i = sb.span.start; i < sb.span.start + sb.span.count; ++i) {
      const uint32_t s = sb.offsets[i], e = sb.offsets[i + 1];
      const T* R = &sb.rot9[9 * static_cast<size_t>(i)];
      const T m00 = R[0], m01 = R[1], m02 = R[2], m10 = R[3], m11 = R[4], m12 = R[5], m20 = R[6],
              m21 = R[7], m22 = R[8];
      const T tr = m00 + m11 + m22;
      T qx = 0, qy = 0, qz = 0, qw = 1;
      if (tr > 0) {
        const T sq = static_cast<T>(0.5) / std::sqrt(tr + static_cast<T>(1));
        qw = static_cast<T>(0.25) / sq;
        qx = (m21 - m12) * sq;
        qy = (m02 - m20) * sq;
        qz = (m10 - m01) * sq;
      } else if (m00 > m11 && m00 > m22) {
        const T sq = static_cast<T>(2) * std::sqrt(static_cast<T>(1) + m00 - m11 - m22);
        qw = (m21 - m12) / sq;
        qx = static_cast<T>(0.25) * sq;
        qy = (m01 + m10) / sq;
        qz = (m02 + m20) / sq;
      } else if (m11 > m22) {
        const T sq = static_cast<T>(2) * std::sqrt(static_cast<T>(1) + m11 - m00 - m22);
        qw = (m02 - m20) / sq;
        qx = (m01 + m10) / sq;
        qy = static_cast<T>(0.25) * sq;
        qz = (m12 + m21) / sq;
      } else {
        const T sq = static_cast<T>(2) * std::sqrt(static_cast<T>(1) + m22 - m00 - m11);
        qw = (m10 - m01) / sq;
        qx = (m02 + m20) / sq;
        qy = (m12 + m21) / sq;
        qz = static_cast<T>(0.25) * sq;
      }
      const T d = rot[4 * i] * qx + rot[4 * i + 1] * qy + rot[4 * i + 2] * qz + rot[4 * i + 3] * qw;
      const T flip = d < 0 ? static_cast<T>(-1) : static_cast<T>(1);
      if (e > s) {
        prot[4 * i] = qx * flip;
        prot[4 * i + 1] = qy * flip;
        prot[4 * i + 2] = qz * flip;
        prot[4 * i + 3] = qw * flip;
      }
    }
  }

  // shapeMatch.ts:53-109 / 136-229: one 256-thread workgroup per body; the
  // per-thread strided partial sums and the tree reduction are kept in order.
  void body_frame(Softbodies<T>& sb) {
    const uint32_t W = 256;
    for (size_t b = 0; b < sb.bodies.size(); ++b) {
      const uint32_t start = sb.bodies[b].range.start, count = sb.bodies[b].range.count;
      std::vector<T> s4(4 * W, 0), r9(9 * W, 0);
      for (uint32_t tid = 0; tid < W; ++tid) {
        for (uint32_t li = tid; li < count; li += W) {
          const uint32_t g = start + li;
          const T mi = static_cast<T>(sb.weights[g]);
          const V3<T> xi = p3(pred, g);
          s4[4 * tid] += xi.x * mi;
          s4[4 * tid + 1] += xi.y * mi;
          s4[4 * tid + 2] += xi.z * mi;
          s4[4 * tid + 3] += mi;
          const V3<T> xw = xi * mi;
          const V3<T> ri = v3<T>(sb.restOffsets[4 * g], sb.restOffsets[4 * g + 1], sb.restOffsets[4 * g + 2]);
          const V3<T> a0 = ri * xw.x, a1 = ri * xw.y, a2 = ri * xw.z;
          T* r = &r9[9 * tid];
          r[0] += a0.x; r[1] += a0.y; r[2] += a0.z;
          r[3] += a1.x; r[4] += a1.y; r[5] += a1.z;
          r[6] += a2.x; r[7] += a2.y; r[8] += a2.z;
        }
      }
      for (uint32_t s = W >> 1; s > 0; s >>= 1)
        for (uint32_t tid = 0; tid < s; ++tid) {
          for (int c = 0; c < 4; ++c) s4[4 * tid + c] += s4[4 * (tid + s) + c];
          for (int c = 0; c < 9; ++c) r9[9 * tid + c] += r9[9 * (tid + s) + c];
        }
      sb.bodyCenters[b] = v3(s4[0], s4[1], s4[2]) / s4[3];
      T r[9];
      polar(&r9[0], r);
      for (int m = 0; m < 9; ++m) sb.bodyRot9[9 * b + m] = r[m];
    }
  }
  // shapeMatch.ts:277-351
  void global_delta_apply(Softbodies<T>& sb) {
    for (size_t b = 0; b < sb.bodies.size(); ++b) {
      const uint32_t start = sb.bodies[b].range.start, count = sb.bodies[b].range.count;
      const T* R = &sb.bodyRot9[9 * b];
      const V3<T> R0 = v3(R[0], R[1], R[2]), R1 = v3(R[3], R[4], R[5]), R2 = v3(R[6], R[7], R[8]);
      const V3<T> c = sb.bodyCenters[b];
      const T alphaTilde = static_cast<T>(sb.bodyCompliance[b]) / (dt * dt);
      for (uint32_t li = 0; li < count; ++li) {
        const uint32_t g = start + li;
        const V3<T> ri = v3<T>(sb.restOffsets[4 * g], sb.restOffsets[4 * g + 1], sb.restOffsets[4 * g + 2]);
        const V3<T> goal = v3(dot(R0, ri), dot(R1, ri), dot(R2, ri)) + c;
        const V3<T> xs = p3(pred, g);
        const V3<T> C = xs - goal;
        const V3<T> lo = sb.lambdaG[g];
        const T w = invMass[g];
        const V3<T> dl = (neg(C) - lo * alphaTilde) / (w + alphaTilde);
        sb.lambdaG[g] = lo + dl;
        set3(pred, g, xs + dl * w, 0);
      }
    }
  }

  // ----------------------------------------------------------- cloth ----
  // distance.ts:264-288
  void cloth_solve(Cloth<T>& cl) {
    for (const auto& grp : cl.groups) {
      for (uint32_t c : grp) {
        const uint32_t i = cl.pairs[2 * c], j = cl.pairs[2 * c + 1];
        const V3<T> xi = p3(pred, i), xj = p3(pred, j);
        const T wi = invMass[i], wj = invMass[j];
        const T wSum = wi + wj;
        const V3<T> off = xi - xj;
        const T len = length(off);
        if (wSum <= 0 || len < static_cast<T>(1e-12)) continue;
        const V3<T> n = off / len;
        const T lc = cl.lambda[c];
        const T alphaTilde = cl.compliance[c] / (dt * dt);
        const T dl = (-(len - cl.rest[c]) - alphaTilde * lc) / (wSum + alphaTilde);
        set3(pred, i, xi + n * (wi * dl), 0);
        set3(pred, j, xj - n * (wj * dl), 0);
        cl.lambda[c] = lc + dl;
      }
    }
    // bending.ts:130-235, after the stretch colours (ClothSystem.ts:193-212)
    for (const auto& grp : cl.bendGroups) {
      for (uint32_t c : grp) {
        const uint32_t* t = cl.bend.data() + 4 * static_cast<size_t>(c);
        const V3<T> x1 = p3(pred, t[0]), x2 = p3(pred, t[1]), x3 = p3(pred, t[2]), x4 = p3(pred, t[3]);
        const T w1 = invMass[t[0]], w2 = invMass[t[1]], w3 = invMass[t[2]], w4 = invMass[t[3]];
        const V3<T> E = x2 - x1;
        const T e2 = dot(E, E);
        if (e2 < static_cast<T>(1e-24)) continue;
        const T el = std::sqrt(e2);
        const V3<T> a3 = x3 - x1, b3 = x3 - x2, n1 = cross(a3, b3);
        const V3<T> a4 = x4 - x2, b4 = x4 - x1, n2 = cross(a4, b4);
        const T n1s = dot(n1, n1), n2s = dot(n2, n2);
        if (n1s < static_cast<T>(1e-24) || n2s < static_cast<T>(1e-24)) continue;
        const T theta = std::atan2(dot(cross(n1, n2), E), dot(n1, n2) * el);
        const T C = theta - cl.bendRest[c];
        const V3<T> N1 = n1 / n1s, N2 = n2 / n2s;
        const V3<T> g3 = neg(N1 * el), g4 = neg(N2 * el);
        const T c31 = dot(b3, E) / el, c32 = dot(a4, E) / el, c41 = dot(a3, E) / el, c42 = dot(b4, E) / el;
        const V3<T> g1 = neg(N1 * c31 + N2 * c32);
        const V3<T> g2 = N1 * c41 + N2 * c42;
        const T sg = dot(g1, g1) * w1 + dot(g2, g2) * w2 + dot(g3, g3) * w3 + dot(g4, g4) * w4;
        if (sg <= static_cast<T>(1e-30)) continue;
        const T lc = cl.bendLambda[c];
        const T at = cl.bendCompliance / (dt * dt);
        const T dl = (-C - at * lc) / (sg + at);
        set3(pred, t[0], x1 + g1 * (w1 * dl), 0);
        set3(pred, t[1], x2 + g2 * (w2 * dl), 0);
        set3(pred, t[2], x3 + g3 * (w3 * dl), 0);
        set3(pred, t[3], x4 + g4 * (w4 * dl), 0);
        cl.bendLambda[c] = lc + dl;
      }
    }
    // tether.ts:117-154, after the bending colours (ClothSystem.ts:213-224)
    for (const auto& grp : cl.tetherGroups) {
      for (uint32_t c : grp) {
        const uint32_t i = cl.tether[2 * c], a = cl.tether[2 * c + 1];
        const V3<T> x = p3(pred, i);
        const T w = invMass[i];
        if (w <= 0) continue;
        const V3<T> d = x - p3(pred, a);
        const T len = length(d);
        if (len <= cl.tetherRest[c]) {
          cl.tetherLambda[c] = 0;
          continue;
        }
        if (len < static_cast<T>(1e-12)) continue;
        const T lc = cl.tetherLambda[c];
        const T at = cl.tetherCompliance / (dt * dt);
        const T dl = (-(len - cl.tetherRest[c]) - at * lc) / (w + at);
        set3(pred, i, x + (d / len) * (w * dl), 0);
        cl.tetherLambda[c] = lc + dl;
      }
    }
  }

  // aero.ts:203-283: per cloth vertex, a third of the drag and lift of each
  // incident triangle from committed positions and velocities; the sum moves
  // the predicted position by dt^2 w F. Each vertex writes only its own slot.
  void cloth_aero(Cloth<T>& cl) {
    if (cl.tris.empty()) return;
    const V3<T> wind = v3<T>(cl.wind[0], cl.wind[1], cl.wind[2]);
    const T drag = cl.drag, lift = cl.lift, three = 3;
    for (uint32_t v = 0; v < cl.n; ++v) {
      const uint32_t i = cl.offset + v;
      const T w = invMass[i];
      if (w <= 0) continue;
      V3<T> f = v3<T>(0, 0, 0);
      for (uint32_t m = cl.incOff[v]; m < cl.incOff[v + 1]; ++m) {
        const uint32_t* t = cl.tris.data() + 3 * static_cast<size_t>(cl.incTri[m]);
        const V3<T> vrel = (p3(vel, t[0]) + p3(vel, t[1]) + p3(vel, t[2])) / three - wind;
        const T vrs = dot(vrel, vrel);
        if (!(vrs > static_cast<T>(1e-12))) continue;
        const V3<T> x1 = p3(pos, t[0]);
        const V3<T> nraw = cross(p3(pos, t[1]) - x1, p3(pos, t[2]) - x1);
        const T nms = dot(nraw, nraw);
        if (!(nms > static_cast<T>(1e-12))) continue;
        const T nm = std::sqrt(nms);
        const T area = nm * static_cast<T>(0.5);
        const V3<T> nunit = nraw / nm;
        const V3<T> nbar = nunit * (dot(nunit, vrel) < 0 ? static_cast<T>(-1) : static_cast<T>(1));
        const V3<T> vhat = vrel / std::sqrt(vrs);
        const V3<T> fdrag = neg(vhat * (drag * vrs * area * dot(nbar, vhat)));
        const V3<T> flift = cross(cross(nbar, vhat), vhat) * (lift * vrs * area);
        f = f + (fdrag + flift) / three;
      }
      set3(pred, i, p3(pred, i) + f * (dt * dt * w), 0);
    }
  }

  // ClothSystem.ts:249-287: blend each velocity toward the mean of the
  // particle's edge neighbours (mix(v, mean, damping)); pinned particles keep
  // theirs.
  void cloth_damping(Cloth<T>& cl) {
    if (!cl.hasDamping) return;
    const T t = cl.damping, one = 1;
    std::vector<V3<T>> sm(cl.n);
    for (uint32_t v = 0; v < cl.n; ++v) {
      V3<T> sum = v3<T>(0, 0, 0);
      const uint32_t m0 = cl.dampOff[v], m1 = cl.dampOff[v + 1];
      for (uint32_t m = m0; m < m1; ++m) sum = sum + p3(vel, cl.offset + cl.dampNbr[m]);
      const V3<T> mean = sum / static_cast<T>(std::max(m1 - m0, 1u));
      sm[v] = p3(vel, cl.offset + v) * (one - t) + mean * t;
    }
    for (uint32_t v = 0; v < cl.n; ++v) {
      const uint32_t i = cl.offset + v;
      if (invMass[i] > 0) set3(vel, i, sm[v], vel[4 * i + 3]);
    }
  }

  // ---------------------------------------------------------- contacts ----
  // f32 -> i32 toward zero, saturating (the shader's toInt()).
  static int32_t lam_ticks(T v) { return sat_i32(std::trunc(static_cast<double>(v * static_cast<T>(1048576)))); }
  static int32_t wrap_add(int32_t a, int32_t b) {
    return static_cast<int32_t>(static_cast<uint32_t>(a) + static_cast<uint32_t>(b));
  }

  // generate.ts:53-88: every particle outside the noSelfContacts ranges, in
  // index order, walks its 27 buckets; a pair of two emitters is kept by the
  // lower index. Pairs past maxContacts are counted, not stored.
  void contact_generate() {
    contacts.clear();
    contactCount = 0;
    for (uint32_t i = 0; i < cap; ++i) {
      if (quiet[i]) continue;
      const V3<T> xi = p3(pred, i);
      const uint32_t gi = group[i];
      const T wi = invMass[i];
      for_each_neighbor(xi, [&](uint32_t j, uint32_t) {
        if (j == i) return;
        if (!quiet[j] && j < i) return;
        if (gi != 0 && gi == group[j]) return;
        if (wi <= 0 && invMass[j] <= 0) return;
        const V3<T> d = xi - p3(pred, j);
        if (dot(d, d) >= cCand2) return;
        if (contactCount < maxContacts) contacts.push_back({i, j, 0, 0, v3<T>(0, 0, 0)});
        ++contactCount;
      });
    }
  }

  // solve.ts:115-150, then the accumulator applied to the committed and the
  // predicted positions (loop.ts:388-394).
  void contact_stabilize() {
    for (const Contact& c : contacts) {
      const V3<T> off = p3(pos, c.i) - p3(pos, c.j);
      const T d = length(off);
      const T wi = invMass[c.i], wj = invMass[c.j], ws = wi + wj;
      if (d <= static_cast<T>(1e-8) || d >= cDist || ws <= 0) continue;
      const V3<T> n = off / d;
      const T dl = (cDist - d) / ws;
      accPos.add(c.i, n * (wi * dl));
      accPos.add(c.j, neg(n * (wj * dl)));
    }
    for (uint32_t i = 0; i < cap; ++i) {
      const V3<T> ch = accPos.take(i, &accPos.flag);
      set3(pos, i, p3(pos, i) + ch, pos[4 * i + 3]);
      set3(pred, i, p3(pred, i) + ch, pred[4 * i + 3]);
    }
  }

  // solve.ts:34-104: non-penetration and static friction, scattered.
  void contact_solve() {
    const T inv = static_cast<T>(1) / static_cast<T>(1048576);
    for (Contact& c : contacts) {
      const V3<T> xi = p3(pred, c.i), xj = p3(pred, c.j);
      const V3<T> off = xi - xj;
      const T d = length(off);
      const T wi = invMass[c.i], wj = invMass[c.j], ws = wi + wj;
      if (d <= static_cast<T>(1e-8) || d >= cDist || ws <= 0) continue;
      const V3<T> n = off / d;
      const T dln = (cDist - d) / ws;
      c.ln = wrap_add(c.ln, lam_ticks(dln));
      c.n = n;
      const V3<T> slip = (xi - p3(pos, c.i)) - (xj - p3(pos, c.j));
      const V3<T> tang = slip - n * dot(slip, n);
      const T tl = length(tang);
      const T ln = static_cast<T>(c.ln) * inv, lt = static_cast<T>(c.lt) * inv;
      const T dlt = tl / ws;
      const bool sticks = tl > static_cast<T>(1e-10) && dlt <= cMuS * ln - lt;
      const V3<T> ni = n * (wi * dln), nj = neg(n * (wj * dln));
      accPos.add(c.i, sticks ? ni + neg(tang * (wi / ws)) : ni);
      accPos.add(c.j, sticks ? nj + tang * (wj / ws) : nj);
      c.lt = wrap_add(c.lt, lam_ticks(sticks ? dlt : static_cast<T>(0)));
    }
  }

  // solve.ts:158-189: kinetic friction on the velocities, scattered.
  void contact_friction() {
    const T inv = static_cast<T>(1) / static_cast<T>(1048576);
    for (const Contact& c : contacts) {
      const T wi = invMass[c.i], wj = invMass[c.j], ws = wi + wj;
      const T ln = static_cast<T>(c.ln) * inv;
      if (ws <= 0 || ln <= 0) continue;
      const V3<T> n = c.n;
      const V3<T> v = p3(vel, c.i) - p3(vel, c.j);
      const V3<T> vt = v - n * dot(n, v);
      const T vtl = length(vt);
      if (vtl < static_cast<T>(1e-6)) continue;
      const T change = tmin(cMuK * ln * ws / dt, vtl);
      const V3<T> imp = neg((vt / vtl) * change) / ws;
      accVel.add(c.i, imp * wi);
      accVel.add(c.j, neg(imp * wj));
    }
  }

  // --------------------------------------------------------- the loop ----
  void frame_start() {
    if (hasAcc()) {
      accPos.flag = 0;
      accVel.flag = 0;
    }
    if (hasColliders) clock = dt * (uSubsteps - static_cast<T>(1));
  }

  void substep() {
    predict();
    for (auto& sb : softs)
      if (sb.local) rotation_predict(sb);
    // preSolve
    if (hasAcc()) accPos.reset();
    if (hasGrid) rebuild_grid(pred);
    if (hasContact) {
      contact_generate();
      contact_stabilize();
    }
    if (hasColliders) {
      std::fill(primLambda.begin(), primLambda.end(), static_cast<T>(0));
      std::fill(sdfLambda.begin(), sdfLambda.end(), static_cast<T>(0));
    }
    for (auto& m : materials) {
      if (m.first == MAT_FLUID) {
        Fluid<T>& f = fluids[m.second];
        for (size_t b = 0; b < f.boundaries.size(); ++b)
          if (!f.boundaryStatic[b]) boundary_volume(f, f.boundaries[b], pred);
        build_neighbors(f);
        // FluidSystem.ts:233-255: impulses once per substep, before the solve
        if (f.hasSurfaceTension || f.hasAdhesion) {
          f.impulses.reset();
          if (f.hasSurfaceTension) {
            color_normal(f);
            surface_tension(f);
          }
          if (f.hasAdhesion) adhesion(f);
          for (uint32_t i = f.range.start; i < f.range.start + f.range.count; ++i) {
            const V3<T> c = f.impulses.take(i, &f.impulses.flag);
            set3(vel, i, p3(vel, i) + c, vel[4 * i + 3]);
            set3(pred, i, p3(pred, i) + c * dt, pred[4 * i + 3]);
          }
        }
        if (f.hasReaction) {
          f.reaction.reset();
          f.reaction.flag = 0;
        }
      } else if (m.first == MAT_SOFT) {
        Softbodies<T>& sb = softs[m.second];
        if (sb.local) {
          sb.acc.reset();
          sb.acc.flag = 0;
          std::fill(sb.pairLambda.begin(), sb.pairLambda.end(), v3<T>(0, 0, 0));
        } else {
          std::fill(sb.lambdaG.begin(), sb.lambdaG.end(), v3<T>(0, 0, 0));
        }
      } else {
        Cloth<T>& cl = cloths[m.second];
        std::fill(cl.lambda.begin(), cl.lambda.end(), static_cast<T>(0));
        std::fill(cl.bendLambda.begin(), cl.bendLambda.end(), static_cast<T>(0));
        std::fill(cl.tetherLambda.begin(), cl.tetherLambda.end(), static_cast<T>(0));
        // ClothSystem.ts:226-238: drag and lift after the multiplier resets
        cloth_aero(cl);
      }
    }
    for (uint32_t it = 0; it < iterations; ++it) {
      for (auto& m : materials) {
        if (m.first == MAT_FLUID) {
          Fluid<T>& f = fluids[m.second];
          fluid_lambda(f);
          fluid_delta(f);
          fluid_apply(f);
          if (f.hasReaction) fluid_reaction_apply(f);
        } else if (m.first == MAT_SOFT) {
          Softbodies<T>& sb = softs[m.second];
          if (sb.local) {
            sm_center(sb);
            sm_moment_polar(sb);
            sm_scatter(sb);
            apply_acc(sb.acc, pred, 0, cap);
            sm_qp_write(sb);
          } else {
            body_frame(sb);
            global_delta_apply(sb);
          }
        } else {
          cloth_solve(cloths[m.second]);
        }
      }
      if (hasAcc()) {
        if (hasContact) contact_solve();
        if (hasColliders) {
          collider_solve();
          sdf_solve();
        }
        apply_acc(accPos, pred, 0, cap);
      }
    }
    advect();
    for (auto& m : materials) {
      if (m.first == MAT_FLUID) {
        Fluid<T>& f = fluids[m.second];
        if (f.hasViscosity || f.hasVorticity) fluid_velocity(f);
      } else if (m.first == MAT_SOFT) {
        Softbodies<T>& sb = softs[m.second];
        if (sb.local) {
          rotation_advect(sb);
          body_frame(sb);
        }
      } else {
        cloth_damping(cloths[m.second]);
      }
    }
    if (hasAcc()) {
      accVel.reset();
      if (hasContact) contact_friction();
      if (hasColliders) {
        collider_friction();
        sdf_friction();
      }
      apply_acc(accVel, vel, 0, cap);
    }
    if (hasColliders) clock = tmax(clock - dt, static_cast<T>(0));
  }

  void init_pass() {
    // Static boundaries: their volume is computed once from committed
    // positions after a grid rebuild (FluidSystem.ts:228-231, loop.ts:237).
    bool any = false;
    for (auto& f : fluids)
      for (size_t b = 0; b < f.boundaries.size(); ++b) any = any || f.boundaryStatic[b];
    if (!any) return;
    if (hasGrid) rebuild_grid(pred);
    for (auto& f : fluids)
      for (size_t b = 0; b < f.boundaries.size(); ++b)
        if (f.boundaryStatic[b]) boundary_volume(f, f.boundaries[b], pos);
  }

  void step(double frameDt) {
    dt = static_cast<T>(frameDt / substeps);
    if (!initialized) {
      init_pass();
      initialized = true;
    }
    frame_start();
    for (uint32_t s = 0; s < substeps; ++s) substep();
  }
};

// ---------------------------------------------------- scene wrapper ----

struct Scene {
  int precision = 32;
  std::unique_ptr<Engine<float>> f32;
  std::unique_ptr<Engine<double>> f64;
  template <typename F>
  void visit(F&& fn) {
    if (f32)
      fn(*f32);
    else
      fn(*f64);
  }
};

template <typename T>
void engine_init(Engine<T>& e, uint32_t cap, double radius) {
  e.cap = cap;
  e.radius = radius;
  e.pos.assign(4 * static_cast<size_t>(cap), 0);
  e.pred.assign(4 * static_cast<size_t>(cap), 0);
  e.vel.assign(4 * static_cast<size_t>(cap), 0);
  e.rot.assign(4 * static_cast<size_t>(cap), 0);
  e.prot.assign(4 * static_cast<size_t>(cap), 0);
  e.angv.assign(4 * static_cast<size_t>(cap), 0);
  for (uint32_t i = 0; i < cap; ++i) e.rot[4 * i + 3] = e.prot[4 * i + 3] = 1;
  e.invMass.assign(cap, 0);
  e.bvol.assign(cap, 0);
  e.group.assign(cap, 0);
}

bool range_ok(uint32_t cap, pf_range r) {
  return r.count > 0 && static_cast<uint64_t>(r.start) + r.count <= cap;
}

uint32_t next_pow2(uint64_t n) {
  if (n <= 1) return 1;
  uint64_t p = 1;
  while (p < n) p <<= 1;
  return static_cast<uint32_t>(p);
}

// Greedy colouring in constraint order (types.ts:95-150).
std::vector<std::vector<uint32_t>> color_constraints(const std::vector<uint32_t>& pairs, uint32_t n,
                                                     int arity = 2) {
  std::vector<uint32_t> groupOf(n);
  std::vector<std::vector<uint32_t>> particleGroups;
  uint32_t maxP = 0;
  for (uint32_t v : pairs) maxP = std::max(maxP, v);
  particleGroups.resize(static_cast<size_t>(maxP) + 1);
  uint32_t numGroups = 0;
  for (uint32_t c = 0; c < n; ++c) {
    uint32_t g = 0;
    for (;;) {
      bool conflict = false;
      for (int k = 0; k < arity && !conflict; ++k) {
        const auto& owned = particleGroups[pairs[static_cast<size_t>(arity) * c + k]];
        conflict = std::find(owned.begin(), owned.end(), g) != owned.end();
      }
      if (!conflict) break;
      ++g;
    }
    groupOf[c] = g;
    numGroups = std::max(numGroups, g + 1);
    for (int k = 0; k < arity; ++k) {
      auto& owned = particleGroups[pairs[static_cast<size_t>(arity) * c + k]];
      if (std::find(owned.begin(), owned.end(), g) == owned.end()) owned.push_back(g);
    }
  }
  std::vector<std::vector<uint32_t>> groups(numGroups);
  for (uint32_t c = 0; c < n; ++c) groups[groupOf[c]].push_back(c);
  return groups;
}

}  // namespace

// ================================================================ C API ===

extern "C" {

const char* or_last_error(void) { return g_err.c_str(); }

uint32_t or_part1by2(uint32_t n) { return part1by2(n); }
uint32_t or_morton(int32_t cx, int32_t cy, int32_t cz) { return morton_unmasked(cx, cy, cz); }

void or_set_threads(int n) { g_threads = n > 0 ? n : 1; }

int or_max_threads(void) { return g_threads; }
int or_hardware_threads(void) { return static_cast<int>(std::thread::hardware_concurrency()); }

uint64_t or_grid_cells(const pf_grid_desc* g) { return g ? grid_cells(*g) : 0; }

// Stable counting sort (the oracle of pf_sort). Host arrays.
int or_sort(const float* pos4, uint32_t n, const pf_grid_desc* g, uint32_t* keys, uint32_t* perm,
            uint32_t* start, uint32_t* count, uint32_t* overflow) {
  if (!g || !grid_cells(*g)) return fail(PF_ERR_INVALID, "HashGrid: invalid grid descriptor");
  if (!(g->cell_size > 0) || !std::isfinite(g->cell_size))
    return fail(PF_ERR_INVALID, "HashGrid: cellSize must be a positive finite number");
  std::vector<uint32_t> k(n);
  stable_count_sort<float>(*g, n, pos4, keys ? keys : k.data(), perm, start, count, overflow);
  return PF_OK;
}

// 27-cell candidate walk of query.ts for one query point over a grid built by
// or_sort with a Morton descriptor; writes the particle indices visited.
int or_walk(const float* query3, const pf_grid_desc* g, const uint32_t* perm, const uint32_t* start,
            const uint32_t* count, uint32_t* out, uint32_t cap_out, uint32_t* n_out) {
  Engine<float> e;
  e.grid = *g;
  const uint64_t C = grid_cells(*g);
  e.cellStart.assign(start, start + C);
  e.counts.assign(count, count + C);
  uint32_t maxSlot = 0;
  for (uint64_t c = 0; c < C; ++c) maxSlot = std::max(maxSlot, start[c] + count[c]);
  e.sorted.assign(perm, perm + maxSlot);
  uint32_t n = 0;
  e.for_each_neighbor(v3(query3[0], query3[1], query3[2]), [&](uint32_t j, uint32_t) {
    if (n < cap_out) out[n] = j;
    ++n;
  });
  *n_out = n;
  return PF_OK;
}

// 3x3 polar decomposition (polarDecomp.ts), row-major in and out.
void or_polar(const float* a, float* r) {
  float rr[9];
  Engine<float>::polar(a, rr);
  std::memcpy(r, rr, sizeof(rr));
}
void or_polar_f64(const double* a, double* r) { Engine<double>::polar(a, r); }

// Greedy colouring: groupOf per constraint, returns the number of groups.
uint32_t or_color_constraints(const uint32_t* pairs, uint32_t n, uint32_t* group_of) {
  std::vector<uint32_t> p(pairs, pairs + 2 * static_cast<size_t>(n));
  auto groups = color_constraints(p, n);
  for (uint32_t g = 0; g < groups.size(); ++g)
    for (uint32_t c : groups[g]) group_of[c] = g;
  return static_cast<uint32_t>(groups.size());
}

void* or_scene_create(const pf_scene_desc* d, int precision) {
  if (!d || d->capacity == 0 || !(d->particle_radius > 0)) {
    fail(PF_ERR_INVALID, "ParticleSystem: capacity must be a positive integer");
    return nullptr;
  }
  Scene* s = new Scene;
  s->precision = precision;
  if (precision == 64) {
    s->f64.reset(new Engine<double>);
    engine_init(*s->f64, d->capacity, d->particle_radius);
  } else {
    s->f32.reset(new Engine<float>);
    engine_init(*s->f32, d->capacity, d->particle_radius);
  }
  return s;
}

void or_scene_destroy(void* h) { delete static_cast<Scene*>(h); }

int or_upload_particles(void* h, const float* pos4, const float* vel4, const float* inv_mass,
                        const uint32_t* group, uint32_t start, uint32_t n) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    if (static_cast<uint64_t>(start) + n > e.cap) {
      rc = fail(PF_ERR_INVALID, "ParticleSystem.uploadParticles: invalid particle range");
      return;
    }
    for (uint32_t k = 0; k < n; ++k) {
      const uint32_t i = start + k;
      for (int c = 0; c < 3; ++c) {
        e.pos[4 * i + c] = pos4[4 * k + c];
        e.pred[4 * i + c] = pos4[4 * k + c];
        e.vel[4 * i + c] = vel4 ? vel4[4 * k + c] : 0;
      }
      e.pos[4 * i + 3] = e.pred[4 * i + 3] = e.vel[4 * i + 3] = 0;
      e.invMass[i] = inv_mass ? inv_mass[k] : 1.0f;
      e.group[i] = group ? group[k] : 0;
    }
  });
  return rc;
}

int or_set_inv_mass(void* h, pf_range r, float w) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    if (!range_ok(e.cap, r)) {
      rc = fail(PF_ERR_INVALID, "ParticleSystem.setInvMass: invalid particle range");
      return;
    }
    for (uint32_t i = r.start; i < r.start + r.count; ++i) e.invMass[i] = w;
  });
  return rc;
}

int or_add_fluid(void* h, const pf_fluid_desc* d, uint32_t* mat) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    using T = typename std::remove_reference<decltype(e.pos[0])>::type;
    Fluid<T> f;
    f.range.start = d->range.count ? d->range.start : 0;
    f.range.count = d->range.count ? d->range.count : e.cap;
    if (!range_ok(e.cap, {f.range.start, f.range.count})) {
      rc = fail(PF_ERR_INVALID, "FluidSystem: invalid particle range");
      return;
    }
    // FluidSystem.ts:96-118
    f.restDensity = d->rest_density > 0 ? d->rest_density : 1000.0;
    f.spacing = d->particle_spacing > 0 ? d->particle_spacing : 2.0 * e.radius;
    f.h = d->smoothing_radius > 0 ? d->smoothing_radius : 2.0 * f.spacing;
    f.compliance = d->compliance >= 0 ? d->compliance : 1e-4;
    f.hasViscosity = (d->flags & PF_FLUID_VISCOSITY) != 0;
    f.viscosity = d->viscosity;
    f.hasVorticity = (d->flags & PF_FLUID_VORTICITY) != 0;
    f.vorticity = d->vorticity;
    f.hasSurfaceTension = (d->flags & PF_FLUID_SURFACE_TENSION) != 0;
    f.surfaceTension = d->surface_tension;
    f.hasAdhesion = (d->flags & PF_FLUID_ADHESION) != 0;
    f.adhesion = d->adhesion;
    const double mass = f.restDensity * f.spacing * f.spacing * f.spacing;
    for (uint32_t b = 0; b < d->n_boundaries; ++b) {
      f.boundaries.push_back({d->boundaries[b].start, d->boundaries[b].count});
      f.boundaryStatic.push_back(d->boundary_static ? d->boundary_static[b] : 0);
    }
    // Uniforms: JS doubles stored as f32 uniforms (sph/kernels.ts:221-225,
    // FluidSystem.ts:200-213); the FP64 engine keeps them in double.
    const bool dbl = sizeof(T) == 8;
    auto U = [&](double v) { return dbl ? static_cast<T>(v) : static_cast<T>(static_cast<float>(v)); };
    f.uRho0 = U(f.restDensity);
    f.uVolume = U(f.spacing * f.spacing * f.spacing);
    f.uMass = U(mass);
    f.uH = U(f.h);
    f.uHSq = U(f.h * f.h);
    f.uPoly6 = U(315.0 / (64.0 * M_PI * std::pow(f.h, 9)));
    f.uSpiky = U(45.0 / (M_PI * std::pow(f.h, 6)));
    f.uCompliance = U(f.compliance);
    f.uC = U(f.viscosity);
    f.uEps = U(f.vorticity);
    f.uGamma = U(f.surfaceTension);
    f.uBeta = U(f.adhesion);
    // particles.setInvMass(range, 1 / mass) into a Float32Array.
    const float w = static_cast<float>(1.0 / mass);
    for (uint32_t i = f.range.start; i < f.range.start + f.range.count; ++i) e.invMass[i] = w;
    f.density.assign(e.cap, 0);
    for (uint32_t i = f.range.start; i < f.range.start + f.range.count; ++i)
      f.density[i] = U(f.restDensity);
    f.lambda.assign(e.cap, 0);
    f.deltaX.assign(e.cap, v3<T>(0, 0, 0));
    f.deltaV.assign(e.cap, v3<T>(0, 0, 0));
    f.omega.assign(e.cap, v3<T>(0, 0, 0));
    f.eta.assign(e.cap, v3<T>(0, 0, 0));
    f.omegaLength.assign(e.cap, 0);
    f.normal.assign(e.cap, v3<T>(0, 0, 0));
    f.impulses.init(e.cap, 50.0);
    f.nbrIdx.assign(static_cast<size_t>(f.range.count) * kMaxNeighbors, 0);
    f.nbrCount.assign(f.range.count, 0);
    f.hasReaction = !f.boundaries.empty();
    if (f.hasReaction) f.reaction.init(e.cap, 10.0);
    e.fluids.push_back(std::move(f));
    e.materials.push_back({MAT_FLUID, static_cast<int>(e.fluids.size() - 1)});
    if (mat) *mat = static_cast<uint32_t>(e.materials.size() - 1);
  });
  return rc;
}

int or_add_softbodies(void* h, const pf_softbody_desc* d, uint32_t* mat) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    using T = typename std::remove_reference<decltype(e.pos[0])>::type;
    const bool dbl = sizeof(T) == 8;
    auto U = [&](double v) { return dbl ? static_cast<T>(v) : static_cast<T>(static_cast<float>(v)); };
    if (d->n_bodies == 0) {
      rc = fail(PF_ERR_INVALID, "SoftbodySystem: at least one body is required");
      return;
    }
    Softbodies<T> sb;
    sb.local = d->shape_matching == PF_SHAPE_MATCH_LOCAL;
    sb.selfCollision = d->self_collision != 0;
    sb.restOffsets.assign(4 * static_cast<size_t>(e.cap), 0.0f);
    sb.weights.assign(e.cap, 0.0f);
    sb.bodyCompliance.assign(d->n_bodies, 0.0f);
    uint32_t spanStart = UINT32_MAX, spanEnd = 0;
    for (uint32_t b = 0; b < d->n_bodies; ++b) {
      const pf_softbody_def& def = d->bodies[b];
      if (!range_ok(e.cap, def.range)) {
        rc = fail(PF_ERR_INVALID, "SoftbodySystem body: invalid particle range");
        return;
      }
      Body<T> body;
      body.range = {def.range.start, def.range.count};
      body.surfaceCount = def.surface_count == UINT32_MAX ? def.range.count : def.surface_count;
      body.compliance = def.compliance;
      body.edges.assign(def.edges, def.edges + 2 * static_cast<size_t>(def.n_edges));
      body.restPositions.resize(3 * static_cast<size_t>(def.range.count));
      for (uint32_t k = 0; k < def.range.count; ++k)
        for (int c = 0; c < 3; ++c)
          body.restPositions[3 * k + c] =
              def.rest_positions ? def.rest_positions[3 * k + c]
                                 : static_cast<float>(e.pos[4 * (def.range.start + k) + c]);
      // massWeights (SoftbodySystem.ts:366-372)
      std::vector<double> masses(def.range.count);
      std::vector<double> dyn;
      for (uint32_t k = 0; k < def.range.count; ++k) {
        const double w = static_cast<float>(e.invMass[def.range.start + k]);
        masses[k] = w > 0 ? 1.0 / w : 0.0;
        if (masses[k] > 0) dyn.push_back(masses[k]);
      }
      bool allEq = true;
      for (double m : dyn) allEq = allEq && m == dyn[0];
      std::vector<float> bw(def.range.count, 1.0f);
      if (!allEq) {
        double mean = 0;
        for (double m : dyn) mean += m;
        mean /= dyn.size();
        for (uint32_t k = 0; k < def.range.count; ++k)
          bw[k] = static_cast<float>(masses[k] > 0 ? masses[k] / mean : 1.0);
      }
      double cx = 0, cy = 0, cz = 0, tot = 0;
      for (uint32_t k = 0; k < def.range.count; ++k) {
        cx += static_cast<double>(body.restPositions[3 * k]) * bw[k];
        cy += static_cast<double>(body.restPositions[3 * k + 1]) * bw[k];
        cz += static_cast<double>(body.restPositions[3 * k + 2]) * bw[k];
        tot += bw[k];
      }
      cx /= tot;
      cy /= tot;
      cz /= tot;
      for (uint32_t k = 0; k < def.range.count; ++k) {
        const uint32_t i = def.range.start + k;
        sb.weights[i] = bw[k];
        sb.restOffsets[4 * i] = static_cast<float>(body.restPositions[3 * k] - cx);
        sb.restOffsets[4 * i + 1] = static_cast<float>(body.restPositions[3 * k + 1] - cy);
        sb.restOffsets[4 * i + 2] = static_cast<float>(body.restPositions[3 * k + 2] - cz);
        sb.restOffsets[4 * i + 3] = static_cast<float>(def.compliance);
      }
      sb.bodyCompliance[b] = static_cast<float>(def.compliance);
      spanStart = std::min(spanStart, def.range.start);
      spanEnd = std::max(spanEnd, def.range.start + def.range.count);
      sb.bodies.push_back(std::move(body));
    }
    sb.span = {spanStart, spanEnd - spanStart};
    sb.centers.assign(e.cap, v3<T>(0, 0, 0));
    sb.rot9.assign(9 * static_cast<size_t>(e.cap), 0);
    sb.bodyCenters.assign(d->n_bodies, v3<T>(0, 0, 0));
    sb.bodyRot9.assign(9 * static_cast<size_t>(d->n_bodies), 0);
    for (uint32_t b = 0; b < d->n_bodies; ++b) sb.bodyRot9[9 * b] = sb.bodyRot9[9 * b + 4] = sb.bodyRot9[9 * b + 8] = 1;
    sb.lambdaG.assign(e.cap, v3<T>(0, 0, 0));
    if (sb.local) {
      // buildNeighborGraph (SoftbodySystem.ts:489-514)
      std::vector<uint32_t> degree(e.cap, 0);
      for (auto& body : sb.bodies) {
        for (uint32_t k = 0; k < body.range.count; ++k) degree[body.range.start + k] += 1;
        for (size_t q = 0; q < body.edges.size(); q += 2) {
          degree[body.range.start + body.edges[q]] += 1;
          degree[body.range.start + body.edges[q + 1]] += 1;
        }
      }
      sb.offsets.assign(static_cast<size_t>(e.cap) + 1, 0);
      for (uint32_t i = 0; i < e.cap; ++i) sb.offsets[i + 1] = sb.offsets[i] + degree[i];
      sb.indices.assign(std::max<uint32_t>(1, sb.offsets[e.cap]), 0);
      std::vector<uint32_t> cursor(sb.offsets.begin(), sb.offsets.begin() + e.cap);
      for (auto& body : sb.bodies) {
        for (uint32_t i = body.range.start; i < body.range.start + body.range.count; ++i)
          sb.indices[cursor[i]++] = i;
        for (size_t q = 0; q < body.edges.size(); q += 2) {
          const uint32_t i = body.range.start + body.edges[q], j = body.range.start + body.edges[q + 1];
          sb.indices[cursor[i]++] = j;
          sb.indices[cursor[j]++] = i;
        }
      }
      // restCenters accumulated into a Float32Array (SoftbodySystem.ts:283-295)
      sb.restCenters.assign(4 * static_cast<size_t>(e.cap), 0.0f);
      for (auto& body : sb.bodies)
        for (uint32_t i = body.range.start; i < body.range.start + body.range.count; ++i) {
          const uint32_t from = sb.offsets[i], to = sb.offsets[i + 1];
          for (uint32_t k = from; k < to; ++k) {
            const uint32_t j = sb.indices[k];
            for (int a = 0; a < 3; ++a)
              sb.restCenters[4 * i + a] = static_cast<float>(
                  static_cast<double>(sb.restCenters[4 * i + a]) +
                  static_cast<double>(sb.restOffsets[4 * j + a]) / static_cast<double>(to - from));
          }
        }
      sb.pairLambda.assign(sb.indices.size(), v3<T>(0, 0, 0));
      sb.acc.init(e.cap, 10.0);
      sb.uAi = U(e.radius * e.radius / 5.0);
      const double maxC = 5.0 * e.radius;
      sb.uMaxC = U(maxC);
      sb.uMaxC2 = U(maxC * maxC);
    }
    e.softs.push_back(std::move(sb));
    e.materials.push_back({MAT_SOFT, static_cast<int>(e.softs.size() - 1)});
    if (mat) *mat = static_cast<uint32_t>(e.materials.size() - 1);
  });
  return rc;
}

int or_add_cloth(void* h, const pf_cloth_desc* d, uint32_t* mat) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    using T = typename std::remove_reference<decltype(e.pos[0])>::type;
    if (!range_ok(e.cap, {d->offset, d->n_particles})) {
      rc = fail(PF_ERR_INVALID, "ClothSystem: invalid particle range");
      return;
    }
    // ClothSystem.ts:131-140: upload graph positions and masses, velocity 0.
    for (uint32_t k = 0; k < d->n_particles; ++k) {
      const uint32_t i = d->offset + k;
      for (int c = 0; c < 3; ++c) {
        e.pos[4 * i + c] = d->positions[3 * k + c];
        e.pred[4 * i + c] = d->positions[3 * k + c];
        e.vel[4 * i + c] = 0;
      }
      e.pos[4 * i + 3] = e.pred[4 * i + 3] = e.vel[4 * i + 3] = 0;
      e.invMass[i] = d->inv_mass[k];
    }
    Cloth<T> cl;
    cl.offset = d->offset;
    cl.n = d->n_particles;
    cl.pairs.resize(2 * static_cast<size_t>(d->n_pairs));
    for (size_t q = 0; q < cl.pairs.size(); ++q) cl.pairs[q] = d->offset + d->pairs[q];
    const double comp = d->stretch_compliance >= 0 ? d->stretch_compliance : 1e-7;
    cl.rest.resize(d->n_pairs);
    cl.compliance.assign(d->n_pairs, static_cast<T>(static_cast<float>(comp)));
    for (uint32_t c = 0; c < d->n_pairs; ++c) cl.rest[c] = d->rest_lengths[c];
    cl.lambda.assign(d->n_pairs, 0);
    cl.groups = color_constraints(cl.pairs, d->n_pairs);
    if (d->n_bending) {
      const double bc = d->bend_compliance >= 0 ? d->bend_compliance : 1e-5;
      cl.bend.resize(4 * static_cast<size_t>(d->n_bending));
      for (size_t q = 0; q < cl.bend.size(); ++q) cl.bend[q] = d->offset + d->bending[q];
      cl.bendRest.resize(d->n_bending);
      for (uint32_t c = 0; c < d->n_bending; ++c) cl.bendRest[c] = d->bending_rest[c];
      cl.bendLambda.assign(d->n_bending, 0);
      cl.bendCompliance = static_cast<T>(static_cast<float>(bc));
      cl.bendGroups = color_constraints(cl.bend, d->n_bending, 4);
    }
    if (d->n_tethers) {
      // tether.ts:100-110: one compliance, colours of arity 1 on the particle
      cl.tether.resize(2 * static_cast<size_t>(d->n_tethers));
      std::vector<uint32_t> who(d->n_tethers);
      for (uint32_t c = 0; c < d->n_tethers; ++c) {
        cl.tether[2 * c] = who[c] = d->offset + d->tether_particle[c];
        cl.tether[2 * c + 1] = d->offset + d->tether_anchor[c];
      }
      cl.tetherRest.resize(d->n_tethers);
      for (uint32_t c = 0; c < d->n_tethers; ++c) cl.tetherRest[c] = d->tether_rest[c];
      cl.tetherLambda.assign(d->n_tethers, 0);
      const double tc = d->tether_compliance >= 0 ? d->tether_compliance : 0.0;
      cl.tetherCompliance = static_cast<T>(static_cast<float>(tc));
      cl.tetherGroups = color_constraints(who, d->n_tethers, 1);
    }
    if (d->n_triangles) {
      // aero.ts:160-183: incidence CSR in triangle order
      cl.tris.resize(3 * static_cast<size_t>(d->n_triangles));
      cl.incOff.assign(d->n_particles + 1, 0);
      for (size_t q = 0; q < cl.tris.size(); ++q) {
        cl.tris[q] = d->offset + d->triangles[q];
        ++cl.incOff[d->triangles[q] + 1];
      }
      for (uint32_t v = 0; v < d->n_particles; ++v) cl.incOff[v + 1] += cl.incOff[v];
      cl.incTri.resize(cl.incOff.back());
      std::vector<uint32_t> cur(cl.incOff.begin(), cl.incOff.end() - 1);
      for (uint32_t t = 0; t < d->n_triangles; ++t)
        for (int k = 0; k < 3; ++k) cl.incTri[cur[d->triangles[3 * t + k]]++] = t;
    }
    for (int a = 0; a < 3; ++a) cl.wind[a] = d->wind[a];
    cl.drag = d->drag >= 0 ? d->drag : 0.6125f;
    cl.lift = d->lift >= 0 ? d->lift : 0.3f;
    if (d->has_damping) {
      // ClothSystem.ts:252-263: neighbours in pair order, both directions
      cl.hasDamping = true;
      cl.damping = d->damping;
      cl.dampOff.assign(d->n_particles + 1, 0);
      for (uint32_t q = 0; q < 2 * d->n_pairs; ++q) ++cl.dampOff[d->pairs[q] + 1];
      for (uint32_t v = 0; v < d->n_particles; ++v) cl.dampOff[v + 1] += cl.dampOff[v];
      cl.dampNbr.resize(cl.dampOff.back());
      std::vector<uint32_t> cur(cl.dampOff.begin(), cl.dampOff.end() - 1);
      for (uint32_t q = 0; q < d->n_pairs; ++q) {
        const uint32_t i = d->pairs[2 * q], j = d->pairs[2 * q + 1];
        cl.dampNbr[cur[i]++] = j;
        cl.dampNbr[cur[j]++] = i;
      }
    }
    e.cloths.push_back(std::move(cl));
    e.materials.push_back({MAT_CLOTH, static_cast<int>(e.cloths.size() - 1)});
    if (mat) *mat = static_cast<uint32_t>(e.materials.size() - 1);
  });
  return rc;
}

// ClothSystem.wind / drag / lift / damping / bendCompliance setters
// (ClothSystem.ts:143-188).
int or_cloth_set_params(void* h, uint32_t mat, const pf_cloth_params* p) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    using T = typename std::remove_reference<decltype(e.pos[0])>::type;
    if (mat >= e.materials.size() || e.materials[mat].first != MAT_CLOTH) {
      rc = fail(PF_ERR_INVALID, "ClothSystem: material is not a cloth");
      return;
    }
    auto& cl = e.cloths[e.materials[mat].second];
    for (int a = 0; a < 3; ++a) cl.wind[a] = p->wind[a];
    cl.drag = p->drag;
    cl.lift = p->lift;
    cl.damping = p->damping;
    cl.bendCompliance = static_cast<T>(p->bend_compliance);
  });
  return rc;
}

int or_add_primitive(void* h, const pf_primitive* p, uint32_t* slot) {
  Scene* s = static_cast<Scene*>(h);
  s->visit([&](auto& e) {
    Prim q;
    std::memcpy(&q, p, sizeof(q));
    e.prims.push_back(q);
    if (slot) *slot = static_cast<uint32_t>(e.prims.size() - 1);
  });
  return PF_OK;
}

int or_set_primitive(void* h, uint32_t slot, const pf_primitive* p) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    if (slot >= e.prims.size()) {
      rc = fail(PF_ERR_INVALID, "PrimitiveSet: no primitive in slot");
      return;
    }
    std::memcpy(&e.prims[slot], p, sizeof(Prim));
  });
  return rc;
}

int or_add_sdf_collider(void* h, const pf_sdf_desc* d, uint32_t* slot) {
  Scene* s = static_cast<Scene*>(h);
  if (!d || !d->data) return fail(PF_ERR_INVALID, "SDFCollider: no distance data");
  s->visit([&](auto& e) {
    SdfGrid g;
    const size_t n = static_cast<size_t>(d->res[0]) * d->res[1] * d->res[2];
    for (int a = 0; a < 3; ++a) {
      g.res[a] = d->res[a];
      g.origin[a] = d->origin[a];
      g.voxel[a] = d->voxel_size[a];
      g.invVoxel[a] = static_cast<float>(1.0 / static_cast<double>(d->voxel_size[a]));
    }
    g.phi.resize(n);
    for (size_t i = 0; i < n; ++i) g.phi[i] = half_round(d->data[i]);
    g.thickness = d->thickness;
    g.muS = d->mu_s;
    g.muK = d->mu_k;
    sdf_set_transform(g, d->position, d->rotation, d->scale);
    e.sdfs.push_back(std::move(g));
    if (slot) *slot = static_cast<uint32_t>(e.sdfs.size() - 1);
  });
  return PF_OK;
}

int or_set_sdf_transform(void* h, uint32_t slot, const float* pos, const float* rot, float scale) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    if (slot >= e.sdfs.size()) {
      rc = fail(PF_ERR_INVALID, "SDFCollider: no collider in slot");
      return;
    }
    sdf_set_transform(e.sdfs[slot], pos, rot, scale);
  });
  return rc;
}

// SDF sample at points (tests): phi and the world gradient per point.
int or_sdf_sample(const pf_sdf_desc* d, const float* pts, uint32_t n, float* phi, float* grad) {
  SdfGrid g;
  const size_t nv = static_cast<size_t>(d->res[0]) * d->res[1] * d->res[2];
  for (int a = 0; a < 3; ++a) {
    g.res[a] = d->res[a];
    g.origin[a] = d->origin[a];
    g.voxel[a] = d->voxel_size[a];
    g.invVoxel[a] = static_cast<float>(1.0 / static_cast<double>(d->voxel_size[a]));
  }
  g.phi.resize(nv);
  for (size_t i = 0; i < nv; ++i) g.phi[i] = half_round(d->data[i]);
  g.thickness = d->thickness;
  sdf_set_transform(g, d->position, d->rotation, d->scale);
  for (uint32_t i = 0; i < n; ++i) {
    float p;
    V3<float> gr;
    Engine<float>::sdf_sample(g, v3<float>(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), &p, &gr);
    phi[i] = p;
    grad[3 * i] = gr.x;
    grad[3 * i + 1] = gr.y;
    grad[3 * i + 2] = gr.z;
  }
  return PF_OK;
}

int or_loop_build(void* h, const pf_loop_desc* d, uint32_t table_size) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    using T = typename std::remove_reference<decltype(e.pos[0])>::type;
    e.substeps = d->substeps ? d->substeps : 4;
    e.iterations = d->iterations;
    e.gx = static_cast<T>(d->gravity[0]);
    e.gy = static_cast<T>(d->gravity[1]);
    e.gz = static_cast<T>(d->gravity[2]);
    e.uSubsteps = static_cast<T>(e.substeps);
    // loop.ts:148-160: one grid, cells sized for the widest query
    e.hasContact = d->contact != 0;
    double nr = e.hasContact ? 2.0 * e.radius * 1.1 : 0.0;
    for (auto& f : e.fluids) nr = std::max(nr, f.h);
    e.hasGrid = nr > 0;
    if (e.hasContact) {
      const double cr = 2.0 * e.radius * 1.1;
      e.cMuS = static_cast<T>(d->contact_mu_s >= 0 ? d->contact_mu_s : 0.5f);
      e.cMuK = static_cast<T>(d->contact_mu_k >= 0 ? d->contact_mu_k : 0.4f);
      e.cDist = static_cast<T>(static_cast<float>(2.0 * e.radius));
      e.cCand2 = static_cast<T>(static_cast<float>(cr * cr));
      e.maxContacts = d->max_contacts ? d->max_contacts : static_cast<uint32_t>(8ull * e.cap);
      e.quiet.assign(e.cap, 0);
      for (auto& f : e.fluids)
        for (uint32_t i = f.range.start; i < f.range.start + f.range.count; ++i) e.quiet[i] = 1;
      for (auto& q : e.quietRanges)
        for (uint32_t i = q.start; i < q.start + q.count; ++i) e.quiet[i] = 1;
    }
    // loop.ts:163-166, SoftbodySystem.ts:218-234: collision groups for the
    // soft bodies that have none, above every uploaded group
    {
      uint32_t next = 1;
      for (uint32_t g : e.group) next = std::max(next, g + 1);
      for (auto& m : e.materials) {
        if (m.first != MAT_SOFT || e.softs[m.second].selfCollision) continue;
        for (auto& b : e.softs[m.second].bodies) {
          const uint32_t g0 = e.group[b.range.start];
          bool shared = true;
          for (uint32_t i = b.range.start; i < b.range.start + b.range.count; ++i) shared = shared && e.group[i] == g0;
          if (shared && g0 != 0) continue;
          if (!shared) {
            rc = fail(PF_ERR_INVALID, "SoftbodySystem: a body has mixed collision groups");
            return;
          }
          for (uint32_t i = b.range.start; i < b.range.start + b.range.count; ++i) e.group[i] = next;
          ++next;
        }
      }
    }
    if (e.hasGrid) {
      e.grid.key_kind = PF_KEY_MORTON;
      for (int c = 0; c < 3; ++c) e.grid.origin[c] = d->hash_origin[c];
      e.grid.cell_size = static_cast<float>(nr);
      e.grid.table_size = table_size ? table_size
                                     : std::min<uint32_t>(next_pow2(2ull * e.cap), 1u << 20);
    }
    e.hasColliders = !e.prims.empty() || !e.sdfs.empty();
    if (e.hasAcc()) {
      e.accPos.init(e.cap, 10.0);
      e.accVel.init(e.cap, 50.0);
    }
    if (e.hasColliders) {
      e.primCap = static_cast<uint32_t>(e.prims.size());
      e.primLambda.assign(2 * static_cast<size_t>(e.cap) * e.primCap, 0);
      e.sdfLambda.assign(2 * static_cast<size_t>(e.cap) * e.sdfs.size(), 0);
    }
    e.built = true;
  });
  return rc;
}

int or_step(void* h, double dt) {
  Scene* s = static_cast<Scene*>(h);
  if (!(dt > 0) || !std::isfinite(dt))
    return fail(PF_ERR_INVALID, "SimLoop: step dt must be a positive finite number");
  int rc = PF_OK;
  s->visit([&](auto& e) {
    if (!e.built) {
      rc = fail(PF_ERR_STATE, "SimLoop: build the loop before stepping");
      return;
    }
    e.step(dt);
  });
  return rc;
}

// Field readback (pf_field numbering); float fields are converted to float32,
// or written as float64 when as_f64 is set.
// Whole-field write in particle order (positions, predicted, velocities with
// w set to 0 as the reference's buffers hold it; inverse mass).
int or_write(void* h, uint32_t field, const float* src, size_t bytes) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    using T = typename std::remove_reference<decltype(e.pos[0])>::type;
    const size_t cap = e.cap;
    auto put4 = [&](auto& dst) {
      if (bytes < 16 * cap) { rc = fail(PF_ERR_INVALID, "write: source too small"); return; }
      for (size_t i = 0; i < cap; ++i) {
        for (int c = 0; c < 3; ++c) dst[4 * i + c] = static_cast<T>(src[4 * i + c]);
        dst[4 * i + 3] = 0;
      }
    };
    switch (field) {
      case PF_FIELD_POSITIONS: put4(e.pos); break;
      case PF_FIELD_PREDICTED: put4(e.pred); break;
      case PF_FIELD_VELOCITIES: put4(e.vel); break;
      case PF_FIELD_INV_MASS:
        if (bytes < 4 * cap) { rc = fail(PF_ERR_INVALID, "write: source too small"); return; }
        for (size_t i = 0; i < cap; ++i) e.invMass[i] = static_cast<T>(src[i]);
        break;
      default: rc = fail(PF_ERR_INVALID, "write: field cannot be written");
    }
  });
  return rc;
}

int or_readback(void* h, uint32_t field, void* dst, size_t bytes, int as_f64) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    const size_t cap = e.cap;
    auto put = [&](const auto& src, size_t n) {
      if (as_f64) {
        if (bytes < n * 8) { rc = fail(PF_ERR_INVALID, "readback: buffer too small"); return; }
        double* o = static_cast<double*>(dst);
        for (size_t i = 0; i < n; ++i) o[i] = static_cast<double>(src[i]);
      } else {
        if (bytes < n * 4) { rc = fail(PF_ERR_INVALID, "readback: buffer too small"); return; }
        float* o = static_cast<float*>(dst);
        for (size_t i = 0; i < n; ++i) o[i] = static_cast<float>(src[i]);
      }
    };
    switch (field) {
      case PF_FIELD_POSITIONS: put(e.pos, 4 * cap); break;
      case PF_FIELD_PREDICTED: put(e.pred, 4 * cap); break;
      case PF_FIELD_VELOCITIES: put(e.vel, 4 * cap); break;
      case PF_FIELD_INV_MASS: put(e.invMass, cap); break;
      case PF_FIELD_BOUNDARY_VOLUME: put(e.bvol, cap); break;
      case PF_FIELD_ROTATION: put(e.rot, 4 * cap); break;
      case PF_FIELD_PREDICTED_ROTATION: put(e.prot, 4 * cap); break;
      case PF_FIELD_ANGULAR_VELOCITY: put(e.angv, 4 * cap); break;
      case PF_FIELD_DENSITY:
      case PF_FIELD_LAMBDA: {
        using T = typename std::remove_reference<decltype(e.pos[0])>::type;
        std::vector<T> out(cap, 0);
        for (auto& f : e.fluids)
          for (uint32_t i = f.range.start; i < f.range.start + f.range.count; ++i)
            out[i] = field == PF_FIELD_DENSITY ? f.density[i] : f.lambda[i];
        put(out, cap);
        break;
      }
      case PF_FIELD_NEIGHBOR_COUNT:
      case PF_FIELD_NEIGHBORS: {
        const size_t rows = field == PF_FIELD_NEIGHBORS ? kMaxNeighbors : 1;
        if (bytes < cap * rows * 4) { rc = fail(PF_ERR_INVALID, "readback: buffer too small"); return; }
        uint32_t* o = static_cast<uint32_t*>(dst);
        std::fill(o, o + cap * rows, field == PF_FIELD_NEIGHBORS ? UINT32_MAX : 0u);
        for (auto& f : e.fluids)
          for (uint32_t li = 0; li < f.range.count; ++li) {
            const uint32_t i = f.range.start + li;
            if (field == PF_FIELD_NEIGHBOR_COUNT) {
              o[i] = f.nbrCount[li];
            } else {
              for (uint32_t k = 0; k < f.nbrCount[li]; ++k)
                o[static_cast<size_t>(i) * kMaxNeighbors + k] = f.nbrIdx[static_cast<size_t>(k) * f.range.count + li];
            }
          }
        break;
      }
      default:
        rc = fail(PF_ERR_INVALID, "readback: unknown field");
    }
  });
  return rc;
}

int or_add_no_self_contacts(void* h, pf_range r) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    if (!range_ok(e.cap, r)) {
      rc = fail(PF_ERR_INVALID, "Material: invalid noSelfContacts range");
      return;
    }
    e.quietRanges.push_back({r.start, r.count});
  });
  return rc;
}

// The last substep's pairs (particle indices, each pair ascending, sorted)
// and its pair count including dropped ones.
int or_contacts_read(void* h, uint32_t* pairs, uint32_t capacity, uint32_t* count, uint32_t* stored) {
  Scene* s = static_cast<Scene*>(h);
  int rc = PF_OK;
  s->visit([&](auto& e) {
    if (!e.hasContact) {
      rc = fail(PF_ERR_STATE, "contacts: the SimLoop was built without contact");
      return;
    }
    std::vector<std::pair<uint32_t, uint32_t>> out;
    for (auto& c : e.contacts) out.push_back({std::min(c.i, c.j), std::max(c.i, c.j)});
    std::sort(out.begin(), out.end());
    if (count) *count = e.contactCount;
    if (stored) *stored = static_cast<uint32_t>(out.size());
    for (size_t q = 0; pairs && q < out.size() && q < capacity; ++q) {
      pairs[2 * q] = out[q].first;
      pairs[2 * q + 1] = out[q].second;
    }
  });
  return rc;
}

int or_overflow_read(void* h, pf_overflow* o) {
  Scene* s = static_cast<Scene*>(h);
  s->visit([&](auto& e) {
    std::memset(o, 0, sizeof(*o));
    o->positions = e.accPos.flag;
    o->velocities = e.accVel.flag;
    o->grid = e.gridOverflow;
    o->contacts = e.hasContact && e.contactCount > e.maxContacts;
    for (auto& f : e.fluids) o->neighbors |= f.nbrOverflow;
  });
  return PF_OK;
}

}  // extern "C"
