// Mesh -> particle setup on the GPU: the voxeliser (src/softbody/voxelize.ts)
// and the signed-distance baker (src/sdf/bake.ts).
//
// Both are brute force in the reference (every grid point against every
// triangle, in JavaScript doubles); here one thread per grid point walks the
// triangles, tiled through shared memory, in the reference's order and in
// double precision. This file is compiled with -fmad=false, so every double
// multiply and add is rounded on its own as the reference's arithmetic is,
// and the occupancy, hit counts and distances equal the reference's. The
// integer bookkeeping that follows the inside test (largest piece, surface
// classification, ordering, edges) runs on the host, in O(cells).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "common.cuh"
#include "pfsim.h"

namespace pf {
namespace {

constexpr uint32_t kTileTris = 128;

// One triangle as the kernels read it: the three corners (f32, as the
// mesh's Float32Array holds them) and its bounding box.
struct MeshTri {
  float a[3], b[3], c[3], lo[3], hi[3];
};

// Shared-memory staging of triangles [t0, t0 + kTileTris).
__device__ __forceinline__ uint32_t stage_tris(MeshTri* st, const MeshTri* __restrict__ tris, uint32_t t0,
                                               uint32_t n_tris) {
  const uint32_t cnt = min(kTileTris, n_tris - t0);
  const float* src = reinterpret_cast<const float*>(tris + t0);
  float* dst = reinterpret_cast<float*>(st);
  for (uint32_t i = threadIdx.x; i < cnt * 15u; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  return cnt;
}

// voxelize.ts:178-228: Moller-Trumbore, the ray parameter of the hit or -1.
__device__ __forceinline__ double ray_tri_t(double ox, double oy, double oz, double dx, double dy, double dz,
                                            const MeshTri& T) {
  const double ax = T.a[0], ay = T.a[1], az = T.a[2];
  const double e1x = (double)T.b[0] - ax, e1y = (double)T.b[1] - ay, e1z = (double)T.b[2] - az;
  const double e2x = (double)T.c[0] - ax, e2y = (double)T.c[1] - ay, e2z = (double)T.c[2] - az;
  const double hx = dy * e2z - dz * e2y;
  const double hy = dz * e2x - dx * e2z;
  const double hz = dx * e2y - dy * e2x;
  const double a = e1x * hx + e1y * hy + e1z * hz;
  if (a > -1e-9 && a < 1e-9) return -1.0;
  const double f = 1.0 / a;
  const double sx = ox - ax, sy = oy - ay, sz = oz - az;
  const double u = f * (sx * hx + sy * hy + sz * hz);
  if (u < 0.0 || u > 1.0) return -1.0;
  const double qx = sy * e1z - sz * e1y;
  const double qy = sz * e1x - sx * e1z;
  const double qz = sx * e1y - sy * e1x;
  const double v = f * (dx * qx + dy * qy + dz * qz);
  if (v < 0.0 || u + v > 1.0) return -1.0;
  const double t = f * (e2x * qx + e2y * qy + e2z * qz);
  if (t < 1e-9) return -1.0;
  return t;
}

// voxelize.ts:86-90, 234-259: grid point `cell` of an nx x ny x nz lattice
// at min + r + 2r i, inside the mesh when a slightly off-axis ray crosses it
// an odd number of times.
__global__ void __launch_bounds__(256) k_vox_mesh(const MeshTri* __restrict__ tris, uint32_t n_tris, double mnx,
                                                  double mny, double mnz, double r, double spacing, uint32_t nx,
                                                  uint32_t ny, uint64_t cells, uint8_t* __restrict__ occ) {
  __shared__ MeshTri st[kTileTris];
  const uint64_t cell = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = cell < cells;
  double px = 0, py = 0, pz = 0;
  if (live) {
    px = mnx + r + spacing * (double)(cell % nx);
    py = mny + r + spacing * (double)((cell / nx) % ny);
    pz = mnz + r + spacing * (double)(cell / ((uint64_t)nx * ny));
  }
  uint32_t crossings = 0;
  for (uint32_t t0 = 0; t0 < n_tris; t0 += kTileTris) {
    const uint32_t cnt = stage_tris(st, tris, t0, n_tris);
    if (live)
      for (uint32_t t = 0; t < cnt; ++t)
        if (ray_tri_t(px, py, pz, 1.0, 0.00137, 0.00241, st[t]) > 0.0) ++crossings;
    __syncthreads();
  }
  if (live) occ[cell] = (crossings & 1u) ? 1 : 0;
}

// sample.ts:12-47 in doubles over the f32 field.
__device__ __forceinline__ double sample_field(const float* __restrict__ data, uint32_t rx, uint32_t ry,
                                               uint32_t rz, double ox, double oy, double oz, double vx,
                                               double vy, double vz, double x, double y, double z) {
  const double gx = (x - ox) / vx - 0.5, gy = (y - oy) / vy - 0.5, gz = (z - oz) / vz - 0.5;
  auto clampi = [](double v, double hi) { return v < 0.0 ? 0.0 : (v > hi ? hi : v); };
  const double i0 = clampi(floor(gx), (double)(rx - 2)), j0 = clampi(floor(gy), (double)(ry - 2)),
               k0 = clampi(floor(gz), (double)(rz - 2));
  auto c01 = [](double t) { return t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t); };
  const double tx = c01(gx - i0), ty = c01(gy - j0), tz = c01(gz - k0);
  const uint64_t stride = rx, slice = (uint64_t)rx * ry;
  const uint64_t base = (uint64_t)i0 + (uint64_t)j0 * stride + (uint64_t)k0 * slice;
  auto lerp = [](double a, double b, double t) { return a + (b - a) * t; };
  const double c00 = lerp(data[base], data[base + 1], tx);
  const double c10 = lerp(data[base + stride], data[base + stride + 1], tx);
  const double c01v = lerp(data[base + slice], data[base + slice + 1], tx);
  const double c11 = lerp(data[base + slice + stride], data[base + slice + stride + 1], tx);
  const double c0 = lerp(c00, c10, ty), c1 = lerp(c01v, c11, ty);
  return lerp(c0, c1, tz);
}

// voxelize.ts:173-177: inside where the sampled field is below `dilation`.
__global__ void __launch_bounds__(256) k_vox_sdf(const float* __restrict__ data, uint32_t rx, uint32_t ry,
                                                 uint32_t rz, double ox, double oy, double oz, double vx, double vy,
                                                 double vz, double dilation, double r, double spacing, uint32_t nx,
                                                 uint32_t ny, uint64_t cells, uint8_t* __restrict__ occ) {
  const uint64_t cell = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= cells) return;
  const double px = ox + r + spacing * (double)(cell % nx);
  const double py = oy + r + spacing * (double)((cell / nx) % ny);
  const double pz = oz + r + spacing * (double)(cell / ((uint64_t)nx * ny));
  occ[cell] = sample_field(data, rx, ry, rz, ox, oy, oz, vx, vy, vz, px, py, pz) < dilation ? 1 : 0;
}

// bake.ts:297-368: squared distance from P to a triangle (Ericson RTCD
// 5.1.5, the seven Voronoi regions).
__device__ __forceinline__ double point_tri_d2(double px, double py, double pz, const MeshTri& T) {
  const double ax = T.a[0], ay = T.a[1], az = T.a[2];
  const double bx = T.b[0], by = T.b[1], bz = T.b[2];
  const double cx = T.c[0], cy = T.c[1], cz = T.c[2];
  const double abx = bx - ax, aby = by - ay, abz = bz - az;
  const double acx = cx - ax, acy = cy - ay, acz = cz - az;
  const double apx = px - ax, apy = py - ay, apz = pz - az;
  const double d1 = abx * apx + aby * apy + abz * apz;
  const double d2 = acx * apx + acy * apy + acz * apz;
  if (d1 <= 0.0 && d2 <= 0.0) return apx * apx + apy * apy + apz * apz;
  const double bpx = px - bx, bpy = py - by, bpz = pz - bz;
  const double d3 = abx * bpx + aby * bpy + abz * bpz;
  const double d4 = acx * bpx + acy * bpy + acz * bpz;
  if (d3 >= 0.0 && d4 <= d3) return bpx * bpx + bpy * bpy + bpz * bpz;
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
    const double v = d1 / (d1 - d3);
    const double qx = apx - v * abx, qy = apy - v * aby, qz = apz - v * abz;
    return qx * qx + qy * qy + qz * qz;
  }
  const double cpx = px - cx, cpy = py - cy, cpz = pz - cz;
  const double d5 = abx * cpx + aby * cpy + abz * cpz;
  const double d6 = acx * cpx + acy * cpy + acz * cpz;
  if (d6 >= 0.0 && d5 <= d6) return cpx * cpx + cpy * cpy + cpz * cpz;
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
    const double w = d2 / (d2 - d6);
    const double qx = apx - w * acx, qy = apy - w * acy, qz = apz - w * acz;
    return qx * qx + qy * qy + qz * qz;
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0.0 && d4 - d3 >= 0.0 && d5 - d6 >= 0.0) {
    const double w = (d4 - d3) / (d4 - d3 + (d5 - d6));
    const double qx = bpx - w * (cx - bx), qy = bpy - w * (cy - by), qz = bpz - w * (cz - bz);
    return qx * qx + qy * qy + qz * qz;
  }
  const double denom = 1.0 / (va + vb + vc);
  const double v = vb * denom, w = vc * denom;
  const double qx = apx - v * abx - w * acx, qy = apy - v * aby - w * acy, qz = apz - v * abz - w * acz;
  return qx * qx + qy * qy + qz * qz;
}

__device__ __forceinline__ double outside(double p, double lo, double hi) {
  return p < lo ? lo - p : (p > hi ? p - hi : 0.0);
}

// bake.ts:460-486: the axis ray along +x, +y or +z against one triangle.
__device__ __forceinline__ bool axis_hit(double px, double py, double pz, int axis, const MeshTri& T) {
  const double ax = T.a[0], ay = T.a[1], az = T.a[2];
  const double e1x = (double)T.b[0] - ax, e1y = (double)T.b[1] - ay, e1z = (double)T.b[2] - az;
  const double e2x = (double)T.c[0] - ax, e2y = (double)T.c[1] - ay, e2z = (double)T.c[2] - az;
  double hx, hy, hz;
  if (axis == 0) {
    hx = 0.0;
    hy = -e2z;
    hz = e2y;
  } else if (axis == 1) {
    hx = e2z;
    hy = 0.0;
    hz = -e2x;
  } else {
    hx = -e2y;
    hy = e2x;
    hz = 0.0;
  }
  const double a = e1x * hx + e1y * hy + e1z * hz;
  if (fabs(a) < 1e-7) return false;
  const double inv = 1.0 / a;
  const double sx = px - ax, sy = py - ay, sz = pz - az;
  const double u = inv * (sx * hx + sy * hy + sz * hz);
  if (u < 0.0 || u > 1.0) return false;
  const double qx = sy * e1z - sz * e1y;
  const double qy = sz * e1x - sx * e1z;
  const double qz = sx * e1y - sy * e1x;
  const double v = inv * (axis == 0 ? qx : (axis == 1 ? qy : qz));
  if (v < 0.0 || u + v > 1.0) return false;
  return inv * (e2x * qx + e2y * qy + e2z * qz) > 1e-7;
}

// bake.ts:422-448 with its bounding-box culls.
__device__ __forceinline__ bool axis_ray_counts(double px, double py, double pz, int axis, const MeshTri& T) {
  if (axis == 0) {
    if (py < T.lo[1] || py > T.hi[1] || pz < T.lo[2] || pz > T.hi[2] || px > T.hi[0]) return false;
  } else if (axis == 1) {
    if (px < T.lo[0] || px > T.hi[0] || pz < T.lo[2] || pz > T.hi[2] || py > T.hi[1]) return false;
  } else {
    if (px < T.lo[0] || px > T.hi[0] || py < T.lo[1] || py > T.hi[1] || pz > T.hi[2]) return false;
  }
  return axis_hit(px, py, pz, axis, T);
}

// bake.ts:106-127: per voxel centre, the closest triangle (triangles in mesh
// order, each skipped when its box is no closer than the best so far), the
// three jittered axis-ray parities and their majority.
__global__ void __launch_bounds__(256) k_bake(const MeshTri* __restrict__ tris, uint32_t n_tris, uint32_t res,
                                              double ox, double oy, double oz, double voxel, double jitter,
                                              float* __restrict__ data, unsigned long long* __restrict__ inconsistent) {
  __shared__ MeshTri st[kTileTris];
  const uint64_t n = (uint64_t)res * res * res;
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = idx < n;
  const uint32_t xi = live ? (uint32_t)(idx % res) : 0u, yi = live ? (uint32_t)((idx / res) % res) : 0u,
                 zi = live ? (uint32_t)(idx / ((uint64_t)res * res)) : 0u;
  const double px = ox + ((double)xi + 0.5) * voxel;
  const double py = oy + ((double)yi + 0.5) * voxel;
  const double pz = oz + ((double)zi + 0.5) * voxel;
  const double ja = jitter * 1.4142135623730951, jb = jitter * 3.141592653589793;
  double best = INFINITY;
  uint32_t hx = 0, hy = 0, hz = 0;
  for (uint32_t t0 = 0; t0 < n_tris; t0 += kTileTris) {
    const uint32_t cnt = stage_tris(st, tris, t0, n_tris);
    if (live)
      for (uint32_t t = 0; t < cnt; ++t) {
        const MeshTri& T = st[t];
        const double dx = outside(px, T.lo[0], T.hi[0]), dy = outside(py, T.lo[1], T.hi[1]),
                     dz = outside(pz, T.lo[2], T.hi[2]);
        if (!(dx * dx + dy * dy + dz * dz >= best)) {
          const double d = point_tri_d2(px, py, pz, T);
          if (d < best) best = d;
        }
        hx += axis_ray_counts(px, py + ja, pz + jb, 0, T) ? 1u : 0u;
        hy += axis_ray_counts(px + jb, py, pz + ja, 1, T) ? 1u : 0u;
        hz += axis_ray_counts(px + ja, py + jb, pz, 2, T) ? 1u : 0u;
      }
    __syncthreads();
  }
  if (!live) return;
  const uint32_t votes = (hx & 1u) + (hy & 1u) + (hz & 1u);
  if (votes == 1 || votes == 2) atomicAdd(inconsistent, 1ull);
  const double dist = sqrt(best);
  data[idx] = (float)(votes >= 2 ? -dist : dist);
}

// toTriangleMesh + validated (src/core/mesh.ts:16-56).
pf_status read_mesh(const pf_mesh* m, std::vector<MeshTri>* out) {
  if (!m) return fail(PF_ERR_INVALID, "toTriangleMesh: expected a mesh");
  if (m->n_vertices && !m->vertices) return fail(PF_ERR_INVALID, "TriangleMesh: vertices are NULL");
  if (m->n_indices && !m->indices) return fail(PF_ERR_INVALID, "TriangleMesh: indices are NULL");
  if (m->n_indices % 3 != 0)
    return fail(PF_ERR_INVALID, "TriangleMesh: indices length " + std::to_string(m->n_indices) +
                                    " is not a multiple of 3");
  for (uint32_t i = 0; i < m->n_indices; ++i)
    if (m->indices[i] >= m->n_vertices)
      return fail(PF_ERR_INVALID, "TriangleMesh: index " + std::to_string(m->indices[i]) + " is out of range");
  out->resize(m->n_indices / 3);
  for (size_t t = 0; t < out->size(); ++t) {
    MeshTri& T = (*out)[t];
    const float* v[3] = {m->vertices + 3ull * m->indices[3 * t], m->vertices + 3ull * m->indices[3 * t + 1],
                         m->vertices + 3ull * m->indices[3 * t + 2]};
    for (int a = 0; a < 3; ++a) {
      T.a[a] = v[0][a];
      T.b[a] = v[1][a];
      T.c[a] = v[2][a];
      T.lo[a] = std::min(std::min(v[0][a], v[1][a]), v[2][a]);
      T.hi[a] = std::max(std::max(v[0][a], v[1][a]), v[2][a]);
    }
  }
  return PF_OK;
}

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

pf_status to_device(const std::vector<MeshTri>& tris, DevBuf* d) {
  const size_t bytes = std::max<size_t>(1, tris.size()) * sizeof(MeshTri);
  PF_CUDA(cudaMalloc(&d->p, bytes));
  if (!tris.empty()) PF_CUDA(cudaMemcpy(d->p, tris.data(), tris.size() * sizeof(MeshTri), cudaMemcpyHostToDevice));
  return PF_OK;
}

// voxelize.ts:92-161 from the occupancy: the largest face-connected piece
// (when asked), surface cells (a face neighbour missing) first, positions
// at the grid points, face-adjacent pairs.
pf_status finish_voxels(std::vector<uint8_t>& occ, const double mn[3], double r, double spacing, uint32_t nx,
                        uint32_t ny, uint32_t nz, bool largest, pf_voxels* out) {
  const uint64_t cells = (uint64_t)nx * ny * nz;
  auto nbrs = [&](uint64_t cell, uint64_t* o) {
    const uint64_t x = cell % nx, y = (cell / nx) % ny, z = cell / ((uint64_t)nx * ny);
    int n = 0;
    if (x > 0 && occ[cell - 1]) o[n++] = cell - 1;
    if (x + 1 < nx && occ[cell + 1]) o[n++] = cell + 1;
    if (y > 0 && occ[cell - nx]) o[n++] = cell - nx;
    if (y + 1 < ny && occ[cell + nx]) o[n++] = cell + nx;
    if (z > 0 && occ[cell - (uint64_t)nx * ny]) o[n++] = cell - (uint64_t)nx * ny;
    if (z + 1 < nz && occ[cell + (uint64_t)nx * ny]) o[n++] = cell + (uint64_t)nx * ny;
    return n;
  };
  if (largest) {
    std::vector<int64_t> piece(cells, -1);
    std::vector<uint64_t> best, members;
    uint64_t nb[6];
    for (uint64_t seed = 0; seed < cells; ++seed) {
      if (!occ[seed] || piece[seed] != -1) continue;
      members.assign(1, seed);
      piece[seed] = (int64_t)seed;
      for (size_t k = 0; k < members.size(); ++k) {
        const int c = nbrs(members[k], nb);
        for (int q = 0; q < c; ++q)
          if (piece[nb[q]] == -1) {
            piece[nb[q]] = (int64_t)seed;
            members.push_back(nb[q]);
          }
      }
      if (members.size() > best.size()) best.swap(members);
    }
    std::fill(occ.begin(), occ.end(), 0);
    for (uint64_t c : best) occ[c] = 1;
  }
  std::vector<uint64_t> surf, inner;
  uint64_t nb[6];
  for (uint64_t cell = 0; cell < cells; ++cell) {
    if (!occ[cell]) continue;
    (nbrs(cell, nb) < 6 ? surf : inner).push_back(cell);
  }
  const uint64_t count = surf.size() + inner.size();
  if (count > 0xffffffffull) return fail(PF_ERR_INVALID, "voxelize: too many particles");
  out->count = (uint32_t)count;
  out->surface_count = (uint32_t)surf.size();
  std::vector<uint32_t> particle_of;
  std::vector<uint64_t> ordered(surf);
  ordered.insert(ordered.end(), inner.begin(), inner.end());
  // cell -> particle through a sorted lookup (cells can be many)
  std::vector<std::pair<uint64_t, uint32_t>> lut(count);
  for (uint32_t i = 0; i < count; ++i) lut[i] = {ordered[i], i};
  std::sort(lut.begin(), lut.end());
  auto pid = [&](uint64_t cell) {
    return std::lower_bound(lut.begin(), lut.end(), std::make_pair(cell, 0u))->second;
  };
  if (out->positions && out->capacity >= count)
    for (uint32_t i = 0; i < count; ++i) {
      const uint64_t cell = ordered[i];
      const uint64_t ix[3] = {cell % nx, (cell / nx) % ny, cell / ((uint64_t)nx * ny)};
      for (int a = 0; a < 3; ++a) out->positions[3ull * i + a] = (float)(mn[a] + r + spacing * (double)ix[a]);
    }
  uint64_t ne = 0;
  for (uint32_t i = 0; i < count; ++i) {
    const int c = nbrs(ordered[i], nb);
    for (int q = 0; q < c; ++q) {
      const uint32_t j = pid(nb[q]);
      if (i < j) {
        if (out->edges && ne < out->edge_capacity) {
          out->edges[2 * ne] = i;
          out->edges[2 * ne + 1] = j;
        }
        ++ne;
      }
    }
  }
  out->edge_count = (uint32_t)ne;
  return PF_OK;
}

pf_status occupancy_launch_check() {
  PF_CUDA(cudaGetLastError());
  PF_CUDA(cudaDeviceSynchronize());
  return PF_OK;
}

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" {

pf_status pf_voxelize_mesh(const pf_mesh* mesh, double particle_radius, uint32_t largest_piece, pf_voxels* out) {
  if (!out) return fail(PF_ERR_INVALID, "voxelize: output is NULL");
  if (!(particle_radius > 0) || !std::isfinite(particle_radius))
    return fail(PF_ERR_INVALID, "voxelize: particleRadius must be positive, got " + std::to_string(particle_radius));
  if (mesh && mesh->n_vertices == 0) return fail(PF_ERR_INVALID, "voxelize: mesh has no vertices");
  std::vector<MeshTri> tris;
  PF_TRY(read_mesh(mesh, &tris));
  // voxelize.ts:164-172: bounds of the vertices
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t v = 0; v < mesh->n_vertices; ++v)
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], (double)mesh->vertices[3ull * v + a]);
      mx[a] = std::max(mx[a], (double)mesh->vertices[3ull * v + a]);
    }
  const double spacing = 2 * particle_radius;
  uint32_t dims[3];
  for (int a = 0; a < 3; ++a) {
    const double d = std::ceil((mx[a] - mn[a]) / spacing);
    if (!(d < 4294967295.0)) return fail(PF_ERR_INVALID, "voxelize: grid too large");
    dims[a] = (uint32_t)std::max(1.0, d);
  }
  const uint64_t cells = (uint64_t)dims[0] * dims[1] * dims[2];
  if (cells > (1ull << 31)) return fail(PF_ERR_INVALID, "voxelize: grid too large");
  DevBuf dt, docc;
  PF_TRY(to_device(tris, &dt));
  PF_CUDA(cudaMalloc(&docc.p, std::max<uint64_t>(cells, 1)));
  k_vox_mesh<<<(unsigned)((cells + 255) / 256), 256>>>(static_cast<const MeshTri*>(dt.p), (uint32_t)tris.size(),
                                                        mn[0], mn[1], mn[2], particle_radius, spacing, dims[0],
                                                        dims[1], cells, static_cast<uint8_t*>(docc.p));
  PF_TRY(occupancy_launch_check());
  std::vector<uint8_t> occ(cells);
  PF_CUDA(cudaMemcpy(occ.data(), docc.p, cells, cudaMemcpyDeviceToHost));
  return finish_voxels(occ, mn, particle_radius, spacing, dims[0], dims[1], dims[2], largest_piece != 0, out);
}

pf_status pf_voxelize_sdf(const float* data, const uint32_t res[3], const double origin[3], const double voxel[3],
                          double particle_radius, double dilation, uint32_t largest_piece, pf_voxels* out) {
  if (!out || !data || !res || !origin || !voxel) return fail(PF_ERR_INVALID, "voxelize: NULL argument");
  if (!(particle_radius > 0) || !std::isfinite(particle_radius))
    return fail(PF_ERR_INVALID, "voxelize: particleRadius must be positive, got " + std::to_string(particle_radius));
  if (!std::isfinite(dilation))
    return fail(PF_ERR_INVALID, "voxelize: dilation must be a finite number, got " + std::to_string(dilation));
  for (int a = 0; a < 3; ++a) {
    if (res[a] < 2)
      return fail(PF_ERR_INVALID, "sampleSdf: resolution must be integers >= 2, got [" + std::to_string(res[0]) +
                                      ", " + std::to_string(res[1]) + ", " + std::to_string(res[2]) + "]");
    if (!(voxel[a] > 0) || !std::isfinite(voxel[a]) || !std::isfinite(origin[a]))
      return fail(PF_ERR_INVALID, "voxelize: voxelSize must be positive and origin finite");
  }
  // voxelize.ts:173-177: the field's box
  double mn[3], mx[3];
  for (int a = 0; a < 3; ++a) {
    mn[a] = origin[a];
    mx[a] = origin[a] + (double)res[a] * voxel[a];
  }
  const double spacing = 2 * particle_radius;
  uint32_t dims[3];
  for (int a = 0; a < 3; ++a) {
    const double d = std::ceil((mx[a] - mn[a]) / spacing);
    if (!(d < 4294967295.0)) return fail(PF_ERR_INVALID, "voxelize: grid too large");
    dims[a] = (uint32_t)std::max(1.0, d);
  }
  const uint64_t cells = (uint64_t)dims[0] * dims[1] * dims[2];
  const uint64_t nv = (uint64_t)res[0] * res[1] * res[2];
  if (cells > (1ull << 31) || nv > (1ull << 31)) return fail(PF_ERR_INVALID, "voxelize: grid too large");
  DevBuf dd, docc;
  PF_CUDA(cudaMalloc(&dd.p, 4 * nv));
  PF_CUDA(cudaMemcpy(dd.p, data, 4 * nv, cudaMemcpyHostToDevice));
  PF_CUDA(cudaMalloc(&docc.p, std::max<uint64_t>(cells, 1)));
  k_vox_sdf<<<(unsigned)((cells + 255) / 256), 256>>>(static_cast<const float*>(dd.p), res[0], res[1], res[2],
                                                       origin[0], origin[1], origin[2], voxel[0], voxel[1], voxel[2],
                                                       dilation, particle_radius, spacing, dims[0], dims[1], cells,
                                                       static_cast<uint8_t*>(docc.p));
  PF_TRY(occupancy_launch_check());
  std::vector<uint8_t> occ(cells);
  PF_CUDA(cudaMemcpy(occ.data(), docc.p, cells, cudaMemcpyDeviceToHost));
  return finish_voxels(occ, mn, particle_radius, spacing, dims[0], dims[1], dims[2], largest_piece != 0, out);
}

pf_status pf_bake_sdf(const pf_mesh* mesh, uint32_t resolution, double padding, float* data, double origin[3],
                      double* voxel_size, uint64_t* inconsistent) {
  if (!data || !origin || !voxel_size) return fail(PF_ERR_INVALID, "bakeMeshToSdf: NULL argument");
  std::vector<MeshTri> tris;
  PF_TRY(read_mesh(mesh, &tris));
  // bake.ts:142-172
  if (resolution < 4)
    return fail(PF_ERR_INVALID, "bakeMeshToSdf: resolution must be an integer >= 4, got " + std::to_string(resolution));
  const bool default_pad = padding < 0;
  if (!default_pad && !std::isfinite(padding))
    return fail(PF_ERR_INVALID, "bakeMeshToSdf: padding must be a non-negative finite number, got " +
                                    std::to_string(padding));
  if (tris.empty()) return fail(PF_ERR_INVALID, "bakeMeshToSdf: mesh has zero triangles");
  if ((uint64_t)resolution * resolution * resolution > (1ull << 31))
    return fail(PF_ERR_INVALID, "bakeMeshToSdf: resolution too large");
  // bake.ts:216-255: a cubic grid around the triangles' box
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (const MeshTri& T : tris)
    for (int a = 0; a < 3; ++a) {
      if (T.lo[a] < mn[a]) mn[a] = T.lo[a];
      if (T.hi[a] > mx[a]) mx[a] = T.hi[a];
    }
  if (default_pad) {
    const double extent = std::max(std::max(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]);
    const double k = resolution >= 8 ? 2 : 1;
    padding = (k * extent) / ((double)resolution - 2 * k);
  }
  for (int a = 0; a < 3; ++a) {
    mn[a] -= padding;
    mx[a] += padding;
  }
  const double side = std::max(std::max(mx[0] - mn[0], mx[1] - mn[1]), mx[2] - mn[2]);
  const double vs = side / (double)resolution;
  for (int a = 0; a < 3; ++a) origin[a] = 0.5 * (mn[a] + mx[a]) - 0.5 * side;
  *voxel_size = vs;
  const uint64_t n = (uint64_t)resolution * resolution * resolution;
  DevBuf dt, dd, dc;
  PF_TRY(to_device(tris, &dt));
  PF_CUDA(cudaMalloc(&dd.p, 4 * n));
  PF_CUDA(cudaMalloc(&dc.p, 8));
  PF_CUDA(cudaMemset(dc.p, 0, 8));
  k_bake<<<(unsigned)((n + 255) / 256), 256>>>(static_cast<const MeshTri*>(dt.p), (uint32_t)tris.size(), resolution,
                                                origin[0], origin[1], origin[2], vs, vs * 1e-4,
                                                static_cast<float*>(dd.p), static_cast<unsigned long long*>(dc.p));
  PF_TRY(occupancy_launch_check());
  PF_CUDA(cudaMemcpy(data, dd.p, 4 * n, cudaMemcpyDeviceToHost));
  unsigned long long bad = 0;
  PF_CUDA(cudaMemcpy(&bad, dc.p, 8, cudaMemcpyDeviceToHost));
  if (inconsistent) *inconsistent = bad;
  // bake.ts:129-138
  const double frac = (double)bad / (double)n;
  if (frac > 0.01) {
    char pct[32];
    std::snprintf(pct, sizeof pct, "%.2f", frac * 100);
    return fail(PF_ERR_INVALID, "bakeMeshToSdf: mesh appears non-watertight - " + std::to_string(bad) + " of " +
                                    std::to_string(n) + " voxels (" + pct +
                                    "%) had disagreeing axis sign votes. Threshold is 1.00%. Check the input mesh "
                                    "for holes, T-junctions, or non-manifold edges.");
  }
  return PF_OK;
}

}  // extern "C"
