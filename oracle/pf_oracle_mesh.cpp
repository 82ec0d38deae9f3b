// CPU oracle of the mesh -> particle setup (TEST INFRASTRUCTURE ONLY: the
// checker of pf_voxelize_mesh / pf_voxelize_sdf / pf_bake_sdf; never part of
// the product). Plain loops over grid points and triangles in the order of
// src/softbody/voxelize.ts and src/sdf/bake.ts, in doubles, compiled with
// -ffp-contract=off so each multiply and add is rounded on its own.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "pfsim.h"

namespace {

struct Tri {
  double a[3], b[3], c[3], lo[3], hi[3];
};

std::vector<Tri> tris_of(const pf_mesh* m) {
  std::vector<Tri> out(m->n_indices / 3);
  for (size_t t = 0; t < out.size(); ++t) {
    Tri& T = out[t];
    for (int a = 0; a < 3; ++a) {
      T.a[a] = m->vertices[3 * m->indices[3 * t] + a];
      T.b[a] = m->vertices[3 * m->indices[3 * t + 1] + a];
      T.c[a] = m->vertices[3 * m->indices[3 * t + 2] + a];
      T.lo[a] = std::min(std::min(T.a[a], T.b[a]), T.c[a]);
      T.hi[a] = std::max(std::max(T.a[a], T.b[a]), T.c[a]);
    }
  }
  return out;
}

// voxelize.ts:178-228
double ray_triangle(const double o[3], const double d[3], const Tri& T) {
  const double e1[3] = {T.b[0] - T.a[0], T.b[1] - T.a[1], T.b[2] - T.a[2]};
  const double e2[3] = {T.c[0] - T.a[0], T.c[1] - T.a[1], T.c[2] - T.a[2]};
  const double h[3] = {d[1] * e2[2] - d[2] * e2[1], d[2] * e2[0] - d[0] * e2[2], d[0] * e2[1] - d[1] * e2[0]};
  const double a = e1[0] * h[0] + e1[1] * h[1] + e1[2] * h[2];
  if (a > -1e-9 && a < 1e-9) return -1;
  const double f = 1 / a;
  const double s[3] = {o[0] - T.a[0], o[1] - T.a[1], o[2] - T.a[2]};
  const double u = f * (s[0] * h[0] + s[1] * h[1] + s[2] * h[2]);
  if (u < 0 || u > 1) return -1;
  const double q[3] = {s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
  const double v = f * (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]);
  if (v < 0 || u + v > 1) return -1;
  const double t = f * (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]);
  if (t < 1e-9) return -1;
  return t;
}

// sample.ts:12-47
double sample(const float* data, const uint32_t res[3], const double o[3], const double vs[3], const double p[3]) {
  double g[3], t[3];
  int64_t i[3];
  for (int a = 0; a < 3; ++a) {
    g[a] = (p[a] - o[a]) / vs[a] - 0.5;
    double f = std::floor(g[a]);
    const double hi = (double)res[a] - 2;
    f = f < 0 ? 0 : (f > hi ? hi : f);
    i[a] = (int64_t)f;
    const double tt = g[a] - f;
    t[a] = tt < 0 ? 0 : (tt > 1 ? 1 : tt);
  }
  const int64_t sy = res[0], sz = (int64_t)res[0] * res[1];
  const int64_t b = i[0] + i[1] * sy + i[2] * sz;
  auto L = [](double x, double y, double w) { return x + (y - x) * w; };
  const double c00 = L(data[b], data[b + 1], t[0]), c10 = L(data[b + sy], data[b + sy + 1], t[0]);
  const double c01 = L(data[b + sz], data[b + sz + 1], t[0]), c11 = L(data[b + sz + sy], data[b + sz + sy + 1], t[0]);
  return L(L(c00, c10, t[1]), L(c01, c11, t[1]), t[2]);
}

// voxelize.ts:80-161 from an inside predicate.
template <typename In>
void voxels(const double mn[3], const double mx[3], double r, bool largest, In inside, pf_voxels* out) {
  const double sp = 2 * r;
  uint32_t n[3];
  for (int a = 0; a < 3; ++a) n[a] = (uint32_t)std::max(1.0, std::ceil((mx[a] - mn[a]) / sp));
  const uint64_t cells = (uint64_t)n[0] * n[1] * n[2];
  auto ctr = [&](uint64_t cell, int a) {
    const uint64_t idx[3] = {cell % n[0], (cell / n[0]) % n[1], cell / ((uint64_t)n[0] * n[1])};
    return mn[a] + r + sp * (double)idx[a];
  };
  std::vector<uint8_t> occ(cells);
  for (uint64_t c = 0; c < cells; ++c) occ[c] = inside(ctr(c, 0), ctr(c, 1), ctr(c, 2)) ? 1 : 0;
  auto nb = [&](uint64_t c) {
    std::vector<uint64_t> o;
    const uint64_t x = c % n[0], y = (c / n[0]) % n[1], z = c / ((uint64_t)n[0] * n[1]);
    const uint64_t sxy = (uint64_t)n[0] * n[1];
    if (x > 0) o.push_back(c - 1);
    if (x + 1 < n[0]) o.push_back(c + 1);
    if (y > 0) o.push_back(c - n[0]);
    if (y + 1 < n[1]) o.push_back(c + n[0]);
    if (z > 0) o.push_back(c - sxy);
    if (z + 1 < n[2]) o.push_back(c + sxy);
    std::vector<uint64_t> k;
    for (uint64_t q : o)
      if (occ[q]) k.push_back(q);
    return k;
  };
  if (largest) {
    std::vector<int64_t> piece(cells, -1);
    std::vector<uint64_t> big;
    for (uint64_t s = 0; s < cells; ++s) {
      if (!occ[s] || piece[s] != -1) continue;
      std::vector<uint64_t> mem{s};
      piece[s] = (int64_t)s;
      for (size_t k = 0; k < mem.size(); ++k)
        for (uint64_t q : nb(mem[k]))
          if (piece[q] == -1) {
            piece[q] = (int64_t)s;
            mem.push_back(q);
          }
      if (mem.size() > big.size()) big = mem;
    }
    std::fill(occ.begin(), occ.end(), 0);
    for (uint64_t c : big) occ[c] = 1;
  }
  std::vector<uint64_t> order, inner;
  for (uint64_t c = 0; c < cells; ++c)
    if (occ[c]) (nb(c).size() < 6 ? order : inner).push_back(c);
  out->surface_count = (uint32_t)order.size();
  order.insert(order.end(), inner.begin(), inner.end());
  out->count = (uint32_t)order.size();
  std::vector<int64_t> pid(cells, -1);
  for (size_t i = 0; i < order.size(); ++i) pid[order[i]] = (int64_t)i;
  if (out->positions && out->capacity >= out->count)
    for (size_t i = 0; i < order.size(); ++i)
      for (int a = 0; a < 3; ++a) out->positions[3 * i + a] = (float)ctr(order[i], a);
  uint32_t e = 0;
  for (size_t i = 0; i < order.size(); ++i)
    for (uint64_t q : nb(order[i])) {
      const uint32_t j = (uint32_t)pid[q];
      if (i < j) {
        if (out->edges && e < out->edge_capacity) {
          out->edges[2 * e] = (uint32_t)i;
          out->edges[2 * e + 1] = j;
        }
        ++e;
      }
    }
  out->edge_count = e;
}

// bake.ts:297-368
double tri_d2(const double p[3], const Tri& T) {
  double ab[3], ac[3], ap[3];
  for (int a = 0; a < 3; ++a) {
    ab[a] = T.b[a] - T.a[a];
    ac[a] = T.c[a] - T.a[a];
    ap[a] = p[a] - T.a[a];
  }
  auto dot = [](const double* x, const double* y) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
  const double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0 && d2 <= 0) return dot(ap, ap);
  double bp[3];
  for (int a = 0; a < 3; ++a) bp[a] = p[a] - T.b[a];
  const double d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0 && d4 <= d3) return dot(bp, bp);
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    const double v = d1 / (d1 - d3);
    const double q[3] = {ap[0] - v * ab[0], ap[1] - v * ab[1], ap[2] - v * ab[2]};
    return dot(q, q);
  }
  double cp[3];
  for (int a = 0; a < 3; ++a) cp[a] = p[a] - T.c[a];
  const double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0 && d5 <= d6) return dot(cp, cp);
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    const double w = d2 / (d2 - d6);
    const double q[3] = {ap[0] - w * ac[0], ap[1] - w * ac[1], ap[2] - w * ac[2]};
    return dot(q, q);
  }
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0 && d4 - d3 >= 0 && d5 - d6 >= 0) {
    const double w = (d4 - d3) / (d4 - d3 + (d5 - d6));
    const double q[3] = {bp[0] - w * (T.c[0] - T.b[0]), bp[1] - w * (T.c[1] - T.b[1]), bp[2] - w * (T.c[2] - T.b[2])};
    return dot(q, q);
  }
  const double den = 1.0 / (va + vb + vc);
  const double v = vb * den, w = vc * den;
  const double q[3] = {ap[0] - v * ab[0] - w * ac[0], ap[1] - v * ab[1] - w * ac[1], ap[2] - v * ab[2] - w * ac[2]};
  return dot(q, q);
}

// bake.ts:422-486
uint32_t axis_hits(const double p[3], int axis, const std::vector<Tri>& tris) {
  // the box test on the two perpendicular axes, then the one behind the ray
  const int pa = axis == 0 ? 1 : 0, pb = axis == 2 ? 1 : 2;
  uint32_t hits = 0;
  for (const Tri& T : tris) {
    if (p[pa] < T.lo[pa] || p[pa] > T.hi[pa]) continue;
    if (p[pb] < T.lo[pb] || p[pb] > T.hi[pb]) continue;
    if (p[axis] > T.hi[axis]) continue;
    double e1[3], e2[3];
    for (int a = 0; a < 3; ++a) {
      e1[a] = T.b[a] - T.a[a];
      e2[a] = T.c[a] - T.a[a];
    }
    double h[3];
    if (axis == 0) {
      h[0] = 0;
      h[1] = -e2[2];
      h[2] = e2[1];
    } else if (axis == 1) {
      h[0] = e2[2];
      h[1] = 0;
      h[2] = -e2[0];
    } else {
      h[0] = -e2[1];
      h[1] = e2[0];
      h[2] = 0;
    }
    const double a = e1[0] * h[0] + e1[1] * h[1] + e1[2] * h[2];
    if (std::fabs(a) < 1e-7) continue;
    const double ia = 1 / a;
    const double s[3] = {p[0] - T.a[0], p[1] - T.a[1], p[2] - T.a[2]};
    const double u = ia * (s[0] * h[0] + s[1] * h[1] + s[2] * h[2]);
    if (u < 0 || u > 1) continue;
    const double q[3] = {s[1] * e1[2] - s[2] * e1[1], s[2] * e1[0] - s[0] * e1[2], s[0] * e1[1] - s[1] * e1[0]};
    const double v = ia * q[axis];
    if (v < 0 || u + v > 1) continue;
    if (ia * (e2[0] * q[0] + e2[1] * q[1] + e2[2] * q[2]) > 1e-7) ++hits;
  }
  return hits;
}

}  // namespace

extern "C" {

int or_voxelize_mesh(const pf_mesh* m, double r, uint32_t largest, pf_voxels* out) {
  const std::vector<Tri> tris = tris_of(m);
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t v = 0; v < m->n_vertices; ++v)
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], (double)m->vertices[3 * v + a]);
      mx[a] = std::max(mx[a], (double)m->vertices[3 * v + a]);
    }
  const double dir[3] = {1, 0.00137, 0.00241};
  voxels(mn, mx, r, largest != 0,
         [&](double x, double y, double z) {
           const double o[3] = {x, y, z};
           uint32_t c = 0;
           for (const Tri& T : tris)
             if (ray_triangle(o, dir, T) > 0) ++c;
           return (c & 1) == 1;
         },
         out);
  return 0;
}

int or_voxelize_sdf(const float* data, const uint32_t res[3], const double origin[3], const double vs[3], double r,
                    double dilation, uint32_t largest, pf_voxels* out) {
  double mn[3], mx[3];
  for (int a = 0; a < 3; ++a) {
    mn[a] = origin[a];
    mx[a] = origin[a] + res[a] * vs[a];
  }
  voxels(mn, mx, r, largest != 0,
         [&](double x, double y, double z) {
           const double p[3] = {x, y, z};
           return sample(data, res, origin, vs, p) < dilation;
         },
         out);
  return 0;
}

int or_bake_sdf(const pf_mesh* m, uint32_t res, double padding, float* data, double origin[3], double* voxel,
                uint64_t* inconsistent) {
  const std::vector<Tri> tris = tris_of(m);
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (const Tri& T : tris)
    for (int a = 0; a < 3; ++a) {
      if (T.lo[a] < mn[a]) mn[a] = T.lo[a];
      if (T.hi[a] > mx[a]) mx[a] = T.hi[a];
    }
  if (padding < 0) {
    const double ext = std::max(mx[0] - mn[0], std::max(mx[1] - mn[1], mx[2] - mn[2]));
    const double k = res >= 8 ? 2 : 1;
    padding = (k * ext) / (res - 2 * k);
  }
  for (int a = 0; a < 3; ++a) {
    mn[a] -= padding;
    mx[a] += padding;
  }
  const double side = std::max(mx[0] - mn[0], std::max(mx[1] - mn[1], mx[2] - mn[2]));
  const double vs = side / res;
  for (int a = 0; a < 3; ++a) origin[a] = 0.5 * (mn[a] + mx[a]) - 0.5 * side;
  *voxel = vs;
  const double jit = vs * 1e-4, ja = jit * 1.4142135623730951, jb = jit * 3.141592653589793;
  uint64_t bad = 0;
  for (uint32_t z = 0; z < res; ++z)
    for (uint32_t y = 0; y < res; ++y)
      for (uint32_t x = 0; x < res; ++x) {
        const double p[3] = {origin[0] + (x + 0.5) * vs, origin[1] + (y + 0.5) * vs, origin[2] + (z + 0.5) * vs};
        double best = INFINITY;
        for (const Tri& T : tris) {
          double d[3];
          for (int a = 0; a < 3; ++a) d[a] = p[a] < T.lo[a] ? T.lo[a] - p[a] : (p[a] > T.hi[a] ? p[a] - T.hi[a] : 0);
          if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] >= best) continue;
          const double e = tri_d2(p, T);
          if (e < best) best = e;
        }
        const double px[3] = {p[0], p[1] + ja, p[2] + jb}, py[3] = {p[0] + jb, p[1], p[2] + ja},
                     pz[3] = {p[0] + ja, p[1] + jb, p[2]};
        const int votes = (int)(axis_hits(px, 0, tris) & 1) + (int)(axis_hits(py, 1, tris) & 1) +
                          (int)(axis_hits(pz, 2, tris) & 1);
        if (votes == 1 || votes == 2) ++bad;
        const double dist = std::sqrt(best);
        data[x + (size_t)res * (y + (size_t)res * z)] = (float)(votes >= 2 ? -dist : dist);
      }
  *inconsistent = bad;
  return 0;
}

}  // extern "C"
