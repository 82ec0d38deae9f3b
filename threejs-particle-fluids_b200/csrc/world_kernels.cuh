// world_kernels.cuh — device helpers shared by the solver stage kernels:
// SPH kernels, primitive SDFs, fixed-point accumulation, 3x3 polar
// decomposition and the 27-cell stencil walk over the sorted slots.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "world.cuh"

namespace pf {

__device__ __forceinline__ uint32_t lane_of() { return threadIdx.x & 31u; }

__device__ __forceinline__ const DevScene& scene_at(const WorldView& V, uint32_t slot) {
  return V.scenes[V.chunk_scene[slot >> 8]];
}
__device__ __forceinline__ uint32_t scene_index(const WorldView& V, uint32_t slot) {
  return V.chunk_scene[slot >> 8];
}
// Slot of the g-th slot of a chunk list (launch index g over its chunks).
__device__ __forceinline__ uint32_t chunk_slot(const uint32_t* __restrict__ list, uint32_t g) {
  return __ldg(list + g / kSegAlign) * kSegAlign + g % kSegAlign;
}

// ----------------------------------------------------------- vector math ----
struct f3 {
  float x, y, z;
};
__device__ __forceinline__ f3 mk(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ f3 xyz(float4 a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ f3 operator+(f3 a, f3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ f3 operator-(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ f3 operator*(f3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ f3 operator/(f3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ f3 neg(f3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ f3 cross(f3 a, f3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float len(f3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float4 with_w(f3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

// |a|^2 without fused multiply-add: the neighbour-list acceptance test must
// round exactly like the reference's separately rounded products and sums.
__device__ __forceinline__ float dot_rn(f3 a) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)), __fmul_rn(a.z, a.z));
}
__device__ __forceinline__ float dot_rn(f3 a, f3 b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
// dot_rn(xi - xj) with the x and y lanes in packed f32x2 operations (each
// lane rounded as its scalar form, so the result is the same bits): the
// list build's acceptance test.
__device__ __forceinline__ float dist2_rn(f3 xi, float4 xj) {
  float r;
  asm("{\n\t.reg .b64 a, b, d;\n\t.reg .f32 sx, sy, dz;\n\t"
      "mov.b64 a, {%1, %2};\n\tmov.b64 b, {%4, %5};\n\t"
      "sub.rn.f32x2 d, a, b;\n\tmul.rn.f32x2 d, d, d;\n\t"
      "mov.b64 {sx, sy}, d;\n\tadd.rn.f32 sx, sx, sy;\n\t"
      "sub.rn.f32 dz, %3, %6;\n\tmul.rn.f32 dz, dz, dz;\n\tadd.rn.f32 %0, sx, dz;\n\t}"
      : "=f"(r)
      : "f"(xi.x), "f"(xi.y), "f"(xi.z), "f"(xj.x), "f"(xj.y), "f"(xj.z));
  return r;
}

// collider.ts:53-89, the static-friction cone of one contact: the slip's
// tangential part and whether the particle sticks (the tangential
// displacement fits the remaining budget mu_s * lambda_n - lambda_t). A
// sticking particle returns to where it was, a sliding one keeps its slip, so
// the decision is a step: it is formed with separately rounded products and
// sums, as the reference's arithmetic rounds them.
struct StickTest {
  f3 tang;
  float tl;
  bool sticks;
};
__device__ __forceinline__ StickTest stick_test(f3 slip, f3 nrm, float w, float mu_s, float ln, float lt) {
  const float sn = dot_rn(slip, nrm);
  StickTest r;
  r.tang = mk(__fsub_rn(slip.x, __fmul_rn(nrm.x, sn)), __fsub_rn(slip.y, __fmul_rn(nrm.y, sn)),
              __fsub_rn(slip.z, __fmul_rn(nrm.z, sn)));
  r.tl = __fsqrt_rn(dot_rn(r.tang));
  r.sticks = r.tl > 1e-10f && (__fdiv_rn(r.tl, w) <= __fsub_rn(__fmul_rn(mu_s, ln), lt));
  return r;
}

// ------------------------------------------------------------ SPH kernels ----
// sph/kernels.ts:254-298
__device__ __forceinline__ float poly6(float rsq, const DevFluid& F) {
  const float d = fmaxf(F.hsq - rsq, 0.0f);
  return d * d * d * F.poly6;
}
__device__ __forceinline__ f3 spiky_grad(f3 r, const DevFluid& F) {
  const float rl = sqrtf(dot(r, r));
  const float t = fmaxf(F.h - rl, 0.0f);
  const float rs = fmaxf(rl, 1e-20f);
  const f3 rhat = r / rs;
  const float mag = -(t * t * F.spiky);
  return rhat * mag;
}
// shared.ts:52-62: the neighbour's SPH mass (boundary psi = rho0 * V).
__device__ __forceinline__ float neighbor_mass(float bv, float w, float rho0) {
  return bv > 0.0f ? rho0 * bv : (w > 0.0f ? 1.0f / w : 0.0f);
}

// The mass code of a slot (its lm.y): the boundary volume of a boundary
// particle, minus its own mass otherwise; and the mass a fluid with rest
// density rho0 sees from it.
__device__ __forceinline__ float mass_code(float bv, float w) {
  return bv > 0.0f ? bv : -(w > 0.0f ? 1.0f / w : 0.0f);
}
__device__ __forceinline__ float code_mass(float q, float rho0) { return q > 0.0f ? rho0 * q : -q; }

// The same quantities in the form the per-neighbour loops use: one
// reciprocal square root instead of a square root and three divisions, and
// an approximate reciprocal for the particle mass. Within the solver's
// tolerance of the exactly rounded forms above.
__device__ __forceinline__ float neighbor_mass_fast(float bv, float w, float rho0) {
  return bv > 0.0f ? rho0 * bv : (w > 0.0f ? __fdividef(1.0f, w) : 0.0f);
}
// -45/(pi h^6) (h - r)^2 / r, the factor that turns r_vec into the Spiky
// gradient; zero at r = 0 (rsqrt of the floored square stays finite).
__device__ __forceinline__ float spiky_factor(float rsq, const DevFluid& F) {
  const float inv_r = rsqrtf(fmaxf(rsq, 1e-40f));
  const float t = fmaxf(F.h - rsq * inv_r, 0.0f);
  return -(t * t * F.spiky) * inv_r;
}

// (h - r)^2 / r from r^2, without the -45/(pi h^6) constant (the slot
// kernels apply it once to their sums): zero at r = 0.
__device__ __forceinline__ float spiky_shape(float rsq, const DevFluid& F) {
  const float inv_r = rsqrtf(fmaxf(rsq, 1e-40f));
  const float t = fmaxf(F.h - rsq * inv_r, 0.0f);
  return t * t * inv_r;
}

// The forms the neighbour loops call. A build with PF_EXACT_ROUNDING (and
// -fmad=false) uses the exactly rounded reference forms instead; it is a
// diagnostic build that reproduces the oracle's FP32 arithmetic bit for bit.
#ifdef PF_EXACT_ROUNDING
__device__ __forceinline__ float nbr_mass(float bv, float w, float rho0) { return neighbor_mass(bv, w, rho0); }
__device__ __forceinline__ f3 spiky_vec(f3 off, float, const DevFluid& F) { return spiky_grad(off, F); }
#else
__device__ __forceinline__ float nbr_mass(float bv, float w, float rho0) { return neighbor_mass_fast(bv, w, rho0); }
__device__ __forceinline__ f3 spiky_vec(f3 off, float rsq, const DevFluid& F) { return off * spiky_factor(rsq, F); }
#endif

// ------------------------------------------------- fixed-point accumulation ----
// accumulator.ts:108-115: round(v * scale) with ties to even, saturating.
__device__ __forceinline__ int to_ticks(float v, float scale) { return __float2int_rn(v * scale); }
__device__ __forceinline__ void acc_add(int4* acc, uint32_t slot, f3 v, float scale) {
  int* p = reinterpret_cast<int*>(acc + slot);
  atomicAdd(p + 0, to_ticks(v.x, scale));
  atomicAdd(p + 1, to_ticks(v.y, scale));
  atomicAdd(p + 2, to_ticks(v.z, scale));
}
// accumulator.ts:148-178: ticks -> float change, saturation test, clear.
__device__ __forceinline__ f3 ticks_change(int tx, int ty, int tz, float inv, bool* sat) {
  const float fx = (float)tx, fy = (float)ty, fz = (float)tz;
  const float m = fmaxf(fmaxf(fabsf(fx), fabsf(fy)), fabsf(fz));
  if (m >= 1073741824.0f) *sat = true;
  return mk(fx * inv, fy * inv, fz * inv);
}

// --------------------------------------------------------- grid stencil ----
__device__ __forceinline__ int32_t cell_of(float p, float o, float cell) {
  return __float2int_rz(floorf(__fdiv_rn(__fsub_rn(p, o), cell)));
}

__device__ __forceinline__ int32_t clampi(int64_t v, int32_t lo, int32_t hi) {
  return (int32_t)(v < lo ? lo : (v > hi ? hi : v));
}

// Cell coordinates outside the reference's Morton range raise its grid
// overflow flag (cellIndex.ts:145-169, mortonHash.ts:71-79: bias 512).
constexpr int32_t kMortonBias = 512;
__device__ __forceinline__ bool morton_over(int32_t c) { return c < -kMortonBias || c >= kMortonBias; }

// Local (grid) cell of a position, clamped into the grid window; `clamped`
// reports a clamp, `ref_over` a cell the reference's hash flags.
__device__ __forceinline__ void local_cell(const DevScene& S, f3 p, int32_t* cx, int32_t* cy, int32_t* cz,
                                           bool* clamped, bool* ref_over = nullptr) {
  const int32_t rx = cell_of(p.x, S.ox, S.cell), ry = cell_of(p.y, S.oy, S.cell), rz = cell_of(p.z, S.oz, S.cell);
  const int64_t ax = (int64_t)rx - S.lo[0];
  const int64_t ay = (int64_t)ry - S.lo[1];
  const int64_t az = (int64_t)rz - S.lo[2];
  *cx = clampi(ax, 0, (int32_t)S.dims[0] - 1);
  *cy = clampi(ay, 0, (int32_t)S.dims[1] - 1);
  *cz = clampi(az, 0, (int32_t)S.dims[2] - 1);
  if (clamped) *clamped = (*cx != ax) || (*cy != ay) || (*cz != az);
  if (ref_over) *ref_over = morton_over(rx) || morton_over(ry) || morton_over(rz);
}

// Adds the cells of this block's positions (`in` lanes) to the scene's
// bounds (V.bbox[6 s ...]): a block reduction, then six atomics. Every
// thread of the block must call it; the block belongs to scene s.
__device__ __forceinline__ void bbox_block_add(const WorldView& V, const DevScene& S, uint32_t s, bool in, f3 p) {
  __shared__ int32_t sb[kBlock / 32][6];
  int32_t c[6];
  if (in) {
    c[0] = c[3] = cell_of(p.x, S.ox, S.cell);
    c[1] = c[4] = cell_of(p.y, S.oy, S.cell);
    c[2] = c[5] = cell_of(p.z, S.oz, S.cell);
  } else {
    c[0] = c[1] = c[2] = INT32_MAX;
    c[3] = c[4] = c[5] = INT32_MIN;
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    c[a] = __reduce_min_sync(0xffffffffu, c[a]);
    c[a + 3] = __reduce_max_sync(0xffffffffu, c[a + 3]);
  }
  const uint32_t w = threadIdx.x >> 5;
  if ((threadIdx.x & 31u) == 0)
#pragma unroll
    for (int a = 0; a < 6; ++a) sb[w][a] = c[a];
  __syncthreads();
  if (threadIdx.x < 6) {
    const int a = (int)threadIdx.x;
    int32_t v = sb[0][a];
    for (uint32_t q = 1; q < blockDim.x / 32; ++q) v = a < 3 ? min(v, sb[q][a]) : max(v, sb[q][a]);
    if (a < 3 ? v != INT32_MAX : v != INT32_MIN) {
      if (a < 3) atomicMin(V.bbox + 6 * s + a, v);
      else atomicMax(V.bbox + 6 * s + a, v);
    }
  }
}

// Visit the sorted slots of the 27 cells around p in the reference's order
// (query.ts:37-66: dz, dy, dx; within a cell ascending particle index). With
// linear keys the three cells of one (dy, dz) row are consecutive keys, so a
// row is one contiguous slot range. fn(slot) returns false to stop early.
template <typename F>
__device__ __forceinline__ void walk27(const DevScene& S, const uint32_t* __restrict__ cstart,
                                       const uint32_t* __restrict__ ccount, f3 p, F&& fn) {
  int32_t cx, cy, cz;
  local_cell(S, p, &cx, &cy, &cz, nullptr);
  const int32_t x0 = max(cx - 1, 0), x1 = min(cx + 1, (int32_t)S.dims[0] - 1);
  for (int dz = -1; dz <= 1; ++dz) {
    const int32_t z = cz + dz;
    if (z < 0 || z >= (int32_t)S.dims[2]) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int32_t y = cy + dy;
      if (y < 0 || y >= (int32_t)S.dims[1]) continue;
      const uint32_t row = S.cell_base + S.dims[0] * ((uint32_t)y + S.dims[1] * (uint32_t)z);
      const uint32_t k0 = row + (uint32_t)x0, k1 = row + (uint32_t)x1;
      const uint32_t s0 = __ldg(cstart + k0);
      const uint32_t s1 = __ldg(cstart + k1) + __ldg(ccount + k1);
      for (uint32_t j = s0; j < s1; ++j)
        if (!fn(j)) return;
    }
  }
}

// ------------------------------------------------------------ quaternions ----
__device__ __forceinline__ f3 qrot(float4 q, f3 v) {
  const f3 qv = mk(q.x, q.y, q.z);
  const f3 t = cross(qv, v) * 2.0f;
  return v + t * q.w + cross(qv, t);
}

// ------------------------------------------------------ primitive SDFs ----
// primitives.ts:158-171
__device__ __forceinline__ f3 prim_pivot(const pf_primitive& p) {
  const f3 d0 = mk(p.data0[0], p.data0[1], p.data0[2]);
  const f3 d1 = mk(p.data1[0], p.data1[1], p.data1[2]);
  if (p.kind == PF_PRIM_PLANE) return d1;
  if (p.kind == PF_PRIM_CAPSULE) return (d0 + d1) * 0.5f;
  return d0;
}

// primitives.ts:203-335 with the PrimitiveSet fields (velocity and spin).
__device__ __forceinline__ void prim_sdf(const pf_primitive& p, f3 xw, float rewind, float* phi_out, f3* grad_out) {
  if (p.kind == PF_PRIM_PLANE && !(p.flags & PF_PRIM_SWEEP) && p.spin[0] == 0.0f && p.spin[1] == 0.0f &&
      p.spin[2] == 0.0f) {
    // an unswept, unspun plane: the general path below with t = 0 and the
    // identity turn, term for term (x = pivot + (x_w - pivot))
    const f3 d0 = mk(p.data0[0], p.data0[1], p.data0[2]);
    const f3 d1 = mk(p.data1[0], p.data1[1], p.data1[2]);
    const f3 x = d1 + ((xw + mk(p.velocity[0], p.velocity[1], p.velocity[2]) * 0.0f) - d1);
    const float phi = dot_rn(d0, x - d1);
    const bool inv = (p.flags & PF_PRIM_INVERT) != 0;
    *phi_out = inv ? -phi : phi;
    *grad_out = inv ? neg(d0) : d0;
    return;
  }
  const float t = (p.flags & PF_PRIM_SWEEP) ? rewind : 0.0f;
  const f3 shifted = xw + mk(p.velocity[0], p.velocity[1], p.velocity[2]) * t;
  const f3 pivot = prim_pivot(p);
  const f3 spin = mk(p.spin[0], p.spin[1], p.spin[2]);
  const float rate = len(spin);
  const float half = rate * t * 0.5f;
  float4 turn = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
  f3 x;
  if (half != 0.0f) {
    const f3 axis = spin / fmaxf(rate, 1e-8f);
    float sh, ch;
    sincosf(half, &sh, &ch);
    turn = make_float4(axis.x * sh, axis.y * sh, axis.z * sh, ch);
    x = pivot + qrot(turn, shifted - pivot);
  } else {
    // rotating by the identity quaternion returns its argument exactly
    x = pivot + (shifted - pivot);
  }
  const float4 unturn = make_float4(-turn.x, -turn.y, -turn.z, turn.w);
  const f3 d0 = mk(p.data0[0], p.data0[1], p.data0[2]);
  const f3 d1 = mk(p.data1[0], p.data1[1], p.data1[2]);
  float phi = 0.0f;
  f3 g = mk(0.0f, 0.0f, 0.0f);
  if (p.kind == PF_PRIM_PLANE) {
    phi = dot(d0, x - d1);
    g = d0;
  } else if (p.kind == PF_PRIM_SPHERE) {
    const f3 diff = x - d0;
    const float l = len(diff);
    phi = l - p.data0[3];
    g = diff / fmaxf(l, 1e-8f);
  } else if (p.kind == PF_PRIM_BOX) {
    const float4 rot = make_float4(p.rotation[0], p.rotation[1], p.rotation[2], p.rotation[3]);
    const float4 conj = make_float4(-rot.x, -rot.y, -rot.z, rot.w);
    const f3 xl = qrot(conj, x - d0);
    const f3 q = mk(fabsf(xl.x), fabsf(xl.y), fabsf(xl.z)) - d1;
    const f3 qp = mk(fmaxf(q.x, 0.0f), fmaxf(q.y, 0.0f), fmaxf(q.z, 0.0f));
    const float outside = len(qp);
    const float inside = fminf(fmaxf(fmaxf(q.x, q.y), q.z), 0.0f);
    phi = outside + inside;
    const f3 sg = mk(xl.x >= 0.0f ? 1.0f : -1.0f, xl.y >= 0.0f ? 1.0f : -1.0f, xl.z >= 0.0f ? 1.0f : -1.0f);
    const bool is_out = outside > 1e-8f;
    const bool dx = q.x >= q.y && q.x >= q.z;
    const bool dy = q.y >= q.x && q.y >= q.z;
    const f3 in_dir = mk(dx ? sg.x : 0.0f, (!dx && dy) ? sg.y : 0.0f, (!dx && !dy) ? sg.z : 0.0f);
    const f3 lg = is_out ? mk(qp.x * sg.x, qp.y * sg.y, qp.z * sg.z) / fmaxf(outside, 1e-8f) : in_dir;
    g = qrot(rot, lg);
  } else if (p.kind == PF_PRIM_CAPSULE) {
    const f3 ab = d1 - d0;
    const f3 ax = x - d0;
    const float ab2 = fmaxf(dot(ab, ab), 1e-8f);
    const float tt = fminf(fmaxf(dot(ax, ab) / ab2, 0.0f), 1.0f);
    const f3 closest = d0 + ab * tt;
    const f3 diff = x - closest;
    const float l = len(diff);
    phi = l - p.data0[3];
    g = diff / fmaxf(l, 1e-8f);
  }
  if (p.flags & PF_PRIM_INVERT) {
    phi = -phi;
    g = neg(g);
  }
  *phi_out = phi;
  *grad_out = half != 0.0f ? qrot(unturn, g) : g;
}

// primitives.ts:342-360
__device__ __forceinline__ f3 prim_surface_velocity(const pf_primitive& p, f3 xw, float rewind) {
  const f3 vel = mk(p.velocity[0], p.velocity[1], p.velocity[2]);
  const float t = (p.flags & PF_PRIM_SWEEP) ? rewind : 0.0f;
  const f3 arm = (xw - prim_pivot(p)) + vel * t;
  return vel + cross(mk(p.spin[0], p.spin[1], p.spin[2]), arm);
}

// -------------------------------------------------- polar decomposition ----
// polarDecomp.ts:34-264: Jacobi on A^T A (8 sweeps over the (0,1), (0,2),
// (1,2) planes), S^-1 = Q diag(1/sqrt(lambda)) Q^T, R = A S^-1. All in
// registers.
__device__ __forceinline__ void jacobi_coeffs(float app, float aqq, float apq, float* t, float* c, float* s) {
  const float tau = (aqq - app) / (apq * 2.0f);
  const float sg = tau >= 0.0f ? 1.0f : -1.0f;
  const float ta = fabsf(tau);
  *t = sg / (ta + sqrtf(ta * ta + 1.0f));
  *c = 1.0f / sqrtf(*t * *t + 1.0f);
  *s = *t * *c;
}

// sample.ts:12-53 trilinear filter at continuous grid coordinate g (voxel
// (i, j, k) centred at g = (i + 0.5, j + 0.5, k + 0.5)), clamp to edge.
__device__ __forceinline__ float sdf_trilinear(const uint16_t* __restrict__ d, const DevSdf& G, float gx, float gy,
                                               float gz) {
  gx -= 0.5f;
  gy -= 0.5f;
  gz -= 0.5f;
  const int nx = (int)G.res[0], ny = (int)G.res[1], nz = (int)G.res[2];
  const int i0 = min(max((int)floorf(gx), 0), nx - 2);
  const int j0 = min(max((int)floorf(gy), 0), ny - 2);
  const int k0 = min(max((int)floorf(gz), 0), nz - 2);
  const float tx = fminf(fmaxf(gx - (float)i0, 0.0f), 1.0f);
  const float ty = fminf(fmaxf(gy - (float)j0, 0.0f), 1.0f);
  const float tz = fminf(fmaxf(gz - (float)k0, 0.0f), 1.0f);
  const size_t sy = (size_t)nx, sz = (size_t)nx * ny;
  const uint16_t* b = d + G.data_off + (size_t)i0 + j0 * sy + k0 * sz;
  auto h = [](uint16_t v) { return __half2float(__ushort_as_half(v)); };
  auto lerp = [](float a, float c, float t) { return a + (c - a) * t; };
  const float c00 = lerp(h(__ldg(b)), h(__ldg(b + 1)), tx);
  const float c10 = lerp(h(__ldg(b + sy)), h(__ldg(b + sy + 1)), tx);
  const float c01 = lerp(h(__ldg(b + sz)), h(__ldg(b + sz + 1)), tx);
  const float c11 = lerp(h(__ldg(b + sz + sy)), h(__ldg(b + sz + sy + 1)), tx);
  return lerp(lerp(c00, c10, ty), lerp(c01, c11, ty), tz);
}

// sdf.ts:107-147 (emitSampleSdf): world -> local frame, phi by the trilinear
// filter, the gradient by central differences one voxel apart, back to world.
__device__ __forceinline__ void sdf_sample(const uint16_t* __restrict__ d, const DevSdf& G, f3 x, float* phi,
                                           f3* grad) {
  const f3 off = mk(x.x - G.position[0], x.y - G.position[1], x.z - G.position[2]);
  const float* I = G.inv_rot;
  const f3 xl = mk(I[0] * off.x + I[1] * off.y + I[2] * off.z, I[3] * off.x + I[4] * off.y + I[5] * off.z,
                   I[6] * off.x + I[7] * off.y + I[8] * off.z) *
                G.inv_scale;
  const float gx = (xl.x - G.origin[0]) * G.inv_voxel[0];
  const float gy = (xl.y - G.origin[1]) * G.inv_voxel[1];
  const float gz = (xl.z - G.origin[2]) * G.inv_voxel[2];
  const float p0 = sdf_trilinear(d, G, gx, gy, gz);
  const f3 gl = mk((sdf_trilinear(d, G, gx + 1.0f, gy, gz) - sdf_trilinear(d, G, gx - 1.0f, gy, gz)) / (2.0f * G.voxel[0]),
                   (sdf_trilinear(d, G, gx, gy + 1.0f, gz) - sdf_trilinear(d, G, gx, gy - 1.0f, gz)) / (2.0f * G.voxel[1]),
                   (sdf_trilinear(d, G, gx, gy, gz + 1.0f) - sdf_trilinear(d, G, gx, gy, gz - 1.0f)) / (2.0f * G.voxel[2]));
  const float* R = G.rot;
  *phi = p0 * G.scale;
  *grad = mk(R[0] * gl.x + R[1] * gl.y + R[2] * gl.z, R[3] * gl.x + R[4] * gl.y + R[5] * gl.z,
             R[6] * gl.x + R[7] * gl.y + R[8] * gl.z);
}

__device__ __forceinline__ void polar3(const float a[9], float r[9]) {
  float m00 = a[0] * a[0] + a[3] * a[3] + a[6] * a[6];
  float m01 = a[0] * a[1] + a[3] * a[4] + a[6] * a[7];
  float m02 = a[0] * a[2] + a[3] * a[5] + a[6] * a[8];
  float m11 = a[1] * a[1] + a[4] * a[4] + a[7] * a[7];
  float m12 = a[1] * a[2] + a[4] * a[5] + a[7] * a[8];
  float m22 = a[2] * a[2] + a[5] * a[5] + a[8] * a[8];
  float q00 = 1, q01 = 0, q02 = 0, q10 = 0, q11 = 1, q12 = 0, q20 = 0, q21 = 0, q22 = 1;
  const float eps = 1e-12f;
#pragma unroll 1
  for (int sweep = 0; sweep < 8; ++sweep) {
    if (fabsf(m01) > eps) {
      float t, c, s;
      const float apq = m01, app = m00, aqq = m11;
      jacobi_coeffs(app, aqq, apq, &t, &c, &s);
      const float o02 = m02, o12 = m12, a0 = q00, a1 = q01, b0 = q10, b1 = q11, c0 = q20, c1 = q21;
      m00 = app - t * apq;
      m11 = aqq + t * apq;
      m01 = 0.0f;
      m02 = c * o02 - s * o12;
      m12 = s * o02 + c * o12;
      q00 = c * a0 - s * a1;
      q01 = s * a0 + c * a1;
      q10 = c * b0 - s * b1;
      q11 = s * b0 + c * b1;
      q20 = c * c0 - s * c1;
      q21 = s * c0 + c * c1;
    }
    if (fabsf(m02) > eps) {
      float t, c, s;
      const float apq = m02, app = m00, aqq = m22;
      jacobi_coeffs(app, aqq, apq, &t, &c, &s);
      const float o01 = m01, o12 = m12, a0 = q00, a2 = q02, b0 = q10, b2 = q12, c0 = q20, c2 = q22;
      m00 = app - t * apq;
      m22 = aqq + t * apq;
      m02 = 0.0f;
      m01 = c * o01 - s * o12;
      m12 = s * o01 + c * o12;
      q00 = c * a0 - s * a2;
      q02 = s * a0 + c * a2;
      q10 = c * b0 - s * b2;
      q12 = s * b0 + c * b2;
      q20 = c * c0 - s * c2;
      q22 = s * c0 + c * c2;
    }
    if (fabsf(m12) > eps) {
      float t, c, s;
      const float apq = m12, app = m11, aqq = m22;
      jacobi_coeffs(app, aqq, apq, &t, &c, &s);
      const float o01 = m01, o02 = m02, a1 = q01, a2 = q02, b1 = q11, b2 = q12, c1 = q21, c2 = q22;
      m11 = app - t * apq;
      m22 = aqq + t * apq;
      m12 = 0.0f;
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
  const float i0 = 1.0f / sqrtf(fmaxf(m00, 1e-20f));
  const float i1 = 1.0f / sqrtf(fmaxf(m11, 1e-20f));
  const float i2 = 1.0f / sqrtf(fmaxf(m22, 1e-20f));
  const float s00 = q00 * q00 * i0 + q01 * q01 * i1 + q02 * q02 * i2;
  const float s01 = q00 * q10 * i0 + q01 * q11 * i1 + q02 * q12 * i2;
  const float s02 = q00 * q20 * i0 + q01 * q21 * i1 + q02 * q22 * i2;
  const float s11 = q10 * q10 * i0 + q11 * q11 * i1 + q12 * q12 * i2;
  const float s12 = q10 * q20 * i0 + q11 * q21 * i1 + q12 * q22 * i2;
  const float s22 = q20 * q20 * i0 + q21 * q21 * i1 + q22 * q22 * i2;
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

// The colliders of particle k's scene against its predicted position xs4
// (w = inverse mass), their multipliers updated; the fixed-point position
// changes summed in registers, on top of the ticks `start` that particle
// contacts scattered for k, and applied. Returns whether xs4 changed.
__device__ __forceinline__ bool collide_particle(const WorldView& V, const DevScene& S, uint32_t s, uint32_t k,
                                                 float4& xs4, const pf_primitive* __restrict__ prims,
                                                 int4 start = make_int4(0, 0, 0, 0)) {
  const float w = xs4.w;
  const bool moves = w > 0.0f;
  const uint32_t n_prim = moves ? S.prim_count : 0u, n_sdf = moves ? S.sdf_count : 0u;
  const f3 xstar = xyz(xs4);
  // the displacement this substep, read on the first contact only (most
  // particles touch no collider)
  f3 disp_v = mk(0.0f, 0.0f, 0.0f);
  bool have_disp = false;
  auto disp = [&]() {
    if (!have_disp) {
      disp_v = xstar - xyz(V.cur.x[k]);
      have_disp = true;
    }
    return disp_v;
  };
  // collider multipliers: entry i < 32 is valid once bit i of the slot's
  // mask is set this substep (zero before)
  uint32_t mask = n_prim + n_sdf ? V.cmask[k] : 0u;
  const uint32_t mask0 = mask;
  auto lam_at = [&](uint32_t i) {
    return (i >= 32 || ((mask >> i) & 1u)) ? V.plam[(size_t)k * V.prim_stride + i] : make_float2(0.0f, 0.0f);
  };
  auto lam_put = [&](uint32_t i, float2 lam) {
    V.plam[(size_t)k * V.prim_stride + i] = lam;
    if (i < 32) mask |= 1u << i;
  };
  const float clock = V.clocks[s];
  const float radius = S.radius;
  uint32_t tx = (uint32_t)start.x, ty = (uint32_t)start.y, tz = (uint32_t)start.z;
  bool any = (start.x | start.y | start.z) != 0;
  for (uint32_t p = 0; p < n_prim; ++p) {
    float phi;
    f3 nrm;
    if (S.planes_fast) {
      // prim_sdf's unswept plane, term for term, from the compact table
      const float4 a = __ldg(V.plane4 + 2 * ((size_t)S.prim_base + p));
      const float4 b = __ldg(V.plane4 + 2 * ((size_t)S.prim_base + p) + 1);
      const f3 d0 = xyz(a), d1 = xyz(b);
      const f3 x = d1 + (xstar - d1);
      const float ph = dot_rn(d0, x - d1);
      const bool inv = a.w != 0.0f;
      phi = inv ? -ph : ph;
      nrm = inv ? neg(d0) : d0;
    } else {
      prim_sdf(prims[p], xstar, clock, &phi, &nrm);
    }
    if (!(phi < radius)) continue;
    const pf_primitive& P = prims[p];
    const f3 coldisp = prim_surface_velocity(P, xstar, clock) * S.dt;
    const float depth = radius - phi;
    float2 lam = lam_at(p);
    const float ln = lam.x + depth / w;
    const f3 slip = disp() - coldisp;
    const StickTest st = stick_test(slip, nrm, w, P.data1[3], ln, lam.y);
    const bool sticks = st.sticks;
    const float tl = st.tl;
    const f3 push = nrm * depth;
    const f3 c = sticks ? push - st.tang : push;
    tx += (uint32_t)to_ticks(c.x, S.pos_scale);
    ty += (uint32_t)to_ticks(c.y, S.pos_scale);
    tz += (uint32_t)to_ticks(c.z, S.pos_scale);
    lam.x = ln;
    lam.y = lam.y + (sticks ? tl / w : 0.0f);
    lam_put(p, lam);
    any = true;
  }
  // SDFCollider.ts:256-281: static surface, reach = radius + thickness
  for (uint32_t q = 0; q < n_sdf; ++q) {
    const DevSdf& G = V.sdfs[S.sdf_base + q];
    float phi;
    f3 g;
    sdf_sample(V.sdf_half, G, xstar, &phi, &g);
    const float gl = len(g);
    if (!(gl > 1e-6f)) continue;
    const float reach = radius + G.thickness;
    if (!(phi < reach)) continue;
    const f3 nrm = g / gl;
    const float depth = reach - phi;
    const uint32_t li = S.prim_count + q;
    float2 lam = lam_at(li);
    const float ln = lam.x + depth / w;
    const StickTest st = stick_test(disp(), nrm, w, G.mu_s, ln, lam.y);
    const bool sticks = st.sticks;
    const float tl = st.tl;
    const f3 push = nrm * depth;
    const f3 c = sticks ? push - st.tang : push;
    tx += (uint32_t)to_ticks(c.x, S.pos_scale);
    ty += (uint32_t)to_ticks(c.y, S.pos_scale);
    tz += (uint32_t)to_ticks(c.z, S.pos_scale);
    lam.x = ln;
    lam.y = lam.y + (sticks ? tl / w : 0.0f);
    lam_put(li, lam);
    any = true;
  }
  if (mask != mask0) V.cmask[k] = mask;
  if (!any) return false;
  bool sat = false;
  const f3 c = ticks_change((int)tx, (int)ty, (int)tz, S.pos_inv, &sat);
  xs4 = with_w(xstar + c, w);
  if (sat) atomicOr(V.flags + s * kNumFlags + FLAG_POS, 1u);
  return true;
}

}  // namespace pf
