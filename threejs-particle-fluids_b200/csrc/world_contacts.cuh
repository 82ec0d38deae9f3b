// Particle-particle contacts (src/core/contact/generate.ts, solve.ts,
// ContactBuffer.ts; scheduled by loop.ts:180-242, 347-417).
//
// The reference appends pairs to one buffer through an atomic counter, so
// its pair order (and, past maxContacts, which pairs it drops) is whatever
// order the threads reach the counter. Here every emitting slot keeps its own
// partner list (column-major, entry m of slot k at m * n + k, at most
// kMaxContacts), and a per-scene prefix over the slots numbers the pairs in
// slot order: the first max_contacts pairs of that order are solved. Each
// pair's multipliers and normal belong to the one thread of its emitting
// slot, and the position and velocity corrections are fixed-point sums, so
// the results do not depend on which side of a pair emits it (swapping the
// pair negates every vector exactly) nor on the order of the atomic adds.
#pragma once

#include "world_kernels.cuh"

namespace pf {

// ContactBuffer.ts:16: multipliers are kept in ticks of 2^-20 kg m.
constexpr float kLambdaScale = 1048576.0f;
constexpr float kLambdaInv = 1.0f / 1048576.0f;
// generate.ts:20
constexpr double kContactRadiusExpansion = 1.1;

// f32 -> i32 toward zero, saturating (the shader's toInt()).
__device__ __forceinline__ int lam_ticks(float v) { return __float2int_rz(v * kLambdaScale); }

// Exclusive prefix of v over the block (blockDim.x a multiple of 32, at most
// 1024); *total receives the block's sum. `ws` holds 32 words.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t v, uint32_t* ws, uint32_t* total) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t inc = v;
#pragma unroll
  for (uint32_t d = 1; d < 32; d <<= 1) {
    const uint32_t o = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += o;
  }
  if (lane == 31) ws[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = lane < nw ? ws[lane] : 0u;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_up_sync(0xffffffffu, t, d);
      if (lane >= d) t += o;
    }
    ws[lane] = t;  // inclusive prefix of the warp totals
  }
  __syncthreads();
  const uint32_t before = warp ? ws[warp - 1] : 0u;
  *total = ws[nw - 1];
  __syncthreads();  // ws is reused by the caller
  return before + inc - v;
}

// generate.ts:53-88: each slot outside the noSelfContacts ranges walks the 27
// cells around its predicted position and keeps every partner closer than
// 2r * 1.1, outside its non-zero collision group, not both pinned; a pair of
// two emitting slots is kept by the lower slot. The block is one 256-slot
// chunk: it also forms the slots' prefix inside the chunk and the chunk's sum.
__global__ void __launch_bounds__(kBlock) k_con_gen(WorldView V, uint32_t sub) {
  __shared__ uint32_t ws[32];
  const uint32_t k = blockIdx.x * kBlock + threadIdx.x;  // the grid covers n exactly
  const DevScene& S = scene_at(V, k);
  uint32_t cnt = 0;
  if (S.contact && sub < S.substeps) {
    const uint32_t id = V.ids[k];
    if (id < S.seg_start + S.cap && !V.cquiet[id]) {
      const float4 xi4 = V.cur.xs[k];
      const f3 xi = xyz(xi4);
      const float wi = xi4.w;
      const uint32_t gi = V.cgroup[id];
      const size_t n = V.n;
      int32_t cx, cy, cz;
      local_cell(S, xi, &cx, &cy, &cz, nullptr);
      const int32_t x0 = max(cx - 1, 0), x1 = min(cx + 1, (int32_t)S.dims[0] - 1);
      for (int r = 0; r < 9; ++r) {
        const int32_t z = cz + r / 3 - 1, y = cy + r % 3 - 1;
        if (z < 0 || z >= (int32_t)S.dims[2] || y < 0 || y >= (int32_t)S.dims[1]) continue;
        const uint32_t row = S.cell_base + S.dims[0] * ((uint32_t)y + S.dims[1] * (uint32_t)z);
        const uint32_t e = V.cstart[row + x1] + V.ccount[row + x1];
        for (uint32_t j = V.cstart[row + x0]; j < e; ++j) {
          if (j == k) continue;
          const float4 xj = V.cur.xs[j];
          const f3 d = xi - xyz(xj);
          if (dot(d, d) >= S.c_cand2) continue;
          const uint32_t jd = V.ids[j];
          if (jd >= S.seg_start + S.cap) continue;
          if (!V.cquiet[jd] && j < k) continue;
          if (gi != 0u && gi == V.cgroup[jd]) continue;
          if (wi <= 0.0f && xj.w <= 0.0f) continue;
          if (cnt < kMaxContacts) {
            V.con_nbr[cnt * n + k] = j;
            V.con_lam[cnt * n + k] = make_int2(0, 0);
          }
          ++cnt;
        }
      }
    }
  }
  V.con_cnt[k] = cnt;
  uint32_t total;
  V.con_pre[k] = block_exclusive(cnt, ws, &total);
  uint32_t dropped;
  (void)block_exclusive(cnt > kMaxContacts ? cnt - kMaxContacts : 0u, ws, &dropped);
  if (threadIdx.x == 0) {
    V.chunk_sum[blockIdx.x] = total;
    V.chunk_drop[blockIdx.x] = dropped;
  }
}

// The chunks' first pair index inside their scene (one block per scene), and
// the scene's pair count of this substep (ContactBuffer.counter).
__global__ void __launch_bounds__(1024) k_con_scan(WorldView V, uint32_t sub) {
  __shared__ uint32_t ws[32];
  const DevScene& S = V.scenes[blockIdx.x];
  if (!S.contact || sub >= S.substeps) return;
  const uint32_t c0 = S.seg_start / kSegAlign, c1 = S.seg_end / kSegAlign;
  uint32_t carry = 0, drop = 0;
  for (uint32_t base = c0; base < c1; base += blockDim.x) {
    const uint32_t c = base + threadIdx.x;
    const uint32_t v = c < c1 ? V.chunk_sum[c] : 0u;
    const uint32_t dv = c < c1 ? V.chunk_drop[c] : 0u;
    uint32_t t, td;
    const uint32_t ex = block_exclusive(v, ws, &t);
    (void)block_exclusive(dv, ws, &td);
    if (c < c1) V.chunk_off[c] = carry + ex;
    carry += t;
    drop += td;
  }
  if (threadIdx.x == 0) V.con_stat[blockIdx.x] = make_uint2(carry, drop);
}

// Entry m of slot k is solved when it was stored and falls inside the
// scene's first max_contacts pairs.
__device__ __forceinline__ uint32_t con_live(const WorldView& V, const DevScene& S, uint32_t k) {
  const uint32_t cnt = min(V.con_cnt[k], kMaxContacts);
  if (!cnt) return 0;
  const uint32_t first = V.chunk_off[k / kSegAlign] + V.con_pre[k];
  return first >= S.max_contacts ? 0u : min(cnt, S.max_contacts - first);
}

// solve.ts:115-150: pairs that overlap at the start of the substep are
// separated, the change going to both the committed and the predicted
// positions (applied by k_con_apply2).
__global__ void __launch_bounds__(kBlock) k_con_stab(WorldView V, uint32_t sub) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= V.n) return;
  const DevScene& S = scene_at(V, k);
  if (!S.contact || sub >= S.substeps) return;
  const uint32_t live = con_live(V, S, k);
  if (!live) return;
  const float4 xk = V.cur.x[k];
  const size_t n = V.n;
  for (uint32_t m = 0; m < live; ++m) {
    const uint32_t j = V.con_nbr[m * n + k];
    const float4 xj = V.cur.x[j];
    const f3 off = xyz(xk) - xyz(xj);
    const float d = len(off);
    const float ws = xk.w + xj.w;
    if (d <= 1e-8f || d >= S.c_dist || ws <= 0.0f) continue;
    const f3 nrm = off / d;
    const float dl = (S.c_dist - d) / ws;
    acc_add(V.acc_con, k, nrm * (xk.w * dl), S.pos_scale);
    acc_add(V.acc_con, j, neg(nrm * (xj.w * dl)), S.pos_scale);
  }
}

// accumulator.ts:101-131 over [positions, predictedPositions] (loop.ts:393).
__global__ void __launch_bounds__(kBlock) k_con_apply2(WorldView V, uint32_t sub) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= V.n) return;
  const uint32_t s = scene_index(V, k);
  const DevScene& S = V.scenes[s];
  if (!S.contact || sub >= S.substeps) return;
  const int4 t = V.acc_con[k];
  if (!(t.x | t.y | t.z)) return;
  V.acc_con[k] = make_int4(0, 0, 0, 0);
  bool sat = false;
  const f3 c = ticks_change(t.x, t.y, t.z, S.pos_inv, &sat);
  const float4 x = V.cur.x[k], xs = V.cur.xs[k];
  V.cur.x[k] = with_w(xyz(x) + c, x.w);
  V.cur.xs[k] = with_w(xyz(xs) + c, xs.w);
  if (sat) atomicOr(V.flags + s * kNumFlags + FLAG_POS, 1u);
}

// solve.ts:34-104: non-penetration along the pair's normal and static
// friction inside the cone lambda_t <= mu_s lambda_n, scattered into the
// position sums that the collider pass applies.
__global__ void __launch_bounds__(kBlock) k_con_solve(WorldView V, uint32_t sub, uint32_t it) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= V.n) return;
  const DevScene& S = scene_at(V, k);
  if (!S.contact || sub >= S.substeps || it >= S.iterations) return;
  const uint32_t live = con_live(V, S, k);
  if (!live) return;
  const float4 pk = V.cur.xs[k];
  const f3 xk = xyz(pk), dk = xk - xyz(V.cur.x[k]);
  const float wk = pk.w;
  const size_t n = V.n;
  for (uint32_t m = 0; m < live; ++m) {
    const size_t e = m * n + k;
    const uint32_t j = V.con_nbr[e];
    const float4 pj = V.cur.xs[j];
    const f3 off = xk - xyz(pj);
    const float d = len(off);
    const float wj = pj.w, ws = wk + wj;
    if (d <= 1e-8f || d >= S.c_dist || ws <= 0.0f) continue;
    const f3 nrm = off / d;
    const float dln = (S.c_dist - d) / ws;
    int2 L = V.con_lam[e];
    L.x += lam_ticks(dln);
    V.con_nrm[e] = with_w(nrm, 0.0f);
    const f3 slip = dk - (xyz(pj) - xyz(V.cur.x[j]));
    const f3 tang = slip - nrm * dot(slip, nrm);
    const float tl = len(tang);
    const float ln = (float)L.x * kLambdaInv, lt = (float)L.y * kLambdaInv;
    const float dlt = tl / ws;
    const bool sticks = tl > 1e-10f && dlt <= S.c_mus * ln - lt;
    const f3 ni = nrm * (wk * dln), nj = neg(nrm * (wj * dln));
    acc_add(V.acc_con, k, sticks ? ni + neg(tang * (wk / ws)) : ni, S.pos_scale);
    acc_add(V.acc_con, j, sticks ? nj + tang * (wj / ws) : nj, S.pos_scale);
    L.y += lam_ticks(sticks ? dlt : 0.0f);
    V.con_lam[e] = L;
  }
}

// solve.ts:158-189: kinetic friction, the tangential relative velocity
// reduced by at most mu_k lambda_n / dt, into the velocity sums that the
// friction pass applies.
__global__ void __launch_bounds__(kBlock) k_con_friction(WorldView V, uint32_t sub) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= V.n) return;
  const DevScene& S = scene_at(V, k);
  if (!S.contact || sub >= S.substeps) return;
  const uint32_t live = con_live(V, S, k);
  if (!live) return;
  const float wk = V.cur.x[k].w;
  const f3 vk = xyz(V.cur.v[k]);
  const size_t n = V.n;
  for (uint32_t m = 0; m < live; ++m) {
    const size_t e = m * n + k;
    const uint32_t j = V.con_nbr[e];
    const float wj = V.cur.x[j].w, ws = wk + wj;
    const float ln = (float)V.con_lam[e].x * kLambdaInv;
    if (ws <= 0.0f || ln <= 0.0f) continue;
    const f3 nrm = xyz(V.con_nrm[e]);
    const f3 v = vk - xyz(V.cur.v[j]);
    const f3 vt = v - nrm * dot(nrm, v);
    const float vtl = len(vt);
    if (vtl < 1e-6f) continue;
    const float change = fminf(S.c_muk * ln * ws / S.dt, vtl);
    const f3 imp = neg((vt / vtl) * change) / ws;
    acc_add(V.acc_con, k, imp * wk, S.vel_scale);
    acc_add(V.acc_con, j, neg(imp * wj), S.vel_scale);
  }
}

}  // namespace pf
