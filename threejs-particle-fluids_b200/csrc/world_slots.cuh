// world_slots.cuh — the fluid neighbour passes with one thread per slot.
//
// Each thread owns one particle (slot k, cell order) and gathers its
// neighbours' state straight from the slot arrays; particles are in cell
// order, so a warp's gathers fall on a few hundred consecutive slots that L1
// holds. The neighbour list is blocked by warp: 16-bit offsets from a
// per-warp base slot in groups of eight per slot, so a warp reads a round of
// 2, 4 or 8 entries per slot as one coalesced vector load per lane (32-bit
// slots, one line per entry index, where a warp's rows reach further). The
// loops fetch the list and
// the neighbours several at a time before using them: independent loads in
// flight per round instead of a dependent load per neighbour, with the sums
// still formed in list order.
//
// The depth of that fetch (kNbrUnroll: 2, 4 or 8 entries per round) trades
// loads in flight against registers and so occupancy; the autotuner of
// World::tune picks it, the block size, and this path or the warp-tile path
// (world_tiles.cuh) per world.
#pragma once

#include <type_traits>

#include "world_kernels.cuh"

namespace pf {

// A list entry, or 2, 4 or 8 16-bit entries of one group (read-only for the
// kernel). A miss fetches 256 bytes into L2: with the warp-blocked layout
// that is the warp's neighbouring entries too.
__device__ __forceinline__ uint32_t ld_entry(const uint32_t* p) {
  uint32_t v;
  asm("ld.global.nc.L2::256B.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
template <uint32_t kN>
__device__ __forceinline__ void ld_group(const uint16_t* p, uint32_t (&w)[kN / 2]) {
  static_assert(kN == 2 || kN == 4 || kN == 8, "2, 4 or 8 entries");
  if constexpr (kN == 8)
    asm("ld.global.nc.L2::256B.v4.u32 {%0, %1, %2, %3}, [%4];"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3])
        : "l"(p));
  else if constexpr (kN == 4)
    asm("ld.global.nc.L2::256B.v2.u32 {%0, %1}, [%2];" : "=r"(w[0]), "=r"(w[1]) : "l"(p));
  else
    asm("ld.global.nc.L2::256B.u32 %0, [%1];" : "=r"(w[0]) : "l"(p));
}

// The list of slot k: its warp's base (kNbrWide: 32-bit entries) and the
// first entry of either width.
struct NbrList {
  uint32_t base;
  const uint32_t* w32;  // entry m at w32[m * kNbrStride]
  const uint16_t* w16;  // entry m at w16[(m / 8) * 256 + m % 8]
  __device__ __forceinline__ bool wide() const { return (base & kNbrWide) != 0; }
  __device__ __forceinline__ uint32_t entry(uint32_t m) const {
    return wide() ? __ldg(w32 + m * kNbrStride)
                  : base + __ldg(w16 + (m / kNbrGroup) * (kNbrStride * kNbrGroup) + m % kNbrGroup);
  }
};
__device__ __forceinline__ NbrList nbr_list(const WorldView& V, uint32_t k) {
  NbrList L;
  L.base = V.nbr_base[k >> 5];
  L.w32 = V.nbr + nbr_col(k);
  L.w16 = reinterpret_cast<const uint16_t*>(V.nbr) + nbr16_col(k);
  return L;
}

// Before a walk: one lane of the warp has its list block's first max(cnt)
// entry lines (contiguous) fetched into L2 in one bulk prefetch, so the
// later rounds' entries come from L2 instead of DRAM.
__device__ __forceinline__ void prefetch_list(const NbrList& L, uint32_t cnt) {
  const uint32_t act = __activemask();
  const uint32_t most = __reduce_max_sync(act, cnt);
  if (most && (threadIdx.x & 31u) == (uint32_t)(__ffs(act) - 1)) {
    const uint32_t lane = threadIdx.x & 31u;
    const void* base = L.wide() ? (const void*)(L.w32 - lane) : (const void*)(L.w16 - lane * kNbrGroup);
    const uint32_t bytes = L.wide() ? most * kNbrStride * 4u : div_up(most, kNbrGroup) * kNbrStride * kNbrGroup * 2u;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(base), "r"(bytes) : "memory");
  }
}

// Walks list entries [0, cnt) (entries(m, j) gives the slots of entries m
// to m + kU - 1, m a multiple of kU), kU per round, in list order: a round
// gathers its neighbours' records (fetch), then fetches the next round's
// list entries, then uses the records (use). The list entries come from
// DRAM and the records mostly from L1, so the next round's entries are in
// flight while this round's records arrive and are used. The last partial
// round is one batch as well (its entries past cnt are read, not used).
template <uint32_t kU, typename Entries, typename Fetch, typename Use>
__device__ __forceinline__ void walk_list(Entries entries, uint32_t cnt, Fetch fetch, Use use) {
  using Rec = decltype(fetch(0u));
  uint32_t jn[kU];
  if (cnt) entries(0u, jn);
  uint32_t m = 0;
  for (; m + kU <= cnt; m += kU) {
    uint32_t j[kU];
    Rec r[kU];
#pragma unroll
    for (uint32_t q = 0; q < kU; ++q) {
      j[q] = jn[q];
      r[q] = fetch(j[q]);
    }
    if (m + kU < cnt) entries(m + kU, jn);
#pragma unroll
    for (uint32_t q = 0; q < kU; ++q) use(j[q], r[q]);
  }
  if (m < cnt) {
    Rec r[kU];
#pragma unroll
    for (uint32_t q = 0; q < kU; ++q)
      if (m + q < cnt) r[q] = fetch(jn[q]);
#pragma unroll
    for (uint32_t q = 0; q < kU; ++q)
      if (m + q < cnt) use(jn[q], r[q]);
  }
}

// walk_list over slot k's list in whichever width its warp stored (a
// warp-uniform branch): 16-bit entries a group at a time. kFresh: the list
// was written by this same thread in this kernel, so its entries are read
// with plain (coherent) loads.
template <uint32_t kU, bool kFresh = false, typename Fetch, typename Use>
__device__ __forceinline__ void walk_nbrs(const NbrList& L, uint32_t cnt, Fetch fetch, Use use) {
  static_assert(kNbrGroup % kU == 0, "a round lies in one group");
  if (L.wide()) {
    const uint32_t* p = L.w32;
    walk_list<kU>(
        [&](uint32_t m, uint32_t(&j)[kU]) {
#pragma unroll
          for (uint32_t q = 0; q < kU; ++q) j[q] = kFresh ? p[(m + q) * kNbrStride] : ld_entry(p + (m + q) * kNbrStride);
        },
        cnt, fetch, use);
  } else {
    const uint16_t* p = L.w16;
    const uint32_t b = L.base;
    walk_list<kU>(
        [&](uint32_t m, uint32_t(&j)[kU]) {
          const uint16_t* g = p + (m / kNbrGroup) * (kNbrStride * kNbrGroup) + m % kNbrGroup;
          uint32_t w[kU / 2];
          if (kFresh) {
#pragma unroll
            for (uint32_t q = 0; q < kU / 2; ++q) w[q] = reinterpret_cast<const uint32_t*>(g)[q];
          } else {
            ld_group<kU>(g, w);
          }
#pragma unroll
          for (uint32_t q = 0; q < kU / 2; ++q) {
            j[2 * q] = b + (w[q] & 0xffffu);
            j[2 * q + 1] = b + (w[q] >> 16);
          }
        },
        cnt, fetch, use);
  }
}

// neighbour records gathered by the list walks
struct NbrXQ {  // predicted position (w = inverse mass) and mass code
  float4 x;
  float q;
};
struct NbrXL {  // predicted position and (lambda, mass code)
  float4 x;
  float2 lq;
};
struct NbrXV {  // committed position, velocity (or curl) and mass code (or volume)
  float4 x, v;
  float q;
};

// lambda.ts:60-71: density and the multiplier from the neighbour sums (in
// the fast path the kernel constants are applied here).
__device__ __forceinline__ void finish_lambda(const WorldView& V, const DevScene& S, const DevFluid& F, uint32_t k,
                                              float4 xi4, float rho, f3 gs, float gss) {
  const float wi = xi4.w;
#ifndef PF_EXACT_ROUNDING
  rho *= F.poly6;
  gs = gs * -F.spiky;
  gss *= F.spiky * F.spiky;
#endif
  V.cur.dens[k] = rho;
  const float C = rho * F.inv_rho0 - 1.0f;
  float lam = 0.0f;
  if (C > 0.0f) {
    const float gn = (dot(gs, gs) * wi + gss) * (F.inv_rho0 * F.inv_rho0);
    const float at = F.compliance / (S.dt * S.dt);
    lam = -C / fmaxf(gn + at, 1e-20f);
  }
  // the position pass of a single-fluid scene of one mass reads (x*, lambda)
  // from xl, the others lambda from lm (the warp-tile path keeps its own)
  if (S.homog)
    V.xl[k] = make_float4(xi4.x, xi4.y, xi4.z, lam);
  else
    V.lm[k].x = lam;
}

// lambda.ts:41-59: one neighbour's terms of the density and constraint-
// gradient sums.
__device__ __forceinline__ void lambda_terms(const DevFluid& F, f3 xi, float4 xj, float qj, float& rho, f3& gs,
                                             float& gss) {
  const float mass = code_mass(qj, F.rho0);
  const f3 off = xi - xyz(xj);
  const float rsq = dot(off, off);
#ifdef PF_EXACT_ROUNDING
  rho += mass * poly6(rsq, F);
  const f3 g = spiky_vec(off, rsq, F) * mass;
  gs = gs + g;
  gss += dot(g, g) * xj.w;
#else
  // The kernel constants leave the sums: rho = poly6 * sum m d^3,
  // sum grad = -spiky * sum f r, sum |grad|^2 w = spiky^2 * sum f^2 r^2 w
  // with f = m (h - r)^2 / r.
  const float d = fmaxf(F.hsq - rsq, 0.0f);
  rho += mass * (d * d * d);
  const float f = spiky_shape(rsq, F) * mass;
  gs = gs + off * f;
  gss += (f * f) * (rsq * xj.w);
#endif
}

// neighborList.ts:48-71: up to 64 neighbours within h at the predicted
// positions of this substep, in walk order (query.ts:37-66: rows dz, dy;
// inside a row ascending cell, inside a cell ascending index), self
// included. The nine row ranges are fetched first, then each row's
// candidates several at a time.
//
// With kDens, a fluid that is its scene's first material also forms the
// density and lambda of its first solver iteration from the same hits, in
// the same order (nothing moves between the list and that pass when the
// world has no surface impulses and no late drag and lift).
// kFlat: the nine rows are walked as one sequence, kNbrUnroll candidates
// per round across row ends, so a warp waits for its longest walk rather
// than, row by row, for each row's longest (the same candidates in the same
// order; the autotuner picks the faster form).
template <uint32_t kNbrUnroll, bool kDens, bool kFlat>
__global__ void k_s_neighbors(WorldView V, uint32_t sub) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_fchunk * kSegAlign) return;     // whole warps
  const uint32_t k = chunk_slot(V.fchunk, g);  // slots of the scenes with a fluid
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps) return;               // whole chunks
  const uint32_t f = tag_fluid(V.cur.tag[k]);
  // every lane of the warp takes part in choosing the list width; lanes of
  // other materials (f == 0) leave after that
  const DevFluid& F = V.fluids[f ? f - 1 : 0];
  const float4 xi4 = V.cur.xs[k];
  const f3 xi = xyz(xi4);
  const bool dens = kDens && F.rank == 0 && S.iterations > 0;
  float rho = 0.0f, gss = 0.0f;
  f3 gs = mk(0.0f, 0.0f, 0.0f);
  const float* __restrict__ q_of = reinterpret_cast<const float*>(V.lm) + 1;
  const float hsq = F.hsq;
  int32_t cx, cy, cz;
  local_cell(S, xi, &cx, &cy, &cz, nullptr);
  const int32_t x0 = max(cx - 1, 0), x1 = min(cx + 1, (int32_t)S.dims[0] - 1);
  // Cells whose box lies at least h away cannot hold a neighbour, so they
  // are left out of the walk; the hits, and their order, stay those of the
  // full 27-cell walk. Border cells (which hold the clamped particles) are
  // never left out.
  auto gap = [&](float p, int32_t c, int a, float o) {
    const float lo = o + (float)(S.lo[a] + c) * S.cell, hi = lo + S.cell;
    const float d = fmaxf(fmaxf(lo - p, p - hi), 0.0f);
    return fmaxf(d - S.prune_slack, 0.0f);
  };
  const int32_t nx = (int32_t)S.dims[0], ny = (int32_t)S.dims[1], nz = (int32_t)S.dims[2];
  const float gl = (x0 < cx && x0 > 0) ? gap(xi.x, x0, 0, S.ox) : 0.0f;
  const float gr = (x1 > cx && x1 < nx - 1) ? gap(xi.x, x1, 0, S.ox) : 0.0f;
  const bool can_l = x0 < cx && x0 > 0, can_r = x1 > cx && x1 < nx - 1;
  uint32_t rs[9], re[9];
#pragma unroll
  for (int r = 0; r < 9; ++r) {
    const int32_t z = cz + r / 3 - 1, y = cy + r % 3 - 1;
    if (z < 0 || z >= nz || y < 0 || y >= ny) {
      rs[r] = re[r] = 0;
      continue;
    }
    int32_t a0 = x0, a1 = x1;
    if (y > 0 && y < ny - 1 && z > 0 && z < nz - 1) {
      const float gy = y != cy ? gap(xi.y, y, 1, S.oy) : 0.0f, gz = z != cz ? gap(xi.z, z, 2, S.oz) : 0.0f;
      const float perp = gy * gy + gz * gz;
      if (perp >= hsq) {
        rs[r] = re[r] = 0;
        continue;
      }
      if (can_l && perp + gl * gl >= hsq) a0 = cx;
      if (can_r && perp + gr * gr >= hsq) a1 = cx;
    }
    const uint32_t row = S.cell_base + S.dims[0] * ((uint32_t)y + S.dims[1] * (uint32_t)z);
    rs[r] = __ldg(V.cstart + row + a0);
    re[r] = __ldg(V.cstart + row + a1) + __ldg(V.ccount + row + a1);
  }
  // The warp's entries are 16-bit offsets from the lowest slot its rows
  // reach when every reachable slot lies within 65,536 of it.
  // (No reduction when the world keeps whole slots in every warp.)
  bool narrow = false;
  uint32_t base = kNbrWide;
  if (!V.nbr_wide_only) {  // uniform over the launch
    uint32_t lo = 0xffffffffu, hi = 0;
#pragma unroll
    for (int r = 0; r < 9; ++r) {
      if (!f) rs[r] = re[r] = 0;
      if (re[r] > rs[r]) {
        lo = min(lo, rs[r]);
        hi = max(hi, re[r]);
      }
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    narrow = hi <= lo || hi - lo <= 65536u;
    base = narrow ? (hi > lo ? lo : 0u) : kNbrWide;
  }
  if ((threadIdx.x & 31u) == 0) V.nbr_base[k >> 5] = base;
  if (!f) return;
  // Every candidate is tested; the first kMaxNbr hits in walk order are
  // stored (as the reference's list keeps them) and any further hit only
  // marks the overflow. The walk is compiled once per entry width (the width
  // is uniform over the warp), and a 16-bit entry is stored without a branch
  // on the count: hits past the kMaxNbr-th land in the group after the last,
  // which the 16-bit layout leaves unused (a block has room for 2 kMaxNbr
  // entries per slot).
  uint32_t cnt = 0;
  uint32_t* __restrict__ out = V.nbr + nbr_col(k);
  uint16_t* __restrict__ out16 = reinterpret_cast<uint16_t*>(V.nbr) + nbr16_col(k);
  auto walk = [&](auto narrow_tag) {
    constexpr bool kNarrow = decltype(narrow_tag)::value;
    auto test = [&](uint32_t j, float4 xj) {
      const bool hit = dist2_rn(xi, xj) < hsq;
      if (kNarrow) {
        if (hit)
          out16[(min(cnt, kMaxNbr) / kNbrGroup) * (kNbrStride * kNbrGroup) + cnt % kNbrGroup] = (uint16_t)(j - base);
      } else {
        if (hit && cnt < kMaxNbr) out[cnt * kNbrStride] = j;
      }
      cnt += hit ? 1u : 0u;
    };
    if (kFlat) {
      // the row pointer moves on at each row's end (empty rows skipped); the
      // rows stay in registers (constant indices after unrolling)
      int r = 0;
      uint32_t j = rs[0], e = re[0];
      auto pick = [](const uint32_t(&a)[9], int q) {
        uint32_t v = a[0];
#pragma unroll
        for (int t = 1; t < 9; ++t) v = q == t ? a[t] : v;
        return v;
      };
      auto advance = [&]() {
        while (j >= e && r < 8) {
          ++r;
          j = pick(rs, r);
          e = pick(re, r);
        }
      };
      advance();
      while (j < e) {
        uint32_t c[kNbrUnroll];
        bool live[kNbrUnroll];
#pragma unroll
        for (uint32_t q = 0; q < kNbrUnroll; ++q) {
          live[q] = j < e;
          c[q] = j;
          if (live[q]) {
            ++j;
            if (j >= e) advance();
          }
        }
        float4 xj[kNbrUnroll];
#pragma unroll
        for (uint32_t q = 0; q < kNbrUnroll; ++q)
          if (live[q]) xj[q] = __ldg(V.cur.xs + c[q]);
#pragma unroll
        for (uint32_t q = 0; q < kNbrUnroll; ++q)
          if (live[q]) test(c[q], xj[q]);
      }
    } else {
#pragma unroll
      for (int r = 0; r < 9; ++r) {
        uint32_t j = rs[r];
        const uint32_t e = re[r];
        // whole rounds, then the row's last 1 to kNbrUnroll - 1 candidates as
        // one guarded round (their loads in flight together)
        for (; j + kNbrUnroll <= e; j += kNbrUnroll) {
          float4 xj[kNbrUnroll];
#pragma unroll
          for (uint32_t q = 0; q < kNbrUnroll; ++q) xj[q] = __ldg(V.cur.xs + j + q);
#pragma unroll
          for (uint32_t q = 0; q < kNbrUnroll; ++q) test(j + q, xj[q]);
        }
        if (j < e) {
          float4 xj[kNbrUnroll];
#pragma unroll
          for (uint32_t q = 0; q < kNbrUnroll; ++q)
            if (j + q < e) xj[q] = __ldg(V.cur.xs + j + q);
#pragma unroll
          for (uint32_t q = 0; q < kNbrUnroll; ++q)
            if (j + q < e) test(j + q, xj[q]);
        }
      }
    }
  };
  if (narrow)
    walk(std::true_type{});
  else
    walk(std::false_type{});
  const bool over = cnt > kMaxNbr;
  cnt = min(cnt, kMaxNbr);
  V.ncount[k] = cnt;
  if (over) atomicOr(V.flags + scene_index(V, k) * kNumFlags + FLAG_NBR, 1u);
  if (kDens && dens) {
    // the density pass over the list just written (still in cache), in list
    // order, outside the divergent walk
    NbrList L;
    L.base = base;
    L.w32 = V.nbr + nbr_col(k);
    L.w16 = reinterpret_cast<const uint16_t*>(V.nbr) + nbr16_col(k);
    const float qh = -S.homog_mass;
    const bool homog = S.homog;
    walk_nbrs<kNbrUnroll, true>(
        L, cnt, [&](uint32_t j) { return NbrXQ{__ldg(V.cur.xs + j), homog ? qh : __ldg(q_of + 2 * (size_t)j)}; },
        [&](uint32_t, const NbrXQ& r) { lambda_terms(F, xi, r.x, r.q, rho, gs, gss); });
    finish_lambda(V, S, F, k, xi4, rho, gs, gss);
  }
}

// lambda.ts:41-71
template <uint32_t kNbrUnroll>
__global__ void __maxnreg__(kNbrUnroll == 8 ? 80 : 48) k_s_lambda(WorldView V, uint32_t rank, uint32_t sub, uint32_t it) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_fchunk * kSegAlign) return;
  const uint32_t k = chunk_slot(V.fchunk, g);  // slots of the scenes with a fluid
  const uint32_t f = tag_fluid(V.cur.tag[k]);
  if (!f) return;
  const DevFluid& F = V.fluids[f - 1];
  if (F.rank != rank) return;
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps || it >= S.iterations) return;
  const float4 xi4 = V.cur.xs[k];
  const f3 xi = xyz(xi4);
  float rho = 0.0f, gss = 0.0f;
  f3 gs = mk(0.0f, 0.0f, 0.0f);
  const uint32_t cnt = V.ncount[k];
  const NbrList nl = nbr_list(V, k);
  prefetch_list(nl, cnt);
  const float* __restrict__ q_of = reinterpret_cast<const float*>(V.lm) + 1;  // lm[j].y
  if (S.homog) {
    // one fluid, one mass: no mass gather
    const float qh = -S.homog_mass;
    walk_nbrs<kNbrUnroll>(
        nl, cnt, [&](uint32_t j) { return __ldg(V.cur.xs + j); },
        [&](uint32_t, const float4& xj) { lambda_terms(F, xi, xj, qh, rho, gs, gss); });
  } else {
    walk_nbrs<kNbrUnroll>(
        nl, cnt, [&](uint32_t j) { return NbrXQ{__ldg(V.cur.xs + j), __ldg(q_of + 2 * (size_t)j)}; },
        [&](uint32_t, const NbrXQ& r) { lambda_terms(F, xi, r.x, r.q, rho, gs, gss); });
  }
  finish_lambda(V, S, F, k, xi4, rho, gs, gss);
}

// positionDelta.ts:41-85 (the reaction on dynamic boundary neighbours goes
// into the fixed-point reaction sums by slot).
//
// With `apply`, the slots of single-fluid scenes of one mass (S.homog) also
// take the apply of k_fluid_apply in the same thread: x* += delta, then the
// scene's colliders when they follow the fluid. Their neighbours' positions
// come from xl (written by the density pass), not from x*, so x* of the slot
// is rewritten in place; the arithmetic is that of the separate apply.
template <uint32_t kNbrUnroll, bool kReact>
__global__ void __maxnreg__(kNbrUnroll == 8 ? 96 : 56) k_s_delta(WorldView V, uint32_t rank, uint32_t sub, uint32_t it, uint32_t apply) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_fchunk * kSegAlign) return;
  const uint32_t k = chunk_slot(V.fchunk, g);  // slots of the scenes with a fluid
  const uint32_t f = tag_fluid(V.cur.tag[k]);
  if (!f) return;
  const DevFluid& F = V.fluids[f - 1];
  if (F.rank != rank) return;
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps || it >= S.iterations) return;
  const float4 xi4 = V.cur.xs[k];
  const f3 xi = xyz(xi4);
  const float li = S.homog ? V.xl[k].w : V.lm[k].x;
  const bool react = kReact && F.react_lo != F.react_hi && li != 0.0f;
  // each fluid reads its own multipliers, zero for other particles (the
  // reference keeps one lambda buffer per fluid)
  const bool multi = S.fluid_count > 1;
  f3 sum = mk(0.0f, 0.0f, 0.0f);
  const uint32_t cnt = V.ncount[k];
  const NbrList nl = nbr_list(V, k);
  prefetch_list(nl, cnt);
  auto one = [&](uint32_t j, float4 xj, float2 lq) {
    const float bvj = lq.y;
    const float lj = (multi && tag_fluid(__ldg(V.cur.tag + j)) != f) ? 0.0f : lq.x;
    const float mass = code_mass(bvj, F.rho0);
    const f3 off = xi - xyz(xj);
#ifdef PF_EXACT_ROUNDING
    const f3 g = spiky_vec(off, dot(off, off), F);
    sum = sum + g * ((li + lj) * mass);
#else
    // sum stays without the -spiky constant until the end; the gradient is
    // formed only for a reaction
    const float rsq = dot(off, off);
    const float shape = spiky_shape(rsq, F);
    sum = sum + off * (shape * ((li + lj) * mass));
    const f3 g = off * (shape * -F.spiky);
#endif
    if (react && bvj > 0.0f && xj.w > 0.0f) {
      const uint32_t idj = V.ids[j];
      bool in = false;
      for (uint32_t b = 0; b < F.bnd_count; ++b) {
        const DevBoundary B = V.bnds[F.bnd_first + b];
        in = in || (idj >= B.start && idj < B.start + B.count);
      }
      if (in) acc_add(V.acc_react, j, g * (-(li / F.rho0) * (F.rho0 * bvj) * xj.w), F.react_scale);
    }
  };
  if (S.homog) {
    // one fluid, one mass: (x*, lambda) of a neighbour in one gather
    const float qh = -S.homog_mass;
    walk_nbrs<kNbrUnroll>(
        nl, cnt, [&](uint32_t j) { return __ldg(V.xl + j); },
        [&](uint32_t j, const float4& xj) { one(j, xj, make_float2(xj.w, qh)); });
  } else {
    walk_nbrs<kNbrUnroll>(
        nl, cnt, [&](uint32_t j) { return NbrXL{__ldg(V.cur.xs + j), __ldg(V.lm + j)}; },
        [&](uint32_t j, const NbrXL& r) { one(j, r.x, r.lq); });
  }
#ifndef PF_EXACT_ROUNDING
  sum = sum * -F.spiky;
#endif
  const float4 d = with_w((sum / F.rho0) * xi4.w, 0.0f);
  if (apply && S.homog) {
    float4 x = xi4;
    x.x += d.x;
    x.y += d.y;
    x.z += d.z;
    if (S.collide_rank1 == rank + 1) collide_particle(V, S, scene_index(V, k), k, x, V.prims + S.prim_base);
    V.cur.xs[k] = x;
    return;
  }
  V.dx[k] = d;
}

// velocity.ts:43-70: one walk over the list at the committed positions for
// the XSPH change (Delta v = c sum V_j (v_j - v_i) W) and, with vorticity
// confinement, the curl omega = sum V_j (v_i - v_j) x grad W.
template <uint32_t kNbrUnroll, bool kBnd>
__global__ void k_s_xsph(WorldView V, uint32_t rank, uint32_t sub) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_fchunk * kSegAlign) return;
  const uint32_t k = chunk_slot(V.fchunk, g);  // slots of the scenes with a fluid
  const uint32_t f = tag_fluid(V.cur.tag[k]);
  if (!f) return;
  const DevFluid& F = V.fluids[f - 1];
  const bool visc = F.has_visc, vort = F.has_vort;
  if (F.rank != rank || !(visc || vort)) return;
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps) return;
  const f3 xi = xyz(V.cur.x[k]);
  const f3 vi = xyz(V.cur.v[k]);
  f3 sm = mk(0.0f, 0.0f, 0.0f), curl = mk(0.0f, 0.0f, 0.0f);
  const uint32_t cnt = V.ncount[k];
  const NbrList nl = nbr_list(V, k);
  prefetch_list(nl, cnt);
  const float* __restrict__ q_of = reinterpret_cast<const float*>(V.lm) + 1;  // lm[j].y: volume if > 0
  // without boundaries in the world every neighbour has the fluid volume
  auto one = [&](float4 xj, float4 vj, float bvj) {
    const f3 off = xi - xyz(xj);
    const float vol = (kBnd && bvj > 0.0f) ? bvj : F.volume;
    const float rsq = dot(off, off);
    if (vort) curl = curl + cross(vi - xyz(vj), spiky_vec(off, rsq, F)) * vol;
#ifdef PF_EXACT_ROUNDING
    if (visc) sm = sm + ((xyz(vj) - vi) * poly6(rsq, F)) * vol;
#else
    if (visc) {
      const float d = fmaxf(F.hsq - rsq, 0.0f);
      sm = sm + (xyz(vj) - vi) * ((d * d * d) * vol);
    }
#endif
  };
  walk_nbrs<kNbrUnroll>(
      nl, cnt,
      [&](uint32_t j) { return NbrXV{__ldg(V.cur.x + j), __ldg(V.cur.v + j), kBnd ? __ldg(q_of + 2 * (size_t)j) : 0.0f}; },
      [&](uint32_t, const NbrXV& r) { one(r.x, r.v, r.q); });
#ifndef PF_EXACT_ROUNDING
  sm = sm * F.poly6;
#endif
  if (visc) V.dv[k] = with_w(sm * F.c_xsph, 0.0f);
  if (vort) V.vort[k] = with_w(curl, len(curl));
}

// velocity.ts:75-92: eta = sum over fluid neighbours (no boundary volume) of
// grad W (|omega_j| - |omega_i|) V, into dx (free after the iterations).
template <uint32_t kNbrUnroll>
__global__ void k_s_vort_grad(WorldView V, uint32_t rank, uint32_t sub) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_fchunk * kSegAlign) return;
  const uint32_t k = chunk_slot(V.fchunk, g);  // slots of the scenes with a fluid
  const uint32_t f = tag_fluid(V.cur.tag[k]);
  if (!f) return;
  const DevFluid& F = V.fluids[f - 1];
  if (F.rank != rank || !F.has_vort) return;
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps) return;
  const f3 xi = xyz(V.cur.x[k]);
  const float wi = V.vort[k].w;
  f3 eta = mk(0.0f, 0.0f, 0.0f);
  const uint32_t cnt = V.ncount[k];
  const NbrList nl = nbr_list(V, k);
  prefetch_list(nl, cnt);
  walk_nbrs<kNbrUnroll>(
      nl, cnt, [&](uint32_t j) { return NbrXV{__ldg(V.cur.x + j), V.vort[j], __ldg(V.cur.bv + j)}; },
      [&](uint32_t, const NbrXV& r) {
        if (r.q > 0.0f) return;
        const f3 off = xi - xyz(r.x);
        eta = eta + spiky_vec(off, dot(off, off), F) * ((r.v.w - wi) * F.volume);
      });
  V.dx[k] = with_w(eta, 0.0f);
}

// cohesion.ts:33-48: n_i = h sum_j V_j grad W(x*_i - x*_j), at this
// substep's predicted positions.
template <uint32_t kNbrUnroll>
__global__ void k_s_color_normal(WorldView V, uint32_t rank, uint32_t sub) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_fchunk * kSegAlign) return;
  const uint32_t k = chunk_slot(V.fchunk, g);  // slots of the scenes with a fluid
  const uint32_t f = tag_fluid(V.cur.tag[k]);
  if (!f) return;
  const DevFluid& F = V.fluids[f - 1];
  if (F.rank != rank || !F.has_st) return;
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps) return;
  const f3 xi = xyz(V.cur.xs[k]);
  f3 sum = mk(0.0f, 0.0f, 0.0f);
  const uint32_t cnt = V.ncount[k];
  const NbrList nl = nbr_list(V, k);
  prefetch_list(nl, cnt);
  walk_nbrs<kNbrUnroll>(
      nl, cnt, [&](uint32_t j) { return NbrXQ{__ldg(V.cur.xs + j), __ldg(V.cur.bv + j)}; },
      [&](uint32_t, const NbrXQ& r) {
        const f3 off = xi - xyz(r.x);
        sum = sum + spiky_vec(off, dot(off, off), F) * (r.q > 0.0f ? r.q : F.volume);
      });
  V.normal[k] = with_w(sum * F.h, 0.0f);
}

// cohesion.ts:54-66: the cohesion spline C(r).
__device__ __forceinline__ float cohesion_spline(float r, const DevFluid& F) {
  const float gap = fmaxf(F.h - r, 0.0f);
  const float shared = gap * gap * gap * (r * r * r);
  const float value = r * 2.0f > F.h ? shared : shared * 2.0f - F.coh_h6_64;
  return (r > 0.0f && r <= F.h) ? value * F.coh_coef : 0.0f;
}
// adhesion.ts:33-47: the adhesion spline A(r), non-zero on (h/2, h].
__device__ __forceinline__ float adhesion_spline(float r, const DevFluid& F) {
  const float inner = fmaxf(r * r * F.adh_m4h + r * 6.0f - F.adh_2h, 0.0f);
  const float root = sqrtf(sqrtf(inner));
  return (r * 2.0f > F.h && r <= F.h) ? root * F.adh_coef : 0.0f;
}

// cohesion.ts:75-120 and adhesion.ts:55-76 in one walk: surface tension on
// each fluid pair once (partner id above this one, inside the fluid's range;
// the negated change goes to the partner), adhesion toward boundary
// neighbours on the fluid side only; both as fixed-point velocity changes.
template <uint32_t kNbrUnroll>
__global__ void k_s_impulses(WorldView V, uint32_t rank, uint32_t sub) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= V.n_fchunk * kSegAlign) return;
  const uint32_t k = chunk_slot(V.fchunk, g);  // slots of the scenes with a fluid
  const uint32_t f = tag_fluid(V.cur.tag[k]);
  if (!f) return;
  const DevFluid& F = V.fluids[f - 1];
  if (F.rank != rank || !(F.has_st || F.has_ad)) return;
  const DevScene& S = scene_at(V, k);
  if (sub >= S.substeps) return;
  const f3 xi = xyz(V.cur.xs[k]);
  const uint32_t idi = V.ids[k];
  const f3 ni = F.has_st ? xyz(V.normal[k]) : mk(0.0f, 0.0f, 0.0f);
  const float rhoi = V.cur.dens[k];
  const float dt = S.dt;
  const uint32_t cnt = V.ncount[k];
  const NbrList nl = nbr_list(V, k);
  for (uint32_t m = 0; m < cnt; ++m) {
    const uint32_t j = nl.entry(m);
    const f3 off = xi - xyz(__ldg(V.cur.xs + j));
    if (F.has_st) {
      const uint32_t idj = V.ids[j];
      if (idj > idi && idj < F.range_end) {
        const float r = len(off);
        if (!(r < 1e-20f)) {
          const float corr = (F.rho0 * 2.0f) / fmaxf(rhoi + V.cur.dens[j], 1.0f);
          const f3 coh = (off / r) * -(F.gamma * F.mass * F.mass * cohesion_spline(r, F));
          const f3 curv = (ni - xyz(V.normal[j])) * -(F.gamma * F.mass);
          const f3 dv = (coh + curv) * corr / F.mass * dt;
          acc_add(V.acc_imp, k, dv, F.imp_scale);
          acc_add(V.acc_imp, j, neg(dv), F.imp_scale);
        }
      }
    }
    if (F.has_ad) {
      const float vol = __ldg(V.cur.bv + j);
      if (vol > 0.0f) {
        const float r = len(off);
        if (!(r < 1e-20f)) {
          const f3 force = (off / r) * -(F.beta * F.mass * (F.rho0 * vol) * adhesion_spline(r, F));
          acc_add(V.acc_imp, k, force / F.mass * dt, F.imp_scale);
        }
      }
    }
  }
}

}  // namespace pf
