// world_tiles.cuh — the neighbour passes of the fluid over shared-memory
// tiles of the 27-cell stencil.
//
// After each grid rebuild the fluid scenes' grid rows are cut into tiles: a
// run of consecutive cells of one (y, z) row holding at most 32 particles,
// one per lane of a warp. Particles are sorted by cell, so a tile's own
// particles are one contiguous slot range, and the union of their 27-cell
// stencils is nine contiguous slot ranges (the rows y-1..y+1, z-1..z+1 over
// cells x0-1..x1+1): the tile's halo. Each warp takes tiles on its own,
// stages the halo into its slice of shared memory with asynchronous copies
// (cp.async) and synchronises with __syncwarp only, so no warp waits for
// another; every neighbour read after staging is a shared-memory read.
//
// The neighbour list keeps the reference's semantics (neighborList.ts:48-71:
// neighbours within h at the substep's predicted positions, 27-cell walk
// order, ascending index inside a cell, at most 64) but stores each entry as
// a 16-bit index into the tile's halo sequence, which every later pass of the
// substep rebuilds identically from the same tile.
#pragma once

#include "world_kernels.cuh"

namespace pf {

constexpr uint32_t kTileCells = 32;    // cells of one tile, at most
constexpr uint32_t kTileMax = 32;      // particles of one tile (one per lane), unless one cell holds more
constexpr uint32_t kWarpHalo = 512;    // halo particles one warp stages in shared memory
constexpr uint32_t kTileWarps = 4;     // warps (independent tiles) per CTA
constexpr uint32_t kTileThreads = 32 * kTileWarps;

// Halo rows of a tile: 9 rows in (dz, dy) order over cells [xa, xb].
__device__ __forceinline__ void tile_rows(const DevScene& S, const uint32_t* __restrict__ cstart,
                                          const uint32_t* __restrict__ ccount, int32_t y, int32_t z, int32_t x0,
                                          int32_t x1, uint32_t rs[9], uint32_t len[9]) {
  const int32_t xa = max(x0 - 1, 0), xb = min(x1 + 1, (int32_t)S.dims[0] - 1);
  int r = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy, ++r) {
      const int32_t yy = y + dy, zz = z + dz;
      if (yy < 0 || yy >= (int32_t)S.dims[1] || zz < 0 || zz >= (int32_t)S.dims[2]) {
        rs[r] = 0;
        len[r] = 0;
        continue;
      }
      const uint32_t row = S.cell_base + S.dims[0] * ((uint32_t)yy + S.dims[1] * (uint32_t)zz);
      const uint32_t a = cstart[row + xa];
      rs[r] = a;
      len[r] = cstart[row + xb] + ccount[row + xb] - a;
    }
}

// Next tile of a row starting at cell x (>= one occupied cell): at most
// kTileMax particles and kTileCells cells, shrunk until its halo fits in a
// warp's shared memory (a single cell always forms a tile).
__device__ __forceinline__ int32_t next_tile(const DevScene& S, const uint32_t* __restrict__ cstart,
                                            const uint32_t* __restrict__ ccount, uint32_t rowk, int32_t y, int32_t z,
                                            int32_t x0, uint32_t rs[9], uint32_t len[9], uint32_t* halo) {
  const int32_t nx = (int32_t)S.dims[0];
  int32_t x = x0;
  uint32_t parts = 0;
  while (x < nx && x - x0 < (int32_t)kTileCells) {
    const uint32_t c = ccount[rowk + x];
    if (parts > 0 && parts + c > kTileMax) break;
    parts += c;
    ++x;
  }
  int32_t x1 = x - 1;
  for (;;) {
    tile_rows(S, cstart, ccount, y, z, x0, x1, rs, len);
    uint32_t hsum = 0;
    for (int r = 0; r < 9; ++r) hsum += len[r];
    *halo = hsum;
    if (hsum <= kWarpHalo || x1 == x0) break;
    x1 = x0 + (x1 - x0) / 2;
  }
  return x1;
}

// Cut every grid row of the fluid scenes into tiles: one thread per row,
// counted first, one atomic per warp for the warp's tile range, then emitted.
__global__ void __launch_bounds__(kBlock) k_build_tiles(WorldView V, uint32_t sub) {
  const uint32_t R = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31u;
  bool valid = R < V.n_rows;
  uint32_t s = 0, rowk = 0;
  int32_t y = 0, z = 0;
  const DevScene* Sp = nullptr;
  if (valid) {
    uint32_t lo = 0, hi = V.n_grid_scenes;  // row_base[lo] <= R < row_base[lo + 1]
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (V.row_base[mid] <= R) lo = mid; else hi = mid;
    }
    s = V.grid_scene[lo];
    Sp = &V.scenes[s];
    if (sub >= Sp->substeps) valid = false;
    const uint32_t lr = R - V.row_base[lo];
    y = (int32_t)(lr % Sp->dims[1]);
    z = (int32_t)(lr / Sp->dims[1]);
    rowk = Sp->cell_base + Sp->dims[0] * ((uint32_t)y + Sp->dims[1] * (uint32_t)z);
  }
  uint32_t rs[9], len[9], halo;
  uint32_t ntile = 0;
  if (valid) {
    const int32_t nx = (int32_t)Sp->dims[0];
    for (int32_t x = 0; x < nx;) {
      if (V.ccount[rowk + x] == 0) { ++x; continue; }
      x = next_tile(*Sp, V.cstart, V.ccount, rowk, y, z, x, rs, len, &halo) + 1;
      ++ntile;
    }
  }
  // warp-aggregated reservation of this warp's tiles
  uint32_t incl = ntile;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= (uint32_t)off) incl += v;
  }
  const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
  uint32_t base = 0;
  if (lane == 31 && total) base = atomicAdd(V.tile_count, total);
  base = __shfl_sync(0xffffffffu, base, 31) + incl - ntile;
  if (!valid || !ntile) return;
  const int32_t nx = (int32_t)Sp->dims[0];
  uint32_t t = base;
  for (int32_t x = 0; x < nx;) {
    if (V.ccount[rowk + x] == 0) { ++x; continue; }
    const int32_t x1 = next_tile(*Sp, V.cstart, V.ccount, rowk, y, z, x, rs, len, &halo);
    if (t >= V.max_tiles) {
      atomicOr(V.flags + s * kNumFlags + FLAG_DEVICE, 1u);
      return;
    }
    Tile& T = V.tiles[t++];
    T.scene = s;
    T.p0 = V.cstart[rowk + x];
    T.p1 = V.cstart[rowk + x1] + V.ccount[rowk + x1];
    T.halo = halo;
    uint32_t off = 0;
    for (int r = 0; r < 9; ++r) {
      T.rs[r] = rs[r];
      T.roff[r] = off;
      off += len[r];
    }
    T.roff[9] = off;
    x = x1 + 1;
  }
}

// Slot of halo index h of tile T (rows are consecutive in the halo sequence).
__device__ __forceinline__ uint32_t halo_slot(const Tile& T, uint32_t h) {
  int r = 0;
  while (r < 8 && h >= T.roff[r + 1]) ++r;
  return T.rs[r] + (h - T.roff[r]);
}

// Asynchronous global -> shared copy of one element (4, 8 or 16 bytes).
template <typename E>
__device__ __forceinline__ void cp_async_elem(E* dst, const E* src) {
  static_assert(sizeof(E) == 4 || sizeof(E) == 8 || sizeof(E) == 16, "cp.async element size");
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(d), "l"(src), "n"(sizeof(E)) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// A warp's view of its current tile: the descriptor's 23 words spread over
// the lanes (word w in lane w), read with shuffles.
struct WarpTile {
  uint32_t word;
  __device__ __forceinline__ uint32_t get(int w) const { return __shfl_sync(0xffffffffu, word, w); }
  __device__ __forceinline__ uint32_t scene() const { return get(0); }
  __device__ __forceinline__ uint32_t p0() const { return get(1); }
  __device__ __forceinline__ uint32_t p1() const { return get(2); }
  __device__ __forceinline__ uint32_t halo() const { return get(3); }
};

__device__ __forceinline__ WarpTile load_warp_tile(const Tile* tiles, uint32_t t) {
  const uint32_t lane = threadIdx.x & 31u;
  WarpTile w;
  w.word = lane < 23 ? reinterpret_cast<const uint32_t*>(tiles + t)[lane] : 0u;
  return w;
}

// Stage a tile's halo of per-slot data into the warp's shared memory with
// asynchronous copies, row by row (coalesced within a row).
template <typename E>
__device__ __forceinline__ void stage_rows(const WarpTile& W, const E* __restrict__ src, E* dst) {
  const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
  for (int r = 0; r < 9; ++r) {
    const uint32_t rs = W.get(4 + r), ro = W.get(13 + r), len = W.get(14 + r) - ro;
    for (uint32_t o = lane; o < len; o += 32) cp_async_elem(dst + ro + o, src + rs + o);
  }
}

// Visit a particle's list entries in order, fetching four halo indices per
// round so their loads overlap.
template <typename Fn>
__device__ __forceinline__ void for_each_h(const uint16_t* __restrict__ nl, size_t n, uint32_t cnt, Fn&& one) {
  uint32_t m = 0;
  for (; m + 4 <= cnt; m += 4) {
    uint32_t h[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) h[q] = __ldg(nl + (m + q) * n);
#pragma unroll
    for (int q = 0; q < 4; ++q) one(h[q]);
  }
  for (; m < cnt; ++m) one(__ldg(nl + m * n));
}

// neighborList.ts:48-71 over warp tiles: candidates are the 27 cells of the
// particle's own cell; entries are halo indices of the tile.
__global__ void __launch_bounds__(kTileThreads) k_t_neighbors(WorldView V, uint32_t sub) {
  extern __shared__ float4 smem4[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  float4* hx = smem4 + warp * kWarpHalo;
  const uint32_t ntiles = min(*V.tile_count, V.max_tiles);
  const uint32_t n = V.n;
  for (uint32_t t = blockIdx.x * kTileWarps + warp; t < ntiles; t += gridDim.x * kTileWarps) {
    const WarpTile W = load_warp_tile(V.tiles, t);
    const uint32_t sc = W.scene(), p0 = W.p0(), p1 = W.p1(), halo = W.halo();
    const DevScene& S = V.scenes[sc];
    const bool staged = halo <= kWarpHalo;
    if (staged) stage_rows(W, V.cur.xs, hx);
    cp_async_wait_all();
    __syncwarp();
    const Tile& T = V.tiles[t];
    for (uint32_t i = p0 + lane; i < p1; i += 32) {
      V.slot_tile[i] = t;
      const uint32_t f = tag_fluid(V.cur.tag[i]);
      if (!f) continue;
      const DevFluid& F = V.fluids[f - 1];
      const f3 xi = xyz(V.cur.xs[i]);
      int32_t cx, cy, cz;
      local_cell(S, xi, &cx, &cy, &cz, nullptr);
      const int32_t xa = max(cx - 1, 0), xb = min(cx + 1, (int32_t)S.dims[0] - 1);
      uint32_t cnt = 0;
      bool over = false;
      int r = 0;
      for (int dz = -1; dz <= 1 && !over; ++dz)
        for (int dy = -1; dy <= 1 && !over; ++dy, ++r) {
          const int32_t yy = cy + dy, zz = cz + dz;
          if (yy < 0 || yy >= (int32_t)S.dims[1] || zz < 0 || zz >= (int32_t)S.dims[2]) continue;
          const uint32_t row = S.cell_base + S.dims[0] * ((uint32_t)yy + S.dims[1] * (uint32_t)zz);
          const uint32_t a = __ldg(V.cstart + row + xa);
          const uint32_t b = __ldg(V.cstart + row + xb) + __ldg(V.ccount + row + xb);
          const uint32_t base = T.roff[r] - T.rs[r];
          for (uint32_t j = a; j < b; ++j) {
            const uint32_t h = base + j;
            const f3 off = xi - xyz(staged ? hx[h] : V.cur.xs[j]);
            if (dot_rn(off) < F.hsq) {
              if (cnt < kMaxNbr && h <= 0xffffu) {
                V.nbr16[(size_t)cnt * n + i] = (uint16_t)h;
                ++cnt;
              } else {
                over = true;
                break;
              }
            }
          }
        }
      V.ncount[i] = cnt;
      if (over) atomicOr(V.flags + sc * kNumFlags + FLAG_NBR, 1u);
    }
    __syncwarp();
  }
}

// lambda.ts:41-71 over warp tiles.
__global__ void __launch_bounds__(kTileThreads) k_t_lambda(WorldView V, uint32_t rank, uint32_t sub, uint32_t it) {
  extern __shared__ float4 smem4[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  float4* hx = smem4 + warp * kWarpHalo;
  float* hb = reinterpret_cast<float*>(smem4 + kTileWarps * kWarpHalo) + warp * kWarpHalo;
  const uint32_t ntiles = min(*V.tile_count, V.max_tiles);
  const uint32_t n = V.n;
  for (uint32_t t = blockIdx.x * kTileWarps + warp; t < ntiles; t += gridDim.x * kTileWarps) {
    const WarpTile W = load_warp_tile(V.tiles, t);
    const uint32_t p0 = W.p0(), p1 = W.p1(), halo = W.halo();
    const DevScene& S = V.scenes[W.scene()];
    if (sub >= S.substeps || it >= S.iterations) continue;  // uniform over the warp
    const bool staged = halo <= kWarpHalo;
    if (staged) {
      stage_rows(W, V.cur.xs, hx);
      stage_rows(W, V.cur.bv, hb);
    }
    cp_async_wait_all();
    __syncwarp();
    for (uint32_t i = p0 + lane; i < p1; i += 32) {
      const uint32_t f = tag_fluid(V.cur.tag[i]);
      if (!f) continue;
      const DevFluid& F = V.fluids[f - 1];
      if (F.rank != rank) continue;
      const float4 xi4 = V.cur.xs[i];
      const f3 xi = xyz(xi4);
      float rho = 0.0f, gss = 0.0f;
      f3 gs = mk(0.0f, 0.0f, 0.0f);
      const uint32_t cnt = V.ncount[i];
      auto one = [&](uint32_t h) {
        float4 xj;
        float bvj;
        if (staged) {
          xj = hx[h];
          bvj = hb[h];
        } else {
          const uint32_t j = halo_slot(V.tiles[t], h);
          xj = V.cur.xs[j];
          bvj = V.cur.bv[j];
        }
        const float mass = nbr_mass(bvj, xj.w, F.rho0);
        const f3 off = xi - xyz(xj);
        const float rsq = dot(off, off);
        rho += mass * poly6(rsq, F);
        const f3 g = spiky_vec(off, rsq, F) * mass;
        gs = gs + g;
        gss += dot(g, g) * xj.w;
      };
      for_each_h(V.nbr16 + i, n, cnt, one);
      V.cur.dens[i] = rho;
      const float C = rho * F.inv_rho0 - 1.0f;
      if (C <= 0.0f) {
        V.lambda[i] = 0.0f;
        continue;
      }
      const float gn = (dot(gs, gs) * xi4.w + gss) * (F.inv_rho0 * F.inv_rho0);
      const float at = F.compliance / (S.dt * S.dt);
      V.lambda[i] = -C / fmaxf(gn + at, 1e-20f);
    }
    __syncwarp();
  }
}

// positionDelta.ts:41-85 over warp tiles (the reaction on dynamic boundary
// neighbours goes into the fixed-point reaction sums by slot).
__global__ void __launch_bounds__(kTileThreads) k_t_delta(WorldView V, uint32_t rank, uint32_t sub, uint32_t it) {
  extern __shared__ float4 smem4[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  float4* hx = smem4 + warp * kWarpHalo;
  float* hb = reinterpret_cast<float*>(smem4 + kTileWarps * kWarpHalo) + warp * kWarpHalo;
  float* hl = reinterpret_cast<float*>(smem4 + kTileWarps * kWarpHalo) + kTileWarps * kWarpHalo + warp * kWarpHalo;
  const uint32_t ntiles = min(*V.tile_count, V.max_tiles);
  const uint32_t n = V.n;
  for (uint32_t t = blockIdx.x * kTileWarps + warp; t < ntiles; t += gridDim.x * kTileWarps) {
    const WarpTile W = load_warp_tile(V.tiles, t);
    const uint32_t p0 = W.p0(), p1 = W.p1(), halo = W.halo();
    const DevScene& S = V.scenes[W.scene()];
    if (sub >= S.substeps || it >= S.iterations) continue;
    const bool staged = halo <= kWarpHalo;
    if (staged) {
      stage_rows(W, V.cur.xs, hx);
      stage_rows(W, V.cur.bv, hb);
      stage_rows(W, (const float*)V.lambda, hl);
    }
    cp_async_wait_all();
    __syncwarp();
    for (uint32_t i = p0 + lane; i < p1; i += 32) {
      const uint32_t f = tag_fluid(V.cur.tag[i]);
      if (!f) continue;
      const DevFluid& F = V.fluids[f - 1];
      if (F.rank != rank) continue;
      const float4 xi4 = V.cur.xs[i];
      const f3 xi = xyz(xi4);
      const float li = V.lambda[i];
      const bool react = F.react_lo != F.react_hi && li != 0.0f;
      f3 sum = mk(0.0f, 0.0f, 0.0f);
      const uint32_t cnt = V.ncount[i];
      auto one = [&](uint32_t h) {
        float4 xj;
        float bvj, lj;
        if (staged) {
          xj = hx[h];
          bvj = hb[h];
          lj = hl[h];
        } else {
          const uint32_t j = halo_slot(V.tiles[t], h);
          xj = V.cur.xs[j];
          bvj = V.cur.bv[j];
          lj = V.lambda[j];
        }
        const float mass = nbr_mass(bvj, xj.w, F.rho0);
        const f3 off = xi - xyz(xj);
        const f3 g = spiky_vec(off, dot(off, off), F);
        sum = sum + g * ((li + lj) * mass);
        if (react && bvj > 0.0f && xj.w > 0.0f) {
          const uint32_t j = halo_slot(V.tiles[t], h);
          const uint32_t idj = V.ids[j];
          bool in = false;
          for (uint32_t b = 0; b < F.bnd_count; ++b) {
            const DevBoundary B = V.bnds[F.bnd_first + b];
            in = in || (idj >= B.start && idj < B.start + B.count);
          }
          if (in) acc_add(V.acc_react, j, g * (-(li / F.rho0) * (F.rho0 * bvj) * xj.w), F.react_scale);
        }
      };
      for_each_h(V.nbr16 + i, n, cnt, one);
      V.dx[i] = with_w((sum / F.rho0) * xi4.w, 0.0f);
    }
    __syncwarp();
  }
}

// velocity.ts:43-70 (XSPH) over warp tiles: committed positions and velocities.
__global__ void __launch_bounds__(kTileThreads) k_t_xsph(WorldView V, uint32_t rank, uint32_t sub) {
  extern __shared__ float4 smem4[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  float4* hx = smem4 + warp * kWarpHalo;
  float4* hv = smem4 + kTileWarps * kWarpHalo + warp * kWarpHalo;
  float* hb = reinterpret_cast<float*>(smem4 + 2 * kTileWarps * kWarpHalo) + warp * kWarpHalo;
  const uint32_t ntiles = min(*V.tile_count, V.max_tiles);
  const uint32_t n = V.n;
  for (uint32_t t = blockIdx.x * kTileWarps + warp; t < ntiles; t += gridDim.x * kTileWarps) {
    const WarpTile W = load_warp_tile(V.tiles, t);
    const uint32_t p0 = W.p0(), p1 = W.p1(), halo = W.halo();
    const DevScene& S = V.scenes[W.scene()];
    if (sub >= S.substeps) continue;
    const bool staged = halo <= kWarpHalo;
    if (staged) {
      stage_rows(W, V.cur.x, hx);
      stage_rows(W, V.cur.v, hv);
      stage_rows(W, V.cur.bv, hb);
    }
    cp_async_wait_all();
    __syncwarp();
    for (uint32_t i = p0 + lane; i < p1; i += 32) {
      const uint32_t f = tag_fluid(V.cur.tag[i]);
      if (!f) continue;
      const DevFluid& F = V.fluids[f - 1];
      if (F.rank != rank || !F.has_visc) continue;
      const f3 xi = xyz(V.cur.x[i]);
      const f3 vi = xyz(V.cur.v[i]);
      f3 sm = mk(0.0f, 0.0f, 0.0f);
      const uint32_t cnt = V.ncount[i];
      auto one = [&](uint32_t h) {
        float4 xj, vj;
        float bvj;
        if (staged) {
          xj = hx[h];
          vj = hv[h];
          bvj = hb[h];
        } else {
          const uint32_t j = halo_slot(V.tiles[t], h);
          xj = V.cur.x[j];
          vj = V.cur.v[j];
          bvj = V.cur.bv[j];
        }
        const f3 off = xi - xyz(xj);
        const float vol = bvj > 0.0f ? bvj : F.volume;
        sm = sm + ((xyz(vj) - vi) * poly6(dot(off, off), F)) * vol;
      };
      for_each_h(V.nbr16 + i, n, cnt, one);
      V.dv[i] = with_w(sm * F.c_xsph, 0.0f);
    }
    __syncwarp();
  }
}

constexpr size_t kSmemNbr = 16ull * kWarpHalo * kTileWarps;
constexpr size_t kSmemLambda = 20ull * kWarpHalo * kTileWarps;
constexpr size_t kSmemDelta = 24ull * kWarpHalo * kTileWarps;
constexpr size_t kSmemXsph = 36ull * kWarpHalo * kTileWarps;

}  // namespace pf
