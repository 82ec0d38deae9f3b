// grid_sort.cu — stable counting sort of particles by hash-grid cell key.
//
// Replaces the reference's 8-kernel HashGrid rebuild (src/core/hashGrid/
// cellIndex.ts:113-170, sort.ts:72-192): the same histogram -> exclusive scan
// -> scatter structure, re-planned for B200:
//   * the histogram aggregates equal keys inside a warp with __match_any_sync,
//     so a warp issues one L2 atomic per distinct key;
//   * the scan is a single-pass decoupled look-back over 4096-entry tiles, so
//     the bucket count is not capped at 1024^2 as in the two-level
//     workgroup scan (sort.ts:22-28);
//   * the scatter is stable: equal keys inside a warp are ranked by lane, and
//     the (rare at low occupancy) cells filled by several warps are re-sorted
//     by a fix-up that runs only over those cells.
// Every spin-wait is bounded and reports DEV_ERR_LOOKBACK_TIMEOUT.

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>

#include "grid_sort.cuh"

namespace pf {

namespace {

constexpr uint32_t kHistThreads = 256;
constexpr uint32_t kScanThreads = 256;
constexpr uint32_t kScanItems = 16;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;  // 4096
constexpr uint32_t kSmallMax = 16;     // thread-per-cell fix-up
constexpr uint32_t kMidMax = 4096;     // CTA bitonic fix-up in shared memory
constexpr uint32_t kFixThreads = 256;
constexpr uint32_t kMortonBias = 512;
constexpr int32_t kCellCoordMax = 1 << 30;

__device__ __forceinline__ uint32_t part1by2(uint32_t n) {
  uint32_t m = n & 0x000003ffu;
  m = (m | (m << 16)) & 0xff0000ffu;
  m = (m | (m << 8)) & 0x0300f00fu;
  m = (m | (m << 4)) & 0x030c30c3u;
  m = (m | (m << 2)) & 0x09249249u;
  return m;
}

// floor((p - o) / cell) as a saturating i32 (NaN -> 0), with the IEEE
// subtract and divide the reference's WGSL performs (no contraction).
__device__ __forceinline__ int32_t cell_coord(float p, float o, float cell) {
  return __float2int_rz(floorf(__fdiv_rn(__fsub_rn(p, o), cell)));
}

__device__ __forceinline__ uint32_t cell_key(const KeyFn& k, float px, float py, float pz,
                                             uint32_t* over) {
  const int32_t cxr = cell_coord(px, k.ox, k.cell);
  const int32_t cyr = cell_coord(py, k.oy, k.cell);
  const int32_t czr = cell_coord(pz, k.oz, k.cell);
  if (k.kind == PF_KEY_LINEAR) {
    const int64_t ax = (int64_t)cxr - k.lo[0], ay = (int64_t)cyr - k.lo[1], az = (int64_t)czr - k.lo[2];
    const int64_t cx = ax < 0 ? 0 : (ax >= (int64_t)k.dims[0] ? (int64_t)k.dims[0] - 1 : ax);
    const int64_t cy = ay < 0 ? 0 : (ay >= (int64_t)k.dims[1] ? (int64_t)k.dims[1] - 1 : ay);
    const int64_t cz = az < 0 ? 0 : (az >= (int64_t)k.dims[2] ? (int64_t)k.dims[2] - 1 : az);
    *over = (cx != ax || cy != ay || cz != az) ? 1u : 0u;
    return (uint32_t)cx + k.dims[0] * ((uint32_t)cy + k.dims[1] * (uint32_t)cz);
  }
  const int32_t cx = min(max(cxr, -kCellCoordMax), kCellCoordMax - 1);
  const int32_t cy = min(max(cyr, -kCellCoordMax), kCellCoordMax - 1);
  const int32_t cz = min(max(czr, -kCellCoordMax), kCellCoordMax - 1);
  const int32_t b = (int32_t)kMortonBias;
  const bool o = cxr != cx || cyr != cy || czr != cz || cx < -b || cx >= b || cy < -b || cy >= b ||
                 cz < -b || cz >= b;
  *over = o ? 1u : 0u;
  const uint32_t ux = (uint32_t)cx + kMortonBias, uy = (uint32_t)cy + kMortonBias,
                 uz = (uint32_t)cz + kMortonBias;
  return (part1by2(ux) | (part1by2(uy) << 1) | (part1by2(uz) << 2)) & k.mask;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---------------------------------------------------------------- keys ----
__global__ void __launch_bounds__(kHistThreads)
k_keys_hist(const float4* __restrict__ pos, uint32_t n, KeyFn kf, uint32_t* __restrict__ keys,
            uint32_t* __restrict__ counts, uint32_t* __restrict__ overflow) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  uint32_t key = 0, over = 0;
  if (valid) {
    const float4 p = __ldg(pos + i);
    key = cell_key(kf, p.x, p.y, p.z, &over);
    keys[i] = key;
  }
  const uint32_t active = __ballot_sync(0xffffffffu, valid);
  if (valid) {
    const uint32_t peers = __match_any_sync(active, key);
    if (lane_id() == (uint32_t)(__ffs(peers) - 1)) atomicAdd(counts + key, (uint32_t)__popc(peers));
  }
  if (__any_sync(0xffffffffu, over) && lane_id() == 0) atomicOr(overflow, 1u);
}

// ---------------------------------------------------------------- scan ----
// Tile status word: high 32 bits flag (0 none, 1 aggregate, 2 inclusive
// prefix), low 32 bits value. One 64-bit store publishes both.
constexpr uint64_t kFlagAgg = 1ull << 32;
constexpr uint64_t kFlagInc = 2ull << 32;

__device__ __forceinline__ uint64_t load_status(const uint64_t* p) {
  return *reinterpret_cast<const volatile unsigned long long*>(p);
}
__device__ __forceinline__ void store_status(uint64_t* p, uint64_t v) {
  atomicExch(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}

__global__ void __launch_bounds__(kScanThreads)
k_scan(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t* __restrict__ zero_out,
       uint64_t n, uint64_t* __restrict__ status, uint32_t* __restrict__ counters) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t s_prefix;
  if (threadIdx.x == 0) s_tile = atomicAdd(counters + kCounterTicket, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t base = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  const bool full = base + kScanItems <= n;
  if (full) {
    const uint4* src = reinterpret_cast<const uint4*>(in + base);
#pragma unroll
    for (int q = 0; q < (int)kScanItems / 4; ++q) {
      const uint4 w = src[q];
      v[4 * q] = w.x;
      v[4 * q + 1] = w.y;
      v[4 * q + 2] = w.z;
      v[4 * q + 3] = w.w;
    }
  } else {
#pragma unroll
    for (int k = 0; k < (int)kScanItems; ++k) v[k] = (base + k < n) ? in[base + k] : 0u;
  }
  uint32_t sum = 0;
#pragma unroll
  for (int k = 0; k < (int)kScanItems; ++k) {
    const uint32_t t = v[k];
    v[k] = sum;
    sum += t;
  }
  // Warp inclusive scan of the per-thread sums.
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  uint32_t x = sum;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= (uint32_t)off) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, wi, off);
      if (lane >= (uint32_t)off) wi += y;
    }
    const uint32_t aggregate = __shfl_sync(0xffffffffu, wi, kScanThreads / 32 - 1);
    if (lane < kScanThreads / 32) s_warp[lane] = wi - w;  // exclusive warp offsets
    // Decoupled look-back (single pass).
    uint32_t excl = 0;
    if (tile == 0) {
      if (lane == 0) store_status(status, kFlagInc | aggregate);
    } else {
      if (lane == 0) store_status(status + tile, kFlagAgg | aggregate);
      int64_t pred = (int64_t)tile - 1 - (int64_t)lane;
      bool timed_out = false;
      for (;;) {
        uint64_t st = kFlagInc;  // lanes past tile 0 contribute nothing
        if (pred >= 0) {
          uint32_t spins = 0;
          st = load_status(status + pred);
          while ((st >> 32) == 0 && spins < kLookbackSpinLimit) {
            __nanosleep(32);
            st = load_status(status + pred);
            ++spins;
          }
          if ((st >> 32) == 0) {
            timed_out = true;
            st = kFlagInc;
          }
        }
        const uint32_t inc = __ballot_sync(0xffffffffu, (st >> 32) == 2 || pred < 0);
        const uint32_t stop = inc ? (uint32_t)(__ffs(inc) - 1) : 31u;
        uint32_t val = (lane <= stop && pred >= 0) ? (uint32_t)st : 0u;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) val += __shfl_xor_sync(0xffffffffu, val, off);
        excl += val;
        if (inc) break;
        pred -= 32;
      }
      if (__any_sync(0xffffffffu, timed_out) && lane == 0) atomicOr(counters + kCounterError, DEV_ERR_LOOKBACK_TIMEOUT);
      if (lane == 0) store_status(status + tile, kFlagInc | (excl + aggregate));
    }
    if (lane == 0) s_prefix = excl;
  }
  __syncthreads();
  const uint32_t prefix = s_prefix + s_warp[warp] + (x - sum);
  if (full) {
    uint4* dst = reinterpret_cast<uint4*>(out + base);
#pragma unroll
    for (int q = 0; q < (int)kScanItems / 4; ++q)
      dst[q] = make_uint4(prefix + v[4 * q], prefix + v[4 * q + 1], prefix + v[4 * q + 2], prefix + v[4 * q + 3]);
    if (zero_out) {
      uint4* z = reinterpret_cast<uint4*>(zero_out + base);
#pragma unroll
      for (int q = 0; q < (int)kScanItems / 4; ++q) z[q] = make_uint4(0, 0, 0, 0);
    }
  } else {
#pragma unroll
    for (int k = 0; k < (int)kScanItems; ++k)
      if (base + k < n) {
        out[base + k] = prefix + v[k];
        if (zero_out) zero_out[base + k] = 0;
      }
  }
}

// ------------------------------------------------------------- scatter ----
struct Lists {
  uint32_t* small;
  uint32_t* mid;
  uint32_t* giant;
  uint32_t small_cap, mid_cap, giant_cap;
};

__global__ void __launch_bounds__(kHistThreads)
k_scatter(const uint32_t* __restrict__ keys, uint32_t n, const uint32_t* __restrict__ start,
          const uint32_t* __restrict__ counts, uint32_t* __restrict__ fill, uint32_t* __restrict__ perm,
          uint32_t* __restrict__ dirty_bits, Lists lists, uint32_t* __restrict__ counters) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n;
  const uint32_t key = valid ? keys[i] : 0u;
  const uint32_t active = __ballot_sync(0xffffffffu, valid);
  if (!valid) return;
  const uint32_t peers = __match_any_sync(active, key);
  const uint32_t leader = (uint32_t)(__ffs(peers) - 1);
  uint32_t base = 0;
  // 0: nothing to record; 1/2/3: this lane's cell goes on the small / mid /
  // giant fix-up list (its run was started by another warp)
  uint32_t need = 0;
  if (lane_id() == leader) {
    const uint32_t old = atomicAdd(fill + key, (uint32_t)__popc(peers));
    base = start[key] + old;
    if (old != 0) {
      const uint32_t bit = 1u << (key & 31u);
      const uint32_t prev = atomicOr(dirty_bits + (key >> 5), bit);
      if (!(prev & bit)) {
        const uint32_t c = counts[key];
        need = c <= kSmallMax ? 1u : (c <= kMidMax ? 2u : 3u);
      }
    }
  }
  // one counter atomic per warp and list for the cells this warp records
#pragma unroll
  for (uint32_t l = 1; l <= 3; ++l) {
    const uint32_t mask = __ballot_sync(active, need == l);
    if (!mask) continue;
    const uint32_t first = (uint32_t)(__ffs(mask) - 1);
    const uint32_t ctr = l == 1 ? kCounterSmall : (l == 2 ? kCounterMid : kCounterGiant);
    uint32_t at = 0;
    if (lane_id() == first) at = atomicAdd(counters + ctr, (uint32_t)__popc(mask));
    at = __shfl_sync(active, at, first) + __popc(mask & lanemask_lt());
    if (need == l) {
      uint32_t* list = l == 1 ? lists.small : (l == 2 ? lists.mid : lists.giant);
      const uint32_t cap = l == 1 ? lists.small_cap : (l == 2 ? lists.mid_cap : lists.giant_cap);
      if (at < cap) list[at] = key;
      else atomicOr(counters + kCounterError, DEV_ERR_SORT_CAPACITY);
    }
  }
  base = __shfl_sync(active, base, leader);
  const uint32_t slot = base + __popc(peers & lanemask_lt());
  if (slot < n)
    perm[slot] = i;
  else
    atomicOr(counters + kCounterError, DEV_ERR_SORT_CAPACITY);
}

// -------------------------------------------------------------- fix-up ----
__device__ __forceinline__ void cswap(uint32_t& a, uint32_t& b) {
  const uint32_t lo = min(a, b), hi = max(a, b);
  a = lo;
  b = hi;
}

__global__ void __launch_bounds__(kFixThreads)
k_fix_small(const uint32_t* __restrict__ list, const uint32_t* __restrict__ counters_len,
            const uint32_t* __restrict__ start, const uint32_t* __restrict__ counts,
            uint32_t* __restrict__ perm, uint32_t cap) {
  const uint32_t total = min(*counters_len, cap);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const uint32_t c = list[t];
    const uint32_t s = start[c], m = counts[c];
    uint32_t v[kSmallMax];
#pragma unroll
    for (int k = 0; k < (int)kSmallMax; ++k) v[k] = (uint32_t)k < m ? perm[s + k] : 0xffffffffu;
    // Odd-even transposition network: kSmallMax rounds sort kSmallMax keys.
#pragma unroll
    for (int r = 0; r < (int)kSmallMax; ++r) {
#pragma unroll
      for (int k = r & 1; k + 1 < (int)kSmallMax; k += 2) cswap(v[k], v[k + 1]);
    }
#pragma unroll
    for (int k = 0; k < (int)kSmallMax; ++k)
      if ((uint32_t)k < m) perm[s + k] = v[k];
  }
}

__global__ void __launch_bounds__(kFixThreads)
k_fix_mid(const uint32_t* __restrict__ list, const uint32_t* __restrict__ counters_len,
          const uint32_t* __restrict__ start, const uint32_t* __restrict__ counts,
          uint32_t* __restrict__ perm, uint32_t cap) {
  __shared__ uint32_t sh[kMidMax];
  const uint32_t total = min(*counters_len, cap);
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t c = list[t];
    const uint32_t s = start[c], m = counts[c];
    uint32_t P = 32;
    while (P < m) P <<= 1;
    for (uint32_t k = threadIdx.x; k < P; k += blockDim.x) sh[k] = k < m ? perm[s + k] : 0xffffffffu;
    __syncthreads();
    for (uint32_t size = 2; size <= P; size <<= 1) {
      for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
        for (uint32_t k = threadIdx.x; k < P; k += blockDim.x) {
          const uint32_t j = k ^ stride;
          if (j > k) {
            const uint32_t a = sh[k], b = sh[j];
            const bool up = (k & size) == 0;
            if ((a > b) == up) {
              sh[k] = b;
              sh[j] = a;
            }
          }
        }
        __syncthreads();
      }
    }
    for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) perm[s + k] = sh[k];
    __syncthreads();
  }
}

// Giant cells (> kMidMax elements): one CTA runs a stable LSD radix sort
// (8-bit digits) over the cell's run, ping-ponging with the same range of a
// scratch buffer, 256 elements per round.
__global__ void __launch_bounds__(kFixThreads)
k_fix_giant(const uint32_t* __restrict__ list, const uint32_t* __restrict__ counters_len,
            const uint32_t* __restrict__ start, const uint32_t* __restrict__ counts,
            uint32_t* __restrict__ perm, uint32_t* __restrict__ tmp, uint32_t cap, uint32_t value_bits) {
  __shared__ uint32_t hist[256];
  __shared__ uint32_t offs[256];
  __shared__ uint32_t wcount[kFixThreads / 32][256];
  const uint32_t total = min(*counters_len, cap);
  const uint32_t lane = lane_id(), warp = threadIdx.x >> 5;
  const uint32_t passes = (value_bits + 7) / 8;
  for (uint32_t t = blockIdx.x; t < total; t += gridDim.x) {
    const uint32_t c = list[t];
    const uint32_t s = start[c], m = counts[c];
    uint32_t* src = perm + s;
    uint32_t* dst = tmp + s;
    for (uint32_t pass = 0; pass < passes; ++pass) {
      const uint32_t shift = 8 * pass;
      hist[threadIdx.x] = 0;
      for (uint32_t w = 0; w < kFixThreads / 32; ++w) wcount[w][threadIdx.x] = 0;
      __syncthreads();
      for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) atomicAdd(&hist[(src[k] >> shift) & 255u], 1u);
      __syncthreads();
      if (warp == 0) {
        uint32_t run = 0;
        for (uint32_t q = 0; q < 8; ++q) {
          const uint32_t d = q * 32 + lane;
          const uint32_t h = hist[d];
          uint32_t x = h;
#pragma unroll
          for (int off = 1; off < 32; off <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= (uint32_t)off) x += y;
          }
          offs[d] = run + x - h;
          run += __shfl_sync(0xffffffffu, x, 31);
        }
      }
      __syncthreads();
      for (uint32_t r = 0; r < m; r += blockDim.x) {
        const uint32_t k = r + threadIdx.x;
        const bool valid = k < m;
        const uint32_t val = valid ? src[k] : 0u;
        const uint32_t d = (val >> shift) & 255u;
        const uint32_t active = __ballot_sync(0xffffffffu, valid);
        uint32_t peers = 0, rank = 0;
        if (valid) {
          peers = __match_any_sync(active, d);
          rank = __popc(peers & lanemask_lt());
          if (lane == (uint32_t)(__ffs(peers) - 1)) wcount[warp][d] = __popc(peers);
        }
        __syncthreads();
        if (valid) {
          uint32_t before = 0;
          for (uint32_t w = 0; w < warp; ++w) before += wcount[w][d];
          dst[offs[d] + before + rank] = val;
        }
        __syncthreads();
        {
          const uint32_t dd = threadIdx.x;
          uint32_t add = 0;
          for (uint32_t w = 0; w < kFixThreads / 32; ++w) {
            add += wcount[w][dd];
            wcount[w][dd] = 0;
          }
          offs[dd] += add;
        }
        __syncthreads();
      }
      uint32_t* sw = src;
      src = dst;
      dst = sw;
      __syncthreads();
    }
    if (src != perm + s) {
      for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) perm[s + k] = src[k];
    }
    __syncthreads();
  }
}

}  // namespace

bool make_key_fn(const pf_grid_desc& g, KeyFn* out, uint64_t* cells) {
  KeyFn k{};
  k.kind = g.key_kind;
  k.ox = g.origin[0];
  k.oy = g.origin[1];
  k.oz = g.origin[2];
  k.cell = g.cell_size;
  if (!(g.cell_size > 0) || !std::isfinite(g.cell_size)) return false;
  uint64_t C = 0;
  if (g.key_kind == PF_KEY_LINEAR) {
    if (!g.dims[0] || !g.dims[1] || !g.dims[2]) return false;
    C = (uint64_t)g.dims[0] * g.dims[1] * g.dims[2];
    for (int a = 0; a < 3; ++a) {
      k.lo[a] = 0;
      k.dims[a] = g.dims[a];
    }
  } else if (g.key_kind == PF_KEY_MORTON) {
    if (!g.table_size || (g.table_size & (g.table_size - 1))) return false;
    C = g.table_size;
    k.mask = g.table_size - 1;
  } else {
    return false;
  }
  if (C > 0x7fffffffull) return false;
  *out = k;
  *cells = C;
  return true;
}

uint32_t scan_tiles(uint64_t n) { return (uint32_t)((n + kScanTile - 1) / kScanTile); }

namespace {
struct ListCaps {
  uint32_t small, mid, giant;
};
ListCaps list_caps(uint32_t n, uint64_t C) {
  const uint64_t cmax = std::min<uint64_t>(C, n / 2 + 1);
  ListCaps c;
  c.small = (uint32_t)cmax;
  c.mid = (uint32_t)std::min<uint64_t>(C, n / (kSmallMax + 1) + 1);
  c.giant = (uint32_t)std::min<uint64_t>(C, n / (kMidMax + 1) + 1);
  return c;
}
size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
}  // namespace

size_t sort_scratch_bytes(uint32_t n, uint64_t C) {
  const ListCaps lc = list_caps(n, C);
  size_t b = 0;
  b += align256(4ull * n);                    // keys
  b += align256(4ull * C);                    // fill
  b += align256(4ull * ((C + 31) / 32));      // dirty bits
  b += align256(4ull * ((uint64_t)lc.small + lc.mid + lc.giant));  // lists
  b += align256(8ull * scan_tiles(C));        // tile status
  b += align256(4ull * kNumCounters);         // counters
  b += align256(4ull * n);                    // radix tmp
  return b;
}

void sort_scratch_carve(void* base, uint32_t n, uint64_t C, SortScratch* s) {
  const ListCaps lc = list_caps(n, C);
  char* p = static_cast<char*>(base);
  s->keys = reinterpret_cast<uint32_t*>(p);
  p += align256(4ull * n);
  s->fill = reinterpret_cast<uint32_t*>(p);
  p += align256(4ull * C);
  s->dirty_bits = reinterpret_cast<uint32_t*>(p);
  p += align256(4ull * ((C + 31) / 32));
  s->lists = reinterpret_cast<uint32_t*>(p);
  p += align256(4ull * ((uint64_t)lc.small + lc.mid + lc.giant));
  s->tile_status = reinterpret_cast<uint64_t*>(p);
  p += align256(8ull * scan_tiles(C));
  s->counters = reinterpret_cast<uint32_t*>(p);
  p += align256(4ull * kNumCounters);
  s->radix_tmp = reinterpret_cast<uint32_t*>(p);
  s->n_cap = n;
  s->c_cap = (uint32_t)C;
  s->list_cap = lc.small;
  s->tiles_cap = scan_tiles(C);
}

void launch_keys_hist(const float4* pos, uint32_t n, const KeyFn& kf, uint32_t* keys, uint32_t* counts,
                      uint32_t* overflow, cudaStream_t st) {
  if (n == 0) return;
  k_keys_hist<<<div_up(n, kHistThreads), kHistThreads, 0, st>>>(pos, n, kf, keys, counts, overflow);
}

void launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t* zero_out, uint64_t n,
                           uint64_t* tile_status, uint32_t* counters, cudaStream_t st) {
  if (n == 0) return;
  const uint32_t tiles = scan_tiles(n);
  cudaMemsetAsync(tile_status, 0, 8ull * tiles, st);
  cudaMemsetAsync(counters + kCounterTicket, 0, 4, st);
  k_scan<<<tiles, kScanThreads, 0, st>>>(in, out, zero_out, n, tile_status, counters);
}

void launch_sort_from_hist(const uint32_t* keys, uint32_t n, uint64_t C, const uint32_t* counts,
                           uint32_t* start, uint32_t* perm, const SortScratch& s, cudaStream_t st) {
  if (C == 0) return;
  const ListCaps lc = list_caps(n, C);
  // Reset the fix-up lists and dirty bits (the error word is left to the caller).
  cudaMemsetAsync(s.counters + kCounterSmall, 0, 3 * 4, st);
  cudaMemsetAsync(s.dirty_bits, 0, 4ull * ((C + 31) / 32), st);
  launch_exclusive_scan(counts, start, s.fill, C, s.tile_status, s.counters, st);
  if (n == 0) return;
  Lists L;
  L.small = s.lists;
  L.mid = s.lists + lc.small;
  L.giant = s.lists + lc.small + lc.mid;
  L.small_cap = lc.small;
  L.mid_cap = lc.mid;
  L.giant_cap = lc.giant;
  k_scatter<<<div_up(n, kHistThreads), kHistThreads, 0, st>>>(keys, n, start, counts, s.fill, perm,
                                                             s.dirty_bits, L, s.counters);
  const int sms = sm_count();
  k_fix_small<<<sms * 8, kFixThreads, 0, st>>>(L.small, s.counters + kCounterSmall, start, counts, perm,
                                               L.small_cap);
  k_fix_mid<<<sms * 4, kFixThreads, 0, st>>>(L.mid, s.counters + kCounterMid, start, counts, perm,
                                             L.mid_cap);
  uint32_t bits = 1;
  while (bits < 32 && (1ull << bits) < n) ++bits;
  k_fix_giant<<<sms, kFixThreads, 0, st>>>(L.giant, s.counters + kCounterGiant, start, counts, perm,
                                           s.radix_tmp, L.giant_cap, bits);
}

}  // namespace pf
