// grid_sort.cu — stable counting sort of particles by hash-grid cell key.
//
// Replaces the reference's 8-kernel HashGrid rebuild (src/core/hashGrid/
// cellIndex.ts:113-170, sort.ts:72-192): the reference's histogram ->
// exclusive scan -> scatter becomes, for B200,
//   * keys with every radix pass's digit counts, from shared-memory
//     histograms (one global atomic per digit per block);
//   * one least-significant-digit radix pass per 11 key bits (two for a
//     128^3 grid), each three steps: every tile of 4096 elements counts its
//     digits; the counts are scanned over the tiles per digit (in chunks of
//     32 tiles, then over the chunks); every tile ranks its elements by digit
//     in element order with warp-aggregated ranks (__match_any_sync) and
//     writes them out run by run through shared memory. The passes are
//     stable, unlike the reference's atomic write cursor (sort.ts:187-192),
//     so the permutation lists each cell's particles in ascending index;
//   * cell counts from the sorted keys (one atomic per run of equal keys in a
//     warp) and a single-pass decoupled look-back scan to the cell starts,
//     so the bucket count is not capped at 1024^2 as in the two-level
//     workgroup scan (sort.ts:22-28).
// The one spin-wait (the start scan's look-back) is bounded and reports
// DEV_ERR_LOOKBACK_TIMEOUT.

#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <set>
#include <string>

#include "grid_sort.cuh"

namespace pf {

namespace {

constexpr uint32_t kHistThreads = 256;
constexpr uint32_t kKeysUnroll = 4;
constexpr uint32_t kScanThreads = 256;
constexpr uint32_t kScanItems = 16;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;  // 4096
// radix scatter: 512 threads x 8 elements per tile, elements warp-striped
// (warp w ranks elements [256 w, 256 w + 256) of its tile, 32 per round)
constexpr uint32_t kOsThreads = 512;
constexpr uint32_t kOsItems = 8;
constexpr uint32_t kOsWarps = kOsThreads / 32;
constexpr uint32_t kOsStripe = kOsItems * 32;
static_assert(kOsThreads * kOsItems == kRadixTile, "tile size");
// shared memory of a scatter, in words: two tile buffers of keys (and two of
// values unless the values are the element indices); the staged tile (keys
// then values); the warp histograms (u16); each digit's first tile position
// and first output position
__host__ __device__ constexpr size_t scatter_smem_bytes(uint32_t digits, bool first) {
  return 4ull * ((first ? 2ull : 4ull) * kRadixTile + 2ull * kRadixTile + kOsWarps * digits / 2 + 2ull * digits);
}
constexpr size_t kOsSmemBytes = scatter_smem_bytes(kRadixMaxDigits, false);  // the largest
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
       uint64_t n, uint64_t* __restrict__ status, uint32_t* __restrict__ counters, uint32_t vec) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t s_prefix;
  if (threadIdx.x == 0) s_tile = atomicAdd(counters + kCounterTicket, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t base = (uint64_t)tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  // 16-byte loads and stores when every array is 16-byte aligned
  const bool full = vec && base + kScanItems <= n;
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


// -------------------------------------------------------- keys + digits ----
// Keys of every element with the radix digit counts of every pass, in a
// grid-stride loop: each block keeps its digit histograms in shared memory
// and adds them to the global counts once.
__global__ void __launch_bounds__(kHistThreads)
k_keys_digits(const float4* __restrict__ pos, uint32_t n, KeyFn kf, DigitHist h, uint32_t* __restrict__ keys,
              uint32_t* __restrict__ overflow) {
  extern __shared__ uint32_t sh[];
  digit_hist_zero(sh, h);
  __syncthreads();
  uint32_t over_any = 0;
  const uint32_t stride = gridDim.x * blockDim.x;
  // kKeysUnroll positions in flight per thread before their keys
  for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += kKeysUnroll * stride) {
    float4 p[kKeysUnroll];
#pragma unroll
    for (uint32_t q = 0; q < kKeysUnroll; ++q)
      if (i0 + q * stride < n) p[q] = __ldg(pos + i0 + q * stride);
#pragma unroll
    for (uint32_t q = 0; q < kKeysUnroll; ++q) {
      const uint32_t i = i0 + q * stride;
      if (i >= n) break;
      uint32_t over = 0;
      const uint32_t key = cell_key(kf, p[q].x, p[q].y, p[q].z, &over);
      keys[i] = key;
      over_any |= over;
      digit_hist_add(sh, h, key);
    }
  }
  if (__any_sync(0xffffffffu, over_any) && lane_id() == 0) atomicOr(overflow, 1u);
  __syncthreads();
  digit_hist_flush(sh, h);
}

// Each pass's digit counts -> each digit's first output position (one block
// of 1024 threads per pass, two digits per thread).
__global__ void __launch_bounds__(1024) k_digit_first(uint32_t* __restrict__ dc, uint32_t digits) {
  __shared__ uint32_t s_warp[32];
  uint32_t* c = dc + blockIdx.x * kRadixMaxDigits;
  const uint32_t t = threadIdx.x, lane = lane_id(), warp = t >> 5;
  const uint32_t a = 2 * t < digits ? c[2 * t] : 0u, b = 2 * t + 1 < digits ? c[2 * t + 1] : 0u;
  const uint32_t own = a + b;
  uint32_t x = own;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= (uint32_t)off) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  uint32_t before = 0;
  for (uint32_t w = 0; w < warp; ++w) before += s_warp[w];
  const uint32_t excl = before + x - own;
  if (2 * t < digits) c[2 * t] = excl;
  if (2 * t + 1 < digits) c[2 * t + 1] = excl + a;
}

// ------------------------------------------------------------ radix pass ----
// A pass over digit (key >> shift) & (digits - 1) runs as three kernels: each
// tile of kRadixTile elements counts its digits (k_tile_counts); the counts
// are scanned over the tiles per digit, in chunks of kScanChunk tiles
// (k_tile_scan_chunk, k_tile_scan_chunks), giving each tile its first output
// position per digit; each tile then ranks its elements by digit in element
// order and writes them out digit run by digit run (k_radix_scatter). No
// kernel waits on another block.
constexpr uint32_t kScanChunk = 32;  // tiles per chunk of the tile-count scan
constexpr uint32_t kCountThreads = 256;
constexpr uint32_t kCountItems = kRadixTile / kCountThreads;  // 16: four 16-byte loads
static_assert(kCountItems % 4 == 0, "tile count loads");

// Digit counts of tile blockIdx.x: row tile of `tcount` (digits entries).
// `vec`: kin is 16-byte aligned (whole tiles load four keys at a time).
__global__ void __launch_bounds__(kCountThreads)
k_tile_counts(const uint32_t* __restrict__ kin, uint32_t n, uint32_t shift, uint32_t digits,
              uint32_t* __restrict__ tcount, uint32_t vec) {
  __shared__ uint32_t h[kRadixMaxDigits];
  for (uint32_t d = threadIdx.x; d < digits; d += kCountThreads) h[d] = 0u;
  __syncthreads();
  const uint32_t mask = digits - 1u;
  const size_t base = (size_t)blockIdx.x * kRadixTile;
  if (vec && base + kRadixTile <= n) {
    const uint4* src = reinterpret_cast<const uint4*>(kin + base);
    uint4 v[kCountItems / 4];
#pragma unroll
    for (uint32_t q = 0; q < kCountItems / 4; ++q) v[q] = __ldg(src + threadIdx.x + q * kCountThreads);
#pragma unroll
    for (uint32_t q = 0; q < kCountItems / 4; ++q) {
      atomicAdd(h + ((v[q].x >> shift) & mask), 1u);
      atomicAdd(h + ((v[q].y >> shift) & mask), 1u);
      atomicAdd(h + ((v[q].z >> shift) & mask), 1u);
      atomicAdd(h + ((v[q].w >> shift) & mask), 1u);
    }
  } else {
#pragma unroll 4
    for (uint32_t i = threadIdx.x; i < kRadixTile; i += kCountThreads) {
      const size_t e = base + i;
      if (e < n) atomicAdd(h + ((__ldg(kin + e) >> shift) & mask), 1u);
    }
  }
  __syncthreads();
  uint32_t* row = tcount + (size_t)blockIdx.x * digits;
  for (uint32_t d = threadIdx.x; d < digits; d += kCountThreads) row[d] = h[d];
}

// Per digit (one thread each), the exclusive running sum over the tiles of
// chunk blockIdx.x, in place, and the chunk's total into `csum`. With
// `first` (a pass of one chunk), csum gets the digit's first output position
// instead, so no scan over the chunks is needed.
__global__ void __launch_bounds__(256)
k_tile_scan_chunk(uint32_t* __restrict__ tcount, uint32_t tiles, uint32_t digits, uint32_t* __restrict__ csum,
                  const uint32_t* __restrict__ first) {
  const uint32_t d = blockIdx.y * blockDim.x + threadIdx.x;
  if (d >= digits) return;
  const uint32_t t0 = blockIdx.x * kScanChunk, t1 = min(t0 + kScanChunk, tiles);
  uint32_t v[kScanChunk];
#pragma unroll
  for (uint32_t q = 0; q < kScanChunk; ++q) v[q] = t0 + q < t1 ? tcount[(size_t)(t0 + q) * digits + d] : 0u;
  uint32_t run = 0;
#pragma unroll
  for (uint32_t q = 0; q < kScanChunk; ++q) {
    if (t0 + q < t1) tcount[(size_t)(t0 + q) * digits + d] = run;
    run += v[q];
  }
  csum[(size_t)blockIdx.x * digits + d] = first ? first[d] : run;
}

// Per digit (one warp each, 32 chunks per round), the chunk totals -> each
// chunk's first output position (the digit's first position plus the counts
// of the chunks before), in place.
__global__ void __launch_bounds__(256)
k_tile_scan_chunks(uint32_t* __restrict__ csum, uint32_t chunks, uint32_t digits, const uint32_t* __restrict__ first) {
  const uint32_t d = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const uint32_t lane = lane_id();
  if (d >= digits) return;  // whole warps
  uint32_t run = first[d];
  for (uint32_t c0 = 0; c0 < chunks; c0 += 32) {
    const uint32_t c = c0 + lane;
    const uint32_t v = c < chunks ? csum[(size_t)c * digits + d] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
      if (lane >= (uint32_t)off) x += y;
    }
    if (c < chunks) csum[(size_t)c * digits + d] = run + x - v;
    run += __shfl_sync(0xffffffffu, x, 31);
  }
}

// Asynchronous global -> shared copies (cp.async): 16 bytes with zero fill
// past src_bytes, or one 4-byte element.
__device__ __forceinline__ void cp_async16(uint32_t* dst, const uint32_t* src, uint32_t src_bytes) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t* dst, const uint32_t* src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Copy tile `tile` of `src` (its elements below n) into dst[0, kRadixTile):
// 16-byte copies when src is 16-byte aligned, else element by element.
__device__ __forceinline__ void tile_fetch(uint32_t* dst, const uint32_t* __restrict__ src, uint32_t tile,
                                           uint32_t n, bool vec) {
  const uint32_t base = tile * kRadixTile;  // n < 2^30
  const uint32_t valid = min(kRadixTile, n - base);
  if (vec) {
#pragma unroll
    for (uint32_t c = threadIdx.x; c < kRadixTile / 4; c += kOsThreads) {
      const uint32_t e = 4 * c;
      if (e < valid) cp_async16(dst + e, src + base + e, 4 * min(4u, valid - e));
    }
  } else {
    for (uint32_t e = threadIdx.x; e < valid; e += kOsThreads) cp_async4(dst + e, src + base + e);
  }
}

// The lanes of `active` whose digit d (of `bits` bits) equals this lane's:
// one ballot per digit bit, each keeping the lanes that agree on that bit.
// Called by every lane of `active` together.
// kW > 0: the digits have exactly kW bits (bits is then ignored).
template <uint32_t kW>
__device__ __forceinline__ uint32_t digit_peers(uint32_t d, uint32_t bits, uint32_t active) {
  uint32_t m = active;
#pragma unroll
  for (uint32_t b = 0; b < (kW ? kW : kRadixMaxBits); ++b)
    if (kW || b < bits) {  // uniform over the warp
      const bool set = (d >> b) & 1u;
      const uint32_t v = __ballot_sync(active, set);
      m &= set ? v : ~v;
    }
  return m;
}

// The scatter of one stable LSD pass, a persistent kernel: each block takes
// tiles blockIdx.x, blockIdx.x + gridDim.x, ... and copies the next tile's
// keys (and values) into shared memory while it ranks the current one. A
// tile ranks its elements by digit in element order (warp-striped rounds of
// 32: equal digits found by digit_peers (kBallot) or __match_any_sync, ranked
// against a per-warp digit histogram; then the warps' counts scanned per
// digit), stages them in digit order in shared
// memory and writes each digit's run to the run's first output position (the
// tile's scanned count plus its chunk's base).
// kFirst: the values are the element indices (no value input).
// kW: the digit width when it is fixed at compile time (0: any width).
// kLast: the keys are not written out; instead the staged tile, which is in
// key order, adds the length of every run of equal keys in a warp's 32
// entries to count[key] (the cell counts of the sort).
template <bool kFirst, bool kLast, bool kBallot, uint32_t kW>
__global__ void __launch_bounds__(kOsThreads, 2)
k_radix_scatter(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t n,
                uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, uint32_t shift, uint32_t digits,
                const uint32_t* __restrict__ tcount, const uint32_t* __restrict__ csum,
                uint32_t* __restrict__ count, uint32_t vec) {
  extern __shared__ __align__(16) uint32_t sm[];
  uint32_t* in_k = sm;                                                  // [2][kRadixTile]
  uint32_t* in_v = sm + 2 * kRadixTile;                                 // [2][kRadixTile], not with kFirst
  uint32_t* stage_k = sm + (kFirst ? 2 : 4) * kRadixTile;                    // the tile in digit order
  uint32_t* stage_v = stage_k + kRadixTile;
  uint16_t* whist = reinterpret_cast<uint16_t*>(stage_v + kRadixTile);       // [warp][digit]
  uint32_t* lstart = stage_v + kRadixTile + kOsWarps * digits / 2;           // first tile position of each digit
  uint32_t* gstart = lstart + digits;                                        // first output position of each digit
  __shared__ uint32_t s_wsum[kOsWarps];
  const uint32_t tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
  const uint32_t tiles = div_up(n, kRadixTile);
  const uint32_t mask = digits - 1u;
  const uint32_t width = 31u - __clz(digits);
  uint32_t tile = blockIdx.x, buf = 0;
  if (tile < tiles) {
    tile_fetch(in_k, kin, tile, n, vec);
    if (!kFirst) tile_fetch(in_v, vin, tile, n, vec);
  }
  cp_async_commit();
  for (; tile < tiles; tile += gridDim.x, buf ^= 1u) {
    // the next tile's copies go out first; the buffer they fill was last
    // read before the previous iteration's closing barrier
    const uint32_t next = tile + gridDim.x;
    if (next < tiles) {
      tile_fetch(in_k + (buf ^ 1u) * kRadixTile, kin, next, n, vec);
      if (!kFirst) tile_fetch(in_v + (buf ^ 1u) * kRadixTile, vin, next, n, vec);
    }
    cp_async_commit();
    {
      const uint32_t* trow = tcount + (size_t)tile * digits;
      const uint32_t* crow = csum + (size_t)(tile / kScanChunk) * digits;
      for (uint32_t d = tid; d < digits; d += kOsThreads) gstart[d] = __ldg(trow + d) + __ldg(crow + d);
    }
    uint32_t* wrow = reinterpret_cast<uint32_t*>(whist + warp * digits);  // digits is even
    for (uint32_t w = lane; w < digits / 2; w += 32) wrow[w] = 0u;
    cp_async_wait_prev();  // this thread's copies of this tile have landed
    __syncthreads();       // and everyone's
    const uint32_t* ik = in_k + buf * kRadixTile;
    const uint32_t tbase = tile * kRadixTile;
    const uint32_t valid = min(kRadixTile, n - tbase);
    const uint32_t wbase = warp * kOsStripe;
    // rank in element order inside the warp's stripe: a round's equal digits
    // by lane, after the counts of the warp's earlier rounds. The rounds'
    // peer masks depend on nothing in shared memory, so they are all formed
    // first (their latencies overlap); then the rounds run through the warp's
    // histogram in order.
    uint32_t key[kOsItems], pos[kOsItems], peers[kOsItems];
    uint16_t* wh = whist + warp * digits;
    const uint32_t lt = lanemask_lt();
    if (valid == kRadixTile) {  // a whole tile (uniform over the block)
#pragma unroll
      for (uint32_t i = 0; i < kOsItems; ++i) key[i] = ik[wbase + i * 32u + lane];
#pragma unroll
      for (uint32_t i = 0; i < kOsItems; ++i) {
        const uint32_t d = (key[i] >> shift) & mask;
        peers[i] = kBallot ? digit_peers<kW>(d, width, 0xffffffffu) : __match_any_sync(0xffffffffu, d);
      }
#pragma unroll
      for (uint32_t i = 0; i < kOsItems; ++i) {
        const uint32_t d = (key[i] >> shift) & mask;
        const uint32_t old = wh[d];
        pos[i] = old + __popc(peers[i] & lt);
        __syncwarp();
        if (lane == (uint32_t)(__ffs(peers[i]) - 1)) wh[d] = (uint16_t)(old + __popc(peers[i]));
        __syncwarp();
      }
    } else {
#pragma unroll
      for (uint32_t i = 0; i < kOsItems; ++i) {
        const uint32_t l = wbase + i * 32u + lane;
        const bool ok = l < valid;
        key[i] = ok ? ik[l] : 0u;
        const uint32_t vm = __ballot_sync(0xffffffffu, ok);
        pos[i] = 0;
        if (!vm) continue;  // warp-uniform
        const uint32_t d = (key[i] >> shift) & mask;
        uint32_t pm = 0, old = 0;
        if (ok) {
          pm = kBallot ? digit_peers<kW>(d, width, vm) : __match_any_sync(vm, d);
          old = wh[d];
          pos[i] = old + __popc(pm & lt);
        }
        __syncwarp();
        if (ok && lane == (uint32_t)(__ffs(pm) - 1)) wh[d] = (uint16_t)(old + __popc(pm));
        __syncwarp();
      }
    }
    __syncthreads();
    // per digit: the warps' counts -> exclusive offsets over warps; the tile's count
    for (uint32_t d = tid; d < digits; d += kOsThreads) {
      uint32_t sum = 0;
#pragma unroll
      for (uint32_t w = 0; w < kOsWarps; ++w) {
        const uint32_t c = whist[w * digits + d];
        whist[w * digits + d] = (uint16_t)sum;
        sum += c;
      }
      lstart[d] = sum;
    }
    __syncthreads();
    // exclusive scan of the tile's digit counts (a run of digits per thread)
    {
      const uint32_t per = (digits + kOsThreads - 1) / kOsThreads, d0 = tid * per;
      uint32_t run = 0;
      for (uint32_t q = 0; q < per; ++q)
        if (d0 + q < digits) run += lstart[d0 + q];
      uint32_t x = run;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= (uint32_t)off) x += y;
      }
      if (lane == 31) s_wsum[warp] = x;
      __syncthreads();
      uint32_t acc = x - run;
      for (uint32_t w = 0; w < warp; ++w) acc += s_wsum[w];
      for (uint32_t q = 0; q < per; ++q)
        if (d0 + q < digits) {
          const uint32_t c = lstart[d0 + q];
          lstart[d0 + q] = acc;
          acc += c;
        }
    }
    __syncthreads();
    // each digit's output position for tile position 0 of its run
    for (uint32_t d = tid; d < digits; d += kOsThreads) gstart[d] -= lstart[d];
    // tile positions, and the tile staged in digit order (the stage holds
    // nothing else)
    const uint32_t* iv = in_v + buf * kRadixTile;
#pragma unroll
    for (uint32_t i = 0; i < kOsItems; ++i) {
      const uint32_t l = wbase + i * 32u + lane;
      if (l < valid) {
        const uint32_t d = (key[i] >> shift) & mask;
        const uint32_t p = pos[i] + lstart[d] + whist[warp * digits + d];
        stage_k[p] = key[i];
        stage_v[p] = kFirst ? tbase + l : iv[l];
      }
    }
    __syncthreads();
    // out run by run: consecutive threads write consecutive positions of a digit
#pragma unroll 2
    for (uint32_t k0 = 0; k0 < valid; k0 += kOsThreads) {  // uniform over the block
      const uint32_t k = k0 + tid;
      const bool ok = k < valid;
      const uint32_t kk = ok ? stage_k[k] : 0xffffffffu;
      if (ok) {
        const uint32_t dst = gstart[(kk >> shift) & mask] + k;
        if (!kLast) kout[dst] = kk;
        vout[dst] = stage_v[k];
      }
      if (kLast) {
        // one atomic per run of equal keys in the warp's 32 entries
        const uint32_t prev = __shfl_up_sync(0xffffffffu, kk, 1);
        const bool starts = ok && (lane == 0 || kk != prev);
        const uint32_t heads = __ballot_sync(0xffffffffu, starts);
        const uint32_t live = __ballot_sync(0xffffffffu, ok);
        if (starts) {
          const uint32_t later = heads & ~((2u << lane) - 1u);  // heads after this lane (lane 31: none)
          const uint32_t end = later ? (uint32_t)(__ffs(later) - 1) : 32u - __clz(live);
          atomicAdd(count + kk, end - lane);
        }
      }
    }
    __syncthreads();  // the stage, histograms and this tile's buffer are free again
  }
}

// A plan of no passes (one cell): the identity permutation.
__global__ void __launch_bounds__(256) k_identity(uint32_t* __restrict__ perm, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) perm[i] = i;
}

// Cell counts from the sorted keys: one atomic per run of equal keys in a
// warp (a run's first lane in the warp adds the run's length there).
__global__ void __launch_bounds__(256) k_run_counts(const uint32_t* __restrict__ sk, uint32_t n,
                                                    uint32_t* __restrict__ count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = lane_id();
  const bool valid = i < n;
  const uint32_t key = valid ? __ldg(sk + i) : 0xffffffffu;
  const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
  const bool starts = valid && (lane == 0 || key != prev);
  const uint32_t heads = __ballot_sync(0xffffffffu, starts);
  const uint32_t live = __ballot_sync(0xffffffffu, valid);
  if (!starts) return;
  const uint32_t later = heads & ~((2u << lane) - 1u);  // heads after this lane (lane 31: none)
  const uint32_t end = later ? (uint32_t)(__ffs(later) - 1) : 32u - __clz(live);
  atomicAdd(count + key, end - lane);
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

pf_status validate_sort(uint32_t n, const pf_grid_desc* grid, KeyFn* kf, uint64_t* C) {
  if (!grid) return fail(PF_ERR_INVALID, "HashGrid: grid descriptor is NULL");
  if (!make_key_fn(*grid, kf, C)) {
    if (!(grid->cell_size > 0) || !std::isfinite(grid->cell_size))
      return fail(PF_ERR_INVALID, "HashGrid: cellSize must be a positive finite number, got " +
                                      std::to_string(grid->cell_size));
    if (grid->key_kind == PF_KEY_MORTON)
      return fail(PF_ERR_INVALID, "HashGrid: hashTableSize must be a positive power of two, got " +
                                      std::to_string(grid->table_size));
    return fail(PF_ERR_INVALID, "HashGrid: invalid grid descriptor");
  }
  if (n >= (1u << 30)) return fail(PF_ERR_INVALID, "HashGrid: too many particles (at most 2^30 - 1)");
  return PF_OK;
}

pf_status validate_sort_buffers(uint32_t n, const void* pos4, const void* perm, const void* start, const void* count,
                                const void* keys, const void* overflow) {
  if (n > 0 && (!pos4 || !perm)) return fail(PF_ERR_INVALID, "HashGrid: NULL positions or perm");
  if (!start || !count) return fail(PF_ERR_INVALID, "HashGrid: NULL start or count");
  if (reinterpret_cast<uintptr_t>(pos4) & 15u)
    return fail(PF_ERR_INVALID, "HashGrid: positions must be 16-byte aligned (float4 elements)");
  const uintptr_t words = reinterpret_cast<uintptr_t>(perm) | reinterpret_cast<uintptr_t>(start) |
                          reinterpret_cast<uintptr_t>(count) | reinterpret_cast<uintptr_t>(keys) |
                          reinterpret_cast<uintptr_t>(overflow);
  if (words & 3u) return fail(PF_ERR_INVALID, "HashGrid: perm, start, count, keys and overflow must be 4-byte aligned");
  return PF_OK;
}

uint32_t radix_digit_bits() {
  static const uint32_t b = [] {
    const char* e = std::getenv("PFSIM_RADIX_BITS");
    const int v = e ? std::atoi(e) : 8;
    return (uint32_t)std::min(std::max(v, 4), (int)kRadixMaxBits);
  }();
  return b;
}

RadixPlan radix_plan(uint64_t cells) {
  uint32_t bits = 0;
  while (bits < 40 && (1ull << bits) < cells) ++bits;
  const uint32_t dbits = radix_digit_bits();
  RadixPlan p;
  p.passes = (bits + dbits - 1) / dbits;
  p.width = p.passes ? (bits + p.passes - 1) / p.passes : 0;
  p.digits = 1u << p.width;
  return p;
}

uint32_t scan_tiles(uint64_t n) { return (uint32_t)((n + kScanTile - 1) / kScanTile); }

uint32_t keys_grid(uint32_t n, uint32_t threads) {
  return std::max<uint32_t>(1, std::min<uint32_t>(div_up(std::max<uint32_t>(n, 1), threads), (uint32_t)sm_count() * 8));
}

namespace {
size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
uint32_t radix_tiles(uint32_t n) { return std::max<uint32_t>(1, div_up(n, kRadixTile)); }
}  // namespace

size_t sort_scratch_bytes(uint32_t n, uint64_t C) {
  size_t b = 0;
  b += 5 * align256(4ull * n);                                          // keys, ka, va, kb, vb
  b += align256(4ull * kRadixMaxPasses * kRadixMaxDigits);             // digit counts
  b += align256(4ull * radix_tiles(n) * kRadixMaxDigits);                 // tile digit counts
  b += align256(4ull * div_up(radix_tiles(n), kScanChunk) * kRadixMaxDigits);  // chunk bases
  b += align256(8ull * scan_tiles(std::max<uint64_t>(C, 1)));           // scan tile status
  b += align256(4ull * kNumCounters);                                   // counters
  return b;
}

void sort_scratch_carve(void* base, uint32_t n, uint64_t C, SortScratch* s) {
  char* p = static_cast<char*>(base);
  auto take = [&](size_t bytes) {
    char* q = p;
    p += align256(bytes);
    return q;
  };
  s->keys = reinterpret_cast<uint32_t*>(take(4ull * n));
  s->ka = reinterpret_cast<uint32_t*>(take(4ull * n));
  s->va = reinterpret_cast<uint32_t*>(take(4ull * n));
  s->kb = reinterpret_cast<uint32_t*>(take(4ull * n));
  s->vb = reinterpret_cast<uint32_t*>(take(4ull * n));
  s->digit_count = reinterpret_cast<uint32_t*>(take(4ull * kRadixMaxPasses * kRadixMaxDigits));
  s->tiles_cap = radix_tiles(n);
  s->tcount = reinterpret_cast<uint32_t*>(take(4ull * s->tiles_cap * kRadixMaxDigits));
  s->csum = reinterpret_cast<uint32_t*>(take(4ull * div_up(s->tiles_cap, kScanChunk) * kRadixMaxDigits));
  s->scan_tiles_cap = scan_tiles(std::max<uint64_t>(C, 1));
  s->scan_status = reinterpret_cast<uint64_t*>(take(8ull * s->scan_tiles_cap));
  s->counters = reinterpret_cast<uint32_t*>(take(4ull * kNumCounters));
  s->n_cap = n;
  s->c_cap = (uint32_t)C;
}

cudaError_t sort_scratch_zero(const SortScratch& s, cudaStream_t st) {
  // the digit counts, tile counts, chunk bases, scan status and counters
  const char* a = reinterpret_cast<const char*>(s.digit_count);
  const char* b = reinterpret_cast<const char*>(s.counters) + 4ull * kNumCounters;
  return cudaMemsetAsync(const_cast<char*>(a), 0, (size_t)(b - a), st);
}

void launch_keys_digits(const float4* pos, uint32_t n, const KeyFn& kf, const RadixPlan& plan, uint32_t* keys,
                        uint32_t* overflow, const SortScratch& s, cudaStream_t st) {
  if (n == 0) return;
  const DigitHist h = digit_hist(plan, s);
  k_keys_digits<<<keys_grid(n, kHistThreads), kHistThreads, 4ull * plan.passes * plan.digits, st>>>(pos, n, kf, h, keys,
                                                                                                   overflow);
}

cudaError_t launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t* zero_out, uint64_t n,
                                  uint64_t* tile_status, uint32_t* counters, cudaStream_t st) {
  if (n == 0) return cudaSuccess;
  const uint32_t tiles = scan_tiles(n);
  if (cudaError_t e = cudaMemsetAsync(tile_status, 0, 8ull * tiles, st); e != cudaSuccess) return e;
  if (cudaError_t e = cudaMemsetAsync(counters + kCounterTicket, 0, 4, st); e != cudaSuccess) return e;
  const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out) |
                     reinterpret_cast<uintptr_t>(zero_out)) & 15u) == 0;
  k_scan<<<tiles, kScanThreads, 0, st>>>(in, out, zero_out, n, tile_status, counters, vec ? 1u : 0u);
  return cudaGetLastError();
}

namespace {
// Per device: shared memory per SM, for the blocks per SM of the persistent
// scatter (two by its launch bounds when shared memory allows).
int g_smem_per_sm[64];

// Equal digits in a warp round by ballots (default) or by __match_any_sync
// (PFSIM_RADIX_RANK=match); the results are the same.
bool radix_rank_ballot() {
  static const bool b = [] {
    const char* e = std::getenv("PFSIM_RADIX_RANK");
    return !(e && std::string(e) == "match");
  }();
  return b;
}

template <bool kFirst, bool kLast, bool kBallot, uint32_t kW>
cudaError_t launch_scatter_as(const uint32_t* kin, const uint32_t* vin, uint32_t n, uint32_t* kout, uint32_t* vout,
                              uint32_t shift, const RadixPlan& plan, const SortScratch& s, uint32_t* count,
                              cudaStream_t st) {
  int dev = 0;
  if (cudaError_t e = cudaGetDevice(&dev); e != cudaSuccess) return e;
  const size_t smem = scatter_smem_bytes(plan.digits, kFirst);
  const int per_sm = dev < 64 ? g_smem_per_sm[dev] : 0;
  const uint32_t blocks = per_sm > 0 ? (uint32_t)std::min<size_t>(2, std::max<size_t>(1, per_sm / (smem + 1024))) : 1u;
  const uint32_t grid = std::min<uint32_t>(radix_tiles(n), blocks * (uint32_t)sm_count());
  const bool vec = (reinterpret_cast<uintptr_t>(kin) & 15u) == 0 &&
                   (kFirst || (reinterpret_cast<uintptr_t>(vin) & 15u) == 0);
  k_radix_scatter<kFirst, kLast, kBallot, kW><<<grid, kOsThreads, smem, st>>>(
      kin, vin, n, kout, vout, shift, plan.digits, s.tcount, s.csum, count, vec ? 1u : 0u);
  return cudaGetLastError();
}

// The digit widths of the common plans get their own ballot kernels.
#define PF_SCATTER_WIDTHS(X) X(6) X(7) X(8)

template <bool kFirst, bool kLast>
cudaError_t launch_scatter(const uint32_t* kin, const uint32_t* vin, uint32_t n, uint32_t* kout, uint32_t* vout,
                           uint32_t shift, const RadixPlan& plan, const SortScratch& s, uint32_t* count,
                           cudaStream_t st) {
  if (!radix_rank_ballot())
    return launch_scatter_as<kFirst, kLast, false, 0>(kin, vin, n, kout, vout, shift, plan, s, count, st);
  switch (plan.width) {
#define PF_CASE(w) \
  case w:          \
    return launch_scatter_as<kFirst, kLast, true, w>(kin, vin, n, kout, vout, shift, plan, s, count, st);
    PF_SCATTER_WIDTHS(PF_CASE)
#undef PF_CASE
    default:
      return launch_scatter_as<kFirst, kLast, true, 0>(kin, vin, n, kout, vout, shift, plan, s, count, st);
  }
}

template <bool kFirst, bool kLast, bool kBallot, uint32_t kW>
cudaError_t scatter_allow_smem() {
  return cudaFuncSetAttribute(k_radix_scatter<kFirst, kLast, kBallot, kW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)kOsSmemBytes);
}
template <bool kFirst, bool kLast>
cudaError_t scatter_allow_smem_all() {
  for (cudaError_t e : {scatter_allow_smem<kFirst, kLast, false, 0>(), scatter_allow_smem<kFirst, kLast, true, 0>()
#define PF_ALLOW(w) , scatter_allow_smem<kFirst, kLast, true, w>()
                            PF_SCATTER_WIDTHS(PF_ALLOW)
#undef PF_ALLOW
       })
    if (e != cudaSuccess) return e;
  return cudaSuccess;
}
}  // namespace

uint32_t grid_sort_launches(const RadixPlan& plan, uint32_t n) {
  if (n == 0) return 1;                        // the start scan
  if (plan.passes == 0) return 3;              // identity, run counts, start scan
  // digit scan, per pass four (three when the tiles form one chunk), start scan
  const uint32_t per_pass = div_up(radix_tiles(n), kScanChunk) > 1 ? 4u : 3u;
  return 1 + per_pass * plan.passes + 1;
}

cudaError_t launch_grid_sort(const uint32_t* keys, uint32_t n, uint64_t C, const RadixPlan& plan, uint32_t* count,
                             uint32_t* start, uint32_t* perm, const SortScratch& s, cudaStream_t st) {
  if (C == 0) return cudaSuccess;
  if (cudaError_t e = cudaMemsetAsync(count, 0, 4ull * C, st); e != cudaSuccess) return e;
  if (n > 0) {
    const uint32_t tiles = radix_tiles(n);
    if (plan.passes == 0) {
      k_identity<<<div_up(n, 256), 256, 0, st>>>(perm, n);
      k_run_counts<<<div_up(n, 256), 256, 0, st>>>(keys, n, count);
    } else {
      if (cudaError_t e = radix_prepare(); e != cudaSuccess) return e;
      k_digit_first<<<plan.passes, 1024, 0, st>>>(s.digit_count, plan.digits);
      const uint32_t chunks = div_up(tiles, kScanChunk);
      const bool kvec = (reinterpret_cast<uintptr_t>(keys) & 15u) == 0;
      const uint32_t* kin = keys;
      const uint32_t* vin = nullptr;
      for (uint32_t p = 0; p < plan.passes; ++p) {
        const bool first = p == 0, last = p + 1 == plan.passes;
        // pass outputs: even passes -> (ka, va), odd -> (kb, vb); the last
        // writes the permutation and the cell counts, no keys
        uint32_t* kout = last ? nullptr : ((p & 1u) ? s.kb : s.ka);
        uint32_t* vout = last ? perm : ((p & 1u) ? s.vb : s.va);
        const uint32_t shift = p * plan.width;
        k_tile_counts<<<tiles, kCountThreads, 0, st>>>(kin, n, shift, plan.digits, s.tcount,
                                                       (first ? kvec : true) ? 1u : 0u);
        const uint32_t* first_pos = s.digit_count + p * kRadixMaxDigits;
        k_tile_scan_chunk<<<dim3(chunks, div_up(plan.digits, 256)), 256, 0, st>>>(
            s.tcount, tiles, plan.digits, s.csum, chunks == 1 ? first_pos : nullptr);
        if (chunks > 1)
          k_tile_scan_chunks<<<div_up(plan.digits, 8), 256, 0, st>>>(s.csum, chunks, plan.digits, first_pos);
        cudaError_t e;
        if (first && last)
          e = launch_scatter<true, true>(kin, vin, n, kout, vout, shift, plan, s, count, st);
        else if (first)
          e = launch_scatter<true, false>(kin, vin, n, kout, vout, shift, plan, s, count, st);
        else if (last)
          e = launch_scatter<false, true>(kin, vin, n, kout, vout, shift, plan, s, count, st);
        else
          e = launch_scatter<false, false>(kin, vin, n, kout, vout, shift, plan, s, count, st);
        if (e != cudaSuccess) return e;
        kin = kout;
        vin = vout;
      }
    }
  }
  if (cudaError_t e = cudaGetLastError(); e != cudaSuccess) return e;
  return launch_exclusive_scan(count, start, nullptr, C, s.scan_status, s.counters, st);
}

cudaError_t radix_prepare() {
  static std::mutex m;
  static std::set<int> ready;
  int dev = 0;
  if (cudaError_t e = cudaGetDevice(&dev); e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(m);
  if (ready.count(dev)) return cudaSuccess;
  for (cudaError_t e : {scatter_allow_smem_all<true, true>(), scatter_allow_smem_all<true, false>(),
                        scatter_allow_smem_all<false, true>(), scatter_allow_smem_all<false, false>()})
    if (e != cudaSuccess) return e;
  int per_sm = 0;
  if (cudaError_t e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
      e != cudaSuccess)
    return e;
  if (dev < 64) g_smem_per_sm[dev] = per_sm;
  (void)sm_count();  // cached outside any stream capture
  ready.insert(dev);
  return cudaSuccess;
}

cudaError_t sort_run(const float4* pos, uint32_t n, const KeyFn& kf, uint64_t C, uint32_t* perm, uint32_t* start,
                     uint32_t* count, uint32_t* keys, uint32_t* overflow, const SortScratch& s, cudaStream_t st) {
  const RadixPlan plan = radix_plan(C);
  if (cudaError_t e = cudaMemsetAsync(s.counters, 0, 4ull * kNumCounters, st); e != cudaSuccess) return e;
  if (cudaError_t e = cudaMemsetAsync(s.digit_count, 0, 4ull * kRadixMaxPasses * kRadixMaxDigits, st);
      e != cudaSuccess)
    return e;
  uint32_t* ovf = overflow ? overflow : s.counters + kCounterOverflow;
  if (overflow)
    if (cudaError_t e = cudaMemsetAsync(overflow, 0, 4, st); e != cudaSuccess) return e;
  launch_keys_digits(pos, n, kf, plan, keys, ovf, s, st);
  return launch_grid_sort(keys, n, C, plan, count, start, perm, s, st);
}

}  // namespace pf
