// grid_sort.cuh — stable counting sort of particle indices by cell key.
//
// Pipeline (one call of SortPlan::run):
//   clear      counts[C] = 0, fill state reset
//   key+hist   key of every element, warp-aggregated histogram (one atomic
//              per distinct key per warp), overflow flag
//   scan       decoupled look-back exclusive scan counts -> start, fill = 0
//   scatter    warp-stable atomic scatter into each cell's run; a cell that
//              receives groups from more than one warp is queued for fix-up
//   fix-up     each queued cell's run is sorted ascending (thread, CTA and
//              chunked-radix tiers by run length)
// The result equals a stable counting sort of elements 0..n-1: within a cell,
// elements appear in ascending element index.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace pf {

// Device view of a key function (pf_grid_desc resolved on the host).
struct KeyFn {
  uint32_t kind;        // PF_KEY_LINEAR / PF_KEY_MORTON
  float ox, oy, oz;     // origin
  float cell;           // cell size
  int32_t lo[3];        // linear: lowest cell coordinate per axis (usually 0)
  uint32_t dims[3];     // linear: cells per axis
  uint32_t mask;        // morton: table_size - 1
};

bool make_key_fn(const pf_grid_desc& g, KeyFn* out, uint64_t* cells);

// Scratch of one sort, sized for n elements and C cells.
struct SortScratch {
  uint32_t* keys = nullptr;      // n
  uint32_t* fill = nullptr;      // C   running fill per cell
  uint32_t* dirty_bits = nullptr;  // ceil(C/32)
  uint32_t* lists = nullptr;     // 3 * list_cap dirty cells by tier
  uint64_t* tile_status = nullptr;  // scan tiles
  uint32_t* counters = nullptr;  // [0] scan tile ticket, [1..3] tier list lengths, [4] error word, [5] overflow
  uint32_t* radix_tmp = nullptr;   // n, giant-cell ping-pong buffer
  uint32_t n_cap = 0, c_cap = 0, list_cap = 0, tiles_cap = 0;
};

constexpr int kCounterTicket = 0;
constexpr int kCounterSmall = 1;
constexpr int kCounterMid = 2;
constexpr int kCounterGiant = 3;
constexpr int kCounterError = 4;
constexpr int kCounterOverflow = 5;
constexpr int kNumCounters = 8;

// Bytes of scratch for n elements and C cells.
size_t sort_scratch_bytes(uint32_t n, uint64_t C);
// Carve a scratch layout out of one device allocation of sort_scratch_bytes.
void sort_scratch_carve(void* base, uint32_t n, uint64_t C, SortScratch* s);

// Keys from float4 positions by element index, fused with the histogram.
void launch_keys_hist(const float4* pos, uint32_t n, const KeyFn& kf, uint32_t* keys,
                      uint32_t* counts, uint32_t* overflow, cudaStream_t st);

// The sort proper from precomputed keys (keys[e] < C for every element).
// Writes perm[n], start[C]; counts[C] must already hold the histogram.
void launch_sort_from_hist(const uint32_t* keys, uint32_t n, uint64_t C, const uint32_t* counts,
                           uint32_t* start, uint32_t* perm, const SortScratch& s, cudaStream_t st);

// Exclusive scan of n uint32 values (decoupled look-back); also zeroes
// `zero_out` (n entries) when it is not null.
void launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t* zero_out, uint64_t n,
                           uint64_t* tile_status, uint32_t* counters, cudaStream_t st);
uint32_t scan_tiles(uint64_t n);

}  // namespace pf
