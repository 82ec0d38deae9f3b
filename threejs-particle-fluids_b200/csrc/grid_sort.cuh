// grid_sort.cuh — stable counting sort of particle indices by cell key.
//
// Pipeline (launch_grid_sort after the keys and their digit counts exist):
//   keys+digits  key of every element (or the caller's keys), and the count
//                of every radix digit of every pass, from shared-memory
//                histograms flushed once per block
//   digit scan   the counts of each pass turned into each digit's first
//                output position
//   passes       one LSD radix pass per 8 (or fewer; PFSIM_RADIX_BITS) key
//                bits, each three steps: every tile of 4096 elements counts
//                its digits; the tile counts are scanned per digit over the
//                tiles; a persistent scatter ranks each tile's elements by
//                digit in element order (warp-aggregated with
//                __match_any_sync), copying the next tile into shared memory
//                meanwhile, and writes them out digit run by digit run
//   runs         the last pass writes no keys: it counts every cell from its
//                staged tiles, which are in key order (one atomic per run of
//                equal keys in a warp)
//   scan         decoupled look-back exclusive scan counts -> start
// LSD passes are stable, so the result equals a stable counting sort of the
// elements 0..n-1: within a cell, elements appear in ascending index.
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

// Checks a sort request as HashGrid's constructor and rebuild do and
// resolves its key function; the reference's error text on failure.
pf_status validate_sort(uint32_t n, const pf_grid_desc* grid, KeyFn* kf, uint64_t* cells);
// Checks the device buffers of a standalone sort: positions and perm present
// unless n is 0, start and count present, positions 16-byte aligned (they are
// read as float4), the other buffers (keys and overflow may be NULL) 4-byte
// aligned. Other alignments are handled inside the sort.
pf_status validate_sort_buffers(uint32_t n, const void* pos4, const void* perm, const void* start, const void* count,
                                const void* keys, const void* overflow);

// Radix plan for keys in [0, C): `passes` LSD passes of `width` bits, at
// most radix_digit_bits() bits each (8 unless PFSIM_RADIX_BITS sets 4 to 11).
constexpr uint32_t kRadixMaxBits = 11;
constexpr uint32_t kRadixMaxDigits = 1u << kRadixMaxBits;  // 2048
constexpr uint32_t kRadixMaxPasses = 4;                     // 32 bits of 8 >= any key below 2^31
constexpr uint32_t kRadixTile = 4096;                       // elements per tile of a radix pass
uint32_t radix_digit_bits();
struct RadixPlan {
  uint32_t passes = 0, width = 0, digits = 1;
};
RadixPlan radix_plan(uint64_t cells);

// Scratch of one sort, carved for a capacity of n_cap elements and c_cap
// cells.
struct SortScratch {
  uint32_t* keys = nullptr;      // n_cap: keys by element when the caller keeps none
  uint32_t* ka = nullptr;        // n_cap: keys after pass 0
  uint32_t* va = nullptr;        // n_cap: element indices after pass 0
  uint32_t* kb = nullptr;        // n_cap: keys after odd passes, or the sorted keys
  uint32_t* vb = nullptr;        // n_cap
  uint32_t* digit_count = nullptr;  // kRadixMaxPasses x kRadixMaxDigits: counts, then first positions
  uint32_t* tcount = nullptr;    // tiles_cap x kRadixMaxDigits: digit counts per tile, then their scan
  uint32_t* csum = nullptr;      // tiles_cap / 32 x kRadixMaxDigits: per chunk of 32 tiles, its first positions
  uint64_t* scan_status = nullptr;  // look-back tiles of the count -> start scan
  uint32_t* counters = nullptr;  // kNumCounters words
  uint32_t n_cap = 0, c_cap = 0, tiles_cap = 0, scan_tiles_cap = 0;
};

constexpr int kCounterTicket = 0;  // scan tile ticket
constexpr int kCounterError = 4;
constexpr int kCounterOverflow = 5;
constexpr int kNumCounters = 8;

// Bytes of scratch for a capacity of n elements and C cells.
size_t sort_scratch_bytes(uint32_t n, uint64_t C);
// Carve a scratch layout out of one device allocation of sort_scratch_bytes.
// sort_scratch_zero clears its counters and counts (a fresh block once).
void sort_scratch_carve(void* base, uint32_t n, uint64_t C, SortScratch* s);
cudaError_t sort_scratch_zero(const SortScratch& s, cudaStream_t st);

// Keys from float4 positions by element index, with the radix digit counts
// of `plan` (s.digit_count must be zero) and the overflow flag.
void launch_keys_digits(const float4* pos, uint32_t n, const KeyFn& kf, const RadixPlan& plan, uint32_t* keys,
                        uint32_t* overflow, const SortScratch& s, cudaStream_t st);

// The sort proper from keys by element (keys[e] < C) whose digit counts are
// in s.digit_count: writes perm[n], count[C] and start[C]. Clears what it
// needs itself except s.digit_count (zeroed before the digit counts) and the
// caller's error word.
cudaError_t launch_grid_sort(const uint32_t* keys, uint32_t n, uint64_t C, const RadixPlan& plan,
                             uint32_t* count, uint32_t* start, uint32_t* perm, const SortScratch& s,
                             cudaStream_t st);

// Kernel launches of launch_grid_sort for a plan and element count.
uint32_t grid_sort_launches(const RadixPlan& plan, uint32_t n);

// Per device, once: the radix passes' shared-memory size above the default
// limit. Call it outside stream capture before the first sort on a device
// (the sort calls it itself; a world calls it when it is built).
cudaError_t radix_prepare();

// The whole standalone sort on device buffers: clears the counts and
// counters it needs, computes keys (into `keys`) and the overflow flag, and
// sorts. `overflow` may be null (the flag then goes to a scratch counter).
cudaError_t sort_run(const float4* pos, uint32_t n, const KeyFn& kf, uint64_t C, uint32_t* perm, uint32_t* start,
                     uint32_t* count, uint32_t* keys, uint32_t* overflow, const SortScratch& s, cudaStream_t st);

// Records `counters` as the counter block of the latest standalone sort on
// (current device, st): pf_sort_device_errors reads its error word.
void sort_note_counters(cudaStream_t st, uint32_t* counters);

// Shared-memory digit histogram of a block, flushed into s.digit_count.
// Used by the key kernels (standalone sort and the solver's k_keys).
struct DigitHist {
  uint32_t passes, width, digits;
  uint32_t* global;  // kRadixMaxPasses x kRadixMaxDigits
};
__device__ __forceinline__ void digit_hist_add(uint32_t* sh, const DigitHist& h, uint32_t key) {
  for (uint32_t p = 0; p < h.passes; ++p) atomicAdd(sh + p * h.digits + ((key >> (p * h.width)) & (h.digits - 1u)), 1u);
}
__device__ __forceinline__ void digit_hist_zero(uint32_t* sh, const DigitHist& h) {
  for (uint32_t b = threadIdx.x; b < h.passes * h.digits; b += blockDim.x) sh[b] = 0;
}
__device__ __forceinline__ void digit_hist_flush(const uint32_t* sh, const DigitHist& h) {
  for (uint32_t b = threadIdx.x; b < h.passes * h.digits; b += blockDim.x) {
    const uint32_t v = sh[b];
    if (v) atomicAdd(h.global + (b / h.digits) * kRadixMaxDigits + b % h.digits, v);
  }
}
inline DigitHist digit_hist(const RadixPlan& p, const SortScratch& s) {
  return DigitHist{p.passes, p.width, p.digits, s.digit_count};
}
// Blocks of a grid-stride key kernel: enough to fill the GPU, few enough
// that each block's histogram flush is cheap.
uint32_t keys_grid(uint32_t n, uint32_t threads);

// Exclusive scan of n uint32 values (decoupled look-back); also zeroes
// `zero_out` (n entries) when it is not null.
cudaError_t launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t* zero_out, uint64_t n,
                                  uint64_t* tile_status, uint32_t* counters, cudaStream_t st);
uint32_t scan_tiles(uint64_t n);

}  // namespace pf
