// sort_noalloc.cu — pf_sort_noalloc: the stable grid sort without any
// device allocation.
//
// Who needs this: callers that must not allocate GPU memory while they run.
// Examples are a host that has handed all of the device's memory to its own
// pool allocator and treats any cudaMalloc behind its back as a leak, and
// real-time loops where an allocation (which can synchronise the device) is
// not allowed once the frame loop has started. pf_sort takes its scratch from
// a workspace that it grows with cudaMalloc; this entry point instead uses one
// fixed block of device memory that is part of the library image.
//
// The scratch block below is a file-scope __device__ array of
// kNoAllocScratchBytes (23 MiB). Its size caps the problem: at most
// kNoAllocMaxParticles particles and kNoAllocMaxCells cells per call. The
// CUDA runtime loads this file's device code lazily (CUDA 12 defaults to
// lazy module loading), so the block is reserved on a device by the first
// call there, when the address lookup below loads the module, and it stays
// reserved until the process exits. A caller whose own pool takes the
// device's memory should therefore make one call per device before the pool
// claims it; a call with n = 0 and no start/count buffers does only this
// set-up. The lookup is also why that first call must come before any stream
// capture begins.
//
// In host code the name g_noalloc_scratch is only a stand-in for the device
// symbol, not a device address: passing it to a kernel would fault, or on a
// system where the GPU can reach host memory, silently use the wrong memory.
// The real address comes from cudaGetSymbolAddress, once per device, with
// that device current.
//
// All calls share the one block and it keeps the last call's contents: each
// call clears what must start at zero itself, and two calls whose GPU work
// overlaps (for example on two streams) race on the block and corrupt each
// other's results. Serialise them.
//
// Errors found on the device (a bounded look-back wait that expired) go to
// the block's error word; pf_sort_device_errors on the call's stream reads
// and clears it, as it does for pf_sort.

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "common.cuh"
#include "grid_sort.cuh"

namespace pf {
namespace {

constexpr uint32_t kNoAllocMaxParticles = 1u << 20;  // 1,048,576
constexpr uint64_t kNoAllocMaxCells = 1ull << 21;    // 2,097,152 (a 128^3 grid)
constexpr size_t kNoAllocScratchBytes = 23ull << 20; // >= sort_scratch_bytes(max particles, max cells)

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch block on the current device (set-up on the
// first call per device).
pf_status noalloc_scratch(void** out) {
  int dev = 0;
  PF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(PF_ERR_INVALID, "HashGrid: device index out of range");
  std::lock_guard<std::mutex> g(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(PF_ERR_CUDA, std::string("HashGrid: cudaGetSymbolAddress of the fixed sort scratch failed: ") +
                                   cudaGetErrorString(e));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return PF_OK;
}

}  // namespace
}  // namespace pf

using namespace pf;

extern "C" pf_status pf_sort_noalloc(const float* d_pos4, uint32_t n, const pf_grid_desc* grid,
                                     uint32_t* d_perm, uint32_t* d_start, uint32_t* d_count,
                                     uint32_t* d_keys, uint32_t* d_overflow, void* stream) {
  KeyFn kf;
  uint64_t C = 0;
  PF_TRY(validate_sort(n, grid, &kf, &C));
  if (n > kNoAllocMaxParticles)
    return fail(PF_ERR_INVALID, "HashGrid: pf_sort_noalloc takes at most " + std::to_string(kNoAllocMaxParticles) +
                                    " particles, got " + std::to_string(n) + " (use pf_sort)");
  if (C > kNoAllocMaxCells)
    return fail(PF_ERR_INVALID, "HashGrid: pf_sort_noalloc takes at most " + std::to_string(kNoAllocMaxCells) +
                                    " cells, got " + std::to_string(C) + " (use pf_sort)");
  if (sort_scratch_bytes(kNoAllocMaxParticles, kNoAllocMaxCells) > kNoAllocScratchBytes)
    return fail(PF_ERR_INVALID, "HashGrid: pf_sort_noalloc scratch block is smaller than its limits need");
  void* base = nullptr;
  // set-up only: the block's address on this device (see the file comment)
  if (n == 0 && !d_start && !d_count) return noalloc_scratch(&base);
  PF_TRY(validate_sort_buffers(n, d_pos4, d_perm, d_start, d_count, d_keys, d_overflow));

  PF_TRY(noalloc_scratch(&base));
  // carved for the block's limits, whatever this call's size
  SortScratch s;
  sort_scratch_carve(base, kNoAllocMaxParticles, kNoAllocMaxCells, &s);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  PF_CUDA(sort_run(reinterpret_cast<const float4*>(d_pos4), n, kf, C, d_perm, d_start, d_count,
                   d_keys ? d_keys : s.keys, d_overflow, s, st));
  sort_note_counters(st, s.counters);
  return PF_OK;
}
