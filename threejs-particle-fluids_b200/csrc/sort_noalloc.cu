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
// The scratch block below is a file-scope __device__ array, so every GPU that
// loads libpfsim.so holds it (kNoAllocScratchBytes, about 21 MB) until the
// process exits. Its size caps the problem: at most kNoAllocMaxParticles
// particles and kNoAllocMaxCells cells per call.
//
// In host code the name g_noalloc_scratch is only a stand-in for the device
// symbol, not a device address: passing it to a kernel would fault, or on a
// system where the GPU can reach host memory, silently use the wrong memory.
// The real address comes from cudaGetSymbolAddress, once per device, with
// that device current; the first pf_sort_noalloc call on a device does this
// set-up, so make that first call before any stream capture begins.
//
// All calls share the one block and it keeps the last call's contents: each
// call clears what must start at zero itself, and two calls whose GPU work
// overlaps (for example on two streams) race on the block and corrupt each
// other's results. Serialise them.

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "common.cuh"
#include "grid_sort.cuh"

namespace pf {
namespace {

constexpr uint32_t kNoAllocMaxParticles = 1u << 20;  // 1,048,576
constexpr uint64_t kNoAllocMaxCells = 1ull << 21;    // 2,097,152 (a 128^3 grid)
constexpr size_t kNoAllocScratchBytes = 21ull << 20; // >= sort_scratch_bytes(max particles, max cells)

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
  if (!grid) return fail(PF_ERR_INVALID, "HashGrid: grid descriptor is NULL");
  KeyFn kf;
  uint64_t C = 0;
  if (!make_key_fn(*grid, &kf, &C)) return fail(PF_ERR_INVALID, "HashGrid: invalid grid descriptor");
  if (n > kNoAllocMaxParticles)
    return fail(PF_ERR_INVALID, "HashGrid: pf_sort_noalloc takes at most " + std::to_string(kNoAllocMaxParticles) +
                                    " particles, got " + std::to_string(n) + " (use pf_sort)");
  if (C > kNoAllocMaxCells)
    return fail(PF_ERR_INVALID, "HashGrid: pf_sort_noalloc takes at most " + std::to_string(kNoAllocMaxCells) +
                                    " cells, got " + std::to_string(C) + " (use pf_sort)");
  if (sort_scratch_bytes(n, C) > kNoAllocScratchBytes)
    return fail(PF_ERR_INVALID, "HashGrid: pf_sort_noalloc scratch too small for this size (use pf_sort)");
  if (n > 0 && (!d_pos4 || !d_perm)) return fail(PF_ERR_INVALID, "HashGrid: NULL positions or perm");
  if (!d_start || !d_count) return fail(PF_ERR_INVALID, "HashGrid: NULL start or count");

  void* base = nullptr;
  PF_TRY(noalloc_scratch(&base));
  SortScratch s;
  sort_scratch_carve(base, n, C, &s);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // What must start at zero: the histogram, the counters and the flag.
  PF_CUDA(cudaMemsetAsync(d_count, 0, 4ull * C, st));
  PF_CUDA(cudaMemsetAsync(s.counters, 0, 4ull * kNumCounters, st));
  uint32_t* ovf = d_overflow ? d_overflow : s.counters + kCounterOverflow;
  if (d_overflow) PF_CUDA(cudaMemsetAsync(d_overflow, 0, 4, st));
  launch_keys_hist(reinterpret_cast<const float4*>(d_pos4), n, kf, d_keys ? d_keys : s.keys, d_count, ovf, st);
  launch_sort_from_hist(d_keys ? d_keys : s.keys, n, C, d_count, d_start, d_perm, s, st);
  PF_CUDA(cudaGetLastError());
  return PF_OK;
}
