// devmem.cu — device memory of worlds: one stream-ordered pool per device.
//
// A world's arena, its grid cell arrays and its sort scratch come from a
// pool (cudaMallocFromPoolAsync on the world's stream) whose release
// threshold is unbounded: what a destroyed world or a re-laid-out grid
// frees (cudaFreeAsync) stays mapped in the pool, and the next world or grid
// of the process takes it from there. Freeing then neither waits for the
// whole device (cudaFree does) nor unmaps pages, and building maps none
// after the first time: in a serving loop that builds and frees cohorts of
// tens of GB every few ticks, those were ticks of hundreds of milliseconds.
// pf_trim_device_memory hands the unused part back to the device; an
// allocation that finds no room trims and tries once more. Devices without
// memory pools use cudaMalloc and cudaFree.

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>

#include "common.cuh"
#include "devmem.cuh"

namespace pf {

namespace {

std::mutex g_pool_mutex;
std::map<int, cudaMemPool_t> g_pools;  // device -> pool (nullptr: no pool support)

cudaMemPool_t pool_for_current_device() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> g(g_pool_mutex);
  auto it = g_pools.find(dev);
  if (it != g_pools.end()) return it->second;
  cudaMemPool_t pool = nullptr;
  int supported = 0;
  if (cudaDeviceGetAttribute(&supported, cudaDevAttrMemoryPoolsSupported, dev) == cudaSuccess && supported) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if (cudaMemPoolCreate(&pool, &props) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess) {
        cudaMemPoolDestroy(pool);
        pool = nullptr;
      }
    } else {
      pool = nullptr;
    }
  }
  cudaGetLastError();  // an unsupported attribute leaves no sticky error
  g_pools[dev] = pool;
  return pool;
}

}  // namespace

cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t st) {
  *p = nullptr;
  cudaMemPool_t pool = pool_for_current_device();
  if (!pool) return cudaMalloc(p, bytes);
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes, pool, st);
  if (e == cudaErrorMemoryAllocation) {
    // memory other worlds freed is still held by the pool: hand it back
    // (after the frees in flight on this stream) and try once more
    cudaGetLastError();
    cudaStreamSynchronize(st);
    cudaMemPoolTrimTo(pool, 0);
    e = cudaMallocFromPoolAsync(p, bytes, pool, st);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return e;
  }
  // the carvers place buffers at 256-byte offsets from the base
  if (reinterpret_cast<uintptr_t>(*p) & 255u) {
    cudaFreeAsync(*p, st);
    *p = nullptr;
    return cudaErrorMisalignedAddress;
  }
  return cudaSuccess;
}

void dev_free(void* p, cudaStream_t st) {
  if (!p) return;
  if (!pool_for_current_device()) {
    cudaFree(p);
    return;
  }
  cudaFreeAsync(p, st);
}

cudaError_t dev_trim() {
  cudaMemPool_t pool = pool_for_current_device();
  if (!pool) return cudaSuccess;
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return e;
  return cudaMemPoolTrimTo(pool, 0);
}

}  // namespace pf

extern "C" {

PF_API pf_status pf_trim_device_memory(void) {
  if (const cudaError_t e = pf::dev_trim(); e != cudaSuccess)
    return pf::fail(PF_ERR_CUDA, std::string("pf_trim_device_memory: ") + cudaGetErrorString(e));
  return PF_OK;
}

}  // extern "C"
