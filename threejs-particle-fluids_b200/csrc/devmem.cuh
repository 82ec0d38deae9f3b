// devmem.cuh — device memory of worlds (arena, grid cell arrays, sort
// scratch) from a stream-ordered pool per device that keeps freed memory
// for the next world; devmem.cu says why.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace pf {

// Allocate `bytes` in stream order on `st` (256-byte aligned). The memory
// is usable on other streams once `st` has reached this point (a
// synchronize of `st`, or an event recorded after it).
cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t st);
// Free in stream order on `st`: every stream that used `p` must have been
// ordered before this point of `st` (synchronized, or joined by an event).
void dev_free(void* p, cudaStream_t st);
// Wait for the device, then hand the pool's unused memory back.
cudaError_t dev_trim();

}  // namespace pf
