// common.cuh — shared helpers of libpfsim: status/error plumbing, device
// error words, launch-shape constants and small vector math.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdlib>
#include <string>

#include "pfsim.h"

namespace pf {

// Thread-local error text behind pf_last_error().
void set_error(const std::string& msg);
const std::string& get_error();

// PFSIM_VERBOSE set: host-side events (grid window growth, graph captures,
// the phases of a serving tick) and their times go to stderr.
inline bool verbose() {
  static const bool v = std::getenv("PFSIM_VERBOSE") != nullptr;
  return v;
}

// Returns a pf_status and records msg.
inline pf_status fail(pf_status s, const std::string& msg) {
  set_error(msg);
  return s;
}

// CUDA call check inside functions returning pf_status.
#define PF_CUDA(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return ::pf::fail(PF_ERR_CUDA, std::string("CUDA: ") + #call + ": " +                \
                                         cudaGetErrorString(e_));                          \
  } while (0)

#define PF_TRY(expr)                \
  do {                              \
    pf_status s_ = (expr);          \
    if (s_ != PF_OK) return s_;     \
  } while (0)

// Number of SMs on the current device (148 on B200), cached per device.
int sm_count();

// Device-side error word bits, written by kernels that give up a bounded
// wait or find an inconsistent input; read back by the host after a call.
enum DeviceError : uint32_t {
  DEV_ERR_LOOKBACK_TIMEOUT = 1u << 0,
};

// Upper bound on spins of a decoupled look-back before it reports
// DEV_ERR_LOOKBACK_TIMEOUT and returns (forward progress is guaranteed by
// tile ids taken in launch order, so this only triggers on a bug).
constexpr uint32_t kLookbackSpinLimit = 1u << 24;

__host__ __device__ inline uint32_t div_up(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

}  // namespace pf
