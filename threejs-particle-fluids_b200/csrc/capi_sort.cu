// capi_sort.cu — C ABI of the standalone neighbour-grid sort and the
// library-wide error plumbing (pf_last_error, pf_abi_version).

#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <utility>

#include "common.cuh"
#include "grid_sort.cuh"

namespace pf {

namespace {
thread_local std::string t_error;
}

void set_error(const std::string& msg) { t_error = msg; }
const std::string& get_error() { return t_error; }

int sm_count() {
  static std::mutex m;
  static std::map<int, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> g(m);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  cache[dev] = n;
  return n;
}

namespace {

// Scratch of the standalone sort, one per (device, stream): calls on one
// stream run in order and reuse it; calls on different streams get their own.
struct Workspace {
  void* scratch = nullptr;
  uint32_t n_cap = 0;
  uint64_t c_cap = 0;
  SortScratch s{};
  // staging for pf_sort_host
  void* io = nullptr;
  size_t io_bytes = 0;
  // counters of the most recent sort on this stream: pf_sort's own, or the
  // fixed block's after a pf_sort_noalloc; pf_sort_device_errors reads its
  // error word
  uint32_t* counters = nullptr;
};

std::mutex g_ws_mutex;
std::map<std::pair<int, cudaStream_t>, Workspace> g_ws;

pf_status ensure_io(void** ptr, size_t* have, size_t need) {
  if (*have >= need && *ptr) return PF_OK;
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  *have = 0;
  const size_t grow = need + need / 4;
  if (cudaMalloc(ptr, grow) != cudaSuccess) {
    cudaGetLastError();
    return fail(PF_ERR_OOM, "HashGrid: out of device memory for sort staging");
  }
  *have = grow;
  return PF_OK;
}

// Grows the workspace's sort scratch to hold n elements and C cells. The
// layout follows the capacity, not the call, and a new block starts zeroed.
pf_status ensure_scratch(Workspace& ws, uint32_t n, uint64_t C, cudaStream_t st) {
  if (ws.scratch && ws.n_cap >= n && ws.c_cap >= C) return PF_OK;
  if (ws.scratch) {
    PF_CUDA(cudaStreamSynchronize(st));
    cudaFree(ws.scratch);
  }
  ws.scratch = nullptr;
  ws.counters = nullptr;
  const uint32_t n_cap =
      (uint32_t)std::min<uint64_t>(std::max<uint64_t>(ws.n_cap, (uint64_t)n + n / 4), (1u << 30) - 1);
  const uint64_t c_cap = std::max<uint64_t>(ws.c_cap, C + C / 4);
  if (cudaMalloc(&ws.scratch, sort_scratch_bytes(n_cap, c_cap)) != cudaSuccess) {
    cudaGetLastError();
    ws.scratch = nullptr;
    ws.n_cap = 0;
    ws.c_cap = 0;
    return fail(PF_ERR_OOM, "HashGrid: out of device memory for sort scratch");
  }
  ws.n_cap = n_cap;
  ws.c_cap = c_cap;
  sort_scratch_carve(ws.scratch, n_cap, c_cap, &ws.s);
  PF_CUDA(sort_scratch_zero(ws.s, st));
  return PF_OK;
}

Workspace& workspace_for(cudaStream_t st) {
  int dev = 0;
  cudaGetDevice(&dev);
  return g_ws[{dev, st}];
}

}  // namespace

void sort_note_counters(cudaStream_t st, uint32_t* counters) {
  std::lock_guard<std::mutex> g(g_ws_mutex);
  workspace_for(st).counters = counters;
}

}  // namespace pf

using namespace pf;

extern "C" {

const char* pf_last_error(void) { return get_error().c_str(); }
int pf_abi_version(void) { return PFSIM_ABI_VERSION; }

uint64_t pf_grid_cells(const pf_grid_desc* grid) {
  KeyFn kf;
  uint64_t C = 0;
  if (!grid || !make_key_fn(*grid, &kf, &C)) return 0;
  return C;
}

pf_status pf_sort(const float* d_pos4, uint32_t n, const pf_grid_desc* grid, uint32_t* d_perm,
                  uint32_t* d_start, uint32_t* d_count, uint32_t* d_keys, uint32_t* d_overflow,
                  void* stream) {
  KeyFn kf;
  uint64_t C = 0;
  PF_TRY(validate_sort(n, grid, &kf, &C));
  PF_TRY(validate_sort_buffers(n, d_pos4, d_perm, d_start, d_count, d_keys, d_overflow));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> g(g_ws_mutex);
  Workspace& ws = workspace_for(st);
  PF_TRY(ensure_scratch(ws, n, C, st));
  ws.counters = ws.s.counters;
  PF_CUDA(sort_run(reinterpret_cast<const float4*>(d_pos4), n, kf, C, d_perm, d_start, d_count,
                   d_keys ? d_keys : ws.s.keys, d_overflow, ws.s, st));
  return PF_OK;
}

// Synchronises `stream` and returns (and clears) the device error word of the
// most recent standalone sort on that stream: pf_sort's workspace, or the
// fixed block of pf_sort_noalloc when that ran last.
pf_status pf_sort_device_errors(void* stream, uint32_t* bits) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> g(g_ws_mutex);
  Workspace& ws = workspace_for(st);
  uint32_t e = 0;
  PF_CUDA(cudaStreamSynchronize(st));
  if (ws.counters) {
    PF_CUDA(cudaMemcpy(&e, ws.counters + kCounterError, 4, cudaMemcpyDeviceToHost));
    PF_CUDA(cudaMemset(ws.counters + kCounterError, 0, 4));
  }
  if (bits) *bits = e;
  return PF_OK;
}

pf_status pf_sort_host(const float* h_pos4, uint32_t n, const pf_grid_desc* grid, uint32_t* h_perm,
                       uint32_t* h_start, uint32_t* h_count, uint32_t* h_keys, uint32_t* h_overflow) {
  KeyFn kf;
  uint64_t C = 0;
  PF_TRY(validate_sort(n, grid, &kf, &C));
  if (n > 0 && !h_pos4) return fail(PF_ERR_INVALID, "HashGrid: NULL positions");
  cudaStream_t st = nullptr;
  std::lock_guard<std::mutex> g(g_ws_mutex);
  Workspace& ws = workspace_for(st);
  auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t io = al(16ull * n) + al(4ull * n) + al(4ull * C) + al(4ull * C) + al(4ull * n) + al(4);
  PF_TRY(ensure_io(&ws.io, &ws.io_bytes, io));
  PF_TRY(ensure_scratch(ws, n, C, st));
  ws.counters = ws.s.counters;
  char* p = static_cast<char*>(ws.io);
  float4* d_pos = reinterpret_cast<float4*>(p);
  p += al(16ull * n);
  uint32_t* d_perm = reinterpret_cast<uint32_t*>(p);
  p += al(4ull * n);
  uint32_t* d_start = reinterpret_cast<uint32_t*>(p);
  p += al(4ull * C);
  uint32_t* d_count = reinterpret_cast<uint32_t*>(p);
  p += al(4ull * C);
  uint32_t* d_keys = reinterpret_cast<uint32_t*>(p);
  p += al(4ull * n);
  uint32_t* d_ovf = reinterpret_cast<uint32_t*>(p);
  const SortScratch& s = ws.s;
  if (n) PF_CUDA(cudaMemcpyAsync(d_pos, h_pos4, 16ull * n, cudaMemcpyHostToDevice, st));
  PF_CUDA(sort_run(d_pos, n, kf, C, d_perm, d_start, d_count, d_keys, d_ovf, s, st));
  uint32_t err = 0;
  PF_CUDA(cudaMemcpyAsync(&err, s.counters + kCounterError, 4, cudaMemcpyDeviceToHost, st));
  if (h_perm && n) PF_CUDA(cudaMemcpyAsync(h_perm, d_perm, 4ull * n, cudaMemcpyDeviceToHost, st));
  if (h_start) PF_CUDA(cudaMemcpyAsync(h_start, d_start, 4ull * C, cudaMemcpyDeviceToHost, st));
  if (h_count) PF_CUDA(cudaMemcpyAsync(h_count, d_count, 4ull * C, cudaMemcpyDeviceToHost, st));
  if (h_keys && n) PF_CUDA(cudaMemcpyAsync(h_keys, d_keys, 4ull * n, cudaMemcpyDeviceToHost, st));
  if (h_overflow) PF_CUDA(cudaMemcpyAsync(h_overflow, d_ovf, 4, cudaMemcpyDeviceToHost, st));
  PF_CUDA(cudaStreamSynchronize(st));
  if (err) return fail(PF_ERR_DEVICE, "HashGrid: device error word " + std::to_string(err));
  return PF_OK;
}

}  // extern "C"
