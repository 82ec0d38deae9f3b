// capi_sort.cu — C ABI of the standalone neighbour-grid sort and the
// library-wide error plumbing (pf_last_error, pf_abi_version).

#include <cuda_runtime.h>

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
  size_t scratch_bytes = 0;
  // staging for pf_sort_host
  void* io = nullptr;
  size_t io_bytes = 0;
  // counters of the most recent call (its error word is read by
  // pf_sort_device_errors)
  uint32_t* counters = nullptr;
};

std::mutex g_ws_mutex;
std::map<std::pair<int, cudaStream_t>, Workspace> g_ws;

pf_status ensure(void** ptr, size_t* have, size_t need) {
  if (*have >= need && *ptr) return PF_OK;
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  *have = 0;
  const size_t grow = need + need / 4;
  if (cudaMalloc(ptr, grow) != cudaSuccess) {
    cudaGetLastError();
    return fail(PF_ERR_OOM, "HashGrid: out of device memory for sort scratch");
  }
  *have = grow;
  return PF_OK;
}

Workspace& workspace_for(cudaStream_t st) {
  int dev = 0;
  cudaGetDevice(&dev);
  return g_ws[{dev, st}];
}

pf_status validate(uint32_t n, const pf_grid_desc* grid, KeyFn* kf, uint64_t* C) {
  if (!grid) return fail(PF_ERR_INVALID, "HashGrid: grid descriptor is NULL");
  if (!make_key_fn(*grid, kf, C)) {
    if (!(grid->cell_size > 0))
      return fail(PF_ERR_INVALID, "HashGrid: cellSize must be a positive finite number, got " +
                                      std::to_string(grid->cell_size));
    if (grid->key_kind == PF_KEY_MORTON)
      return fail(PF_ERR_INVALID, "HashGrid: hashTableSize must be a positive power of two, got " +
                                      std::to_string(grid->table_size));
    return fail(PF_ERR_INVALID, "HashGrid: invalid grid descriptor");
  }
  if (n > 0x7fffffffu) return fail(PF_ERR_INVALID, "HashGrid: too many particles");
  return PF_OK;
}

// Runs the sort on prepared device buffers with scratch `s`.
void run_sort(const float4* pos, uint32_t n, const KeyFn& kf, uint64_t C, uint32_t* perm, uint32_t* start,
              uint32_t* count, uint32_t* keys, uint32_t* overflow, const SortScratch& s, cudaStream_t st) {
  cudaMemsetAsync(count, 0, 4ull * C, st);
  cudaMemsetAsync(s.counters, 0, 4ull * kNumCounters, st);
  uint32_t* ovf = overflow ? overflow : s.counters + kCounterOverflow;
  if (overflow) cudaMemsetAsync(overflow, 0, 4, st);
  launch_keys_hist(pos, n, kf, keys, count, ovf, st);
  launch_sort_from_hist(keys, n, C, count, start, perm, s, st);
}

}  // namespace
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
  PF_TRY(validate(n, grid, &kf, &C));
  if (n > 0 && (!d_pos4 || !d_perm)) return fail(PF_ERR_INVALID, "HashGrid: NULL positions or perm");
  if (!d_start || !d_count) return fail(PF_ERR_INVALID, "HashGrid: NULL start or count");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  std::lock_guard<std::mutex> g(g_ws_mutex);
  Workspace& ws = workspace_for(st);
  PF_TRY(ensure(&ws.scratch, &ws.scratch_bytes, sort_scratch_bytes(n, C)));
  SortScratch s;
  sort_scratch_carve(ws.scratch, n, C, &s);
  ws.counters = s.counters;
  run_sort(reinterpret_cast<const float4*>(d_pos4), n, kf, C, d_perm, d_start, d_count,
           d_keys ? d_keys : s.keys, d_overflow, s, st);
  PF_CUDA(cudaGetLastError());
  return PF_OK;
}

// Synchronises `stream` and returns (and clears) the device error word of the
// standalone sort's workspace on that stream.
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
  PF_TRY(validate(n, grid, &kf, &C));
  if (n > 0 && !h_pos4) return fail(PF_ERR_INVALID, "HashGrid: NULL positions");
  cudaStream_t st = nullptr;
  std::lock_guard<std::mutex> g(g_ws_mutex);
  Workspace& ws = workspace_for(st);
  auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
  const size_t io = al(16ull * n) + al(4ull * n) + al(4ull * C) + al(4ull * C) + al(4ull * n) + al(4);
  PF_TRY(ensure(&ws.io, &ws.io_bytes, io));
  PF_TRY(ensure(&ws.scratch, &ws.scratch_bytes, sort_scratch_bytes(n, C)));
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
  SortScratch s;
  sort_scratch_carve(ws.scratch, n, C, &s);
  if (n) PF_CUDA(cudaMemcpyAsync(d_pos, h_pos4, 16ull * n, cudaMemcpyHostToDevice, st));
  run_sort(d_pos, n, kf, C, d_perm, d_start, d_count, d_keys, d_ovf, s, st);
  PF_CUDA(cudaGetLastError());
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
