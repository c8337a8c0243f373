// bpf_alloc.cu — allocation wrappers with live-allocation tracking and a one-shot
// injected failure (see bpf_alloc.cuh). The injected failure returns
// cudaErrorMemoryAllocation without calling the runtime, as a real out-of-memory
// allocation would, so callers take their ordinary error path.
#include <atomic>
#include <mutex>
#include <unordered_set>

#include "bpf_alloc.cuh"
#include "../../include/gpu_bpf.h"

namespace {
std::mutex g_mutex;
std::unordered_set<void*> g_live;        // live device and pinned allocations
long long g_fail_in = -1;                 // allocations to let through before the injected failure
long long g_count = 0;                    // allocations attempted since load

// true when this allocation is the one to fail
bool take_failure() {
  std::lock_guard<std::mutex> lock(g_mutex);
  ++g_count;
  if (g_fail_in < 0) return false;
  if (g_fail_in == 0) { g_fail_in = -1; return true; }
  --g_fail_in;
  return false;
}

cudaError_t track(cudaError_t e, void** p) {
  if (e == cudaSuccess && *p) {
    std::lock_guard<std::mutex> lock(g_mutex);
    g_live.insert(*p);
  }
  return e;
}

void untrack(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lock(g_mutex);
  g_live.erase(p);
}
}  // namespace

cudaError_t bpf_malloc_raw(void** p, size_t bytes) {
  if (take_failure()) { *p = nullptr; return cudaErrorMemoryAllocation; }
  return track(cudaMalloc(p, bytes), p);
}
cudaError_t bpf_malloc_host_raw(void** p, size_t bytes) {
  if (take_failure()) { *p = nullptr; return cudaErrorMemoryAllocation; }
  return track(cudaMallocHost(p, bytes), p);
}
cudaError_t bpf_host_alloc_raw(void** p, size_t bytes, unsigned flags) {
  if (take_failure()) { *p = nullptr; return cudaErrorMemoryAllocation; }
  return track(cudaHostAlloc(p, bytes, flags), p);
}
cudaError_t bpf_free(void* p) {
  untrack(p);
  return cudaFree(p);
}
cudaError_t bpf_free_host(void* p) {
  untrack(p);
  return cudaFreeHost(p);
}

extern "C" {

int gpu_bpf_debug_fail_alloc(long long k) {
  std::lock_guard<std::mutex> lock(g_mutex);
  g_fail_in = k < 0 ? -1 : k;
  return BPF_OK;
}

long long gpu_bpf_debug_alloc_count(void) {
  std::lock_guard<std::mutex> lock(g_mutex);
  return g_count;
}

long long gpu_bpf_debug_live_allocs(void) {
  std::lock_guard<std::mutex> lock(g_mutex);
  return (long long)g_live.size();
}

}  // extern "C"
