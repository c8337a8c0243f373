// bpf_alloc.cuh — every device and pinned allocation the library makes goes through
// these wrappers (except the allocation-free entry point, which makes none). They
// keep the set of live allocations and can be told to fail one allocation on
// purpose (gpu_bpf_debug_fail_alloc), the host-side fault injection with which the
// cleanup of every create path is tested: no GPU fault is involved.
#pragma once
#include <cstddef>
#include <cuda_runtime.h>

cudaError_t bpf_malloc_raw(void** p, size_t bytes);
cudaError_t bpf_malloc_host_raw(void** p, size_t bytes);
cudaError_t bpf_host_alloc_raw(void** p, size_t bytes, unsigned flags);
cudaError_t bpf_free(void* p);
cudaError_t bpf_free_host(void* p);

template <typename T>
inline cudaError_t bpf_malloc(T** p, size_t bytes) { return bpf_malloc_raw(reinterpret_cast<void**>(p), bytes); }
template <typename T>
inline cudaError_t bpf_malloc_host(T** p, size_t bytes) { return bpf_malloc_host_raw(reinterpret_cast<void**>(p), bytes); }
template <typename T>
inline cudaError_t bpf_host_alloc(T** p, size_t bytes, unsigned flags) {
  return bpf_host_alloc_raw(reinterpret_cast<void**>(p), bytes, flags);
}
