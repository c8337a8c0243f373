// bpf_block.cuh — warp/CTA reductions and scans, PTX helpers (dependent
// launch, mbarrier, bulk async copy, global timer) and fixed-point helpers
// shared by the plain and batched filter kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "bpf_common.cuh"

namespace bpf {

// ---------------------------------------------------------------------------
// PTX helpers: dependent launch, mbarrier, bulk async copy, timer
// ---------------------------------------------------------------------------
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// 1-D bulk copy global -> shared, completion counted on the mbarrier.
// Both addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Wait for phase `parity` of the mbarrier; gives up after ~1 s and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_addr(bar);
  const uint64_t t0 = global_timer_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (global_timer_ns() - t0 > 1000000000ull) return false;
  }
}

// ---------------------------------------------------------------------------
// Block-wide reductions and scans for NT threads (NT a multiple of 32)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ int warp_max_i(int v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Sums over lanes 0..WIDTH-1 (WIDTH a power of two <= 32), complete in those lanes. When the
// other lanes hold zeros, lane 0 gets the same value as warp_sum_d / warp_sum_u64 (their extra
// steps only add exact zeros).
template <int WIDTH>
__device__ __forceinline__ double warp_sum_d_w(double v) {
#pragma unroll
  for (int o = WIDTH / 2; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <int WIDTH>
__device__ __forceinline__ unsigned long long warp_sum_u64_w(unsigned long long v) {
#pragma unroll
  for (int o = WIDTH / 2; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Barrier of a block-level helper run by NT threads: the whole CTA, or, for NT = 32, the one
// warp that runs it while the rest of the CTA does something else.
template <int NT>
__device__ __forceinline__ void nt_sync() {
  if constexpr (NT == 32) __syncwarp();
  else __syncthreads();
}

template <typename T>
__device__ __forceinline__ T warp_incl_scan_add(T v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  return v;
}
// Exclusive prefix sum over the NT threads of a CTA; *total gets the sum.
// sh holds NT/32 + 1 entries. All threads must call it (it has barriers).
// TRAIL = false leaves out the last barrier: the caller then passes another
// barrier before sh is written again.
template <int NT, typename T, bool TRAIL = true>
__device__ T block_excl_scan_add(T v, T* total, T* sh) {
  constexpr int W = NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const T inc = warp_incl_scan_add(v, lane);
  if (lane == 31) sh[warp] = inc;
  nt_sync<NT>();
  if (warp == 0) {
    const T t = lane < W ? sh[lane] : T(0);
    const T ti = warp_incl_scan_add(t, lane);
    __syncwarp();
    if (lane < W) sh[lane] = ti - t;
    if (lane == W - 1) sh[W] = ti;
  }
  nt_sync<NT>();
  const T r = sh[warp] + inc - v;
  *total = sh[W];
  if constexpr (TRAIL) nt_sync<NT>();
  return r;
}
template <int NT>
__device__ int block_max_i(int v, int* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_max_i(v);
  if (lane == 0) sh[warp] = v;
  nt_sync<NT>();
  int m = sh[0];
#pragma unroll
  for (int w = 1; w < NT / 32; ++w) m = max(m, sh[w]);
  nt_sync<NT>();
  return m;
}

// 2^e as a double (exact IEEE encoding; 0 below the normal range).
__device__ __forceinline__ double pow2d(int e) {
  if (e < -1022) return 0.0;
  if (e > 1023) return __longlong_as_double(0x7FF0000000000000LL);
  return __longlong_as_double((long long)(e + 1023) << 52);
}
__device__ __forceinline__ unsigned long long shr64(unsigned long long x, int r) {
  return r >= 64 ? 0ull : (x >> r);
}
__host__ __device__ inline int ceil_log2_u(unsigned n) {
#ifdef __CUDA_ARCH__
  return n <= 1u ? 0 : 32 - __clz((int)(n - 1u));
#else
  int c = 0;
  while ((1ull << c) < (unsigned long long)n) ++c;
  return c;
#endif
}

// #{ i in [0,N) : base + i*delta < c } (targets strictly below c)
__device__ __forceinline__ int targets_below(unsigned long long c, unsigned long long base,
                                             unsigned long long delta, unsigned long long magic, int N) {
  if (c <= base) return 0;
  const unsigned long long q = udiv_magic(c - base - 1ull, delta, magic) + 1ull;
  return q >= (unsigned long long)N ? N : (int)q;
}

}  // namespace bpf
