// bpf_batch.cuh — many independent SV filters (different theta, N and seed)
// sharing one observation series, in one persistent launch per size class.
//
// A CTA owns one filter at a time and keeps its particles, weights and
// ancestor slots in shared memory for all T ticks, so the per-tick HBM
// traffic is zero; the kernel is bound by instruction issue and shared
// memory. Filters are taken from a per-class work counter in LPT order
// (largest N first). The arithmetic per particle is the plain filter's
// (same PCG32 draw, inverse CDF, propagation, log2-weight, tile-relative
// weights over 4096-particle tiles and the same fixed-point systematic
// resampling), so a batched filter reproduces the plain filter with the same
// theta, N and seed: identical ancestors and particles, log-likelihood equal
// up to the order of floating-point sums.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "bpf_common.cuh"
#include "../../include/gpu_bpf.h"

namespace bpf {

constexpr int kBatchMaxN = 16384;          // largest filter the shared-memory layout holds
constexpr int kBatchMaxTiles = kBatchMaxN / kTile;

struct BatchFilterDev {                    // 48 bytes, one per filter
  float mu, rho, sigma, std_stat;
  float nu, c_obs, inv_nu, nu_p1h;
  int n, seed;
  int nu_int;                              // Student-t state noise dof round(nu_state), 0 = Gaussian
  float nu_state;
};

// Resumable state of one filter between launches (runs that continue from a
// saved tick: the IMM step and any caller that steps the batch a few ticks at
// a time). The particle and carried-weight arrays live at st_off[b] in st_h/st_w.
struct BatchFilterState {
  double logS_prev, ll_total;
  unsigned long long ustate;   // resampling-uniform PCG32 state
  int carry, n_res;
  float carry_off[kBatchMaxTiles];
  float hm_last;
  int pad;
};

struct BatchArgs {
  const BatchFilterDev* filters;
  const int* order;           // filter indices of this class, largest N first
  int n_order;
  int* counter;               // work counter of this class (zeroed before the launch)
  const float* y;             // observations [T]
  int T;
  float ess_threshold;
  double* loglik;             // [B] total log-likelihood (FP64)
  double* dll;                // [B*T] per-tick increments, or null
  float* hmean;               // [B*T] filtered means, or null
  float* h_final;             // [B] filtered mean at the last tick
  int* resamples;             // [B] resampling count
  int32_t* anc;               // [B*T*kBatchMaxN] ancestors, or null (testing)
  float* particles;           // [B*kBatchMaxN] final particles, or null (testing)
  // gradient runs: tape of the launch's CTA slots (one filter at a time per slot), all null otherwise.
  // Strides use the class's largest N (maxn); per-slot bases are taken from blockIdx.x.
  unsigned short* g_list;     // [slots][T][maxn] first child of every parent, in thread-chunk order
  float* g_ckpt;              // [slots][ceil(T/K)][maxn] particles entering every K-th tick
  float2* g_norm;             // [slots][T] {1/S, nM}: W_i = 2^(x_i - nM) / S
  float* g_seg;               // [slots][K][maxn] recomputed particles of one checkpoint segment
  const ulonglong2* g_AB;     // [T+1] PCG32 jump constants (A^t, sum_{k<t} A^k)
  int g_K;                    // checkpoint interval
  double* grad;               // [3B] d loglik / d(mu, rho, sigma_z)
  // resumable runs (all null for a run from tick 0 that keeps nothing)
  const int* t0_dev;          // first tick of this launch (device); y, dll, hmean are indexed from it
  BatchFilterState* st;       // [B] state saved at the end and, when *t0_dev > 0, loaded at the start
  float* st_h;                // particles of every filter at st_off[b]
  float* st_w;                // carried weights of every filter at st_off[b]
  const long long* st_off;    // [B]
  int y_abs;                  // 1: y is indexed by the absolute tick (y[t]) instead of from t0
  // correlated-noise runs (all null otherwise): the auxiliary noise of filter b is an area at
  // nz_out + nz_out_off[b] of batch_noise_stride(n) floats per absolute tick: the particles'
  // standard normals (tick 0: the initial draw), then the normal of the tick's resampling
  // uniform. With nz_in, noise = cp_rho * (nz_in + nz_in_off[b])[...] + cp_scale * fresh.
  // Particles are sorted by value before every resampling. One tile (n <= 4096) and Gaussian
  // state noise only.
  const float* nz_in;
  float* nz_out;
  const long long* nz_in_off; // [B]
  const long long* nz_out_off;// [B]
  float cp_rho, cp_scale;
  // Launch epilogue of resumable steps (null ep_done: none, the host zeroes the
  // counter before the launch): the CTA that finishes last of the ep_total CTAs
  // launched over all classes zeroes the ep_n work counters and ep_done and
  // adds ep_add to *ep_tick, so a step is one kernel node per class.
  int* ep_done;
  int* ep_counters;
  int* ep_tick;
  int ep_total, ep_n, ep_add;
};

// Floats per tick in a correlated-noise area of a filter of n particles.
__host__ __device__ inline int batch_noise_stride(int n) { return ((n + 3) & ~3) + 4; }

// Dynamic shared memory of the class kernel for filters of at most maxn particles (with
// sort_perm: plus the sort permutation of correlated-noise runs that record ancestors).
size_t batch_smem_bytes(int maxn, bool sort_perm = false);
// Launches the kernel instance with `threads` threads per CTA (64..1024, power of 2).
cudaError_t launch_batch_class(const BatchArgs& a, int threads, int maxn, int grid, cudaStream_t s);
// CTAs per SM the class kernel can keep resident.
int batch_occupancy(int threads, int maxn);

// Gradient form: every CTA runs a filter's taped forward and then its adjoint
// backward (segment recompute from checkpoints and child lists, lambda in
// shared memory) before taking the next filter.
size_t batch_grad_smem_bytes(int maxn);
cudaError_t launch_batch_grad_class(const BatchArgs& a, int threads, int maxn, int grid, cudaStream_t s);
int batch_grad_occupancy(int threads, int maxn);
// Filter j of a correlated-noise buffer takes the first `floats` floats (a multiple of 4) of the
// area at src_off[j] into the area at dst_off[j] (16-byte aligned areas that do not overlap).
cudaError_t launch_noise_gather(float* nz, const long long* src_off, const long long* dst_off, long long floats,
                                int B, cudaStream_t s);
// Filter j of dst takes the resumable state and table entry of filter idx[j] of src (every j, or
// those with mask[j] != 0); with new_seed, filter j continues with seed new_seed[j] (fresh noise
// streams and resampling uniforms). Filters have n particles each at offsets off[]; src and dst
// must not alias.
cudaError_t launch_batch_gather(BatchFilterDev* dst_tab, BatchFilterState* dst_st, float* dst_h, float* dst_w,
                                const BatchFilterDev* src_tab, const BatchFilterState* src_st, const float* src_h,
                                const float* src_w, const long long* off, const int* idx, const int* mask,
                                const int* new_seed, int n, int B, cudaStream_t s);

}  // namespace bpf
