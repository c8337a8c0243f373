// bpf_plain.cuh — device-memory layout and launchers of the plain filter.
//
// HBM layout of one filter of N particles, G = ceil(N/4096) tiles
// (every particle array is padded to G*4096 floats so tile loads never
// leave the allocation):
//   h[2][G*4096]  f32  particle ping-pong (current buffer index in DevState)
//   w[G*4096]     f32  tile-relative log2-weights d_i = x_i - n_k <= 0 (weight 2^d_i)
//   tile records  rec[G] f32x4 {S=sum w, Q=sum w^2, H=sum w h, n_k bits},
//                 nexp[G] i32 (n_k again), E[G] u64 exact fixed-point mass
//   P[G] u64 exclusive tile prefix of the fixed-point CDF, ofirst[G+1] i32
//   items[G + N/8192 + 1] int4 pass-2 work items (tile, first out, end out, flags)
//   DevState      scalars carried from tick to tick
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "bpf_alloc.cuh"
#include "bpf_common.cuh"
#include "../../include/gpu_bpf.h"

namespace bpf {

// Scalars that live on the device from tick to tick (no host round trip).
struct DevState {
  uint64_t k1, k2;          // PCG32 stream constants of the next tick t: slot i's state is
                            // k1 + k2 inc_i, k1 = A^t A^2 seed, k2 = A^t (A+1) + sum_{k<t} A^k;
                            // tick to tick k1 <- A k1, k2 <- A k2 + 1
  uint64_t u_state;         // resampling-uniform PCG32 (gpu_bpf_ptx_full.cu:353)
  uint64_t base, delta;     // systematic targets t_i = base + i*delta (fixed point)
  uint64_t delta_magic;     // floor((2^64-1)/delta)
  uint64_t total;           // fixed-point CDF total
  double   logS_prev;       // ln(sum of carried weights) in the carry frame; ln N after a resample
  double   ll_total;        // FP64 running log-likelihood
  double   ll_ref;          // log-evidence since the last resample
  int      tick;            // index of the next tick
  int      cur;             // h buffer holding the current particles
  int      src;             // pass-2 gather source buffer
  int      resampled_prev;  // previous tick resampled (1 before tick 0)
  int      nM_prev;         // global tile exponent of the previous tick
  int      do_resample;     // current tick resamples
  int      nM;              // global tile exponent of the current tick
  int      Fg;              // global-frame fraction bits
  int      n_items;         // pass-2 work items of the current tick
  uint32_t u23;             // resampling uniform of the current tick
  int      resample_count;
  int      dirs;            // tile orders (1 = decreasing): bit 0 the next pass 1, bit 1 this tick's pass 2
  int      error;           // sticky BPF_* error code
  int      seed;            // filter seed (PCG32 streams, resampling uniform)
  double   learn[4];        // online learning sums since the last update: sum_t of
                            // sum W dlw, sum W dlw^2, sum W dlw (h_prev-mu), sum W dlw^2 (h_prev-mu)^2
  double   hm;              // filtered mean of the current tick (FP64): the centre of Silverman jitter
  uint64_t jk1, jk2;        // PCG32 stream constants of the current tick's jitter draw
  float    bw;              // Silverman jitter bandwidth of the current tick
  int      seq;             // host request number of the current tick (copied into the mirror)
};
static_assert(sizeof(DevState) == 200, "DevState layout");

struct Plan {
  int N, G, max_items;
  float* h0; float* h1; float* w;
  int* nexp; unsigned long long* E; float4* rec;
  float4* rec2;              // per tile, online learning only: tile-frame sums of w dlw, w dlw^2, w dlw dh, w dlw^2 dh^2
  unsigned long long* P; int* ofirst; int4* items;
  double* jpart;             // per tile, Silverman jitter only: sum of (h - hm)^2 over the tile's particles
  unsigned* jticket;         // CTAs of the jitter-variance kernel done this tick (the last one resets it)
  unsigned* pticket;         // pass-1 CTAs done this tick when the last one runs the plan (it resets it)
  DevState* st;
};

// Host-mapped mirror of the state a synchronous tick reads back (zero-copy): written by the
// plan kernel at the end of every tick it is given to, and by pass 2 when it records an error.
struct TickMirror {
  int resample_count;
  int tick;                  // ticks completed
  int error;                 // DevState::error
  int seq;                   // host request number of the tick that wrote it (written last, after a
                             // system fence: the host may take the record once it sees its number)
};

struct TickArgs {
  float mu, rho, sigma;
  float ess_threshold;
  double log_n;              // ln N
  ObsModel obs;              // obs.y is used when y_ptr == nullptr
  const float* y_ptr;        // device pointer to this tick's observation, or null
  BpfTickRecord* rec;        // device record slot written by the last pass-1 CTA
  int32_t* anc;              // ancestors of this tick (N ints) or null
  int nu_int;                // Student-t state noise: round(nu_state) degrees of freedom, 0 = Gaussian
  float nu_state;            // Student-t state noise scale parameter
  int learn;                 // accumulate the online-learning score sums of this tick (needs p.rec2)
  int apf;                   // auxiliary particle filter stage: 0 = bootstrap tick, 1 = first stage
                             // (weights p(y | mu + rho (h - mu)), particles unchanged, tick not
                             // advanced), 2 = second stage (propagate, weights p(y|h) / p(y|m))
  // gradient tape (all null outside a taped run)
  float* ckpt;               // copy of the particles pass 1 reads this tick (G*4096 floats) or null
  int32_t* csr;              // on resampling ticks: first child slot of every parent (N ints) or null
  float2* aux;               // {1/S, nM}: normalised weight W_i = 2^(x_i - nM) / S of this tick, or null
  TickMirror* mirror;        // host-mapped mirror of this tick's outcome, or null
  int seq;                   // host request number of this tick (pass 1 stores it in the device state)
  int tail_plan;             // the last pass-1 CTA runs the plan (G <= kTailTiles; no plan launch)
  float silverman;           // Silverman jitter shrink after resampling (0 = off; needs p.jpart)
};

// Device buffers of a plan for N particles (G, max_items set; DevState included).
cudaError_t plan_alloc(Plan& p, int N);
void plan_free(Plan& p);

// Host-side launchers (stream-ordered, no synchronisation).
// Draws h_0 for `seed` and (re)initialises the DevState on the device.
cudaError_t launch_init(const Plan& p, float mu, float std_stat, int seed, cudaStream_t s);
// pdl = programmatic dependent launch on the previous kernel in the stream.
cudaError_t launch_pass1(const Plan& p, const TickArgs& a, cudaStream_t s, bool pdl);
// Filters of at most kTailTiles tiles may run the plan in pass 1's last CTA (a.tail_plan):
// the same plan code on 256 threads, one tile per thread, so the results equal the plan
// kernel's bit for bit; bootstrap ticks without learning or a gradient tape only.
constexpr int kTailTiles = 256;
bool tail_plan_eligible(const Plan& p, const TickArgs& a);
cudaError_t launch_plan(const Plan& p, const TickArgs& a, cudaStream_t s, bool pdl);
cudaError_t launch_pass2(const Plan& p, const TickArgs& a, int grid, cudaStream_t s, bool pdl);
// Silverman jitter of a resampling tick (both kernels exit at once on other ticks): the bandwidth
// from the resampled particles' spread about the tick's filtered mean, then h += bw z clamped to
// [mu - 8, mu + 8], z from the particle slot's next PCG32 draw.
cudaError_t launch_jitter(const Plan& p, const TickArgs& a, cudaStream_t s, bool pdl);
// Fused small-filter tick (N <= kSmallMaxN): one launch of one CTA runs n_ticks consecutive
// ticks (pass 1, plan and resampling), bit-identical to the three-kernel tick. a.y_ptr and
// a.rec point at the run's first tick (a.obs.y is the observation when y_ptr is null and
// n_ticks is 1). Not for learning, auxiliary-filter, Silverman or taped ticks.
bool small_eligible(const Plan& p, const TickArgs& a);
cudaError_t launch_small(const Plan& p, const TickArgs& a, int n_ticks, cudaStream_t s, bool pdl);
int pass2_grid_size(int device);
// Tiles the fused tick takes on this device (16, else 8; 4 before pass2_grid_size configured it).
int small_max_tiles(int device);
size_t pass2_smem_bytes();
cudaError_t launch_debug_pcg(int seed, int n, int t, uint32_t* d_out, float* d_norm, cudaStream_t s);
// w_out[i] = 2^d_i of the stored tile-relative log2-weights (N floats, device).
cudaError_t launch_tile_weights(const Plan& p, float* w_out, cudaStream_t s);

}  // namespace bpf

// Status and launch bookkeeping shared by the C entry points (bpf_api.cu).
int bpf_record_error(int code);          // sets gpu_bpf_last_error() for this thread, returns code
void bpf_note_launches(long long n);     // adds to gpu_bpf_launch_count()
