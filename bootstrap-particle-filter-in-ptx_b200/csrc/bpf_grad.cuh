// bpf_grad.cuh — adjoint (reverse-mode) gradient of the plain filter's total
// log-likelihood with the resampling ancestors held fixed, and an FP64 replay
// of a taped run with forward-mode tangents.
//
// Tape written by a taped forward run (the plain tick kernels with TickArgs
// ckpt/csr/aux set):
//   csr[t][j]   first child slot of parent j after the resampling of tick t;
//               children of j are the slots [csr[t][j], csr[t][j+1]) (the
//               ancestors of systematic resampling are non-decreasing, so the
//               children of a parent are contiguous; csr[t][N] = N)
//   ckpt[s]     the particles pass 1 read at tick s*K (checkpoint every K ticks)
//   aux[t]      {1/S_t, nM_t}: normalised weight W_t,i = 2^(x_t,i - nM_t) / S_t
// Backward, per checkpoint segment from the last to the first: the segment's
// particles h_t are recomputed forward from the checkpoint, the tape's child
// lists and the counter-based PCG32 noise (nothing per particle-step is stored
// except the child lists), then the adjoint runs backward through it:
//   lambda_t,j = W_t,j g_t(h_t,j) + rho * sum_{i in children_t(j)} lambda_t+1,i
//   g_t(h)     = d log p(y_t | h) / dh
// and the parameter adjoints accumulate per CTA in FP64:
//   dL/dmu    += (1-rho) sum_i lambda_t+1,i          (h_t+1 = mu(1-rho) + rho h~ + sigma eps)
//   dL/drho   += sum_j cs_t,j (h_t,j - mu)           (cs = children sum)
//   dL/dsigma += sum_i lambda_t+1,i eps_t+1,i       (eps Gaussian or Student-t state noise)
// plus the stationary initial draw h_0 = mu + sigma z / sqrt(1-rho^2).
//
// Reference: tests/diff_bpf.py:186-237 differentiates the same loss by autograd
// with the resampling indices detached (:35-56, :230-231); the PTX edition's
// bpf_grad_alpha (ptx_assembly/bpf_kernels_full.ptx:1116-1384) is a one-step
// score, not a pathwise derivative.
#pragma once
#include "bpf_plain.cuh"

namespace bpf {

constexpr int kGradThreads = 256;
constexpr int kGradGroup   = 4;                          // consecutive parents per thread
constexpr int kGradTile    = kGradThreads * kGradGroup;  // parents per CTA
constexpr int kGradHeavy   = 32;                         // children per group above which the warp shares the walk
constexpr int kGradAcc     = 5;                          // FP64 accumulators per CTA

// Per-CTA accumulator slots
//   0: sum of children sums            -> dmu  (times 1-rho)
//   1: sum cs_j (h_j - mu)             -> drho
//   2: sum lambda_i eps_i              -> dsigma
//   3: sum lambda_0,i                  -> dmu  (initial draw)
//   4: sum lambda_0,i z_0,i            -> drho, dsigma (initial draw)

struct GradAdjArgs {
  int N;
  float mu, rho, sigma;
  ObsModel obs;
  const float* y;          // y_t (device)
  const float* h;          // h_t
  const int32_t* csr;      // children of tick t, null on the last tick
  const float* lam_next;   // lambda_t+1, null on the last tick
  float* lam;              // lambda_t (out)
  const float2* aux;       // {1/S_t, nM_t}
  PcgTick pc_next;         // noise constants of tick t+1
  PcgTick pc0;             // draw-0 constants (initial particles)
  int first;               // t == 0
  int nu_int;              // Student-t state noise dof (0 = Gaussian)
  float nu_state;
  double* acc;             // [CTAs][kGradAcc]
};

struct ReplayArgs {
  int N;
  double mu, rho, sigma;
  ObsModel obs;            // nu, c_obs used in FP64
  const float* y;          // y_t (device)
  const int32_t* csr;      // children of tick t-1 (null at t = 0)
  const double* hp;        // state of tick t-1: h[N4], dh/dmu, dh/drho, dh/dsigma at stride N4
  double* hc;              // state of tick t (out)
  int stride;              // N4
  PcgTick pc;              // noise constants of tick t
  int nu_int;              // Student-t state noise dof (0 = Gaussian)
  float nu_state;
  double* part;            // [CTAs][5]: (max, sum, sum*g*dh/dmu, .. drho, .. dsigma) of this tick
};

inline int grad_ctas(int N) { return (N + kGradTile - 1) / kGradTile; }
inline int grad_stride(int N) { return grad_ctas(N) * kGradTile; }

cudaError_t launch_grad_seed(int N, const float* ckpt, float* h_out, PcgTick pc, int propagate, float mu,
                             float rho, float sigma, int nu_int, float nu_state, cudaStream_t s, bool pdl);
cudaError_t launch_grad_recompute(int N, const int32_t* csr, const float* hp, float* hc, PcgTick pc, float mu,
                                  float rho, float sigma, int nu_int, float nu_state, cudaStream_t s, bool pdl);
cudaError_t launch_grad_adjoint(const GradAdjArgs& a, cudaStream_t s, bool pdl);
cudaError_t launch_grad_finish(int ctas, const double* acc, float mu, float rho, float sigma, double* grad,
                               cudaStream_t s, bool pdl);
cudaError_t launch_replay_init(const ReplayArgs& a, cudaStream_t s);
cudaError_t launch_replay_tick(const ReplayArgs& a, cudaStream_t s);
cudaError_t launch_replay_reduce(int T, int ctas, const double* part, double log_n, double* per_tick,
                                 double* total, cudaStream_t s);

}  // namespace bpf
