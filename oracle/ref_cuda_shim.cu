// TEST INFRASTRUCTURE ONLY: a C-linkage face over the reference's CUDA-C
// edition (gpu_bpf/gpu_bpf.cu behind gpu_bpf/gpu_bpf.cuh, the header this
// build's C ABI replaces), compiled with the reference source where it lies
// into oracle/_ref/librefcuda.so by oracle/build_ref.py. The tests use it as a
// statistical checker of the plain tick and of IMM (its noise is cuRAND
// XORWOW, so comparisons are statistical). This edition turns Silverman jitter
// on by default (gpu_bpf.cu:406-407); the wrappers take the shrink factor, so
// the tests run it with the jitter off, as this build's filter is. The product
// never links or loads this library.
#include "gpu_bpf.cuh"

#include <cuda_runtime.h>

extern "C" {

// gpu_bpf_create (gpu_bpf.cu:380-442) with the Silverman shrink and the ESS threshold set.
void* refc_create(int n, float rho, float sigma_z, float mu, float nu_state, float nu_obs, int seed,
                  float silverman, float ess_threshold) {
  GpuBpfState* s = gpu_bpf_create(n, rho, sigma_z, mu, nu_state, nu_obs, seed);
  if (!s) return nullptr;
  s->silverman_shrink = silverman;
  gpu_bpf_set_ess_threshold(s, ess_threshold);
  return s;
}

void refc_destroy(void* s) { gpu_bpf_destroy(static_cast<GpuBpfState*>(s)); }

int refc_resample_count(void* s) { return gpu_bpf_get_resample_count(static_cast<GpuBpfState*>(s)); }

// T ticks of gpu_bpf_step, one BpfResult per tick.
int refc_run(void* sv, const float* y, int T, float* h_mean, float* log_lik) {
  GpuBpfState* s = static_cast<GpuBpfState*>(sv);
  for (int t = 0; t < T; ++t) {
    const BpfResult r = gpu_bpf_step(s, y[t]);
    h_mean[t] = r.h_mean;
    log_lik[t] = r.log_lik;
  }
  return (int)cudaGetLastError();
}

// gpu_imm_create (gpu_bpf.cu:955-1015) from K x {rho, sigma_z, mu, nu_state, nu_obs}, then the
// Silverman shrink and the ESS threshold of every model's filter set. gpu_imm_step mixes each
// filter's BpfResult.log_lik, the log-evidence since its last resample; with threshold 0 every
// filter resamples each tick and that is the tick's increment.
void* refc_imm_create(const float* models, int K, int n, const float* transition, int seed, float silverman,
                      float ess_threshold) {
  ImmModelParams* m = new ImmModelParams[K];
  for (int k = 0; k < K; ++k) {
    m[k].rho = models[5 * k]; m[k].sigma_z = models[5 * k + 1]; m[k].mu = models[5 * k + 2];
    m[k].nu_state = models[5 * k + 3]; m[k].nu_obs = models[5 * k + 4];
  }
  GpuImmState* s = gpu_imm_create(m, K, n, transition, seed);
  delete[] m;
  if (!s) return nullptr;
  for (int k = 0; k < K; ++k) {
    s->filters[k]->silverman_shrink = silverman;
    gpu_bpf_set_ess_threshold(s->filters[k], ess_threshold);
  }
  return s;
}

void refc_imm_destroy(void* s) { gpu_imm_destroy(static_cast<GpuImmState*>(s)); }

// T ticks of gpu_imm_step (gpu_bpf.cu:1017-1080): mixed mean, log Z, best model per tick and the
// model probabilities after the last tick.
int refc_imm_run(void* sv, const float* y, int T, float* h_mean, float* log_lik, int* best, float* probs) {
  GpuImmState* s = static_cast<GpuImmState*>(sv);
  for (int t = 0; t < T; ++t) {
    const ImmResult r = gpu_imm_step(s, y[t]);
    h_mean[t] = r.h_mean;
    log_lik[t] = r.log_lik;
    best[t] = r.best_model;
  }
  if (probs) gpu_imm_get_probs(s, probs);
  return (int)cudaGetLastError();
}

}  // extern "C"
