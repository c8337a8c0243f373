// TEST INFRASTRUCTURE ONLY: a C-linkage face over the reference's own GPU
// filter (the PTX edition: gpu_bpf/gpu_bpf_ptx_full.cu driving the hand-written
// ptx_assembly/bpf_kernels_full.ptx), compiled together with the reference
// sources into oracle/_ref/ by oracle/build_ref.py. The tests use it to pin the
// oracle and the CUDA path against the reference itself run on the same GPU;
// bench.py's reference arm times it beside the CPU baseline. The product never
// links or loads it.
//
// The reference exports C++ names (gpu_bpf_full.cuh has no extern "C" block)
// and loads its PTX module from the current directory on the first create
// (gpu_bpf_ptx_full.cu:121-183), so create runs with the working directory
// switched to the directory of this library, where the build put the module.
#include "gpu_bpf_full.cuh"

#include <cuda_runtime.h>
#include <dlfcn.h>
#include <limits.h>
#include <string.h>
#include <unistd.h>

#include <chrono>
#include <string>

namespace {

std::string lib_dir() {
  Dl_info info;
  if (!dladdr(reinterpret_cast<void*>(&lib_dir), &info) || !info.dli_fname) return ".";
  std::string p(info.dli_fname);
  const size_t slash = p.rfind('/');
  return slash == std::string::npos ? std::string(".") : p.substr(0, slash);
}

}  // namespace

extern "C" {

// gpu_bpf_create (gpu_bpf_ptx_full.cu:340-438): allocates, seeds the PCG32
// streams (draw 0 feeds the initial particles) and synchronises.
void* refgpu_create(int n, float rho, float sigma_z, float mu, float nu_state, float nu_obs, int seed) {
  char cwd[PATH_MAX];
  const bool have_cwd = getcwd(cwd, sizeof(cwd)) != nullptr;
  if (chdir(lib_dir().c_str()) != 0) return nullptr;
  GpuBpfState* s = gpu_bpf_create(n, rho, sigma_z, mu, nu_state, nu_obs, seed);
  if (have_cwd && chdir(cwd) != 0) return s;
  return s;
}

void refgpu_destroy(void* s) { gpu_bpf_destroy(static_cast<GpuBpfState*>(s)); }

// gpu_bpf_set_ess_threshold (gpu_bpf_ptx_full.cu:858-860); 0 = always resample.
void refgpu_set_ess(void* s, float thr) { gpu_bpf_set_ess_threshold(static_cast<GpuBpfState*>(s), thr); }

int refgpu_resample_count(void* s) { return gpu_bpf_get_resample_count(static_cast<GpuBpfState*>(s)); }

int refgpu_timestep(void* s) { return static_cast<GpuBpfState*>(s)->timestep; }

// T ticks of gpu_bpf_step (gpu_bpf_ptx_full.cu:764-775), one BpfResult per tick.
int refgpu_run(void* sv, const float* y, int T, float* h_mean, float* log_lik) {
  GpuBpfState* s = static_cast<GpuBpfState*>(sv);
  for (int t = 0; t < T; ++t) {
    const BpfResult r = gpu_bpf_step(s, y[t]);
    h_mean[t] = r.h_mean;
    log_lik[t] = r.log_lik;
  }
  return (int)cudaGetLastError();
}

// T ticks of gpu_bpf_step_async (gpu_bpf_ptx_full.cu:550-752), the reference's
// fastest tick loop, and one gpu_bpf_get_result at the end. Returns the wall
// time in milliseconds from the first launch to the synchronised end of the
// last tick; the host round trips of the ESS decision are part of it.
double refgpu_time_run(void* sv, const float* y, int T, float* last) {
  GpuBpfState* s = static_cast<GpuBpfState*>(sv);
  cudaStreamSynchronize(s->stream);
  const auto t0 = std::chrono::steady_clock::now();
  for (int t = 0; t < T; ++t) gpu_bpf_step_async(s, y[t]);
  cudaStreamSynchronize(s->stream);
  const auto t1 = std::chrono::steady_clock::now();
  const BpfResult r = gpu_bpf_get_result(s);
  if (last) { last[0] = r.h_mean; last[1] = r.log_lik; }
  return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

// Wall time in milliseconds of `warmup` untimed then T timed ticks of the synchronous per-tick
// API gpu_bpf_step (gpu_bpf_ptx_full.cu:764-775), the loop of the reference's matched-DGP
// throughput test (tests/test_bpf_matched_dgp.cu:560-603): warm-up ticks take y[t % T].
double refgpu_time_steps(void* sv, const float* y, int T, int warmup) {
  GpuBpfState* s = static_cast<GpuBpfState*>(sv);
  for (int t = 0; t < warmup; ++t) gpu_bpf_step(s, y[t % T]);
  cudaDeviceSynchronize();
  const auto t0 = std::chrono::steady_clock::now();
  for (int t = 0; t < T; ++t) gpu_bpf_step(s, y[t]);
  cudaDeviceSynchronize();
  const auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

// Online mu / rho learning of the reference (gpu_bpf_full.cuh:197-210, gpu_bpf_ptx_full.cu:469-544,
// 777-828).
void refgpu_enable_mu_learning(void* s, int mode, int K, float c, float t0, float gamma) {
  gpu_bpf_enable_mu_learning(static_cast<GpuBpfState*>(s), mode, K, c, t0, gamma);
}
void refgpu_enable_rho_learning(void* s, int enable) {
  gpu_bpf_enable_rho_learning(static_cast<GpuBpfState*>(s), enable);
}
float refgpu_get_mu(void* s) { return gpu_bpf_get_mu(static_cast<GpuBpfState*>(s)); }
float refgpu_get_rho(void* s) { return gpu_bpf_get_rho(static_cast<GpuBpfState*>(s)); }

// Device state read-back: the PCG32 states [state, inc] per particle
// (gpu_bpf_full.cuh:87), the particles and the normalised weights of the last tick.
int refgpu_copy_rng(void* sv, unsigned long long* out, int n) {
  GpuBpfState* s = static_cast<GpuBpfState*>(sv);
  cudaStreamSynchronize(s->stream);
  return (int)cudaMemcpy(out, s->d_rng, (size_t)n * 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
}

int refgpu_copy_h(void* sv, float* out, int n) {
  GpuBpfState* s = static_cast<GpuBpfState*>(sv);
  cudaStreamSynchronize(s->stream);
  return (int)cudaMemcpy(out, s->d_h, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
}

// After a resampling tick the reference's scratch buffer holds the propagated,
// pre-resampling particles of that tick (the resample gathers into it and the
// buffers swap, gpu_bpf_ptx_full.cu:698-706).
int refgpu_copy_h2(void* sv, float* out, int n) {
  GpuBpfState* s = static_cast<GpuBpfState*>(sv);
  cudaStreamSynchronize(s->stream);
  return (int)cudaMemcpy(out, s->d_h2, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
}

int refgpu_copy_w(void* sv, float* out, int n) {
  GpuBpfState* s = static_cast<GpuBpfState*>(sv);
  cudaStreamSynchronize(s->stream);
  return (int)cudaMemcpy(out, s->d_w, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
}

// The reference's auxiliary particle filter (gpu_bpf_ptx_full.cu:1050-1175;
// cuRAND state noise, so comparisons with it are statistical).
void* refgpu_apf_create(int n, float rho, float sigma_z, float mu, float nu_state, float nu_obs, int seed) {
  return gpu_apf_create(n, rho, sigma_z, mu, nu_state, nu_obs, seed);
}

void refgpu_apf_destroy(void* s) { gpu_apf_destroy(static_cast<GpuApfState*>(s)); }

int refgpu_apf_run(void* sv, const float* y, int T, float* h_mean, float* log_lik) {
  GpuApfState* s = static_cast<GpuApfState*>(sv);
  for (int t = 0; t < T; ++t) {
    const BpfResult r = gpu_apf_step(s, y[t]);
    h_mean[t] = r.h_mean;
    log_lik[t] = r.log_lik;
  }
  return (int)cudaGetLastError();
}

// Wall time in milliseconds of T reference APF ticks (gpu_apf_step, synchronous per tick).
double refgpu_apf_time(void* sv, const float* y, int T) {
  GpuApfState* s = static_cast<GpuApfState*>(sv);
  cudaStreamSynchronize(s->stream);
  const auto t0 = std::chrono::steady_clock::now();
  for (int t = 0; t < T; ++t) gpu_apf_step(s, y[t]);
  cudaStreamSynchronize(s->stream);
  const auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

}  // extern "C"
