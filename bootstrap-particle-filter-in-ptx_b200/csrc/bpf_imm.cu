// bpf_imm.cu — IMM (interacting multiple model) over K SV models: the
// reference's gpu_imm_* entry points (gpu_bpf/gpu_bpf.cuh:131-164, behaviour
// gpu_bpf/gpu_bpf.cu:947-1122).
//
// The reference steps K independent filters on K streams (about 15 launches
// per filter per tick, one device-wide synchronisation) and mixes the model
// probabilities on the host. Here the K filters are one resumable batch
// (gpu_bpf_batch_step_device): every tick is one graph launch for all models,
// one 4-byte upload and one download of the K increments and means. Filters
// with more than 16384 particles (beyond the batched kernel's shared-memory
// layout) are stepped as K plain filters instead. Model k uses the seed
// seed + 7919 k and the plain filter's default ESS threshold 0.5, as the
// reference's gpu_bpf_create calls do, so each model's particles equal a
// plain filter's with those arguments.
//
// Update (reference gpu_bpf.cu:1029-1064): log pi_k^- = LSE_j(log T[j,k] +
// log pi_j); log pi_k = log pi_k^- + l_k - log Z, with l_k the model's
// log-likelihood increment of the tick (the reference passes BpfResult.log_lik,
// which after a skipped resample is the log-evidence since the last
// resample; the increment is the quantity the Bayes update needs).
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/gpu_bpf.h"
#include "bpf_alloc.cuh"

int bpf_record_error(int code);

namespace {

constexpr int kImmMaxModels = 64;            // IMM_MAX_MODELS, gpu_bpf/gpu_bpf.cuh:15
constexpr int kImmMaxBatchN = 16384;         // largest filter of the batched kernel

double lse(const double* x, int n) {
  double m = -INFINITY;
  for (int i = 0; i < n; ++i) m = std::fmax(m, x[i]);
  if (!std::isfinite(m)) return m;
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += std::exp(x[i] - m);
  return m + std::log(s);
}

// The tick's observation and the models' increments and means live in host-mapped memory: the
// batched kernel reads y and writes its outputs there directly (the *_dev pointers are device
// views of the *_pin allocations), so a tick is one graph launch and one synchronise, no copies.
struct ImmImpl {
  int device = 0;
  GpuBpfBatch* batch = nullptr;
  cudaStream_t stream = nullptr;
  float* y_dev = nullptr;
  float* y_pin = nullptr;
  double* dll_dev = nullptr;
  double* dll_pin = nullptr;
  float* hm_dev = nullptr;
  float* hm_pin = nullptr;
};

void free_impl(ImmImpl* m) {
  if (!m) return;
  if (m->batch) gpu_bpf_batch_destroy(m->batch);
  bpf_free_host(m->y_pin); bpf_free_host(m->dll_pin); bpf_free_host(m->hm_pin);
  delete m;
}

}  // namespace

extern "C" {

GpuImmState* gpu_imm_create(const ImmModelParams* models, int n_models, int n_particles_per_model,
                            const float* transition_matrix, int seed) {
  if (!models || n_models <= 0 || n_models > kImmMaxModels || n_particles_per_model <= 0) {
    bpf_record_error(BPF_ERR_ARG);
    return nullptr;
  }
  const int K = n_models, N = n_particles_per_model;
  GpuImmState* s = (GpuImmState*)calloc(1, sizeof(GpuImmState));
  if (!s) { bpf_record_error(BPF_ERR_ALLOC); return nullptr; }
  s->n_models = K;
  s->n_particles_per_model = N;
  s->log_pi = (double*)malloc(K * sizeof(double));
  s->log_pi_pred = (double*)malloc(K * sizeof(double));
  s->log_T = (double*)malloc((size_t)K * K * sizeof(double));
  ImmImpl* m = new ImmImpl();
  s->impl = m;
  auto fail = [&](int code) -> GpuImmState* {
    gpu_imm_destroy(s);
    bpf_record_error(code);
    return nullptr;
  };
  if (!s->log_pi || !s->log_pi_pred || !s->log_T) return fail(BPF_ERR_ALLOC);
  for (int k = 0; k < K; ++k) s->log_pi[k] = -std::log((double)K);
  if (transition_matrix) {                                   // gpu_bpf.cu:993-995
    for (int i = 0; i < K * K; ++i) s->log_T[i] = std::log(std::fmax((double)transition_matrix[i], 1e-30));
  } else {                                                   // gpu_bpf.cu:996-1001
    const double p_stay = 0.95, p_switch = (K > 1) ? (1.0 - p_stay) / (K - 1) : 0.0;
    for (int i = 0; i < K; ++i)
      for (int j = 0; j < K; ++j) s->log_T[i * K + j] = std::log(std::fmax(i == j ? p_stay : p_switch, 1e-30));
  }

  if (N <= kImmMaxBatchN) {
    std::vector<BpfBatchFilter> fl(K);
    for (int k = 0; k < K; ++k) {
      fl[k].mu = models[k].mu; fl[k].rho = models[k].rho; fl[k].sigma_z = models[k].sigma_z;
      fl[k].nu_obs = models[k].nu_obs; fl[k].nu_state = models[k].nu_state;
      fl[k].n_particles = N;
      fl[k].seed = seed + k * 7919;                          // gpu_bpf.cu:979-985
    }
    m->batch = gpu_bpf_batch_create(fl.data(), K, 0.5f);     // gpu_bpf_create's default threshold
    if (!m->batch) return fail(gpu_bpf_last_error());
    if (cudaGetDevice(&m->device) != cudaSuccess) return fail(BPF_ERR_CUDA);
    m->stream = (cudaStream_t)gpu_bpf_batch_stream(m->batch);
    if (bpf_host_alloc(&m->y_pin, sizeof(float), cudaHostAllocMapped) != cudaSuccess ||
        bpf_host_alloc(&m->dll_pin, K * sizeof(double), cudaHostAllocMapped) != cudaSuccess ||
        bpf_host_alloc(&m->hm_pin, K * sizeof(float), cudaHostAllocMapped) != cudaSuccess) {
      cudaGetLastError();
      return fail(BPF_ERR_ALLOC);
    }
    if (cudaHostGetDevicePointer(reinterpret_cast<void**>(&m->y_dev), m->y_pin, 0) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void**>(&m->dll_dev), m->dll_pin, 0) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void**>(&m->hm_dev), m->hm_pin, 0) != cudaSuccess) {
      cudaGetLastError();
      return fail(BPF_ERR_CUDA);
    }
  } else {
    s->filters = (GpuBpfState**)calloc(K, sizeof(GpuBpfState*));
    if (!s->filters) return fail(BPF_ERR_ALLOC);
    for (int k = 0; k < K; ++k) {
      s->filters[k] = gpu_bpf_create(N, models[k].rho, models[k].sigma_z, models[k].mu, models[k].nu_state,
                                     models[k].nu_obs, seed + k * 7919);
      if (!s->filters[k]) return fail(gpu_bpf_last_error());
    }
  }
  return s;
}

void gpu_imm_destroy(GpuImmState* s) {
  if (!s) return;
  if (s->filters) {
    for (int k = 0; k < s->n_models; ++k) gpu_bpf_destroy(s->filters[k]);
    free(s->filters);
  }
  free_impl(reinterpret_cast<ImmImpl*>(s->impl));
  free(s->log_pi); free(s->log_pi_pred); free(s->log_T);
  free(s);
}

ImmResult gpu_imm_step(GpuImmState* s, float y_t) {
  ImmResult bad;
  bad.h_mean = NAN; bad.vol = NAN; bad.log_lik = NAN; bad.best_model = -1; bad.best_prob = NAN;
  if (!s || !s->impl) { bpf_record_error(BPF_ERR_STATE); return bad; }
  if (!std::isfinite(y_t)) { bpf_record_error(BPF_ERR_ARG); return bad; }
  ImmImpl* m = reinterpret_cast<ImmImpl*>(s->impl);
  const int K = s->n_models;

  // 1. interaction: log pi_k^- = LSE_j(log T[j,k] + log pi_j)   (gpu_bpf.cu:1029-1034)
  std::vector<double> terms(K), ll(K), hm(K), joint(K);
  for (int k = 0; k < K; ++k) {
    for (int j = 0; j < K; ++j) terms[j] = s->log_T[j * K + k] + s->log_pi[j];
    s->log_pi_pred[k] = lse(terms.data(), K);
  }

  // 2. all models advance one tick
  if (m->batch) {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || (cur != m->device && cudaSetDevice(m->device) != cudaSuccess)) {
      bpf_record_error(BPF_ERR_CUDA);
      return bad;
    }
    *m->y_pin = y_t;                       // the previous tick has completed: nothing reads it now
    if (gpu_bpf_batch_step_device(m->batch, m->y_dev, 1, m->dll_dev, m->hm_dev) != BPF_OK) return bad;
    if (cudaStreamSynchronize(m->stream) != cudaSuccess) {
      cudaGetLastError();
      bpf_record_error(BPF_ERR_CUDA);
      return bad;
    }
    for (int k = 0; k < K; ++k) { ll[k] = m->dll_pin[k]; hm[k] = m->hm_pin[k]; }
  } else {
    for (int k = 0; k < K; ++k) gpu_bpf_step_async(s->filters[k], y_t);
    for (int k = 0; k < K; ++k) {
      BpfTickRecord r;
      if (gpu_bpf_get_record(s->filters[k], &r) != BPF_OK) return bad;
      ll[k] = r.dloglik;
      hm[k] = r.h_mean;
    }
  }

  // 3. update and mix (gpu_bpf.cu:1050-1078)
  for (int k = 0; k < K; ++k) joint[k] = s->log_pi_pred[k] + ll[k];
  const double logZ = lse(joint.data(), K);
  double h_mixed = 0.0, best = -INFINITY;
  int best_k = 0;
  for (int k = 0; k < K; ++k) {
    s->log_pi[k] = joint[k] - logZ;
    h_mixed += std::exp(s->log_pi[k]) * hm[k];
    if (s->log_pi[k] > best) { best = s->log_pi[k]; best_k = k; }
  }
  s->timestep++;
  ImmResult r;
  r.h_mean = (float)h_mixed;
  r.vol = expf((float)h_mixed * 0.5f);
  r.log_lik = (float)logZ;
  r.best_model = best_k;
  r.best_prob = (float)std::exp(best);
  return r;
}

float gpu_imm_get_prob(const GpuImmState* s, int k) {
  if (!s || k < 0 || k >= s->n_models) return 0.0f;        // gpu_bpf.cu:1087-1090
  return (float)std::exp(s->log_pi[k]);
}

void gpu_imm_get_probs(const GpuImmState* s, float* probs_out) {
  if (!s || !probs_out) { bpf_record_error(BPF_ERR_ARG); return; }
  for (int k = 0; k < s->n_models; ++k) probs_out[k] = (float)std::exp(s->log_pi[k]);
}

ImmModelParams* gpu_imm_build_grid(const float* rhos, int n_rho, const float* sigma_zs, int n_sigma, const float* mus,
                                   int n_mu, float nu_state, float nu_obs, int* out_n_models) {
  if (!rhos || !sigma_zs || !mus || !out_n_models || n_rho <= 0 || n_sigma <= 0 || n_mu <= 0) {
    bpf_record_error(BPF_ERR_ARG);
    return nullptr;
  }
  const int total = n_rho * n_sigma * n_mu;                  // gpu_bpf.cu:1101-1121, rho-major order
  ImmModelParams* grid = (ImmModelParams*)malloc((size_t)total * sizeof(ImmModelParams));
  if (!grid) { bpf_record_error(BPF_ERR_ALLOC); return nullptr; }
  int idx = 0;
  for (int r = 0; r < n_rho; ++r)
    for (int q = 0; q < n_sigma; ++q)
      for (int u = 0; u < n_mu; ++u) {
        grid[idx].rho = rhos[r];
        grid[idx].sigma_z = sigma_zs[q];
        grid[idx].mu = mus[u];
        grid[idx].nu_state = nu_state;
        grid[idx].nu_obs = nu_obs;
        ++idx;
      }
  *out_n_models = total;
  return grid;
}

}  // extern "C"
