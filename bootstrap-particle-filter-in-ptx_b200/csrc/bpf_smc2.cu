// bpf_smc2.cu — SMC^2 (Chopin, Jacob & Papaspiliopoulos 2013) for the SV
// parameters theta = (mu, rho, sigma_z), with the batched bootstrap filter as
// the inner filter: the outer loop of the reference's smc2_cuda_update
// (smc2/smc2_rbpf_batch.cu:1329-1502; host API smc2/smc2_rbpf_batch.cuh:461-489)
// on this build's plain SV model.
//
// Per observation: every theta-particle's inner filter advances one tick (one
// graph launch of the resumable batch for all of them) and its outer
// log-weight gains the tick's log-likelihood increment. When the outer ESS
// falls below the threshold, the theta-particles are resampled (systematic;
// the copies' filter states are gathered on the device and given fresh seeds,
// so duplicates do not share future noise) and rejuvenated by particle
// marginal Metropolis-Hastings moves (Andrieu, Doucet & Holenstein 2010):
// random-walk proposals with the scaled empirical covariance of the
// theta-particles, each scored by a fresh inner filter run over the whole
// history (a second batch, one launch), accepted with probability
// min(1, p^(y|theta') p(theta') / p^(y|theta) p(theta)); accepted proposals'
// filter states are gathered into the current batch.
//
// Correlated-noise moves (CPMMH, Deligiannidis, Doucet & Pitt 2018; the
// reference's kernel_cpmmh_rejuvenate_fused, smc2/smc2_rbpf_batch.cu:651-935):
// with cpmmh_rho > 0 every theta-particle's auxiliary noise (its inner filter's
// normals and resampling normals, gpu_bpf_batch_run_correlated's layout) is
// kept on the device in one of two areas; par[j] names theta-particle j's
// current area. The forward ticks record into the current area, a proposal is
// scored with noise rho * current + sqrt(1 - rho^2) * fresh written into the
// other area, and acceptance flips par[j] (no copy; the reference copies the
// accepted noise back, kernel_commit_accepted_noise :959-985). Outer
// resampling copies the ancestors' areas into the other areas and flips every
// par[j]. The reference's regime-switching RBPF inner model is not part of
// this driver.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bpf_batch_internal.cuh"

namespace {

// Host PCG32 (O'Neill 2014) for the driver's own draws: prior, resampling
// uniform, proposals, acceptance uniforms.
struct HostPcg {
  uint64_t s = 0, inc = 1;
  void seed(uint64_t sd, uint64_t stream) {
    inc = (stream << 1) | 1ull;
    s = 0;
    next();
    s += sd;
    next();
  }
  uint32_t next() {
    const uint64_t old = s;
    s = old * kPcgMult + inc;
    const uint32_t xs = (uint32_t)(((old >> 18) ^ old) >> 27), rot = (uint32_t)(old >> 59);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
  }
  double uniform() {   // 53 bits: the first draw's top 27, then the second's top 26
    const uint32_t a = next() >> 5;
    const uint32_t b = next() >> 6;
    return ((double)a * 67108864.0 + (double)b + 0.5) / 9007199254740992.0;
  }
  double normal() {   // Box-Muller
    const double u1 = uniform(), u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925286766559 * u2);
  }
};

struct Theta { double mu, rho, sigma; };

}  // namespace

struct GpuBpfSmc2 {
  int n_theta = 0, n = 0, max_ticks = 0, t = 0;
  BpfSmc2Prior prior{};
  int n_moves = 1;
  float ess_frac = 0.5f;
  float scale = 1.0f;
  GpuBpfBatch* cur = nullptr;
  GpuBpfBatch* prop = nullptr;
  cudaStream_t stream = nullptr;
  float* d_y = nullptr;
  float* y_pin = nullptr;
  double* d_dll = nullptr;                 // device view of dll_pin (host-mapped): the forward tick's increments
  double* dll_pin = nullptr;
  int* d_idx = nullptr;
  int* d_mask = nullptr;
  int* d_seed = nullptr;
  int* i_pin = nullptr;                    // staging for idx / mask / seeds
  BatchFilterState* st_pin = nullptr;
  double* ll_pin = nullptr;
  // scratch filter states for the outer resampling gather
  BatchFilterDev* s_tab = nullptr;
  BatchFilterState* s_st = nullptr;
  float* s_h = nullptr;
  float* s_w = nullptr;
  std::vector<Theta> theta;
  std::vector<double> logw;
  HostPcg rng;
  int next_seed = 0;
  int n_rejuv = 0;
  long long n_prop = 0, n_acc = 0;
  float last_ess = 0.0f;
  // correlated-noise moves
  float cp_rho = 0.0f;
  float* d_nz = nullptr;               // 2 areas per theta-particle, each `area` floats
  long long area = 0;
  long long* d_off_cur = nullptr;      // [M] current areas
  long long* d_off_oth = nullptr;      // [M] the other areas
  long long* d_off_src = nullptr;      // [M] outer resampling: the ancestors' current areas
  long long* off_pin = nullptr;        // [3M] staging
  std::vector<int> par;
  // the last update: forward increments, whether it resampled, the outer ancestors
  bool have_update = false;
  std::vector<double> lu_dll;
  std::vector<int> lu_idx;
  int lu_res = 0;
  // the last PMMH move
  bool have_move = false;
  std::vector<float> lm_theta_prop, lm_theta_cur;
  std::vector<double> lm_ll_prop, lm_ll_cur;
  std::vector<int> lm_acc;
};

namespace {

double log_prior(const BpfSmc2Prior& p, const Theta& th) {
  if (!(th.rho > p.rho_lo && th.rho < p.rho_hi && th.sigma > p.sigma_lo && th.sigma < p.sigma_hi)) return -INFINITY;
  const double z = (th.mu - p.mu_mean) / p.mu_sd;
  return -0.5 * z * z - std::log((double)p.mu_sd) - std::log((double)(p.rho_hi - p.rho_lo)) -
         std::log((double)(p.sigma_hi - p.sigma_lo)) - 0.918938533204672741780329736406;
}

BpfBatchFilter filter_of(const Theta& th, int n, int seed) {
  BpfBatchFilter f{};
  f.mu = (float)th.mu; f.rho = (float)th.rho; f.sigma_z = (float)th.sigma;
  f.nu_obs = 0.0f; f.nu_state = 0.0f;
  f.n_particles = n;
  f.seed = seed;
  return f;
}

void free_smc2(GpuBpfSmc2* s) {
  if (!s) return;
  if (s->cur) gpu_bpf_batch_destroy(s->cur);
  if (s->prop) gpu_bpf_batch_destroy(s->prop);
  bpf_free(s->d_y); bpf_free(s->d_idx); bpf_free(s->d_mask); bpf_free(s->d_seed);
  bpf_free(s->s_tab); bpf_free(s->s_st); bpf_free(s->s_h); bpf_free(s->s_w);
  bpf_free_host(s->y_pin); bpf_free_host(s->dll_pin); bpf_free_host(s->i_pin); bpf_free_host(s->st_pin);
  bpf_free_host(s->ll_pin);
  bpf_free(s->d_nz); bpf_free(s->d_off_cur); bpf_free(s->d_off_oth); bpf_free(s->d_off_src);
  bpf_free_host(s->off_pin);
  delete s;
}

double outer_ess(const std::vector<double>& lw) {
  double m = -INFINITY;
  for (double v : lw) m = std::fmax(m, v);
  double a = 0.0, b = 0.0;
  for (double v : lw) { const double e = std::exp(v - m); a += e; b += e * e; }
  return a * a / b;
}

// Uploads the current / other area offsets of par[] (and waits: off_pin is reused).
int upload_noise_offsets(GpuBpfSmc2* s) {
  const int M = s->n_theta;
  for (int j = 0; j < M; ++j) {
    s->off_pin[j] = (2LL * j + s->par[j]) * s->area;
    s->off_pin[M + j] = (2LL * j + 1 - s->par[j]) * s->area;
  }
  BCK(cudaMemcpyAsync(s->d_off_cur, s->off_pin, M * sizeof(long long), cudaMemcpyHostToDevice, s->stream));
  BCK(cudaMemcpyAsync(s->d_off_oth, s->off_pin + M, M * sizeof(long long), cudaMemcpyHostToDevice, s->stream));
  BCK(cudaStreamSynchronize(s->stream));
  return BPF_OK;
}

// Outer systematic resampling and PMMH rejuvenation at tick count s->t + 1.
int resample_move(GpuBpfSmc2* s) {
  const int M = s->n_theta, T = s->t + 1;
  GpuBpfBatch* cur = s->cur;
  // a. systematic resampling of the theta-particles
  double m = -INFINITY;
  for (double v : s->logw) m = std::fmax(m, v);
  std::vector<double> cdf(M);
  double acc = 0.0;
  for (int j = 0; j < M; ++j) { acc += std::exp(s->logw[j] - m); cdf[j] = acc; }
  const double u0 = s->rng.uniform();
  int k = 0;
  std::vector<int> idx(M);
  for (int j = 0; j < M; ++j) {
    const double tgt = (u0 + j) / M * acc;
    while (k < M - 1 && cdf[k] <= tgt) ++k;
    idx[j] = k;
  }
  s->lu_idx = idx;
  for (int j = 0; j < M; ++j) s->i_pin[j] = idx[j];
  for (int j = 0; j < M; ++j) s->i_pin[M + j] = s->next_seed++;
  BCK(cudaMemcpyAsync(s->d_idx, s->i_pin, M * sizeof(int), cudaMemcpyHostToDevice, s->stream));
  BCK(cudaMemcpyAsync(s->d_seed, s->i_pin + M, M * sizeof(int), cudaMemcpyHostToDevice, s->stream));
  BCK(launch_batch_gather(s->s_tab, s->s_st, s->s_h, s->s_w, cur->d_filters, cur->d_st, cur->d_sth, cur->d_stw,
                          cur->d_stoff, s->d_idx, nullptr, s->d_seed, s->n, M, s->stream));
  const size_t nh = (size_t)M * ((s->n + 3) & ~3);
  BCK(cudaMemcpyAsync(cur->d_filters, s->s_tab, M * sizeof(BatchFilterDev), cudaMemcpyDeviceToDevice, s->stream));
  BCK(cudaMemcpyAsync(cur->d_st, s->s_st, M * sizeof(BatchFilterState), cudaMemcpyDeviceToDevice, s->stream));
  BCK(cudaMemcpyAsync(cur->d_sth, s->s_h, nh * sizeof(float), cudaMemcpyDeviceToDevice, s->stream));
  BCK(cudaMemcpyAsync(cur->d_stw, s->s_w, nh * sizeof(float), cudaMemcpyDeviceToDevice, s->stream));
  const bool cp = s->cp_rho > 0.0f;
  const long long used = (long long)T * batch_noise_stride(s->n);   // floats of ticks 0..T-1
  if (cp) {
    // the copies take their ancestors' noise (into their other areas), then those become current
    for (int j = 0; j < M; ++j) s->off_pin[2 * M + j] = (2LL * idx[j] + s->par[idx[j]]) * s->area;
    BCK(cudaMemcpyAsync(s->d_off_src, s->off_pin + 2 * M, M * sizeof(long long), cudaMemcpyHostToDevice, s->stream));
    BCK(launch_noise_gather(s->d_nz, s->d_off_src, s->d_off_oth, used, M, s->stream));
    for (int j = 0; j < M; ++j) s->par[j] ^= 1;
    const int rc = upload_noise_offsets(s);
    if (rc) return rc;
  }
  std::vector<Theta> th(M);
  for (int j = 0; j < M; ++j) th[j] = s->theta[idx[j]];
  s->theta = th;
  std::fill(s->logw.begin(), s->logw.end(), 0.0);
  ++s->n_rejuv;

  // b. PMMH moves
  const double c = s->scale * 2.38 * 2.38 / 3.0;
  for (int mv = 0; mv < s->n_moves; ++mv) {
    double mean[3] = {0, 0, 0}, cov[3][3] = {{0}};
    for (const Theta& q : s->theta) { mean[0] += q.mu; mean[1] += q.rho; mean[2] += q.sigma; }
    for (double& v : mean) v /= M;
    for (const Theta& q : s->theta) {
      const double d[3] = {q.mu - mean[0], q.rho - mean[1], q.sigma - mean[2]};
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) cov[a][b] += d[a] * d[b] / M;
    }
    double L[3][3] = {{0}};
    for (int a = 0; a < 3; ++a) {                         // Cholesky of c * cov + jitter
      for (int b = 0; b <= a; ++b) {
        double v = c * cov[a][b] + (a == b ? 1e-10 : 0.0);
        for (int q = 0; q < b; ++q) v -= L[a][q] * L[b][q];
        L[a][b] = (a == b) ? std::sqrt(std::fmax(v, 1e-12)) : v / L[b][b];
      }
    }
    std::vector<Theta> pr(M);
    std::vector<double> lp(M), lpn(M);
    std::vector<BpfBatchFilter> fl(M);
    std::vector<int> pseed(M);
    for (int j = 0; j < M; ++j) {
      const double z[3] = {s->rng.normal(), s->rng.normal(), s->rng.normal()};
      const double d0 = L[0][0] * z[0], d1 = L[1][0] * z[0] + L[1][1] * z[1],
                   d2 = L[2][0] * z[0] + L[2][1] * z[1] + L[2][2] * z[2];
      pr[j] = Theta{s->theta[j].mu + d0, s->theta[j].rho + d1, s->theta[j].sigma + d2};
      lp[j] = log_prior(s->prior, s->theta[j]);
      lpn[j] = log_prior(s->prior, pr[j]);
      pseed[j] = s->next_seed++;
      // outside the prior's support: score the current theta instead (the move is rejected)
      fl[j] = filter_of(std::isfinite(lpn[j]) ? pr[j] : s->theta[j], s->n, pseed[j]);
    }
    int rc = batch_set_filters(s->prop, fl.data());
    if (rc) return rc;
    if (cp) {
      NoiseArgs nz;
      nz.in = s->d_nz;
      nz.out = s->d_nz;
      nz.in_off = s->d_off_cur;
      nz.out_off = s->d_off_oth;
      nz.rho = s->cp_rho;
      nz.scale = sqrtf(fmaxf(0.0f, 1.0f - s->cp_rho * s->cp_rho));
      s->prop->step_nz = nz;
    } else {
      s->prop->step_nz = NoiseArgs{};
    }
    rc = batch_set_tick(s->prop, 0);
    if (rc) return rc;
    rc = batch_step_abs(s->prop, s->d_y, T, nullptr);
    if (rc) return rc;
    BCK(cudaMemcpyAsync(s->ll_pin, s->prop->d_loglik, M * sizeof(double), cudaMemcpyDeviceToHost, s->prop->stream));
    BCK(cudaStreamSynchronize(s->prop->stream));
    BCK(cudaMemcpyAsync(s->st_pin, cur->d_st, M * sizeof(BatchFilterState), cudaMemcpyDeviceToHost, s->stream));
    BCK(cudaStreamSynchronize(s->stream));
    s->lm_theta_prop.resize(3 * M); s->lm_theta_cur.resize(3 * M);
    s->lm_ll_prop.resize(M); s->lm_ll_cur.resize(M); s->lm_acc.resize(M);
    for (int j = 0; j < M; ++j) {
      const double la = s->ll_pin[j] + lpn[j] - s->st_pin[j].ll_total - lp[j];
      const bool ok = std::isfinite(lpn[j]) && std::isfinite(s->ll_pin[j]) && std::log(s->rng.uniform()) < la;
      s->i_pin[j] = ok ? 1 : 0;
      s->lm_theta_prop[3 * j] = fl[j].mu; s->lm_theta_prop[3 * j + 1] = fl[j].rho; s->lm_theta_prop[3 * j + 2] = fl[j].sigma_z;
      s->lm_theta_cur[3 * j] = (float)s->theta[j].mu; s->lm_theta_cur[3 * j + 1] = (float)s->theta[j].rho;
      s->lm_theta_cur[3 * j + 2] = (float)s->theta[j].sigma;
      s->lm_ll_prop[j] = s->ll_pin[j]; s->lm_ll_cur[j] = s->st_pin[j].ll_total; s->lm_acc[j] = ok ? 1 : 0;
      if (ok) {
        s->theta[j] = pr[j]; ++s->n_acc;
        if (cp) s->par[j] ^= 1;                             // the proposal's noise becomes current
      }
      ++s->n_prop;
    }
    s->have_move = true;
    BCK(cudaMemcpyAsync(s->d_mask, s->i_pin, M * sizeof(int), cudaMemcpyHostToDevice, s->stream));
    BCK(launch_batch_gather(cur->d_filters, cur->d_st, cur->d_sth, cur->d_stw, s->prop->d_filters, s->prop->d_st,
                            s->prop->d_sth, s->prop->d_stw, cur->d_stoff, nullptr, s->d_mask, nullptr, s->n, M,
                            s->stream));
    BCK(cudaStreamSynchronize(s->stream));
    if (cp) {
      rc = upload_noise_offsets(s);
      if (rc) return rc;
    }
  }
  return BPF_OK;
}

}  // namespace

extern "C" {

GpuBpfSmc2* gpu_bpf_smc2_create(int n_theta, int n_particles, int max_ticks, const BpfSmc2Prior* prior,
                                unsigned long long seed) {
  BpfSmc2Prior p{-1.0f, 0.5f, 0.85f, 0.995f, 0.05f, 0.4f};
  if (prior) p = *prior;
  if (n_theta < 2 || n_particles <= 0 || n_particles > kBatchMaxN || max_ticks <= 0 || !(p.mu_sd > 0.0f) ||
      !(p.rho_lo < p.rho_hi) || !(p.rho_lo > -1.0f) || !(p.rho_hi < 1.0f) || !(p.sigma_lo < p.sigma_hi) ||
      !(p.sigma_lo >= 0.0f)) {
    bpf_record_error(BPF_ERR_ARG);
    return nullptr;
  }
  GpuBpfSmc2* s = new GpuBpfSmc2();
  s->n_theta = n_theta; s->n = n_particles; s->max_ticks = max_ticks; s->prior = p;
  s->rng.seed(seed, 0x5eedull);
  s->next_seed = (int)(seed & 0x3fffffffull) + 1;
  s->theta.resize(n_theta);
  s->logw.assign(n_theta, 0.0);
  std::vector<BpfBatchFilter> fl(n_theta);
  for (int j = 0; j < n_theta; ++j) {                     // draws from the prior
    Theta th;
    th.mu = p.mu_mean + p.mu_sd * s->rng.normal();
    th.rho = p.rho_lo + (p.rho_hi - p.rho_lo) * s->rng.uniform();
    th.sigma = p.sigma_lo + (p.sigma_hi - p.sigma_lo) * s->rng.uniform();
    s->theta[j] = th;
    fl[j] = filter_of(th, n_particles, s->next_seed++);
  }
  auto fail = [&](int code) -> GpuBpfSmc2* { free_smc2(s); bpf_record_error(code); return nullptr; };
  s->cur = gpu_bpf_batch_create(fl.data(), n_theta, 0.5f);
  if (!s->cur) return fail(gpu_bpf_last_error());
  s->prop = gpu_bpf_batch_create(fl.data(), n_theta, 0.5f);
  if (!s->prop) return fail(gpu_bpf_last_error());
  if (batch_prepare_steps(s->cur) || batch_prepare_steps(s->prop)) return fail(gpu_bpf_last_error());
  s->stream = s->cur->stream;
  const size_t nh = (size_t)n_theta * ((n_particles + 3) & ~3);
  cudaError_t e = cudaSuccess;
  auto al = [&](auto** ptr, size_t bytes) { if (e == cudaSuccess) e = bpf_malloc(ptr, bytes); };
  auto ah = [&](auto** ptr, size_t bytes) { if (e == cudaSuccess) e = bpf_malloc_host(ptr, bytes); };
  al(&s->d_y, (size_t)max_ticks * sizeof(float));
  al(&s->d_idx, n_theta * sizeof(int));
  al(&s->d_mask, n_theta * sizeof(int));
  al(&s->d_seed, n_theta * sizeof(int));
  al(&s->s_tab, n_theta * sizeof(BatchFilterDev));
  al(&s->s_st, n_theta * sizeof(BatchFilterState));
  al(&s->s_h, nh * sizeof(float));
  al(&s->s_w, nh * sizeof(float));
  ah(&s->y_pin, sizeof(float));
  if (e == cudaSuccess) e = bpf_host_alloc(&s->dll_pin, n_theta * sizeof(double), cudaHostAllocMapped);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->d_dll), s->dll_pin, 0);
  ah(&s->i_pin, 2 * n_theta * sizeof(int));
  ah(&s->st_pin, n_theta * sizeof(BatchFilterState));
  ah(&s->ll_pin, n_theta * sizeof(double));
  if (e != cudaSuccess) { cudaGetLastError(); return fail(BPF_ERR_ALLOC); }
  s->last_ess = (float)n_theta;
  return s;
}

void gpu_bpf_smc2_destroy(GpuBpfSmc2* s) {
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  free_smc2(s);
}

int gpu_bpf_smc2_set_moves(GpuBpfSmc2* s, int n_moves, float outer_ess_threshold, float proposal_scale) {
  if (!s) return bpf_record_error(BPF_ERR_STATE);
  if (n_moves < 0 || !(outer_ess_threshold >= 0.0f && outer_ess_threshold <= 1.0f) || !(proposal_scale > 0.0f))
    return bpf_record_error(BPF_ERR_ARG);
  s->n_moves = n_moves;
  s->ess_frac = outer_ess_threshold;
  s->scale = proposal_scale;
  return BPF_OK;
}

float gpu_bpf_smc2_update(GpuBpfSmc2* s, float y) {
  if (!s) { bpf_record_error(BPF_ERR_STATE); return NAN; }
  if (!std::isfinite(y)) { bpf_record_error(BPF_ERR_ARG); return NAN; }
  if (s->t >= s->max_ticks) { bpf_record_error(BPF_ERR_ARG); return NAN; }
  int cur_dev = -1;
  if (cudaGetDevice(&cur_dev) != cudaSuccess || (cur_dev != s->cur->device && cudaSetDevice(s->cur->device) != cudaSuccess)) {
    bpf_record_error(BPF_ERR_CUDA);
    return NAN;
  }
  *s->y_pin = y;
  if (cudaMemcpyAsync(s->d_y + s->t, s->y_pin, sizeof(float), cudaMemcpyHostToDevice, s->stream) != cudaSuccess) {
    bpf_record_error(BPF_ERR_CUDA);
    return NAN;
  }
  if (batch_step_abs(s->cur, s->d_y, 1, s->d_dll) != BPF_OK) return NAN;
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) {
    cudaGetLastError();
    bpf_record_error(BPF_ERR_CUDA);
    return NAN;
  }
  for (int j = 0; j < s->n_theta; ++j) s->logw[j] += s->dll_pin[j];
  s->lu_dll.assign(s->dll_pin, s->dll_pin + s->n_theta);
  s->lu_res = 0;
  s->have_update = true;
  double ess = outer_ess(s->logw);
  if (ess < (double)s->ess_frac * s->n_theta) {
    s->lu_res = 1;
    if (resample_move(s) != BPF_OK) return NAN;
    ess = (double)s->n_theta;
  }
  s->t += 1;
  s->last_ess = (float)ess;
  return s->last_ess;
}

float gpu_bpf_smc2_get_outer_ess(GpuBpfSmc2* s) {
  if (!s) { bpf_record_error(BPF_ERR_STATE); return NAN; }
  return s->last_ess;
}

int gpu_bpf_smc2_get_theta(GpuBpfSmc2* s, float* mean, float* sd) {
  if (!s) return bpf_record_error(BPF_ERR_STATE);
  double m = -INFINITY;
  for (double v : s->logw) m = std::fmax(m, v);
  double wsum = 0.0, mu[3] = {0, 0, 0}, m2[3] = {0, 0, 0};
  for (int j = 0; j < s->n_theta; ++j) {
    const double w = std::exp(s->logw[j] - m);
    const double v[3] = {s->theta[j].mu, s->theta[j].rho, s->theta[j].sigma};
    wsum += w;
    for (int a = 0; a < 3; ++a) { mu[a] += w * v[a]; m2[a] += w * v[a] * v[a]; }
  }
  for (int a = 0; a < 3; ++a) {
    const double mean_a = mu[a] / wsum;
    if (mean) mean[a] = (float)mean_a;
    if (sd) sd[a] = (float)std::sqrt(std::fmax(m2[a] / wsum - mean_a * mean_a, 0.0));
  }
  return BPF_OK;
}

int gpu_bpf_smc2_get_particles(GpuBpfSmc2* s, float* theta, double* logw, double* loglik) {
  if (!s) return bpf_record_error(BPF_ERR_STATE);
  for (int j = 0; j < s->n_theta; ++j) {
    if (theta) { theta[3 * j] = (float)s->theta[j].mu; theta[3 * j + 1] = (float)s->theta[j].rho; theta[3 * j + 2] = (float)s->theta[j].sigma; }
    if (logw) logw[j] = s->logw[j];
  }
  if (loglik) {
    if (cudaMemcpyAsync(s->st_pin, s->cur->d_st, s->n_theta * sizeof(BatchFilterState), cudaMemcpyDeviceToHost,
                        s->stream) != cudaSuccess ||
        cudaStreamSynchronize(s->stream) != cudaSuccess) {
      cudaGetLastError();
      return bpf_record_error(BPF_ERR_CUDA);
    }
    for (int j = 0; j < s->n_theta; ++j) loglik[j] = s->st_pin[j].ll_total;
  }
  return BPF_OK;
}

int gpu_bpf_smc2_set_cpmmh_rho(GpuBpfSmc2* s, float rho) {
  if (!s) return bpf_record_error(BPF_ERR_STATE);
  if (!(rho >= 0.0f && rho <= 1.0f)) return bpf_record_error(BPF_ERR_ARG);
  const bool on = rho > 0.0f;
  if (on != (s->cp_rho > 0.0f) && s->t > 0) return bpf_record_error(BPF_ERR_STATE);
  if (on && s->n > kTile) return bpf_record_error(BPF_ERR_UNSUPPORTED);
  int cur_dev = -1;
  if (cudaGetDevice(&cur_dev) != cudaSuccess || (cur_dev != s->cur->device && cudaSetDevice(s->cur->device) != cudaSuccess))
    return bpf_record_error(BPF_ERR_CUDA);
  const int M = s->n_theta;
  if (on && !s->d_nz) {
    s->area = (long long)s->max_ticks * batch_noise_stride(s->n);
    cudaError_t e = bpf_malloc(&s->d_nz, (size_t)(2LL * M * s->area) * sizeof(float));
    if (e == cudaSuccess) e = bpf_malloc(&s->d_off_cur, M * sizeof(long long));
    if (e == cudaSuccess) e = bpf_malloc(&s->d_off_oth, M * sizeof(long long));
    if (e == cudaSuccess) e = bpf_malloc(&s->d_off_src, M * sizeof(long long));
    if (e == cudaSuccess) e = bpf_malloc_host(&s->off_pin, 3 * M * sizeof(long long));
    if (e != cudaSuccess) {
      cudaGetLastError();
      bpf_free(s->d_nz); bpf_free(s->d_off_cur); bpf_free(s->d_off_oth); bpf_free(s->d_off_src);
      bpf_free_host(s->off_pin);
      s->d_nz = nullptr; s->d_off_cur = s->d_off_oth = s->d_off_src = nullptr; s->off_pin = nullptr;
      return bpf_record_error(BPF_ERR_ALLOC);
    }
    s->par.assign(M, 0);
    const int rc = upload_noise_offsets(s);
    if (rc) return rc;
  }
  s->cp_rho = rho;
  if (on) {
    NoiseArgs nz;                                            // forward ticks: fresh noise, recorded
    nz.out = s->d_nz;
    nz.out_off = s->d_off_cur;
    s->cur->step_nz = nz;
  } else {
    s->cur->step_nz = NoiseArgs{};
  }
  return BPF_OK;
}

int gpu_bpf_smc2_get_last_move(GpuBpfSmc2* s, float* theta_prop, float* theta_cur, double* loglik_prop,
                               double* loglik_cur, int* accepted) {
  if (!s || !s->have_move) return bpf_record_error(BPF_ERR_STATE);
  const int M = s->n_theta;
  if (theta_prop) std::copy(s->lm_theta_prop.begin(), s->lm_theta_prop.end(), theta_prop);
  if (theta_cur) std::copy(s->lm_theta_cur.begin(), s->lm_theta_cur.end(), theta_cur);
  if (loglik_prop) std::copy(s->lm_ll_prop.begin(), s->lm_ll_prop.begin() + M, loglik_prop);
  if (loglik_cur) std::copy(s->lm_ll_cur.begin(), s->lm_ll_cur.begin() + M, loglik_cur);
  if (accepted) std::copy(s->lm_acc.begin(), s->lm_acc.begin() + M, accepted);
  return BPF_OK;
}

int gpu_bpf_smc2_get_last_update(GpuBpfSmc2* s, double* dll, int* resampled, int* ancestors) {
  if (!s || !s->have_update) return bpf_record_error(BPF_ERR_STATE);
  const int M = s->n_theta;
  if (dll) std::copy(s->lu_dll.begin(), s->lu_dll.begin() + M, dll);
  if (resampled) *resampled = s->lu_res;
  if (ancestors && s->lu_res) std::copy(s->lu_idx.begin(), s->lu_idx.begin() + M, ancestors);
  return BPF_OK;
}

int gpu_bpf_smc2_get_noise(GpuBpfSmc2* s, int j, int n_ticks, float* out) {
  if (!s) return bpf_record_error(BPF_ERR_STATE);
  if (!(s->cp_rho > 0.0f) || !s->d_nz) return bpf_record_error(BPF_ERR_STATE);
  if (j < 0 || j >= s->n_theta || n_ticks <= 0 || n_ticks > s->t || !out) return bpf_record_error(BPF_ERR_ARG);
  int cur_dev = -1;
  if (cudaGetDevice(&cur_dev) != cudaSuccess || (cur_dev != s->cur->device && cudaSetDevice(s->cur->device) != cudaSuccess))
    return bpf_record_error(BPF_ERR_CUDA);
  if (cudaStreamSynchronize(s->stream) != cudaSuccess ||
      cudaMemcpy(out, s->d_nz + (2LL * j + s->par[j]) * s->area,
                 (size_t)n_ticks * batch_noise_stride(s->n) * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return bpf_record_error(BPF_ERR_CUDA);
  }
  return BPF_OK;
}

int gpu_bpf_smc2_stats(GpuBpfSmc2* s, int* n_rejuvenations, long long* n_proposed, long long* n_accepted) {
  if (!s) return bpf_record_error(BPF_ERR_STATE);
  if (n_rejuvenations) *n_rejuvenations = s->n_rejuv;
  if (n_proposed) *n_proposed = s->n_prop;
  if (n_accepted) *n_accepted = s->n_acc;
  return BPF_OK;
}

}  // extern "C"
