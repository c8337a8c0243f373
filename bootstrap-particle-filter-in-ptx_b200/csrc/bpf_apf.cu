// bpf_apf.cu — auxiliary particle filter: the reference's gpu_apf_* entry
// points (gpu_bpf/gpu_bpf.cuh:114-126; behaviour gpu_bpf/gpu_bpf_ptx_full.cu:
// 990-1190) on the plain filter's three kernels.
//
// The reference runs an APF tick as about 25 launches: first-stage weights,
// five normalisation passes, a thrust scan, a paired resample, propagate +
// correction weights, five more passes, a second scan and resample, with a
// host round trip. Here a tick is two passes of the plain tick machinery:
//   stage 1  pass 1 (APF=1): log2 v_i = log2 p(y | m_i), m_i = mu + rho (h_i - mu),
//            particles untouched; plan (always resample, tick not advanced);
//            pass 2 resamples the particles by v (the predicted means are not
//            stored: stage 2 recomputes m from the resampled parent with the
//            same operations, so no second array moves)
//   stage 2  pass 1 (APF=2): h_i = m_i + sigma eps_i,t, log2 w_i = log2 p(y | h_i) -
//            log2 p(y | m_i); plan (always resample; the record and the tick
//            advance); pass 2 resamples by w
// Tick 0 is a bootstrap tick (weights from h_0, resample), as in the reference.
// eps is draw t of slot i's PCG32 stream (Student-t scaled when nu_state > 0),
// where the reference draws cuRAND XORWOW states (apf_init_rng_k); both
// resampling uniforms come from the host-formula PCG32 stream, in the
// reference's order. BpfResult.log_lik is the reference's value, log mean w
// (the second-stage weights); BpfTickRecord.dloglik is the APF estimate of
// log p(y_t | y_{1:t-1}) = log mean v + log mean w, with its FP64 running sum.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "bpf_plain.cuh"

using namespace bpf;

namespace {

constexpr int kApfChunk = 64;   // ticks per captured graph in gpu_apf_step_many

inline int set_err(int code) { return bpf_record_error(code); }

#define ACK(call)                                                         \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) {                                              \
      if (e_ == cudaErrorMemoryAllocation) return set_err(BPF_ERR_ALLOC); \
      if (e_ == cudaErrorNoDevice || e_ == cudaErrorNoKernelImageForDevice || \
          e_ == cudaErrorInsufficientDriver) return set_err(BPF_ERR_NODEVICE); \
      return set_err(BPF_ERR_CUDA);                                       \
    }                                                                     \
  } while (0)

struct ApfImpl {
  int device = 0;
  Plan plan{};
  int pass2_grid = 0;
  cudaStream_t stream = nullptr;
  BpfTickRecord* rec_dev = nullptr;   // [1 + kApfChunk]: slot 0 single step, 1.. graph ticks
  BpfTickRecord* rec_pin = nullptr;
  DevState* st_pin = nullptr;
  float* y_dev = nullptr;             // [kApfChunk]
  float* y_pin = nullptr;
  int32_t* anc_dev = nullptr;         // when recording: first stage, then second stage at anc_stride
  bool record_anc = false;
  int ticks = 0;                      // ticks enqueued since create
  int sticky_error = BPF_OK;
  bool pdl = true;
  ObsModel obs{};
  cudaGraphExec_t graph = nullptr;    // kApfChunk ticks after tick 0, keyed by the baked arguments
  float g_mu = NAN, g_rho = NAN, g_sigma = NAN;
  bool g_anc = false;
};

inline ApfImpl* impl_of(GpuApfState* s) { return s ? reinterpret_cast<ApfImpl*>(s->impl) : nullptr; }

// Offset of the second stage's ancestors in anc_dev: N rounded up to 4 slots
// (16 bytes), so both halves start aligned.
inline size_t anc_stride(const ApfImpl* m) { return ((size_t)m->plan.N + 3) & ~(size_t)3; }

int ensure_device(ApfImpl* m) {
  int cur = -1;
  ACK(cudaGetDevice(&cur));
  if (cur != m->device) ACK(cudaSetDevice(m->device));
  return BPF_OK;
}

int check_params(const GpuApfState* s) {
  if (!std::isfinite(s->mu) || !std::isfinite(s->rho) || !std::isfinite(s->sigma_z)) return set_err(BPF_ERR_ARG);
  if (!(std::fabs(s->rho) < 1.0f) || !(s->sigma_z > 0.0f)) return set_err(BPF_ERR_ARG);
  return BPF_OK;
}

TickArgs make_args(const GpuApfState* s, const ApfImpl* m, float y, const float* y_ptr) {
  TickArgs a{};
  a.mu = s->mu; a.rho = s->rho; a.sigma = s->sigma_z;
  a.ess_threshold = 0.0f;                                             // both stages always resample
  a.log_n = std::log((double)m->plan.N);
  a.obs = m->obs;
  a.obs.y = y;
  a.y_ptr = y_ptr;
  a.nu_int = (s->nu_state > 0.0f) ? (int)(s->nu_state + 0.5f) : 0;
  a.nu_state = s->nu_state;
  return a;
}

cudaError_t launch3(ApfImpl* m, const TickArgs& a) {
  cudaError_t e = launch_pass1(m->plan, a, m->stream, m->pdl);
  if (e == cudaSuccess) e = launch_plan(m->plan, a, m->stream, m->pdl);
  if (e == cudaSuccess) e = launch_pass2(m->plan, a, m->pass2_grid, m->stream, m->pdl);
  return e;
}

// One APF tick (tick index `t` on the host): a bootstrap tick at t = 0, else
// the two stages. Returns the kernels launched, or -1 on a launch error.
int enqueue_tick(const GpuApfState* s, ApfImpl* m, int t, float y, const float* y_ptr, BpfTickRecord* rec) {
  TickArgs a = make_args(s, m, y, y_ptr);
  int32_t* anc2 = m->record_anc ? m->anc_dev + anc_stride(m) : nullptr;
  if (t == 0) {
    a.apf = 0; a.rec = rec; a.anc = anc2;
    return launch3(m, a) == cudaSuccess ? 3 : -1;
  }
  TickArgs a1 = a;
  a1.apf = 1; a1.rec = nullptr; a1.anc = m->record_anc ? m->anc_dev : nullptr;
  if (launch3(m, a1) != cudaSuccess) return -1;
  TickArgs a2 = a;
  a2.apf = 2; a2.rec = rec; a2.anc = anc2;
  return launch3(m, a2) == cudaSuccess ? 6 : -1;
}

int free_impl(ApfImpl* m) {
  if (!m) return BPF_OK;
  if (m->graph) cudaGraphExecDestroy(m->graph);
  plan_free(m->plan);
  bpf_free(m->rec_dev); bpf_free(m->y_dev); bpf_free(m->anc_dev);
  bpf_free_host(m->rec_pin); bpf_free_host(m->st_pin); bpf_free_host(m->y_pin);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return BPF_OK;
}

int create_impl(GpuApfState* s, ApfImpl* m, int seed) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return set_err(BPF_ERR_NODEVICE); }
  ACK(cudaGetDevice(&m->device));
  ACK(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  ACK(plan_alloc(m->plan, s->n_particles));
  ACK(bpf_malloc(&m->rec_dev, (1 + kApfChunk) * sizeof(BpfTickRecord)));
  ACK(bpf_malloc(&m->y_dev, kApfChunk * sizeof(float)));
  ACK(bpf_malloc_host(&m->rec_pin, (1 + kApfChunk) * sizeof(BpfTickRecord)));
  ACK(bpf_malloc_host(&m->st_pin, sizeof(DevState)));
  ACK(bpf_malloc_host(&m->y_pin, kApfChunk * sizeof(float)));
  ACK(cudaMemsetAsync(m->rec_dev, 0, (1 + kApfChunk) * sizeof(BpfTickRecord), m->stream));
  m->pass2_grid = pass2_grid_size(m->device);
  if (const char* v = std::getenv("BPF_DISABLE_PDL")) m->pdl = (v[0] == '0');
  const float nu_obs = s->nu_obs;
  m->obs.nu = nu_obs;
  if (nu_obs > 0.0f) {
    m->obs.c_obs = (float)(std::lgamma((nu_obs + 1.0) / 2.0) - std::lgamma(nu_obs / 2.0) -
                           0.5 * std::log(nu_obs * 3.14159265358979323846));
    m->obs.inv_nu = 1.0f / nu_obs;
    m->obs.nu_p1h = (nu_obs + 1.0f) * 0.5f;
  }
  const float std_stat = sqrtf((s->sigma_z * s->sigma_z) / fmaxf(1.0f - s->rho * s->rho, 1e-6f));
  ACK(launch_init(m->plan, s->mu, std_stat, seed, m->stream));
  bpf_note_launches(1);
  ACK(cudaStreamSynchronize(m->stream));
  s->stream = (void*)m->stream;
  return BPF_OK;
}

int build_graph(GpuApfState* s, ApfImpl* m) {
  if (m->graph) { cudaGraphExecDestroy(m->graph); m->graph = nullptr; }
  cudaGraph_t g = nullptr;
  ACK(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaMemcpyAsync(m->y_dev, m->y_pin, kApfChunk * sizeof(float), cudaMemcpyHostToDevice, m->stream);
  for (int k = 0; k < kApfChunk && err == cudaSuccess; ++k)
    if (enqueue_tick(s, m, 1, 0.0f, m->y_dev + k, m->rec_dev + 1 + k) < 0) err = cudaErrorLaunchFailure;
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(m->rec_pin + 1, m->rec_dev + 1, kApfChunk * sizeof(BpfTickRecord), cudaMemcpyDeviceToHost,
                          m->stream);
  cudaError_t e2 = cudaStreamEndCapture(m->stream, &g);
  if (err != cudaSuccess || e2 != cudaSuccess) { if (g) cudaGraphDestroy(g); cudaGetLastError(); return set_err(BPF_ERR_CUDA); }
  cudaError_t e3 = cudaGraphInstantiate(&m->graph, g, 0);
  cudaGraphDestroy(g);
  if (e3 != cudaSuccess) { m->graph = nullptr; return set_err(BPF_ERR_CUDA); }
  m->g_mu = s->mu; m->g_rho = s->rho; m->g_sigma = s->sigma_z; m->g_anc = m->record_anc;
  return BPF_OK;
}

bool graph_stale(const GpuApfState* s, const ApfImpl* m) {
  return !m->graph || m->g_mu != s->mu || m->g_rho != s->rho || m->g_sigma != s->sigma_z || m->g_anc != m->record_anc;
}

int sync_state(GpuApfState* s, ApfImpl* m) {
  ACK(cudaMemcpyAsync(m->st_pin, m->plan.st, sizeof(DevState), cudaMemcpyDeviceToHost, m->stream));
  ACK(cudaStreamSynchronize(m->stream));
  s->timestep = m->st_pin->tick;
  if (m->st_pin->error != BPF_OK) { m->sticky_error = m->st_pin->error; return set_err(m->st_pin->error); }
  return BPF_OK;
}

BpfResult to_result(const BpfTickRecord& r) {
  BpfResult o;
  o.h_mean = r.h_mean;
  o.log_lik = (float)r.loglik_ref;
  return o;
}

}  // namespace

extern "C" {

GpuApfState* gpu_apf_create(int n_particles, float rho, float sigma_z, float mu, float nu_state, float nu_obs,
                            int seed) {
  bpf_record_error(BPF_OK);
  if (n_particles <= 0 || n_particles > (1 << 30) || !std::isfinite(rho) || !std::isfinite(sigma_z) ||
      !std::isfinite(mu) || !(std::fabs(rho) < 1.0f) || !(sigma_z > 0.0f) || !(nu_obs >= 0.0f) ||
      !std::isfinite(nu_obs) || !(nu_state >= 0.0f) || (nu_state > 0.0f && nu_state < 0.5f) ||
      !std::isfinite(nu_state)) {
    set_err(BPF_ERR_ARG);
    return nullptr;
  }
  GpuApfState* s = (GpuApfState*)calloc(1, sizeof(GpuApfState));
  if (!s) { set_err(BPF_ERR_ALLOC); return nullptr; }
  s->n_particles = n_particles;
  s->rho = rho; s->sigma_z = sigma_z; s->mu = mu;
  s->nu_state = nu_state; s->nu_obs = nu_obs;
  ApfImpl* m = new ApfImpl();
  s->impl = m;
  const int rc = create_impl(s, m, seed);
  if (rc != BPF_OK) {
    free_impl(m);
    free(s);
    set_err(rc);
    return nullptr;
  }
  return s;
}

void gpu_apf_destroy(GpuApfState* s) {
  if (!s) return;
  ApfImpl* m = impl_of(s);
  if (m) { ensure_device(m); cudaStreamSynchronize(m->stream); free_impl(m); }
  s->impl = nullptr;
  free(s);
}

int gpu_apf_step_many(GpuApfState* s, const float* y, int n_ticks, BpfResult* out, BpfTickRecord* rec) {
  ApfImpl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  if (n_ticks < 0 || (n_ticks > 0 && !y)) return set_err(BPF_ERR_ARG);
  for (int t = 0; t < n_ticks; ++t) if (!std::isfinite(y[t])) return set_err(BPF_ERR_ARG);
  int rc = check_params(s);
  if (rc) return rc;
  rc = ensure_device(m);
  if (rc) return rc;
  int t = 0;
  while (t < n_ticks) {
    const int n = std::min(kApfChunk, n_ticks - t);
    if (n == kApfChunk && m->ticks > 0) {
      if (graph_stale(s, m)) { rc = build_graph(s, m); if (rc) return rc; }
      std::memcpy(m->y_pin, y + t, kApfChunk * sizeof(float));
      ACK(cudaGraphLaunch(m->graph, m->stream));
      bpf_note_launches(6LL * kApfChunk);
    } else {
      for (int k = 0; k < n; ++k) {
        const int launched = enqueue_tick(s, m, m->ticks + k, y[t + k], nullptr, m->rec_dev + 1 + k);
        if (launched < 0) return set_err(BPF_ERR_CUDA);
        bpf_note_launches(launched);
      }
      ACK(cudaMemcpyAsync(m->rec_pin + 1, m->rec_dev + 1, n * sizeof(BpfTickRecord), cudaMemcpyDeviceToHost,
                          m->stream));
    }
    ACK(cudaStreamSynchronize(m->stream));
    m->ticks += n;
    for (int k = 0; k < n; ++k) {
      if (out) out[t + k] = to_result(m->rec_pin[1 + k]);
      if (rec) rec[t + k] = m->rec_pin[1 + k];
    }
    // slot 0 keeps the last tick's record for gpu_apf_get_record
    ACK(cudaMemcpyAsync(m->rec_dev, m->rec_dev + n, sizeof(BpfTickRecord), cudaMemcpyDeviceToDevice, m->stream));
    t += n;
  }
  if (n_ticks > 0) return sync_state(s, m);
  return BPF_OK;
}

BpfResult gpu_apf_step(GpuApfState* s, float y_t) {
  BpfResult r;
  r.h_mean = NAN; r.log_lik = NAN;
  if (gpu_apf_step_many(s, &y_t, 1, &r, nullptr) != BPF_OK) {
    r.h_mean = NAN; r.log_lik = NAN;
  }
  return r;
}

int gpu_apf_get_record(GpuApfState* s, BpfTickRecord* out) {
  ApfImpl* m = impl_of(s);
  if (!m || !out) return set_err(!m ? BPF_ERR_STATE : BPF_ERR_ARG);
  if (m->ticks == 0) return set_err(BPF_ERR_STATE);
  int rc = ensure_device(m);
  if (rc) return rc;
  ACK(cudaMemcpyAsync(m->rec_pin, m->rec_dev, sizeof(BpfTickRecord), cudaMemcpyDeviceToHost, m->stream));
  ACK(cudaStreamSynchronize(m->stream));
  *out = m->rec_pin[0];
  return BPF_OK;
}

double gpu_apf_get_loglik_total(GpuApfState* s) {
  ApfImpl* m = impl_of(s);
  if (!m) { set_err(BPF_ERR_STATE); return NAN; }
  if (ensure_device(m)) return NAN;
  if (cudaMemcpyAsync(m->st_pin, m->plan.st, sizeof(DevState), cudaMemcpyDeviceToHost, m->stream) != cudaSuccess ||
      cudaStreamSynchronize(m->stream) != cudaSuccess) {
    set_err(BPF_ERR_CUDA);
    return NAN;
  }
  return m->st_pin->ll_total;
}

int gpu_apf_get_particles(GpuApfState* s, float* h_out) {
  ApfImpl* m = impl_of(s);
  if (!m || !h_out) return set_err(!m ? BPF_ERR_STATE : BPF_ERR_ARG);
  int rc = ensure_device(m);
  if (rc) return rc;
  ACK(cudaMemcpyAsync(m->st_pin, m->plan.st, sizeof(DevState), cudaMemcpyDeviceToHost, m->stream));
  ACK(cudaStreamSynchronize(m->stream));
  const float* src = m->st_pin->cur ? m->plan.h1 : m->plan.h0;
  ACK(cudaMemcpy(h_out, src, (size_t)m->plan.N * sizeof(float), cudaMemcpyDeviceToHost));
  return BPF_OK;
}

int gpu_apf_record_ancestors(GpuApfState* s, int enable) {
  ApfImpl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  int rc = ensure_device(m);
  if (rc) return rc;
  if (enable && !m->anc_dev) {
    ACK(bpf_malloc(&m->anc_dev, 2 * anc_stride(m) * sizeof(int32_t)));
    ACK(cudaMemsetAsync(m->anc_dev, 0xff, 2 * anc_stride(m) * sizeof(int32_t), m->stream));
  }
  m->record_anc = enable != 0;
  return BPF_OK;
}

int gpu_apf_get_ancestors(GpuApfState* s, int32_t* anc_first, int32_t* anc_second) {
  ApfImpl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  if (!m->anc_dev || m->ticks == 0) return set_err(BPF_ERR_STATE);
  int rc = ensure_device(m);
  if (rc) return rc;
  ACK(cudaStreamSynchronize(m->stream));
  const size_t n = (size_t)m->plan.N;
  if (anc_first) ACK(cudaMemcpy(anc_first, m->anc_dev, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (anc_second) ACK(cudaMemcpy(anc_second, m->anc_dev + anc_stride(m), n * sizeof(int32_t), cudaMemcpyDeviceToHost));
  return BPF_OK;
}

double gpu_apf_run_rmse(const double* returns, const double* true_h, int n_ticks, int n_particles, float rho,
                        float sigma_z, float mu, float nu_state, float nu_obs, int seed) {
  if (!returns || !true_h || n_ticks <= 100) { set_err(BPF_ERR_ARG); return NAN; }
  GpuApfState* f = gpu_apf_create(n_particles, rho, sigma_z, mu, nu_state, nu_obs, seed);
  if (!f) return NAN;
  float* y = (float*)malloc(sizeof(float) * n_ticks);
  BpfResult* out = (BpfResult*)malloc(sizeof(BpfResult) * n_ticks);
  int rc = (y && out) ? BPF_OK : BPF_ERR_ALLOC;
  if (rc == BPF_OK) {
    for (int t = 0; t < n_ticks; ++t) y[t] = (float)returns[t];
    rc = gpu_apf_step_many(f, y, n_ticks, out, nullptr);
  }
  double sse = 0.0;
  int count = 0;
  if (rc == BPF_OK)
    for (int t = 100; t < n_ticks; ++t) {            // gpu_bpf_ptx_full.cu:1183-1186
      const double e = (double)out[t].h_mean - true_h[t];
      sse += e * e;
      ++count;
    }
  free(y);
  free(out);
  gpu_apf_destroy(f);
  if (rc != BPF_OK) { set_err(rc); return NAN; }
  return std::sqrt(sse / (double)count);
}

}  // extern "C"
