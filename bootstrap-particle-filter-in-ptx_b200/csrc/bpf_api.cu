// bpf_api.cu — extern "C" entry points of libgpubpf.so (include/gpu_bpf.h).
//
// Host tick driver: replaces gpu_bpf/gpu_bpf_ptx_full.cu:340-864. Every tick
// is two stream-ordered launches (pass 1, pass 2); the resampling decision,
// the resampling uniform and the buffer swap live on the device, so a tick
// never waits for the host and runs of ticks are captured in CUDA graphs.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bpf_plain.cuh"

using namespace bpf;

// ---------------------------------------------------------------------------
// Status plumbing
// ---------------------------------------------------------------------------
static thread_local int g_last_error = BPF_OK;
static std::atomic<long long> g_launches{0};

static inline int set_err(int code) { g_last_error = code; return code; }

int bpf_record_error(int code) { return set_err(code); }
void bpf_note_launches(long long n) { g_launches += n; }

#define CK(call)                                                        \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess) {                                            \
      if (e_ == cudaErrorMemoryAllocation) return set_err(BPF_ERR_ALLOC); \
      if (e_ == cudaErrorNoDevice || e_ == cudaErrorNoKernelImageForDevice || \
          e_ == cudaErrorInsufficientDriver) return set_err(BPF_ERR_NODEVICE); \
      return set_err(BPF_ERR_CUDA);                                     \
    }                                                                   \
  } while (0)

namespace {

constexpr int kGraphChunk = 64;   // ticks per captured graph

struct Impl {
  int device = 0;
  int seed = 0;
  Plan plan{};
  int pass2_grid = 0;
  cudaStream_t stream = nullptr;

  BpfTickRecord* rec_dev = nullptr;     // [1 + kGraphChunk]: slot 0 single step, 1.. graph ticks
  BpfTickRecord* rec_pin = nullptr;     // pinned mirror
  DevState* st_pin = nullptr;           // pinned DevState snapshot
  // single ticks (gpu_bpf_step / step_async) write their record and outcome straight into
  // host-mapped memory, so reading the result back is one stream synchronise and no copy
  BpfTickRecord* rec_map = nullptr;     // host view
  BpfTickRecord* rec_map_dev = nullptr; // device view of the same memory
  TickMirror* mir_map = nullptr;
  TickMirror* mir_map_dev = nullptr;
  bool last_in_map = false;             // the last enqueued tick wrote rec_map (not rec_dev[0])
  int seq = 0;                          // request number of the last tick that writes the mirror
  float* y_dev = nullptr;               // [kGraphChunk]
  float* y_pin = nullptr;               // [kGraphChunk]
  int32_t* anc_dev = nullptr;           // [N] when recording
  bool record_anc = false;
  int ll_mode = 0;
  int ticks_enqueued = 0;
  int sticky_error = BPF_OK;

  // graph of kGraphChunk ticks, keyed by the launch arguments baked into it
  cudaGraphExec_t graph = nullptr;
  float g_mu = NAN, g_rho = NAN, g_sigma = NAN, g_thr = NAN, g_nus = NAN, g_silv = NAN;
  bool g_anc = false;

  // graph of one tick for single steps (gpu_bpf_step / step_async), keyed likewise: pass 1's
  // node gets the tick's observation by a parameter update of the instantiated graph, so a tick
  // is one graph launch instead of three kernel launches. t_g (the captured graph) stays alive
  // because the update names pass 1's node in it; t_params points at t_plan / t_args.
  cudaGraph_t t_g = nullptr;
  cudaGraphExec_t tgraph = nullptr;
  cudaGraphNode_t t_pass1 = nullptr;
  cudaKernelNodeParams t_params{};
  Plan t_plan{};
  TickArgs t_args{};
  int t_n = 1;                          // the fused kernel's tick count
  void* t_argv[3] = {nullptr, nullptr, nullptr};
  float t_mu = NAN, t_rho = NAN, t_sigma = NAN, t_thr = NAN, t_nus = NAN, t_silv = NAN;
  bool t_anc = false;

  // graph of a whole device-resident run (step_many_device), keyed likewise
  cudaGraphExec_t dgraph = nullptr;
  const float* dg_y = nullptr;
  BpfTickRecord* dg_rec = nullptr;
  int dg_n = 0;
  float dg_mu = NAN, dg_rho = NAN, dg_sigma = NAN, dg_thr = NAN, dg_nus = NAN, dg_silv = NAN;
  bool dg_anc = false;

  // programmatic dependent launch between consecutive kernels (off while profiling)
  bool pdl = true;

  // filters of at most kSmallMaxN particles run each tick (or each captured run of ticks) as one
  // fused launch (gpu_bpf_set_fused_small)
  bool fused_small = true;
  int small_tiles = 4;                  // largest fused cluster on the filter's device (tiles)

  // profiling
  bool profiling = false;

  // online mu / rho learning (gpu_bpf_ptx_full.cu:469-544, settings :363-371,777-800)
  int learn_mode = 0, learn_rho = 0, update_K = 50, grad_count = 0, rm_step = 0;
  float rm_c = 0.1f, rm_t0 = 10.0f, rm_gamma = 0.667f, grad_clip = 5.0f;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<cudaEvent_t> ev_pending;   // quadruples: before pass 1, after pass 1, after plan, after pass 2
  double prof_p1_ms = 0.0, prof_plan_ms = 0.0, prof_p2_ms = 0.0;
  int prof_n1 = 0, prof_n2 = 0;

  ObsModel obs{};
};

inline Impl* impl_of(GpuBpfState* s) { return s ? reinterpret_cast<Impl*>(s->impl) : nullptr; }

int ensure_device(Impl* m) {
  int cur = -1;
  CK(cudaGetDevice(&cur));
  if (cur != m->device) CK(cudaSetDevice(m->device));
  return BPF_OK;
}

// A tick runs as the fused small-filter kernel when the filter is small enough and the tick
// needs nothing that only the three-kernel path provides (learning, Silverman jitter, per-kernel
// profiling); the two give bit-identical results.
bool use_small(const Impl* m, const TickArgs& a) {
  return m->fused_small && !m->profiling && m->plan.G <= m->small_tiles && small_eligible(m->plan, a);
}

// Filters of at most kTailTiles tiles run the plan in pass 1's last CTA instead of a plan
// launch (the same results; per-kernel profiling keeps the separate plan kernel).
bool use_tail(const Impl* m, const TickArgs& a) {
  return !m->profiling && tail_plan_eligible(m->plan, a);
}

// Kernels one tick launches: the fused kernel alone, or pass 1, the plan (unless pass 1 runs
// it), pass 2 and the two Silverman jitter kernels when on.
int tick_launches(const Impl* m, const TickArgs& a) {
  if (use_small(m, a)) return 1;
  return (use_tail(m, a) ? 2 : 3) + (a.silverman > 0.0f ? 2 : 0);
}

cudaError_t launch_tick3(Impl* m, const TickArgs& a) {
  if (use_small(m, a)) return launch_small(m->plan, a, 1, m->stream, m->pdl);
  TickArgs at = a;
  at.tail_plan = use_tail(m, a) ? 1 : 0;
  cudaError_t e = launch_pass1(m->plan, at, m->stream, m->pdl);
  if (e == cudaSuccess && !at.tail_plan) e = launch_plan(m->plan, at, m->stream, m->pdl);
  if (e == cudaSuccess) e = launch_pass2(m->plan, at, m->pass2_grid, m->stream, m->pdl);
  if (e == cudaSuccess && a.silverman > 0.0f) e = launch_jitter(m->plan, at, m->stream, m->pdl);
  return e;
}

TickArgs make_args(GpuBpfState* s, Impl* m, float y, const float* y_ptr, BpfTickRecord* rec) {
  TickArgs a{};
  a.mu = s->mu; a.rho = s->rho; a.sigma = s->sigma_z;
  a.ess_threshold = s->ess_threshold;
  a.log_n = std::log((double)m->plan.N);
  a.obs = m->obs;
  a.obs.y = y;
  a.y_ptr = y_ptr;
  a.rec = rec;
  a.anc = m->record_anc ? m->anc_dev : nullptr;
  a.nu_int = (s->nu_state > 0.0f) ? (int)(s->nu_state + 0.5f) : 0;   // gpu_bpf_ptx_full.cu:392
  a.nu_state = s->nu_state;
  a.learn = m->learn_mode ? 1 : 0;
  a.silverman = s->silverman_shrink > 0.0f ? s->silverman_shrink : 0.0f;   // gpu_bpf_ptx_full.cu:709
  return a;
}

int check_options(GpuBpfState* s) {
  if (!std::isfinite(s->mu) || !std::isfinite(s->rho) || !std::isfinite(s->sigma_z)) return set_err(BPF_ERR_ARG);
  if (!(std::fabs(s->rho) < 1.0f) || !(s->sigma_z > 0.0f)) return set_err(BPF_ERR_ARG);
  if (!std::isfinite(s->silverman_shrink)) return set_err(BPF_ERR_ARG);
  if (!(s->nu_state == 0.0f || (s->nu_state >= 0.5f && std::isfinite(s->nu_state)))) return set_err(BPF_ERR_ARG);
  if (std::isnan(s->ess_threshold)) return set_err(BPF_ERR_ARG);
  return BPF_OK;
}

cudaEvent_t take_event(Impl* m) {
  if (!m->ev_pool.empty()) { cudaEvent_t e = m->ev_pool.back(); m->ev_pool.pop_back(); return e; }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

int drain_profile(Impl* m) {
  for (size_t i = 0; i + 3 < m->ev_pending.size(); i += 4) {
    float a = 0.f, b = 0.f, c = 0.f;
    CK(cudaEventSynchronize(m->ev_pending[i + 3]));
    CK(cudaEventElapsedTime(&a, m->ev_pending[i], m->ev_pending[i + 1]));
    CK(cudaEventElapsedTime(&b, m->ev_pending[i + 1], m->ev_pending[i + 2]));
    CK(cudaEventElapsedTime(&c, m->ev_pending[i + 2], m->ev_pending[i + 3]));
    m->prof_p1_ms += a; m->prof_plan_ms += b; m->prof_p2_ms += c;
    m->prof_n1 += 1; m->prof_n2 += 1;
  }
  for (cudaEvent_t e : m->ev_pending) m->ev_pool.push_back(e);
  m->ev_pending.clear();
  return BPF_OK;
}

int zero_learning_sums(Impl* m) {
  CK(cudaMemsetAsync(&m->plan.st->learn[0], 0, sizeof(m->plan.st->learn), m->stream));
  return BPF_OK;
}

// Robbins-Monro natural-gradient step on alpha = mu (1 - rho) and on rho from the
// score sums of the last update_K ticks (gpu_bpf_ptx_full.cu:489-543): step size
// c / (k + t0)^gamma, direction mean score / mean Fisher information (mode 1; the
// mean score itself in mode 2), clipped to +-5, gated by min(SNR / 2, 1) with
// SNR = |mean score| / sqrt(mean Fisher / K). Waits for the filter's stream.
int learning_update(GpuBpfState* s, Impl* m) {
  CK(cudaMemcpyAsync(m->st_pin, m->plan.st, sizeof(DevState), cudaMemcpyDeviceToHost, m->stream));
  CK(cudaStreamSynchronize(m->stream));
  const double* sums = m->st_pin->learn;
  m->rm_step += 1;
  const double eta = m->rm_c / std::pow((double)m->rm_step + m->rm_t0, (double)m->rm_gamma);
  const double K = (double)m->grad_count;
  auto step = [&](double g_sum, double f_sum) {
    const double mean_g = g_sum / K, mean_f = f_sum / K;
    double dir = (m->learn_mode == 2) ? mean_g : mean_g / std::fmax(mean_f, 1e-8);
    if (m->grad_clip > 0.0f && std::fabs(dir) > m->grad_clip) dir *= m->grad_clip / std::fabs(dir);
    const double snr = std::fabs(mean_g) / std::fmax(std::sqrt(mean_f / K), 1e-10);
    return eta * std::fmin(snr / 2.0, 1.0) * dir;
  };
  const double rho = s->rho;
  const double alpha = (double)s->mu * (1.0 - rho) + step(sums[0], sums[1]);
  s->mu = (float)std::fmax(std::fmin(alpha / std::fmax(1.0 - rho, 1e-6), 2.0), -5.0);
  if (m->learn_rho) s->rho = (float)std::fmax(std::fmin(rho + step(sums[2], sums[3]), 0.999), 0.001);
  m->grad_count = 0;
  return zero_learning_sums(m);
}

// Enqueue one tick (pass 1, plan, pass 2) on the filter's stream.
int enqueue_tick(GpuBpfState* s, Impl* m, const TickArgs& a) {
  if (m->profiling) {
    cudaEvent_t ev[4] = {take_event(m), take_event(m), take_event(m), take_event(m)};
    CK(cudaEventRecord(ev[0], m->stream));
    CK(launch_pass1(m->plan, a, m->stream, false));
    CK(cudaEventRecord(ev[1], m->stream));
    CK(launch_plan(m->plan, a, m->stream, false));
    CK(cudaEventRecord(ev[2], m->stream));
    CK(launch_pass2(m->plan, a, m->pass2_grid, m->stream, false));
    if (a.silverman > 0.0f) CK(launch_jitter(m->plan, a, m->stream, false));   // timed with pass 2
    CK(cudaEventRecord(ev[3], m->stream));
    for (cudaEvent_t e : ev) m->ev_pending.push_back(e);
    if (m->ev_pending.size() >= 4 * 4096) { int rc = drain_profile(m); if (rc) return rc; }
  } else {
    CK(launch_tick3(m, a));
  }
  g_launches += tick_launches(m, a);
  const int tick = m->ticks_enqueued;
  m->ticks_enqueued += 1;
  if (m->learn_mode && tick > 0 && ++m->grad_count >= m->update_K) return learning_update(s, m);
  return BPF_OK;
}

// Waits until the last single tick's outcome is in host-mapped memory: the plan writes the
// record, then (after a system-scope fence) the mirror carrying the tick's request number, so
// seeing that number means the record is complete although the tick's resampling may still run
// on the stream (later work on the stream is ordered after it). The wait spins on the mirror for
// up to 2 ms, then falls back to a stream synchronise, which also reports launch failures.
int wait_single_tick(Impl* m) {
  const volatile int* seq = &m->mir_map->seq;
  const auto t0 = std::chrono::steady_clock::now();
  for (int i = 0;; ++i) {
    if (*seq == m->seq) {
      std::atomic_thread_fence(std::memory_order_acquire);
      return BPF_OK;
    }
    if ((i & 255) == 255 && std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(2)) break;
  }
  CK(cudaStreamSynchronize(m->stream));
  return BPF_OK;
}

int read_back(GpuBpfState* s, Impl* m, int slot, BpfTickRecord* out) {
  if (slot == 0 && m->last_in_map) {
    const int rc = wait_single_tick(m);
    if (rc) return rc;
    *out = *m->rec_map;                    // written by this tick's plan before its mirror
    const TickMirror mm = *m->mir_map;
    s->did_resample = out->resampled;
    s->resample_count = mm.resample_count;
    s->timestep = mm.tick;
    s->last_h_est = out->h_mean;
    if (mm.error != BPF_OK) m->sticky_error = mm.error;
    return BPF_OK;
  }
  CK(cudaMemcpyAsync(m->rec_pin + slot, m->rec_dev + slot, sizeof(BpfTickRecord), cudaMemcpyDeviceToHost, m->stream));
  CK(cudaMemcpyAsync(m->st_pin, m->plan.st, sizeof(DevState), cudaMemcpyDeviceToHost, m->stream));
  CK(cudaStreamSynchronize(m->stream));
  *out = m->rec_pin[slot];
  s->did_resample = out->resampled;
  s->resample_count = m->st_pin->resample_count;
  s->timestep = m->st_pin->tick;
  s->last_h_est = out->h_mean;
  if (m->st_pin->error != BPF_OK) m->sticky_error = m->st_pin->error;
  return BPF_OK;
}

BpfResult to_result(const Impl* m, const BpfTickRecord& r) {
  BpfResult o;
  o.h_mean = r.h_mean;
  o.log_lik = (float)(m->ll_mode ? r.loglik_ref : r.dloglik);
  return o;
}

int free_impl(Impl* m) {
  if (!m) return BPF_OK;
  if (m->graph) cudaGraphExecDestroy(m->graph);
  if (m->dgraph) cudaGraphExecDestroy(m->dgraph);
  if (m->tgraph) cudaGraphExecDestroy(m->tgraph);
  if (m->t_g) cudaGraphDestroy(m->t_g);
  for (cudaEvent_t e : m->ev_pending) cudaEventDestroy(e);
  for (cudaEvent_t e : m->ev_pool) cudaEventDestroy(e);
  plan_free(m->plan);
  bpf_free(m->rec_dev); bpf_free(m->y_dev); bpf_free(m->anc_dev);
  bpf_free_host(m->rec_pin); bpf_free_host(m->st_pin); bpf_free_host(m->y_pin);
  bpf_free_host(m->rec_map); bpf_free_host(m->mir_map);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return BPF_OK;
}

int build_graph(GpuBpfState* s, Impl* m) {
  if (m->graph) { cudaGraphExecDestroy(m->graph); m->graph = nullptr; }
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaMemcpyAsync(m->y_dev, m->y_pin, kGraphChunk * sizeof(float), cudaMemcpyHostToDevice, m->stream);
  const TickArgs a0 = make_args(s, m, 0.0f, m->y_dev, m->rec_dev + 1);
  if (err == cudaSuccess && use_small(m, a0)) {
    err = launch_small(m->plan, a0, kGraphChunk, m->stream, m->pdl);     // the chunk as one launch
  } else {
    for (int k = 0; k < kGraphChunk && err == cudaSuccess; ++k) {
      TickArgs a = make_args(s, m, 0.0f, m->y_dev + k, m->rec_dev + 1 + k);
      err = launch_tick3(m, a);
    }
  }
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(m->rec_pin + 1, m->rec_dev + 1, kGraphChunk * sizeof(BpfTickRecord), cudaMemcpyDeviceToHost, m->stream);
  cudaError_t e2 = cudaStreamEndCapture(m->stream, &g);
  if (err != cudaSuccess || e2 != cudaSuccess) { if (g) cudaGraphDestroy(g); cudaGetLastError(); return set_err(BPF_ERR_CUDA); }
  cudaError_t e3 = cudaGraphInstantiate(&m->graph, g, 0);
  cudaGraphDestroy(g);
  if (e3 != cudaSuccess) { m->graph = nullptr; return set_err(BPF_ERR_CUDA); }
  m->g_mu = s->mu; m->g_rho = s->rho; m->g_sigma = s->sigma_z; m->g_thr = s->ess_threshold; m->g_nus = s->nu_state;
  m->g_silv = s->silverman_shrink;
  m->g_anc = m->record_anc;
  return BPF_OK;
}

constexpr int kMaxGraphTicks = 16384;   // larger device runs launch directly

int build_device_graph(GpuBpfState* s, Impl* m, const float* y_dev, int n, BpfTickRecord* rec_dev) {
  if (m->dgraph) { cudaGraphExecDestroy(m->dgraph); m->dgraph = nullptr; }
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t err = cudaSuccess;
  const TickArgs a0 = make_args(s, m, 0.0f, y_dev, rec_dev);
  if (use_small(m, a0)) {
    err = launch_small(m->plan, a0, n, m->stream, m->pdl);              // the whole run as one launch
  } else {
    for (int k = 0; k < n && err == cudaSuccess; ++k) {
      TickArgs a = make_args(s, m, 0.0f, y_dev + k, rec_dev + k);
      err = launch_tick3(m, a);
    }
  }
  cudaError_t e2 = cudaStreamEndCapture(m->stream, &g);
  if (err != cudaSuccess || e2 != cudaSuccess) { if (g) cudaGraphDestroy(g); cudaGetLastError(); return set_err(BPF_ERR_CUDA); }
  cudaError_t e3 = cudaGraphInstantiate(&m->dgraph, g, 0);
  cudaGraphDestroy(g);
  if (e3 != cudaSuccess) { m->dgraph = nullptr; return set_err(BPF_ERR_CUDA); }
  m->dg_y = y_dev; m->dg_rec = rec_dev; m->dg_n = n;
  m->dg_mu = s->mu; m->dg_rho = s->rho; m->dg_sigma = s->sigma_z; m->dg_thr = s->ess_threshold;
  m->dg_nus = s->nu_state;
  m->dg_silv = s->silverman_shrink;
  m->dg_anc = m->record_anc;
  return BPF_OK;
}

bool tick_graph_stale(GpuBpfState* s, Impl* m) {
  return !m->tgraph || m->t_mu != s->mu || m->t_rho != s->rho || m->t_sigma != s->sigma_z ||
         m->t_thr != s->ess_threshold || m->t_nus != s->nu_state || m->t_silv != s->silverman_shrink ||
         m->t_anc != m->record_anc;
}

// Captures one tick (pass 1, plan, pass 2 with their programmatic dependencies) writing its
// record and outcome into the host-mapped slot, and finds pass 1's node: the graph's only root.
int build_tick_graph(GpuBpfState* s, Impl* m) {
  if (m->tgraph) { cudaGraphExecDestroy(m->tgraph); m->tgraph = nullptr; }
  if (m->t_g) { cudaGraphDestroy(m->t_g); m->t_g = nullptr; }
  m->t_pass1 = nullptr;
  TickArgs a = make_args(s, m, 0.0f, nullptr, m->rec_map_dev);
  a.mirror = m->mir_map_dev;
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
  const cudaError_t err = launch_tick3(m, a);
  const cudaError_t e2 = cudaStreamEndCapture(m->stream, &g);
  if (err != cudaSuccess || e2 != cudaSuccess) { if (g) cudaGraphDestroy(g); cudaGetLastError(); return set_err(BPF_ERR_CUDA); }
  size_t nroot = 0;
  cudaGraphNode_t root = nullptr;
  cudaGraphNodeType type = cudaGraphNodeTypeEmpty;
  if (cudaGraphGetRootNodes(g, nullptr, &nroot) != cudaSuccess || nroot != 1 ||
      cudaGraphGetRootNodes(g, &root, &nroot) != cudaSuccess || cudaGraphNodeGetType(root, &type) != cudaSuccess ||
      type != cudaGraphNodeTypeKernel || cudaGraphKernelNodeGetParams(root, &m->t_params) != cudaSuccess) {
    cudaGraphDestroy(g);
    cudaGetLastError();
    return set_err(BPF_ERR_CUDA);
  }
  cudaGraphExec_t ex = nullptr;
  if (cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) { cudaGraphDestroy(g); cudaGetLastError(); return set_err(BPF_ERR_CUDA); }
  m->t_g = g;
  m->tgraph = ex;
  m->t_pass1 = root;
  m->t_plan = m->plan;                     // the root kernel's arguments, as its launcher passed them
  m->t_n = 1;
  m->t_args = a;
  m->t_args.tail_plan = use_tail(m, a) ? 1 : 0;  // as launch_tick3 passed it to the root (pass 1)
  m->t_argv[0] = &m->t_plan;
  m->t_argv[1] = &m->t_args;
  m->t_argv[2] = &m->t_n;                  // read only by the fused kernel (three parameters)
  m->t_params.kernelParams = m->t_argv;
  m->t_params.extra = nullptr;
  m->t_mu = s->mu; m->t_rho = s->rho; m->t_sigma = s->sigma_z; m->t_thr = s->ess_threshold; m->t_nus = s->nu_state;
  m->t_silv = s->silverman_shrink;
  m->t_anc = m->record_anc;
  return BPF_OK;
}

bool graph_stale(GpuBpfState* s, Impl* m) {
  return !m->graph || m->g_mu != s->mu || m->g_rho != s->rho || m->g_sigma != s->sigma_z ||
         m->g_thr != s->ess_threshold || m->g_nus != s->nu_state || m->g_silv != s->silverman_shrink ||
         m->g_anc != m->record_anc;
}

}  // namespace

// ===========================================================================
// Reference API
// ===========================================================================
extern "C" {

int gpu_bpf_last_error(void) { return g_last_error; }

const char* gpu_bpf_error_string(int code) {
  switch (code) {
    case BPF_OK: return "ok";
    case BPF_ERR_ARG: return "invalid argument";
    case BPF_ERR_CUDA: return "CUDA runtime error";
    case BPF_ERR_ALLOC: return "allocation failed";
    case BPF_ERR_UNSUPPORTED: return "option not supported by this build";
    case BPF_ERR_STATE: return "invalid filter state";
    case BPF_ERR_DEGENERATE: return "all particle weights underflowed";
    case BPF_ERR_NODEVICE: return "no usable CUDA device";
    default: return "unknown error";
  }
}

long long gpu_bpf_launch_count(void) { return g_launches.load(); }

static int create_impl(GpuBpfState* s, Impl* m, int n, float rho, float sigma_z, float mu, float nu_obs, int seed) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return set_err(BPF_ERR_NODEVICE); }
  CK(cudaGetDevice(&m->device));
  m->seed = seed;
  Plan& p = m->plan;
  CK(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  CK(plan_alloc(p, n));
  CK(bpf_malloc(&m->rec_dev, (1 + kGraphChunk) * sizeof(BpfTickRecord)));
  CK(bpf_malloc(&m->y_dev, kGraphChunk * sizeof(float)));
  CK(bpf_malloc_host(&m->rec_pin, (1 + kGraphChunk) * sizeof(BpfTickRecord)));
  CK(bpf_malloc_host(&m->st_pin, sizeof(DevState)));
  CK(bpf_malloc_host(&m->y_pin, kGraphChunk * sizeof(float)));
  CK(bpf_host_alloc(&m->rec_map, sizeof(BpfTickRecord), cudaHostAllocMapped));
  CK(bpf_host_alloc(&m->mir_map, sizeof(TickMirror), cudaHostAllocMapped));
  CK(cudaHostGetDevicePointer(reinterpret_cast<void**>(&m->rec_map_dev), m->rec_map, 0));
  CK(cudaHostGetDevicePointer(reinterpret_cast<void**>(&m->mir_map_dev), m->mir_map, 0));
  std::memset(m->rec_map, 0, sizeof(BpfTickRecord));
  std::memset(m->mir_map, 0, sizeof(TickMirror));
  CK(cudaMemsetAsync(m->rec_dev, 0, (1 + kGraphChunk) * sizeof(BpfTickRecord), m->stream));
  m->pass2_grid = pass2_grid_size(m->device);
  m->small_tiles = small_max_tiles(m->device);
  if (const char* v = std::getenv("BPF_DISABLE_PDL")) m->pdl = (v[0] == '0');

  // observation model (gpu_bpf_ptx_full.cu:406-412)
  m->obs.nu = nu_obs;
  if (nu_obs > 0.0f) {
    m->obs.c_obs = (float)(std::lgamma((nu_obs + 1.0) / 2.0) - std::lgamma(nu_obs / 2.0) -
                           0.5 * std::log(nu_obs * 3.14159265358979323846));
    m->obs.inv_nu = 1.0f / nu_obs;
    m->obs.nu_p1h = (nu_obs + 1.0f) * 0.5f;
  }

  const float std_stat = sqrtf((sigma_z * sigma_z) / fmaxf(1.0f - rho * rho, 1e-6f));   // :430
  CK(launch_init(p, mu, std_stat, seed, m->stream));
  g_launches += 1;
  CK(cudaStreamSynchronize(m->stream));
  s->stream = (void*)m->stream;
  return BPF_OK;
}

GpuBpfState* gpu_bpf_create(int n_particles, float rho, float sigma_z, float mu,
                            float nu_state, float nu_obs, int seed) {
  g_last_error = BPF_OK;
  if (n_particles <= 0 || n_particles > (1 << 30) || !std::isfinite(rho) || !std::isfinite(sigma_z) ||
      !std::isfinite(mu) || !(std::fabs(rho) < 1.0f) || !(sigma_z > 0.0f) || !(nu_obs >= 0.0f) ||
      !std::isfinite(nu_obs) || !(nu_state >= 0.0f)) {
    set_err(BPF_ERR_ARG);
    return nullptr;
  }
  if (nu_state > 0.0f && nu_state < 0.5f) { set_err(BPF_ERR_ARG); return nullptr; }   // round(nu_state) >= 1
  GpuBpfState* s = (GpuBpfState*)calloc(1, sizeof(GpuBpfState));
  if (!s) { set_err(BPF_ERR_ALLOC); return nullptr; }
  s->n_particles = n_particles;
  s->rho = rho; s->sigma_z = sigma_z; s->mu = mu;
  s->nu_state = nu_state; s->nu_obs = nu_obs;
  s->silverman_shrink = 0.0f;
  s->ess_threshold = 0.5f;           // gpu_bpf_ptx_full.cu:356
  s->did_resample = 1;
  s->last_h_est = mu;
  Impl* m = new Impl();
  s->impl = m;
  int rc = create_impl(s, m, n_particles, rho, sigma_z, mu, nu_obs, seed);
  if (rc != BPF_OK) {
    free_impl(m);
    free(s);
    set_err(rc);
    return nullptr;
  }
  return s;
}

void gpu_bpf_destroy(GpuBpfState* s) {
  if (!s) return;
  Impl* m = impl_of(s);
  if (m) { ensure_device(m); cudaStreamSynchronize(m->stream); free_impl(m); }
  s->impl = nullptr;
  free(s);
}

// One tick enqueued. A synchronous step (one_shot) launches the single-tick graph (less host
// time per tick); consecutive asynchronous steps launch the kernels directly, so each tick's
// pass 1 overlaps the previous tick's pass 2 through programmatic dependent launch.
static int step_async_rc(GpuBpfState* s, float y_t, bool one_shot) {
  Impl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  if (!std::isfinite(y_t)) return set_err(BPF_ERR_ARG);
  int rc = check_options(s);
  if (rc) return rc;
  rc = ensure_device(m);
  if (rc) return rc;
  if (one_shot && !m->profiling && !m->learn_mode) {  // learning updates need the host every K ticks
    if (tick_graph_stale(s, m)) { rc = build_tick_graph(s, m); if (rc) return rc; }
    m->t_args.obs.y = y_t;
    m->t_args.seq = ++m->seq;
    CK(cudaGraphExecKernelNodeSetParams(m->tgraph, m->t_pass1, &m->t_params));
    CK(cudaGraphLaunch(m->tgraph, m->stream));
    g_launches += tick_launches(m, m->t_args);
    m->ticks_enqueued += 1;
    m->last_in_map = true;
    return BPF_OK;
  }
  TickArgs a = make_args(s, m, y_t, nullptr, m->rec_map_dev);
  a.mirror = m->mir_map_dev;
  a.seq = ++m->seq;
  rc = enqueue_tick(s, m, a);
  if (rc == BPF_OK) m->last_in_map = true;
  return rc;
}

void gpu_bpf_step_async(GpuBpfState* s, float y_t) { step_async_rc(s, y_t, false); }

BpfResult gpu_bpf_get_result(GpuBpfState* s) {
  BpfResult bad; bad.h_mean = NAN; bad.log_lik = NAN;
  Impl* m = impl_of(s);
  if (!m) { set_err(BPF_ERR_STATE); return bad; }
  if (m->ticks_enqueued == 0) { set_err(BPF_ERR_STATE); return bad; }
  if (ensure_device(m)) return bad;
  BpfTickRecord r;
  if (read_back(s, m, 0, &r) != BPF_OK) return bad;
  return to_result(m, r);
}

BpfResult gpu_bpf_step(GpuBpfState* s, float y_t) {
  BpfResult bad; bad.h_mean = NAN; bad.log_lik = NAN;
  if (step_async_rc(s, y_t, true) != BPF_OK) return bad;
  return gpu_bpf_get_result(s);
}

double gpu_bpf_run_rmse(const double* returns, const double* true_h, int n_ticks,
                        int n_particles, float rho, float sigma_z, float mu,
                        float nu_state, float nu_obs, int seed) {
  if (!returns || !true_h || n_ticks <= 100) { set_err(BPF_ERR_ARG); return NAN; }
  GpuBpfState* f = gpu_bpf_create(n_particles, rho, sigma_z, mu, nu_state, nu_obs, seed);
  if (!f) return NAN;
  std::vector<float> y(n_ticks);
  for (int t = 0; t < n_ticks; ++t) y[t] = (float)returns[t];
  std::vector<BpfResult> out(n_ticks);
  int rc = gpu_bpf_step_many(f, y.data(), n_ticks, out.data(), nullptr);
  gpu_bpf_destroy(f);
  if (rc != BPF_OK) { set_err(rc); return NAN; }
  double sse = 0.0;
  int count = 0;
  for (int t = 100; t < n_ticks; ++t) {            // gpu_bpf_ptx_full.cu:841-848
    const double e = (double)out[t].h_mean - true_h[t];
    sse += e * e;
    ++count;
  }
  return std::sqrt(sse / (double)count);
}

void gpu_bpf_set_bands(int n_particles, int n_bands, const float* fracs, const float* scales) {
  (void)n_particles; (void)fracs;
  if (n_bands == 1 && scales && scales[0] == 1.0f) { g_last_error = BPF_OK; return; }
  set_err(BPF_ERR_UNSUPPORTED);
}

void gpu_bpf_set_adaptive_bands(int, const float*, const float*, int, const float*, const float*, int,
                                const float*, const float*, int, float, float) {
  set_err(BPF_ERR_UNSUPPORTED);
}

void gpu_bpf_set_ess_threshold(GpuBpfState* s, float threshold) {
  if (!s) { set_err(BPF_ERR_STATE); return; }
  s->ess_threshold = threshold;
}

int gpu_bpf_get_resample_count(GpuBpfState* s) {
  Impl* m = impl_of(s);
  if (!m) { set_err(BPF_ERR_STATE); return -1; }
  if (ensure_device(m)) return -1;
  if (cudaMemcpyAsync(m->st_pin, m->plan.st, sizeof(DevState), cudaMemcpyDeviceToHost, m->stream) != cudaSuccess ||
      cudaStreamSynchronize(m->stream) != cudaSuccess) { set_err(BPF_ERR_CUDA); return -1; }
  s->resample_count = m->st_pin->resample_count;
  return s->resample_count;
}

float gpu_bpf_get_mu(GpuBpfState* s) { return s ? s->mu : NAN; }
float gpu_bpf_get_rho(GpuBpfState* s) { return s ? s->rho : NAN; }
// An external parameter push restarts the Robbins-Monro schedule (gpu_bpf_ptx_full.cu:812-828).
static void restart_learning(GpuBpfState* s) {
  Impl* m = impl_of(s);
  if (!m) return;
  m->rm_step = 0;
  m->grad_count = 0;
  if (ensure_device(m) == BPF_OK) zero_learning_sums(m);
}
void gpu_bpf_set_mu(GpuBpfState* s, float mu) {
  if (!s || !std::isfinite(mu)) { set_err(BPF_ERR_ARG); return; }
  s->mu = mu;
  restart_learning(s);
}
void gpu_bpf_set_rho(GpuBpfState* s, float rho) {
  if (!s || !std::isfinite(rho)) { set_err(BPF_ERR_ARG); return; }
  s->rho = fmaxf(fminf(rho, 0.999f), 0.001f);       // gpu_bpf_ptx_full.cu:822
  restart_learning(s);
}
void gpu_bpf_enable_mu_learning(GpuBpfState* s, int mode, int K, float c, float t0, float gamma) {
  Impl* m = impl_of(s);
  if (!m) { set_err(BPF_ERR_STATE); return; }
  if (mode < 0 || mode > 2 || K < 1 || !(c > 0.0f) || !(t0 >= 0.0f) || !(gamma > 0.0f)) { set_err(BPF_ERR_ARG); return; }
  m->learn_mode = mode;                              // gpu_bpf_ptx_full.cu:777-790
  m->update_K = K;
  m->grad_clip = 5.0f;
  m->rm_c = c; m->rm_t0 = t0; m->rm_gamma = gamma;
  restart_learning(s);
}
void gpu_bpf_disable_mu_learning(GpuBpfState* s) {
  Impl* m = impl_of(s);
  if (!m) { set_err(BPF_ERR_STATE); return; }
  m->learn_mode = 0;
  m->learn_rho = 0;
}
void gpu_bpf_enable_rho_learning(GpuBpfState* s, int enable) {
  Impl* m = impl_of(s);
  if (!m) { set_err(BPF_ERR_STATE); return; }
  m->learn_rho = enable ? 1 : 0;
}
int gpu_bpf_get_learning_sums(GpuBpfState* s, double* sums4, int* ticks) {
  Impl* m = impl_of(s);
  if (!m || !sums4) return set_err(!m ? BPF_ERR_STATE : BPF_ERR_ARG);
  int rc = ensure_device(m);
  if (rc) return rc;
  CK(cudaMemcpyAsync(m->st_pin, m->plan.st, sizeof(DevState), cudaMemcpyDeviceToHost, m->stream));
  CK(cudaStreamSynchronize(m->stream));
  for (int i = 0; i < 4; ++i) sums4[i] = m->st_pin->learn[i];
  if (ticks) *ticks = m->grad_count;
  return BPF_OK;
}

// ===========================================================================
// Additions
// ===========================================================================
int gpu_bpf_step_many(GpuBpfState* s, const float* y, int n_ticks, BpfResult* out, BpfTickRecord* rec) {
  Impl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  if (n_ticks < 0 || (n_ticks > 0 && !y)) return set_err(BPF_ERR_ARG);
  for (int t = 0; t < n_ticks; ++t) if (!std::isfinite(y[t])) return set_err(BPF_ERR_ARG);
  int rc = check_options(s);
  if (rc) return rc;
  rc = ensure_device(m);
  if (rc) return rc;
  int t = 0;
  if (!m->profiling && !m->learn_mode) {            // learning updates need the host every K ticks
    while (n_ticks - t >= kGraphChunk) {
      if (graph_stale(s, m)) { rc = build_graph(s, m); if (rc) return rc; }
      std::memcpy(m->y_pin, y + t, kGraphChunk * sizeof(float));
      CK(cudaGraphLaunch(m->graph, m->stream));
      CK(cudaStreamSynchronize(m->stream));
      g_launches += use_small(m, make_args(s, m, 0.0f, nullptr, nullptr))
                        ? 1 : (long long)tick_launches(m, make_args(s, m, 0.0f, nullptr, nullptr)) * kGraphChunk;
      m->ticks_enqueued += kGraphChunk;
      for (int k = 0; k < kGraphChunk; ++k) {
        if (out) out[t + k] = to_result(m, m->rec_pin[1 + k]);
        if (rec) rec[t + k] = m->rec_pin[1 + k];
      }
      t += kGraphChunk;
    }
  }
  // remainder (and the profiled path): direct launches into the same record slots
  while (t < n_ticks) {
    const int n = std::min(kGraphChunk, n_ticks - t);
    for (int k = 0; k < n; ++k) {
      rc = enqueue_tick(s, m, make_args(s, m, y[t + k], nullptr, m->rec_dev + 1 + k));
      if (rc) return rc;
    }
    CK(cudaMemcpyAsync(m->rec_pin + 1, m->rec_dev + 1, n * sizeof(BpfTickRecord), cudaMemcpyDeviceToHost, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    for (int k = 0; k < n; ++k) {
      if (out) out[t + k] = to_result(m, m->rec_pin[1 + k]);
      if (rec) rec[t + k] = m->rec_pin[1 + k];
    }
    t += n;
  }
  // keep slot 0 = last tick so get_result/get_record see it
  if (n_ticks > 0) {
    m->last_in_map = false;
    const int last = (n_ticks - 1) % kGraphChunk;
    const BpfTickRecord& lr = m->rec_pin[1 + last];
    CK(cudaMemcpyAsync(m->rec_dev, m->rec_dev + 1 + last, sizeof(BpfTickRecord), cudaMemcpyDeviceToDevice, m->stream));
    CK(cudaMemcpyAsync(m->st_pin, m->plan.st, sizeof(DevState), cudaMemcpyDeviceToHost, m->stream));
    CK(cudaStreamSynchronize(m->stream));
    s->did_resample = lr.resampled;
    s->last_h_est = lr.h_mean;
    s->resample_count = m->st_pin->resample_count;
    s->timestep = m->st_pin->tick;
    if (m->st_pin->error != BPF_OK) { m->sticky_error = m->st_pin->error; return set_err(m->st_pin->error); }
  }
  return BPF_OK;
}

int gpu_bpf_step_many_device(GpuBpfState* s, const float* y_dev, int n_ticks, BpfTickRecord* rec_dev) {
  Impl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  if (n_ticks < 0 || (n_ticks > 0 && (!y_dev || !rec_dev))) return set_err(BPF_ERR_ARG);
  int rc = check_options(s);
  if (rc) return rc;
  rc = ensure_device(m);
  if (rc) return rc;
  if (!m->profiling && !m->learn_mode && n_ticks > 0 && n_ticks <= kMaxGraphTicks) {
    const bool stale = !m->dgraph || m->dg_y != y_dev || m->dg_rec != rec_dev || m->dg_n != n_ticks ||
                       m->dg_mu != s->mu || m->dg_rho != s->rho || m->dg_sigma != s->sigma_z ||
                       m->dg_thr != s->ess_threshold || m->dg_nus != s->nu_state ||
                       m->dg_silv != s->silverman_shrink || m->dg_anc != m->record_anc;
    if (stale) { rc = build_device_graph(s, m, y_dev, n_ticks, rec_dev); if (rc) return rc; }
    CK(cudaGraphLaunch(m->dgraph, m->stream));
    g_launches += use_small(m, make_args(s, m, 0.0f, nullptr, nullptr))
                      ? 1 : (long long)tick_launches(m, make_args(s, m, 0.0f, nullptr, nullptr)) * n_ticks;
    m->ticks_enqueued += n_ticks;
  } else {
    for (int t = 0; t < n_ticks; ++t) {
      rc = enqueue_tick(s, m, make_args(s, m, 0.0f, y_dev + t, rec_dev + t));
      if (rc) return rc;
    }
  }
  if (n_ticks > 0) {
    CK(cudaMemcpyAsync(m->rec_dev, rec_dev + n_ticks - 1, sizeof(BpfTickRecord), cudaMemcpyDeviceToDevice, m->stream));
    m->last_in_map = false;
  }
  return BPF_OK;
}

int gpu_bpf_reset(GpuBpfState* s, int seed) {
  Impl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  int rc = check_options(s);
  if (rc) return rc;
  rc = ensure_device(m);
  if (rc) return rc;
  m->seed = seed;
  const float std_stat = sqrtf((s->sigma_z * s->sigma_z) / fmaxf(1.0f - s->rho * s->rho, 1e-6f));
  CK(launch_init(m->plan, s->mu, std_stat, seed, m->stream));   // also resets the DevState
  g_launches += 1;
  m->ticks_enqueued = 0;
  m->last_in_map = false;
  m->grad_count = 0;                               // the init kernel zeroes the device sums
  s->timestep = 0; s->did_resample = 1; s->resample_count = 0; s->last_h_est = s->mu;
  return BPF_OK;
}

int gpu_bpf_get_record(GpuBpfState* s, BpfTickRecord* out) {
  Impl* m = impl_of(s);
  if (!m || !out) return set_err(!m ? BPF_ERR_STATE : BPF_ERR_ARG);
  if (m->ticks_enqueued == 0) return set_err(BPF_ERR_STATE);
  int rc = ensure_device(m);
  if (rc) return rc;
  return read_back(s, m, 0, out);
}

float gpu_bpf_get_ess(GpuBpfState* s) {
  BpfTickRecord r;
  if (gpu_bpf_get_record(s, &r) != BPF_OK) return NAN;
  return r.ess;
}

double gpu_bpf_get_loglik_total(GpuBpfState* s) {
  Impl* m = impl_of(s);
  if (!m) { set_err(BPF_ERR_STATE); return NAN; }
  if (ensure_device(m)) return NAN;
  if (cudaMemcpyAsync(m->st_pin, m->plan.st, sizeof(DevState), cudaMemcpyDeviceToHost, m->stream) != cudaSuccess ||
      cudaStreamSynchronize(m->stream) != cudaSuccess) { set_err(BPF_ERR_CUDA); return NAN; }
  return m->st_pin->ll_total;
}

int gpu_bpf_set_loglik_semantics(GpuBpfState* s, int mode) {
  Impl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  if (mode != 0 && mode != 1) return set_err(BPF_ERR_ARG);
  m->ll_mode = mode;
  return BPF_OK;
}

int gpu_bpf_get_particles(GpuBpfState* s, float* h_out) {
  Impl* m = impl_of(s);
  if (!m || !h_out) return set_err(!m ? BPF_ERR_STATE : BPF_ERR_ARG);
  int rc = ensure_device(m);
  if (rc) return rc;
  CK(cudaMemcpyAsync(m->st_pin, m->plan.st, sizeof(DevState), cudaMemcpyDeviceToHost, m->stream));
  CK(cudaStreamSynchronize(m->stream));
  const float* src = m->st_pin->cur ? m->plan.h1 : m->plan.h0;
  CK(cudaMemcpy(h_out, src, (size_t)m->plan.N * sizeof(float), cudaMemcpyDeviceToHost));
  return BPF_OK;
}

int gpu_bpf_record_ancestors(GpuBpfState* s, int enable) {
  Impl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  int rc = ensure_device(m);
  if (rc) return rc;
  if (enable && !m->anc_dev) {
    CK(bpf_malloc(&m->anc_dev, (size_t)m->plan.N * sizeof(int32_t)));
    CK(cudaMemsetAsync(m->anc_dev, 0xff, (size_t)m->plan.N * sizeof(int32_t), m->stream));
  }
  m->record_anc = enable != 0;
  return BPF_OK;
}

int gpu_bpf_get_ancestors(GpuBpfState* s, int32_t* anc_out) {
  Impl* m = impl_of(s);
  if (!m || !anc_out) return -set_err(!m ? BPF_ERR_STATE : BPF_ERR_ARG);
  if (!m->anc_dev || m->ticks_enqueued == 0) return -set_err(BPF_ERR_STATE);
  if (ensure_device(m)) return -BPF_ERR_CUDA;
  BpfTickRecord r;
  int rc = read_back(s, m, 0, &r);
  if (rc) return -rc;
  // the ancestors are written by the tick's resampling, which may still run after its record
  if (cudaStreamSynchronize(m->stream) != cudaSuccess ||
      cudaMemcpy(anc_out, m->anc_dev, (size_t)m->plan.N * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
    return -set_err(BPF_ERR_CUDA);
  return r.resampled ? 1 : 0;
}

int gpu_bpf_get_resample_inputs(GpuBpfState* s, float* w_out, int32_t* tile_exp_out, uint32_t* u23_out) {
  Impl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  int rc = ensure_device(m);
  if (rc) return rc;
  CK(cudaMemcpyAsync(m->st_pin, m->plan.st, sizeof(DevState), cudaMemcpyDeviceToHost, m->stream));
  CK(cudaStreamSynchronize(m->stream));
  if (w_out) {
    float* w_dev = nullptr;
    CK(bpf_malloc(&w_dev, (size_t)m->plan.N * sizeof(float)));
    cudaError_t e = launch_tile_weights(m->plan, w_dev, m->stream);
    g_launches += 1;
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    if (e == cudaSuccess) e = cudaMemcpy(w_out, w_dev, (size_t)m->plan.N * sizeof(float), cudaMemcpyDeviceToHost);
    bpf_free(w_dev);
    CK(e);
  }
  if (tile_exp_out) CK(cudaMemcpy(tile_exp_out, m->plan.nexp, (size_t)m->plan.G * sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (u23_out) *u23_out = m->st_pin->u23;
  return BPF_OK;
}

// ---------------------------------------------------------------------------
// Checkpoint / resume: the filter's whole stochastic state in one byte string.
// The PCG32 streams are counter-based, so the state holds no RNG arrays: the
// device state's stream constants and tick index, plus the resampling-uniform
// stream position, determine every later draw.
// ---------------------------------------------------------------------------
namespace {
struct CkptHeader {
  char magic[8];                 // "GPUBPF\0\1"
  uint32_t version;              // 1
  uint32_t devstate_bytes;       // sizeof(DevState)
  int32_t n, G;
  float rho, sigma_z, mu, nu_state, nu_obs, ess_threshold, silverman_shrink;
  int32_t seed;
};
constexpr char kCkptMagic[8] = {'G', 'P', 'U', 'B', 'P', 'F', 0, 1};

size_t ckpt_bytes(const Impl* m) {
  return sizeof(CkptHeader) + sizeof(DevState) + (size_t)m->plan.G * sizeof(int32_t) +
         2 * (size_t)m->plan.N * sizeof(float);
}
}  // namespace

size_t gpu_bpf_checkpoint_bytes(GpuBpfState* s) {
  Impl* m = impl_of(s);
  if (!m) { set_err(BPF_ERR_STATE); return 0; }
  return ckpt_bytes(m);
}

int gpu_bpf_save(GpuBpfState* s, void* buf, size_t cap) {
  Impl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  if (!buf || cap < ckpt_bytes(m)) return set_err(BPF_ERR_ARG);
  int rc = ensure_device(m);
  if (rc) return rc;
  CK(cudaStreamSynchronize(m->stream));
  unsigned char* out = static_cast<unsigned char*>(buf);
  CkptHeader h{};
  std::memcpy(h.magic, kCkptMagic, sizeof(h.magic));
  h.version = 1;
  h.devstate_bytes = (uint32_t)sizeof(DevState);
  h.n = m->plan.N; h.G = m->plan.G;
  h.rho = s->rho; h.sigma_z = s->sigma_z; h.mu = s->mu; h.nu_state = s->nu_state; h.nu_obs = s->nu_obs;
  h.ess_threshold = s->ess_threshold; h.silverman_shrink = s->silverman_shrink;
  h.seed = m->seed;
  std::memcpy(out, &h, sizeof(h));
  out += sizeof(h);
  DevState st;
  CK(cudaMemcpy(&st, m->plan.st, sizeof(DevState), cudaMemcpyDeviceToHost));
  std::memcpy(out, &st, sizeof(st));
  out += sizeof(st);
  const size_t nb = (size_t)m->plan.N * sizeof(float);
  CK(cudaMemcpy(out, m->plan.nexp, (size_t)m->plan.G * sizeof(int32_t), cudaMemcpyDeviceToHost));
  out += (size_t)m->plan.G * sizeof(int32_t);
  CK(cudaMemcpy(out, st.cur ? m->plan.h1 : m->plan.h0, nb, cudaMemcpyDeviceToHost));
  out += nb;
  CK(cudaMemcpy(out, m->plan.w, nb, cudaMemcpyDeviceToHost));
  return BPF_OK;
}

int gpu_bpf_load(GpuBpfState* s, const void* buf, size_t len) {
  Impl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  if (!buf || len < ckpt_bytes(m)) return set_err(BPF_ERR_ARG);
  const unsigned char* in = static_cast<const unsigned char*>(buf);
  CkptHeader h;
  std::memcpy(&h, in, sizeof(h));
  if (std::memcmp(h.magic, kCkptMagic, sizeof(h.magic)) != 0 || h.version != 1 ||
      h.devstate_bytes != (uint32_t)sizeof(DevState) || h.n != m->plan.N || h.G != m->plan.G)
    return set_err(BPF_ERR_ARG);
  if (!std::isfinite(h.rho) || !(std::fabs(h.rho) < 1.0f) || !(h.sigma_z > 0.0f) || !std::isfinite(h.mu) ||
      !(h.nu_obs >= 0.0f) || !std::isfinite(h.nu_obs) || !(h.nu_state == 0.0f || h.nu_state >= 0.5f))
    return set_err(BPF_ERR_ARG);
  int rc = ensure_device(m);
  if (rc) return rc;
  in += sizeof(h);
  DevState st;
  std::memcpy(&st, in, sizeof(st));
  in += sizeof(st);
  const size_t nb = (size_t)m->plan.N * sizeof(float);
  CK(cudaStreamSynchronize(m->stream));
  CK(cudaMemcpy(m->plan.st, &st, sizeof(DevState), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(m->plan.nexp, in, (size_t)m->plan.G * sizeof(int32_t), cudaMemcpyHostToDevice));
  in += (size_t)m->plan.G * sizeof(int32_t);
  CK(cudaMemcpy(st.cur ? m->plan.h1 : m->plan.h0, in, nb, cudaMemcpyHostToDevice));
  in += nb;
  CK(cudaMemcpy(m->plan.w, in, nb, cudaMemcpyHostToDevice));
  s->rho = h.rho; s->sigma_z = h.sigma_z; s->mu = h.mu; s->nu_state = h.nu_state; s->nu_obs = h.nu_obs;
  s->ess_threshold = h.ess_threshold; s->silverman_shrink = h.silverman_shrink;
  m->seed = h.seed;
  m->obs = ObsModel{};
  m->obs.nu = h.nu_obs;
  if (h.nu_obs > 0.0f) {
    m->obs.c_obs = (float)(std::lgamma((h.nu_obs + 1.0) / 2.0) - std::lgamma(h.nu_obs / 2.0) -
                           0.5 * std::log(h.nu_obs * 3.14159265358979323846));
    m->obs.inv_nu = 1.0f / h.nu_obs;
    m->obs.nu_p1h = (h.nu_obs + 1.0f) * 0.5f;
  }
  // captured graphs hold the observation model and parameters of their capture: drop them
  if (m->graph) { cudaGraphExecDestroy(m->graph); m->graph = nullptr; }
  if (m->dgraph) { cudaGraphExecDestroy(m->dgraph); m->dgraph = nullptr; }
  if (m->tgraph) { cudaGraphExecDestroy(m->tgraph); m->tgraph = nullptr; }
  if (m->t_g) { cudaGraphDestroy(m->t_g); m->t_g = nullptr; }
  m->ticks_enqueued = 0;
  m->last_in_map = false;
  m->grad_count = 0;
  s->timestep = st.tick;
  s->resample_count = st.resample_count;
  s->did_resample = st.resampled_prev;
  return BPF_OK;
}

int gpu_bpf_set_fused_small(GpuBpfState* s, int enable) {
  Impl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  const bool on = enable != 0;
  if (on != m->fused_small) {              // captured graphs hold the other path's launches
    int rc = ensure_device(m);
    if (rc) return rc;
    CK(cudaStreamSynchronize(m->stream));
    if (m->graph) { cudaGraphExecDestroy(m->graph); m->graph = nullptr; }
    if (m->dgraph) { cudaGraphExecDestroy(m->dgraph); m->dgraph = nullptr; }
    if (m->tgraph) { cudaGraphExecDestroy(m->tgraph); m->tgraph = nullptr; }
    if (m->t_g) { cudaGraphDestroy(m->t_g); m->t_g = nullptr; }
    m->fused_small = on;
  }
  return BPF_OK;
}

int gpu_bpf_profile(GpuBpfState* s, int enable) {
  Impl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  int rc = ensure_device(m);
  if (rc) return rc;
  rc = drain_profile(m);
  if (rc) return rc;
  m->profiling = enable != 0;
  m->prof_p1_ms = m->prof_plan_ms = m->prof_p2_ms = 0.0;
  m->prof_n1 = m->prof_n2 = 0;
  return BPF_OK;
}

int gpu_bpf_profile_read(GpuBpfState* s, double* p1, double* plan, double* p2, int* n1, int* n2) {
  Impl* m = impl_of(s);
  if (!m) return set_err(BPF_ERR_STATE);
  int rc = ensure_device(m);
  if (rc) return rc;
  rc = drain_profile(m);
  if (rc) return rc;
  if (p1) *p1 = m->prof_p1_ms;
  if (plan) *plan = m->prof_plan_ms;
  if (p2) *p2 = m->prof_p2_ms;
  if (n1) *n1 = m->prof_n1;
  if (n2) *n2 = m->prof_n2;
  return BPF_OK;
}

static int debug_probe(int seed, int n, int t, uint32_t* out, float* norm) {
  if (n <= 0 || t < 0 || (!out && !norm)) return set_err(BPF_ERR_ARG);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return set_err(BPF_ERR_NODEVICE); }
  uint32_t* d_out = nullptr;
  float* d_norm = nullptr;
  CK(bpf_malloc(&d_out, n * sizeof(uint32_t)));
  CK(bpf_malloc(&d_norm, n * sizeof(float)));
  cudaError_t e = launch_debug_pcg(seed, n, t, d_out, d_norm, 0);
  g_launches += 1;
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess && out) e = cudaMemcpy(out, d_out, n * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && norm) e = cudaMemcpy(norm, d_norm, n * sizeof(float), cudaMemcpyDeviceToHost);
  bpf_free(d_out);
  bpf_free(d_norm);
  CK(e);
  return BPF_OK;
}

int gpu_bpf_debug_pcg32(int seed, int n, int t, uint32_t* out) { return debug_probe(seed, n, t, out, nullptr); }
int gpu_bpf_debug_normals(int seed, int n, int t, float* out) { return debug_probe(seed, n, t, nullptr, out); }

}  // extern "C"
