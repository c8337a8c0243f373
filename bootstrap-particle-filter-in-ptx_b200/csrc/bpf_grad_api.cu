// bpf_grad_api.cu — extern "C" entry points of the gradient form
// (include/gpu_bpf.h, "Gradient").
//
// A GpuBpfGrad owns one plain-filter plan, its stream and a tape sized for up
// to max_ticks ticks. gpu_bpf_grad_forward runs the plain tick kernels with
// the tape hooks on (child lists, checkpoints, weight normalisers);
// gpu_bpf_grad_backward recomputes each checkpoint segment and runs the
// adjoint through it; gpu_bpf_grad_replay re-runs the taped noise and child
// lists in FP64 at any theta. Forward and backward are each replayed as one
// CUDA graph; a change of theta, seed or buffers re-captures the launches and
// updates the instantiated graph in place.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "bpf_grad.cuh"

using namespace bpf;

#define GCK(call)                                                             \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      cudaGetLastError();                                                     \
      return bpf_record_error(e_ == cudaErrorMemoryAllocation ? BPF_ERR_ALLOC : BPF_ERR_CUDA); \
    }                                                                         \
  } while (0)

namespace {

constexpr int kDefaultCheckpoint = 16;

struct FwdKey {
  int T = -1, seed = 0;
  float mu = NAN, rho = NAN, sigma = NAN, nu = NAN, nu_state = NAN;
  const float* y = nullptr;
  double* ll = nullptr;
  bool operator==(const FwdKey& o) const {
    return T == o.T && seed == o.seed && mu == o.mu && rho == o.rho && sigma == o.sigma && nu == o.nu &&
           nu_state == o.nu_state &&
           y == o.y && ll == o.ll;
  }
};
struct BwdKey {
  FwdKey f;
  double* grad = nullptr;
  bool operator==(const BwdKey& o) const { return f == o.f && grad == o.grad; }
};

int nu_int_of(float nu_state) { return nu_state > 0.0f ? (int)(nu_state + 0.5f) : 0; }   // gpu_bpf_ptx_full.cu:392

ObsModel make_obs(float nu_obs) {
  ObsModel o{};
  o.nu = nu_obs;
  if (nu_obs > 0.0f) {
    o.c_obs = (float)(std::lgamma((nu_obs + 1.0) / 2.0) - std::lgamma(nu_obs / 2.0) -
                      0.5 * std::log(nu_obs * 3.14159265358979323846));
    o.inv_nu = 1.0f / nu_obs;
    o.nu_p1h = (nu_obs + 1.0f) * 0.5f;
  }
  return o;
}

// Replace *exec by the graph captured in g (update in place when the topology allows).
cudaError_t install_graph(cudaGraphExec_t* exec, cudaGraph_t g) {
  if (*exec) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(*exec, g, &info) == cudaSuccess) return cudaSuccess;
    cudaGetLastError();
    cudaGraphExecDestroy(*exec);
    *exec = nullptr;
  }
  return cudaGraphInstantiate(exec, g, 0);
}

}  // namespace

struct GpuBpfGrad {
  int device = 0;
  int N = 0, G1 = 0, N4 = 0, T_max = 0, K = kDefaultCheckpoint, n_ckpt = 0;
  size_t ckpt_stride = 0;
  Plan plan{};
  int pass2_grid = 0;
  cudaStream_t stream = nullptr;
  bool pdl = true;

  // tape
  int32_t* csr = nullptr;            // [T_max][N4]
  float* ckpt = nullptr;             // [n_ckpt][G*4096]
  float2* aux = nullptr;             // [T_max]
  BpfTickRecord* rec = nullptr;      // [T_max]
  float* seg = nullptr;              // [K][N4]
  float* lam[2] = {nullptr, nullptr};
  double* acc = nullptr;             // [G1][kGradAcc]

  // FP64 replay (allocated on first use)
  double* rs[2] = {nullptr, nullptr};   // [4][N4] each
  double* part = nullptr;               // [T_max][G1][5]
  double* per_tick = nullptr;           // [T_max][4]
  double* rtotal = nullptr;             // [4]

  // the taped run
  bool have_fwd = false;
  FwdKey cur;
  std::vector<PcgTick> pcs;          // noise constants of ticks 0..T

  cudaGraphExec_t fgraph = nullptr, bgraph = nullptr;
  FwdKey fkey;
  BwdKey bkey;
};

namespace {

void free_grad(GpuBpfGrad* g) {
  if (!g) return;
  if (g->fgraph) cudaGraphExecDestroy(g->fgraph);
  if (g->bgraph) cudaGraphExecDestroy(g->bgraph);
  plan_free(g->plan);
  bpf_free(g->csr); bpf_free(g->ckpt); bpf_free(g->aux); bpf_free(g->rec); bpf_free(g->seg);
  bpf_free(g->lam[0]); bpf_free(g->lam[1]); bpf_free(g->acc);
  bpf_free(g->rs[0]); bpf_free(g->rs[1]); bpf_free(g->part); bpf_free(g->per_tick); bpf_free(g->rtotal);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

int ensure_dev(GpuBpfGrad* g) {
  int cur = -1;
  GCK(cudaGetDevice(&cur));
  if (cur != g->device) GCK(cudaSetDevice(g->device));
  return BPF_OK;
}

// init + T ticks of the plain filter with the tape hooks, then loglik_total -> ll
cudaError_t enqueue_forward(GpuBpfGrad* g, const FwdKey& k) {
  const float std_stat = sqrtf((k.sigma * k.sigma) / fmaxf(1.0f - k.rho * k.rho, 1e-6f));   // gpu_bpf_ptx_full.cu:430
  cudaError_t e = launch_init(g->plan, k.mu, std_stat, k.seed, g->stream);
  const ObsModel obs = make_obs(k.nu);
  for (int t = 0; t < k.T && e == cudaSuccess; ++t) {
    TickArgs a{};
    a.mu = k.mu; a.rho = k.rho; a.sigma = k.sigma;
    a.ess_threshold = 0.0f;
    a.log_n = std::log((double)g->N);
    a.obs = obs;
    a.y_ptr = k.y + t;
    a.rec = g->rec + t;
    a.ckpt = (t % g->K == 0) ? g->ckpt + (size_t)(t / g->K) * g->ckpt_stride : nullptr;
    a.csr = g->csr + (size_t)t * g->N4;
    a.aux = g->aux + t;
    a.nu_int = nu_int_of(k.nu_state);
    a.nu_state = k.nu_state;
    e = launch_pass1(g->plan, a, g->stream, g->pdl);
    if (e == cudaSuccess) e = launch_plan(g->plan, a, g->stream, g->pdl);
    if (e == cudaSuccess) e = launch_pass2(g->plan, a, g->pass2_grid, g->stream, g->pdl);
  }
  if (e == cudaSuccess && k.T > 0)
    e = cudaMemcpyAsync(k.ll, &g->rec[k.T - 1].loglik_total, sizeof(double), cudaMemcpyDeviceToDevice, g->stream);
  return e;
}

cudaError_t enqueue_backward(GpuBpfGrad* g, const BwdKey& bk) {
  const FwdKey& k = bk.f;
  const int T = k.T, N = g->N, K = g->K;
  const ObsModel obs = make_obs(k.nu);
  const int nui = nu_int_of(k.nu_state);
  cudaError_t e = cudaMemsetAsync(g->acc, 0, (size_t)g->G1 * kGradAcc * sizeof(double), g->stream);
  const int nseg = (T + K - 1) / K;
  for (int s = nseg - 1; s >= 0 && e == cudaSuccess; --s) {
    const int c = s * K, last = std::min(c + K, T) - 1;
    // recompute h_c .. h_last into seg[0 .. last-c]
    e = launch_grad_seed(N, g->ckpt + (size_t)s * g->ckpt_stride, g->seg, g->pcs[c], c > 0 ? 1 : 0, k.mu, k.rho,
                         k.sigma, nui, k.nu_state, g->stream, g->pdl);
    for (int t = c + 1; t <= last && e == cudaSuccess; ++t)
      e = launch_grad_recompute(N, g->csr + (size_t)(t - 1) * g->N4, g->seg + (size_t)(t - 1 - c) * g->N4,
                                g->seg + (size_t)(t - c) * g->N4, g->pcs[t], k.mu, k.rho, k.sigma, nui,
                                k.nu_state, g->stream, g->pdl);
    // adjoint last .. c
    for (int t = last; t >= c && e == cudaSuccess; --t) {
      GradAdjArgs a{};
      a.N = N;
      a.mu = k.mu; a.rho = k.rho; a.sigma = k.sigma;
      a.obs = obs;
      a.y = k.y + t;
      a.h = g->seg + (size_t)(t - c) * g->N4;
      a.csr = (t < T - 1) ? g->csr + (size_t)t * g->N4 : nullptr;
      a.lam_next = (t < T - 1) ? g->lam[(t + 1) & 1] : nullptr;
      a.lam = g->lam[t & 1];
      a.aux = g->aux + t;
      a.pc_next = g->pcs[t + 1];
      a.pc0 = g->pcs[0];
      a.first = (t == 0);
      a.nu_int = nui;
      a.nu_state = k.nu_state;
      a.acc = g->acc;
      e = launch_grad_adjoint(a, g->stream, g->pdl);
    }
  }
  if (e == cudaSuccess) e = launch_grad_finish(g->G1, g->acc, k.mu, k.rho, k.sigma, bk.grad, g->stream, g->pdl);
  return e;
}

template <typename F>
cudaError_t capture(GpuBpfGrad* g, cudaGraphExec_t* exec, F&& body) {
  cudaGraph_t gr = nullptr;
  cudaError_t e = cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  cudaError_t eb = body();
  cudaError_t ec = cudaStreamEndCapture(g->stream, &gr);
  if (eb != cudaSuccess || ec != cudaSuccess) {
    if (gr) cudaGraphDestroy(gr);
    cudaGetLastError();
    return eb != cudaSuccess ? eb : ec;
  }
  e = install_graph(exec, gr);
  cudaGraphDestroy(gr);
  return e;
}

}  // namespace

extern "C" {

size_t gpu_bpf_grad_tape_bytes(int n_particles, int max_ticks, int checkpoint_every) {
  if (n_particles <= 0 || max_ticks <= 0) return 0;
  const int K = checkpoint_every > 0 ? checkpoint_every : kDefaultCheckpoint;
  const size_t N4 = (size_t)grad_stride(n_particles);
  const size_t G = (size_t)((n_particles + kTile - 1) / kTile) * kTile;
  const size_t n_ckpt = (size_t)((max_ticks + K - 1) / K);
  return (size_t)max_ticks * N4 * 4 + n_ckpt * G * 4 + (size_t)max_ticks * (sizeof(float2) + sizeof(BpfTickRecord)) +
         (size_t)K * N4 * 4 + 2 * N4 * 4 + (size_t)grad_ctas(n_particles) * kGradAcc * 8;
}

GpuBpfGrad* gpu_bpf_grad_create(int n_particles, int max_ticks, int checkpoint_every) {
  bpf_record_error(BPF_OK);
  if (n_particles <= 0 || n_particles > (1 << 30) || max_ticks <= 0 || checkpoint_every < 0) {
    bpf_record_error(BPF_ERR_ARG);
    return nullptr;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    bpf_record_error(BPF_ERR_NODEVICE);
    return nullptr;
  }
  GpuBpfGrad* g = new GpuBpfGrad();
  auto fail = [&](cudaError_t e) -> GpuBpfGrad* {
    cudaGetLastError();
    bpf_record_error(e == cudaErrorMemoryAllocation ? BPF_ERR_ALLOC : BPF_ERR_CUDA);
    free_grad(g);
    return nullptr;
  };
  cudaError_t e = cudaGetDevice(&g->device);
  if (e != cudaSuccess) return fail(e);
  g->N = n_particles;
  g->G1 = grad_ctas(n_particles);
  g->N4 = grad_stride(n_particles);
  g->T_max = max_ticks;
  g->K = checkpoint_every > 0 ? checkpoint_every : kDefaultCheckpoint;
  g->n_ckpt = (max_ticks + g->K - 1) / g->K;
  if (const char* v = std::getenv("BPF_DISABLE_PDL")) g->pdl = (v[0] == '0');
  if ((e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
  if ((e = plan_alloc(g->plan, n_particles)) != cudaSuccess) return fail(e);
  g->ckpt_stride = (size_t)g->plan.G * kTile;
  g->pass2_grid = pass2_grid_size(g->device);
  const size_t N4 = (size_t)g->N4;
  auto al = [&](auto** p, size_t bytes) { if (e == cudaSuccess) e = bpf_malloc(p, bytes); };
  al(&g->csr, (size_t)max_ticks * N4 * sizeof(int32_t));
  al(&g->ckpt, (size_t)g->n_ckpt * g->ckpt_stride * sizeof(float));
  al(&g->aux, (size_t)max_ticks * sizeof(float2));
  al(&g->rec, (size_t)max_ticks * sizeof(BpfTickRecord));
  al(&g->seg, (size_t)g->K * N4 * sizeof(float));
  al(&g->lam[0], N4 * sizeof(float));
  al(&g->lam[1], N4 * sizeof(float));
  al(&g->acc, (size_t)g->G1 * kGradAcc * sizeof(double));
  if (e != cudaSuccess) return fail(e);
  return g;
}

void gpu_bpf_grad_destroy(GpuBpfGrad* g) {
  if (!g) return;
  ensure_dev(g);
  cudaStreamSynchronize(g->stream);
  free_grad(g);
}

void* gpu_bpf_grad_stream(GpuBpfGrad* g) { return g ? (void*)g->stream : nullptr; }

int gpu_bpf_grad_checkpoint_every(GpuBpfGrad* g) { return g ? g->K : -bpf_record_error(BPF_ERR_STATE); }

int gpu_bpf_grad_forward(GpuBpfGrad* g, float mu, float rho, float sigma_z, float nu_state, float nu_obs, int seed,
                         float ess_threshold, const float* y_dev, int n_ticks, double* loglik_dev) {
  if (!g) return bpf_record_error(BPF_ERR_STATE);
  if (!y_dev || !loglik_dev || n_ticks <= 0 || n_ticks > g->T_max) return bpf_record_error(BPF_ERR_ARG);
  if (!std::isfinite(mu) || !std::isfinite(rho) || !std::isfinite(sigma_z) || !(std::fabs(rho) < 1.0f) ||
      !(sigma_z > 0.0f) || !(nu_obs >= 0.0f) || !std::isfinite(nu_obs) ||
      !(nu_state == 0.0f || (nu_state >= 0.5f && std::isfinite(nu_state))))
    return bpf_record_error(BPF_ERR_ARG);
  if (ess_threshold != 0.0f) return bpf_record_error(BPF_ERR_UNSUPPORTED);   // always-resample tapes only
  int rc = ensure_dev(g);
  if (rc) return rc;
  FwdKey k;
  k.T = n_ticks; k.seed = seed; k.mu = mu; k.rho = rho; k.sigma = sigma_z; k.nu = nu_obs; k.nu_state = nu_state;
  k.y = y_dev; k.ll = loglik_dev;
  if (!g->fgraph || !(g->fkey == k)) {
    GCK(capture(g, &g->fgraph, [&]() { return enqueue_forward(g, k); }));
    g->fkey = k;
  }
  GCK(cudaGraphLaunch(g->fgraph, g->stream));
  bpf_note_launches(1 + 3LL * n_ticks);
  g->cur = k;
  g->have_fwd = true;
  g->pcs.resize(n_ticks + 1);
  uint64_t At = 1ull, Bt = 0ull;
  for (int t = 0; t <= n_ticks; ++t) {
    g->pcs[t] = pcg_tick_consts(seed, At, Bt);
    At *= kPcgMult;
    Bt = Bt * kPcgMult + 1ull;
  }
  return BPF_OK;
}

int gpu_bpf_grad_backward(GpuBpfGrad* g, double* grad_dev) {
  if (!g) return bpf_record_error(BPF_ERR_STATE);
  if (!grad_dev) return bpf_record_error(BPF_ERR_ARG);
  if (!g->have_fwd) return bpf_record_error(BPF_ERR_STATE);
  int rc = ensure_dev(g);
  if (rc) return rc;
  BwdKey bk;
  bk.f = g->cur;
  bk.grad = grad_dev;
  if (!g->bgraph || !(g->bkey == bk)) {
    GCK(capture(g, &g->bgraph, [&]() { return enqueue_backward(g, bk); }));
    g->bkey = bk;
  }
  GCK(cudaGraphLaunch(g->bgraph, g->stream));
  const int T = g->cur.T;
  bpf_note_launches(2LL * T + 1);
  return BPF_OK;
}

int gpu_bpf_grad_replay(GpuBpfGrad* g, double mu, double rho, double sigma_z, double* out_dev,
                        double* per_tick_dev) {
  if (!g) return bpf_record_error(BPF_ERR_STATE);
  if (!out_dev) return bpf_record_error(BPF_ERR_ARG);
  if (!g->have_fwd) return bpf_record_error(BPF_ERR_STATE);
  if (!std::isfinite(mu) || !std::isfinite(rho) || !std::isfinite(sigma_z) || !(std::fabs(rho) < 1.0) ||
      !(sigma_z > 0.0))
    return bpf_record_error(BPF_ERR_ARG);
  int rc = ensure_dev(g);
  if (rc) return rc;
  const size_t N4 = (size_t)g->N4;
  cudaError_t e = cudaSuccess;
  auto al = [&](auto** p, size_t bytes) { if (e == cudaSuccess && !*p) e = bpf_malloc(p, bytes); };
  al(&g->rs[0], 4 * N4 * sizeof(double));
  al(&g->rs[1], 4 * N4 * sizeof(double));
  al(&g->part, (size_t)g->T_max * g->G1 * 5 * sizeof(double));
  al(&g->per_tick, (size_t)g->T_max * 4 * sizeof(double));
  al(&g->rtotal, 4 * sizeof(double));
  GCK(e);
  const FwdKey& k = g->cur;
  ReplayArgs a{};
  a.N = g->N;
  a.mu = mu; a.rho = rho; a.sigma = sigma_z;
  a.obs = make_obs(k.nu);
  a.nu_int = nu_int_of(k.nu_state);
  a.nu_state = k.nu_state;
  a.stride = g->N4;
  for (int t = 0; t < k.T; ++t) {
    a.y = k.y + t;
    a.pc = g->pcs[t];
    a.part = g->part + (size_t)t * g->G1 * 5;
    a.hc = g->rs[t & 1];
    if (t == 0) {
      a.csr = nullptr; a.hp = nullptr;
      GCK(launch_replay_init(a, g->stream));
    } else {
      a.csr = g->csr + (size_t)(t - 1) * g->N4;
      a.hp = g->rs[(t - 1) & 1];
      GCK(launch_replay_tick(a, g->stream));
    }
  }
  GCK(launch_replay_reduce(k.T, g->G1, g->part, std::log((double)g->N), g->per_tick, g->rtotal, g->stream));
  GCK(cudaMemcpyAsync(out_dev, g->rtotal, 4 * sizeof(double), cudaMemcpyDeviceToDevice, g->stream));
  if (per_tick_dev)
    GCK(cudaMemcpyAsync(per_tick_dev, g->per_tick, (size_t)k.T * 4 * sizeof(double), cudaMemcpyDeviceToDevice,
                        g->stream));
  bpf_note_launches(k.T + 2LL);
  return BPF_OK;
}

int gpu_bpf_grad_get_records(GpuBpfGrad* g, BpfTickRecord* out, int n) {
  if (!g || !g->have_fwd) return bpf_record_error(BPF_ERR_STATE);
  if (!out || n < 0 || n > g->cur.T) return bpf_record_error(BPF_ERR_ARG);
  int rc = ensure_dev(g);
  if (rc) return rc;
  GCK(cudaStreamSynchronize(g->stream));
  GCK(cudaMemcpy(out, g->rec, (size_t)n * sizeof(BpfTickRecord), cudaMemcpyDeviceToHost));
  return BPF_OK;
}

int gpu_bpf_grad_get_children(GpuBpfGrad* g, int tick, int32_t* first_child) {
  if (!g || !g->have_fwd) return bpf_record_error(BPF_ERR_STATE);
  if (!first_child || tick < 0 || tick >= g->cur.T) return bpf_record_error(BPF_ERR_ARG);
  int rc = ensure_dev(g);
  if (rc) return rc;
  GCK(cudaStreamSynchronize(g->stream));
  GCK(cudaMemcpy(first_child, g->csr + (size_t)tick * g->N4, (size_t)g->N * sizeof(int32_t),
                 cudaMemcpyDeviceToHost));
  return BPF_OK;
}

}  // extern "C"
