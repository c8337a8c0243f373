// bpf_batch_api.cu — extern "C" entry points of the batched filter
// (include/gpu_bpf.h, "Batched filters").
//
// Filters are grouped into five size classes by particle count (at most
// 1024, 2048, 4096, 8192, 16384). Each class runs as one persistent launch
// whose CTAs pull filters from a work counter in LPT order (largest N
// first); the classes run concurrently on their own streams, forked from and
// joined to the batch stream, and a whole run is replayed as one CUDA graph.
// The threads per CTA of every class are the tile shape the autotuner picks.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "bpf_batch.cuh"
#include "bpf_plain.cuh"

using namespace bpf;

#include "bpf_batch_internal.cuh"


namespace {

void free_batch(GpuBpfBatch* b) {
  if (!b) return;
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->ggraph) cudaGraphExecDestroy(b->ggraph);
  if (b->sgraph) cudaGraphExecDestroy(b->sgraph);
  bpf_free(b->d_st); bpf_free(b->d_sth); bpf_free(b->d_stw); bpf_free(b->d_stoff); bpf_free(b->d_tick);
  bpf_free(b->d_scounters);
  for (int c = 0; c < kClasses; ++c) bpf_free(b->g_tape[c]);
  bpf_free(b->d_AB);
  bpf_free(b->d_nzoff);
  bpf_free(b->d_filters); bpf_free(b->d_order); bpf_free(b->d_counters);
  bpf_free(b->d_hfinal); bpf_free(b->d_resamples); bpf_free(b->d_loglik); bpf_free(b->d_y);
  for (int c = 0; c < kClasses; ++c) {
    if (b->cls_stream[c]) cudaStreamDestroy(b->cls_stream[c]);
    if (b->join[c]) cudaEventDestroy(b->join[c]);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

int class_of(int n) {
  for (int c = 0; c < kClasses; ++c)
    if (n <= kClassMaxN[c]) return c;
  return -1;
}

BatchArgs class_args(GpuBpfBatch* b, int c, const float* y, int T, double* loglik, double* dll, float* hmean,
                     int32_t* anc, float* particles, const NoiseArgs* nz = nullptr) {
  BatchArgs a{};
  if (nz && nz->out) {
    a.nz_in = nz->in; a.nz_out = nz->out; a.nz_in_off = nz->in_off; a.nz_out_off = nz->out_off;
    a.cp_rho = nz->rho; a.cp_scale = nz->scale;
  }
  a.filters = b->d_filters;
  a.order = b->d_order + b->class_off[c];
  a.n_order = b->class_cnt[c];
  a.counter = b->d_counters + c;
  a.y = y;
  a.T = T;
  a.ess_threshold = b->ess_threshold;
  a.loglik = loglik;
  a.dll = dll;
  a.hmean = hmean;
  a.h_final = b->d_hfinal;
  a.resamples = b->d_resamples;
  a.anc = anc;
  a.particles = particles;
  return a;
}

// Grid of every class for its current CTA shape (sets the kernel attributes).
void configure_classes(GpuBpfBatch* b) {
  for (int c = 0; c < kClasses; ++c) {
    const int occ = std::max(1, batch_occupancy(b->threads[c], kClassMaxN[c]));
    b->grid[c] = std::max(1, std::min(b->class_cnt[c], b->sms * occ));
  }
}

// Enqueue one run: zero the work counters, fork the classes (largest first),
// join them back onto the batch stream.
cudaError_t enqueue_run(GpuBpfBatch* b, const float* y, int T, double* loglik, double* dll, float* hmean,
                        int32_t* anc, float* particles, int only_class = -1, const NoiseArgs* nz = nullptr) {
  cudaError_t e = cudaMemsetAsync(b->d_counters, 0, kClasses * sizeof(int), b->stream);
  if (e != cudaSuccess) return e;
  e = cudaEventRecord(b->fork, b->stream);
  if (e != cudaSuccess) return e;
  for (int c = kClasses - 1; c >= 0; --c) {
    if (!b->class_cnt[c] || (only_class >= 0 && c != only_class)) continue;
    e = cudaStreamWaitEvent(b->cls_stream[c], b->fork, 0);
    if (e == cudaSuccess)
      e = launch_batch_class(class_args(b, c, y, T, loglik, dll, hmean, anc, particles, nz), b->threads[c],
                             kClassMaxN[c], b->grid[c], b->cls_stream[c]);
    if (e == cudaSuccess) e = cudaEventRecord(b->join[c], b->cls_stream[c]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join[c], 0);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

constexpr int kGradK = 8;   // checkpoint interval of batched gradient runs

// Per-slot tape layout of class c for T ticks (see BatchArgs::g_*).
struct SlotLayout {
  size_t list, ckpt, norm, seg, total;   // byte offsets inside one slot, and the slot size
};
SlotLayout slot_layout(int maxn, int T) {
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t nck = (size_t)((T + kGradK - 1) / kGradK);
  SlotLayout L;
  L.list = 0;
  L.ckpt = al((size_t)T * maxn * sizeof(unsigned short));
  L.norm = L.ckpt + al(nck * maxn * sizeof(float));
  L.seg = L.norm + al((size_t)T * sizeof(float2));
  L.total = L.seg + al((size_t)kGradK * maxn * sizeof(float));
  return L;
}

// Grid of every class's gradient kernel and its tape for T ticks.
int prepare_grad(GpuBpfBatch* b, int T) {
  for (int c = 0; c < kClasses; ++c) {
    if (!b->class_cnt[c]) continue;
    const int occ = std::max(1, batch_grad_occupancy(b->threads[c], kClassMaxN[c]));
    b->g_grid[c] = std::max(1, std::min(b->class_cnt[c], b->sms * occ));
    const size_t need = slot_layout(kClassMaxN[c], T).total * (size_t)b->g_grid[c];
    if (b->g_tape_bytes[c] < need) {
      bpf_free(b->g_tape[c]);
      b->g_tape[c] = nullptr;
      b->g_tape_bytes[c] = 0;
      BCK(bpf_malloc(&b->g_tape[c], need));
      b->g_tape_bytes[c] = need;
    }
  }
  if (b->ab_T < T + 1) {
    bpf_free(b->d_AB);
    b->d_AB = nullptr;
    b->ab_T = 0;
    BCK(bpf_malloc(&b->d_AB, (size_t)(T + 1) * sizeof(ulonglong2)));
    std::vector<ulonglong2> ab(T + 1);
    unsigned long long At = 1ull, Bt = 0ull;
    for (int t = 0; t <= T; ++t) {
      ab[t].x = At; ab[t].y = Bt;
      At *= kPcgMult;
      Bt = Bt * kPcgMult + 1ull;
    }
    BCK(cudaMemcpy(b->d_AB, ab.data(), (size_t)(T + 1) * sizeof(ulonglong2), cudaMemcpyHostToDevice));
    b->ab_T = T + 1;
  }
  return BPF_OK;
}

cudaError_t enqueue_grad(GpuBpfBatch* b, const float* y, int T, double* loglik, double* grad) {
  cudaError_t e = cudaMemsetAsync(b->d_counters, 0, kClasses * sizeof(int), b->stream);
  if (e != cudaSuccess) return e;
  e = cudaEventRecord(b->fork, b->stream);
  if (e != cudaSuccess) return e;
  for (int c = kClasses - 1; c >= 0; --c) {
    if (!b->class_cnt[c]) continue;
    BatchArgs a = class_args(b, c, y, T, loglik, nullptr, nullptr, nullptr, nullptr);
    const SlotLayout L = slot_layout(kClassMaxN[c], T);
    // slot-major tape: every field is an array over slots with the per-slot stride the kernel uses
    unsigned char* base = b->g_tape[c];
    const size_t slots = (size_t)b->g_grid[c];
    a.g_list = reinterpret_cast<unsigned short*>(base);
    a.g_ckpt = reinterpret_cast<float*>(base + slots * L.ckpt);
    a.g_norm = reinterpret_cast<float2*>(base + slots * L.norm);
    a.g_seg = reinterpret_cast<float*>(base + slots * L.seg);
    a.g_AB = b->d_AB;
    a.g_K = kGradK;
    a.grad = grad;
    e = cudaStreamWaitEvent(b->cls_stream[c], b->fork, 0);
    if (e == cudaSuccess)
      e = launch_batch_grad_class(a, b->threads[c], kClassMaxN[c], b->g_grid[c], b->cls_stream[c]);
    if (e == cudaSuccess) e = cudaEventRecord(b->join[c], b->cls_stream[c]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join[c], 0);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace

int batch_prepare_steps(GpuBpfBatch* b) {
  if (b->d_st) return BPF_OK;
  std::vector<long long> off(b->B);
  long long tot = 0;
  for (int i = 0; i < b->B; ++i) { off[i] = tot; tot += (b->n_of[i] + 3) & ~3; }
  BCK(bpf_malloc(&b->d_st, (size_t)b->B * sizeof(BatchFilterState)));
  BCK(bpf_malloc(&b->d_sth, (size_t)tot * sizeof(float)));
  BCK(bpf_malloc(&b->d_stw, (size_t)tot * sizeof(float)));
  BCK(bpf_malloc(&b->d_stoff, (size_t)b->B * sizeof(long long)));
  BCK(bpf_malloc(&b->d_tick, sizeof(int)));
  BCK(bpf_malloc(&b->d_scounters, (kClasses + 1) * sizeof(int)));
  BCK(cudaMemcpy(b->d_stoff, off.data(), (size_t)b->B * sizeof(long long), cudaMemcpyHostToDevice));
  BCK(cudaMemset(b->d_tick, 0, sizeof(int)));
  BCK(cudaMemset(b->d_scounters, 0, (kClasses + 1) * sizeof(int)));
  b->host_tick = 0;
  return BPF_OK;
}

namespace {

// Advance every filter by T ticks from its saved state (tick 0 = fresh start).
// The step path has its own work counters, left at zero by every step launch
// (the last CTA resets them and advances the device tick), so the captured step
// holds the class kernels alone.
cudaError_t enqueue_step(GpuBpfBatch* b, const float* y, int T, double* dll, float* hmean, int y_abs) {
  cudaError_t e = cudaEventRecord(b->fork, b->stream);
  if (e != cudaSuccess) return e;
  int ctas = 0;
  for (int c = 0; c < kClasses; ++c) if (b->class_cnt[c]) ctas += b->grid[c];
  for (int c = kClasses - 1; c >= 0; --c) {
    if (!b->class_cnt[c]) continue;
    BatchArgs a = class_args(b, c, y, T, b->d_loglik, dll, hmean, nullptr, nullptr, &b->step_nz);
    a.t0_dev = b->d_tick;
    a.st = b->d_st;
    a.st_h = b->d_sth;
    a.st_w = b->d_stw;
    a.st_off = b->d_stoff;
    a.y_abs = y_abs;
    a.counter = b->d_scounters + c;
    a.ep_done = b->d_scounters + kClasses;
    a.ep_counters = b->d_scounters;
    a.ep_tick = b->d_tick;
    a.ep_total = ctas;
    a.ep_n = kClasses;
    a.ep_add = T;
    e = cudaStreamWaitEvent(b->cls_stream[c], b->fork, 0);
    if (e == cudaSuccess) e = launch_batch_class(a, b->threads[c], kClassMaxN[c], b->grid[c], b->cls_stream[c]);
    if (e == cudaSuccess) e = cudaEventRecord(b->join[c], b->cls_stream[c]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, b->join[c], 0);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

int ensure_device_b(GpuBpfBatch* b) {
  int cur = -1;
  BCK(cudaGetDevice(&cur));
  if (cur != b->device) BCK(cudaSetDevice(b->device));
  return BPF_OK;
}

std::string gpu_key(int device) {
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return "unknown";
  std::string s = p.name;
  for (char& ch : s) if (ch == ' ' || ch == '"') ch = '_';
  return s + "_sm" + std::to_string(p.multiProcessorCount);
}

// Autotune cache: one line per entry, "<gpu_key> <class> <threads>".
bool cache_lookup(const char* path, const std::string& key, int cls, int* threads) {
  if (!path) return false;
  std::ifstream in(path);
  std::string k;
  int c, t;
  bool found = false;
  while (in >> k >> c >> t)
    if (k == key && c == cls) { *threads = t; found = true; }
  return found;
}
void cache_store(const char* path, const std::string& key, int cls, int threads) {
  if (!path) return;
  std::ofstream out(path, std::ios::app);
  out << key << " " << cls << " " << threads << "\n";
}

}  // namespace

// Device table entry of one filter; false for invalid parameters.
static bool make_filter_dev(const BpfBatchFilter& f, BatchFilterDev* out) {
  if (f.n_particles <= 0 || f.n_particles > kBatchMaxN || !std::isfinite(f.mu) || !std::isfinite(f.rho) ||
      !std::isfinite(f.sigma_z) || !(std::fabs(f.rho) < 1.0f) || !(f.sigma_z > 0.0f) || !std::isfinite(f.nu_obs) ||
      !(f.nu_obs >= 0.0f) || !(f.nu_state == 0.0f || (f.nu_state >= 0.5f && std::isfinite(f.nu_state))))
    return false;
  BatchFilterDev d{};
  d.mu = f.mu; d.rho = f.rho; d.sigma = f.sigma_z;
  d.std_stat = sqrtf((f.sigma_z * f.sigma_z) / fmaxf(1.0f - f.rho * f.rho, 1e-6f));   // gpu_bpf_ptx_full.cu:430
  d.nu = f.nu_obs;
  if (f.nu_obs > 0.0f) {
    d.c_obs = (float)(std::lgamma((f.nu_obs + 1.0) / 2.0) - std::lgamma(f.nu_obs / 2.0) -
                      0.5 * std::log(f.nu_obs * 3.14159265358979323846));
    d.inv_nu = 1.0f / f.nu_obs;
    d.nu_p1h = (f.nu_obs + 1.0f) * 0.5f;
  }
  d.n = f.n_particles;
  d.seed = f.seed;
  d.nu_int = (f.nu_state > 0.0f) ? (int)(f.nu_state + 0.5f) : 0;   // gpu_bpf_ptx_full.cu:392
  d.nu_state = f.nu_state;
  *out = d;
  return true;
}

int batch_set_filters(GpuBpfBatch* b, const BpfBatchFilter* filters) {
  if (!b) return bpf_record_error(BPF_ERR_STATE);
  if (!filters) return bpf_record_error(BPF_ERR_ARG);
  std::vector<BatchFilterDev> tab(b->B);
  for (int i = 0; i < b->B; ++i)
    if (filters[i].n_particles != b->n_of[i] || !make_filter_dev(filters[i], &tab[i])) return bpf_record_error(BPF_ERR_ARG);
  BCK(cudaMemcpyAsync(b->d_filters, tab.data(), (size_t)b->B * sizeof(BatchFilterDev), cudaMemcpyHostToDevice,
                      b->stream));
  BCK(cudaStreamSynchronize(b->stream));   // the host table goes out of scope
  for (int i = 0; i < b->B; ++i) b->nus_of[i] = filters[i].nu_state;
  return BPF_OK;
}

int batch_check_correlated(const GpuBpfBatch* b) {
  for (int i = 0; i < b->B; ++i)
    if (b->n_of[i] > kTile || b->nus_of[i] != 0.0f) return bpf_record_error(BPF_ERR_UNSUPPORTED);
  return BPF_OK;
}

extern "C" {

int gpu_bpf_batch_set_filters(GpuBpfBatch* b, const BpfBatchFilter* filters) {
  if (b) {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || (cur != b->device && cudaSetDevice(b->device) != cudaSuccess))
      return bpf_record_error(BPF_ERR_CUDA);
  }
  return batch_set_filters(b, filters);
}

GpuBpfBatch* gpu_bpf_batch_create(const BpfBatchFilter* filters, int n_filters, float ess_threshold) {
  if (!filters || n_filters <= 0 || std::isnan(ess_threshold)) { bpf_record_error(BPF_ERR_ARG); return nullptr; }
  std::vector<BatchFilterDev> tab(n_filters);
  for (int i = 0; i < n_filters; ++i)
    if (!make_filter_dev(filters[i], &tab[i])) {
      bpf_record_error(BPF_ERR_ARG);
      return nullptr;
    }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); bpf_record_error(BPF_ERR_NODEVICE); return nullptr; }

  GpuBpfBatch* b = new GpuBpfBatch();
  b->B = n_filters;
  b->ess_threshold = ess_threshold;
  std::copy(kDefaultThreads, kDefaultThreads + kClasses, b->threads);
  b->n_of.resize(n_filters);
  for (int i = 0; i < n_filters; ++i) b->n_of[i] = tab[i].n;
  b->nus_of.resize(n_filters);
  for (int i = 0; i < n_filters; ++i) b->nus_of[i] = filters[i].nu_state;
  // LPT order inside each class: largest N first
  std::vector<int> order(n_filters);
  for (int i = 0; i < n_filters; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    const int cx = class_of(tab[x].n), cy = class_of(tab[y].n);
    if (cx != cy) return cx < cy;
    return tab[x].n > tab[y].n;
  });
  for (int i = 0; i < n_filters; ++i) b->class_cnt[class_of(tab[order[i]].n)]++;
  for (int c = 1; c < kClasses; ++c) b->class_off[c] = b->class_off[c - 1] + b->class_cnt[c - 1];

  auto fail = [&](int code) { free_batch(b); bpf_record_error(code); return (GpuBpfBatch*)nullptr; };
  if (cudaGetDevice(&b->device) != cudaSuccess) return fail(BPF_ERR_CUDA);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(BPF_ERR_CUDA);
  for (int c = 0; c < kClasses; ++c) {
    if (cudaStreamCreateWithFlags(&b->cls_stream[c], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->join[c], cudaEventDisableTiming) != cudaSuccess)
      return fail(BPF_ERR_CUDA);
  }
  if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) return fail(BPF_ERR_CUDA);
  if (bpf_malloc(&b->d_filters, n_filters * sizeof(BatchFilterDev)) != cudaSuccess ||
      bpf_malloc(&b->d_order, n_filters * sizeof(int)) != cudaSuccess ||
      bpf_malloc(&b->d_counters, kClasses * sizeof(int)) != cudaSuccess ||
      bpf_malloc(&b->d_hfinal, n_filters * sizeof(float)) != cudaSuccess ||
      bpf_malloc(&b->d_resamples, n_filters * sizeof(int)) != cudaSuccess ||
      bpf_malloc(&b->d_loglik, n_filters * sizeof(double)) != cudaSuccess)
    return fail(BPF_ERR_ALLOC);
  if (cudaMemcpy(b->d_filters, tab.data(), n_filters * sizeof(BatchFilterDev), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->d_order, order.data(), n_filters * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(BPF_ERR_CUDA);
  configure_classes(b);
  return b;
}

void gpu_bpf_batch_destroy(GpuBpfBatch* b) {
  if (!b) return;
  ensure_device_b(b);
  cudaStreamSynchronize(b->stream);
  free_batch(b);
}

void* gpu_bpf_batch_stream(GpuBpfBatch* b) { return b ? (void*)b->stream : nullptr; }

int gpu_bpf_batch_size_class(int n_particles) { return class_of(n_particles); }

int gpu_bpf_batch_set_threads(GpuBpfBatch* b, int size_class, int threads) {
  if (!b || size_class < 0 || size_class >= kClasses) return bpf_record_error(BPF_ERR_ARG);
  bool ok = false;
  for (int t : kThreadChoices) ok |= (t == threads);
  if (!ok) return bpf_record_error(BPF_ERR_ARG);
  int rc = ensure_device_b(b);
  if (rc) return rc;
  if (batch_occupancy(threads, kClassMaxN[size_class]) < 1) return bpf_record_error(BPF_ERR_UNSUPPORTED);
  b->threads[size_class] = threads;
  configure_classes(b);
  return BPF_OK;
}

int gpu_bpf_batch_get_threads(GpuBpfBatch* b, int size_class) {
  if (!b || size_class < 0 || size_class >= kClasses) return -bpf_record_error(BPF_ERR_ARG);
  return b->threads[size_class];
}

int gpu_bpf_batch_run_device(GpuBpfBatch* b, const float* y_dev, int n_ticks, double* loglik_dev, double* dll_dev,
                             float* hmean_dev) {
  if (!b) return bpf_record_error(BPF_ERR_STATE);
  if (n_ticks <= 0 || !y_dev || !loglik_dev) return bpf_record_error(BPF_ERR_ARG);
  int rc = ensure_device_b(b);
  if (rc) return rc;
  GraphKey k;
  k.y = y_dev; k.T = n_ticks; k.loglik = loglik_dev; k.dll = dll_dev; k.hmean = hmean_dev;
  std::copy(b->threads, b->threads + kClasses, k.threads);
  if (!b->graph || !(k == b->key)) {
    if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
    cudaGraph_t g = nullptr;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_run(b, y_dev, n_ticks, loglik_dev, dll_dev, hmean_dev, nullptr, nullptr);
    cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) { if (g) cudaGraphDestroy(g); cudaGetLastError(); return bpf_record_error(BPF_ERR_CUDA); }
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { b->graph = nullptr; cudaGetLastError(); return bpf_record_error(BPF_ERR_CUDA); }
    b->key = k;
  }
  BCK(cudaGraphLaunch(b->graph, b->stream));
  bpf_note_launches(kClasses);
  return BPF_OK;
}

int gpu_bpf_batch_grad_run(GpuBpfBatch* b, const float* y_dev, int n_ticks, double* loglik_dev, double* grad_dev) {
  if (!b) return bpf_record_error(BPF_ERR_STATE);
  if (n_ticks <= 0 || !y_dev || !loglik_dev || !grad_dev) return bpf_record_error(BPF_ERR_ARG);
  if (b->ess_threshold != 0.0f) return bpf_record_error(BPF_ERR_UNSUPPORTED);   // always-resample tapes only
  int rc = ensure_device_b(b);
  if (rc) return rc;
  GraphKey k;
  k.y = y_dev; k.T = n_ticks; k.loglik = loglik_dev;
  std::copy(b->threads, b->threads + kClasses, k.threads);
  if (!b->ggraph || !(k == b->gkey) || b->gkey_grad != grad_dev) {
    if (b->ggraph) { cudaGraphExecDestroy(b->ggraph); b->ggraph = nullptr; }
    BCK(cudaStreamSynchronize(b->stream));           // a resized tape must not be in use
    rc = prepare_grad(b, n_ticks);
    if (rc) return rc;
    cudaGraph_t g = nullptr;
    BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_grad(b, y_dev, n_ticks, loglik_dev, grad_dev);
    cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess || e2 != cudaSuccess) { if (g) cudaGraphDestroy(g); cudaGetLastError(); return bpf_record_error(BPF_ERR_CUDA); }
    e = cudaGraphInstantiate(&b->ggraph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { b->ggraph = nullptr; cudaGetLastError(); return bpf_record_error(BPF_ERR_CUDA); }
    b->gkey = k;
    b->gkey_grad = grad_dev;
  }
  BCK(cudaGraphLaunch(b->ggraph, b->stream));
  bpf_note_launches(kClasses);
  return BPF_OK;
}

}  // extern "C"

static int step_common(GpuBpfBatch* b, const float* y_dev, int n_ticks, double* dll_dev, float* hmean_dev,
                       int y_abs) {
  if (!b) return bpf_record_error(BPF_ERR_STATE);
  if (n_ticks <= 0 || !y_dev) return bpf_record_error(BPF_ERR_ARG);
  int rc = ensure_device_b(b);
  if (rc) return rc;
  rc = batch_prepare_steps(b);
  if (rc) return rc;
  GraphKey k;
  k.y = y_dev; k.T = n_ticks; k.dll = dll_dev; k.hmean = hmean_dev; k.y_abs = y_abs;
  k.nz = b->step_nz;
  std::copy(b->threads, b->threads + kClasses, k.threads);
  // Only the observation / output pointers differ from the captured step (a caller
  // walking a device series tick by tick): launch the step directly instead of
  // capturing and instantiating a graph for every call.
  GraphKey shape = k;
  shape.y = b->skey.y; shape.dll = b->skey.dll; shape.hmean = b->skey.hmean;
  if (b->sgraph && !(k == b->skey) && shape == b->skey) {
    BCK(enqueue_step(b, y_dev, n_ticks, dll_dev, hmean_dev, y_abs));
  } else {
    if (!b->sgraph || !(k == b->skey)) {
      if (b->sgraph) { cudaGraphExecDestroy(b->sgraph); b->sgraph = nullptr; }
      cudaGraph_t g = nullptr;
      BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      cudaError_t e = enqueue_step(b, y_dev, n_ticks, dll_dev, hmean_dev, y_abs);
      cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
      if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return bpf_record_error(BPF_ERR_CUDA);
      }
      e = cudaGraphInstantiate(&b->sgraph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) { b->sgraph = nullptr; cudaGetLastError(); return bpf_record_error(BPF_ERR_CUDA); }
      b->skey = k;
    }
    BCK(cudaGraphLaunch(b->sgraph, b->stream));
  }
  int launched = 0;
  for (int c = 0; c < kClasses; ++c) launched += b->class_cnt[c] ? 1 : 0;
  bpf_note_launches(launched);
  b->host_tick += n_ticks;
  return BPF_OK;
}

int batch_step_abs(GpuBpfBatch* b, const float* y_base, int n, double* dll_dev) {
  return step_common(b, y_base, n, dll_dev, nullptr, 1);
}

int batch_set_tick(GpuBpfBatch* b, int tick) {
  int rc = batch_prepare_steps(b);
  if (rc) return rc;
  BCK(cudaMemcpyAsync(b->d_tick, &tick, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  b->host_tick = tick;
  return BPF_OK;
}

extern "C" {

int gpu_bpf_batch_step_device(GpuBpfBatch* b, const float* y_dev, int n_ticks, double* dll_dev, float* hmean_dev) {
  return step_common(b, y_dev, n_ticks, dll_dev, hmean_dev, 0);
}

int gpu_bpf_batch_reset(GpuBpfBatch* b) {
  if (!b) return bpf_record_error(BPF_ERR_STATE);
  int rc = ensure_device_b(b);
  if (rc) return rc;
  if (b->d_tick) BCK(cudaMemsetAsync(b->d_tick, 0, sizeof(int), b->stream));
  b->host_tick = 0;
  return BPF_OK;
}

int gpu_bpf_batch_tick(GpuBpfBatch* b) { return b ? b->host_tick : -bpf_record_error(BPF_ERR_STATE); }

double* gpu_bpf_batch_loglik_device(GpuBpfBatch* b) { return b ? b->d_loglik : nullptr; }

size_t gpu_bpf_batch_grad_tape_bytes(GpuBpfBatch* b, int n_ticks) {
  if (!b || n_ticks <= 0) return 0;
  size_t tot = 0;
  for (int c = 0; c < kClasses; ++c) {
    if (!b->class_cnt[c]) continue;
    const int occ = std::max(1, batch_grad_occupancy(b->threads[c], kClassMaxN[c]));
    const size_t slots = (size_t)std::max(1, std::min(b->class_cnt[c], b->sms * occ));
    tot += slots * slot_layout(kClassMaxN[c], n_ticks).total;
  }
  return tot + (size_t)(n_ticks + 1) * sizeof(ulonglong2);
}

int gpu_bpf_batch_run(GpuBpfBatch* b, const float* y, int n_ticks, double* loglik_out, float* hmean_last_out) {
  if (!b) return bpf_record_error(BPF_ERR_STATE);
  if (n_ticks <= 0 || !y || !loglik_out) return bpf_record_error(BPF_ERR_ARG);
  for (int t = 0; t < n_ticks; ++t) if (!std::isfinite(y[t])) return bpf_record_error(BPF_ERR_ARG);
  int rc = ensure_device_b(b);
  if (rc) return rc;
  if (b->y_cap < n_ticks) {
    bpf_free(b->d_y);
    b->d_y = nullptr;
    b->y_cap = 0;
    BCK(bpf_malloc(&b->d_y, n_ticks * sizeof(float)));
    b->y_cap = n_ticks;
  }
  BCK(cudaMemcpyAsync(b->d_y, y, n_ticks * sizeof(float), cudaMemcpyHostToDevice, b->stream));
  rc = gpu_bpf_batch_run_device(b, b->d_y, n_ticks, b->d_loglik, nullptr, nullptr);
  if (rc) return rc;
  BCK(cudaMemcpyAsync(loglik_out, b->d_loglik, b->B * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
  if (hmean_last_out)
    BCK(cudaMemcpyAsync(hmean_last_out, b->d_hfinal, b->B * sizeof(float), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return BPF_OK;
}

int gpu_bpf_batch_run_debug(GpuBpfBatch* b, const float* y_dev, int n_ticks, double* loglik_dev, double* dll_dev,
                            int32_t* anc_dev, float* particles_dev) {
  if (!b) return bpf_record_error(BPF_ERR_STATE);
  if (n_ticks <= 0 || !y_dev || !loglik_dev) return bpf_record_error(BPF_ERR_ARG);
  int rc = ensure_device_b(b);
  if (rc) return rc;
  BCK(enqueue_run(b, y_dev, n_ticks, loglik_dev, dll_dev, nullptr, anc_dev, particles_dev));
  bpf_note_launches(kClasses);
  return BPF_OK;
}

long long gpu_bpf_batch_noise_offset(GpuBpfBatch* b, int filter, int n_ticks) {
  if (!b || filter < 0 || filter > b->B || n_ticks <= 0) return -bpf_record_error(BPF_ERR_ARG);
  long long off = 0;
  for (int i = 0; i < filter; ++i) off += (long long)n_ticks * batch_noise_stride(b->n_of[i]);
  return off;
}

int gpu_bpf_batch_run_correlated(GpuBpfBatch* b, const float* y_dev, int n_ticks, const float* noise_in_dev,
                                 float* noise_out_dev, float rho, double* loglik_dev, double* dll_dev,
                                 int32_t* anc_dev) {
  if (!b) return bpf_record_error(BPF_ERR_STATE);
  if (n_ticks <= 0 || !y_dev || !loglik_dev || !noise_out_dev || noise_in_dev == noise_out_dev ||
      !(rho >= 0.0f && rho <= 1.0f))
    return bpf_record_error(BPF_ERR_ARG);
  int rc = batch_check_correlated(b);
  if (rc) return rc;
  rc = ensure_device_b(b);
  if (rc) return rc;
  if (b->nz_T != n_ticks) {
    BCK(cudaStreamSynchronize(b->stream));           // the old offsets may be in use
    std::vector<long long> off(b->B);
    for (int i = 0; i < b->B; ++i) off[i] = gpu_bpf_batch_noise_offset(b, i, n_ticks);
    if (!b->d_nzoff) BCK(bpf_malloc(&b->d_nzoff, (size_t)b->B * sizeof(long long)));
    BCK(cudaMemcpy(b->d_nzoff, off.data(), (size_t)b->B * sizeof(long long), cudaMemcpyHostToDevice));
    b->nz_T = n_ticks;
  }
  NoiseArgs nz;
  nz.in = noise_in_dev;
  nz.out = noise_out_dev;
  nz.in_off = b->d_nzoff;
  nz.out_off = b->d_nzoff;
  nz.rho = rho;
  nz.scale = sqrtf(fmaxf(0.0f, 1.0f - rho * rho));
  BCK(enqueue_run(b, y_dev, n_ticks, loglik_dev, dll_dev, nullptr, anc_dev, nullptr, -1, &nz));
  bpf_note_launches(kClasses);
  return BPF_OK;
}

int gpu_bpf_batch_resample_counts(GpuBpfBatch* b, int* counts_out, float* hmean_last_out) {
  if (!b || !counts_out) return bpf_record_error(BPF_ERR_ARG);
  int rc = ensure_device_b(b);
  if (rc) return rc;
  BCK(cudaMemcpyAsync(counts_out, b->d_resamples, b->B * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
  if (hmean_last_out)
    BCK(cudaMemcpyAsync(hmean_last_out, b->d_hfinal, b->B * sizeof(float), cudaMemcpyDeviceToHost, b->stream));
  BCK(cudaStreamSynchronize(b->stream));
  return BPF_OK;
}

int gpu_bpf_batch_autotune(GpuBpfBatch* b, const float* y, int n_ticks, const char* cache_path) {
  if (!b || !y || n_ticks <= 0) return bpf_record_error(BPF_ERR_ARG);
  int rc = ensure_device_b(b);
  if (rc) return rc;
  const std::string key = gpu_key(b->device);
  float* d_y = nullptr;
  double* d_ll = nullptr;
  BCK(bpf_malloc(&d_y, n_ticks * sizeof(float)));
  if (bpf_malloc(&d_ll, b->B * sizeof(double)) != cudaSuccess) { bpf_free(d_y); return bpf_record_error(BPF_ERR_ALLOC); }
  cudaMemcpy(d_y, y, n_ticks * sizeof(float), cudaMemcpyHostToDevice);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int result = BPF_OK;
  for (int c = 0; c < kClasses && result == BPF_OK; ++c) {
    if (!b->class_cnt[c]) continue;
    int cached = 0;
    if (cache_lookup(cache_path, key, c, &cached)) { b->threads[c] = cached; continue; }
    float best_ms = 1e30f;
    int best = b->threads[c];
    for (int t : kThreadChoices) {
      if (t > 4 * kClassMaxN[c] || batch_occupancy(t, kClassMaxN[c]) < 1) continue;
      b->threads[c] = t;
      configure_classes(b);
      float ms_min = 1e30f;
      for (int rep = 0; rep < 2; ++rep) {   // first repetition warms up
        cudaEventRecord(e0, b->stream);
        if (enqueue_run(b, d_y, n_ticks, d_ll, nullptr, nullptr, nullptr, nullptr, c) != cudaSuccess) {
          result = bpf_record_error(BPF_ERR_CUDA);
          break;
        }
        cudaEventRecord(e1, b->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep) ms_min = std::min(ms_min, ms);
      }
      if (result != BPF_OK) break;
      if (ms_min < best_ms) { best_ms = ms_min; best = t; }
    }
    b->threads[c] = best;
    configure_classes(b);
    if (result == BPF_OK) cache_store(cache_path, key, c, best);
  }
  configure_classes(b);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  bpf_free(d_y);
  bpf_free(d_ll);
  if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
  return result;
}

}  // extern "C"
