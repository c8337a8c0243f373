// bpf_batch_internal.cuh — the batch object shared by the batched filter's
// entry points (bpf_batch_api.cu) and the SMC^2 driver built on it (bpf_smc2.cu).
// Not part of the public C ABI.
#pragma once
#include <algorithm>
#include <vector>

#include "bpf_batch.cuh"
#include "bpf_plain.cuh"

using namespace bpf;

namespace bpf_batch_detail {

constexpr int kClasses = 5;
constexpr int kClassMaxN[kClasses] = {1024, 2048, 4096, 8192, 16384};
constexpr int kDefaultThreads[kClasses] = {256, 256, 512, 512, 1024};
constexpr int kThreadChoices[] = {64, 128, 256, 512, 1024};

#define BCK(call)                                                             \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      cudaGetLastError();                                                     \
      return bpf_record_error(e_ == cudaErrorMemoryAllocation ? BPF_ERR_ALLOC : BPF_ERR_CUDA); \
    }                                                                         \
  } while (0)

// Correlated-noise fields of a run (BatchArgs::nz_*); out == nullptr: none.
struct NoiseArgs {
  const float* in = nullptr;
  float* out = nullptr;
  const long long* in_off = nullptr;
  const long long* out_off = nullptr;
  float rho = 0.0f, scale = 1.0f;
  bool operator==(const NoiseArgs& o) const {
    return in == o.in && out == o.out && in_off == o.in_off && out_off == o.out_off && rho == o.rho &&
           scale == o.scale;
  }
};

struct GraphKey {
  const float* y = nullptr;
  int T = 0;
  int y_abs = 0;
  double* loglik = nullptr;
  double* dll = nullptr;
  float* hmean = nullptr;
  int32_t* anc = nullptr;
  float* particles = nullptr;
  int threads[kClasses] = {0, 0, 0, 0, 0};
  NoiseArgs nz;
  bool operator==(const GraphKey& o) const {
    return y == o.y && T == o.T && y_abs == o.y_abs && loglik == o.loglik && dll == o.dll && hmean == o.hmean &&
           anc == o.anc &&
           particles == o.particles && std::equal(threads, threads + kClasses, o.threads) && nz == o.nz;
  }
};

}  // namespace bpf_batch_detail
using namespace bpf_batch_detail;

struct GpuBpfBatch {
  int device = 0;
  int B = 0;
  float ess_threshold = 0.0f;
  int sms = 0;
  BatchFilterDev* d_filters = nullptr;
  int* d_order = nullptr;
  int* d_counters = nullptr;
  float* d_hfinal = nullptr;
  int* d_resamples = nullptr;
  double* d_loglik = nullptr;
  float* d_y = nullptr;
  int y_cap = 0;
  int class_off[kClasses] = {0, 0, 0, 0, 0};
  int class_cnt[kClasses] = {0, 0, 0, 0, 0};
  int threads[kClasses];
  int grid[kClasses] = {1, 1, 1, 1, 1};
  cudaStream_t stream = nullptr;
  cudaStream_t cls_stream[kClasses] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kClasses] = {};
  cudaGraphExec_t graph = nullptr;
  GraphKey key;
  std::vector<int> n_of;      // particle count per filter
  std::vector<float> nus_of;  // Student-t state noise dof per filter (0 = Gaussian)

  // correlated-noise runs: per-filter area offsets of gpu_bpf_batch_run_correlated (for nz_T
  // ticks), and the noise fields resumable steps run with (NoiseArgs::out null: none)
  long long* d_nzoff = nullptr;
  int nz_T = 0;
  NoiseArgs step_nz;

  // gradient runs: per-class tape for the class's CTA slots, PCG jump table, graph
  unsigned char* g_tape[kClasses] = {};
  size_t g_tape_bytes[kClasses] = {0, 0, 0, 0, 0};
  int g_grid[kClasses] = {1, 1, 1, 1, 1};
  ulonglong2* d_AB = nullptr;
  int ab_T = 0;
  cudaGraphExec_t ggraph = nullptr;
  GraphKey gkey;
  double* gkey_grad = nullptr;

  // resumable stepping (allocated on the first step): per-filter state, particle and
  // carried-weight arrays, the device tick counter and the step graph
  BatchFilterState* d_st = nullptr;
  float* d_sth = nullptr;
  float* d_stw = nullptr;
  long long* d_stoff = nullptr;
  int* d_tick = nullptr;
  int* d_scounters = nullptr;       // work counters of the step path ([kClasses]) and its done counter;
                                    // zero between step launches (reset by each launch's last CTA)
  int host_tick = 0;
  cudaGraphExec_t sgraph = nullptr;
  GraphKey skey;
};

// Internal helpers of bpf_batch_api.cu used by the SMC^2 driver.
int batch_prepare_steps(GpuBpfBatch* b);
// Step every filter n ticks, reading y[t] at the absolute tick t (y_base = the series' start).
int batch_step_abs(GpuBpfBatch* b, const float* y_base, int n, double* dll_dev);
// Device tick counter of resumable steps (host mirror updated too).
int batch_set_tick(GpuBpfBatch* b, int tick);
// Replace every filter's parameters and seed (particle counts unchanged); waits.
int batch_set_filters(GpuBpfBatch* b, const BpfBatchFilter* filters);
// BPF_OK if every filter can run with correlated noise (one tile, Gaussian state noise).
int batch_check_correlated(const GpuBpfBatch* b);
