// bpf_static.cu — the allocation-free way to run the plain filter.
//
// Some callers may not allocate device memory while they run: hosts that
// reserve their whole GPU memory budget when they start (for example a
// trading or control loop sharing one GPU with other engines) and forbid any
// later allocation, and latency-critical loops that cannot afford cudaFree's
// implicit device synchronisation or the allocator's locks. For them,
// gpu_bpf_run_static runs a complete filter using only the file-scope device
// array below, which the CUDA module holds from the moment the library is
// loaded on a GPU until the process exits. No cudaMalloc, cudaFree or
// allocating library routine is called on this path.
#include <cmath>
#include <mutex>

#include "bpf_plain.cuh"

using namespace bpf;

namespace {

constexpr int kStaticMaxTiles = BPF_STATIC_MAX_PARTICLES / kTile;
constexpr int kStaticMaxItems =
    kStaticMaxTiles + (BPF_STATIC_MAX_PARTICLES + kOutChunk - 1) / kOutChunk + 1;
static_assert(BPF_STATIC_MAX_PARTICLES % kTile == 0, "static capacity is whole tiles");

// Layout of the scratch area: the same buffers a GpuBpfState allocates,
// sized for BPF_STATIC_MAX_PARTICLES. Every offset is a multiple of 16 bytes
// (bulk async copies of h and w tiles need 16-byte alignment).
struct StaticArea {
  float h0[BPF_STATIC_MAX_PARTICLES];
  float h1[BPF_STATIC_MAX_PARTICLES];
  float w[BPF_STATIC_MAX_PARTICLES];
  float4 rec[kStaticMaxTiles];
  unsigned long long E[kStaticMaxTiles];
  unsigned long long P[kStaticMaxTiles];
  int4 items[kStaticMaxItems];
  int nexp[kStaticMaxTiles];
  int ofirst[kStaticMaxTiles + 1];
  int pad_[3];
  DevState st;
};

// The scratch area itself (about 3 MiB).
static __device__ __align__(256) unsigned char g_static_scratch[sizeof(StaticArea)];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
StaticArea* g_area[kMaxDevices] = {};   // device address of g_static_scratch, per device
int g_pass2_grid[kMaxDevices] = {};

// Once per device, with that device current: the device address of the
// scratch array. In host code the symbol name is only a host-side handle, so
// the address must come from cudaGetSymbolAddress.
int static_setup(int dev, StaticArea** area, int* grid) {
  if (dev < 0 || dev >= kMaxDevices) return BPF_ERR_NODEVICE;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_area[dev]) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (e != cudaSuccess || !ptr) {
      cudaGetLastError();
      return (e == cudaErrorNoKernelImageForDevice || e == cudaErrorNoDevice) ? BPF_ERR_NODEVICE : BPF_ERR_CUDA;
    }
    g_pass2_grid[dev] = pass2_grid_size(dev);
    g_area[dev] = static_cast<StaticArea*>(ptr);
  }
  *area = g_area[dev];
  *grid = g_pass2_grid[dev];
  return BPF_OK;
}

}  // namespace

extern "C" int gpu_bpf_run_static(int n_particles, float rho, float sigma_z, float mu, float nu_obs, int seed,
                                  float ess_threshold, const float* y_dev, int n_ticks, BpfTickRecord* rec_dev,
                                  void* stream) {
  if (n_particles <= 0 || n_particles > BPF_STATIC_MAX_PARTICLES) return bpf_record_error(BPF_ERR_ARG);
  if (!std::isfinite(rho) || !std::isfinite(sigma_z) || !std::isfinite(mu) || !(std::fabs(rho) < 1.0f) ||
      !(sigma_z > 0.0f) || !std::isfinite(nu_obs) || !(nu_obs >= 0.0f) || std::isnan(ess_threshold))
    return bpf_record_error(BPF_ERR_ARG);
  if (n_ticks < 0 || (n_ticks > 0 && (!y_dev || !rec_dev))) return bpf_record_error(BPF_ERR_ARG);

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return bpf_record_error(BPF_ERR_NODEVICE); }
  StaticArea* area = nullptr;
  int grid = 0;
  const int rc = static_setup(dev, &area, &grid);
  if (rc != BPF_OK) return bpf_record_error(rc);

  Plan p{};
  p.N = n_particles;
  p.G = (n_particles + kTile - 1) / kTile;
  p.max_items = p.G + (n_particles + kOutChunk - 1) / kOutChunk + 1;
  p.h0 = area->h0; p.h1 = area->h1; p.w = area->w;
  p.nexp = area->nexp; p.E = area->E; p.rec = area->rec;
  p.P = area->P; p.ofirst = area->ofirst; p.items = area->items;
  p.st = &area->st;

  TickArgs a{};
  a.mu = mu; a.rho = rho; a.sigma = sigma_z;
  a.ess_threshold = ess_threshold;
  a.log_n = std::log((double)n_particles);
  a.obs.nu = nu_obs;
  if (nu_obs > 0.0f) {
    a.obs.c_obs = (float)(std::lgamma((nu_obs + 1.0) / 2.0) - std::lgamma(nu_obs / 2.0) -
                          0.5 * std::log(nu_obs * 3.14159265358979323846));
    a.obs.inv_nu = 1.0f / nu_obs;
    a.obs.nu_p1h = (nu_obs + 1.0f) * 0.5f;
  }
  a.anc = nullptr;

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The init kernel rewrites every particle buffer and the whole device tick
  // state, so no value survives from an earlier call; the per-tile arrays are
  // written each tick before anything reads them.
  const float std_stat = sqrtf((sigma_z * sigma_z) / fmaxf(1.0f - rho * rho, 1e-6f));
  cudaError_t e = launch_init(p, mu, std_stat, seed, s);
  for (int t = 0; t < n_ticks && e == cudaSuccess; ++t) {
    a.y_ptr = y_dev + t;
    a.rec = rec_dev + t;
    e = launch_pass1(p, a, s, true);
    if (e == cudaSuccess) e = launch_plan(p, a, s, true);
    if (e == cudaSuccess) e = launch_pass2(p, a, grid, s, true);
  }
  if (e != cudaSuccess) { cudaGetLastError(); return bpf_record_error(BPF_ERR_CUDA); }
  bpf_note_launches(1 + 3LL * n_ticks);
  return BPF_OK;
}
