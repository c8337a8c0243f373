// bpf_grad.cu — gradient kernels of the plain filter (sm_100a).
//
//   grad_seed       first tick of a checkpoint segment from the checkpoint
//   grad_recompute  one tick forward through the tape's child lists
//                   (parent-centric: every parent writes its children)
//   grad_adjoint    one tick backward: children sums of lambda_t+1, the new
//                   lambda_t and the per-CTA FP64 parameter adjoints
//   grad_finish     fixed-order sum of the per-CTA adjoints -> dL/dtheta
//   replay_*        FP64 re-run of the taped run at any theta with the same
//                   noise and the same child lists, carrying forward-mode
//                   tangents dh/dtheta: log-likelihood and its exact gradient
//                   for the finite-difference and forward-mode checks
//
// Every kernel assigns four consecutive parents to a thread (1024 per CTA).
// Their children are one contiguous run of slots; a thread walks its run
// alone unless it has more than kGradHeavy children, in which case its warp
// walks it together (lanes strided over the children, per-parent sums
// combined by a butterfly). Sums are in a fixed order, so results are
// deterministic run to run.
#include "bpf_grad.cuh"
#include "bpf_block.cuh"
#include <cmath>

namespace bpf {


// First child of each of the thread's four parents and the end of the last
// one's children: children of parent e are [f[e], f[e+1]). Parents at or past
// N have none. Entries are clamped to [0, N], so a child list that no
// resampling wrote (a tick whose weights all underflowed) can never send a
// walk outside the particle arrays.
__device__ __forceinline__ void load_children(const int32_t* __restrict__ csr, int N, int j0, int lane, int f[5]) {
  if (j0 + kGradGroup <= N) {
    const int4 v = *reinterpret_cast<const int4*>(csr + j0);
    f[0] = v.x; f[1] = v.y; f[2] = v.z; f[3] = v.w;
  } else {
#pragma unroll
    for (int e = 0; e < kGradGroup; ++e) f[e] = (j0 + e < N) ? csr[j0 + e] : N;
  }
  const int nx = __shfl_down_sync(0xffffffffu, f[0], 1);
  f[4] = (lane < 31) ? nx : ((j0 + kGradGroup < N) ? csr[j0 + kGradGroup] : N);
#pragma unroll
  for (int e = 0; e < 5; ++e) f[e] = min(max(f[e], 0), N);
}

__device__ __forceinline__ int parent_of(int c, const int g[5]) {
  return (c >= g[1]) + (c >= g[2]) + (c >= g[3]);
}

template <typename T>
__device__ __forceinline__ T pick4(int e, T a0, T a1, T a2, T a3) {
  return e == 0 ? a0 : (e == 1 ? a1 : (e == 2 ? a2 : a3));
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// Recompute
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kGradThreads) grad_seed_kernel(int N, const float* __restrict__ ckpt,
                                                                  float* __restrict__ h_out, PcgTick pc,
                                                                  int propagate_tick, float mu, float rho,
                                                                  float sigma, int nu_int, float nu_state) {
  griddep_wait();
  const int j0 = (blockIdx.x * kGradThreads + threadIdx.x) * kGradGroup;
  float4 h4 = *reinterpret_cast<const float4*>(ckpt + j0);
  if (propagate_tick) {
    float hh[4] = {h4.x, h4.y, h4.z, h4.w};
#pragma unroll
    for (int e = 0; e < kGradGroup; ++e)
      if (j0 + e < N) hh[e] = propagate(hh[e], mu, rho, sigma, state_noise(pc, (uint32_t)(j0 + e), nu_int, nu_state));
    h4 = make_float4(hh[0], hh[1], hh[2], hh[3]);
  }
  *reinterpret_cast<float4*>(h_out + j0) = h4;
  griddep_release();
}

__global__ void __launch_bounds__(kGradThreads) grad_recompute_kernel(int N, const int32_t* __restrict__ csr,
                                                                       const float* __restrict__ hp,
                                                                       float* __restrict__ hc, PcgTick pc,
                                                                       float mu, float rho, float sigma, int nu_int,
                                                                       float nu_state) {
  griddep_wait();
  const int lane = threadIdx.x & 31;
  const int j0 = (blockIdx.x * kGradThreads + threadIdx.x) * kGradGroup;
  int f[5];
  load_children(csr, N, j0, lane, f);
  const float4 h4 = *reinterpret_cast<const float4*>(hp + j0);
  const float hv[4] = {h4.x, h4.y, h4.z, h4.w};
  const bool heavy = f[4] - f[0] > kGradHeavy;
  if (!heavy) {
    int c = f[0];
#pragma unroll
    for (int e = 0; e < kGradGroup; ++e)
      for (; c < f[e + 1]; ++c) hc[c] = propagate(hv[e], mu, rho, sigma, state_noise(pc, (uint32_t)c, nu_int, nu_state));
  }
  unsigned hm = __ballot_sync(0xffffffffu, heavy);
  while (hm) {
    const int src = __ffs(hm) - 1;
    hm &= hm - 1u;
    int g[5];
    float hs[4];
#pragma unroll
    for (int e = 0; e < 5; ++e) g[e] = __shfl_sync(0xffffffffu, f[e], src);
#pragma unroll
    for (int e = 0; e < 4; ++e) hs[e] = __shfl_sync(0xffffffffu, hv[e], src);
    for (int c = g[0] + lane; c < g[4]; c += 32) {
      const float h = pick4(parent_of(c, g), hs[0], hs[1], hs[2], hs[3]);
      hc[c] = propagate(h, mu, rho, sigma, state_noise(pc, (uint32_t)c, nu_int, nu_state));
    }
  }
  griddep_release();
}

// ---------------------------------------------------------------------------
// Adjoint
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kGradThreads) grad_adjoint_kernel(GradAdjArgs a) {
  __shared__ double s_red[kGradAcc][kGradThreads / 32];
  griddep_wait();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int j0 = (blockIdx.x * kGradThreads + tid) * kGradGroup;
  const int N = a.N;
  const float4 h4 = *reinterpret_cast<const float4*>(a.h + j0);
  const float hv[4] = {h4.x, h4.y, h4.z, h4.w};

  // children sums of lambda_t+1 and sum lambda eps over the children
  float cs[4] = {0.f, 0.f, 0.f, 0.f};
  float acc_eps = 0.f;
  if (a.csr) {
    int f[5];
    load_children(a.csr, N, j0, lane, f);
    const bool heavy = f[4] - f[0] > kGradHeavy;
    if (!heavy) {
      int c = f[0];
#pragma unroll
      for (int e = 0; e < kGradGroup; ++e)
        for (; c < f[e + 1]; ++c) {
          const float l = a.lam_next[c];
          cs[e] += l;
          acc_eps = fmaf(l, state_noise(a.pc_next, (uint32_t)c, a.nu_int, a.nu_state), acc_eps);
        }
    }
    unsigned hm = __ballot_sync(0xffffffffu, heavy);
    while (hm) {
      const int src = __ffs(hm) - 1;
      hm &= hm - 1u;
      int g[5];
#pragma unroll
      for (int e = 0; e < 5; ++e) g[e] = __shfl_sync(0xffffffffu, f[e], src);
      float p[4] = {0.f, 0.f, 0.f, 0.f};
      for (int c = g[0] + lane; c < g[4]; c += 32) {
        const float l = a.lam_next[c];
        const int e = parent_of(c, g);
        p[0] += (e == 0) ? l : 0.f;
        p[1] += (e == 1) ? l : 0.f;
        p[2] += (e == 2) ? l : 0.f;
        p[3] += (e == 3) ? l : 0.f;
        acc_eps = fmaf(l, state_noise(a.pc_next, (uint32_t)c, a.nu_int, a.nu_state), acc_eps);
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) p[e] = warp_sum_f(p[e]);
      if (lane == src) {
#pragma unroll
        for (int e = 0; e < 4; ++e) cs[e] += p[e];
      }
    }
  }

  // lambda_t of the four parents
  const float2 ax = *a.aux;
  const float invS = ax.x, nM = (float)__float_as_int(ax.y);
  const float y = *a.y, y2 = y * y;
  const bool gauss = !(a.obs.nu > 0.0f);
  ObsModel obs = a.obs;
  obs.y = y;
  float lam[4];
  float acc_cs = 0.f, acc_csh = 0.f, acc_l0 = 0.f, acc_l0z = 0.f;
#pragma unroll
  for (int e = 0; e < kGradGroup; ++e) {
    const int j = j0 + e;
    float l = 0.f;
    if (j < N) {
      const float h = hv[e];
      float x, g;
      if (gauss) {
        x = obs_log2pdf_gauss(y2, h);
        g = 0.5f * fmaf(y2, ex2_approx(h * -kLog2e), -1.0f);          // -1/2 + y^2 e^{-h}/2
      } else {
        x = obs_log2pdf_t_plus(obs, __fmul_rn(y2, obs.inv_nu), h, __fmul_rn(obs.c_obs, kLog2e));
        const float q = y2 * ex2_approx(h * -kLog2e) * obs.inv_nu;     // y^2 e^{-h} / nu
        g = fmaf(obs.nu_p1h, div_approx(q, 1.0f + q), -0.5f);
      }
      const float W = ex2_approx(x - nM) * invS;
      l = fmaf(a.rho, cs[e], W * g);
      acc_cs += cs[e];
      acc_csh = fmaf(cs[e], h - a.mu, acc_csh);
      if (a.first) {
        const float z0 = state_noise(a.pc0, (uint32_t)j, 0, 0.0f);
        acc_l0 += l;
        acc_l0z = fmaf(l, z0, acc_l0z);
      }
    }
    lam[e] = l;
  }
  *reinterpret_cast<float4*>(a.lam + j0) = make_float4(lam[0], lam[1], lam[2], lam[3]);

  // per-CTA FP64 accumulation (the same CTA index adds in tick order)
  double v[kGradAcc] = {(double)acc_cs, (double)acc_csh, (double)acc_eps, (double)acc_l0, (double)acc_l0z};
#pragma unroll
  for (int k = 0; k < kGradAcc; ++k) v[k] = warp_sum_d(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < kGradAcc; ++k) s_red[k][warp] = v[k];
  }
  __syncthreads();
  if (tid < kGradAcc) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kGradThreads / 32; ++w) t += s_red[tid][w];
    a.acc[(size_t)blockIdx.x * kGradAcc + tid] += t;
  }
  griddep_release();
}

__global__ void __launch_bounds__(kGradThreads) grad_finish_kernel(int ctas, const double* __restrict__ acc,
                                                                    float mu, float rho, float sigma,
                                                                    double* __restrict__ grad) {
  __shared__ double s_red[kGradAcc][kGradThreads / 32];
  griddep_wait();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double v[kGradAcc] = {0.0, 0.0, 0.0, 0.0, 0.0};
  for (int b = tid; b < ctas; b += kGradThreads)
#pragma unroll
    for (int k = 0; k < kGradAcc; ++k) v[k] += acc[(size_t)b * kGradAcc + k];
#pragma unroll
  for (int k = 0; k < kGradAcc; ++k) v[k] = warp_sum_d(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < kGradAcc; ++k) s_red[k][warp] = v[k];
  __syncthreads();
  if (tid == 0) {
    double t[kGradAcc];
#pragma unroll
    for (int k = 0; k < kGradAcc; ++k) {
      t[k] = 0.0;
      for (int w = 0; w < kGradThreads / 32; ++w) t[k] += s_red[k][w];
    }
    // h_0 = mu + sigma z / sqrt(max(1 - rho^2, 1e-6))   (gpu_bpf/gpu_bpf_ptx_full.cu:430)
    const double r = (double)rho, sg = (double)sigma;
    const double one_m = 1.0 - r * r;
    const double s2 = fmax(one_m, 1e-6), sd = sqrt(s2);
    const double ds_drho = one_m > 1e-6 ? sg * r / (s2 * sd) : 0.0;
    grad[0] = (1.0 - r) * t[0] + t[3];
    grad[1] = t[1] + t[4] * ds_drho;
    grad[2] = t[2] + t[4] / sd;
  }
  griddep_release();
}

// ---------------------------------------------------------------------------
// FP64 replay with forward-mode tangents
// ---------------------------------------------------------------------------
struct OnlineLse {
  double m, s, s1, s2, s3;   // running max, sum e^{lw-m}, sums e^{lw-m} * g * dh/dtheta_k
  __device__ void init() { m = -INFINITY; s = s1 = s2 = s3 = 0.0; }
  __device__ void add(double lw, double g0, double g1, double g2) {
    if (lw > m) {
      const double sc = (m == -INFINITY) ? 0.0 : exp(m - lw);
      s *= sc; s1 *= sc; s2 *= sc; s3 *= sc;
      m = lw;
    }
    const double e = exp(lw - m);
    s += e; s1 = fma(e, g0, s1); s2 = fma(e, g1, s2); s3 = fma(e, g2, s3);
  }
  __device__ void merge(const OnlineLse& o) {
    const double mm = fmax(m, o.m);
    if (mm == -INFINITY) return;
    const double fa = (m == -INFINITY) ? 0.0 : exp(m - mm);
    const double fb = (o.m == -INFINITY) ? 0.0 : exp(o.m - mm);
    s = s * fa + o.s * fb; s1 = s1 * fa + o.s1 * fb; s2 = s2 * fa + o.s2 * fb; s3 = s3 * fa + o.s3 * fb;
    m = mm;
  }
};

__device__ __forceinline__ OnlineLse shfl_xor_lse(const OnlineLse& a, int o) {
  OnlineLse b;
  b.m = __shfl_xor_sync(0xffffffffu, a.m, o);
  b.s = __shfl_xor_sync(0xffffffffu, a.s, o);
  b.s1 = __shfl_xor_sync(0xffffffffu, a.s1, o);
  b.s2 = __shfl_xor_sync(0xffffffffu, a.s2, o);
  b.s3 = __shfl_xor_sync(0xffffffffu, a.s3, o);
  return b;
}

// log p(y | h) and its h-derivative in FP64 (PTX :414-451 model)
__device__ __forceinline__ void obs_f64(const ObsModel& o, double y, double h, double* lw, double* g) {
  const double q = y * y * exp(-h);
  if (o.nu > 0.0f) {
    const double nu = (double)o.nu;
    *lw = (double)o.c_obs - 0.5 * (nu + 1.0) * log1p(q / nu) - 0.5 * h;
    *g = -0.5 + 0.5 * (nu + 1.0) * (q / nu) / (1.0 + q / nu);
  } else {
    *lw = -0.918938533204672741780329736406 - 0.5 * q - 0.5 * h;
    *g = -0.5 + 0.5 * q;
  }
}

__device__ void lse_block_store(OnlineLse acc, double* out) {
  __shared__ OnlineLse s_w[kGradThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc.merge(shfl_xor_lse(acc, o));
  if (lane == 0) s_w[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    OnlineLse t = s_w[0];
    for (int w = 1; w < kGradThreads / 32; ++w) t.merge(s_w[w]);
    out[0] = t.m; out[1] = t.s; out[2] = t.s1; out[3] = t.s2; out[4] = t.s3;
  }
}

__global__ void __launch_bounds__(kGradThreads) replay_init_kernel(ReplayArgs a) {
  const int j0 = (blockIdx.x * kGradThreads + threadIdx.x) * kGradGroup;
  const double mu = a.mu, rho = a.rho, sg = a.sigma;
  const double one_m = 1.0 - rho * rho;
  const double s2 = fmax(one_m, 1e-6), sd = sqrt(s2);
  const double sstat = sg / sd, ds_drho = one_m > 1e-6 ? sg * rho / (s2 * sd) : 0.0, ds_dsig = 1.0 / sd;
  const double y = (double)*a.y;
  OnlineLse acc;
  acc.init();
  for (int e = 0; e < kGradGroup; ++e) {
    const int j = j0 + e;
    if (j >= a.N) break;
    const double z = (double)state_noise(a.pc, (uint32_t)j, 0, 0.0f);
    const double h = fma(sstat, z, mu), d0 = 1.0, d1 = z * ds_drho, d2 = z * ds_dsig;
    a.hc[j] = h; a.hc[a.stride + j] = d0; a.hc[2 * (size_t)a.stride + j] = d1; a.hc[3 * (size_t)a.stride + j] = d2;
    double lw, g;
    obs_f64(a.obs, y, h, &lw, &g);
    acc.add(lw, g * d0, g * d1, g * d2);
  }
  lse_block_store(acc, a.part + (size_t)blockIdx.x * 5);
}

__global__ void __launch_bounds__(kGradThreads) replay_tick_kernel(ReplayArgs a) {
  const int lane = threadIdx.x & 31;
  const int j0 = (blockIdx.x * kGradThreads + threadIdx.x) * kGradGroup;
  const size_t S = (size_t)a.stride;
  const double mu = a.mu, rho = a.rho, sg = a.sigma;
  const double y = (double)*a.y;
  int f[5];
  load_children(a.csr, a.N, j0, lane, f);
  double ph[4], p0[4], p1[4], p2[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    ph[e] = a.hp[j0 + e]; p0[e] = a.hp[S + j0 + e]; p1[e] = a.hp[2 * S + j0 + e]; p2[e] = a.hp[3 * S + j0 + e];
  }
  OnlineLse acc;
  acc.init();
  auto child = [&](int c, double hpar, double d0p, double d1p, double d2p) {
    const double eps = (double)state_noise(a.pc, (uint32_t)c, a.nu_int, a.nu_state);
    const double h = mu + rho * (hpar - mu) + sg * eps;
    const double d0 = (1.0 - rho) + rho * d0p, d1 = (hpar - mu) + rho * d1p, d2 = eps + rho * d2p;
    a.hc[c] = h; a.hc[S + c] = d0; a.hc[2 * S + c] = d1; a.hc[3 * S + c] = d2;
    double lw, g;
    obs_f64(a.obs, y, h, &lw, &g);
    acc.add(lw, g * d0, g * d1, g * d2);
  };
  const bool heavy = f[4] - f[0] > kGradHeavy;
  if (!heavy) {
    int c = f[0];
#pragma unroll
    for (int e = 0; e < kGradGroup; ++e)
      for (; c < f[e + 1]; ++c) child(c, ph[e], p0[e], p1[e], p2[e]);
  }
  unsigned hm = __ballot_sync(0xffffffffu, heavy);
  while (hm) {
    const int src = __ffs(hm) - 1;
    hm &= hm - 1u;
    int g[5];
    double qh[4], q0[4], q1[4], q2[4];
#pragma unroll
    for (int e = 0; e < 5; ++e) g[e] = __shfl_sync(0xffffffffu, f[e], src);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      qh[e] = __shfl_sync(0xffffffffu, ph[e], src);
      q0[e] = __shfl_sync(0xffffffffu, p0[e], src);
      q1[e] = __shfl_sync(0xffffffffu, p1[e], src);
      q2[e] = __shfl_sync(0xffffffffu, p2[e], src);
    }
    for (int c = g[0] + lane; c < g[4]; c += 32) {
      const int e = parent_of(c, g);
      child(c, pick4(e, qh[0], qh[1], qh[2], qh[3]), pick4(e, q0[0], q0[1], q0[2], q0[3]),
            pick4(e, q1[0], q1[1], q1[2], q1[3]), pick4(e, q2[0], q2[1], q2[2], q2[3]));
    }
  }
  lse_block_store(acc, a.part + (size_t)blockIdx.x * 5);
}

// one CTA per tick: dll_t = LSE_t - ln N and d dll_t / dtheta
__global__ void __launch_bounds__(kGradThreads) replay_reduce_kernel(int ctas, const double* __restrict__ part,
                                                                      double log_n, double* __restrict__ per_tick) {
  const int t = blockIdx.x;
  OnlineLse acc;
  acc.init();
  for (int b = threadIdx.x; b < ctas; b += kGradThreads) {
    const double* q = part + ((size_t)t * ctas + b) * 5;
    OnlineLse o;
    o.m = q[0]; o.s = q[1]; o.s1 = q[2]; o.s2 = q[3]; o.s3 = q[4];
    acc.merge(o);
  }
  __shared__ double out[5];
  lse_block_store(acc, out);
  __syncthreads();
  if (threadIdx.x == 0) {
    double* r = per_tick + (size_t)t * 4;
    r[0] = out[0] + log(out[1]) - log_n;
    r[1] = out[2] / out[1];
    r[2] = out[3] / out[1];
    r[3] = out[4] / out[1];
  }
}

__global__ void __launch_bounds__(kGradThreads) replay_total_kernel(int T, const double* __restrict__ per_tick,
                                                                     double* __restrict__ total) {
  __shared__ double s_red[4][kGradThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  for (int t = tid; t < T; t += kGradThreads)
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] += per_tick[(size_t)t * 4 + k];
#pragma unroll
  for (int k = 0; k < 4; ++k) v[k] = warp_sum_d(v[k]);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) s_red[k][warp] = v[k];
  __syncthreads();
  if (tid < 4) {
    double t = 0.0;
    for (int w = 0; w < kGradThreads / 32; ++w) t += s_red[tid][w];
    total[tid] = t;
  }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kern)(KArgs...), int grid, cudaStream_t s, bool pdl, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kGradThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl ? attr : nullptr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

cudaError_t launch_grad_seed(int N, const float* ckpt, float* h_out, PcgTick pc, int propagate_tick, float mu,
                             float rho, float sigma, int nu_int, float nu_state, cudaStream_t s, bool pdl) {
  return launch_pdl(grad_seed_kernel, grad_ctas(N), s, pdl, N, ckpt, h_out, pc, propagate_tick, mu, rho, sigma,
                    nu_int, nu_state);
}
cudaError_t launch_grad_recompute(int N, const int32_t* csr, const float* hp, float* hc, PcgTick pc, float mu,
                                  float rho, float sigma, int nu_int, float nu_state, cudaStream_t s, bool pdl) {
  return launch_pdl(grad_recompute_kernel, grad_ctas(N), s, pdl, N, csr, hp, hc, pc, mu, rho, sigma, nu_int,
                    nu_state);
}
cudaError_t launch_grad_adjoint(const GradAdjArgs& a, cudaStream_t s, bool pdl) {
  return launch_pdl(grad_adjoint_kernel, grad_ctas(a.N), s, pdl, a);
}
cudaError_t launch_grad_finish(int ctas, const double* acc, float mu, float rho, float sigma, double* grad,
                               cudaStream_t s, bool pdl) {
  return launch_pdl(grad_finish_kernel, 1, s, pdl, ctas, acc, mu, rho, sigma, grad);
}
cudaError_t launch_replay_init(const ReplayArgs& a, cudaStream_t s) {
  replay_init_kernel<<<grad_ctas(a.N), kGradThreads, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_replay_tick(const ReplayArgs& a, cudaStream_t s) {
  replay_tick_kernel<<<grad_ctas(a.N), kGradThreads, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_replay_reduce(int T, int ctas, const double* part, double log_n, double* per_tick,
                                 double* total, cudaStream_t s) {
  replay_reduce_kernel<<<T, kGradThreads, 0, s>>>(ctas, part, log_n, per_tick);
  replay_total_kernel<<<1, kGradThreads, 0, s>>>(T, per_tick, total);
  return cudaGetLastError();
}

}  // namespace bpf
