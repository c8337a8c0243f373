// bpf_common.cuh — device building blocks shared by the plain, batched and
// gradient particle-filter kernels (sm_100a).
//
// Model (stochastic volatility, reference gpu_bpf/gpu_bpf.cuh:44 names):
//   h_t = mu + rho*(h_{t-1} - mu) + sigma_z*eps_t,   y_t = exp(h_t/2)*eta_t
//
// Random numbers: the reference gives every particle slot i its own PCG32
// stream (ptx_assembly/bpf_kernels_full.ptx:74-91 seeds it, :140-157 steps
// it) and never moves a stream with a resampled particle. Slot i's draw t is
// therefore a pure function of (seed, i, t):
//   inc_i = (2i+1) mod 2^32 (zero-extended), s0_i = (seed*A + inc_i)*A + inc_i
//   s_t   = A^t * s0_i + (sum_{k<t} A^k) * inc_i            (mod 2^64)
//         = K1_t + K2_t * inc_i,  K1_t = A^t*A^2*seed, K2_t = A^t*(A+1) + B_t
// (LCG jump-ahead, F. Brown, "Random number generation with arbitrary
// strides", 1994). The kernels hold no RNG state in HBM at all.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bpf {

// ---------------------------------------------------------------------------
// Tiling constants of the plain filter
// ---------------------------------------------------------------------------
constexpr int kThreads   = 256;              // threads per CTA (pass 1 and pass 2)
constexpr int kPerThread = 16;               // particles per thread
constexpr int kTile      = kThreads * kPerThread;   // 4096 particles per tile
constexpr int kOutChunk  = 4096;             // outputs per pass-2 work item
constexpr int kFixF      = 50;               // tile-frame fraction bits: 62 - log2(kTile)
constexpr int kNkEmpty   = -(1 << 30);       // tile exponent of a tile with no mass

constexpr uint64_t kPcgMult = 6364136223846793005ULL;        // PTX :81
constexpr uint64_t kHostInc = 1442695040888963407ULL;        // gpu_bpf_ptx_full.cu:243

// Uniform clamp of the reference: max.f32 0f358637BD, min.f32 0f3F7FFBCE
// (bpf_kernels_full.ptx:163-164). The upper constant is 0.99993598, not
// 1-1e-6 as the PTX comment says; it is mirrored bit-for-bit so the particle
// noise has the reference's distribution.
__host__ __device__ inline float uclamp_lo() { return 9.99999997475242708e-07f; }   // 0x358637BD
__host__ __device__ inline float uclamp_hi() { return 0.999935984611511230f; }      // 0x3F7FFBCE

// ---------------------------------------------------------------------------
// PCG32 (O'Neill 2014), XSH-RR output of the pre-step state
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pcg_output(uint64_t old) {
  const uint32_t lo = (uint32_t)old, hi = (uint32_t)(old >> 32);
  // low 32 bits of ((old >> 18) ^ old) >> 27  ==  (old >> 27) ^ (old >> 45)
  const uint32_t xsh = __funnelshift_r(lo, hi, 27) ^ (hi >> 13);
  const uint32_t rot = hi >> 27;
  return __funnelshift_r(xsh, xsh, rot);   // rotate right by rot
}

// Per-tick stream constants for a filter with integer seed `seed`.
struct PcgTick {
  uint64_t k1, k2;   // s_{t,i} = k1 + k2 * inc_i
};
__host__ __device__ inline PcgTick pcg_tick_consts(int seed, uint64_t At, uint64_t Bt) {
  const uint64_t s = (uint64_t)(int64_t)seed;   // (unsigned long long)seed, PTX param is u64
  PcgTick c;
  c.k1 = At * (kPcgMult * kPcgMult) * s;
  c.k2 = At * (kPcgMult + 1ULL) + Bt;
  return c;
}
__host__ __device__ inline uint64_t pcg_inc(uint32_t i) { return (uint64_t)(uint32_t)(2u * i + 1u); }

// u in (0,1): (out >> 9) * 2^-23, clamped like the reference (PTX :159-164)
__device__ __forceinline__ float pcg_uniform(uint32_t out) {
  float u = __uint2float_rn(out >> 9) * 1.1920928955078125e-07f;
  u = fmaxf(u, uclamp_lo());
  u = fminf(u, uclamp_hi());
  return u;
}

// ---------------------------------------------------------------------------
// Hardware approximate transcendental instructions (MUFU), written as PTX.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float ex2_approx(float x) {
  float r; asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r;
}
__device__ __forceinline__ float lg2_approx(float x) {
  float r; asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r;
}
__device__ __forceinline__ float sqrt_approx(float x) {
  float r; asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r;
}
__device__ __forceinline__ float div_approx(float a, float b) {
  float r; asm("div.approx.ftz.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b)); return r;
}

constexpr float kLog2e = 1.44269504088896340736f;
constexpr float kLn2   = 0.693147180559945309417f;

// ---------------------------------------------------------------------------
// Inverse normal CDF. The reference evaluates P. J. Acklam's rational
// approximation in FP32 (PTX :166-205); in FP32 its central rational loses
// about three digits to cancellation near |u-1/2| = 0.47 (absolute error up to
// 2.7e-4 in z). This build evaluates M. J. Wichura's algorithm AS 241 (PPND7,
// Applied Statistics 37, 1988), designed for single precision: positive
// coefficients in the central branch, absolute error below ~1.1e-6 over the
// clamped uniform range. Coefficients are Wichura's published ones. The
// uniform clamp keeps u in [1e-6, 0.99994], so the far-tail branch of AS 241
// (sqrt(-ln p) > 5) is never reached.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float icdf_normal(float u) {
  const float q = u - 0.5f;
  if (fabsf(q) <= 0.425f) {
    const float r = 0.180625f - q * q;
    float num = fmaf(5.9109374720e+01f, r, 1.5929113202e+02f);
    num = fmaf(num, r, 5.0434271938e+01f);
    num = fmaf(num, r, 3.3871327179e+00f);
    float den = fmaf(6.7187563600e+01f, r, 7.8757757664e+01f);
    den = fmaf(den, r, 1.7895169469e+01f);
    den = fmaf(den, r, 1.0f);
    return div_approx(q * num, den);
  }
  const float p = (q < 0.0f) ? u : 1.0f - u;
  const float r = sqrt_approx(-kLn2 * lg2_approx(p)) - 1.6f;
  float num = fmaf(1.7023821103e-01f, r, 1.3067284816e+00f);
  num = fmaf(num, r, 2.7568153900e+00f);
  num = fmaf(num, r, 1.4234372777e+00f);
  float den = fmaf(1.2021132975e-01f, r, 7.3700164250e-01f);
  den = fmaf(den, r, 1.0f);
  const float z = div_approx(num, den);
  return (q < 0.0f) ? -z : z;
}

// ---------------------------------------------------------------------------
// Observation log-density log p(y | h) (PTX :414-451; gpu_bpf.cu:226)
//   Gaussian:  -1/2 ln(2 pi) - 1/2 y^2 e^{-h} - 1/2 h
//   Student-t: C_obs - (nu+1)/2 ln(1 + y^2 e^{-h}/nu) - 1/2 h
// ---------------------------------------------------------------------------
struct ObsModel {
  float y;          // observation
  float nu;         // 0 = Gaussian
  float c_obs;      // lgamma((nu+1)/2) - lgamma(nu/2) - ln(nu pi)/2
  float inv_nu;     // 1/nu
  float nu_p1h;     // (nu+1)/2
};

__device__ __forceinline__ float obs_logpdf(const ObsModel& m, float h) {
  const float e = ex2_approx(h * -0.5f * kLog2e);   // exp(-h/2)
  const float eta = m.y * e;
  const float eta2 = eta * eta;
  if (m.nu > 0.0f) {
    const float t = fmaf(eta2, m.inv_nu, 1.0f);
    const float lt = -m.nu_p1h * (kLn2 * lg2_approx(t));
    return fmaf(-0.5f, h, m.c_obs + lt);
  }
  float lw = fmaf(-0.5f, eta2, -0.918938533204672742f);   // -1/2 ln(2 pi)
  return fmaf(-0.5f, h, lw);
}

// OU transition with the reference's operation order (PTX :406-411):
//   dev = rho*(h-mu); h = mu + dev; h = fma(sigma, eps, h)
__device__ __forceinline__ float propagate(float h, float mu, float rho, float sigma, float eps) {
  const float dev = __fmul_rn(rho, __fsub_rn(h, mu));
  return fmaf(sigma, eps, __fadd_rn(mu, dev));
}

// ---------------------------------------------------------------------------
// Exact fixed-point weight of a tile-relative FP32 weight w in [0, 1]:
// floor(w * 2^kFixF). The product is an exact power-of-two scaling, so the
// result is reproducible bit-for-bit by any IEEE host.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t fix_weight(float w) {
  return __float2ull_rz(w * 1125899906842624.0f);   // 2^50
}

// Unsigned 64-bit floor division by a constant d, through the reciprocal
// m = floor((2^64-1)/d) and an exact remainder correction.
__device__ __forceinline__ uint64_t udiv_magic(uint64_t a, uint64_t d, uint64_t m) {
  uint64_t q = __umul64hi(a, m);
  uint64_t r = a - q * d;
  while (r >= d) { ++q; r -= d; }
  return q;
}

}  // namespace bpf
