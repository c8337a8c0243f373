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
constexpr int kOutChunk  = 2 * kTile;        // outputs per pass-2 work item (2x the mean per tile)
constexpr int kPlanThreads = 1024;           // threads of the single-CTA plan kernel
constexpr int kPlanSmemTiles = 12800;        // tiles the plan kernel stages in shared memory (N <= 52.4M)
constexpr int kSmallTiles = 16;             // tiles of the fused small-filter tick (one CTA each)
constexpr int kSmallMaxN  = kSmallTiles * kTile;    // 65536 particles
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

// Jump constants of draw t: A^t and sum_{k<t} A^k (mod 2^64), by composing the
// affine maps x -> A x + 1 in O(log t) steps.
__host__ __device__ inline void pcg_jump(uint64_t t, uint64_t* At, uint64_t* Bt) {
  uint64_t am = 1ull, ap = 0ull, cm = kPcgMult, cp = 1ull;
  while (t) {
    if (t & 1ull) { am *= cm; ap = ap * cm + cp; }
    cp = (cm + 1ull) * cp;
    cm *= cm;
    t >>= 1;
  }
  *At = am;
  *Bt = ap;
}

// u in (0,1): (out >> 9) * 2^-23, clamped like the reference (PTX :159-164).
// Formed from the float bit pattern 1.m - 1 (exact) instead of an int->float
// conversion.
__device__ __forceinline__ float pcg_uniform(uint32_t out) {
  float u = __uint_as_float(0x3F800000u | (out >> 9)) - 1.0f;
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
// Inverse normal CDF, z = sqrt(2) * erfinv(2u - 1), by M. Giles' single-
// precision erfinv approximation ("Approximating the erfinv function", GPU
// Computing Gems Jade Edition, 2011; published coefficients). The argument
// w = -ln(1 - x^2) is formed as -ln(4u(1-u)) straight from u, so there is no
// cancellation near the clamped ends. Absolute error in z is below 1e-6 over
// the whole clamped range [1e-6, 0.99994]; the common branch (w < 5, i.e.
// 0.0017 < u < 0.9983) costs one MUFU lg2 and nine FMAs with no division.
// The reference evaluates P. J. Acklam's rational approximation in FP32 (PTX
// :166-205), whose central rational cancels to ~3e-4 absolute error near
// |u-1/2| = 0.47; the uniform clamp and PCG32 draw are kept bit-for-bit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float icdf_central_poly(float l2) {      // w < 5
  const float w = fmaf(-kLn2, l2, -2.0f * kLn2 - 2.5f);                // w - 2.5
  float p = 2.81022636e-08f;
  p = fmaf(p, w, 3.43273939e-07f);
  p = fmaf(p, w, -3.5233877e-06f);
  p = fmaf(p, w, -4.39150654e-06f);
  p = fmaf(p, w, 0.00021858087f);
  p = fmaf(p, w, -0.00125372503f);
  p = fmaf(p, w, -0.00417768164f);
  p = fmaf(p, w, 0.246640727f);
  p = fmaf(p, w, 1.50140941f);
  return p;
}
__device__ __forceinline__ float icdf_tail_poly(float l2) {         // w >= 5
  const float w = sqrt_approx(fmaf(-kLn2, l2, -2.0f * kLn2)) - 3.0f;
  float p = -0.000200214257f;
  p = fmaf(p, w, 0.000100950558f);
  p = fmaf(p, w, 0.00134934322f);
  p = fmaf(p, w, -0.00367342844f);
  p = fmaf(p, w, 0.00573950773f);
  p = fmaf(p, w, -0.0076224613f);
  p = fmaf(p, w, 0.00943887047f);
  p = fmaf(p, w, 1.00167406f);
  p = fmaf(p, w, 2.83297682f);
  return p;
}
constexpr float kIcdfTailL2 = -9.21347810f;   // w = -ln(4u(1-u)) < 5  <=>  log2(u(1-u)) > -5/ln2 - 2

__device__ __forceinline__ float icdf_normal(float u) {
  const float t = u * (1.0f - u);
  const float l2 = lg2_approx(t);                                       // log2(u(1-u))
  const float xs = fmaf(2.82842712474619010f, u, -1.41421356237309505f);  // sqrt2 * (2u - 1)
  const float p = (l2 > kIcdfTailL2) ? icdf_central_poly(l2) : icdf_tail_poly(l2);
  return p * xs;
}

// The same function for a full warp in convergent code: the tail polynomial
// (u < 0.0017 or u > 0.9983, about one draw in 290) runs behind a warp vote,
// so the common case costs the central polynomial alone. Results are identical
// to icdf_normal bit for bit.
__device__ __forceinline__ float icdf_normal_warp(float u) {
  const float t = u * (1.0f - u);
  const float l2 = lg2_approx(t);
  const float xs = fmaf(2.82842712474619010f, u, -1.41421356237309505f);
  float p = icdf_central_poly(l2);
  const bool tail = !(l2 > kIcdfTailL2);
  if (__any_sync(0xffffffffu, tail)) {
    const float pt = icdf_tail_poly(l2);
    if (tail) p = pt;
  }
  return p * xs;
}

// The same for code whose warp may be partly active (a loop over particles whose trip count
// differs between lanes): the vote covers the active lanes only.
__device__ __forceinline__ float icdf_normal_active(float u) {
  const float t = u * (1.0f - u);
  const float l2 = lg2_approx(t);
  const float xs = fmaf(2.82842712474619010f, u, -1.41421356237309505f);
  float p = icdf_central_poly(l2);
  const bool tail = !(l2 > kIcdfTailL2);
  if (__any_sync(__activemask(), tail)) {
    const float pt = icdf_tail_poly(l2);
    if (tail) p = pt;
  }
  return p * xs;
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

// log2 p(y | h) for the Gaussian model with y2 = y^2:
//   -log2(e)/2 * (y^2 e^{-h} + h) - log2(e) ln(2 pi)/2
constexpr float kGaussLog2C = -1.32574806473616f;               // -log2(e) ln(2 pi)/2
__device__ __forceinline__ float obs_log2pdf_gauss_plus(float y2, float h, float c) {   // + (c - kGaussLog2C)
  const float e = ex2_approx(h * -kLog2e);                       // e^{-h}
  const float s = (y2 > 0.0f) ? fmaf(y2, e, h) : h;
  return fmaf(-0.5f * kLog2e, s, c);
}
__device__ __forceinline__ float obs_log2pdf_gauss(float y2, float h) {
  return obs_log2pdf_gauss_plus(y2, h, kGaussLog2C);
}

// Tile-relative weight 2^d of a tile-relative log2-weight d <= 0 (the stored
// form). Pass 1 and pass 2 both evaluate it with this one instruction sequence,
// so the fixed-point masses agree bit for bit.
__device__ __forceinline__ float tile_weight(float d) { return fminf(ex2_approx(d), 1.0f); }

// log2 p(y | h) for the Student-t model, from y2nu = y^2 / nu and
// c = log2(e) c_obs (+ any offset):
//   c - (nu+1)/2 log2(1 + y^2 e^{-h} / nu) - log2(e) h / 2
__device__ __forceinline__ float obs_log2pdf_t_plus(const ObsModel& m, float y2nu, float h, float c) {
  const float e = ex2_approx(h * -kLog2e);                       // e^{-h}
  const float t = (y2nu > 0.0f) ? fmaf(y2nu, e, 1.0f) : 1.0f;
  return fmaf(-m.nu_p1h, lg2_approx(t), fmaf(-0.5f * kLog2e, h, c));
}

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

// ---------------------------------------------------------------------------
// Student-t state noise (nu_state > 0). The reference scales the normal draw by
// rsqrt(chi2 / nu_state), chi2 the sum of round(nu_state) squared normals from
// a separate cuRAND stream (gpu_bpf/gpu_bpf_ptx_full.cu:392-400,574-583;
// ptx_assembly/bpf_kernels_full.ptx:394-404). Here chi2 with k = round(nu_state)
// degrees of freedom is drawn exactly and statelessly: -2 ln(U_1 ... U_{k/2})
// (a sum of k/2 exponentials of mean 2) plus Z^2 when k is odd. Component c of
// slot i at tick t is draw t of the PCG32 stream with the particle's seed and
// increment ((c+1) << 33) | (2i+1), which no particle stream uses (their
// increments are below 2^32), so the counter-based jump of the tick applies
// unchanged. The log is summed in log2 (no underflow for large k).
// ---------------------------------------------------------------------------
__host__ __device__ inline uint64_t tstate_inc(uint32_t i, int c) {
  return ((uint64_t)(c + 1) << 33) | (uint64_t)(2u * i + 1u);
}

__device__ __forceinline__ float tstate_scale(const PcgTick& pc, uint32_t i, int nu_int, float nu_state) {
  const int pairs = nu_int >> 1;
  float l2sum = 0.0f;
  for (int c = 0; c < pairs; ++c)
    l2sum += lg2_approx(pcg_uniform(pcg_output(pc.k1 + pc.k2 * tstate_inc(i, c))));
  float chi2 = (-2.0f * kLn2) * l2sum;
  if (nu_int & 1) {
    const float z = icdf_normal(pcg_uniform(pcg_output(pc.k1 + pc.k2 * tstate_inc(i, pairs))));
    chi2 = fmaf(z, z, chi2);
  }
  return sqrt_approx(div_approx(nu_state, chi2));
}

// The same scale from slot i's own stream state s = k1 + k2 inc_i of the tick
// (component c's increment is inc_i + (c+1) 2^33, so its state is
// s + (c+1) k33 with k33 = k2 2^33): no 64-bit multiply per component. For a
// full, convergent warp (the odd component's normal uses the warp-vote form).
// Values are identical to tstate_scale.
__device__ __forceinline__ float tstate_scale_warp(uint64_t s, uint64_t k33, int nu_int, float nu_state) {
  const int pairs = nu_int >> 1;
  float l2sum = 0.0f;
  for (int c = 0; c < pairs; ++c) {
    s += k33;
    l2sum += lg2_approx(pcg_uniform(pcg_output(s)));
  }
  float chi2 = (-2.0f * kLn2) * l2sum;
  if (nu_int & 1) {
    const float z = icdf_normal_warp(pcg_uniform(pcg_output(s + k33)));
    chi2 = fmaf(z, z, chi2);
  }
  return sqrt_approx(div_approx(nu_state, chi2));
}

// State noise eps of slot i at the tick of pc: N(0,1), or Student-t when nu_int > 0.
__device__ __forceinline__ float state_noise(const PcgTick& pc, uint32_t i, int nu_int, float nu_state) {
  float z = icdf_normal(pcg_uniform(pcg_output(pc.k1 + pc.k2 * pcg_inc(i))));
  if (nu_int > 0) z *= tstate_scale(pc, i, nu_int, nu_state);
  return z;
}

// OU transition h' = mu + rho (h - mu) + sigma eps (PTX :406-411 evaluates
// mu + rho*(h-mu) in three roundings); here rho h + mu (1 - rho) as one FMA
// with the constant rounded once, then fma(sigma, eps, .). Every kernel that
// propagates (pass 1, the batched kernels, the gradient recompute, the APF)
// goes through these two helpers, so their particles agree bit for bit.
__device__ __forceinline__ float propagate_mean(float h, float mu, float rho) {
  return fmaf(rho, h, __fmul_rn(mu, __fsub_rn(1.0f, rho)));
}
__device__ __forceinline__ float propagate(float h, float mu, float rho, float sigma, float eps) {
  return fmaf(sigma, eps, propagate_mean(h, mu, rho));
}

// ---------------------------------------------------------------------------
// Exact fixed-point weight of a tile-relative FP32 weight w in [0, 1]:
// floor(w * 2^kFixF). The product is an exact power-of-two scaling, so the
// result is reproducible bit-for-bit by any IEEE host.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t fix_weight(float w) {
  return __float2ull_rz(w * 1125899906842624.0f);   // 2^50
}

// floor(a / b) for 1 <= b and a < 2^62: FP64 estimate, exact integer correction.
__device__ __forceinline__ uint64_t udiv_fp64(uint64_t a, uint64_t b) {
  uint64_t q = __double2ull_rz((double)a / (double)b);
  while (q > 0ull && q * b > a) --q;
  while (a - q * b >= b) ++q;
  return q;
}
// The same quotient from an FP64 reciprocal rb of b (1/b rounded once): for a / b < 2^50 the
// estimate is within one of the quotient, and the same corrections make it exact.
__device__ __forceinline__ uint64_t udiv_fp64_rcp(uint64_t a, uint64_t b, double rb) {
  uint64_t q = __double2ull_rz((double)a * rb);
  while (q > 0ull && q * b > a) --q;
  while (a - q * b >= b) ++q;
  return q;
}
// Reciprocal for udiv_magic: m <= floor((2^64-1)/d) with a relative deficit
// below 2^-48, so the quotient estimate is short by at most 3 for a/d < 2^31.
__device__ __forceinline__ uint64_t udiv_magic_of(uint64_t d) {
  return __double2ull_rz(18446744073709551615.0 / (double)d * (1.0 - 0x1p-49));
}

// Unsigned 64-bit floor division by a constant d, through a reciprocal
// m <= floor((2^64-1)/d) and an exact remainder correction.
__device__ __forceinline__ uint64_t udiv_magic(uint64_t a, uint64_t d, uint64_t m) {
  uint64_t q = __umul64hi(a, m);
  uint64_t r = a - q * d;
  while (r >= d) { ++q; r -= d; }
  return q;
}

}  // namespace bpf
