// bpf_plain.cu — the plain SV bootstrap-filter tick as three sm_100a kernels.
//
//   pass 1  (one CTA per 4096-particle tile, streaming)
//           counter-PCG32 -> inverse-CDF normal (x Student-t scale when
//           nu_state > 0) -> OU propagate -> log2-weight
//           (+ carried log2-weight on ESS-skipped ticks). The tile max becomes a
//           power-of-two exponent n_k; the tile-relative log2-weights
//           d = x - n_k <= 0 are written once (w = 2^d is re-derived by pass 2
//           and by the next tick's carry without a log), with the tile partials
//           S=sum w, Q=sum w^2, H=sum w h and the exact fixed-point tile mass
//           E = sum floor(w 2^50).
//   plan    (one CTA of 512 threads)
//           FP64 combine of the tile partials in the global frame 2^nM:
//           log-likelihood increment, ESS, filtered mean, the resampling
//           decision and the next tick's device state; on resampling ticks
//           also the fixed-point CDF (tile prefixes, total, target spacing)
//           and the pass-2 work list. No host synchronisation per tick.
//   pass 2  (persistent CTAs over work items: one tile, a run of outputs)
//           systematic resampling: exact integer prefix of the tile weights,
//           each element counts the evenly spaced targets it owns and marks
//           the first of them, a warp max-scan over the marks gives every
//           output its ancestor, gather of h[ancestor] from a bulk-async
//           (TMA) copy of the tile, 16-byte vector stores. Four CTAs per SM,
//           each staging one item's tiles at a time (the next item's copy is
//           issued as soon as the buffer is free). Early exit on ticks that
//           do not resample.
// Pass 1 and pass 2 walk the tiles (items) in the order opposite to the pass
// before them, so each starts on the tiles still in L2.
// Consecutive kernels use programmatic dependent launch: each waits on its
// predecessor with griddepcontrol.wait and releases its successor after its
// last store, so launch latency overlaps the predecessor's tail.
//
// Reference tick this replaces: gpu_bpf/gpu_bpf_ptx_full.cu:550-748 (~15
// launches, float atomics, a host sync for ESS, thrust scan) with kernels
// ptx_assembly/bpf_kernels_full.ptx:231-842.
#include "bpf_plain.cuh"
#include "bpf_block.cuh"
#include <cooperative_groups.h>
#include <cmath>
#include <mutex>
#include <type_traits>

namespace bpf {

// ---------------------------------------------------------------------------
// Init: h_0 = mu + std_stat * z(draw 0)  (bpf_kernels_full.ptx:103-218);
// thread 0 also (re)initialises the device state.
// ---------------------------------------------------------------------------
__global__ void init_kernel(Plan p, float mu, float std_stat, int seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int npad = p.G * kTile;
  if (i == 0) {
    DevState d{};
    const PcgTick c0 = pcg_tick_consts(seed, 1ull, 0ull);       // tick 0 uses draw index 0
    d.k1 = c0.k1; d.k2 = c0.k2;
    d.u_state = (unsigned long long)seed * 67890ULL + 12345ULL;  // gpu_bpf_ptx_full.cu:353
    d.logS_prev = log((double)p.N);
    d.resampled_prev = 1;                                        // gpu_bpf_ptx_full.cu:357
    d.seed = seed;
    *p.st = d;
  }
  if (i >= npad) return;
  float h = 0.0f;
  if (i < p.N) {
    const PcgTick c = pcg_tick_consts(seed, 1ull, 0ull);
    const uint64_t s = c.k1 + c.k2 * pcg_inc((uint32_t)i);
    const float z = icdf_normal(pcg_uniform(pcg_output(s)));
    h = fmaf(std_stat, z, mu);
  }
  p.h0[i] = h;
  p.h1[i] = h;
  p.w[i] = 0.0f;
}

constexpr int kStWords = (int)(sizeof(DevState) / 8);

// ---------------------------------------------------------------------------
// Pass 1
// ---------------------------------------------------------------------------
// Shared memory of one tile's pass 1 (one group of kThreads threads).
struct Pass1Shared {
  float s_max[kThreads / 32];
  float s_part[3][kThreads];
  unsigned long long s_E[kThreads];
  double s_red[3][kThreads / 32];          // online-learning sums
  unsigned long long s_redE[kThreads / 32];
  double s_red4[kThreads / 32];
};

// Barrier of one group of kThreads threads: barrier 0 is the whole CTA of the
// pass-1 kernel; the fused small-filter kernel gives each tile's group its own.
__device__ __forceinline__ void group_sync(int bar) {
  asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(kThreads) : "memory");
}

// APF = 0: bootstrap tick; 1 / 2: the two stages of an auxiliary-particle-filter
// tick (gpu_bpf_ptx_full.cu:990-1047): stage 1 weights each particle by
// p(y | m), m = mu + rho (h - mu), and leaves the particles in place; stage 2
// runs on the particles resampled by those weights, propagates them
// (h = m + sigma eps, the same operations as a bootstrap tick) and weights them
// by p(y | h) / p(y | m).
// GAUSS: the observation model is Gaussian (a.obs.nu == 0), fixed at compile
// time so the per-particle code carries no model branch.
// Pass 1 of tile k by one group of kThreads threads (tid = 0..kThreads-1 inside
// the group, `bar` its barrier), reading the tick's state from st.
template <bool TSTATE, bool LEARN, int APF, bool GAUSS>
__device__ __forceinline__ void pass1_tile(const Plan& p, const TickArgs& a, const DevState* st, int k, int tid,
                                           int bar, Pass1Shared& sh) {
  float* s_max = sh.s_max;
  float (*s_part)[kThreads] = sh.s_part;
  unsigned long long* s_E = sh.s_E;
  double (*s_red)[kThreads / 32] = sh.s_red;
  unsigned long long* s_redE = sh.s_redE;
  const int lane = tid & 31, warp = tid >> 5;
  const int tick = st->tick;
  const bool carry = APF == 0 && st->resampled_prev == 0;
  const int nM_prev = st->nM_prev;
  PcgTick c;
  c.k1 = st->k1; c.k2 = st->k2;
  float* hb = st->cur ? p.h1 : p.h0;

  const float y = a.y_ptr ? __ldg(a.y_ptr) : a.obs.y;
  constexpr bool gauss = GAUSS;
  ObsModel obs = a.obs;
  obs.y = y;
  const float y2 = y * y;

  float carry_off = 0.0f;
  if (carry) {
    const int nkp = p.nexp[k];
    carry_off = (nkp == kNkEmpty) ? -INFINITY : (float)(nkp - nM_prev);
  }
  const float gauss_c = kGaussLog2C + carry_off;   // the carry offset folded into the density's constant
  const float t_c0 = __fmul_rn(obs.c_obs, kLog2e);
  const float t_c = t_c0 + carry_off;
  const float y2nu = __fmul_rn(y2, obs.inv_nu);

  const int tile0 = k * kTile;
  const bool full = tile0 + kTile <= p.N;      // every slot of the tile holds a particle
  float4 h4[4], w4[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i0 = tile0 + 4 * (tid + kThreads * r);
    h4[r] = *reinterpret_cast<const float4*>(hb + i0);
    if (carry) w4[r] = *reinterpret_cast<const float4*>(p.w + i0);
    else w4[r] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  if (a.ckpt) {
#pragma unroll
    for (int r = 0; r < 4; ++r) *reinterpret_cast<float4*>(a.ckpt + tile0 + 4 * (tid + kThreads * r)) = h4[r];
  }

  float x[kPerThread], hv[kPerThread];
  float hpv[LEARN ? kPerThread : 1];     // particles before this tick's propagation (learning only)
  const unsigned long long step2 = 2ull * c.k2;
  const unsigned long long k33 = c.k2 << 33;          // Student-t component streams (tstate_scale_warp)
  // state of the first particle of group r + 1 from the state after group r's
  // four draws: inc advances by 2 * 4 * kThreads slots
  const unsigned long long group_step = (unsigned long long)(2 * 4 * kThreads - 8) * c.k2;
  const unsigned long long s_first = c.k1 + c.k2 * pcg_inc((uint32_t)(tile0 + 4 * tid));
  // the per-particle loop, compiled once with and once without the propagation
  // (tick 0 only weights the initial draw), so no particle tests the tick
  auto particles = [&](auto prop_tag) {
  constexpr bool PROP = decltype(prop_tag)::value;
  unsigned long long s = s_first;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i0 = tile0 + 4 * (tid + kThreads * r);
    if (r > 0) s += group_step;
    float hh[4] = {h4[r].x, h4[r].y, h4[r].z, h4[r].w};
    const float wp[4] = {w4[r].x, w4[r].y, w4[r].z, w4[r].w};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float h = hh[e];
      if (LEARN) hpv[4 * r + e] = h;
      float xx;
      if (APF == 0) {
        if (PROP) {
          float z = icdf_normal_warp(pcg_uniform(pcg_output(s)));
          if (TSTATE) z *= tstate_scale_warp(s, k33, a.nu_int, a.nu_state);
          h = propagate(h, a.mu, a.rho, a.sigma, z);
        }
        xx = gauss ? obs_log2pdf_gauss_plus(y2, h, gauss_c) : obs_log2pdf_t_plus(obs, y2nu, h, t_c);
      } else {
        const float m = propagate_mean(h, a.mu, a.rho);
        const float lm = gauss ? obs_log2pdf_gauss(y2, m) : obs_log2pdf_t_plus(obs, y2nu, m, t_c0);
        if (APF == 1) {
          xx = lm;
        } else {
          float z = icdf_normal_warp(pcg_uniform(pcg_output(s)));
          if (TSTATE) z *= tstate_scale_warp(s, k33, a.nu_int, a.nu_state);
          h = fmaf(a.sigma, z, m);
          xx = (gauss ? obs_log2pdf_gauss(y2, h) : obs_log2pdf_t_plus(obs, y2nu, h, t_c0)) - lm;
        }
      }
      s += step2;
      if (carry) xx += wp[e];                      // carried log2-weight (offset already added)
      hh[e] = h;
      x[4 * r + e] = xx;
      hv[4 * r + e] = h;
    }
    if (APF != 1) *reinterpret_cast<float4*>(hb + i0) = make_float4(hh[0], hh[1], hh[2], hh[3]);
  }
  };
  if (APF != 0 || tick > 0) particles(std::true_type{});
  else particles(std::false_type{});
  if (!full) {                                   // the last tile's padding slots carry no weight
#pragma unroll
    for (int idx = 0; idx < kPerThread; ++idx)
      if (tile0 + 4 * (tid + kThreads * (idx >> 2)) + (idx & 3) >= p.N) x[idx] = -INFINITY;
  }

  // tile max -> power-of-two exponent n_k (all tile weights <= 1)
  float mx = x[0];
#pragma unroll
  for (int e = 1; e < kPerThread; ++e) mx = fmaxf(mx, x[e]);
  mx = warp_max_f(mx);
  if (lane == 0) s_max[warp] = mx;
  group_sync(bar);
  mx = s_max[0];
#pragma unroll
  for (int w = 1; w < kThreads / 32; ++w) mx = fmaxf(mx, s_max[w]);
  const int nk = (mx == -INFINITY) ? kNkEmpty : (int)ceilf(fmaxf(mx, -1.0e9f));
  // an empty tile (every log-weight -inf) gets the frame +inf: 2^(-inf) = 0 for all of it
  const float fnk = (nk == kNkEmpty) ? INFINITY : (float)nk;

  float fS = 0.f, fQ = 0.f, fH = 0.f;
  float lG0 = 0.f, lF0 = 0.f, lG1 = 0.f, lF1 = 0.f;   // online-learning score sums (tile frame)
  unsigned long long E = 0ull;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i0 = tile0 + 4 * (tid + kThreads * r);
    float dv[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int idx = 4 * r + e;
      const float d = x[idx] - fnk;
      const float w = tile_weight(d);
      dv[e] = d;
      fS += w;
      fQ = fmaf(w, w, fQ);
      fH = fmaf(w, hv[idx], fH);
      E += fix_weight(w);
      if (LEARN) {
        // d log p(y|h)/dh at h_t (PTX :1187-1204) and d h_t / d rho = h_{t-1} - mu
        const float q = y2 * ex2_approx(hv[idx] * -kLog2e);
        const float dlw = gauss ? 0.5f * (q - 1.0f)
                                : fmaf(obs.nu_p1h, div_approx(q * obs.inv_nu, 1.0f + q * obs.inv_nu), -0.5f);
        const float dh = hpv[idx] - a.mu;
        const float wd = w * dlw, wd2 = wd * dlw;
        lG0 += wd;
        lF0 += wd2;
        lG1 = fmaf(wd, dh, lG1);
        lF1 = fmaf(wd2, dh * dh, lF1);
      }
    }
    *reinterpret_cast<float4*>(p.w + i0) = make_float4(dv[0], dv[1], dv[2], dv[3]);
  }
  // tile partials: the per-thread FP32 sums are staged in shared memory and one
  // warp adds them in FP64 (and the exact masses in u64), in a fixed order
  s_part[0][tid] = fS; s_part[1][tid] = fQ; s_part[2][tid] = fH; s_E[tid] = E;
  group_sync(bar);
  if (warp == 0) {
    double tS = 0.0, tQ = 0.0, tH = 0.0;
    unsigned long long tE = 0ull;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
      tS += (double)s_part[0][lane + 32 * w];
      tQ += (double)s_part[1][lane + 32 * w];
      tH += (double)s_part[2][lane + 32 * w];
      tE += s_E[lane + 32 * w];
    }
    tS = warp_sum_d(tS); tQ = warp_sum_d(tQ); tH = warp_sum_d(tH);
    tE = warp_sum_u64(tE);
    if (lane == 0) {
      p.nexp[k] = nk;
      p.E[k] = tE;
      p.rec[k] = make_float4((float)tS, (float)tQ, (float)tH, __int_as_float(nk));
    }
  }
  if (LEARN) {
    group_sync(bar);                                 // s_red is reused
    const double g0 = warp_sum_d((double)lG0), f0 = warp_sum_d((double)lF0);
    const double g1 = warp_sum_d((double)lG1), f1 = warp_sum_d((double)lF1);
    if (lane == 0) { s_red[0][warp] = g0; s_red[1][warp] = f0; s_red[2][warp] = g1; s_redE[warp] = 0ull; }
    double* s_red4 = sh.s_red4;
    if (lane == 0) s_red4[warp] = f1;
    group_sync(bar);
    if (tid == 0) {
      double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w) { t0 += s_red[0][w]; t1 += s_red[1][w]; t2 += s_red[2][w]; t3 += s_red4[w]; }
      p.rec2[k] = make_float4((float)t0, (float)t1, (float)t2, (float)t3);
    }
  }
}

__device__ __forceinline__ void tail_plan(const Plan& p, const TickArgs& a);

// TAIL: the last CTA to finish (a ticket taken after each CTA's tile record is out) runs the
// plan for the whole filter, in place of the plan kernel (filters of at most kTailTiles tiles).
template <bool TSTATE, bool LEARN, int APF, bool GAUSS, bool TAIL>
__global__ void __launch_bounds__(kThreads, 4) pass1_kernel(Plan p, TickArgs a) {
  __shared__ Pass1Shared sh;
  griddep_wait();
  const DevState* st = p.st;
  if (a.mirror && blockIdx.x == 0 && threadIdx.x == 0) p.st->seq = a.seq;   // for the plan's mirror
  // Each pass walks the tiles in the order opposite to the previous pass over
  // the particle arrays, so it starts on the tiles that pass wrote last, still
  // in L2 (the arrays are rewritten in place every tick).
  const int k = (st->dirs & 1) ? (p.G - 1 - (int)blockIdx.x) : (int)blockIdx.x;
  pass1_tile<TSTATE, LEARN, APF, GAUSS>(p, a, st, k, (int)threadIdx.x, 0, sh);
  if constexpr (TAIL) tail_plan(p, a);
  griddep_release();
}

// ---------------------------------------------------------------------------
// Plan: one CTA of kPlanThreads threads. Every tick it combines the tile
// records and takes the resampling decision; on resampling ticks it stages
// the tile exponents and fixed-point masses in shared memory with coalesced
// loads and builds the prefix, the target spacing and the work list there.
// ---------------------------------------------------------------------------
template <int NT>
struct PlanShared {
  int red_i[NT / 32];
  double red[3][NT / 32];
  double learn3[NT / 32];
  double tot[3];
  double res[4];
  unsigned long long scan_u[NT / 32 + 1];
  int scan_i[NT / 32 + 1];
  unsigned long long b_base, b_delta, b_magic;
  int b_resample, b_Fg;
};

__host__ __device__ constexpr size_t plan_smem_bytes(int G) {
  return G <= kPlanSmemTiles ? (size_t)G * 8 + (size_t)(2 * G + 1) * 4 : 0;
}

// The tick's outcome from its statistics, by one thread: the log-likelihood increment and the
// tick's record, the resampling decision and the device state of the next tick.
// res = {log-sum of the weights in the carry frame, ESS, filtered mean, ln S}.
// Returns the resampling decision.
__device__ __forceinline__ int plan_decide(const TickArgs& a, DevState* st, int N, int nM, bool degenerate,
                                           const double* res, double tS, BpfTickRecord* rec_out) {
  const int tick = st->tick, cur = st->cur;
  double dll, ess, hm;
  int resample = 0;
  if (degenerate) {
    dll = -INFINITY; ess = 0.0; hm = __longlong_as_double(0x7FF8000000000000LL);
    st->error = BPF_ERR_DEGENERATE;
  } else {
    dll = res[0] - st->logS_prev;
    ess = res[1];
    hm = res[2];
    resample = (a.ess_threshold <= 0.0f) || (ess / (double)N < (double)a.ess_threshold);
  }
  // Auxiliary particle filter: the first stage leaves log mean v (its weights)
  // in ll_ref for the second, whose increment is log mean v + log mean w; the
  // record's loglik_ref is log mean w, the value the reference reports
  // (gpu_bpf_ptx_full.cu:1155-1164). The tick advances after the second stage.
  double rec_dll = dll, ll_ref;
  if (a.apf == 1) {
    ll_ref = dll;
  } else if (a.apf == 2) {
    rec_dll = st->ll_ref + dll;
    ll_ref = dll;
  } else {
    ll_ref = (st->resampled_prev ? 0.0 : st->ll_ref) + dll;
  }
  st->ll_ref = ll_ref;
  st->hm = degenerate ? 0.0 : hm;
  if (a.apf != 1) st->ll_total += rec_dll;
  if (a.aux) *a.aux = degenerate ? make_float2(0.0f, __int_as_float(0))
                                 : make_float2((float)(1.0 / tS), __int_as_float(nM));
  if (rec_out) {
    BpfTickRecord r;
    r.dloglik = rec_dll; r.loglik_ref = ll_ref; r.loglik_total = st->ll_total;
    r.h_mean = (float)hm; r.ess = (float)ess; r.resampled = resample; r.tick = tick;
    *rec_out = r;
  }
  {
    // pass 2 runs opposite to this pass 1; the next pass 1 opposite to the
    // last pass that wrote the particles (pass 2 on a resampling tick)
    const int d1 = st->dirs & 1;
    st->dirs = (resample ? d1 : (d1 ^ 1)) | ((d1 ^ 1) << 1);
  }
  if (a.apf != 1) {
    st->k1 = st->k1 * kPcgMult;          // next tick's stream constants
    st->k2 = st->k2 * kPcgMult + 1ull;
    st->tick = tick + 1;
  }
  st->do_resample = resample;
  st->nM = nM;
  if (resample) {
    const uint64_t old = st->u_state;
    st->u_state = old * kPcgMult + kHostInc;
    st->u23 = pcg_output(old) >> 9;
    st->logS_prev = a.log_n;
    st->resampled_prev = 1;
    st->resample_count += 1;
    st->src = cur;
    st->cur = cur ^ 1;
  } else if (degenerate) {
    st->logS_prev = a.log_n;             // restart from uniform weights
    st->resampled_prev = 1;
  } else {
    st->logS_prev = res[3];
    st->resampled_prev = 0;
    st->nM_prev = nM;
  }
  return resample;
}

// Where the plan finds the tile records of the tick and puts the tile prefixes: the plan
// kernel reads the global copies pass 1 wrote (through L2) and writes P to global memory.
struct PlanGlobalIO {
  const Plan* p;
  static constexpr bool kStoreState = true;      // write the device state back to p.st
  __device__ __forceinline__ float4 rec(int k) const { return __ldcg(p->rec + k); }
  __device__ __forceinline__ int nexp(int k) const { return __ldcg(p->nexp + k); }
  __device__ __forceinline__ unsigned long long E(int k) const { return __ldcg(p->E + k); }
  __device__ __forceinline__ void set_P(int k, unsigned long long v) const { p->P[k] = v; }
};

// The plan of one tick by a CTA of NT threads on the device state s_st held in
// shared memory (the body's first barrier comes before its first read of s_st);
// it ends by writing s_st back to p.st when IO::kStoreState. ITEMS: also write pass 2's
// work items.
template <int NT, bool ITEMS, class IO>
__device__ __forceinline__ void plan_body(const Plan& p, const TickArgs& a, DevState& s_st, PlanShared<NT>& sh,
                                          unsigned char* plan_smem, const IO& io, BpfTickRecord* rec_out,
                                          TickMirror* mirror_out) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int G = p.G, N = p.N;
  DevState* st = &s_st;
  auto store_state = [&]() {
    nt_sync<NT>();
    if (!IO::kStoreState) return;
    if (tid < kStWords)
      reinterpret_cast<unsigned long long*>(p.st)[tid] = reinterpret_cast<const unsigned long long*>(&s_st)[tid];
    if (tid == 0 && mirror_out) {
      __threadfence_system();                 // the record first, then the mirror naming its request
      TickMirror mm;
      mm.resample_count = st->resample_count; mm.tick = st->tick; mm.error = st->error; mm.seq = st->seq;
      *mirror_out = mm;
    }
  };

  // 1. FP64 combine of the tile partials (one 16-byte record per tile, eight in
  //    flight per thread), per thread in a running frame 2^nrun
  int nrun = kNkEmpty;
  double S = 0.0, Q = 0.0, H = 0.0;
  for (int k0 = 0; k0 < G; k0 += 8 * NT) {
    float4 r8[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int k = k0 + u * NT + tid;
      r8[u] = (k < G) ? io.rec(k) : make_float4(0.f, 0.f, 0.f, __int_as_float(kNkEmpty));
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int nk = __float_as_int(r8[u].w);
      if (nk == kNkEmpty) continue;
      if (nk > nrun) {
        const double sc = (nrun == kNkEmpty) ? 0.0 : pow2d(nrun - nk);
        S *= sc; Q *= sc * sc; H *= sc;
        nrun = nk;
      }
      const double sc = pow2d(nk - nrun);
      S += (double)r8[u].x * sc; Q += (double)r8[u].y * (sc * sc); H += (double)r8[u].z * sc;
    }
  }
  // 2. global frame 2^nM, FP64 block sums
  const int nM = block_max_i<NT>(nrun, sh.red_i);   // barrier: s_st loaded
  if (nrun != kNkEmpty) {
    const double sc = pow2d(nrun - nM);
    S *= sc; Q *= sc * sc; H *= sc;
  } else {
    S = Q = H = 0.0;
  }
  S = warp_sum_d(S); Q = warp_sum_d(Q); H = warp_sum_d(H);
  if (lane == 0) { sh.red[0][warp] = S; sh.red[1][warp] = Q; sh.red[2][warp] = H; }
  nt_sync<NT>();

  // 3. tick statistics: the FP64 transcendental/division chains (on different warps
  //    of a full CTA; in every lane of a single warp, which avoids serialising
  //    divergent branches), then thread 0 takes the decision
  constexpr double kLn2d = 0.693147180559945309417232121458;
  double tS, tQ, tH;
  if constexpr (NT == 32) {
    tS = S; tQ = Q; tH = H;                        // the warp sums, complete in every lane
  } else {
    if (lane == 0 && warp < 3) {
      double v = 0.0;
      for (int w = 0; w < NT / 32; ++w) v += sh.red[warp][w];
      sh.tot[warp] = v;
    }
    nt_sync<NT>();
    tS = sh.tot[0]; tQ = sh.tot[1]; tH = sh.tot[2];
  }
  const bool degenerate = (nM == kNkEmpty) || !(tS > 0.0);
  if (!degenerate) {
    if constexpr (NT == 32) {
      const double L = log(tS);
      const double r0 = __fma_rn((double)nM, kLn2d, L), r1 = tS * tS / tQ, r2 = tH / tS;
      if (lane == 0) { sh.res[0] = r0; sh.res[1] = r1; sh.res[2] = r2; sh.res[3] = L; }
    } else if (lane == 0) {
      if (warp == 0) sh.res[0] = __fma_rn((double)nM, kLn2d, log(tS));   // log-sum in the carry frame
      if (warp == 1) sh.res[1] = tS * tS / tQ;                            // ESS
      if (warp == 2) sh.res[2] = tH / tS;                                 // filtered mean
      if (warp == 3) sh.res[3] = log(tS);
    }
  }
  nt_sync<NT>();
  // online learning: normalised score sums of this tick, FP64 in the global frame
  if (a.learn && p.rec2 && st->tick > 0 && !degenerate) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k = tid; k < G; k += NT) {
      const int nk = __float_as_int(io.rec(k).w);
      if (nk == kNkEmpty) continue;
      const float4 r2 = __ldcg(p.rec2 + k);
      const double sc = pow2d(nk - nM);
      v[0] += (double)r2.x * sc; v[1] += (double)r2.y * sc; v[2] += (double)r2.z * sc; v[3] += (double)r2.w * sc;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = warp_sum_d(v[q]);
    nt_sync<NT>();                                  // sh.red is free again
    if (lane == 0) { sh.red[0][warp] = v[0]; sh.red[1][warp] = v[1]; sh.red[2][warp] = v[2]; }
    if (lane == 0) sh.learn3[warp] = v[3];
    nt_sync<NT>();
    if (tid < 4) {
      double t = 0.0;
      for (int w = 0; w < NT / 32; ++w) t += (tid < 3) ? sh.red[tid][w] : sh.learn3[w];
      st->learn[tid] += t / tS;
    }
    nt_sync<NT>();
  }
  if (tid == 0) {
    sh.b_resample = plan_decide(a, st, N, nM, degenerate, sh.res, tS, rec_out);
    sh.b_Fg = min(kFixF, 62 - ceil_log2_u((unsigned)N));
  }
  nt_sync<NT>();
  if (!sh.b_resample) {
    store_state();
    return;
  }

  // staging arrays: shared memory when the tile count fits, else the global copies
  const bool in_smem = G <= kPlanSmemTiles;
  unsigned long long* e_s = in_smem ? reinterpret_cast<unsigned long long*>(plan_smem) : p.E;
  int* n_s = in_smem ? reinterpret_cast<int*>(plan_smem + (size_t)G * 8) : p.nexp;
  int* o_s = in_smem ? n_s + G : p.ofirst;
  if (in_smem) {
    for (int k0 = 0; k0 < G; k0 += 4 * NT) {
      int nk[4]; unsigned long long e4[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int k = k0 + u * NT + tid;
        if (k < G) { nk[u] = io.nexp(k); e4[u] = io.E(k); }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int k = k0 + u * NT + tid;
        if (k < G) { n_s[k] = nk[u]; e_s[k] = e4[u]; }
      }
    }
  }
  nt_sync<NT>();

  // 4. fixed-point CDF over contiguous runs of tiles: masses in the global
  //    frame, prefix and total
  const int Fg = sh.b_Fg;
  const int C = (G + NT - 1) / NT;
  const int k0 = min(tid * C, G), k1 = min(k0 + C, G);
  auto ehat = [&](int k) -> unsigned long long {
    const int nk = n_s[k];
    if (nk == kNkEmpty) return 0ull;
    return shr64(e_s[k], nM - nk + kFixF - Fg);
  };
  unsigned long long part = 0ull;
  for (int k = k0; k < k1; ++k) part += ehat(k);
  unsigned long long total;
  const unsigned long long excl = block_excl_scan_add<NT>(part, &total, sh.scan_u);
  if (tid == 0) {
    unsigned long long delta = udiv_fp64(total, (unsigned long long)N);
    if (delta == 0ull) { delta = 1ull; st->error = BPF_ERR_DEGENERATE; }
    const unsigned long long u = st->u23;
    const unsigned long long hi = __umul64hi(u, delta), lo = u * delta;
    sh.b_base = (hi << 41) | (lo >> 23);          // floor(u * delta / 2^23)
    sh.b_delta = delta;
    sh.b_magic = udiv_magic_of(delta);
    st->base = sh.b_base; st->delta = delta; st->delta_magic = sh.b_magic; st->total = total;
    st->Fg = Fg;
  }
  nt_sync<NT>();
  const unsigned long long base = sh.b_base, delta = sh.b_delta, magic = sh.b_magic;

  // 5. per tile: prefix, first output index, number of work items (a taped
  //    run gives every tile an item, so pass 2 writes every parent's first child)
  const int min_items = a.csr ? 1 : 0;
  unsigned long long run = excl;
  int o = targets_below(run, base, delta, magic, N);
  int n_it = 0;
  for (int k = k0; k < k1; ++k) {
    io.set_P(k, run);
    o_s[k] = o;
    run += ehat(k);
    const int o_next = targets_below(run, base, delta, magic, N);
    n_it += max((o_next - o + kOutChunk - 1) / kOutChunk, min_items);
    o = o_next;
  }
  const int o_end = o;     // first output of the next thread's first tile (N for the last)
  int n_items_total;
  const int it0 = block_excl_scan_add<NT>(n_it, &n_items_total, sh.scan_i);

  // 6. work items (tile, first output, end output, flags: 1 = first item of the
  //    tile, 2 = the only one, holding all of the tile's outputs);
  //    heavy tiles are split
  int ib = it0;
  for (int k = k0; ITEMS && k < k1; ++k) {
    const int o0 = o_s[k];
    const int o1 = (k + 1 < k1) ? o_s[k + 1] : o_end;
    const int ni = max((o1 - o0 + kOutChunk - 1) / kOutChunk, min_items);
    for (int u = 0; u < ni; ++u) {
      const int oo = o0 + u * kOutChunk;
      p.items[ib++] = make_int4(k, oo, min(o1, oo + kOutChunk), (u == 0 ? 1 : 0) | (ni == 1 ? 2 : 0));
    }
  }
  if (tid == 0) st->n_items = n_items_total;
  store_state();
}

// The plan in pass 1's last CTA: every CTA's tile record is out before its ticket (a fence
// between), so the CTA that takes the last ticket sees them all after a second fence.
__device__ __forceinline__ void tail_plan(const Plan& p, const TickArgs& a) {
  __shared__ PlanShared<kThreads> sh;
  __shared__ __align__(16) DevState s_st;
  __shared__ __align__(16) unsigned char stage[plan_smem_bytes(kTailTiles)];
  __shared__ unsigned s_last;
  __syncthreads();                               // the tile record of this CTA is written
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = (atomicAdd(p.pticket, 1u) == (unsigned)(p.G - 1)) ? 1u : 0u;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  if (threadIdx.x < kStWords)
    reinterpret_cast<unsigned long long*>(&s_st)[threadIdx.x] =
        __ldcg(reinterpret_cast<const unsigned long long*>(p.st) + threadIdx.x);
  if (threadIdx.x == 0) *p.pticket = 0u;          // for the next tick
  plan_body<kThreads, true>(p, a, s_st, sh, stage, PlanGlobalIO{&p}, a.rec, a.mirror);
}

__global__ void __launch_bounds__(kPlanThreads, 1) plan_kernel(Plan p, TickArgs a) {
  __shared__ PlanShared<kPlanThreads> sh;
  __shared__ __align__(16) DevState s_st;
  extern __shared__ __align__(16) unsigned char plan_smem[];
  griddep_wait();
  // the device state lives in shared memory for the whole kernel (one load, one store)
  if (threadIdx.x < kStWords)
    reinterpret_cast<unsigned long long*>(&s_st)[threadIdx.x] =
        __ldcg(reinterpret_cast<const unsigned long long*>(p.st) + threadIdx.x);
  plan_body<kPlanThreads, true>(p, a, s_st, sh, plan_smem, PlanGlobalIO{&p}, a.rec, a.mirror);
  griddep_release();
}

// ---------------------------------------------------------------------------
// Pass 2: persistent CTAs, four per SM; the tiles (h and w) of a work item
// are fetched by bulk async copies into shared memory as soon as the previous
// item has released the buffer (the other CTAs on the SM hide the latency).
// ---------------------------------------------------------------------------
constexpr size_t kTileBytes = (size_t)kTile * 4;
// u16 ancestor (tile-local + 1) per output slot of a window; a window starts
// at its item's first output rounded down to a multiple of 4 (up to 3 extra
// slots), rounded up to whole 256-slot steps of the gather (8 slots a lane)
constexpr int kGatherStep = 256;
constexpr size_t kMarkBytes = ((size_t)kOutChunk + kGatherStep) * 2;
constexpr size_t kMarkOffset = 2 * kTileBytes;                 // after the staged h and w tiles
constexpr size_t kPass2Smem = kMarkOffset + kMarkBytes;         // one staged tile (h, w) + marks
static_assert(kMarkOffset % 16 == 0 && kMarkBytes % 16 == 0, "marks are cleared with 16-byte stores");
static_assert((size_t)kOutChunk % kGatherStep == 0, "the gather reads marks in steps of 256 slots");

// Tile-frame thresholds of the child count are kept relative to the thread's first
// element and capped here: a thread's 16 fixed-point weights sum to at most 16 * 2^50
// < kThCap, so a capped threshold is never reached, and threshold + c * spacing stays
// below 2^57 for every count c the loop forms.
constexpr unsigned long long kThCap = 1ull << 55;

// Exact count of targets up to element `upto` of a thread's 16 staged log2-weights d:
// #{m >= 0 : R0 + m D <= sum_{i <= upto} floor(2^d_i 2^50)}, at most cap. The rare path of
// the FP32 estimate in pass 2's child count.
__device__ __noinline__ int exact_count(const float* d, int upto, unsigned long long R0, unsigned long long D,
                                        int cap) {
  unsigned long long l = 0ull;
  for (int i = 0; i <= upto; ++i) l += fix_weight(tile_weight(d[i]));
  if (l < R0) return 0;
  const unsigned long long c = udiv_fp64(l - R0, D) + 1ull;
  return c >= (unsigned long long)cap ? cap : (int)c;
}

__device__ __forceinline__ void pass2_fetch(const Plan& p, const float* hsrc, int it, unsigned char* buf,
                                            uint64_t* bar) {
  const int k = p.items[it].x;
  mbar_expect_tx(bar, 2u * (uint32_t)kTileBytes);
  bulk_load(buf, hsrc + (size_t)k * kTile, (uint32_t)kTileBytes, bar);
  bulk_load(buf + kTileBytes, p.w + (size_t)k * kTile, (uint32_t)kTileBytes, bar);
}

__global__ void __launch_bounds__(kThreads, 4) pass2_kernel(Plan p, TickArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned short* marks = reinterpret_cast<unsigned short*>(smem + kMarkOffset);
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ unsigned long long s_scan[kThreads / 32 + 1];
  __shared__ unsigned s_wmax[kThreads / 32];
  __shared__ int s_err;

  griddep_wait();
  const DevState* st = p.st;
  if (!st->do_resample) {
    griddep_release();
    return;
  }
  const int n_items = st->n_items;
  const bool rev = ((st->dirs >> 1) & 1) != 0;     // item order opposite to this tick's pass 1
  const unsigned long long base = st->base, delta = st->delta, magic = st->delta_magic;
  const int nM = st->nM, Fg = st->Fg, N = p.N;
  const int src = st->src;
  const float* hsrc = src ? p.h1 : p.h0;
  float* hdst = src ? p.h0 : p.h1;
  // the ancestor record takes vector stores only from a 16-byte aligned base
  const bool anc_vec = ((reinterpret_cast<uintptr_t>(a.anc) & 15u) == 0u);
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_err = 0;
    mbar_init(&mbar[0], 1);
    if ((int)blockIdx.x < n_items) pass2_fetch(p, hsrc, rev ? n_items - 1 - (int)blockIdx.x : (int)blockIdx.x, smem, &mbar[0]);
  }
  __syncthreads();

  const float* hs = reinterpret_cast<const float*>(smem);
  const float* ws = reinterpret_cast<const float*>(smem + kTileBytes);
  int n = 0;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x, ++n) {

    const int4 item = p.items[rev ? n_items - 1 - it : it];
    const int k = item.x, oa = item.y, ob = item.z;
    const int wa = oa & ~3;                          // window origin: 16-byte aligned output slot
    const int j0 = k * kTile;
    const int nA = min(kTile, N - j0);
    const int nB = ob - wa;                          // window slots [wa, ob); [wa, oa) belong to other items
    const int r = nM - p.nexp[k] + kFixF - Fg;       // tile frame -> global frame shift
    const unsigned long long Pk = p.P[k];
    // A staged copy that does not land within the wait's limit ends the CTA's work: the error is
    // recorded, thread 0 waits once more (bounded) for that copy, and no further copy is issued
    // into the buffer, so the CTA never reads a partial tile or leaves with its own copy in flight
    // unless the second wait gives up too.
    if (__syncthreads_or(!mbar_wait_bounded(&mbar[0], (uint32_t)n & 1u))) {
      if (tid == 0) {
        s_err = 1;
        mbar_wait_bounded(&mbar[0], (uint32_t)n & 1u);
      }
      break;
    }

    // clear this window's ancestor marks (the previous item's gather has finished:
    // the loop ends with a barrier; the scan's barriers order this before the marks)
    const int nBs = (nB + kGatherStep - 1) & ~(kGatherStep - 1);
    for (int x = tid; x < nBs / 8; x += kThreads) reinterpret_cast<uint4*>(marks)[x] = make_uint4(0u, 0u, 0u, 0u);

    // Exact fixed-point prefix of the tile: 16 contiguous weights per thread
    // (summed here, rebuilt element by element below from the staged tile).
    // A tile whose shift reaches 64 has no mass in the global frame. Slots past N
    // hold the log2-weight -inf (weight 0), so they need no test here or below.
    const float4* wt = reinterpret_cast<const float4*>(ws + tid * kPerThread);
    const bool massive = r < 64;
    unsigned long long run = 0ull;
    float lfT = 0.0f;            // FP32 sum of the thread's weights, in the child count's order
    if (massive) {
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const float4 f = wt[v];
        const float a0 = tile_weight(f.x), a1 = tile_weight(f.y), a2 = tile_weight(f.z), a3 = tile_weight(f.w);
        run += fix_weight(a0) + fix_weight(a1);
        run += fix_weight(a2) + fix_weight(a3);
        lfT += a0; lfT += a1; lfT += a2; lfT += a3;
      }
    }
    unsigned long long tot;
    // (no trailing barrier: s_scan is next written by the next item's scan, three barriers on)
    const unsigned long long excl = block_excl_scan_add<kThreads, unsigned long long, false>(run, &tot, s_scan);

    // Element j owns the output slots [q_{j-1}, q_j): the targets t_q below its CDF value
    // C_j = P_k + (A_j >> r) (A_j its tile-local inclusive prefix) and not below the previous
    // element's. In the tile's own frame, C_j > t_q  <=>  A_j >= ((t_q - P_k + 1) << r), and
    // consecutive targets are D = delta << r apart there. Relative to the thread's first
    // element (exclusive prefix A_s, first target q0 at relative threshold R0), the count up to
    // element j is c_j = #{m >= 0 : R0 + m D <= l_j}, l_j = A_j - A_s, so q_j = min(q0 + c_j, N).
    // c_j is estimated in FP32 from the FP32 running sum of the weights, with a bound on the
    // estimate's error (every rounding and the fixed-point truncation counted): when no integer
    // boundary lies within the bound the estimate's floor is exact, otherwise (a warp vote)
    // the element recounts in exact 64-bit integers. Each element with children writes one
    // start mark, at its first slot inside this window.
    const int lane = tid & 31, warp = tid >> 5;
    const int q0 = targets_below(Pk + shr64(excl, r), base, delta, magic, N);
    unsigned long long R0 = kThCap, D = kThCap;      // capped: never reached (see kThCap)
    if (massive && q0 < N) {
      const unsigned long long m = base + (unsigned long long)q0 * delta - Pk + 1ull;   // t_q0 >= P_k
      if (m <= (~0ull >> r)) R0 = min((m << r) - excl, kThCap);                          // (m << r) > excl
      if (delta <= (kThCap >> r)) D = delta << r;
    }
    const float R0w = (float)R0 * 0x1p-50f;           // in units of the tile's largest weight
    const float invDw = 1.0f / ((float)D * 0x1p-50f);
    const float R0x = R0w * invDw;                    // the estimate is x = lf invDw - R0x (one FMA)
    // Bound on the estimate's error at an element with running sum lf and estimate x:
    // (lf + R0w) 2^-18 / Dw + 2^-44 / Dw + |x| 2^-21. Every term is non-negative and the
    // roundings are monotone, so it is largest at the thread's largest lf (lfT, the same
    // additions in the same order) and largest |x| (x runs from at least -R0x up to xT): the
    // thread takes that one bound for all its elements. A wider bound only sends more elements
    // to the exact recount. Estimates of 2^22 and more (xT) recount every element.
    const float eL = 0x1p-18f * invDw, e0 = fmaf(R0w, eL, 0x1p-44f * invDw);
    const float xT = fmaf(lfT, invDw, -R0x);
    float err = fmaf(lfT, eL, fmaf(fmaxf(fabsf(xT), R0x), 0x1p-21f, e0));
    if (!(xT < 0x1p22f)) err = 1.0f;
    const float err_hi = 1.0f - err;
    const float* wsel = ws + tid * kPerThread;
    int32_t* csr = (a.csr && (item.w & 1)) ? a.csr + j0 : nullptr;   // children of j: [csr[j], csr[j+1])
    // Output slots below are relative to the window origin wa. The end of element j's children,
    // min(q0 + c_j, N) with c_j = max(floor(x) + 1, 0), is formed from the bits of fl + 2^23
    // (exact for the fl that pass the bound) as min(max(bits - Kq, qlo), nr).
    const int qlo = q0 - wa, nr = N - wa, oar = oa - wa, obr = ob - wa;
    const int Kq = 0x4AFFFFFF - qlo;
    // Compile-time variants: WHOLE (the item holds every output of the tile, so each
    // counted child lands in the window), TAPE (first-child list for the gradient tape).
    const bool whole = (item.w & 2) != 0;
    auto count_children = [&](auto whole_tag, auto tape_tag) {
      constexpr bool WHOLE = decltype(whole_tag)::value;
      constexpr bool TAPE = decltype(tape_tag)::value;
      float lf = 0.0f;
      int qp = qlo;                                  // first slot of the next element's children
#pragma unroll 1
      for (int g = 0; g < 4; ++g) {
        const float4 f4 = wt[g];
        const float ff[4] = {f4.x, f4.y, f4.z, f4.w};
        int qq[4];
        bool rc[4], any = false;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          lf += tile_weight(ff[e]);
          const float x = fmaf(lf, invDw, -R0x);
          const float fl = floorf(x);
          const float fr = x - fl;                       // exact
          rc[e] = !(fr > err && fr < err_hi);
          any |= rc[e];
          qq[e] = min(max(__float_as_int(fl + 0x1p23f) - Kq, qlo), nr);
        }
        if (__any_sync(0xffffffffu, any)) {            // one vote per four elements
#pragma unroll
          for (int e = 0; e < 4; ++e)
            if (rc[e]) qq[e] = min(qlo + exact_count(wsel, 4 * g + e, R0, D, N), nr);
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int j = tid * kPerThread + 4 * g + e;
          if (TAPE && j < nA) csr[j] = qp + wa;
          const int q1 = qq[e];
          if (q1 > qp && (WHOLE || (qp < obr && q1 > oar))) marks[WHOLE ? qp : max(qp, oar)] = (unsigned short)(j + 1);
          qp = q1;
        }
      }
    };
    if (massive) {
      if (csr) count_children(std::false_type{}, std::true_type{});
      else if (whole) count_children(std::true_type{}, std::false_type{});
      else count_children(std::false_type{}, std::false_type{});
    } else if (csr) {
      for (int e = 0; e < kPerThread; ++e)       // no mass: every element's children start at q0
        if (tid * kPerThread + e < nA) csr[tid * kPerThread + e] = q0;
    }
    __syncthreads();

    // Gather: the ancestor of window slot o is the last start mark at or
    // before o (marks increase along the window). Each warp takes a run of
    // slots in steps of 256 (8 per lane): the running maximum of the marks
    // is a lane-local scan, a warp max-scan and a carry from the earlier
    // steps and warps. A lane's 8 slots are 16-byte aligned in the output,
    // so whole groups are written with two vector stores; every slot from
    // the item's first one on has a mark at or before it, so a group that
    // lies inside the item needs no per-slot test.
    const int chunk = ((nB + kThreads / 32 - 1) / (kThreads / 32) + kGatherStep - 1) & ~(kGatherStep - 1);
    const int cs = warp * chunk, ce = min(cs + chunk, nB);
    unsigned wmax = 0u;
    for (int o0 = cs; o0 < ce; o0 += kGatherStep) {
      const uint4 m = reinterpret_cast<const uint4*>(marks + o0)[lane];
      const unsigned v = __vmaxu2(__vmaxu2(m.x, m.y), __vmaxu2(m.z, m.w));
      wmax = max(wmax, max(v & 0xffffu, v >> 16));
    }
    wmax = __reduce_max_sync(0xffffffffu, wmax);
    if (lane == 0) s_wmax[warp] = wmax;
    __syncthreads();
    unsigned carry = 0u;
    for (int w = 0; w < warp; ++w) carry = max(carry, s_wmax[w]);
    {
      const int olo = oa - wa;                       // first slot of this item in the window
      for (int o0 = cs; o0 < ce; o0 += kGatherStep) {
        const uint4 m = reinterpret_cast<const uint4*>(marks + o0)[lane];
        unsigned am[8];
        am[0] = m.x & 0xffffu;
        am[1] = max(am[0], m.x >> 16);
        am[2] = max(am[1], m.y & 0xffffu);
        am[3] = max(am[2], m.y >> 16);
        am[4] = max(am[3], m.z & 0xffffu);
        am[5] = max(am[4], m.z >> 16);
        am[6] = max(am[5], m.w & 0xffffu);
        am[7] = max(am[6], m.w >> 16);
        unsigned x = am[7];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const unsigned t = __shfl_up_sync(0xffffffffu, x, off);
          if (lane >= off) x = max(x, t);
        }
        unsigned pre = __shfl_up_sync(0xffffffffu, x, 1);
        pre = max(carry, lane == 0 ? 0u : pre);
        const int o = o0 + 8 * lane;
        if (o >= olo && o + 7 < ce) {
#pragma unroll
          for (int hf = 0; hf < 2; ++hf) {
            float hv[4];
            int av[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const unsigned jj = max(pre, am[4 * hf + u]);
              hv[u] = hs[jj - 1u];
              av[u] = j0 + (int)(jj - 1u);
            }
            *reinterpret_cast<float4*>(hdst + wa + o + 4 * hf) = make_float4(hv[0], hv[1], hv[2], hv[3]);
            if (a.anc) {
              if (anc_vec) *reinterpret_cast<int4*>(a.anc + wa + o + 4 * hf) = make_int4(av[0], av[1], av[2], av[3]);
              else for (int u = 0; u < 4; ++u) a.anc[wa + o + 4 * hf + u] = av[u];
            }
          }
        } else {
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            if (o + u >= olo && o + u < ce) {
              unsigned jj = max(pre, am[u]);
              if (jj - 1u >= (unsigned)nA) { jj = 1u; s_err = 1; }   // unreachable by construction
              hdst[wa + o + u] = hs[jj - 1u];
              if (a.anc) a.anc[wa + o + u] = j0 + (int)(jj - 1u);
            }
          }
        }
        carry = max(carry, __shfl_sync(0xffffffffu, x, 31));
      }
    }
    __syncthreads();   // the staged tile is free: fetch the next item's
    if (tid == 0 && it + (int)gridDim.x < n_items) {
      const int nx = it + (int)gridDim.x;
      pass2_fetch(p, hsrc, rev ? n_items - 1 - nx : nx, smem, &mbar[0]);
    }
  }
  __syncthreads();
  if (tid == 0 && s_err) {
    p.st->error = BPF_ERR_STATE;
    if (a.mirror) a.mirror->error = BPF_ERR_STATE;
  }
  griddep_release();
}

// ---------------------------------------------------------------------------
// Silverman jitter after a resampling tick (the reference's legacy option,
// gpu_bpf/gpu_bpf_ptx_full.cu:708-738 with kernels ptx_assembly/
// bpf_kernels_full.ptx:846-1060): bandwidth
//   bw = shrink * sigma_hat * 1.05922 * N^-0.2,  sigma_hat^2 = sum_i (h'_i - hm)^2 / N
// over the resampled particles h', hm the tick's filtered mean; then
//   h'_i = clamp(h'_i + bw z_i, mu - 8, mu + 8)
// with z_i the normal of particle slot i's next PCG32 draw. The reference
// draws z from the slot's own stream (bpf_gen_noise steps it), so each jitter
// takes one draw and the next propagation the one after it: here the draw's
// stream constants are the device state's current ones, and the variance
// kernel's last CTA advances them once more.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) jitter_var_kernel(Plan p, float shrink) {
  __shared__ float s_part[kThreads];
  __shared__ double s_red[kThreads / 32];
  __shared__ int s_last;
  griddep_wait();
  DevState* st = p.st;
  if (!st->do_resample) { griddep_release(); return; }
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k = blockIdx.x, tile0 = k * kTile;
  const float* h = st->cur ? p.h1 : p.h0;           // the resampled particles
  const float hmf = (float)st->hm;
  float acc = 0.0f;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i0 = tile0 + 4 * (tid + kThreads * r);
    const float4 v = *reinterpret_cast<const float4*>(h + i0);
    const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (i0 + u < p.N) { const float d = e[u] - hmf; acc = fmaf(d, d, acc); }
  }
  s_part[tid] = acc;
  __syncthreads();
  if (warp == 0) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) t += (double)s_part[lane + 32 * w];
    t = warp_sum_d(t);
    if (lane == 0) {
      p.jpart[k] = t;
      __threadfence();
      s_last = (atomicAdd(p.jticket, 1u) == (unsigned)(p.G - 1));
    }
  }
  __syncthreads();
  if (s_last) {
    // every tile's sum is visible (each was fenced before its ticket); fixed-order FP64 combine
    __threadfence();
    double v = 0.0;
    for (int j = tid; j < p.G; j += kThreads) v += __ldcg(p.jpart + j);
    v = warp_sum_d(v);
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    if (tid == 0) {
      double V = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) V += s_red[w];
      const double n = (double)p.N;
      st->bw = (float)((double)shrink * sqrt(V / n) * 1.05922 * pow(n, -0.2));
      st->jk1 = st->k1;                              // the jitter takes the next draw
      st->jk2 = st->k2;
      st->k1 = st->k1 * kPcgMult;                    // the next propagation the one after it
      st->k2 = st->k2 * kPcgMult + 1ull;
      *p.jticket = 0u;
    }
  }
  griddep_release();
}

__global__ void __launch_bounds__(kThreads) jitter_apply_kernel(Plan p, float mu) {
  griddep_wait();
  const DevState* st = p.st;
  if (!st->do_resample) { griddep_release(); return; }
  const int tid = threadIdx.x;
  const int tile0 = blockIdx.x * kTile;
  float* h = st->cur ? p.h1 : p.h0;
  const float bw = st->bw, lo = mu - 8.0f, hi = mu + 8.0f;
  const uint64_t k1 = st->jk1, k2 = st->jk2;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i0 = tile0 + 4 * (tid + kThreads * r);
    float4 v = *reinterpret_cast<const float4*>(h + i0);
    float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const float z = icdf_normal_warp(pcg_uniform(pcg_output(k1 + k2 * pcg_inc((uint32_t)(i0 + u)))));
      if (i0 + u < p.N) e[u] = fminf(fmaxf(fmaf(bw, z, e[u]), lo), hi);
    }
    *reinterpret_cast<float4*>(h + i0) = make_float4(e[0], e[1], e[2], e[3]);
  }
  griddep_release();
}

// ---------------------------------------------------------------------------
// Fused tick for small filters (N <= kSmallMaxN, at most kSmallTiles tiles): a
// thread-block cluster of one CTA per tile runs n consecutive ticks in one
// launch. The particles, log2-weights and tile records stay in shared memory
// from the first tick to the last; the CTAs read each other's records and write
// each other's resampled particles through distributed shared memory and meet at
// one cluster barrier per tick (two on resampling ticks).
//   pass 1    each CTA runs its tile with pass 1's per-particle arithmetic on
//             twice as many threads and hands the FP32 running sums along in
//             pass 1's element order, so every tile record is bit for bit pass 1's;
//             warps 0..3 form the FP64 record (one sum each); the exact fixed-point
//             masses of the tile's four-slot chunks are scanned only if the tick
//             resamples, beside the forming of the resampling plan;
//   plan      warp 0 of every CTA runs the plan over all the tile records (lane k
//             reads tile k's): the operations of the plan kernel in the same order
//             (so every CTA takes the same decision and holds the same device state);
//             CTA 0 writes the tick's record; warp 1 forms the resampling plan;
//   resample  the same fixed-point rule (integer exact, so the ancestors do not
//             depend on how the work is split): each CTA counts its tile's
//             children (pass 2's FP32 estimate with an exact recount near target
//             boundaries) and each parent writes its particle into its children's
//             output slots, in the shared memory of the CTA that owns each slot;
//             a barrier over the cluster ends the resampling. When every tick
//             resamples, the resampling runs beside the decision (it needs only
//             whether the tick is degenerate, which warp 1 finds from the same sums).
// Results equal the three-kernel tick's bit for bit: both particle buffers, the
// log2-weights and tile exponents are loaded at the start and written back at
// the end of the launch, with the device state.
// ---------------------------------------------------------------------------
constexpr int kSmallThreads = 4 * kThreads;             // 1024 threads per CTA (one tile)
constexpr int kSmallSplit = 2;                          // threads per pass-1 thread in the fused pass 1
constexpr int kChunks = kTile / 4;                      // four-slot chunks of a tile (one per thread)
constexpr int kYStage = kSmallThreads;                  // observations staged per refill
static_assert(kChunks == kSmallThreads, "one four-slot chunk per thread");

// What the finish of a tick's plan needs from its decision (plan_fused_decide -> plan_fused_finish).
struct FusedTail {
  double tS, tH, ess, logS_prev_old;
  int nM, degenerate, resample, resampled_prev_old, tick_old;
};

struct FusedPlan {
  unsigned long long base, delta, magic, total;
  int nM, Fg, items, zero_spacing;
  int live;                                   // threshold 0: the tick resamples (not degenerate)
};

struct FusedShared {
  float h[2][kTile];                          // particle buffers (DevState::cur / src), this CTA's tile
  float w[kTile];                             // log2-weights of the tile
  __align__(16) float z[kTile];               // state noise of the tick's propagation, slot by slot
  unsigned long long chunkE[kChunks];         // exact fixed-point mass of each four-slot chunk
  unsigned long long chunkP[kChunks];         // its exclusive prefix within the tile
  float ys[kYStage];                          // observations of the next ticks
  float4 rec[2];                              // tile record {S, Q, H, n_k}, by tick parity
  unsigned long long E[2];                    // exact fixed-point tile mass, by tick parity
  int nexp[2];                                // tile exponent, by tick parity
  FusedShared* peer[kSmallTiles];             // every CTA's FusedShared (distributed shared memory)
  __align__(16) DevState st;
  unsigned long long P[kSmallTiles];          // the tick's tile prefixes (all tiles)
  FusedPlan pl;                               // the tick's resampling plan
  FusedTail tail;                             // the tick's decision, for the finish of its plan
  float s_max[kSmallThreads / 32];
  float s_part[3][kThreads];
  unsigned long long s_E[kThreads];
  unsigned long long scan2[16];
  unsigned long long knext[2];                // the next tick's PCG32 stream constants k1, k2
};

template <int NCTA>
__device__ __forceinline__ void cluster_sync_all() {
  if constexpr (NCTA == 1) {
    __syncthreads();
  } else {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
  }
}

// Pass 1 of this CTA's tile (global slots tile0 .. tile0 + kTile - 1) on the shared-memory
// copies, by the first kThreads * SPLIT threads: pass-1 thread v's sixteen particles (four
// float4 groups r) go to SPLIT threads, 4 / SPLIT consecutive groups each, with the
// per-particle arithmetic of pass1_tile (the state noise read from sh.z, formed beforehand by
// fused_noise with the same draws); the FP32 tile partials are accumulated in pass 1's
// order by handing the running sums from one of those threads to the next, and warps 0..3 form
// the FP64 tile record in pass 1's order (one sum each). Within a warp the SPLIT threads of v sit 32 / SPLIT
// lanes apart, so the float4 accesses of a warp cover whole 128-byte rows. Group r of v is the
// four-slot chunk c = v + 256 r (slots 4c .. 4c + 3), whose exact mass goes to chunkE.
// nk_prev: the tile's exponent of the previous tick (the carried weights' frame).
template <bool TSTATE, bool GAUSS, int SPLIT>
__device__ __forceinline__ void pass1_fused(const TickArgs& a, float y, int N, int tile0, int par, int nk_prev,
                                            FusedShared& sh) {
  static_assert(SPLIT == 1 || SPLIT == 2 || SPLIT == 4, "four float4 groups per pass-1 thread");
  constexpr int R = 4 / SPLIT;                   // float4 groups of a thread
  constexpr int NT1 = kThreads * SPLIT;          // threads of pass 1
  constexpr int LW = 32 / SPLIT;                 // lanes of a warp with the same s
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int s = lane / LW, v = LW * warp + (lane % LW);
  float wv[4 * R], dv[4 * R], hv[4 * R];
  int nk = kNkEmpty;
  if (tid < NT1) {
    const DevState& st = sh.st;
    const int tick = st.tick;
    const bool carry = st.resampled_prev == 0;
    float* hb = sh.h[st.cur];
    ObsModel obs = a.obs;
    obs.y = y;
    const float y2 = y * y;
    float carry_off = 0.0f;
    if (carry) carry_off = (nk_prev == kNkEmpty) ? -INFINITY : (float)(nk_prev - st.nM_prev);
    const float gauss_c = kGaussLog2C + carry_off;
    const float t_c = __fmul_rn(obs.c_obs, kLog2e) + carry_off;
    const float y2nu = __fmul_rn(y2, obs.inv_nu);
    float x[4 * R];
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      const int l0 = 4 * (v + kThreads * (s * R + rr));
      const float4 h4 = *reinterpret_cast<const float4*>(hb + l0);
      const float4 w4 = carry ? *reinterpret_cast<const float4*>(sh.w + l0) : make_float4(0.f, 0.f, 0.f, 0.f);
      float hh[4] = {h4.x, h4.y, h4.z, h4.w};
      const float wp[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int i = tile0 + l0 + e;
        float h = hh[e];
        if (tick > 0) h = propagate(h, a.mu, a.rho, a.sigma, sh.z[l0 + e]);
        float xx = GAUSS ? obs_log2pdf_gauss_plus(y2, h, gauss_c) : obs_log2pdf_t_plus(obs, y2nu, h, t_c);
        if (carry) xx += wp[e];
        if (i >= N) xx = -INFINITY;               // padding slots carry no weight
        hh[e] = h;
        x[4 * rr + e] = xx;
        hv[4 * rr + e] = h;
      }
      *reinterpret_cast<float4*>(hb + l0) = make_float4(hh[0], hh[1], hh[2], hh[3]);
    }
    float mx = x[0];
#pragma unroll
    for (int e = 1; e < 4 * R; ++e) mx = fmaxf(mx, x[e]);
    mx = warp_max_f(mx);
    if (lane == 0) sh.s_max[warp] = mx;
    if constexpr (NT1 == kSmallThreads) __syncthreads();
    else asm volatile("bar.sync 1, %0;" ::"n"(NT1) : "memory");
    mx = warp_max_f(lane < NT1 / 32 ? sh.s_max[lane] : -INFINITY);
    nk = (mx == -INFINITY) ? kNkEmpty : (int)ceilf(fmaxf(mx, -1.0e9f));
    const float fnk = (nk == kNkEmpty) ? INFINITY : (float)nk;
    unsigned long long E = 0ull;
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      unsigned long long Ec = 0ull;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        dv[4 * rr + e] = x[4 * rr + e] - fnk;
        wv[4 * rr + e] = tile_weight(dv[4 * rr + e]);
        Ec += fix_weight(wv[4 * rr + e]);
      }
      const int c = v + kThreads * (s * R + rr);
      *reinterpret_cast<float4*>(sh.w + 4 * c) = make_float4(dv[4 * rr], dv[4 * rr + 1], dv[4 * rr + 2], dv[4 * rr + 3]);
      sh.chunkE[c] = Ec;
      E += Ec;
    }
    // pass 1's per-thread FP32 sums, in its element order, handed along the SPLIT threads
    float aS = 0.f, aQ = 0.f, aH = 0.f;
#pragma unroll
    for (int step = 0; step < SPLIT; ++step) {
      if (s == step) {
#pragma unroll
        for (int e = 0; e < 4 * R; ++e) {
          aS += wv[e];
          aQ = fmaf(wv[e], wv[e], aQ);
          aH = fmaf(wv[e], hv[e], aH);
        }
      }
      if (step + 1 < SPLIT) {
        const float nS = __shfl_up_sync(0xffffffffu, aS, LW);
        const float nQ = __shfl_up_sync(0xffffffffu, aQ, LW);
        const float nH = __shfl_up_sync(0xffffffffu, aH, LW);
        if (s == step + 1) { aS = nS; aQ = nQ; aH = nH; }
      }
    }
#pragma unroll
    for (int o = LW; o < 32; o <<= 1) E += __shfl_xor_sync(0xffffffffu, E, o);
    if (s == SPLIT - 1) { sh.s_part[0][v] = aS; sh.s_part[1][v] = aQ; sh.s_part[2][v] = aH; }
    if (s == 0) sh.s_E[v] = E;
  }
  __syncthreads();
  if (warp < 3) {                               // pass 1's FP64 tile sums S, Q, H, one a warp, same order
    double tw = 0.0;
    const float* part = sh.s_part[warp];
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) tw += (double)part[lane + 32 * w];
    tw = warp_sum_d(tw);
    if (lane == 0) reinterpret_cast<float*>(&sh.rec[par])[warp] = (float)tw;
  } else if (warp == 3) {                       // and the exact tile mass
    unsigned long long tE = 0ull;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) tE += sh.s_E[lane + 32 * w];
    tE = warp_sum_u64(tE);
    if (lane == 0) {
      sh.nexp[par] = nk;
      sh.E[par] = tE;
      reinterpret_cast<float*>(&sh.rec[par])[3] = __int_as_float(nk);
    }
  }
}

// The state noise of a tick for this CTA's tile into sh.z, by the threads from thread `first` on,
// in steps of `stride` four-slot groups (both multiples of 32, so every warp runs whole groups and the
// normal's warp vote sees all its lanes): slot i's draw of the tick with stream constants (k1, k2),
// pass 1's arithmetic (the draws are counter-based, so they are formed before the tick's particles
// are known, by warps that would otherwise wait).
template <bool TSTATE>
__device__ __forceinline__ void fused_noise(const TickArgs& a, int tile0, uint64_t k1, uint64_t k2, int first,
                                            int stride, FusedShared& sh) {
  const uint64_t k33 = k2 << 33;
  for (int g = (int)threadIdx.x - first; g < kTile / 4; g += stride) {
    float zz[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const uint64_t st64 = k1 + k2 * pcg_inc((uint32_t)(tile0 + 4 * g + e));
      float z = icdf_normal_warp(pcg_uniform(pcg_output(st64)));
      if (TSTATE) z *= tstate_scale_warp(st64, k33, a.nu_int, a.nu_state);
      zz[e] = z;
    }
    *reinterpret_cast<float4*>(sh.z + 4 * g) = make_float4(zz[0], zz[1], zz[2], zz[3]);
  }
}

// Exclusive prefix of the tile's four-slot chunk masses within the tile (chunkP), by warps
// 16..31, two chunks a thread; it is needed only when the tick resamples, and runs beside the
// forming of the resampling plan.
__device__ __forceinline__ void chunk_scan(FusedShared& sh) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int t2 = tid - kSmallThreads / 2;
  const unsigned long long e0 = sh.chunkE[2 * t2], e1 = sh.chunkE[2 * t2 + 1];
  const unsigned long long s2 = e0 + e1;
  const unsigned long long inc = warp_incl_scan_add(s2, lane);
  if (lane == 31) sh.scan2[warp - 16] = inc;
  asm volatile("bar.sync 2, %0;" ::"n"(kSmallThreads / 2) : "memory");
  const unsigned long long off = warp_sum_u64((lane < warp - 16) ? sh.scan2[lane] : 0ull);
  const unsigned long long ex = off + inc - s2;
  sh.chunkP[2 * t2] = ex;
  sh.chunkP[2 * t2 + 1] = ex + e0;
}

// The FP64 sums of a fused tick over all tiles' records, for NCTA <= kSmallTiles tiles, by one
// thread: the operations of plan_body on one warp in the same order. There lane k holds tile k's
// FP64 sums and the lanes past the tiles exact zeros, so lane 0's butterfly sum is the pairwise
// tree below: v_i + v_{i+8}, then i + 4, i + 2, i + 1, each lane's value first normalised by
// adding lane i + 16's zero (every lane holds the same totals). nM: the tick's global exponent.
template <int NCTA>
__device__ __forceinline__ void fused_sums(const FusedShared& sh, int par, int nM, double& tS, double& tQ,
                                           double& tH) {
  static_assert(NCTA >= 1 && NCTA <= 16, "the tree below covers sixteen lanes");
  // lane k's sums: its running frame is its own tile's, then the global frame 2^nM; each is
  // normalised by the butterfly's first addition of a zero lane (v + 0 turns -0 into +0)
  auto lane_sums = [&](int k, double& S, double& Q, double& H) {
    S = Q = H = 0.0;
    const float4 r = sh.peer[k]->rec[par];
    const int nk = __float_as_int(r.w);
    if (nk != kNkEmpty) {
      const double sc = pow2d(nk - nM);
      S = __dmul_rn(__dadd_rn(0.0, (double)r.x), sc);
      Q = __dmul_rn(__dadd_rn(0.0, (double)r.y), __dmul_rn(sc, sc));
      H = __dmul_rn(__dadd_rn(0.0, (double)r.z), sc);
    }
    S = __dadd_rn(S, 0.0); Q = __dadd_rn(Q, 0.0); H = __dadd_rn(H, 0.0);
  };
  // The tree pruned where a subtree holds only zero lanes: x + (+0) is x once x has been
  // normalised, so only the live lanes' additions remain and the result is the full
  // butterfly's bit for bit. Level 8 is formed as the lanes are read.
  double bS[8], bQ[8], bH[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    bS[i] = bQ[i] = bH[i] = 0.0;
    if (i < NCTA) {
      lane_sums(i, bS[i], bQ[i], bH[i]);
      if (i + 8 < NCTA) {
        double s1, q1, h1;
        lane_sums(i + 8, s1, q1, h1);
        bS[i] = __dadd_rn(bS[i], s1); bQ[i] = __dadd_rn(bQ[i], q1); bH[i] = __dadd_rn(bH[i], h1);
      }
    }
  }
  auto tree = [](double* v) {                    // levels 4, 2, 1 into v[0]
#pragma unroll
    for (int w = 4; w >= 1; w >>= 1)
#pragma unroll
      for (int i = 0; i < w; ++i)
        if (i + w < NCTA) v[i] = __dadd_rn(v[i], v[i + w]);
    return v[0];
  };
  tS = tree(bS); tQ = tree(bQ); tH = tree(bH);
}

template <int NCTA>
__device__ __forceinline__ int fused_nM(const FusedShared& sh, int par) {
  int nM = kNkEmpty;
#pragma unroll
  for (int k = 0; k < NCTA; ++k) nM = max(nM, sh.peer[k]->nexp[par]);
  return nM;
}

// The plan of a fused tick by warp 0: the statistics (for more than two tiles lane k reads tile k's
// record and the warp's butterfly forms the sums, which is the tree of fused_sums), then lane 0
// takes the decision, writes the record and the next tick's state.
template <int NCTA>
__device__ __forceinline__ void plan_fused(const TickArgs& a, int N, FusedShared& sh, int par, BpfTickRecord* rec_out) {
  const int lane = threadIdx.x & 31;
  int nM;
  double tS, tQ, tH;
  if constexpr (NCTA <= 2) {
    nM = fused_nM<NCTA>(sh, par);
    fused_sums<NCTA>(sh, par, nM, tS, tQ, tH);
  } else {
    float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
    int nk = kNkEmpty;
    if (lane < NCTA) { r = sh.peer[lane]->rec[par]; nk = __float_as_int(r.w); }
    nM = warp_max_i(nk);
    double S = 0.0, Q = 0.0, H = 0.0;
    if (nk != kNkEmpty) {
      const double sc = pow2d(nk - nM);
      S = __dmul_rn(__dadd_rn(0.0, (double)r.x), sc);
      Q = __dmul_rn(__dadd_rn(0.0, (double)r.y), __dmul_rn(sc, sc));
      H = __dmul_rn(__dadd_rn(0.0, (double)r.z), sc);
    }
    tS = warp_sum_d(S); tQ = warp_sum_d(Q); tH = warp_sum_d(H);
  }
  if (lane != 0) return;
  DevState* st = &sh.st;
  const bool degenerate = (nM == kNkEmpty) || !(tS > 0.0);
  constexpr double kLn2d = 0.693147180559945309417232121458;
  double res[4] = {0.0, 0.0, 0.0, 0.0};
  if (!degenerate) {
    const double L = log(tS);
    res[0] = __fma_rn((double)nM, kLn2d, L);
    res[1] = tS * tS / tQ;
    res[2] = tH / tS;
    res[3] = L;
  }
  plan_decide(a, st, N, nM, degenerate, res, tS, rec_out);
}

// The same plan in two parts, for ticks whose next tick should not wait for the record: the
// decision (plan_fused_decide, warp 0) computes the statistics as plan_fused and writes the
// device-state fields that the next tick's pass 1 and the resampling read: plan_decide's
// operations on them, in its order; the finish (plan_fused_finish, lane 0 of warp 0, later in
// the tick) computes the log-likelihood increment and the filtered mean and writes the record, the
// running sums and, when the tick keeps its particles, the log of its weight sum, from the values
// the decision left in sh.tail. The two parts together write what plan_decide writes, with the
// same arithmetic.
template <int NCTA>
__device__ __forceinline__ void plan_fused_decide(const TickArgs& a, int N, FusedShared& sh, int par) {
  const int lane = threadIdx.x & 31;
  int nM;
  double tS, tQ, tH;
  if constexpr (NCTA <= 2) {
    nM = fused_nM<NCTA>(sh, par);
    fused_sums<NCTA>(sh, par, nM, tS, tQ, tH);
  } else {
    float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
    int nk = kNkEmpty;
    if (lane < NCTA) { r = sh.peer[lane]->rec[par]; nk = __float_as_int(r.w); }
    nM = warp_max_i(nk);
    double S = 0.0, Q = 0.0, H = 0.0;
    if (nk != kNkEmpty) {
      const double sc = pow2d(nk - nM);
      S = __dmul_rn(__dadd_rn(0.0, (double)r.x), sc);
      Q = __dmul_rn(__dadd_rn(0.0, (double)r.y), __dmul_rn(sc, sc));
      H = __dmul_rn(__dadd_rn(0.0, (double)r.z), sc);
    }
    tS = warp_sum_d(S); tQ = warp_sum_d(Q); tH = warp_sum_d(H);
  }
  if (lane != 0) return;
  DevState* st = &sh.st;
  FusedTail& tl = sh.tail;
  const bool degenerate = (nM == kNkEmpty) || !(tS > 0.0);
  double ess = 0.0;
  int resample = 0;
  if (!degenerate) {
    ess = tS * tS / tQ;
    resample = (a.ess_threshold <= 0.0f) || (ess / (double)N < (double)a.ess_threshold);
  }
  tl.tS = tS; tl.tH = tH; tl.ess = ess; tl.nM = nM;
  tl.degenerate = degenerate ? 1 : 0; tl.resample = resample;
  tl.logS_prev_old = st->logS_prev; tl.resampled_prev_old = st->resampled_prev; tl.tick_old = st->tick;
  const int cur = st->cur;
  if (degenerate) st->error = BPF_ERR_DEGENERATE;
  {
    const int d1 = st->dirs & 1;
    st->dirs = (resample ? d1 : (d1 ^ 1)) | ((d1 ^ 1) << 1);
  }
  st->k1 = st->k1 * kPcgMult;
  st->k2 = st->k2 * kPcgMult + 1ull;
  st->tick = tl.tick_old + 1;
  st->do_resample = resample;
  st->nM = nM;
  if (resample) {
    const uint64_t old = st->u_state;
    st->u_state = old * kPcgMult + kHostInc;
    st->u23 = pcg_output(old) >> 9;
    st->logS_prev = a.log_n;
    st->resampled_prev = 1;
    st->resample_count += 1;
    st->src = cur;
    st->cur = cur ^ 1;
  } else if (degenerate) {
    st->logS_prev = a.log_n;
    st->resampled_prev = 1;
  } else {
    st->resampled_prev = 0;
    st->nM_prev = nM;
  }
}

__device__ __forceinline__ void plan_fused_finish(const FusedShared& sh_in, DevState* st, BpfTickRecord* rec_out) {
  const FusedTail& tl = sh_in.tail;
  constexpr double kLn2d = 0.693147180559945309417232121458;
  double dll = -INFINITY, hm = __longlong_as_double(0x7FF8000000000000LL), L = 0.0;
  if (!tl.degenerate) {
    L = log(tl.tS);
    dll = __fma_rn((double)tl.nM, kLn2d, L) - tl.logS_prev_old;
    hm = tl.tH / tl.tS;
  }
  const double ll_ref = (tl.resampled_prev_old ? 0.0 : st->ll_ref) + dll;
  st->ll_ref = ll_ref;
  st->hm = tl.degenerate ? 0.0 : hm;
  st->ll_total += dll;
  if (rec_out) {
    BpfTickRecord r;
    r.dloglik = dll; r.loglik_ref = ll_ref; r.loglik_total = st->ll_total;
    r.h_mean = (float)hm; r.ess = (float)tl.ess; r.resampled = tl.resample; r.tick = tl.tick_old;
    *rec_out = r;
  }
  if (!tl.resample && !tl.degenerate) st->logS_prev = L;
}

// The resampling plan into the device state (on a resampling tick).
__device__ __forceinline__ void store_fused_plan(DevState* st, const FusedShared& sh) {
  const FusedPlan& pl = sh.pl;
  if (pl.zero_spacing) st->error = BPF_ERR_DEGENERATE;
  st->base = pl.base; st->delta = pl.delta; st->delta_magic = pl.magic; st->total = pl.total;
  st->Fg = pl.Fg; st->n_items = pl.items;
}

// The tick's resampling plan by warp 1, lane k for tile k (NCTA <= 32): the fixed-point CDF over
// the tiles (an exact u64 scan), the target spacing, base and reciprocal and the item count, as
// plan_body; lane 0 writes the plan and, when the tick resamples, its fields of the device state.
// u_state: the resampling-uniform state at the start of the tick. ahead (threshold 0, the plan runs
// beside the decision): whether the tick resamples is found here too, as the plan's decision would,
// not degenerate: its FP64 weight sum is a sum of the tiles' non-negative terms, positive exactly
// when no term is NaN and one is positive. Returns whether the plan is stored.
template <int NCTA>
__device__ __forceinline__ bool plan_fused_targets(int N, double rcpN, FusedShared& sh, int par,
                                                   unsigned long long u_state, bool ahead) {
  static_assert(NCTA <= 32, "one lane per tile");
  const int lane = threadIdx.x & 31;
  int nk = kNkEmpty;
  unsigned long long E = 0ull;
  float S = 0.0f;
  if (lane < NCTA) {
    const FusedShared* pk = sh.peer[lane];
    nk = pk->nexp[par];
    E = pk->E[par];
    S = pk->rec[par].x;
  }
  const int nM = warp_max_i(nk);
  const int Fg = min(kFixF, 62 - ceil_log2_u((unsigned)N));
  const unsigned long long mass = (nk != kNkEmpty) ? shr64(E, nM - nk + kFixF - Fg) : 0ull;
  const unsigned long long incl = warp_incl_scan_add(mass, lane);
  const unsigned long long excl = incl - mass;
  const unsigned long long total = __shfl_sync(0xffffffffu, incl, 31);
  unsigned long long delta = udiv_fp64_rcp(total, (unsigned long long)N, rcpN);
  const bool zero_spacing = delta == 0ull;
  if (zero_spacing) delta = 1ull;
  const unsigned long long u = pcg_output(u_state) >> 9;       // the tick's resampling uniform
  const unsigned long long hi = __umul64hi(u, delta), lo = u * delta;
  const unsigned long long base = (hi << 41) | (lo >> 23);     // floor(u * delta / 2^23)
  const unsigned long long magic = udiv_magic_of(delta);
  int ni = 0;
  if (lane < NCTA) {
    const int o = targets_below(excl, base, delta, magic, N), o_next = targets_below(incl, base, delta, magic, N);
    ni = (o_next - o + kOutChunk - 1) / kOutChunk;
    sh.P[lane] = excl;
  }
  const int n_items = __reduce_add_sync(0xffffffffu, ni);
  bool live = true;
  if (ahead) {
    double term = 0.0;
    if (nk != kNkEmpty) term = __dmul_rn((double)S, pow2d(nk - nM));
    live = (nM != kNkEmpty) && !__any_sync(0xffffffffu, term != term) && __any_sync(0xffffffffu, term > 0.0);
  }
  if (lane == 0) {
    FusedPlan& pl = sh.pl;
    pl.base = base; pl.delta = delta; pl.magic = magic; pl.total = total;
    pl.nM = nM; pl.Fg = Fg; pl.items = n_items; pl.zero_spacing = zero_spacing ? 1 : 0;
    pl.live = live ? 1 : 0;
    if (live) store_fused_plan(&sh.st, sh);
  }
  return live;
}

// A chunk of CH consecutive slots of the tile (slots CH c .. CH c + CH - 1) against the tick's
// targets: its weights, their FP32 sum in order, its first target and tile-frame thresholds
// (th = kThCap: no target is reachable from the chunk).
template <int CH>
struct ChunkTargets {
  float wf[CH];
  float lfT;
  unsigned long long th, D;
  int q, c;
};

template <int NCTA, int CH>
__device__ __forceinline__ ChunkTargets<CH> chunk_targets(int N, int k, int par, int c, const FusedShared& sh) {
  static_assert(CH % 4 == 0, "whole four-slot chunks");
  const FusedPlan& pl = sh.pl;
  const int nk = sh.nexp[par];
  const int r = (nk == kNkEmpty) ? 64 : pl.nM - nk + kFixF - pl.Fg;
  const unsigned long long Pk = sh.P[k], base = pl.base, delta = pl.delta;
  const int l0 = CH * c, j0 = k * kTile + l0;
  ChunkTargets<CH> ct;
  ct.c = c;
  ct.lfT = 0.0f;
#pragma unroll
  for (int v = 0; v < CH / 4; ++v) {
    const float4 w4 = *reinterpret_cast<const float4*>(sh.w + l0 + 4 * v);
    ct.wf[4 * v] = tile_weight(w4.x); ct.wf[4 * v + 1] = tile_weight(w4.y);
    ct.wf[4 * v + 2] = tile_weight(w4.z); ct.wf[4 * v + 3] = tile_weight(w4.w);
  }
#pragma unroll
  for (int e = 0; e < CH; ++e) ct.lfT += ct.wf[e];
  const unsigned long long loc = sh.chunkP[l0 / 4];   // exclusive prefix of its first four-slot chunk
  // child counts against tile-frame thresholds, as pass 2
  ct.q = targets_below(Pk + shr64(loc, r), base, delta, pl.magic, N);
  ct.th = kThCap; ct.D = kThCap;
  if (r < 64 && ct.q < N && j0 < N) {
    const unsigned long long m = base + (unsigned long long)ct.q * delta - Pk + 1ull;
    if (m <= (~0ull >> r)) ct.th = min((m << r) - loc, kThCap);
    if (delta <= (kThCap >> r)) ct.D = delta << r;
  }
  return ct;
}

// Resampling of a fused tick, this CTA's part: every parent of its tile writes its particle into
// the output slots of its children, in the particle buffer of the CTA that owns each slot
// (distributed shared memory), then one barrier over the cluster ends the tick's resampling.
// The children of the chunk's elements as in pass 2: the running count c_j = #{m >= 0 :
// th + m D <= l_j} (l_j the exact fixed-point sum of the chunk's weights up to j) estimated in
// FP32 from the running sum of the weights, with pass 2's bound on the estimate's error taken at
// the chunk's largest sum; near a target boundary (one vote per four elements) the element
// recounts in exact 64-bit integers. The output slots of element j are [q_{j-1}, q_j),
// q_j = min(q + c_j, N). A chunk from which no target is reachable (th = kThCap) has no children.
// src / dst: the particle buffers the resampling reads and writes.
template <int NCTA, int CH>
__device__ __forceinline__ void count_write(const TickArgs& a, int N, int k, const ChunkTargets<CH>& ct, int src,
                                            int dst, FusedShared& sh) {
  const int j0 = k * kTile + CH * ct.c;
  const float* d = sh.w + CH * ct.c;               // its log2-weights, for the exact recount
  const float* hs = sh.h[src] + CH * ct.c;         // its particles
  const unsigned long long R0 = ct.th, D = ct.D;
  const bool none = R0 >= kThCap;
  const float R0w = (float)R0 * 0x1p-50f;
  const float invDw = 1.0f / ((float)D * 0x1p-50f);
  const float R0x = R0w * invDw;
  const float eL = 0x1p-18f * invDw, e0 = fmaf(R0w, eL, 0x1p-44f * invDw);
  const float xT = fmaf(ct.lfT, invDw, -R0x);
  float err = fmaf(ct.lfT, eL, fmaf(fmaxf(fabsf(xT), R0x), 0x1p-21f, e0));
  if (!(xT < 0x1p22f)) err = 1.0f;
  const float err_hi = 1.0f - err;
  const int q0 = ct.q, Kq = 0x4AFFFFFF - q0;
  float lf = 0.0f;
  int qe[CH];                                      // q_j: the end of element j's children
#pragma unroll
  for (int g = 0; g < CH / 4; ++g) {
    int qq[4];
    bool rc[4], any = false;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      lf += ct.wf[4 * g + e];
      const float x = fmaf(lf, invDw, -R0x);
      const float fl = floorf(x);
      const float fr = x - fl;                       // exact
      rc[e] = !none && !(fr > err && fr < err_hi);
      any |= rc[e];
      qq[e] = none ? q0 : min(max(__float_as_int(fl + 0x1p23f) - Kq, q0), N);
    }
    if (__any_sync(0xffffffffu, any)) {
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (rc[e]) qq[e] = min(q0 + exact_count(d, 4 * g + e, R0, D, N), N);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) qe[4 * g + e] = qq[e];
  }
  // The chunk's children fill the slots [q0, q_last): slot o belongs to element #{j : q_j <= o}.
  // Each lane writes its run in one loop, starting at an offset rotated by lane / 4: the runs of
  // a warp's lanes start about eight slots apart, so without the rotation eight lanes would store
  // to the same bank at every step.
  const int n_run = qe[CH - 1] - q0;
  if (n_run > 0) {
    int p = (int)(threadIdx.x & 31) >> 2;
    while (p >= n_run) p -= n_run;
    for (int m = 0; m < n_run; ++m) {
      const int o = q0 + p;
      int e = 0;
#pragma unroll
      for (int j = 0; j < CH - 1; ++j) e += (qe[j] <= o) ? 1 : 0;
      const float hv = hs[e];
      if constexpr (NCTA == 1) sh.h[dst][o] = hv;
      else sh.peer[o >> 12]->h[dst][o & (kTile - 1)] = hv;
      if (a.anc) a.anc[o] = j0 + e;
      if (++p == n_run) p = 0;
    }
  }
}

// The barrier that ends a resampling (every child written) when warp 0 is taking the tick's
// decision meanwhile: warp 0 arrives before it starts (it writes no children) and waits after
// it, the other warps arrive and wait together. Barrier 4 for one CTA, the cluster's otherwise.
template <int NCTA>
__device__ __forceinline__ void marks_barrier_arrive() {
  if constexpr (NCTA == 1) asm volatile("bar.arrive 4, %0;" ::"n"(kSmallThreads) : "memory");
  else asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
template <int NCTA>
__device__ __forceinline__ void marks_barrier_wait() {
  if constexpr (NCTA > 1) asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
template <int NCTA>
__device__ __forceinline__ void marks_barrier_sync() {
  if constexpr (NCTA == 1) asm volatile("bar.sync 4, %0;" ::"n"(kSmallThreads) : "memory");
  else cluster_sync_all<NCTA>();
}

template <bool TSTATE, bool GAUSS, int NCTA>
__global__ void __cluster_dims__(NCTA, 1, 1) __launch_bounds__(kSmallThreads, 1)
small_kernel(Plan p, TickArgs a, int n_ticks) {
  extern __shared__ __align__(16) unsigned char small_smem[];
  FusedShared& sh = *reinterpret_cast<FusedShared*>(small_smem);
  const int tid = threadIdx.x;
  int k = 0;
  if constexpr (NCTA > 1) k = (int)cooperative_groups::this_cluster().block_rank();
  const int N = p.N, tile0 = k * kTile;
  griddep_wait();
  if (tid < kStWords)
    reinterpret_cast<unsigned long long*>(&sh.st)[tid] = __ldcg(reinterpret_cast<const unsigned long long*>(p.st) + tid);
  if (tid < NCTA) {
    if constexpr (NCTA > 1) sh.peer[tid] = cooperative_groups::this_cluster().map_shared_rank(&sh, tid);
    else sh.peer[tid] = &sh;
  }
  // A cluster may hold more CTAs than the filter has tiles (5..8 tiles run as 8, 9..16 as 16): a
  // CTA past the last tile holds only padding slots (weight 0, finite particles) and no outputs.
  const bool real = k < p.G;
  if (real) {
    if (tid == 0) sh.nexp[1] = __ldcg(p.nexp + k);    // the exponent the first tick's carry reads
    reinterpret_cast<float4*>(sh.h[0])[tid] = __ldcg(reinterpret_cast<const float4*>(p.h0 + tile0) + tid);
    reinterpret_cast<float4*>(sh.h[1])[tid] = __ldcg(reinterpret_cast<const float4*>(p.h1 + tile0) + tid);
    reinterpret_cast<float4*>(sh.w)[tid] = __ldcg(reinterpret_cast<const float4*>(p.w + tile0) + tid);
  } else {
    if (tid == 0) sh.nexp[1] = kNkEmpty;
    reinterpret_cast<float4*>(sh.h[0])[tid] = make_float4(0.f, 0.f, 0.f, 0.f);
    reinterpret_cast<float4*>(sh.h[1])[tid] = make_float4(0.f, 0.f, 0.f, 0.f);
    reinterpret_cast<float4*>(sh.w)[tid] = make_float4(0.f, 0.f, 0.f, 0.f);
  }

  const double rcpN = 1.0 / (double)N;           // exact division by N: the quotient is corrected
  const bool ahead = a.ess_threshold <= 0.0f;     // every tick that can resample does
  const int warp = tid >> 5;
  __syncthreads();                                // the device state is in shared memory
  if (sh.st.tick > 0) fused_noise<TSTATE>(a, tile0, sh.st.k1, sh.st.k2, 0, kSmallThreads, sh);   // the first tick's
  for (int t = 0; t < n_ticks; ++t) {
    const int par = t & 1;
    if (a.y_ptr && (t & (kYStage - 1)) == 0) {       // the next kYStage observations
      __syncthreads();
      if (t + tid < n_ticks) sh.ys[tid] = __ldg(a.y_ptr + t + tid);
      __syncthreads();
    } else if (ahead || t == 0) {
      // With a threshold the decision barrier (and on resampling ticks the barrier after the
      // children's writes) already orders everything this tick's pass 1 reads: the particles, the
      // noise and the device-state fields the decision wrote; the finish of the previous tick's
      // plan (warp 31, outside pass 1) writes only the record and fields pass 1 does not read, and
      // the next decision reads them after the records barrier, which warp 31 reaches after the
      // finish. When every tick resamples, warp 0 did not wait for the children.
      __syncthreads();
    }
    const float y = a.y_ptr ? sh.ys[t & (kYStage - 1)] : a.obs.y;
    const unsigned long long u_state = sh.st.u_state;
    const int cur0 = sh.st.cur;                    // a resampling reads buffer cur0, writes cur0 ^ 1
    const bool more = t + 1 < n_ticks;             // the launch runs another tick: form its noise
    if (tid == 0) { sh.knext[0] = sh.st.k1 * kPcgMult; sh.knext[1] = sh.st.k2 * kPcgMult + 1ull; }
    pass1_fused<TSTATE, GAUSS, kSmallSplit>(a, y, N, tile0, par, sh.nexp[par ^ 1], sh);
    cluster_sync_all<NCTA>();                   // every tile record of the tick is in place
    if (ahead) {
      // The resampling needs nothing from the decision but whether the tick is degenerate, so
      // warp 0 takes the decision and writes the record beside it: warp 1 forms the plan (and
      // the plan's fields of the device state, which the decision does not touch), warps 16..31
      // count the children of eight-slot chunks and write them.
      if (warp == 0) {
        marks_barrier_arrive<NCTA>();
        plan_fused<NCTA>(a, N, sh, par, (a.rec && k == 0) ? a.rec + t : nullptr);
        __syncwarp();
        marks_barrier_wait<NCTA>();
      } else {
        if (warp == 1) plan_fused_targets<NCTA>(N, rcpN, sh, par, u_state, true);
        else if (warp >= 16) chunk_scan(sh);
        else if (more) fused_noise<TSTATE>(a, tile0, sh.knext[0], sh.knext[1], 64, 14 * 32, sh);   // warps 2..15
        if (warp == 1 || warp >= 16) {             // the plan's producer and its users meet; warps 2..15 do not wait
          asm volatile("bar.sync 3, %0;" ::"n"(32 + kSmallThreads / 2) : "memory");
          if (sh.pl.live && warp >= 16) {
            const ChunkTargets<8> ct = chunk_targets<NCTA, 8>(N, k, par, tid - kSmallThreads / 2, sh);
            count_write<NCTA, 8>(a, N, k, ct, cur0, cur0 ^ 1, sh);
          }
        }
        marks_barrier_sync<NCTA>();               // every child is written
      }
    } else {
      if (warp == 0) plan_fused_decide<NCTA>(a, N, sh, par);
      else if (more) fused_noise<TSTATE>(a, tile0, sh.knext[0], sh.knext[1], 32, kSmallThreads - 32, sh);
      __syncthreads();
      if (sh.st.do_resample) {
        if (warp == 1) plan_fused_targets<NCTA>(N, rcpN, sh, par, u_state, false);
        else if (warp >= 16) chunk_scan(sh);
        __syncthreads();
        const ChunkTargets<4> ct = chunk_targets<NCTA, 4>(N, k, par, tid, sh);
        count_write<NCTA, 4>(a, N, k, ct, cur0, cur0 ^ 1, sh);
        cluster_sync_all<NCTA>();                 // every child is written
      }
      // the tick's record and running sums, on a warp outside pass 1, while the others start the
      // next tick
      if (tid == kSmallThreads - 32) plan_fused_finish(sh, &sh.st, (a.rec && k == 0) ? a.rec + t : nullptr);
    }
  }
  if (tid == 0 && a.mirror) sh.st.seq = a.seq;
  cluster_sync_all<NCTA>();                     // no CTA leaves while another may read its shared memory
  if (real) {
    reinterpret_cast<float4*>(p.h0 + tile0)[tid] = reinterpret_cast<const float4*>(sh.h[0])[tid];
    reinterpret_cast<float4*>(p.h1 + tile0)[tid] = reinterpret_cast<const float4*>(sh.h[1])[tid];
    reinterpret_cast<float4*>(p.w + tile0)[tid] = reinterpret_cast<const float4*>(sh.w)[tid];
  }
  if (real && tid == 0) {
    const int last = (n_ticks - 1) & 1;
    p.nexp[k] = sh.nexp[last];
    p.E[k] = sh.E[last];
    p.rec[k] = sh.rec[last];
  }
  if (k == 0) {
    if (tid < kStWords)
      reinterpret_cast<unsigned long long*>(p.st)[tid] = reinterpret_cast<const unsigned long long*>(&sh.st)[tid];
    if (tid == 0 && a.mirror) {
      __threadfence_system();                 // the record first, then the mirror naming its request
      TickMirror mm;
      mm.resample_count = sh.st.resample_count; mm.tick = sh.st.tick; mm.error = sh.st.error; mm.seq = a.seq;
      *a.mirror = mm;
    }
  }
  griddep_release();
}

// ---------------------------------------------------------------------------
// Debug probe: raw PCG32 output and the derived normal for draw t
// ---------------------------------------------------------------------------
__global__ void debug_pcg_kernel(int seed, int n, unsigned long long At, unsigned long long Bt,
                                 uint32_t* out, float* norm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const PcgTick c = pcg_tick_consts(seed, At, Bt);
  const uint32_t o = pcg_output(c.k1 + c.k2 * pcg_inc((uint32_t)i));
  if (out) out[i] = o;
  if (norm) norm[i] = icdf_normal(pcg_uniform(o));
}

// Linear tile-relative weights 2^d of the stored log2-weights (inspection API).
__global__ void tile_weights_kernel(const float* d, float* w, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) w[i] = tile_weight(d[i]);
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
template <typename... KArgs, typename... Args>
static cudaError_t launch_ex(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                             bool pdl, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = pdl ? attr : nullptr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, args...);
}

cudaError_t plan_alloc(Plan& p, int N) {
  p.N = N;
  p.G = (N + kTile - 1) / kTile;
  p.max_items = p.G + (N + kOutChunk - 1) / kOutChunk + 1;
  const size_t npad = (size_t)p.G * kTile;
  cudaError_t e = cudaSuccess;
  auto al = [&](auto** ptr, size_t bytes) { if (e == cudaSuccess) e = bpf_malloc(ptr, bytes); };
  al(&p.h0, npad * sizeof(float));
  al(&p.h1, npad * sizeof(float));
  al(&p.w, npad * sizeof(float));
  al(&p.nexp, p.G * sizeof(int));
  al(&p.E, p.G * sizeof(unsigned long long));
  al(&p.rec, p.G * sizeof(float4));
  al(&p.rec2, p.G * sizeof(float4));
  al(&p.P, p.G * sizeof(unsigned long long));
  al(&p.ofirst, (p.G + 1) * sizeof(int));
  al(&p.items, p.max_items * sizeof(int4));
  al(&p.jpart, p.G * sizeof(double));
  al(&p.jticket, sizeof(unsigned));
  al(&p.pticket, sizeof(unsigned));
  al(&p.st, sizeof(DevState));
  if (e == cudaSuccess) e = cudaMemset(p.nexp, 0, p.G * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(p.jticket, 0, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(p.pticket, 0, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaDeviceSynchronize();   // visible to every stream before first use
  return e;
}

void plan_free(Plan& p) {
  bpf_free(p.h0); bpf_free(p.h1); bpf_free(p.w);
  bpf_free(p.nexp); bpf_free(p.E); bpf_free(p.rec); bpf_free(p.rec2);
  bpf_free(p.P); bpf_free(p.ofirst); bpf_free(p.items); bpf_free(p.st);
  bpf_free(p.jpart); bpf_free(p.jticket); bpf_free(p.pticket);
  p = Plan{};
}

cudaError_t launch_init(const Plan& p, float mu, float std_stat, int seed, cudaStream_t s) {
  const int n = p.G * kTile;
  init_kernel<<<(n + 255) / 256, 256, 0, s>>>(p, mu, std_stat, seed);
  return cudaGetLastError();
}

size_t pass2_smem_bytes() { return kPass2Smem; }

constexpr int kMaxConfiguredDevices = 64;

template <int NCTA>
static void configure_small() {
  constexpr int bytes = (int)sizeof(FusedShared);
  void (*k[4])(Plan, TickArgs, int) = {small_kernel<false, true, NCTA>, small_kernel<true, true, NCTA>,
                                       small_kernel<false, false, NCTA>, small_kernel<true, false, NCTA>};
  for (auto f : k) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (NCTA > 8) cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  }
}

// Largest fused cluster (in tiles) the device schedules: 16 when a cluster of sixteen 1024-thread
// CTAs with the fused kernel's shared memory fits on one GPC, else 8 (the portable size).
static int small_tiles_on_device() {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(16);
  cfg.blockDim = dim3(kSmallThreads);
  cfg.dynamicSmemBytes = sizeof(FusedShared);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 16; attr[0].val.clusterDim.y = 1; attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, small_kernel<false, true, 16>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  return n >= 1 ? 16 : 8;
}
static int g_small_tiles[kMaxConfiguredDevices] = {};

// Called with `device` current. The shared-memory attributes are set once per
// device (they belong to the device's context), under a lock so filters
// created from several threads do not race.
static std::mutex g_config_lock;

int pass2_grid_size(int device) {
  static bool configured[kMaxConfiguredDevices] = {};
  {
    std::lock_guard<std::mutex> guard(g_config_lock);
    if (device < 0 || device >= kMaxConfiguredDevices || !configured[device]) {
      cudaFuncSetAttribute(pass2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPass2Smem);
      cudaFuncSetAttribute(plan_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)plan_smem_bytes(kPlanSmemTiles));
      configure_small<1>();
      configure_small<2>();
      configure_small<3>();
      configure_small<4>();
      configure_small<8>();
      configure_small<16>();
      if (device >= 0 && device < kMaxConfiguredDevices) g_small_tiles[device] = small_tiles_on_device();
      if (device >= 0 && device < kMaxConfiguredDevices) configured[device] = true;
    }
  }
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pass2_kernel, kThreads, kPass2Smem);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

template <bool GAUSS>
static cudaError_t launch_pass1_model(const Plan& p, const TickArgs& a, cudaStream_t s, bool pdl) {
  const dim3 grid(p.G), block(kThreads);
  if (a.apf == 1) return launch_ex(pass1_kernel<false, false, 1, GAUSS, false>, grid, block, 0, s, pdl, p, a);
  if (a.apf == 2) {
    if (a.nu_int > 0) return launch_ex(pass1_kernel<true, false, 2, GAUSS, false>, grid, block, 0, s, pdl, p, a);
    return launch_ex(pass1_kernel<false, false, 2, GAUSS, false>, grid, block, 0, s, pdl, p, a);
  }
  if (a.learn && p.rec2) {
    if (a.nu_int > 0) return launch_ex(pass1_kernel<true, true, 0, GAUSS, false>, grid, block, 0, s, pdl, p, a);
    return launch_ex(pass1_kernel<false, true, 0, GAUSS, false>, grid, block, 0, s, pdl, p, a);
  }
  if (a.tail_plan) {
    if (!tail_plan_eligible(p, a)) return cudaErrorInvalidValue;
    if (a.nu_int > 0) return launch_ex(pass1_kernel<true, false, 0, GAUSS, true>, grid, block, 0, s, pdl, p, a);
    return launch_ex(pass1_kernel<false, false, 0, GAUSS, true>, grid, block, 0, s, pdl, p, a);
  }
  if (a.nu_int > 0) return launch_ex(pass1_kernel<true, false, 0, GAUSS, false>, grid, block, 0, s, pdl, p, a);
  return launch_ex(pass1_kernel<false, false, 0, GAUSS, false>, grid, block, 0, s, pdl, p, a);
}

bool tail_plan_eligible(const Plan& p, const TickArgs& a) {
  return p.G <= kTailTiles && p.pticket && a.apf == 0 && !a.learn && !a.ckpt && !a.csr && !a.aux;
}

cudaError_t launch_pass1(const Plan& p, const TickArgs& a, cudaStream_t s, bool pdl) {
  return (a.obs.nu > 0.0f) ? launch_pass1_model<false>(p, a, s, pdl) : launch_pass1_model<true>(p, a, s, pdl);
}
cudaError_t launch_plan(const Plan& p, const TickArgs& a, cudaStream_t s, bool pdl) {
  return launch_ex(plan_kernel, dim3(1), dim3(kPlanThreads), plan_smem_bytes(p.G), s, pdl, p, a);
}
cudaError_t launch_pass2(const Plan& p, const TickArgs& a, int grid, cudaStream_t s, bool pdl) {
  return launch_ex(pass2_kernel, dim3(grid), dim3(kThreads), kPass2Smem, s, pdl, p, a);
}

bool small_eligible(const Plan& p, const TickArgs& a) {
  return p.N <= kSmallMaxN && !a.learn && a.apf == 0 && !(a.silverman > 0.0f) && !a.ckpt && !a.csr && !a.aux;
}

template <int NCTA>
static cudaError_t launch_small_cluster(const Plan& p, const TickArgs& a, int n_ticks, cudaStream_t s, bool pdl) {
  const dim3 grid(NCTA), block(kSmallThreads);
  constexpr size_t bytes = sizeof(FusedShared);
  if (a.obs.nu > 0.0f) {
    if (a.nu_int > 0) return launch_ex(small_kernel<true, false, NCTA>, grid, block, bytes, s, pdl, p, a, n_ticks);
    return launch_ex(small_kernel<false, false, NCTA>, grid, block, bytes, s, pdl, p, a, n_ticks);
  }
  if (a.nu_int > 0) return launch_ex(small_kernel<true, true, NCTA>, grid, block, bytes, s, pdl, p, a, n_ticks);
  return launch_ex(small_kernel<false, true, NCTA>, grid, block, bytes, s, pdl, p, a, n_ticks);
}

cudaError_t launch_small(const Plan& p, const TickArgs& a, int n_ticks, cudaStream_t s, bool pdl) {
  if (p.N > kSmallMaxN || p.G < 1 || p.G > kSmallTiles || n_ticks < 1) return cudaErrorInvalidValue;
  if (p.G <= 4) {
    switch (p.G) {
      case 1: return launch_small_cluster<1>(p, a, n_ticks, s, pdl);
      case 2: return launch_small_cluster<2>(p, a, n_ticks, s, pdl);
      case 3: return launch_small_cluster<3>(p, a, n_ticks, s, pdl);
      default: return launch_small_cluster<4>(p, a, n_ticks, s, pdl);
    }
  }
  if (p.G <= 8) return launch_small_cluster<8>(p, a, n_ticks, s, pdl);
  return launch_small_cluster<16>(p, a, n_ticks, s, pdl);
}

int small_max_tiles(int device) {
  if (device < 0 || device >= kMaxConfiguredDevices) return 4;
  std::lock_guard<std::mutex> guard(g_config_lock);
  return g_small_tiles[device] ? g_small_tiles[device] : 4;
}

cudaError_t launch_jitter(const Plan& p, const TickArgs& a, cudaStream_t s, bool pdl) {
  if (!p.jpart || !p.jticket) return cudaErrorInvalidValue;
  cudaError_t e = launch_ex(jitter_var_kernel, dim3(p.G), dim3(kThreads), 0, s, pdl, p, a.silverman);
  if (e == cudaSuccess) e = launch_ex(jitter_apply_kernel, dim3(p.G), dim3(kThreads), 0, s, pdl, p, a.mu);
  return e;
}

cudaError_t launch_tile_weights(const Plan& p, float* w_out, cudaStream_t s) {
  tile_weights_kernel<<<(p.N + 255) / 256, 256, 0, s>>>(p.w, w_out, p.N);
  return cudaGetLastError();
}

cudaError_t launch_debug_pcg(int seed, int n, int t, uint32_t* d_out, float* d_norm, cudaStream_t s) {
  unsigned long long At = 1ull, Bt = 0ull;
  for (int k = 0; k < t; ++k) { At *= kPcgMult; Bt = Bt * kPcgMult + 1ull; }
  debug_pcg_kernel<<<(n + 255) / 256, 256, 0, s>>>(seed, n, At, Bt, d_out, d_norm);
  return cudaGetLastError();
}

}  // namespace bpf
