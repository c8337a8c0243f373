// bpf_plain.cu — the plain SV bootstrap-filter tick as two sm_100a kernels.
//
//   pass 1  (one CTA per 4096-particle tile)
//           counter-PCG32 -> AS241 normal -> OU propagate -> log-weight
//           (+ carried weight on ESS-skipped ticks), tile max as a power-of-two
//           exponent n_k, tile-relative weights w = 2^(x - n_k) written once,
//           tile partial sums S=sum w, Q=sum w^2, H=sum w h (FP64) and the exact
//           fixed-point tile mass E = sum floor(w 2^50).
//           The last CTA to finish (atomic ticket) combines the tiles in FP64:
//           log-likelihood increment, ESS, filtered mean, the resampling
//           decision, and — on resampling ticks — the fixed-point CDF tile
//           prefixes and the pass-2 work list. No host synchronisation.
//   pass 2  (persistent CTAs over work items)
//           systematic resampling: exact integer prefix of the tile weights,
//           merge-path match of the N evenly spaced targets against the CDF,
//           gather of h[ancestor] through shared memory, coalesced store.
//
// Reference tick this replaces: gpu_bpf/gpu_bpf_ptx_full.cu:550-748 (≈15
// launches, float atomics, a host sync for ESS, thrust scan) with kernels
// ptx_assembly/bpf_kernels_full.ptx:231-842.
#include "bpf_plain.cuh"
#include <cmath>

namespace bpf {

// ---------------------------------------------------------------------------
// Small reduction / scan helpers (256-thread CTAs)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ int warp_max_i(int v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned long long warp_incl_scan_u64(unsigned long long v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned long long n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  return v;
}
__device__ __forceinline__ int warp_incl_scan_i(int v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += n;
  }
  return v;
}

// Exclusive scan over the 256 threads of a CTA; *total receives the sum.
// sh must hold 9 entries. Contains barriers: call from all threads.
__device__ unsigned long long block_excl_scan_u64(unsigned long long v, unsigned long long* total,
                                                  unsigned long long* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned long long inc = warp_incl_scan_u64(v, lane);
  if (lane == 31) sh[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const unsigned long long t = lane < kThreads / 32 ? sh[lane] : 0ull;
    const unsigned long long ti = warp_incl_scan_u64(t, lane);
    __syncwarp();
    if (lane < kThreads / 32) sh[lane] = ti - t;
    if (lane == kThreads / 32 - 1) sh[kThreads / 32] = ti;
  }
  __syncthreads();
  const unsigned long long r = sh[warp] + inc - v;
  *total = sh[kThreads / 32];
  __syncthreads();
  return r;
}
__device__ int block_excl_scan_i(int v, int* total, int* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int inc = warp_incl_scan_i(v, lane);
  if (lane == 31) sh[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const int t = lane < kThreads / 32 ? sh[lane] : 0;
    const int ti = warp_incl_scan_i(t, lane);
    __syncwarp();
    if (lane < kThreads / 32) sh[lane] = ti - t;
    if (lane == kThreads / 32 - 1) sh[kThreads / 32] = ti;
  }
  __syncthreads();
  const int r = sh[warp] + inc - v;
  *total = sh[kThreads / 32];
  __syncthreads();
  return r;
}

// 2^e as a double (exact IEEE encoding; 0 below the normal range).
__device__ __forceinline__ double pow2d(int e) {
  if (e < -1022) return 0.0;
  if (e > 1023) return __longlong_as_double(0x7FF0000000000000LL);
  return __longlong_as_double((long long)(e + 1023) << 52);
}
__device__ __forceinline__ unsigned long long shr64(unsigned long long x, int r) {
  return r >= 64 ? 0ull : (x >> r);
}
__host__ __device__ inline int ceil_log2_u(unsigned n) {
  int c = 0;
  while ((1ull << c) < (unsigned long long)n) ++c;
  return c;
}

// ---------------------------------------------------------------------------
// Init: h_0 = mu + std_stat * z(draw 0)   (bpf_kernels_full.ptx:103-218)
// ---------------------------------------------------------------------------
__global__ void init_kernel(Plan p, float mu, float std_stat, int seed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int npad = p.G * kTile;
  if (i == 0) {
    DevState d{};
    d.At = 1ull; d.Bt = 0ull;                                   // tick 0 uses draw index 0
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

// ---------------------------------------------------------------------------
// Pass-1 epilogue: run by all 256 threads of the last CTA to finish.
// ---------------------------------------------------------------------------
struct EpiShared {
  unsigned long long scan_u[kThreads / 32 + 1];
  int scan_i[kThreads / 32 + 1];
  double red[3][kThreads / 32];
  int red_i[kThreads / 32];
  unsigned long long b_base, b_delta, b_magic, b_total;
  int b_resample, b_nM, b_Fg;
};

__device__ __forceinline__ int first_target_at_or_above(unsigned long long c, unsigned long long base,
                                                        unsigned long long delta, unsigned long long magic,
                                                        int N) {
  // #{ i in [0,N) : base + i*delta < c }
  if (c <= base) return 0;
  const unsigned long long q = udiv_magic(c - base - 1ull, delta, magic) + 1ull;
  return q >= (unsigned long long)N ? N : (int)q;
}

__device__ void pass1_epilogue(const Plan& p, const TickArgs& a, int tick, int cur, EpiShared& sh) {
  DevState* st = p.st;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int G = p.G, N = p.N;

  // 1. global tile exponent
  int nM = kNkEmpty;
  for (int k = tid; k < G; k += kThreads) nM = max(nM, __ldcg(p.nexp + k));
  nM = warp_max_i(nM);
  if (lane == 0) sh.red_i[warp] = nM;
  __syncthreads();
  nM = sh.red_i[0];
#pragma unroll
  for (int w = 1; w < kThreads / 32; ++w) nM = max(nM, sh.red_i[w]);

  // 2. FP64 combine of the tile partials, rescaled to the global frame 2^nM
  double S = 0.0, Q = 0.0, H = 0.0;
  if (nM != kNkEmpty) {
    for (int k = tid; k < G; k += kThreads) {
      const int nk = __ldcg(p.nexp + k);
      if (nk == kNkEmpty) continue;
      const double sc = pow2d(nk - nM);
      S += __ldcg(p.S + k) * sc;
      Q += __ldcg(p.Q + k) * (sc * sc);
      H += __ldcg(p.H + k) * sc;
    }
  }
  S = warp_sum_d(S); Q = warp_sum_d(Q); H = warp_sum_d(H);
  if (lane == 0) { sh.red[0][warp] = S; sh.red[1][warp] = Q; sh.red[2][warp] = H; }
  __syncthreads();

  // 3. tick statistics and the resampling decision (thread 0)
  if (tid == 0) {
    S = 0.0; Q = 0.0; H = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) { S += sh.red[0][w]; Q += sh.red[1][w]; H += sh.red[2][w]; }
    const bool degenerate = (nM == kNkEmpty) || !(S > 0.0);
    const double ln2 = 0.693147180559945309417232121458;
    double dll, ess, hm;
    int resample = 0;
    if (degenerate) {
      dll = -INFINITY; ess = 0.0; hm = nan("");
      st->error = BPF_ERR_DEGENERATE;
    } else {
      const double lse = (double)nM * ln2 + log(S);
      dll = lse - st->logS_prev;
      ess = S * S / Q;
      hm = H / S;
      resample = (a.ess_threshold <= 0.0f) || (ess / (double)N < (double)a.ess_threshold);
    }
    const double ll_ref = (st->resampled_prev ? 0.0 : st->ll_ref) + dll;
    st->ll_ref = ll_ref;
    st->ll_total += dll;
    if (a.rec) {
      BpfTickRecord r;
      r.dloglik = dll; r.loglik_ref = ll_ref; r.loglik_total = st->ll_total;
      r.h_mean = (float)hm; r.ess = (float)ess; r.resampled = resample; r.tick = tick;
      *a.rec = r;
    }
    // next tick's PCG constants
    st->At = st->At * kPcgMult;
    st->Bt = st->Bt * kPcgMult + 1ull;
    st->tick = tick + 1;
    st->do_resample = resample;
    if (resample) {
      const uint64_t old = st->u_state;
      st->u_state = old * kPcgMult + kHostInc;
      st->u23 = pcg_output(old) >> 9;
      st->logS_prev = log((double)N);
      st->resampled_prev = 1;
      st->resample_count += 1;
      st->src = cur;
      st->cur = cur ^ 1;
    } else if (degenerate) {
      st->logS_prev = log((double)N);   // restart from uniform weights
      st->resampled_prev = 1;
    } else {
      st->logS_prev = log(S);
      st->resampled_prev = 0;
      st->nM_prev = nM;
    }
    sh.b_resample = resample;
    sh.b_nM = nM;
    sh.b_Fg = min(kFixF, 62 - ceil_log2_u((unsigned)N));
  }
  __syncthreads();
  if (!sh.b_resample) {
    if (tid == 0) st->ticket = 0u;
    return;
  }

  // 4. fixed-point CDF: tile masses in the global frame, prefix, total
  const int Fg = sh.b_Fg;
  const int C = (G + kThreads - 1) / kThreads;
  const int k0 = min(tid * C, G), k1 = min(k0 + C, G);
  auto ehat = [&](int k) -> unsigned long long {
    const int nk = __ldcg(p.nexp + k);
    if (nk == kNkEmpty) return 0ull;
    return shr64(__ldcg(p.E + k), nM - nk + kFixF - Fg);
  };
  unsigned long long part = 0;
  for (int k = k0; k < k1; ++k) part += ehat(k);
  unsigned long long total;
  const unsigned long long excl = block_excl_scan_u64(part, &total, sh.scan_u);
  if (tid == 0) {
    unsigned long long delta = total / (unsigned long long)N;
    if (delta == 0ull) { delta = 1ull; st->error = BPF_ERR_DEGENERATE; }
    const unsigned long long u = st->u23;
    const unsigned long long hi = __umul64hi(u, delta), lo = u * delta;
    sh.b_base = (hi << 41) | (lo >> 23);          // floor(u * delta / 2^23)
    sh.b_delta = delta;
    sh.b_magic = ~0ull / delta;
    sh.b_total = total;
  }
  __syncthreads();
  const unsigned long long base = sh.b_base, delta = sh.b_delta, magic = sh.b_magic;

  // 5. per-tile prefix, first output index, number of work items
  unsigned long long run = excl;
  int o_prev = first_target_at_or_above(run, base, delta, magic, N);
  int n_it = 0;
  for (int k = k0; k < k1; ++k) {
    p.P[k] = run;
    p.ofirst[k] = o_prev;
    run += ehat(k);
    const int o_next = first_target_at_or_above(run, base, delta, magic, N);
    n_it += (o_next - o_prev + kOutChunk - 1) / kOutChunk;
    o_prev = o_next;
  }
  if (tid == 0) p.ofirst[G] = N;
  int n_items_total;
  const int it0 = block_excl_scan_i(n_it, &n_items_total, sh.scan_i);   // barrier: ofirst visible

  // 6. emit work items (tile, first output, end output)
  int ib = it0;
  for (int k = k0; k < k1; ++k) {
    const int o0 = p.ofirst[k], o1 = p.ofirst[k + 1];
    for (int o = o0; o < o1; o += kOutChunk) p.items[ib++] = make_int4(k, o, min(o1, o + kOutChunk), 0);
  }
  if (tid == 0) {
    st->n_items = n_items_total;
    st->base = base; st->delta = delta; st->delta_magic = magic; st->total = sh.b_total;
    st->nM = nM; st->Fg = Fg;
    st->ticket = 0u;
  }
}

// ---------------------------------------------------------------------------
// Pass 1
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 3) pass1_kernel(Plan p, TickArgs a) {
  __shared__ float s_max[kThreads / 32];
  __shared__ double s_red[3][kThreads / 32];
  __shared__ unsigned long long s_redE[kThreads / 32];
  __shared__ int s_last;
  __shared__ EpiShared s_epi;

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k = blockIdx.x;
  const DevState* st = p.st;
  const int tick = st->tick;
  const int cur = st->cur;
  const bool carry = st->resampled_prev == 0;
  const int nM_prev = st->nM_prev;
  const PcgTick c = pcg_tick_consts(st->seed, st->At, st->Bt);
  float* hb = cur ? p.h1 : p.h0;

  ObsModel obs = a.obs;
  if (a.y_ptr) obs.y = __ldg(a.y_ptr);

  float carry_off = 0.0f;
  if (carry) {
    const int nkp = p.nexp[k];
    carry_off = (nkp == kNkEmpty) ? -INFINITY : (float)(nkp - nM_prev);
  }

  const int tile0 = k * kTile;
  float4 h4[4], w4[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i0 = tile0 + 4 * (tid + kThreads * r);
    h4[r] = *reinterpret_cast<const float4*>(hb + i0);
    if (carry) w4[r] = *reinterpret_cast<const float4*>(p.w + i0);
    else w4[r] = make_float4(1.f, 1.f, 1.f, 1.f);
  }

  float x[kPerThread], hv[kPerThread];
  const unsigned long long step2 = 2ull * c.k2;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i0 = tile0 + 4 * (tid + kThreads * r);
    unsigned long long s = c.k1 + c.k2 * pcg_inc((uint32_t)i0);
    float hh[4] = {h4[r].x, h4[r].y, h4[r].z, h4[r].w};
    const float wp[4] = {w4[r].x, w4[r].y, w4[r].z, w4[r].w};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      float h = hh[e];
      if (tick > 0) {
        const float z = icdf_normal(pcg_uniform(pcg_output(s)));
        h = propagate(h, a.mu, a.rho, a.sigma, z);
      }
      s += step2;
      float xx = obs_logpdf(obs, h) * kLog2e;
      if (carry) xx += lg2_approx(wp[e]) + carry_off;
      if (i0 + e >= p.N) xx = -INFINITY;
      hh[e] = h;
      x[4 * r + e] = xx;
      hv[4 * r + e] = h;
    }
    *reinterpret_cast<float4*>(hb + i0) = make_float4(hh[0], hh[1], hh[2], hh[3]);
  }

  // tile max -> power-of-two exponent n_k (all tile weights <= 1)
  float mx = x[0];
#pragma unroll
  for (int e = 1; e < kPerThread; ++e) mx = fmaxf(mx, x[e]);
  mx = warp_max_f(mx);
  if (lane == 0) s_max[warp] = mx;
  __syncthreads();
  mx = s_max[0];
#pragma unroll
  for (int w = 1; w < kThreads / 32; ++w) mx = fmaxf(mx, s_max[w]);
  const int nk = (mx == -INFINITY) ? kNkEmpty : (int)ceilf(fmaxf(mx, -1.0e9f));
  const float fnk = (float)nk;

  float fS = 0.f, fQ = 0.f, fH = 0.f;
  unsigned long long E = 0ull;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i0 = tile0 + 4 * (tid + kThreads * r);
    float wv[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int idx = 4 * r + e;
      const float w = (nk == kNkEmpty) ? 0.0f : fminf(ex2_approx(x[idx] - fnk), 1.0f);
      wv[e] = w;
      fS += w;
      fQ = fmaf(w, w, fQ);
      fH = fmaf(w, hv[idx], fH);
      E += fix_weight(w);
    }
    *reinterpret_cast<float4*>(p.w + i0) = make_float4(wv[0], wv[1], wv[2], wv[3]);
  }
  double dS = warp_sum_d((double)fS), dQ = warp_sum_d((double)fQ), dH = warp_sum_d((double)fH);
  E = warp_sum_u64(E);
  if (lane == 0) { s_red[0][warp] = dS; s_red[1][warp] = dQ; s_red[2][warp] = dH; s_redE[warp] = E; }
  __syncthreads();
  if (tid == 0) {
    double tS = 0.0, tQ = 0.0, tH = 0.0;
    unsigned long long tE = 0ull;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) { tS += s_red[0][w]; tQ += s_red[1][w]; tH += s_red[2][w]; tE += s_redE[w]; }
    p.nexp[k] = nk; p.E[k] = tE; p.S[k] = tS; p.Q[k] = tQ; p.H[k] = tH;
    __threadfence();
    const unsigned t = atomicAdd(&p.st->ticket, 1u);
    s_last = (t == (unsigned)(p.G - 1));
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  pass1_epilogue(p, a, tick, cur, s_epi);
}

// ---------------------------------------------------------------------------
// Pass 2
// ---------------------------------------------------------------------------
constexpr size_t kPass2Smem = (size_t)kTile * 8 + (size_t)kTile * 4 + (size_t)kOutChunk * 8;

__global__ void __launch_bounds__(kThreads, 2) pass2_kernel(Plan p, TickArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  unsigned long long* Cs = reinterpret_cast<unsigned long long*>(smem);
  float* hs = reinterpret_cast<float*>(Cs + kTile);
  float* outb = hs + kTile;
  int* ancb = reinterpret_cast<int*>(outb + kOutChunk);
  __shared__ unsigned long long s_scan[kThreads / 32 + 1];
  __shared__ int s_err;

  const DevState* st = p.st;
  if (!st->do_resample) return;
  const int n_items = st->n_items;
  const unsigned long long base = st->base, delta = st->delta;
  const int nM = st->nM, Fg = st->Fg;
  const int src = st->src;
  const float* hsrc = src ? p.h1 : p.h0;
  float* hdst = src ? p.h0 : p.h1;
  const int tid = threadIdx.x;
  if (tid == 0) s_err = 0;

  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const int4 item = p.items[it];
    const int k = item.x, oa = item.y, ob = item.z;
    const int j0 = k * kTile;
    const int nA = min(kTile, p.N - j0);
    const int nB = ob - oa;
    const int r = nM - p.nexp[k] + kFixF - Fg;
    const unsigned long long Pk = p.P[k];

    // stage the h tile (coalesced float4)
    const float4* hsrc4 = reinterpret_cast<const float4*>(hsrc + j0);
#pragma unroll
    for (int v = 0; v < kTile / 4 / kThreads; ++v)
      reinterpret_cast<float4*>(hs)[tid + kThreads * v] = hsrc4[tid + kThreads * v];

    // exact fixed-point prefix of the tile: 16 contiguous weights per thread
    const float4* wv = reinterpret_cast<const float4*>(p.w + j0 + tid * kPerThread);
    unsigned long long L[kPerThread];
    unsigned long long run = 0ull;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const float4 f = wv[v];
      const float ff[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int j = tid * kPerThread + 4 * v + e;
        run += (j < nA) ? fix_weight(ff[e]) : 0ull;
        L[4 * v + e] = run;
      }
    }
    unsigned long long tot;
    const unsigned long long excl = block_excl_scan_u64(run, &tot, s_scan);
#pragma unroll
    for (int e = 0; e < kPerThread; ++e) Cs[tid * kPerThread + e] = Pk + shr64(excl + L[e], r);
    __syncthreads();

    // merge path: thread's slice [d0, d1) of the merged (elements, targets) order
    const int total = nA + nB;
    const int d0 = (int)(((long long)tid * total) / kThreads);
    const int d1 = (int)(((long long)(tid + 1) * total) / kThreads);
    int lo = max(0, d0 - nB), hi = min(d0, nA);
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      const unsigned long long tt = base + (unsigned long long)(oa + d0 - mid - 1) * delta;
      if (Cs[mid] <= tt) lo = mid + 1; else hi = mid;
    }
    int j = lo, i = d0 - lo;
    unsigned long long ti = base + (unsigned long long)(oa + i) * delta;
    for (int d = d0; d < d1; ++d) {
      if (i < nB && (j >= nA || ti < Cs[j])) {
        int jj = j;
        if (jj >= nA) { jj = nA - 1; s_err = 1; }   // unreachable by construction; keeps the access in bounds
        outb[i] = hs[jj];
        ancb[i] = j0 + jj;
        ++i;
        ti += delta;
      } else {
        ++j;
      }
    }
    __syncthreads();
    for (int q = tid; q < nB; q += kThreads) hdst[oa + q] = outb[q];
    if (a.anc) for (int q = tid; q < nB; q += kThreads) a.anc[oa + q] = ancb[q];
    __syncthreads();
  }
  if (tid == 0 && s_err) p.st->error = BPF_ERR_STATE;
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

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
cudaError_t launch_init(const Plan& p, float mu, float std_stat, int seed, cudaStream_t s) {
  const int n = p.G * kTile;
  init_kernel<<<(n + 255) / 256, 256, 0, s>>>(p, mu, std_stat, seed);
  return cudaGetLastError();
}

cudaError_t launch_pass1(const Plan& p, const TickArgs& a, cudaStream_t s) {
  pass1_kernel<<<p.G, kThreads, 0, s>>>(p, a);
  return cudaGetLastError();
}

size_t pass2_smem_bytes() { return kPass2Smem; }

int pass2_grid_size(int device) {
  static int configured = -1;
  if (configured != device) {
    cudaFuncSetAttribute(pass2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPass2Smem);
    configured = device;
  }
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pass2_kernel, kThreads, kPass2Smem);
  if (per_sm < 1) per_sm = 1;
  return sms * per_sm;
}

cudaError_t launch_pass2(const Plan& p, const TickArgs& a, int grid, cudaStream_t s) {
  pass2_kernel<<<grid, kThreads, kPass2Smem, s>>>(p, a);
  return cudaGetLastError();
}

cudaError_t launch_debug_pcg(int seed, int n, int t, uint32_t* d_out, float* d_norm, cudaStream_t s) {
  unsigned long long At = 1ull, Bt = 0ull;
  for (int k = 0; k < t; ++k) { At *= kPcgMult; Bt = Bt * kPcgMult + 1ull; }
  debug_pcg_kernel<<<(n + 255) / 256, 256, 0, s>>>(seed, n, At, Bt, d_out, d_norm);
  return cudaGetLastError();
}

}  // namespace bpf
