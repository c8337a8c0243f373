// bpf_batch.cu — persistent batched SV filter kernel (one filter per CTA at a
// time, whole filter resident in shared memory for all T ticks).
//
// Per tick and filter (N particles, G = ceil(N/4096) tiles, NT threads):
//   1. propagate + log2-weight (+ carried tile-relative log2-weight), per-tile max
//   2. tile-relative log2-weights d = x - n_k (kept for the next tick's carry),
//      weights 2^d, tile partial sums and exact fixed-point tile masses
//   3. thread 0: FP64 combine, log-likelihood increment, ESS, mean, decision;
//      on resampling ticks the fixed-point CDF tile prefix, total and spacing
//   4. resampling: per-thread contiguous chunk scan, per-element count of the
//      evenly spaced targets, ancestor slots, gather into the other buffer.
// Particle arrays use a swizzled layout (column c of each 32-float row stored
// at c ^ row) so both the lane-strided and the per-thread-contiguous access
// patterns are free of shared-memory bank conflicts.
//
// Gradient form (batch_grad_kernel): after a filter's taped forward, the same
// CTA runs its adjoint backward, checkpoint segment by segment from the last:
// the segment's particles are recomputed from the checkpoint through the
// taped child lists (parent-centric: every parent writes its children) into
// a per-CTA global segment buffer, then lambda goes backward through the
// segment in shared memory. Children sums are taken first (into a scratch
// array), then lambda is overwritten in place, so one lambda array suffices.
// The parameter adjoints accumulate per thread in FP64 and are summed once
// per filter.
#include "bpf_batch.cuh"
#include "bpf_block.cuh"

namespace bpf {

__device__ __forceinline__ int swz(int i) { return (i & ~31) | ((i ^ (i >> 5)) & 31); }

template <int NT>
struct BatchShared {
  float tmax[kBatchMaxTiles][NT / 32];
  double sred[3][kBatchMaxTiles][NT / 32];
  unsigned long long ered[kBatchMaxTiles][NT / 32];
  double tsum[3][kBatchMaxTiles];              // per-tile FP64 sums over the warps
  unsigned long long tmass[kBatchMaxTiles];
  unsigned long long scan[NT / 32 + 1];
  unsigned long long excl[NT];
  unsigned long long Pk[kBatchMaxTiles];
  float carry_off[kBatchMaxTiles];
  int rk[kBatchMaxTiles];
  unsigned long long base, delta, magic;
  int resample, carry, next;
  double gred[5][NT / 32];
  double fin_ll, fin_logS;                     // the log-likelihood keeper's state at the end of a run
};

// The tick's decision runs on thread 0; the FP64 logarithm of the weight sum, the increment and
// the running log-likelihood on the first lane of the second warp (kLogTid), concurrently.
constexpr int kLogTid = 32;

size_t batch_smem_bytes(int maxn, bool sort_perm) {
  const size_t u16 = (((size_t)maxn * 2 + 15) / 16) * 16;
  return (size_t)maxn * 8 + u16 + (sort_perm ? u16 : 0);
}

// Sorts the particles H (keys) with their log2-weights Wt, and perm when given, into ascending
// order of H: a bitonic network whose comparators all put the smaller key at the lower index
// (the first step of every merge compares mirrored positions), so positions n..2^k-1 act as
// +inf and are never stored. Steps whose partners are less than 32 apart run on 32-element
// segments held in registers (one element per lane, partners by warp shuffle); only the wider
// steps go through shared memory with a barrier each. Deterministic for equal keys. Ends with a
// barrier.
template <int NT>
__device__ __noinline__ void sort_particles(float* H, float* Wt, unsigned short* perm, int n) {
  constexpr int W = NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int m = 32;
  while (m < n) m <<= 1;
  // merges k = k_lo..k_hi, each from its step min(k/2, 16) down to 1, segment by segment
  auto warp_steps = [&](int k_lo, int k_hi) {
    for (int sg = warp; sg < (m >> 5); sg += W) {
      const int i = (sg << 5) + lane;
      const bool in = i < n;
      float key = in ? H[swz(i)] : INFINITY;
      float w = in ? Wt[swz(i)] : 0.0f;
      unsigned pm = (perm && in) ? (unsigned)perm[i] : 0u;
      for (int k = k_lo; k <= k_hi; k <<= 1) {
        for (int j = min(k >> 1, 16); j > 0; j >>= 1) {
          const bool mirror = j == (k >> 1);                  // k <= 32: the merge's first step
          const int x = mirror ? k - 1 : j;
          const bool lower = (lane & j) == 0;
          const float pk = __shfl_xor_sync(0xffffffffu, key, x);
          const float pw = __shfl_xor_sync(0xffffffffu, w, x);
          const unsigned pp = perm ? __shfl_xor_sync(0xffffffffu, pm, x) : 0u;
          if (lower ? (key > pk) : (pk > key)) { key = pk; w = pw; pm = pp; }
        }
      }
      if (in) {
        H[swz(i)] = key;
        Wt[swz(i)] = w;
        if (perm) perm[i] = (unsigned short)pm;
      }
    }
    __syncthreads();
  };
  warp_steps(2, 32);
  for (int k = 64; k <= m; k <<= 1) {
    for (int j = k >> 1; j >= 32; j >>= 1) {
      for (int p = threadIdx.x; p < (m >> 1); p += NT) {
        const int off = p & (j - 1);
        const int i = ((p - off) << 1) + off;
        const int l = (j == (k >> 1)) ? i + (k - 1 - 2 * off) : i + j;
        if (l < n) {
          const int si = swz(i), sl = swz(l);
          const float a = H[si], c = H[sl];
          if (a > c) {
            H[si] = c; H[sl] = a;
            const float wa = Wt[si];
            Wt[si] = Wt[sl]; Wt[sl] = wa;
            if (perm) { const unsigned short q = perm[i]; perm[i] = perm[l]; perm[l] = q; }
          }
        }
      }
      __syncthreads();
    }
    warp_steps(k, k);
  }
}

// Resampling uniform of a correlated-noise tick: the 23-bit grid point below Phi(v).
__device__ __forceinline__ unsigned long long u23_of_normal(float v) {
  return (unsigned long long)fminf(floorf(normcdff(v) * 8388608.0f), 8388607.0f);
}

// NOISE: a correlated-noise run (BatchArgs::nz_out set); the other instances carry none of its code.
template <int NT, bool RESUMABLE, bool NOISE = false>
__device__ void batch_run_filter(const BatchArgs& a, const BatchFilterDev& f, int b, float* bufA, float* bufB,
                                 unsigned short* marks, BatchShared<NT>& sh, int maxn,
                                 unsigned short* perm = nullptr) {
  constexpr int W = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int N = f.n;
  const int G = (N + kTile - 1) / kTile;
  const bool gauss = !(f.nu > 0.0f);
  ObsModel obs;
  obs.y = 0.0f; obs.nu = f.nu; obs.c_obs = f.c_obs; obs.inv_nu = f.inv_nu; obs.nu_p1h = f.nu_p1h;
  int chunk = 1;
  while (chunk * NT < N) chunk <<= 1;           // power of two: chunks never straddle a tile
  // correlated-noise areas of this filter (null outside correlated-noise runs)
  const int nzs = batch_noise_stride(N), npad = nzs - 4;
  float* zo = NOISE ? a.nz_out + a.nz_out_off[b] : nullptr;
  const float* zi = (NOISE && a.nz_in) ? a.nz_in + a.nz_in_off[b] : nullptr;
  const float cr = a.cp_rho, cs = a.cp_scale;
  if (!NOISE) perm = nullptr;

  float* H = bufA;
  float* Wt = bufB;
  uint64_t At = 1ull, Bt = 0ull;
  // thread-0 filter state
  const double logN = log((double)N);
  double logS_prev = logN, ll_total = 0.0;     // kept by thread kLogTid
  uint64_t ustate = (unsigned long long)f.seed * 67890ULL + 12345ULL;
  int n_res = 0;
  float hm_last = 0.0f;
  const int t0 = (RESUMABLE && a.t0_dev) ? *a.t0_dev : 0;
  BatchFilterState* fs = (RESUMABLE && a.st) ? a.st + b : nullptr;
  const long long soff = (RESUMABLE && a.st) ? a.st_off[b] : 0;
  if (fs && t0 > 0) {
    // resume from the state saved at the end of the previous launch
    const BatchFilterState r = *fs;
    for (int i = tid; i < N; i += NT) H[swz(i)] = a.st_h[soff + i];
    if (r.carry)
      for (int i = tid; i < N; i += NT) Wt[swz(i)] = a.st_w[soff + i];
    pcg_jump((uint64_t)t0, &At, &Bt);
    logS_prev = r.logS_prev; ll_total = r.ll_total; ustate = r.ustate; n_res = r.n_res; hm_last = r.hm_last;
    if (tid == 0) {
      sh.carry = r.carry;
      for (int k = 0; k < kBatchMaxTiles; ++k) sh.carry_off[k] = r.carry_off[k];
    }
  } else {
    // h_0 from draw 0 (stationary law)
    const PcgTick c = pcg_tick_consts(f.seed, 1ull, 0ull);
    for (int i = tid; i < N; i += NT) {
      const uint64_t s = c.k1 + c.k2 * pcg_inc((uint32_t)i);
      float z = icdf_normal(pcg_uniform(pcg_output(s)));
      if constexpr (NOISE) {
        if (zi) z = fmaf(cr, zi[i], cs * z);
        zo[i] = z;
      }
      bufA[swz(i)] = fmaf(f.std_stat, z, f.mu);
    }
    if (tid == 0) sh.carry = 0;
  }
  __syncthreads();

  for (int t = t0; t < t0 + a.T; ++t) {
    const float y = __ldg(a.y + (a.y_abs ? t : t - t0));
    const float y2 = y * y;
    obs.y = y;
    const bool carry = sh.carry != 0;
    const PcgTick c = pcg_tick_consts(f.seed, At, Bt);
    float* ck = (a.g_ckpt && t % a.g_K == 0) ? a.g_ckpt + (size_t)(t / a.g_K) * maxn : nullptr;

    // 1. propagate + log2-weight, per-tile max
    float tmax[kBatchMaxTiles];
#pragma unroll
    for (int k = 0; k < kBatchMaxTiles; ++k) {
      float m = -INFINITY;
      if (k < G) {
        const float coff = carry ? sh.carry_off[k] : 0.0f;
        const int i1 = min(N, (k + 1) * kTile);
        for (int i = k * kTile + tid; i < i1; i += NT) {
          const int si = swz(i);
          float h = H[si];
          if (ck) ck[i] = h;
          if (t > 0) {
            const uint64_t s = c.k1 + c.k2 * pcg_inc((uint32_t)i);
            float z = icdf_normal_active(pcg_uniform(pcg_output(s)));
            if (f.nu_int > 0) z *= tstate_scale(c, (uint32_t)i, f.nu_int, f.nu_state);
            if constexpr (NOISE) {
              if (zi) z = fmaf(cr, zi[(size_t)t * nzs + i], cs * z);
              zo[(size_t)t * nzs + i] = z;
            }
            h = propagate(h, f.mu, f.rho, f.sigma, z);
            H[si] = h;
          }
          // same operation sequence as the plain filter's pass 1 (bit-identical x)
          float x = gauss ? obs_log2pdf_gauss_plus(y2, h, kGaussLog2C + coff)
                          : obs_log2pdf_t_plus(obs, __fmul_rn(y2, obs.inv_nu), h, __fmul_rn(obs.c_obs, kLog2e) + coff);
          if (carry) x += Wt[si];                  // carried tile-relative log2-weight
          Wt[si] = x;
          m = fmaxf(m, x);
        }
      }
      tmax[k] = m;
    }
    // the reductions run for the filter's G tiles only (G is the same for the whole CTA)
#pragma unroll
    for (int k = 0; k < kBatchMaxTiles; ++k) {
      if (k < G) {
        const float v = warp_max_f(tmax[k]);
        if (lane == 0) sh.tmax[k][warp] = v;
      }
    }
    __syncthreads();
    int nk[kBatchMaxTiles];
#pragma unroll
    for (int k = 0; k < kBatchMaxTiles; ++k) {
      float m = -INFINITY;
      if (k < G) m = warp_max_f(lane < W ? sh.tmax[k][lane] : -INFINITY);   // every warp, the same max
      nk[k] = (m == -INFINITY) ? kNkEmpty : (int)ceilf(fmaxf(m, -1.0e9f));
    }

    // 2. tile-relative weights, partial sums, exact fixed-point tile masses
#pragma unroll
    for (int k = 0; k < kBatchMaxTiles; ++k) {
      float fS = 0.f, fQ = 0.f, fH = 0.f;
      unsigned long long E = 0ull;
      if (k < G) {
        const float fnk = (nk[k] == kNkEmpty) ? INFINITY : (float)nk[k];   // empty tile: every 2^d = 0
        const int i1 = min(N, (k + 1) * kTile);
        for (int i = k * kTile + tid; i < i1; i += NT) {
          const int si = swz(i);
          const float d = Wt[si] - fnk;
          const float w = tile_weight(d);
          Wt[si] = d;                              // stored as the tile-relative log2-weight
          fS += w;
          fQ = fmaf(w, w, fQ);
          fH = fmaf(w, H[si], fH);
          E += fix_weight(w);
        }
      }
      if (k < G) {
        const double dS = warp_sum_d((double)fS), dQ = warp_sum_d((double)fQ), dH = warp_sum_d((double)fH);
        E = warp_sum_u64(E);
        if (lane == 0) { sh.sred[0][k][warp] = dS; sh.sred[1][k][warp] = dQ; sh.sred[2][k][warp] = dH; sh.ered[k][warp] = E; }
      }
    }
    __syncthreads();
    // per-tile sums over the warps, one warp per tile (a fixed shuffle tree over its W lanes)
    for (int k = warp; k < G; k += W) {
      const bool on = lane < W;
      const double s1 = warp_sum_d_w<W>(on ? sh.sred[0][k][lane] : 0.0);
      const double s2 = warp_sum_d_w<W>(on ? sh.sred[1][k][lane] : 0.0);
      const double s3 = warp_sum_d_w<W>(on ? sh.sred[2][k][lane] : 0.0);
      const unsigned long long e = warp_sum_u64_w<W>(on ? sh.ered[k][lane] : 0ull);
      if (lane == 0) { sh.tsum[0][k] = s1; sh.tsum[1][k] = s2; sh.tsum[2][k] = s3; sh.tmass[k] = e; }
    }
    __syncthreads();

    // 3. decision (thread 0) and log-likelihood (thread kLogTid), from the same sums
    if (tid == 0 || tid == kLogTid) {
      int nM = kNkEmpty;
      for (int k = 0; k < G; ++k) nM = max(nM, nk[k]);
      double S = 0.0, Q = 0.0, Hm = 0.0;
      unsigned long long Ek[kBatchMaxTiles];
      for (int k = 0; k < kBatchMaxTiles; ++k) {
        Ek[k] = 0ull;
        if (k >= G || nk[k] == kNkEmpty) continue;
        Ek[k] = sh.tmass[k];
        const double sc = pow2d(nk[k] - nM);
        S += sh.tsum[0][k] * sc; Q += sh.tsum[1][k] * sc * sc; Hm += sh.tsum[2][k] * sc;
      }
      const bool degenerate = (nM == kNkEmpty) || !(S > 0.0);
      int resample = 0;
      if (!degenerate) {
        const double ess = S * S / Q;
        resample = (a.ess_threshold <= 0.0f) || (ess / (double)N < (double)a.ess_threshold);
      }
      if (tid == kLogTid) {
        const double lS = degenerate ? 0.0 : log(S);
        const double dll = degenerate ? -INFINITY
                                      : (double)nM * 0.693147180559945309417232121458 + lS - logS_prev;
        ll_total += dll;
        if (a.dll) a.dll[(size_t)b * a.T + (t - t0)] = dll;
        logS_prev = (resample || degenerate) ? logN : lS;
      } else {
        const float hm = degenerate ? __int_as_float(0x7fc00000) : (float)(Hm / S);
        hm_last = hm;
        if (a.g_norm)
          a.g_norm[t] = degenerate ? make_float2(0.0f, 0.0f) : make_float2((float)(1.0 / S), __int_as_float(nM));
        if (a.hmean) a.hmean[(size_t)b * a.T + (t - t0)] = hm;
        unsigned long long u = 0ull;
        if constexpr (NOISE) {
          // the tick's resampling normal: slot kBatchMaxN of the filter's streams (no particle's)
          float v = icdf_normal(pcg_uniform(pcg_output(c.k1 + c.k2 * pcg_inc((uint32_t)kBatchMaxN))));
          if (zi) v = fmaf(cr, zi[(size_t)t * nzs + npad], cs * v);
          zo[(size_t)t * nzs + npad] = v;
          u = u23_of_normal(v);
        }
        if (resample) {
          if constexpr (!NOISE) {
            const uint64_t old = ustate;
            ustate = old * kPcgMult + kHostInc;
            u = pcg_output(old) >> 9;
          }
          ++n_res;
          const int Fg = min(kFixF, 62 - ceil_log2_u((unsigned)N));
          unsigned long long P = 0ull;
          for (int k = 0; k < kBatchMaxTiles; ++k) {
            const int r = (k < G && nk[k] != kNkEmpty) ? nM - nk[k] + kFixF - Fg : 64;
            sh.rk[k] = r;
            sh.Pk[k] = P;
            P += shr64(Ek[k], r);
          }
          unsigned long long delta = udiv_fp64(P, (unsigned long long)N);
          if (delta == 0ull) delta = 1ull;
          const unsigned long long hi = __umul64hi(u, delta), lo = u * delta;
          sh.base = (hi << 41) | (lo >> 23);
          sh.delta = delta;
          sh.magic = udiv_magic_of(delta);
          sh.carry = 0;
        } else if (degenerate) {
          sh.carry = 0;
        } else {
          for (int k = 0; k < kBatchMaxTiles; ++k)
            sh.carry_off[k] = (k < G && nk[k] != kNkEmpty) ? (float)(nk[k] - nM) : -INFINITY;
          sh.carry = 1;
        }
        sh.resample = resample;
      }
    }
    At = At * kPcgMult;
    Bt = Bt * kPcgMult + 1ull;
    __syncthreads();

    // 4. systematic resampling (fixed-point CDF, same rule as the plain filter); correlated-noise
    // runs first sort the particles by value (one tile: the log2-weights share one offset)
    if (sh.resample) {
      if constexpr (NOISE) {
        if (perm)
          for (int i = tid; i < N; i += NT) perm[i] = (unsigned short)i;
        __syncthreads();
        sort_particles<NT>(H, Wt, perm, N);
      }
      const unsigned long long base = sh.base, delta = sh.delta, magic = sh.magic;
      const int j0 = tid * chunk, j1 = min(N, j0 + chunk);
      unsigned long long run = 0ull;
      for (int j = j0; j < j1; ++j) {            // the thread's chunk: log2-weights -> weights, in place
        const float w = tile_weight(Wt[swz(j)]);
        Wt[swz(j)] = w;
        run += fix_weight(w);
      }
      unsigned long long tot;
      const unsigned long long excl = block_excl_scan_add<NT>(run, &tot, sh.scan);
      sh.excl[tid] = excl;
      __syncthreads();
      int q = 0, k = 0, r = 64;
      unsigned long long Pk = 0ull, loc = 0ull, tq = 0ull;
      if (j0 < N) {
        k = j0 >> 12;
        r = sh.rk[k];
        Pk = sh.Pk[k];
        loc = excl - sh.excl[(k * kTile) / chunk];          // tile-local exclusive prefix
        q = targets_below(Pk + shr64(loc, r), base, delta, magic, N);
        tq = base + (unsigned long long)q * delta;
      }
      unsigned short* lst = a.g_list ? a.g_list + (size_t)t * maxn : nullptr;
      for (int e = 0; e < chunk; ++e) {
        const int j = j0 + e;
        int lo = 0, hi = 0;
        if (lst) lst[e * NT + tid] = (unsigned short)(j < j1 ? q : N);   // children of j start at slot q
        if (j < j1) {
          loc += fix_weight(Wt[swz(j)]);
          const unsigned long long cj = Pk + shr64(loc, r);
          if (q < N && tq < cj) {
            if (((cj - tq) >> 2) > delta) {
              const int q1 = targets_below(cj, base, delta, magic, N);
              lo = q; hi = q1;
              q = q1;
              tq = base + (unsigned long long)q * delta;
            } else {
              do { marks[q] = (unsigned short)(j + 1); ++q; tq += delta; } while (q < N && tq < cj);
            }
          }
        }
        unsigned heavy = __ballot_sync(0xffffffffu, hi > lo);
        while (heavy) {
          const int sl = __ffs(heavy) - 1;
          heavy &= heavy - 1u;
          const int flo = __shfl_sync(0xffffffffu, lo, sl), fhi = __shfl_sync(0xffffffffu, hi, sl);
          const unsigned short v = (unsigned short)(__shfl_sync(0xffffffffu, j, sl) + 1);
          for (int qq = flo + lane; qq < fhi; qq += 32) marks[qq] = v;
        }
      }
      __syncthreads();
      for (int i = tid; i < N; i += NT) {
        const int anc = (int)marks[i] - 1;
        Wt[swz(i)] = H[swz(anc)];
        if (a.anc) a.anc[((size_t)b * a.T + (t - t0)) * kBatchMaxN + i] = perm ? (int)perm[anc] : anc;
      }
      __syncthreads();
      float* tmp = H; H = Wt; Wt = tmp;
    }
  }
  if (a.particles)
    for (int i = tid; i < N; i += NT) a.particles[(size_t)b * kBatchMaxN + i] = H[swz(i)];
  if (fs) {
    for (int i = tid; i < N; i += NT) a.st_h[soff + i] = H[swz(i)];
    if (sh.carry)
      for (int i = tid; i < N; i += NT) a.st_w[soff + i] = Wt[swz(i)];
  }
  if (tid == kLogTid) { sh.fin_ll = ll_total; sh.fin_logS = logS_prev; }
  __syncthreads();
  if (tid == 0) {
    a.loglik[b] = sh.fin_ll;
    a.h_final[b] = hm_last;
    a.resamples[b] = n_res;
    if (fs) {
      BatchFilterState r;
      r.logS_prev = sh.fin_logS; r.ll_total = sh.fin_ll; r.ustate = ustate;
      r.carry = sh.carry; r.n_res = n_res; r.hm_last = hm_last; r.pad = 0;
      for (int k = 0; k < kBatchMaxTiles; ++k) r.carry_off[k] = sh.carry_off[k];
      *fs = r;
    }
  }
  __syncthreads();
}

template <int NT, bool NOISE>
__global__ void __launch_bounds__(NT, (1024 / NT > 0 ? 1024 / NT : 1)) batch_kernel(BatchArgs a, int maxn) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ BatchShared<NT> sh;
  float* bufA = reinterpret_cast<float*>(smem);
  float* bufB = bufA + maxn;
  unsigned short* marks = reinterpret_cast<unsigned short*>(bufB + maxn);
  unsigned short* perm = (NOISE && a.anc) ? marks + ((maxn + 7) & ~7) : nullptr;
  for (;;) {
    if (threadIdx.x == 0) sh.next = atomicAdd(a.counter, 1);
    __syncthreads();
    const int idx = sh.next;
    __syncthreads();
    if (idx >= a.n_order) break;
    const int b = a.order[idx];
    const BatchFilterDev f = a.filters[b];
    batch_run_filter<NT, true, NOISE>(a, f, b, bufA, bufB, marks, sh, maxn, perm);
  }
  // every CTA has taken its last work item and read the tick before it counts
  // itself done, so the last one may reset the counters and advance the tick
  if (a.ep_done && threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(a.ep_done, 1) == a.ep_total - 1) {
      for (int c = 0; c < a.ep_n; ++c) a.ep_counters[c] = 0;
      if (a.ep_tick) *a.ep_tick += a.ep_add;
      *a.ep_done = 0;
      __threadfence();
    }
  }
}

// ---------------------------------------------------------------------------
// Gradient: adjoint backward of one filter after its taped forward
// ---------------------------------------------------------------------------
constexpr int kBatchHeavy = 32;   // children above which a parent's walk is shared by its warp



template <int NT>
__device__ void batch_run_backward(const BatchArgs& a, const BatchFilterDev& f, int b, int maxn, float* lam,
                                   float* hA, float* hB, BatchShared<NT>& sh) {
  constexpr int W = NT / 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int N = f.n, T = a.T, K = a.g_K;
  int chunk = 1;
  while (chunk * NT < N) chunk <<= 1;
  const int j0 = tid * chunk;
  const bool gauss = !(f.nu > 0.0f);
  ObsModel obs;
  obs.y = 0.0f; obs.nu = f.nu; obs.c_obs = f.c_obs; obs.inv_nu = f.inv_nu; obs.nu_p1h = f.nu_p1h;
  const PcgTick pc0 = pcg_tick_consts(f.seed, 1ull, 0ull);
  double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  // first child of the thread's e-th parent; e = chunk is the next thread's first parent
  auto first_child = [&](const unsigned short* lst, int e) -> int {
    int v;
    if (e < chunk) v = (j0 + e < N) ? (int)lst[e * NT + tid] : N;
    else v = (tid + 1 < NT && j0 + chunk < N) ? (int)lst[tid + 1] : N;
    return min(v, N);
  };

  const int nseg = (T + K - 1) / K;
  for (int s = nseg - 1; s >= 0; --s) {
    const int c = s * K, last = min(c + K, T) - 1;
    // 1. particles of tick c from the checkpoint
    {
      const float* ck = a.g_ckpt + (size_t)s * maxn;
      const PcgTick pc = pcg_tick_consts(f.seed, a.g_AB[c].x, a.g_AB[c].y);
      for (int i = tid; i < N; i += NT) {
        float h = ck[i];
        if (c > 0) h = propagate(h, f.mu, f.rho, f.sigma, state_noise(pc, (uint32_t)i, f.nu_int, f.nu_state));
        hA[swz(i)] = h;
        if (last > c) a.g_seg[i] = h;
      }
    }
    __syncthreads();
    float* hp = hA;
    float* hc = hB;
    // 2. ticks c+1..last through the child lists of the previous tick
    for (int t = c + 1; t <= last; ++t) {
      const PcgTick pc = pcg_tick_consts(f.seed, a.g_AB[t].x, a.g_AB[t].y);
      const unsigned short* lst = a.g_list + (size_t)(t - 1) * maxn;
      int lo = first_child(lst, 0);
      for (int e = 0; e < chunk; ++e) {
        const int hi = first_child(lst, e + 1);
        float hpar = 0.0f;
        int wlo = 0, whi = 0;
        if (hi > lo) {
          hpar = hp[swz(j0 + e)];
          if (hi - lo <= kBatchHeavy) {
            for (int i = lo; i < hi; ++i) hc[swz(i)] = propagate(hpar, f.mu, f.rho, f.sigma, state_noise(pc, (uint32_t)i, f.nu_int, f.nu_state));
          } else {
            wlo = lo; whi = hi;
          }
        }
        unsigned heavy = __ballot_sync(0xffffffffu, whi > wlo);
        while (heavy) {
          const int src = __ffs(heavy) - 1;
          heavy &= heavy - 1u;
          const int flo = __shfl_sync(0xffffffffu, wlo, src), fhi = __shfl_sync(0xffffffffu, whi, src);
          const float fh = __shfl_sync(0xffffffffu, hpar, src);
          for (int i = flo + lane; i < fhi; i += 32) hc[swz(i)] = propagate(fh, f.mu, f.rho, f.sigma, state_noise(pc, (uint32_t)i, f.nu_int, f.nu_state));
        }
        lo = max(lo, hi);
      }
      __syncthreads();
      if (t < last) {
        float* sg = a.g_seg + (size_t)(t - c) * maxn;
        for (int i = tid; i < N; i += NT) sg[i] = hc[swz(i)];
      }
      float* tmp = hp; hp = hc; hc = tmp;
    }
    // 3. adjoint, ticks last..c (hp holds h_last)
    for (int t = last; t >= c; --t) {
      if (t < last) {
        const float* sg = a.g_seg + (size_t)(t - c) * maxn;
        for (int i = tid; i < N; i += NT) hp[swz(i)] = sg[i];
        __syncthreads();
      }
      // children sums of lambda_t+1 -> hc, and sum lambda eps over the children
      float acc_eps = 0.0f;
      if (t < T - 1) {
        const PcgTick pcn = pcg_tick_consts(f.seed, a.g_AB[t + 1].x, a.g_AB[t + 1].y);
        const unsigned short* lst = a.g_list + (size_t)t * maxn;
        int lo = first_child(lst, 0);
        for (int e = 0; e < chunk; ++e) {
          const int hi = first_child(lst, e + 1);
          float sum = 0.0f;
          int wlo = 0, whi = 0;
          if (hi - lo <= kBatchHeavy) {
            for (int i = lo; i < hi; ++i) {
              const float l = lam[swz(i)];
              sum += l;
              acc_eps = fmaf(l, state_noise(pcn, (uint32_t)i, f.nu_int, f.nu_state), acc_eps);
            }
          } else {
            wlo = lo; whi = hi;
          }
          unsigned heavy = __ballot_sync(0xffffffffu, whi > wlo);
          while (heavy) {
            const int src = __ffs(heavy) - 1;
            heavy &= heavy - 1u;
            const int flo = __shfl_sync(0xffffffffu, wlo, src), fhi = __shfl_sync(0xffffffffu, whi, src);
            float p = 0.0f;
            for (int i = flo + lane; i < fhi; i += 32) {
              const float l = lam[swz(i)];
              p += l;
              acc_eps = fmaf(l, state_noise(pcn, (uint32_t)i, f.nu_int, f.nu_state), acc_eps);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
            if (lane == src) sum = p;
          }
          if (j0 + e < N) hc[swz(j0 + e)] = sum;
          lo = max(lo, hi);
        }
      }
      __syncthreads();                     // lambda_t+1 fully read
      const float2 nz = a.g_norm[t];
      const float invS = nz.x, nM = (float)__float_as_int(nz.y);
      const float y = __ldg(a.y + t), y2 = y * y;
      obs.y = y;
      float acs = 0.f, acsh = 0.f, al0 = 0.f, al0z = 0.f;
      for (int e = 0; e < chunk; ++e) {
        const int j = j0 + e;
        if (j >= N) break;
        const float h = hp[swz(j)];
        const float cs = (t < T - 1) ? hc[swz(j)] : 0.0f;
        float x, g;
        if (gauss) {
          x = obs_log2pdf_gauss(y2, h);
          g = 0.5f * fmaf(y2, ex2_approx(h * -kLog2e), -1.0f);
        } else {
          x = obs_log2pdf_t_plus(obs, __fmul_rn(y2, obs.inv_nu), h, __fmul_rn(obs.c_obs, kLog2e));
          const float q = y2 * ex2_approx(h * -kLog2e) * obs.inv_nu;
          g = fmaf(obs.nu_p1h, div_approx(q, 1.0f + q), -0.5f);
        }
        const float l = fmaf(f.rho, cs, (ex2_approx(x - nM) * invS) * g);
        lam[swz(j)] = l;
        acs += cs;
        acsh = fmaf(cs, h - f.mu, acsh);
        if (t == 0) {
          const float z0 = state_noise(pc0, (uint32_t)j, 0, 0.0f);
          al0 += l;
          al0z = fmaf(l, z0, al0z);
        }
      }
      acc[0] += (double)acs; acc[1] += (double)acsh; acc[2] += (double)acc_eps;
      acc[3] += (double)al0; acc[4] += (double)al0z;
      __syncthreads();                     // lambda_t complete
    }
  }
  // 4. per-filter sums -> gradient (initial draw h_0 = mu + sigma z / sqrt(max(1-rho^2, 1e-6)))
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const double v = warp_sum_d(acc[k]);
    if (lane == 0) sh.gred[k][warp] = v;
  }
  __syncthreads();
  if (tid == 0) {
    double tt[5];
    for (int k = 0; k < 5; ++k) {
      tt[k] = 0.0;
      for (int w = 0; w < W; ++w) tt[k] += sh.gred[k][w];
    }
    const double r = (double)f.rho, sg = (double)f.sigma;
    const double one_m = 1.0 - r * r;
    const double s2 = fmax(one_m, 1e-6), sd = sqrt(s2);
    const double ds_drho = one_m > 1e-6 ? sg * r / (s2 * sd) : 0.0;
    a.grad[3 * (size_t)b + 0] = (1.0 - r) * tt[0] + tt[3];
    a.grad[3 * (size_t)b + 1] = tt[1] + tt[4] * ds_drho;
    a.grad[3 * (size_t)b + 2] = tt[2] + tt[4] / sd;
  }
  __syncthreads();
}

size_t batch_grad_smem_bytes(int maxn) { return (size_t)maxn * 12; }

__global__ void batch_gather_kernel(BatchFilterDev* dst_tab, BatchFilterState* dst_st, float* dst_h, float* dst_w,
                                    const BatchFilterDev* src_tab, const BatchFilterState* src_st,
                                    const float* __restrict__ src_h, const float* __restrict__ src_w,
                                    const long long* off, const int* idx, const int* mask, const int* new_seed, int n) {
  const int b = blockIdx.x;
  if (mask && !mask[b]) return;
  const int sidx = idx ? idx[b] : b;
  const long long od = off[b], os = off[sidx];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    dst_h[od + i] = src_h[os + i];
    dst_w[od + i] = src_w[os + i];
  }
  if (threadIdx.x == 0) {
    BatchFilterDev f = src_tab[sidx];
    BatchFilterState r = src_st[sidx];
    if (new_seed) {
      f.seed = new_seed[b];
      r.ustate = (unsigned long long)new_seed[b] * 67890ULL + 12345ULL;   // gpu_bpf_ptx_full.cu:353
    }
    dst_tab[b] = f;
    dst_st[b] = r;
  }
}

cudaError_t launch_batch_gather(BatchFilterDev* dst_tab, BatchFilterState* dst_st, float* dst_h, float* dst_w,
                                const BatchFilterDev* src_tab, const BatchFilterState* src_st, const float* src_h,
                                const float* src_w, const long long* off, const int* idx, const int* mask,
                                const int* new_seed, int n, int B, cudaStream_t s) {
  batch_gather_kernel<<<B, 256, 0, s>>>(dst_tab, dst_st, dst_h, dst_w, src_tab, src_st, src_h, src_w, off, idx, mask,
                                        new_seed, n);
  return cudaGetLastError();
}

__global__ void noise_gather_kernel(float* nz, const long long* src_off, const long long* dst_off, long long n4) {
  const int b = blockIdx.y;
  const float4* src = reinterpret_cast<const float4*>(nz + src_off[b]);
  float4* dst = reinterpret_cast<float4*>(nz + dst_off[b]);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

cudaError_t launch_noise_gather(float* nz, const long long* src_off, const long long* dst_off, long long floats,
                                int B, cudaStream_t s) {
  if (B <= 0 || floats <= 0) return cudaSuccess;
  const long long n4 = floats / 4;                 // areas hold whole ticks of a multiple of 4 floats
  const int gx = (int)((n4 + 255) / 256 < 64 ? (n4 + 255) / 256 : 64);
  noise_gather_kernel<<<dim3(gx, B), 256, 0, s>>>(nz, src_off, dst_off, n4);
  return cudaGetLastError();
}

template <int NT>
__global__ void __launch_bounds__(NT, (1024 / NT > 0 ? 1024 / NT : 1)) batch_grad_kernel(BatchArgs a, int maxn) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ BatchShared<NT> sh;
  float* r0 = reinterpret_cast<float*>(smem);
  float* r1 = r0 + maxn;
  float* r2 = r1 + maxn;
  unsigned short* marks = reinterpret_cast<unsigned short*>(r2);
  const int nck = (a.T + a.g_K - 1) / a.g_K;
  BatchArgs s = a;                                   // this CTA slot's tape
  s.g_list = a.g_list + (size_t)blockIdx.x * a.T * maxn;
  s.g_ckpt = a.g_ckpt + (size_t)blockIdx.x * nck * maxn;
  s.g_norm = a.g_norm + (size_t)blockIdx.x * a.T;
  s.g_seg = a.g_seg + (size_t)blockIdx.x * a.g_K * maxn;
  for (;;) {
    if (threadIdx.x == 0) sh.next = atomicAdd(a.counter, 1);
    __syncthreads();
    const int idx = sh.next;
    __syncthreads();
    if (idx >= a.n_order) break;
    const int b = a.order[idx];
    const BatchFilterDev f = a.filters[b];
    batch_run_filter<NT, false>(s, f, b, r0, r1, marks, sh, maxn);
    batch_run_backward<NT>(s, f, b, maxn, r0, r1, r2, sh);
  }
}

// The dynamic shared-memory attribute is set by batch_occupancy (called when
// a class is configured, outside any stream capture).
template <int NT>
static cudaError_t launch_nt(const BatchArgs& a, int maxn, int grid, cudaStream_t s) {
  if (a.nz_out)
    batch_kernel<NT, true><<<grid, NT, batch_smem_bytes(maxn, a.anc != nullptr), s>>>(a, maxn);
  else
    batch_kernel<NT, false><<<grid, NT, batch_smem_bytes(maxn), s>>>(a, maxn);
  return cudaGetLastError();
}

cudaError_t launch_batch_class(const BatchArgs& a, int threads, int maxn, int grid, cudaStream_t s) {
  switch (threads) {
    case 64: return launch_nt<64>(a, maxn, grid, s);
    case 128: return launch_nt<128>(a, maxn, grid, s);
    case 256: return launch_nt<256>(a, maxn, grid, s);
    case 512: return launch_nt<512>(a, maxn, grid, s);
    case 1024: return launch_nt<1024>(a, maxn, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int NT>
static int occ_nt(int maxn) {
  const size_t smem = batch_smem_bytes(maxn);
  cudaFuncSetAttribute(batch_kernel<NT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaFuncSetAttribute(batch_kernel<NT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)batch_smem_bytes(maxn, true));
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_kernel<NT, false>, NT, smem);
  return per;
}

template <int NT>
static cudaError_t launch_grad_nt(const BatchArgs& a, int maxn, int grid, cudaStream_t s) {
  batch_grad_kernel<NT><<<grid, NT, batch_grad_smem_bytes(maxn), s>>>(a, maxn);
  return cudaGetLastError();
}

cudaError_t launch_batch_grad_class(const BatchArgs& a, int threads, int maxn, int grid, cudaStream_t s) {
  switch (threads) {
    case 64: return launch_grad_nt<64>(a, maxn, grid, s);
    case 128: return launch_grad_nt<128>(a, maxn, grid, s);
    case 256: return launch_grad_nt<256>(a, maxn, grid, s);
    case 512: return launch_grad_nt<512>(a, maxn, grid, s);
    case 1024: return launch_grad_nt<1024>(a, maxn, grid, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int NT>
static int grad_occ_nt(int maxn) {
  const size_t smem = batch_grad_smem_bytes(maxn);
  cudaFuncSetAttribute(batch_grad_kernel<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_grad_kernel<NT>, NT, smem);
  return per;
}

int batch_grad_occupancy(int threads, int maxn) {
  switch (threads) {
    case 64: return grad_occ_nt<64>(maxn);
    case 128: return grad_occ_nt<128>(maxn);
    case 256: return grad_occ_nt<256>(maxn);
    case 512: return grad_occ_nt<512>(maxn);
    case 1024: return grad_occ_nt<1024>(maxn);
    default: return 0;
  }
}

int batch_occupancy(int threads, int maxn) {
  switch (threads) {
    case 64: return occ_nt<64>(maxn);
    case 128: return occ_nt<128>(maxn);
    case 256: return occ_nt<256>(maxn);
    case 512: return occ_nt<512>(maxn);
    case 1024: return occ_nt<1024>(maxn);
    default: return 0;
  }
}

}  // namespace bpf
