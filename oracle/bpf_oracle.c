/*
 * bpf_oracle.c — CPU oracle of the SV bootstrap particle filter.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for libgpubpf.so and the
 * timed CPU baseline; nothing in the product links or calls it. It restates
 * the reference algorithm (Tugbars/Bootstrap-Particle-Filter-in-PTX) on the
 * CPU, each function citing the reference lines it follows:
 *
 *   orc_pcg32_*          PCG32 stream of particle slot i
 *                        (ptx_assembly/bpf_kernels_full.ptx:74-91, :140-157;
 *                        known-answer formula tests/test_rng_diag.cu:78-96)
 *   orc_host_pcg32       resampling-uniform stream (gpu_bpf/gpu_bpf_ptx_full.cu:241-251)
 *   orc_acklam_f64       Acklam inverse normal CDF in FP64 (PTX :166-205 in FP32)
 *   orc_icdf_f64         the same plus Acklam's published Halley refinement step
 *                        (erfc-based): the FP64 oracle's inverse normal CDF
 *   orc_f64_*            the same filter stepped one tick at a time (lock-step checks
 *                        of runs of any length), with the reference's Silverman
 *                        jitter after resampling (gpu_bpf_ptx_full.cu:708-738)
 *   orc_filter_f64       FP64 filter in this build's semantics, optionally
 *                        replaying resampling decisions and ancestors
 *   orc_filter_noise_f64 FP64 filter driven by given auxiliary noise, sorting the
 *                        particles before every resampling (the correlated-noise runs
 *                        of the reference's CPMMH moves, smc2/smc2_rbpf_batch.cu:651-935)
 *   orc_apf_f64          FP64 auxiliary particle filter (gpu_bpf_ptx_full.cu:990-1175)
 *                        with the PCG32 streams, optionally replaying ancestors
 *   orc_grad_f64         d loglik / d(mu, rho, sigma) of the FP64 filter with the
 *                        resampling ancestors held fixed (tests/diff_bpf.py:186-237
 *                        with detached indices :35-56), forward-mode tangents or
 *                        reverse-mode adjoint
 *   orc_tstate_scale     Student-t state-noise scale (counter-based chi2 draws)
 *   orc_resample_fixed   exact mirror of the GPU fixed-point systematic resampling
 *   orc_ref_run          FP32 restatement of the reference tick loop
 *                        (gpu_bpf_ptx_full.cu:340-771 with PTX kernels :51-842),
 *                        OpenMP over particles: the CPU baseline
 *   orc_ref_init,        the same initial state, tick and resampling stage by
 *   orc_ref_tick,        stage on given particles (lock-step check against the
 *   orc_ref_resample     reference run on a GPU)
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PCG_A 6364136223846793005ULL
#define HOST_INC 1442695040888963407ULL
#define TILE 4096
#define FIXF 50
#define NK_EMPTY (-(1 << 30))

/* ------------------------------------------------------------------------- */
/* PCG32                                                                      */
/* ------------------------------------------------------------------------- */
uint32_t orc_pcg32_output(uint64_t old) {
    uint32_t xsh = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xsh >> rot) | (xsh << ((-rot) & 31u));
}

/* bpf_init_rng: inc = (2i+1)|1 in 32 bits, state = (seed*A + inc)*A + inc */
void orc_pcg32_init(int seed, uint32_t i, uint64_t* state, uint64_t* inc) {
    uint32_t i2 = 2u * i + 1u;
    uint64_t c = (uint64_t)(i2 | 1u);
    uint64_t s = (uint64_t)(int64_t)seed * PCG_A + c;
    s = s * PCG_A + c;
    *state = s;
    *inc = c;
}

/* Output of draw t (t = 0 is the init draw) by stepping the LCG t times. */
uint32_t orc_pcg32_draw_stepped(int seed, uint32_t i, int t) {
    uint64_t s, inc;
    orc_pcg32_init(seed, i, &s, &inc);
    for (int k = 0; k < t; ++k) s = s * PCG_A + inc;
    return orc_pcg32_output(s);
}

/* Jump-ahead constants A^t and sum_{k<t} A^k (mod 2^64), O(log t). */
void orc_pcg32_jump(uint64_t t, uint64_t* At, uint64_t* Bt) {
    uint64_t acc_mult = 1, acc_plus = 0, cur_mult = PCG_A, cur_plus = 1;
    while (t > 0) {
        if (t & 1) { acc_mult *= cur_mult; acc_plus = acc_plus * cur_mult + cur_plus; }
        cur_plus = (cur_mult + 1) * cur_plus;
        cur_mult *= cur_mult;
        t >>= 1;
    }
    *At = acc_mult; *Bt = acc_plus;
}

uint32_t orc_pcg32_draw_jump(int seed, uint32_t i, int t) {
    uint64_t s0, inc, At, Bt;
    orc_pcg32_init(seed, i, &s0, &inc);
    orc_pcg32_jump((uint64_t)t, &At, &Bt);
    return orc_pcg32_output(At * s0 + Bt * inc);
}

/* u = (out >> 9) * 2^-23 clamped to [0x358637BD, 0x3F7FFBCE] (PTX :159-164) */
float orc_uniform(uint32_t out) {
    float u = (float)(out >> 9) * 1.1920928955078125e-07f;
    const float lo = 9.99999997475242708e-07f, hi = 0.999935984611511230f;
    if (u < lo) u = lo;
    if (u > hi) u = hi;
    return u;
}

/* gpu_bpf_ptx_full.cu:241-251 */
uint32_t orc_host_pcg32(uint64_t* state) {
    uint64_t old = *state;
    *state = old * PCG_A + HOST_INC;
    return orc_pcg32_output(old);
}
uint64_t orc_host_seed(int seed) { return (uint64_t)(int64_t)seed * 67890ULL + 12345ULL; }

/* ------------------------------------------------------------------------- */
/* Acklam inverse normal CDF (P. J. Acklam 2003, published coefficients)      */
/* ------------------------------------------------------------------------- */
static const double AK_A[6] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                               1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00};
static const double AK_B[5] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                               6.680131188771972e+01, -1.328068155288572e+01};
static const double AK_C[6] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                               -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00};
static const double AK_D[4] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                               3.754408661907416e+00};

double orc_acklam_f64(double p) {
    double q = p - 0.5;
    if (fabs(q) < 0.47575) {
        double r = q * q;
        double num = (((((AK_A[0] * r + AK_A[1]) * r + AK_A[2]) * r + AK_A[3]) * r + AK_A[4]) * r + AK_A[5]) * q;
        double den = ((((AK_B[0] * r + AK_B[1]) * r + AK_B[2]) * r + AK_B[3]) * r + AK_B[4]) * r + 1.0;
        return num / den;
    }
    int low = p < 0.5;
    double pp = low ? p : 1.0 - p;
    double s = sqrt(-2.0 * log(pp));
    double num = ((((AK_C[0] * s + AK_C[1]) * s + AK_C[2]) * s + AK_C[3]) * s + AK_C[4]) * s + AK_C[5];
    double den = (((AK_D[0] * s + AK_D[1]) * s + AK_D[2]) * s + AK_D[3]) * s + 1.0;
    double z = num / den;
    return low ? z : -z;
}

/* Acklam's refinement: one Halley step on Phi(z) - p, Phi via erfc. The upper
 * half uses the symmetry z(p) = -z(1-p) so that Phi(z) - p never cancels. */
double orc_icdf_f64(double p) {
    if (p > 0.5) return -orc_icdf_f64(1.0 - p);
    double z = orc_acklam_f64(p);
    const double e = 0.5 * erfc(-z / 1.41421356237309504880) - p;
    const double u = e * 2.50662827463100050242 * exp(0.5 * z * z);
    return z - u / (1.0 + 0.5 * z * u);
}

/* FP32 Acklam with IEEE operations (reference restatement; PTX :166-205) */
static float acklam_f32(float u) {
    float q = u - 0.5f;
    if (fabsf(q) < 0.475749999284744263f) {
        float r = q * q;
        float num = fmaf(-3.969683028665376e+01f, r, 2.209460984245205e+02f);
        num = fmaf(num, r, -2.759285104469687e+02f);
        num = fmaf(num, r, 1.383577518672690e+02f);
        num = fmaf(num, r, -3.066479806614716e+01f);
        num = fmaf(num, r, 2.506628277459239e+00f);
        num = q * num;
        float den = fmaf(-5.447609879822406e+01f, r, 1.615858368580409e+02f);
        den = fmaf(den, r, -1.556989798598866e+02f);
        den = fmaf(den, r, 6.680131188771972e+01f);
        den = fmaf(den, r, -1.328068155288572e+01f);
        den = fmaf(den, r, 1.0f);
        return num / den;
    }
    int low = u < 0.5f;
    float p = low ? u : 1.0f - u;
    float s = sqrtf(-2.0f * logf(p));
    float num = fmaf(-7.784894002430293e-03f, s, -3.223964580411365e-01f);
    num = fmaf(num, s, -2.400758277161838e+00f);
    num = fmaf(num, s, -2.549732539343734e+00f);
    num = fmaf(num, s, 4.374664141464968e+00f);
    num = fmaf(num, s, 2.938163982698783e+00f);
    float den = fmaf(7.784695709041462e-03f, s, 3.224671290700398e-01f);
    den = fmaf(den, s, 2.445134137142996e+00f);
    den = fmaf(den, s, 3.754408661907416e+00f);
    den = fmaf(den, s, 1.0f);
    float z = num / den;
    return low ? z : -z;
}
float orc_acklam_f32(float u) { return acklam_f32(u); }

/* ------------------------------------------------------------------------- */
/* Observation log-density (PTX :414-451)                                     */
/* ------------------------------------------------------------------------- */
static double obs_logpdf_f64(double y, double h, double nu, double c_obs) {
    double eta2 = y * y * exp(-h);
    if (nu > 0.0) return c_obs - 0.5 * (nu + 1.0) * log1p(eta2 / nu) - 0.5 * h;
    return -0.91893853320467274178 - 0.5 * eta2 - 0.5 * h;
}
static double c_obs_of(double nu) {
    if (!(nu > 0.0)) return 0.0;
    return lgamma((nu + 1.0) / 2.0) - lgamma(nu / 2.0) - 0.5 * log(nu * 3.14159265358979323846);
}

/* ------------------------------------------------------------------------- */
/* FP64 filter (this build's semantics: increment log-likelihood, carried      */
/* weights on skipped ticks, resampling drawn from the host-formula U stream)  */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n_particles;
    float rho, sigma_z, mu, nu_obs;
    int seed;
    float ess_threshold;
    float nu_state;        /* Student-t state noise, 0 = Gaussian */
    float silverman;       /* Silverman jitter shrink after resampling, 0 = off (orc_f64_* only) */
} OrcConfig;

/*
 * Student-t state-noise scale sqrt(nu_state / chi2) of slot i at tick t, chi2
 * with k = round(nu_state) degrees of freedom drawn as -2 ln(U_1 ... U_{k/2})
 * (+ Z^2 when k is odd). Component c is draw t of the PCG32 stream with the
 * filter seed and increment ((c+1) << 33) | (2i+1). This build's counter-based
 * restatement of the reference's chi2 pre-pass (gpu_bpf/gpu_bpf_ptx_full.cu:
 * 392-400,574-583, PTX :394-404), evaluated in FP64.
 */
static uint32_t pcg_draw_inc(int seed, uint64_t inc, int t) {
    uint64_t s0 = ((uint64_t)(int64_t)seed * PCG_A + inc) * PCG_A + inc, At, Bt;
    orc_pcg32_jump((uint64_t)t, &At, &Bt);
    return orc_pcg32_output(At * s0 + Bt * inc);
}
double orc_tstate_scale(int seed, uint32_t i, int t, int nu_int, double nu_state) {
    const int pairs = nu_int >> 1;
    double l = 0.0;
    for (int c = 0; c < pairs; ++c) {
        uint64_t inc = ((uint64_t)(c + 1) << 33) | (uint64_t)(2u * i + 1u);
        l += log((double)orc_uniform(pcg_draw_inc(seed, inc, t)));
    }
    double chi2 = -2.0 * l;
    if (nu_int & 1) {
        uint64_t inc = ((uint64_t)(pairs + 1) << 33) | (uint64_t)(2u * i + 1u);
        double z = orc_icdf_f64((double)orc_uniform(pcg_draw_inc(seed, inc, t)));
        chi2 += z * z;
    }
    return sqrt(nu_state / chi2);
}
static int nu_int_of(double nu_state) { return nu_state > 0.0 ? (int)(nu_state + 0.5) : 0; }

static int ceil_log2_u(unsigned n) { int c = 0; while ((1ull << c) < (unsigned long long)n) ++c; return c; }

/*
 * The FP64 filter as an object stepped one tick at a time, so a checker can
 * follow a device run of any length in lock step (replaying each resampling
 * tick's ancestors as it comes) without holding T x N ancestors. The
 * per-particle loops run on OpenMP threads; every sum runs over the
 * particles in index order on one thread, so results do not depend on the
 * thread count.
 */
typedef struct {
    OrcConfig c;
    int N, nu_int, t, prev_res;
    int draw;              /* index of the next draw of every slot's PCG32 stream */
    double mu, rho, sig, nu, cobs, lse_prev, llr;
    uint64_t ustate;
    double *h, *hn, *lw, *lwc, *cdf;
} OrcF64;

void orc_f64_destroy(OrcF64* s) {
    if (!s) return;
    free(s->h); free(s->hn); free(s->lw); free(s->lwc); free(s->cdf);
    free(s);
}

OrcF64* orc_f64_create(const OrcConfig* c) {
    const int N = c->n_particles;
    if (N <= 0) return NULL;
    OrcF64* s = (OrcF64*)calloc(1, sizeof(OrcF64));
    if (!s) return NULL;
    s->c = *c;
    s->N = N;
    s->h = (double*)malloc(sizeof(double) * N);
    s->hn = (double*)malloc(sizeof(double) * N);
    s->lw = (double*)malloc(sizeof(double) * N);
    s->lwc = (double*)malloc(sizeof(double) * N);
    s->cdf = (double*)malloc(sizeof(double) * N);
    if (!s->h || !s->hn || !s->lw || !s->lwc || !s->cdf) { orc_f64_destroy(s); return NULL; }
    s->mu = c->mu; s->rho = c->rho; s->sig = c->sigma_z; s->nu = c->nu_obs; s->cobs = c_obs_of(s->nu);
    s->nu_int = nu_int_of((double)c->nu_state);
    const double sstat = sqrt(s->sig * s->sig / fmax(1.0 - s->rho * s->rho, 1e-6));
    double* h = s->h;
    double* lwc = s->lwc;
    const double mu = s->mu;
    const int seed = c->seed;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        float u = orc_uniform(orc_pcg32_draw_jump(seed, (uint32_t)i, 0));
        h[i] = mu + sstat * orc_icdf_f64((double)u);
        lwc[i] = 0.0;
    }
    s->ustate = orc_host_seed(seed);
    s->prev_res = 1;
    s->lse_prev = log((double)N);
    s->llr = 0.0;
    s->t = 0;
    s->draw = 1;           /* draw 0 is the initial particle */
    return s;
}

/*
 * One tick on observation y. anc: this tick's ancestors [N] used if the tick
 * resamples (NULL = own FP64 systematic resampling); flag: the resampling
 * decision to replay (-1 = own). out5 (may be NULL) receives
 * {dll, ll_ref, hmean, ess, resampled}.
 */
int orc_f64_tick(OrcF64* s, float y, const int32_t* anc, int flag, double* out5) {
    if (!s) return 1;
    const int N = s->N, t = s->t;
    const double mu = s->mu, rho = s->rho, sig = s->sig, nu = s->nu, cobs = s->cobs;
    double* h = s->h;
    double* lw = s->lw;
    double* lwc = s->lwc;
    double* cdf = s->cdf;
    const int seed = s->c.seed, nu_int = s->nu_int, prev_res = s->prev_res;
    const double nu_state = (double)s->c.nu_state;
    if (t > 0) {
        const int draw = s->draw++;
        uint64_t At, Bt;
        orc_pcg32_jump((uint64_t)draw, &At, &Bt);
#pragma omp parallel for schedule(static)
        for (int i = 0; i < N; ++i) {
            uint64_t s0, inc;
            orc_pcg32_init(seed, (uint32_t)i, &s0, &inc);
            float u = orc_uniform(orc_pcg32_output(At * s0 + Bt * inc));
            double eps = orc_icdf_f64((double)u);
            if (nu_int > 0) eps *= orc_tstate_scale(seed, (uint32_t)i, draw, nu_int, nu_state);
            h[i] = mu + rho * (h[i] - mu) + sig * eps;
        }
    }
    double M = -INFINITY;
#pragma omp parallel for schedule(static) reduction(max : M)
    for (int i = 0; i < N; ++i) {
        lw[i] = (prev_res ? 0.0 : lwc[i]) + obs_logpdf_f64((double)y, h[i], nu, cobs);
        if (lw[i] > M) M = lw[i];
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) cdf[i] = exp(lw[i] - M);
    double S = 0.0, Q = 0.0, H = 0.0;
    for (int i = 0; i < N; ++i) {
        const double e = cdf[i];
        S += e; Q += e * e; H += e * h[i];
        cdf[i] = S;
    }
    const double lse = M + log(S);
    const double d = lse - (prev_res ? log((double)N) : s->lse_prev);
    s->llr = (prev_res ? 0.0 : s->llr) + d;
    const double es = S * S / Q;
    const int res = flag >= 0 ? (flag != 0)
                              : ((s->c.ess_threshold <= 0.0f) || (es / (double)N < (double)s->c.ess_threshold));
    if (out5) { out5[0] = d; out5[1] = s->llr; out5[2] = H / S; out5[3] = es; out5[4] = (double)res; }
    if (res) {
        const uint32_t u23 = orc_host_pcg32(&s->ustate) >> 9;
        double* hn = s->hn;
        if (anc) {
            for (int i = 0; i < N; ++i) if (anc[i] < 0 || anc[i] >= N) return 3;
#pragma omp parallel for schedule(static)
            for (int i = 0; i < N; ++i) hn[i] = h[anc[i]];
        } else {
            const double step = S / (double)N, u0 = (double)u23 * 1.1920928955078125e-07;
            int j = 0;
            for (int i = 0; i < N; ++i) {
                double target = (u0 + (double)i) * step;
                while (j < N - 1 && !(cdf[j] > target)) ++j;
                hn[i] = h[j];
            }
        }
        s->hn = h; s->h = hn;
        s->prev_res = 1;
        if (s->c.silverman > 0.0f) {
            /* Silverman jitter (gpu_bpf_ptx_full.cu:708-738, PTX :846-1060): bandwidth from the
             * resampled particles' spread about this tick's filtered mean, noise from every slot's
             * next PCG32 draw, clamp to [mu - 8, mu + 8] */
            const double hm = H / S;
            double V = 0.0;
            for (int i = 0; i < N; ++i) V += (hn[i] - hm) * (hn[i] - hm);
            const double bw = (double)s->c.silverman * sqrt(V / (double)N) * 1.05922 * pow((double)N, -0.2);
            const int draw = s->draw++;
            uint64_t At, Bt;
            orc_pcg32_jump((uint64_t)draw, &At, &Bt);
#pragma omp parallel for schedule(static)
            for (int i = 0; i < N; ++i) {
                uint64_t s0, inc;
                orc_pcg32_init(seed, (uint32_t)i, &s0, &inc);
                const double z = orc_icdf_f64((double)orc_uniform(orc_pcg32_output(At * s0 + Bt * inc)));
                hn[i] = fmin(fmax(hn[i] + bw * z, mu - 8.0), mu + 8.0);
            }
        }
    } else {
        double* tmp = s->lwc; s->lwc = s->lw; s->lw = tmp;   /* the carried log-weights */
        s->lse_prev = lse;
        s->prev_res = 0;
    }
    s->t = t + 1;
    return 0;
}

/* Current particles h[0..N) of the object (after its last tick's resampling). */
int orc_f64_particles(const OrcF64* s, double* out) {
    if (!s || !out) return 1;
    memcpy(out, s->h, sizeof(double) * s->N);
    return 0;
}

/*
 * y[T]; anc_replay: [T][N] ancestors used on resampling ticks (NULL = own FP64
 * systematic resampling); flags_replay: [T] decisions to replay (NULL = own).
 * Outputs (each may be NULL): dll[T], ll_ref[T], hmean[T], ess[T], flags_out[T].
 */
int orc_filter_f64(const OrcConfig* c, const float* y, int T,
                   const int32_t* anc_replay, const int32_t* flags_replay,
                   double* dll, double* ll_ref, double* hmean, double* ess, int32_t* flags_out) {
    if (c->n_particles <= 0 || T < 0) return 1;
    OrcF64* s = orc_f64_create(c);
    if (!s) return 2;
    const int N = c->n_particles;
    for (int t = 0; t < T; ++t) {
        double o[5];
        const int rc = orc_f64_tick(s, y[t], anc_replay ? anc_replay + (size_t)t * N : NULL,
                                    flags_replay ? (flags_replay[t] != 0) : -1, o);
        if (rc) { orc_f64_destroy(s); return rc; }
        if (dll) dll[t] = o[0];
        if (ll_ref) ll_ref[t] = o[1];
        if (hmean) hmean[t] = o[2];
        if (ess) ess[t] = o[3];
        if (flags_out) flags_out[t] = (int32_t)o[4];
    }
    orc_f64_destroy(s);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* FP64 filter driven by given auxiliary noise (correlated-noise runs)         */
/* ------------------------------------------------------------------------- */
/*
 * The auxiliary noise of a correlated pseudo-marginal run (the reference's
 * CPMMH replay, smc2/smc2_rbpf_batch.cu:741-860, which stores the noise per
 * tick and particle and draws the resampling offset from a stored normal):
 * z[t*stride + i] (i < N) are the particles' standard normals at tick t
 * (tick 0: h_0 = mu + s_stat z), z[t*stride + npad] (npad = N rounded up to 4)
 * is the normal v_t of the tick's resampling offset u = Phi(v_t), taken on the
 * 23-bit grid (floor(Phi(v_t) 2^23) 2^-23). Before every resampling the
 * particles are put in ascending order (ties by slot), so resampling maps
 * nearby noise to nearby ancestors (the reference sorts the resampled
 * particles, cpmmh_sort, :836-845). anc_replay: [T][N] slot ancestors (the
 * slot before the sort) the run follows; NULL = its own FP64 systematic
 * resampling. flags_replay as orc_filter_f64. Outputs (each may be NULL): dll,
 * hmean, ess [T], flags_out [T], anc_out [T][N]: on resampling ticks the
 * oracle's own slot ancestors from that tick's particles (with anc_replay, a
 * lock-step check of the replayed ancestors).
 */
static const double* g_sort_key;
static int cmp_slot(const void* a, const void* b) {
    const int i = *(const int*)a, j = *(const int*)b;
    const double x = g_sort_key[i], y = g_sort_key[j];
    if (x < y) return -1;
    if (x > y) return 1;
    return (i > j) - (i < j);
}

int orc_filter_noise_f64(const OrcConfig* c, const float* y, int T, const float* z, int stride,
                         const int32_t* anc_replay, const int32_t* flags_replay,
                         double* dll, double* hmean, double* ess, int32_t* flags_out, int32_t* anc_out) {
    const int N = c->n_particles, npad = (N + 3) & ~3;
    if (N <= 0 || T < 0 || stride < npad + 1 || !z) return 1;
    double* h = (double*)malloc(sizeof(double) * N);
    double* hn = (double*)malloc(sizeof(double) * N);
    double* lw = (double*)malloc(sizeof(double) * N);
    double* lwc = (double*)malloc(sizeof(double) * N);
    double* cdf = (double*)malloc(sizeof(double) * N);
    int* ord = (int*)malloc(sizeof(int) * N);
    if (!h || !hn || !lw || !lwc || !cdf || !ord) {
        free(h); free(hn); free(lw); free(lwc); free(cdf); free(ord);
        return 2;
    }
    const double mu = c->mu, rho = c->rho, sig = c->sigma_z, nu = c->nu_obs, cobs = c_obs_of(nu);
    const double sstat = sqrt(sig * sig / fmax(1.0 - rho * rho, 1e-6));
    for (int i = 0; i < N; ++i) { h[i] = mu + sstat * (double)z[i]; lwc[i] = 0.0; }
    int prev_res = 1;
    double lse_prev = log((double)N);
    for (int t = 0; t < T; ++t) {
        const float* zt = z + (size_t)t * stride;
        if (t > 0)
            for (int i = 0; i < N; ++i) h[i] = mu + rho * (h[i] - mu) + sig * (double)zt[i];
        double M = -INFINITY;
        for (int i = 0; i < N; ++i) {
            lw[i] = (prev_res ? 0.0 : lwc[i]) + obs_logpdf_f64((double)y[t], h[i], nu, cobs);
            if (lw[i] > M) M = lw[i];
        }
        double S = 0.0, Q = 0.0, H = 0.0;
        for (int i = 0; i < N; ++i) {
            const double e = exp(lw[i] - M);
            S += e; Q += e * e; H += e * h[i];
        }
        const double lse = M + log(S);
        const double es = S * S / Q;
        if (dll) dll[t] = lse - (prev_res ? log((double)N) : lse_prev);
        if (hmean) hmean[t] = H / S;
        if (ess) ess[t] = es;
        const int res = flags_replay ? (flags_replay[t] != 0)
                                     : ((c->ess_threshold <= 0.0f) || (es / (double)N < (double)c->ess_threshold));
        if (flags_out) flags_out[t] = res;
        if (res) {
            int32_t* ao = anc_out ? anc_out + (size_t)t * N : NULL;
            if (!anc_replay || ao) {
                for (int i = 0; i < N; ++i) ord[i] = i;
                g_sort_key = h;
                qsort(ord, (size_t)N, sizeof(int), cmp_slot);
                double acc = 0.0;
                for (int p = 0; p < N; ++p) { acc += exp(lw[ord[p]] - M); cdf[p] = acc; }
                double u = 0.5 * erfc(-(double)zt[npad] * 0.70710678118654752440);
                double u23 = floor(u * 8388608.0);
                if (u23 > 8388607.0) u23 = 8388607.0;
                const double step = acc / (double)N, u0 = u23 * 1.1920928955078125e-07;
                int j = 0;
                for (int i = 0; i < N; ++i) {
                    const double target = (u0 + (double)i) * step;
                    while (j < N - 1 && !(cdf[j] > target)) ++j;
                    if (!anc_replay) hn[i] = h[ord[j]];
                    if (ao) ao[i] = ord[j];
                }
            }
            if (anc_replay) {
                const int32_t* a = anc_replay + (size_t)t * N;
                for (int i = 0; i < N; ++i) hn[i] = h[a[i]];
            }
            double* tmp = h; h = hn; hn = tmp;
            prev_res = 1;
        } else {
            memcpy(lwc, lw, sizeof(double) * N);
            lse_prev = lse;
            prev_res = 0;
        }
    }
    free(h); free(hn); free(lw); free(lwc); free(cdf); free(ord);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* FP64 auxiliary particle filter (gpu_bpf/gpu_bpf_ptx_full.cu:990-1175)      */
/* ------------------------------------------------------------------------- */
/*
 * Tick 0 is a bootstrap tick (weights from h_0, resample). Tick t >= 1:
 *   first stage   m_i = mu + rho (h_i - mu), v_i = p(y_t | m_i), resample the
 *                 pairs (h, m) by v (apf_first_stage, apf_resample_pair)
 *   second stage  h_i = m_i + sigma eps_i,t,  w_i = p(y_t | h_i) / p(y_t | m_i)
 *                 (apf_propagate_correct), mean and log-likelihood from w,
 *                 resample by w
 * The reference reports log mean w as BpfResult.log_lik (ll_ref here); the APF
 * estimate of log p(y_t | y_{1:t-1}) is log mean v + log mean w (dll here).
 * eps is draw t of slot i's PCG32 stream (Student-t scaled as the bootstrap
 * filter's); the reference draws it from cuRAND (apf_init_rng_k). Both stages
 * draw their uniform from the host stream, in order. anc1 / anc2: [T][N]
 * ancestors of the two stages to replay (anc1 row 0 unused), NULL = own FP64
 * systematic resampling. Outputs (each may be NULL): dll, ll_ref, hmean, ess [T].
 */
static void sys_resample_f64(int N, const double* cdf, double S, uint32_t u23, int32_t* a) {
    const double step = S / (double)N, u0 = (double)u23 * 1.1920928955078125e-07;
    int j = 0;
    for (int i = 0; i < N; ++i) {
        double target = (u0 + (double)i) * step;
        while (j < N - 1 && !(cdf[j] > target)) ++j;
        a[i] = j;
    }
}

int orc_apf_f64(const OrcConfig* c, const float* y, int T, const int32_t* anc1, const int32_t* anc2,
                double* dll, double* ll_ref, double* hmean, double* ess) {
    const int N = c->n_particles;
    if (N <= 0 || T < 0) return 1;
    double* h = (double*)malloc(sizeof(double) * N);
    double* m = (double*)malloc(sizeof(double) * N);
    double* hn = (double*)malloc(sizeof(double) * N);
    double* mn = (double*)malloc(sizeof(double) * N);
    double* lw = (double*)malloc(sizeof(double) * N);
    double* cdf = (double*)malloc(sizeof(double) * N);
    int32_t* a = (int32_t*)malloc(sizeof(int32_t) * N);
    if (!h || !m || !hn || !mn || !lw || !cdf || !a) {
        free(h); free(m); free(hn); free(mn); free(lw); free(cdf); free(a);
        return 2;
    }
    const double mu = c->mu, rho = c->rho, sig = c->sigma_z, nu = c->nu_obs, cobs = c_obs_of(nu);
    const int nu_int = nu_int_of((double)c->nu_state);
    const double sstat = sqrt(sig * sig / fmax(1.0 - rho * rho, 1e-6)), lnN = log((double)N);
    for (int i = 0; i < N; ++i) {
        float u = orc_uniform(orc_pcg32_draw_jump(c->seed, (uint32_t)i, 0));
        h[i] = mu + sstat * orc_icdf_f64((double)u);
    }
    uint64_t ustate = orc_host_seed(c->seed);
    for (int t = 0; t < T; ++t) {
        const double yt = (double)y[t];
        double lmv = 0.0;
        if (t > 0) {
            /* first stage */
            double M = -INFINITY;
            for (int i = 0; i < N; ++i) {
                m[i] = mu + rho * (h[i] - mu);
                lw[i] = obs_logpdf_f64(yt, m[i], nu, cobs);
                if (lw[i] > M) M = lw[i];
            }
            double S = 0.0;
            for (int i = 0; i < N; ++i) { S += exp(lw[i] - M); cdf[i] = S; }
            lmv = M + log(S) - lnN;
            uint32_t u23 = orc_host_pcg32(&ustate) >> 9;
            const int32_t* ar = anc1 ? anc1 + (size_t)t * N : a;
            if (!anc1) sys_resample_f64(N, cdf, S, u23, a);
            for (int i = 0; i < N; ++i) { hn[i] = h[ar[i]]; mn[i] = m[ar[i]]; }
            double* tmp = h; h = hn; hn = tmp;
            tmp = m; m = mn; mn = tmp;
            /* second stage: propagate from the resampled parents */
            uint64_t At, Bt;
            orc_pcg32_jump((uint64_t)t, &At, &Bt);
            for (int i = 0; i < N; ++i) {
                uint64_t s0, inc;
                orc_pcg32_init(c->seed, (uint32_t)i, &s0, &inc);
                float u = orc_uniform(orc_pcg32_output(At * s0 + Bt * inc));
                double eps = orc_icdf_f64((double)u);
                if (nu_int > 0) eps *= orc_tstate_scale(c->seed, (uint32_t)i, t, nu_int, (double)c->nu_state);
                h[i] = m[i] + sig * eps;
            }
        }
        double M = -INFINITY;
        for (int i = 0; i < N; ++i) {
            lw[i] = obs_logpdf_f64(yt, h[i], nu, cobs);
            if (t > 0) lw[i] -= obs_logpdf_f64(yt, m[i], nu, cobs);
            if (lw[i] > M) M = lw[i];
        }
        double S = 0.0, Q = 0.0, H = 0.0;
        for (int i = 0; i < N; ++i) {
            double e = exp(lw[i] - M);
            S += e; Q += e * e; H += e * h[i];
            cdf[i] = S;
        }
        const double lmw = M + log(S) - lnN;
        if (dll) dll[t] = lmv + lmw;
        if (ll_ref) ll_ref[t] = lmw;
        if (hmean) hmean[t] = H / S;
        if (ess) ess[t] = S * S / Q;
        uint32_t u23 = orc_host_pcg32(&ustate) >> 9;
        const int32_t* ar = anc2 ? anc2 + (size_t)t * N : a;
        if (!anc2) sys_resample_f64(N, cdf, S, u23, a);
        for (int i = 0; i < N; ++i) hn[i] = h[ar[i]];
        double* tmp = h; h = hn; hn = tmp;
    }
    free(h); free(m); free(hn); free(mn); free(lw); free(cdf); free(a);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Gradient with the ancestors held fixed                                     */
/* ------------------------------------------------------------------------- */
static double obs_dlogpdf_f64(double y, double h, double nu) {
    double q = y * y * exp(-h);
    if (nu > 0.0) return -0.5 + 0.5 * (nu + 1.0) * (q / nu) / (1.0 + q / nu);
    return -0.5 + 0.5 * q;
}

static double slot_normal(int seed, int i, int t) {
    return orc_icdf_f64((double)orc_uniform(orc_pcg32_draw_jump(seed, (uint32_t)i, t)));
}

/*
 * Every tick resamples; anc[t][i] is the parent (a slot of tick t) of slot i of
 * tick t+1. The loss is L = sum_t (LSE_t(lw) - ln N). Initial particles
 * h_0 = mu + sigma z_0 / sqrt(max(1-rho^2, 1e-6)) are differentiated too.
 * mode 0: forward-mode tangents dh/dtheta carried with the particles;
 * mode 1: reverse mode, lambda_t,j = W_t,j g_t(h_t,j) + rho sum_{i: anc[t][i]=j} lambda_t+1,i.
 * Outputs: *ll, grad[3], dll[T] (NULL allowed).
 */
int orc_grad_f64(int N, double mu, double rho, double sig, double nu, double nu_state, int seed, const float* y,
                 int T, const int32_t* anc, int mode, double* ll, double* grad, double* dll) {
    if (N <= 0 || T <= 0 || !anc) return 1;
    const double cobs = c_obs_of(nu), logn = log((double)N);
    const int nu_int = nu_int_of(nu_state);
#define STATE_EPS(i_, t_) (slot_normal(seed, (i_), (t_)) * \
                           (nu_int > 0 ? orc_tstate_scale(seed, (uint32_t)(i_), (t_), nu_int, nu_state) : 1.0))
    const double one_m = 1.0 - rho * rho, s2 = fmax(one_m, 1e-6), sd = sqrt(s2);
    const double sstat = sig / sd, dsr = one_m > 1e-6 ? sig * rho / (s2 * sd) : 0.0, dss = 1.0 / sd;
    double* z0 = (double*)malloc(sizeof(double) * N);
    double* lw = (double*)malloc(sizeof(double) * N);
    if (!z0 || !lw) { free(z0); free(lw); return 2; }
    for (int i = 0; i < N; ++i) z0[i] = slot_normal(seed, i, 0);
    double L = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
    int rc = 0;
    if (mode == 0) {
        double* st = (double*)malloc(sizeof(double) * 8 * (size_t)N);   /* h, d0, d1, d2 ping-pong */
        if (!st) { rc = 2; goto out; }
        double *h = st, *d0 = st + N, *d1 = st + 2 * N, *d2 = st + 3 * N;
        double *hn = st + 4 * N, *e0 = st + 5 * N, *e1 = st + 6 * N, *e2 = st + 7 * N;
        for (int i = 0; i < N; ++i) { h[i] = mu + sstat * z0[i]; d0[i] = 1.0; d1[i] = z0[i] * dsr; d2[i] = z0[i] * dss; }
        for (int t = 0; t < T; ++t) {
            if (t > 0) {
                const int32_t* a = anc + (size_t)(t - 1) * N;
                for (int i = 0; i < N; ++i) {
                    const int p = a[i];
                    const double eps = STATE_EPS(i, t);
                    hn[i] = mu + rho * (h[p] - mu) + sig * eps;
                    e0[i] = (1.0 - rho) + rho * d0[p];
                    e1[i] = (h[p] - mu) + rho * d1[p];
                    e2[i] = eps + rho * d2[p];
                }
                double* tmp;
                tmp = h; h = hn; hn = tmp; tmp = d0; d0 = e0; e0 = tmp;
                tmp = d1; d1 = e1; e1 = tmp; tmp = d2; d2 = e2; e2 = tmp;
            }
            double M = -INFINITY;
            for (int i = 0; i < N; ++i) { lw[i] = obs_logpdf_f64((double)y[t], h[i], nu, cobs); if (lw[i] > M) M = lw[i]; }
            double S = 0.0, G0 = 0.0, G1 = 0.0, G2 = 0.0;
            for (int i = 0; i < N; ++i) {
                const double e = exp(lw[i] - M), g = obs_dlogpdf_f64((double)y[t], h[i], nu);
                S += e; G0 += e * g * d0[i]; G1 += e * g * d1[i]; G2 += e * g * d2[i];
            }
            const double d = M + log(S) - logn;
            if (dll) dll[t] = d;
            L += d; g0 += G0 / S; g1 += G1 / S; g2 += G2 / S;
        }
        free(st);
    } else {
        double* H = (double*)malloc(sizeof(double) * (size_t)T * N);
        double* lse = (double*)malloc(sizeof(double) * T);
        double* lam = (double*)calloc((size_t)N, sizeof(double));
        double* lamn = (double*)calloc((size_t)N, sizeof(double));
        double* cs = (double*)malloc(sizeof(double) * N);
        if (!H || !lse || !lam || !lamn || !cs) { free(H); free(lse); free(lam); free(lamn); free(cs); rc = 2; goto out; }
        for (int i = 0; i < N; ++i) H[i] = mu + sstat * z0[i];
        for (int t = 0; t < T; ++t) {
            double* h = H + (size_t)t * N;
            if (t > 0) {
                const int32_t* a = anc + (size_t)(t - 1) * N;
                const double* hp = H + (size_t)(t - 1) * N;
                for (int i = 0; i < N; ++i) h[i] = mu + rho * (hp[a[i]] - mu) + sig * STATE_EPS(i, t);
            }
            double M = -INFINITY, S = 0.0;
            for (int i = 0; i < N; ++i) { lw[i] = obs_logpdf_f64((double)y[t], h[i], nu, cobs); if (lw[i] > M) M = lw[i]; }
            for (int i = 0; i < N; ++i) S += exp(lw[i] - M);
            lse[t] = M + log(S);
            if (dll) dll[t] = lse[t] - logn;
            L += lse[t] - logn;
        }
        double acs = 0.0, acsh = 0.0, aeps = 0.0;
        for (int t = T - 1; t >= 0; --t) {
            const double* h = H + (size_t)t * N;
            for (int j = 0; j < N; ++j) cs[j] = 0.0;
            if (t < T - 1) {
                const int32_t* a = anc + (size_t)t * N;
                for (int i = 0; i < N; ++i) {
                    cs[a[i]] += lamn[i];
                    aeps += lamn[i] * STATE_EPS(i, t + 1);
                }
            }
            for (int j = 0; j < N; ++j) {
                const double W = exp(obs_logpdf_f64((double)y[t], h[j], nu, cobs) - lse[t]);
                lam[j] = W * obs_dlogpdf_f64((double)y[t], h[j], nu) + rho * cs[j];
                acs += cs[j];
                acsh += cs[j] * (h[j] - mu);
            }
            double* tmp = lam; lam = lamn; lamn = tmp;
        }
        double al0 = 0.0, al0z = 0.0;
        for (int j = 0; j < N; ++j) { al0 += lamn[j]; al0z += lamn[j] * z0[j]; }
        g0 = (1.0 - rho) * acs + al0;
        g1 = acsh + al0z * dsr;
        g2 = aeps + al0z * dss;
        free(H); free(lse); free(lam); free(lamn); free(cs);
    }
    if (ll) *ll = L;
    if (grad) { grad[0] = g0; grad[1] = g1; grad[2] = g2; }
out:
    free(z0); free(lw);
    return rc;
#undef STATE_EPS
}

/* ------------------------------------------------------------------------- */
/* Exact mirror of the GPU fixed-point systematic resampling                 */
/* ------------------------------------------------------------------------- */
/*
 * w[N]: tile-relative FP32 weights in [0,1]; nexp[G]: power-of-two exponent of
 * each 4096-particle tile; u23: 23-bit uniform. Element mass (tile frame)
 * I_j = floor(w_j 2^50); tile mass in the global frame Ehat_k = E_k >> r_k with
 * r_k = nM - n_k + 50 - Fg, Fg = min(50, 62 - ceil(log2 N)); global CDF
 * C_j = P_k + (L_j >> r_k) with L_j the tile-local inclusive prefix; targets
 * t_i = base + i*delta, delta = floor(T/N), base = floor(u23*delta/2^23);
 * ancestor a_i = min{ j : C_j > t_i }.
 */
int orc_resample_fixed(int N, const float* w, const int32_t* nexp, uint32_t u23, int32_t* anc) {
    if (N <= 0) return 1;
    const int G = (N + TILE - 1) / TILE;
    int nM = NK_EMPTY;
    for (int k = 0; k < G; ++k) if (nexp[k] > nM) nM = nexp[k];
    if (nM == NK_EMPTY) return 2;
    int Fg = 62 - ceil_log2_u((unsigned)N);
    if (Fg > FIXF) Fg = FIXF;
    uint64_t* C = (uint64_t*)malloc(sizeof(uint64_t) * N);
    if (!C) return 3;
    uint64_t P = 0;
    for (int k = 0; k < G; ++k) {
        const int j0 = k * TILE, j1 = (j0 + TILE < N) ? j0 + TILE : N;
        const int r = (nexp[k] == NK_EMPTY) ? 64 : nM - nexp[k] + FIXF - Fg;
        uint64_t L = 0;
        for (int j = j0; j < j1; ++j) {
            L += (uint64_t)(w[j] * 1125899906842624.0f);
            C[j] = P + (r >= 64 ? 0ull : (L >> r));
        }
        P += (r >= 64 ? 0ull : (L >> r));
    }
    const uint64_t T = P;
    uint64_t delta = T / (uint64_t)N;
    if (delta == 0) delta = 1;
    const unsigned __int128 prod = (unsigned __int128)u23 * delta;
    const uint64_t base = (uint64_t)(prod >> 23);
    int j = 0;
    for (int i = 0; i < N; ++i) {
        const uint64_t t = base + (uint64_t)i * delta;
        while (j < N - 1 && !(C[j] > t)) ++j;
        anc[i] = j;
    }
    free(C);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* FP32 restatement of the reference tick loop (CPU baseline)                 */
/* ------------------------------------------------------------------------- */
/*
 * Follows gpu_bpf_step_async (gpu_bpf_ptx_full.cu:550-748) with 1 band,
 * nu_state = 0, Silverman off, no learning, one stage per helper:
 *   ref_propagate_weight  propagate_weight (PTX :231-458) and the accumulation
 *                         of skipped ticks (:601-604); returns max(lw) (PTX :488-576)
 *   ref_normalise         exp_sub / sum / scale_wh / sum(wh) / compute_loglik
 *                         (PTX :586-775) and sum(w^2) for the ESS (:656-685)
 *   ref_resample          inclusive scan + systematic resample (:691-706, PTX :782-842)
 * Transcendentals use libm in FP32 where the PTX uses approximate MUFU ops.
 */
static const float kRefLog2e = 1.44269504088896340736f, kRefLn2 = 0.693147180559945309417f;

static float ref_propagate_weight(int N, uint64_t* rng, float* h, float* lw, const float* lwp, int do_prop, int acc,
                                  float rho, float sigma_z, float mu, float nu_obs, float c_obs, float yt) {
    float mx = -1e30f;
#pragma omp parallel for schedule(static) reduction(max : mx)
    for (int i = 0; i < N; ++i) {
        float hi = h[i];
        if (do_prop) {
            uint64_t s = rng[2 * (size_t)i], inc = rng[2 * (size_t)i + 1];
            uint32_t o = orc_pcg32_output(s);
            rng[2 * (size_t)i] = s * PCG_A + inc;
            float eps = acklam_f32(orc_uniform(o));
            float dev = rho * (hi - mu);
            hi = fmaf(sigma_z, eps, mu + dev);
            h[i] = hi;
        }
        float eta = yt * exp2f(hi * -0.5f * kRefLog2e);
        float l;
        if (nu_obs > 0.0f) {
            float ta = eta * eta / nu_obs + 1.0f;
            l = fmaf(-0.5f, hi, c_obs + (-(nu_obs + 1.0f) * 0.5f) * (log2f(ta) * kRefLn2));
        } else {
            l = fmaf(-0.5f, hi, fmaf(-0.5f, eta * eta, -0.918938517570496f));
        }
        if (acc) l += lwp[i];
        lw[i] = l;
        if (l > mx) mx = l;
    }
    return mx;
}

/* w = normalised weights; out: h_mean, loglik (the reference BpfResult), sum of w^2 */
static void ref_normalise(int N, const float* lw, float mx, const float* h, float* w,
                          float* hmean, float* loglik, float* sumsq) {
    float sw = 0.0f;
#pragma omp parallel for schedule(static) reduction(+ : sw)
    for (int i = 0; i < N; ++i) { w[i] = exp2f((lw[i] - mx) * kRefLog2e); sw += w[i]; }
    const float inv = 1.0f / sw;
    float hest = 0.0f, sw2 = 0.0f;
#pragma omp parallel for schedule(static) reduction(+ : hest, sw2)
    for (int i = 0; i < N; ++i) { w[i] *= inv; hest += w[i] * h[i]; sw2 += w[i] * w[i]; }
    float r = sw / (float)N;
    if (r < 7.27150555e-31f) r = 7.27150555e-31f;
    *hmean = hest;
    *loglik = log2f(r) * kRefLn2 + mx;
    *sumsq = sw2;
}

/* FP32 inclusive scan of w into cdf (chunked over threads; part holds nchunk+1
 * floats), then anc[i] = lower bound of u + i/N (wrapped below 1) in cdf. */
static void ref_resample(int N, const float* w, float* cdf, float* part, float u, int32_t* anc) {
#pragma omp parallel
    {
        int tid = 0, nt = 1;
#ifdef _OPENMP
        tid = omp_get_thread_num(); nt = omp_get_num_threads();
#endif
        int a = (int)((long long)N * tid / nt), b = (int)((long long)N * (tid + 1) / nt);
        float acc2 = 0.0f;
        for (int i = a; i < b; ++i) { acc2 += w[i]; cdf[i] = acc2; }
        part[tid + 1] = acc2;
#pragma omp barrier
#pragma omp single
        {
            part[0] = 0.0f;
            for (int k = 1; k <= nt; ++k) part[k] += part[k - 1];
        }
        float off = part[tid];
        for (int i = a; i < b; ++i) cdf[i] += off;
    }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        float target = (float)i / (float)N + u;
        if (target >= 1.0f) target -= 1.0f;
        int lo = 0, hi = N - 1;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (cdf[mid] < target) lo = mid + 1; else hi = mid;
        }
        anc[i] = lo;
    }
}

/* bpf_init_rng + bpf_init_particles (PTX :74-91, :103-218; std_stat as
 * gpu_bpf_ptx_full.cu:430): rng [state, inc] after draw 0, h = mu + std_stat z_0 */
static void ref_init(int N, int seed, float rho, float sigma_z, float mu, uint64_t* rng, float* h) {
    const float std_stat = sqrtf((sigma_z * sigma_z) / fmaxf(1.0f - rho * rho, 1e-6f));
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) {
        uint64_t s, inc;
        orc_pcg32_init(seed, (uint32_t)i, &s, &inc);
        uint32_t o = orc_pcg32_output(s);
        s = s * PCG_A + inc;
        h[i] = fmaf(std_stat, acklam_f32(orc_uniform(o)), mu);
        rng[2 * (size_t)i] = s;
        rng[2 * (size_t)i + 1] = inc;
    }
}

static int ref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/*
 * hmean/loglik receive the reference BpfResult of every tick.
 */
int orc_ref_run(int N, float rho, float sigma_z, float mu, float nu_obs, int seed, float ess_threshold,
                const float* y, int T, float* hmean, float* loglik, int nthreads, int* resample_count) {
    if (N <= 0 || T < 0) return 1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    uint64_t* rng = (uint64_t*)malloc(sizeof(uint64_t) * 2 * (size_t)N);
    float* h = (float*)malloc(sizeof(float) * N);
    float* h2 = (float*)malloc(sizeof(float) * N);
    float* lw = (float*)malloc(sizeof(float) * N);
    float* lwp = (float*)malloc(sizeof(float) * N);
    float* w = (float*)malloc(sizeof(float) * N);
    float* cdf = (float*)malloc(sizeof(float) * N);
    int32_t* anc = (int32_t*)malloc(sizeof(int32_t) * N);
    float* part = (float*)malloc(sizeof(float) * (ref_max_threads() + 1));
    if (!rng || !h || !h2 || !lw || !lwp || !w || !cdf || !anc || !part) {
        free(rng); free(h); free(h2); free(lw); free(lwp); free(w); free(cdf); free(anc); free(part);
        return 2;
    }
    const float c_obs = (nu_obs > 0.0f) ? (float)c_obs_of(nu_obs) : 0.0f;
    ref_init(N, seed, rho, sigma_z, mu, rng, h);
    uint64_t host_rng = orc_host_seed(seed);
    int did_resample = 1, count = 0;
    for (int t = 0; t < T; ++t) {
        const float mx = ref_propagate_weight(N, rng, h, lw, lwp, t > 0, (t > 0) && !did_resample,
                                              rho, sigma_z, mu, nu_obs, c_obs, y[t]);
        float sw2;
        ref_normalise(N, lw, mx, h, w, &hmean[t], &loglik[t], &sw2);
        int do_res = 1;
        if (ess_threshold > 0.0f) {
            float essv = 1.0f / fmaxf(sw2, 1e-30f);
            do_res = (essv / (float)N) < ess_threshold;
        }
        if (do_res) {
            did_resample = 1;
            ++count;
            const float u = (float)(orc_host_pcg32(&host_rng) >> 9) * (1.0f / 8388608.0f) / (float)N;
            ref_resample(N, w, cdf, part, u, anc);
#pragma omp parallel for schedule(static)
            for (int i = 0; i < N; ++i) h2[i] = h[anc[i]];
            float* tmp = h; h = h2; h2 = tmp;
        } else {
            did_resample = 0;
            memcpy(lwp, lw, sizeof(float) * N);
        }
    }
    if (resample_count) *resample_count = count;
    free(rng); free(h); free(h2); free(lw); free(lwp); free(w); free(cdf); free(anc); free(part);
    return 0;
}

/* The reference's initial state: PCG32 [state, inc] x N after draw 0 and the initial particles. */
int orc_ref_init(int N, int seed, float rho, float sigma_z, float mu, uint64_t* rng, float* h) {
    if (N <= 0) return 1;
    ref_init(N, seed, rho, sigma_z, mu, rng, h);
    return 0;
}

/*
 * One reference tick on given particles, for a lock-step comparison with the
 * reference run on a GPU: rng [state, inc] x N is advanced in place when
 * propagate != 0, h holds the previous particles on entry and the propagated
 * ones on return, w the normalised weights; out3 = h_mean, loglik, 1/sum(w^2).
 * No carried weights (the always-resample schedule).
 */
int orc_ref_tick(int N, uint64_t* rng, float* h, float rho, float sigma_z, float mu, float nu_obs, float y,
                 int propagate, float* w, float* out3) {
    if (N <= 0) return 1;
    float* lw = (float*)malloc(sizeof(float) * N);
    if (!lw) return 2;
    const float c_obs = (nu_obs > 0.0f) ? (float)c_obs_of(nu_obs) : 0.0f;
    const float mx = ref_propagate_weight(N, rng, h, lw, NULL, propagate, 0, rho, sigma_z, mu, nu_obs, c_obs, y);
    float sw2;
    ref_normalise(N, lw, mx, h, w, &out3[0], &out3[1], &sw2);
    out3[2] = 1.0f / fmaxf(sw2, 1e-30f);
    free(lw);
    return 0;
}

/* The reference's systematic resampling of normalised FP32 weights with offset u = U/N. */
int orc_ref_resample(int N, const float* w, float u, int32_t* anc) {
    if (N <= 0) return 1;
    float* cdf = (float*)malloc(sizeof(float) * N);
    float* part = (float*)malloc(sizeof(float) * (ref_max_threads() + 1));
    if (!cdf || !part) { free(cdf); free(part); return 2; }
    ref_resample(N, w, cdf, part, u, anc);
    free(cdf); free(part);
    return 0;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------------------------
 * Host restatement of the FP32 child-count estimate of the resampling kernels (pass 2 and the
 * fused small-filter tick in bootstrap-particle-filter-in-ptx_b200/csrc/bpf_plain.cu), used to
 * check the error bound that decides when the estimate may be used instead of the exact count.
 *
 * For a run of n <= 16 weights w_j in [0, 1] (FP32, tile frame), a relative threshold R0 and a
 * spacing D (u64 fixed point, 2^-50 units), the exact running count is
 *   c_j = #{m >= 0 : R0 + m D <= l_j},  l_j = sum_{i <= j} floor(w_i 2^50),
 * and the kernels estimate it as floor(x) + 1 (0 for x < 0) with x = fmaf(lf_j, 1/Dw, -R0/Dw) from
 * the FP32 running sum lf_j, trusting the estimate only when x is farther than the run's bound from
 * an integer. The operations below are the kernels' own, in their order (this file is compiled
 * without floating-point contraction). bound_scale multiplies the bound: 1 is the kernels' bound;
 * a smaller value plants a mistake that the check must find.
 * Returns the number of elements declared safe whose estimate differs from the exact count;
 * *n_safe and *n_recount count the two kinds of elements.
 * ------------------------------------------------------------------------------------------ */
long long orc_count_estimate_run(const float* w, int n, uint64_t R0, uint64_t D, float bound_scale,
                                 long long* n_safe, long long* n_recount) {
    long long bad = 0;
    float lfT = 0.0f;
    for (int j = 0; j < n; ++j) lfT += w[j];
    const float R0w = (float)R0 * 0x1p-50f;
    const float invDw = 1.0f / ((float)D * 0x1p-50f);
    const float R0x = R0w * invDw;
    const float eL = 0x1p-18f * invDw, e0 = fmaf(R0w, eL, 0x1p-44f * invDw);
    const float xT = fmaf(lfT, invDw, -R0x);
    float err = fmaf(lfT, eL, fmaf(fmaxf(fabsf(xT), R0x), 0x1p-21f, e0));
    err *= bound_scale;
    if (!(xT < 0x1p22f)) err = 1.0f;
    const float err_hi = 1.0f - err;
    float lf = 0.0f;
    uint64_t l = 0;
    for (int j = 0; j < n; ++j) {
        lf += w[j];
        l += (uint64_t)(w[j] * 0x1p50f);
        const float x = fmaf(lf, invDw, -R0x);
        const float fl = floorf(x);
        const float fr = x - fl;
        const int safe = (fr > err && fr < err_hi);
        const float v = fl + 0x1p23f;
        int32_t bits;
        memcpy(&bits, &v, sizeof bits);
        int c_est = bits - 0x4AFFFFFF;
        if (c_est < 0) c_est = 0;
        const uint64_t c = (l < R0) ? 0u : (l - R0) / D + 1u;
        if (safe) {
            ++*n_safe;
            if ((uint64_t)c_est != c) ++bad;
        } else {
            ++*n_recount;
        }
    }
    return bad;
}

static uint64_t orc_splitmix(uint64_t* s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* n_runs random runs of n weights each (mode 0: weights spread over [0, 1] with tiny values,
 * zeros and exact ones mixed in, thresholds and spacings over many magnitudes; mode 1: the
 * thresholds placed on target boundaries: the m-th target sits exactly on, or one unit either side of, an element's
 * running sum). out3 = {violations, safe elements, recounted elements}. */
void orc_count_estimate_fuzz(uint64_t seed, long long n_runs, int n, int mode, float bound_scale, long long* out3) {
    uint64_t s = seed;
    long long bad = 0, n_safe = 0, n_rec = 0;
    float w[16];
    if (n < 1) n = 1;
    if (n > 16) n = 16;
    for (long long r = 0; r < n_runs; ++r) {
        /* weights */
        const int kind = (mode == 2) ? 0 : (int)(orc_splitmix(&s) % 5);
        for (int j = 0; j < n; ++j) {
            const uint64_t u = orc_splitmix(&s);
            float v;
            switch (kind) {
                case 0: v = (float)((u >> 40) * 0x1p-24); break;                               /* uniform */
                case 1: v = ldexpf((float)((u >> 41) | 1u) * 0x1p-23f, -(int)((u >> 8) % 60)); break;   /* 2^-60 .. 1 */
                case 2: v = (u & 1) ? 1.0f : 0.0f; break;                                        /* ones and zeros */
                case 3: v = ldexpf(1.0f, -(int)((u >> 8) % 52)); break;                          /* powers of two */
                default: v = 1.0f - (float)((u >> 45) * 0x1p-19); break;                          /* near one */
            }
            if (v > 1.0f) v = 1.0f;
            if (v < 0x1p-126f) v = 0.0f;                                                        /* flushed */
            w[j] = v;
        }
        uint64_t l[16], acc = 0;
        for (int j = 0; j < n; ++j) { acc += (uint64_t)(w[j] * 0x1p50f); l[j] = acc; }
        /* spacing: 1 .. 2^55, log-uniform; mode 2: about one target per weight (the mean weight
           times 2^50, within a factor of two either way), as in a filter's resampling */
        const int dexp = (int)(orc_splitmix(&s) % 56);
        uint64_t D = (orc_splitmix(&s) >> (64 - dexp - 1)) | (1ull << dexp);
        if (mode == 2) {
            const double mean = (double)acc / n;
            D = (uint64_t)(mean * (0.5 + 1.5 * (double)(orc_splitmix(&s) >> 11) * 0x1p-53));
        }
        if (D == 0) D = 1;
        if (D > (1ull << 55)) D = 1ull << 55;
        uint64_t R0;
        if (mode == 0 || mode == 2) {
            R0 = 1 + orc_splitmix(&s) % (D > (1ull << 54) ? D : 2 * D);                         /* 1 .. 2D */
            if (mode == 0 && (orc_splitmix(&s) & 31) == 0) R0 = 1ull << 55;                     /* no target */
        } else {
            /* a boundary: R0 + m D = l_j + delta for a random element j, m and delta in {-1, 0, 1} */
            const int j = (int)(orc_splitmix(&s) % n);
            const uint64_t lj = l[j];
            const uint64_t m = lj ? (lj - 1) / D : 0;                                              /* lj - m D in [1, D] */
            const int delta = (int)(orc_splitmix(&s) % 3) - 1;
            int64_t r0 = (int64_t)(lj - m * D) + delta;
            if (r0 < 1) r0 = 1;
            R0 = (uint64_t)r0;
        }
        bad += orc_count_estimate_run(w, n, R0, D, bound_scale, &n_safe, &n_rec);
    }
    out3[0] = bad; out3[1] = n_safe; out3[2] = n_rec;
}
