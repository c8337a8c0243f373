/*
 * gpu_bpf.h — C ABI of the B200 (sm_100a) bootstrap particle filter for the
 * stochastic-volatility model.
 *
 * Drop-in for the reference header gpu_bpf/gpu_bpf.cuh (Tugbars/Bootstrap-
 * Particle-Filter-in-PTX), whose PTX edition gpu_bpf/gpu_bpf_full.cuh declares
 * the same functions. Every reference entry point keeps its name, argument
 * list and meaning; each declaration below cites the line it replaces.
 * Entries marked "addition" have no reference counterpart.
 *
 * Model: h_t = mu + rho*(h_{t-1}-mu) + sigma_z*eps_t,  y_t = exp(h_t/2)*eta_t.
 * Library: libgpubpf.so (plain C ABI, no CUDA or torch types in signatures;
 * `void* stream` is a cudaStream_t).
 */
#ifndef GPU_BPF_H
#define GPU_BPF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes (addition: the reference reports no errors)                   */
/* ------------------------------------------------------------------------ */
#define BPF_OK               0
#define BPF_ERR_ARG          1  /* invalid argument (N<=0, |rho|>=1, sigma<=0, non-finite y, NULL) */
#define BPF_ERR_CUDA         2  /* a CUDA runtime call failed                                       */
#define BPF_ERR_ALLOC        3  /* device or pinned allocation failed                               */
#define BPF_ERR_UNSUPPORTED  4  /* option outside this build (multi-band proposals)                   */
#define BPF_ERR_STATE        5  /* call not valid in the filter's current state                     */
#define BPF_ERR_DEGENERATE   6  /* every particle weight underflowed on a tick                      */
#define BPF_ERR_NODEVICE     7  /* no CUDA device / kernel image for this GPU                       */

/* Per-tick result, reference layout (gpu_bpf/gpu_bpf.cuh:21-24). */
typedef struct {
    float h_mean;   /* filtered mean E[h_t | y_{1:t}]                                */
    float log_lik;  /* log p(y_t | y_{1:t-1}) (see gpu_bpf_set_loglik_semantics)     */
} BpfResult;

/* Full per-tick record (addition). 40 bytes. */
typedef struct {
    double  dloglik;        /* increment log p(y_t | y_{1:t-1}), FP64                         */
    double  loglik_ref;     /* reference value: log-evidence since the last resample           */
    double  loglik_total;   /* FP64 running sum of dloglik since create                        */
    float   h_mean;         /* filtered mean                                                   */
    float   ess;            /* effective sample size 1/sum(W^2) before resampling             */
    int32_t resampled;      /* 1 if this tick resampled                                        */
    int32_t tick;           /* tick index (0-based)                                            */
} BpfTickRecord;

/*
 * Filter state. The reference struct is public (gpu_bpf/gpu_bpf.cuh:30-54;
 * gpu_bpf_full.cuh:80-126) and its tests read or write some fields
 * directly, so those fields keep their names and meaning here. Device
 * buffers live behind `impl`.
 *   rho, sigma_z, mu   may be changed between ticks (read at every step)
 *   ess_threshold      0 = always resample, else resample iff ESS/N < it
 *   silverman_shrink   > 0: Silverman jitter after every resampling, as the
 *                      reference's PTX edition (gpu_bpf_ptx_full.cu:708-738):
 *                      h += bw z clamped to [mu-8, mu+8], bw = shrink * 1.05922
 *                      * N^-0.2 * std of the resampled particles about the
 *                      tick's filtered mean, z from each slot's next PCG32
 *                      draw (so the next propagation takes the draw after
 *                      it, as in the reference); 0 (default) = off
 *   did_resample, resample_count, timestep, last_h_est: refreshed whenever a
 *                      result is read back (gpu_bpf_step / get_result)
 */
typedef struct {
    int    n_particles;
    float  rho, sigma_z, mu, nu_state, nu_obs;
    float  silverman_shrink;
    float  ess_threshold;
    int    did_resample;
    int    resample_count;
    int    timestep;
    float  last_h_est;
    void*  stream;          /* cudaStream_t owned by the filter */
    void*  impl;            /* opaque */
} GpuBpfState;

/* ---- Reference API ------------------------------------------------------- */

/* gpu_bpf/gpu_bpf.cuh:56-57. Seeds the per-slot PCG32 streams and draws h_0
 * from N(mu, sigma_z^2/max(1-rho^2,1e-6)) (gpu_bpf_ptx_full.cu:340-438).
 * Default ess_threshold 0.5 (PTX edition, gpu_bpf_ptx_full.cu:356).
 * Returns NULL on failure (reason in gpu_bpf_last_error()). nu_state > 0 selects
 * Student-t state noise eps = z sqrt(nu_state / chi2), chi2 with round(nu_state)
 * degrees of freedom (the reference's law, drawn from counter-based PCG32 streams
 * instead of a cuRAND pre-pass); 0 < nu_state < 0.5 is rejected (BPF_ERR_ARG). */
GpuBpfState* gpu_bpf_create(int n_particles, float rho, float sigma_z, float mu,
                            float nu_state, float nu_obs, int seed);

/* gpu_bpf/gpu_bpf.cuh:58 (gpu_bpf_ptx_full.cu:444-463). NULL is a no-op. */
void gpu_bpf_destroy(GpuBpfState* state);

/* gpu_bpf/gpu_bpf.cuh:59 (gpu_bpf_ptx_full.cu:764-771): one tick, synchronous.
 * Returns as soon as the tick's result is final (it waits for the tick's record in
 * host-mapped memory); the tick's resampling may still be running on state->stream,
 * ordered before any later work there, and every accessor that reads the particles,
 * ancestors or device state waits for it. On error returns {NaN, NaN} and sets
 * gpu_bpf_last_error(); a device-side error detected by that resampling is reported
 * by the next call that reads a result. */
BpfResult gpu_bpf_step(GpuBpfState* state, float y_t);

/* gpu_bpf/gpu_bpf.cuh:60 (gpu_bpf_ptx_full.cu:550-748): enqueue one tick on
 * state->stream. Never synchronises (the resampling decision is taken on the
 * device). */
void gpu_bpf_step_async(GpuBpfState* state, float y_t);

/* gpu_bpf/gpu_bpf.cuh:61 (gpu_bpf_ptx_full.cu:754-762): result of the last
 * enqueued tick; waits for its result (as gpu_bpf_step). */
BpfResult gpu_bpf_get_result(GpuBpfState* state);

/* gpu_bpf/gpu_bpf.cuh:63-67 (gpu_bpf_ptx_full.cu:834-852): run a filter over a
 * series, RMSE of h_mean vs true_h after the first 100 ticks. Returns NaN on
 * error. */
double gpu_bpf_run_rmse(const double* returns, const double* true_h, int n_ticks,
                        int n_particles, float rho, float sigma_z, float mu,
                        float nu_state, float nu_obs, int seed);

/* gpu_bpf/gpu_bpf.cuh:71-72. Only the single-band identity configuration
 * (n_bands == 1, scale 1) is accepted; anything else records
 * BPF_ERR_UNSUPPORTED. */
void gpu_bpf_set_bands(int n_particles, int n_bands, const float* fracs, const float* scales);

/* gpu_bpf/gpu_bpf.cuh:75-79. Records BPF_ERR_UNSUPPORTED. */
void gpu_bpf_set_adaptive_bands(int n_particles,
                                const float* calm_fracs,  const float* calm_scales,  int calm_nb,
                                const float* alert_fracs, const float* alert_scales, int alert_nb,
                                const float* panic_fracs, const float* panic_scales, int panic_nb,
                                float thresh_alert, float thresh_panic);

/* gpu_bpf/gpu_bpf.cuh:84 (gpu_bpf_ptx_full.cu:858-860; no clamping, as the PTX edition). */
void gpu_bpf_set_ess_threshold(GpuBpfState* state, float threshold);

/* gpu_bpf/gpu_bpf.cuh:85 (gpu_bpf_ptx_full.cu:862-864). Waits for enqueued ticks. */
int gpu_bpf_get_resample_count(GpuBpfState* state);

/* gpu_bpf/gpu_bpf_full.cuh:206-230 (gpu_bpf_ptx_full.cu:802-828): parameter
 * access between ticks. set_rho clamps to (0.001, 0.999) like the reference; both
 * setters restart the online-learning step-size schedule. */
float gpu_bpf_get_mu(GpuBpfState* state);
float gpu_bpf_get_rho(GpuBpfState* state);
void  gpu_bpf_set_mu(GpuBpfState* state, float mu);
void  gpu_bpf_set_rho(GpuBpfState* state, float rho);

/* gpu_bpf/gpu_bpf_full.cuh:176-204 (gpu_bpf_ptx_full.cu:469-544,777-800): online
 * learning of mu (and of rho after enable_rho_learning). Every tick after the first adds the
 * one-step score sums sum W dlw, sum W dlw^2, sum W dlw (h_{t-1}-mu), sum W dlw^2 (h_{t-1}-mu)^2
 * (W the normalised weights, dlw = d log p(y_t|h)/dh at h_t; computed inside pass 1 and the
 * plan kernel); every K such ticks mu is moved through alpha = mu (1 - rho) by a Robbins-Monro
 * step c / (k + t0)^gamma times the direction (mode 1: mean score / mean Fisher information,
 * mode 2: mean score), clipped to +-5 and gated by min(SNR / 2, 1); mu stays in [-5, 2] and rho
 * in [0.001, 0.999]. mode 0 switches learning off. An update reads the device state back, so
 * learning filters synchronise every K ticks (as the reference) and step_many runs them
 * without CUDA graphs. */
void gpu_bpf_enable_mu_learning(GpuBpfState* state, int mode, int K, float c, float t0, float gamma);
void gpu_bpf_disable_mu_learning(GpuBpfState* state);
void gpu_bpf_enable_rho_learning(GpuBpfState* state, int enable);
/* Addition: the score sums accumulated since the last update, and how many ticks they cover. */
int  gpu_bpf_get_learning_sums(GpuBpfState* state, double* sums4, int* ticks);

/* ---- Additions ------------------------------------------------------------ */

/* Last status recorded by any call on this host thread, and its text. */
int         gpu_bpf_last_error(void);
const char* gpu_bpf_error_string(int code);

/* Runs n_ticks ticks on host observations y[0..n_ticks). Inputs are staged
 * through pinned memory; ticks run as CUDA-graph chunks with no host sync
 * inside a chunk. out (may be NULL) receives one BpfResult per tick, rec
 * (may be NULL) one BpfTickRecord per tick. Returns a BPF_* status. */
int gpu_bpf_step_many(GpuBpfState* state, const float* y, int n_ticks,
                      BpfResult* out, BpfTickRecord* rec);

/* Same on device memory: y_dev[n_ticks] and rec_dev[n_ticks] are device
 * pointers; enqueued on state->stream without synchronising. The launch
 * sequence is captured once into a CUDA graph per (y_dev, rec_dev, n_ticks,
 * parameters) and replayed on later calls with the same buffers. */
int gpu_bpf_step_many_device(GpuBpfState* state, const float* y_dev, int n_ticks,
                             BpfTickRecord* rec_dev);

/* Re-seed the filter in place (addition): h_0 redrawn from the stationary
 * law of the current (mu, rho, sigma_z) with the given seed, tick counter,
 * resampling-uniform stream and log-likelihood sums reset. Stream-ordered,
 * no allocation, no host synchronisation. */
int gpu_bpf_reset(GpuBpfState* state, int seed);

/* Full record of the last tick (waits). */
int gpu_bpf_get_record(GpuBpfState* state, BpfTickRecord* out);

/* ESS of the last tick and the FP64 running log-likelihood (wait). */
float  gpu_bpf_get_ess(GpuBpfState* state);
double gpu_bpf_get_loglik_total(GpuBpfState* state);

/* BpfResult.log_lik semantics: 0 (default) = increment log p(y_t|y_{1:t-1});
 * 1 = the reference's value max+ln(sum w/N) over the carried weights, i.e.
 * the log-evidence since the last resample (bpf_kernels_full.ptx:755-775). */
int gpu_bpf_set_loglik_semantics(GpuBpfState* state, int mode);

/* Particles h[0..N) of the current state (waits). */
int gpu_bpf_get_particles(GpuBpfState* state, float* h_out);

/* Ancestor recording: when enabled, every resampling tick stores its
 * ancestor indices; gpu_bpf_get_ancestors copies the last tick's (waits) and
 * returns 1 if that tick resampled, 0 if not, <0 on error. */
int gpu_bpf_record_ancestors(GpuBpfState* state, int enable);
int gpu_bpf_get_ancestors(GpuBpfState* state, int32_t* anc_out);

/* Resampling inputs of the last tick (waits): the tile-relative FP32
 * weights w[0..N), the power-of-two exponent of each 4096-particle tile
 * (n_tiles = ceil(N/4096) entries) and the 23-bit resampling uniform U.
 * Ancestors are a deterministic function of these. */
int gpu_bpf_get_resample_inputs(GpuBpfState* state, float* w_out, int32_t* tile_exp_out,
                                uint32_t* u23_out);

/* Checkpoint / resume (addition). A checkpoint holds the filter's whole
 * stochastic state: particles, carried log2-weights and tile exponents, the
 * device tick state (tick index, PCG32 stream constants, resampling-uniform
 * stream, log-likelihood sums, Silverman and online-learning state) and the
 * parameters (rho, sigma_z, mu, nu_state, nu_obs, ess_threshold,
 * silverman_shrink, seed). The PCG32 streams are counter-based, so no per-particle
 * RNG state is stored. gpu_bpf_save writes gpu_bpf_checkpoint_bytes(state)
 * bytes into buf (waits for the filter's stream); gpu_bpf_load restores them into
 * a filter with the same n_particles (BPF_ERR_ARG otherwise), after which the
 * filter continues exactly as the saved one would have. Host-side settings
 * (online-learning schedule, ancestor recording, log-likelihood semantics,
 * profiling) are not part of the checkpoint; the result of the tick before the
 * save is not either (gpu_bpf_get_result needs a tick after the load). */
size_t gpu_bpf_checkpoint_bytes(GpuBpfState* state);
int    gpu_bpf_save(GpuBpfState* state, void* buf, size_t cap);
int    gpu_bpf_load(GpuBpfState* state, const void* buf, size_t len);

/* Fused small-filter ticks (addition): a filter of at most 65536 particles runs
 * each tick as one launch of a thread-block cluster, one CTA per 4096 particles
 * (pass 1, the resampling decision and the resampling in shared memory, the CTAs
 * reading each other's through distributed shared memory), and a captured run of
 * ticks (gpu_bpf_step_many, gpu_bpf_step_many_device) as one launch for the whole
 * run, with results bit-identical to the three-kernel tick. Filters of more than
 * 32768 particles take it where the device schedules a cluster of 16 CTAs. On by
 * default; enable = 0 selects the three-kernel tick. Learning filters, Silverman
 * jitter and profiled ticks always take the three-kernel path. */
int gpu_bpf_set_fused_small(GpuBpfState* state, int enable);

/* Kernel profiling: when enabled, every tick's three kernels (pass 1, plan,
 * pass 2) are timed with CUDA events on state->stream (launched without
 * programmatic dependent launch so the events bracket each kernel). read
 * returns the summed durations (ms) and the tick counts since enabling. */
int gpu_bpf_profile(GpuBpfState* state, int enable);
int gpu_bpf_profile_read(GpuBpfState* state, double* pass1_ms, double* plan_ms, double* pass2_ms,
                         int* pass1_launches, int* pass2_launches);

/* Allocation-free run (addition; no counterpart in the reference).
 * For callers that may not allocate GPU memory while they run: hosts that
 * reserve their whole device memory budget at start-up and forbid later
 * allocations, and latency-critical loops that cannot take cudaFree's
 * implicit device synchronisation or the allocator's locks.
 * Runs one plain filter (same algorithm and results as gpu_bpf_create +
 * gpu_bpf_step_many_device + gpu_bpf_destroy) of n_particles <=
 * BPF_STATIC_MAX_PARTICLES over the device observations y_dev[0..n_ticks),
 * writing one BpfTickRecord per tick to the device array rec_dev. All filter
 * state lives in one fixed scratch area compiled into the library (about
 * 3 MiB, held by every GPU that loads the library until the process exits);
 * no cudaMalloc, cudaFree or allocating library call is made. Larger sizes
 * return BPF_ERR_ARG.
 * The first call on a device looks the scratch address up with that device
 * current; make that first call before any stream capture. Every call
 * re-initialises the whole state, and all calls share the one scratch area:
 * calls whose GPU work overlaps (other streams or host threads) race and
 * corrupt each other, so serialise them. Enqueued on `stream` (a
 * cudaStream_t, NULL = the legacy default stream); does not synchronise.
 * The return value covers the arguments and the launches only: the run's
 * device-side outcome is in the records (a tick whose every weight underflowed
 * has dloglik = -inf and h_mean = NaN), and a resampling copy that failed to
 * complete on the device, which gpu_bpf_step reports as BPF_ERR_STATE, is not
 * reported by this entry point. */
#define BPF_STATIC_MAX_PARTICLES 262144
int gpu_bpf_run_static(int n_particles, float rho, float sigma_z, float mu, float nu_obs, int seed,
                       float ess_threshold, const float* y_dev, int n_ticks, BpfTickRecord* rec_dev,
                       void* stream);

/* ---- APF: auxiliary particle filter (gpu_bpf/gpu_bpf.cuh:114-126) ---------------
 * Behaviour of gpu_bpf/gpu_bpf_ptx_full.cu:990-1190. Tick 0 is a bootstrap tick; every later
 * tick resamples twice: by the first-stage weights v_i = p(y_t | mu + rho (h_i - mu)), then,
 * after propagating the resampled particles, by w_i = p(y_t | h_i) / p(y_t | m_i). The reference
 * public struct (gpu_bpf_full.cuh:314-337) holds device pointers and cuRAND states; this one keeps
 * the parameter fields and puts the buffers behind `impl`. The state noise is drawn from the
 * per-slot PCG32 streams (draw t of slot i at tick t, as the bootstrap filter's) instead of
 * cuRAND XORWOW; the resampling uniforms come from the reference's host-formula stream, two per
 * tick after tick 0. rho / sigma_z / mu may change between ticks. */
typedef struct {
    int    n_particles;
    float  rho, sigma_z, mu, nu_state, nu_obs;
    int    timestep;        /* refreshed whenever results are read back */
    void*  stream;          /* cudaStream_t owned by the filter */
    void*  impl;            /* opaque */
} GpuApfState;

/* gpu_bpf/gpu_bpf.cuh:119-120 (gpu_bpf_ptx_full.cu:1050-1082). NULL on failure (gpu_bpf_last_error()). */
GpuApfState* gpu_apf_create(int n_particles, float rho, float sigma_z, float mu,
                            float nu_state, float nu_obs, int seed);
/* gpu_bpf/gpu_bpf.cuh:121 (gpu_bpf_ptx_full.cu:1084-1093). NULL is a no-op. */
void gpu_apf_destroy(GpuApfState* state);
/* gpu_bpf/gpu_bpf.cuh:122 (gpu_bpf_ptx_full.cu:1102-1175): one tick, synchronous. log_lik is the
 * reference's value, log mean of the second-stage weights; the APF estimate of
 * log p(y_t | y_{1:t-1}) (adds log mean of the first-stage weights) is BpfTickRecord.dloglik of
 * gpu_apf_get_record. {NaN, NaN} on error. */
BpfResult gpu_apf_step(GpuApfState* state, float y_t);
/* gpu_bpf/gpu_bpf.cuh:124-126 (gpu_bpf_ptx_full.cu:1177-1190): RMSE of h_mean vs true_h after the
 * first 100 ticks. NaN on error. */
double gpu_apf_run_rmse(const double* returns, const double* true_h, int n_ticks,
                        int n_particles, float rho, float sigma_z, float mu,
                        float nu_state, float nu_obs, int seed);
/* Additions: n_ticks ticks in one call (CUDA graphs of 64 ticks after tick 0), results and/or
 * records per tick (either may be NULL); the last tick's record; the FP64 running sum of the
 * APF increments; the particles; the ancestors of both resampling stages of the last tick
 * (after gpu_apf_record_ancestors(state, 1); tick 0 writes only the second). */
int    gpu_apf_step_many(GpuApfState* state, const float* y, int n_ticks, BpfResult* out, BpfTickRecord* rec);
int    gpu_apf_get_record(GpuApfState* state, BpfTickRecord* out);
double gpu_apf_get_loglik_total(GpuApfState* state);
int    gpu_apf_get_particles(GpuApfState* state, float* h_out);
int    gpu_apf_record_ancestors(GpuApfState* state, int enable);
int    gpu_apf_get_ancestors(GpuApfState* state, int32_t* anc_first, int32_t* anc_second);

/* ---- IMM: interacting multiple model (gpu_bpf/gpu_bpf.cuh:131-164) ----------
 * K SV models stepped on the same observations; model probabilities follow a Markov switching
 * prior (transition matrix T[j*K + k] = P(j -> k), row-major; NULL = 0.95 stay, the rest spread
 * evenly) and each tick's log-likelihood increment. Models run as one resumable batch (one graph
 * launch per tick) when n_particles_per_model <= 16384, else as K plain filters. Model k uses the
 * seed seed + 7919 k and the plain filter's default ESS threshold 0.5 (as the reference). */
#define IMM_MAX_MODELS 64

typedef struct {
    float rho, sigma_z, mu, nu_state, nu_obs;
} ImmModelParams;                                            /* gpu_bpf/gpu_bpf.cuh:135-137 */

typedef struct {
    float h_mean, vol, log_lik;    /* mixed filtered mean, exp(h_mean/2), log p(y_t | y_{1:t-1}) */
    int   best_model;
    float best_prob;
} ImmResult;                                                 /* gpu_bpf/gpu_bpf.cuh:139-143 */

typedef struct {
    GpuBpfState** filters;         /* the K plain filters when they are used, else NULL */
    int     n_models, n_particles_per_model;
    double *log_pi, *log_pi_pred, *log_T;
    int     timestep;
    void*   impl;                  /* batched models and staging buffers */
} GpuImmState;                                               /* gpu_bpf/gpu_bpf.cuh:145-150 */

/* gpu_bpf/gpu_bpf.cuh:151-153. NULL when n_models is outside 1..64 or a model is invalid. */
GpuImmState* gpu_imm_create(const ImmModelParams* models, int n_models, int n_particles_per_model,
                            const float* transition_matrix, int seed);
ImmResult    gpu_imm_step(GpuImmState* state, float y_t);           /* gpu_bpf/gpu_bpf.cuh:154; waits */
float        gpu_imm_get_prob(const GpuImmState* state, int k);     /* gpu_bpf/gpu_bpf.cuh:155 */
void         gpu_imm_get_probs(const GpuImmState* state, float* probs_out);   /* gpu_bpf/gpu_bpf.cuh:156 */
void         gpu_imm_destroy(GpuImmState* state);                   /* gpu_bpf/gpu_bpf.cuh:157 */
/* gpu_bpf/gpu_bpf.cuh:159-162: the rho x sigma_z x mu grid (rho-major), malloc'd; free() it. */
ImmModelParams* gpu_imm_build_grid(const float* rhos, int n_rho, const float* sigma_zs, int n_sigma,
                                   const float* mus, int n_mu, float nu_state, float nu_obs, int* out_n_models);

/* ---- Batched filters (addition) -------------------------------------------
 * Many independent SV filters with their own (mu, rho, sigma_z, nu_obs), particle count
 * (1..16384) and seed, all on one observation series: the SMC^2 / PMMH inner loop. The
 * reference runs such filters one per CUDA stream (the IMM pattern, gpu_bpf/gpu_bpf.cu:1033-1047)
 * or as its own per-theta RBPF CTA (smc2/smc2_rbpf_batch.cu:248-398). Here every filter keeps its
 * particles in one CTA's shared memory for the whole run; filters are grouped into five size
 * classes (N <= 1024, 2048, 4096, 8192, 16384), each class is one persistent launch pulling
 * filters largest-first, and a run is replayed as one CUDA graph. A batched filter computes the
 * same per-particle arithmetic and the same fixed-point resampling as gpu_bpf_create with the
 * same parameters and seed. */
typedef struct {
    float mu, rho, sigma_z, nu_obs;
    int   n_particles;
    int   seed;
    float nu_state;   /* Student-t state noise as in gpu_bpf_create (0 = Gaussian) */
} BpfBatchFilter;
typedef struct GpuBpfBatch GpuBpfBatch;

/* ess_threshold as gpu_bpf_set_ess_threshold (0 = resample every tick). NULL on error. */
GpuBpfBatch* gpu_bpf_batch_create(const BpfBatchFilter* filters, int n_filters, float ess_threshold);
void         gpu_bpf_batch_destroy(GpuBpfBatch* batch);
void*        gpu_bpf_batch_stream(GpuBpfBatch* batch);          /* cudaStream_t of the batch */
int          gpu_bpf_batch_size_class(int n_particles);         /* 0..4, or -1 if above 16384 */
/* Threads per CTA (64, 128, 256, 512, 1024) of one size class: the tile shape. */
int          gpu_bpf_batch_set_threads(GpuBpfBatch* batch, int size_class, int threads);
int          gpu_bpf_batch_get_threads(GpuBpfBatch* batch, int size_class);
/* Project autotuner: times every CTA shape of every non-empty class on n_ticks of y and keeps
 * the fastest; results are appended to / read from the text cache file cache_path
 * ("<gpu> <class> <threads>" lines; NULL = no cache). */
int          gpu_bpf_batch_autotune(GpuBpfBatch* batch, const float* y, int n_ticks, const char* cache_path);
/* Host buffers: y[n_ticks] in, loglik[n_filters] (FP64 total log-likelihood) and optionally the
 * last tick's filtered mean out. Synchronous. */
int          gpu_bpf_batch_run(GpuBpfBatch* batch, const float* y, int n_ticks, double* loglik,
                               float* hmean_last);
/* Device buffers, enqueued on the batch stream: loglik_dev[n_filters]; dll_dev[n_filters*n_ticks]
 * per-tick increments and hmean_dev[n_filters*n_ticks] filtered means (either may be NULL). */
int          gpu_bpf_batch_run_device(GpuBpfBatch* batch, const float* y_dev, int n_ticks, double* loglik_dev,
                                      double* dll_dev, float* hmean_dev);
/* Testing aid: as run_device without a graph, also writing every tick's ancestors
 * (anc_dev[(f*n_ticks + t)*16384 + i]) and the final particles (particles_dev[f*16384 + i]). */
int          gpu_bpf_batch_run_debug(GpuBpfBatch* batch, const float* y_dev, int n_ticks, double* loglik_dev,
                                     double* dll_dev, int32_t* anc_dev, float* particles_dev);
/* Resampling count and last filtered mean of every filter after a run (waits). */
int          gpu_bpf_batch_resample_counts(GpuBpfBatch* batch, int* counts, float* hmean_last);
/* Resumable stepping: advance every filter by n_ticks from where the previous step left it
 * (the first step after create or gpu_bpf_batch_reset starts at tick 0), enqueued on the batch
 * stream as one CUDA graph (captured on the first call and whenever n_ticks or the CTA shapes
 * change; a call that differs only in y_dev / dll_dev / hmean_dev launches the same kernels
 * directly, so walking a device series one tick at a time captures nothing). Device buffers: y_dev[n_ticks]; dll_dev[n_filters*n_ticks] and
 * hmean_dev[n_filters*n_ticks] (either may be NULL) receive this step's per-tick increments and
 * filtered means. The filters' state lives on the device between steps (8 B per particle). A
 * batch stepped in pieces is bit-identical to one run over the whole series. */
int          gpu_bpf_batch_step_device(GpuBpfBatch* batch, const float* y_dev, int n_ticks, double* dll_dev,
                                       float* hmean_dev);
int          gpu_bpf_batch_reset(GpuBpfBatch* batch);   /* next step starts again at tick 0 */
/* New (mu, rho, sigma_z, nu_obs, nu_state, seed) for every filter; each n_particles must equal the
 * filter's count at creation. Takes effect at the next run or step; the saved state is kept.
 * Waits for the batch stream. */
int          gpu_bpf_batch_set_filters(GpuBpfBatch* batch, const BpfBatchFilter* filters);
int          gpu_bpf_batch_tick(GpuBpfBatch* batch);    /* ticks stepped since create / reset */
/* Device array [n_filters] of FP64 total log-likelihoods, updated by every run or step. */
double*      gpu_bpf_batch_loglik_device(GpuBpfBatch* batch);
/* Batched gradient (the SMC^2 / PMMH inner loop with gradients): one forward and one backward
 * pass of every filter in one persistent launch per size class (each CTA runs a filter's taped
 * forward, then its adjoint, as gpu_bpf_grad_forward/backward do for one filter), replayed as
 * one CUDA graph. Device buffers: loglik_dev[n_filters] (FP64 total log-likelihood) and
 * grad_dev[3*n_filters] = d loglik / d(mu, rho, sigma_z) per filter, ancestors held fixed.
 * The batch must resample every tick (ess_threshold 0; BPF_ERR_UNSUPPORTED otherwise). */
int          gpu_bpf_batch_grad_run(GpuBpfBatch* batch, const float* y_dev, int n_ticks, double* loglik_dev,
                                    double* grad_dev);
/* Device memory the gradient tape of gpu_bpf_batch_grad_run takes for n_ticks ticks (it is sized
 * for the CTAs in flight, not for the number of filters). */
size_t       gpu_bpf_batch_grad_tape_bytes(GpuBpfBatch* batch, int n_ticks);
/* Correlated-noise runs: the building block of correlated pseudo-marginal MCMC (CPMMH,
 * Deligiannidis, Doucet & Pitt 2018), as the reference's CPMMH rejuvenation kernel uses it
 * (smc2/smc2_rbpf_batch.cu:651-935). Every filter runs ticks 0..n_ticks-1 from a fresh start
 * with its auxiliary noise exposed: filter f's noise is an area of
 * n_ticks * (n_pad + 4) floats, n_pad = n_particles rounded up to a multiple of 4, starting at
 * element gpu_bpf_batch_noise_offset(f) of the noise buffers. Per tick: floats [0, n_particles)
 * are the particles' standard normals (tick 0: the initial draw), float n_pad is the normal v
 * whose Phi(v) is the tick's resampling uniform, the rest are unused. With noise_in_dev NULL the
 * normals are the filters' own PCG32 draws (as an ordinary run); otherwise
 * noise = rho * noise_in + sqrt(1 - rho^2) * the filter's own draw (rho in [0, 1]; rho = 1
 * replays noise_in exactly). The noise used is written to noise_out_dev (which must not be
 * noise_in_dev). Before every resampling the particles are sorted by value, so that nearby
 * noise gives nearby resampling. Filters must have at most 4096 particles and Gaussian state
 * noise (BPF_ERR_UNSUPPORTED otherwise). loglik_dev[n_filters] and dll_dev[n_filters*n_ticks]
 * (or NULL) as in gpu_bpf_batch_run_device; anc_dev (or NULL, a testing aid) as in
 * gpu_bpf_batch_run_debug, each ancestor the particle's slot before the sort. Enqueued on the
 * batch stream. */
int          gpu_bpf_batch_run_correlated(GpuBpfBatch* batch, const float* y_dev, int n_ticks,
                                          const float* noise_in_dev, float* noise_out_dev, float rho,
                                          double* loglik_dev, double* dll_dev, int32_t* anc_dev);
/* First element of filter f's area in the noise buffers of n_ticks-tick correlated-noise runs;
 * with f = n_filters, the buffers' length in floats. */
long long    gpu_bpf_batch_noise_offset(GpuBpfBatch* batch, int filter, int n_ticks);

/* ---- Gradient (addition) ---------------------------------------------------
 * d loglik / d(mu, rho, sigma_z) of the plain filter with the resampling ancestors held fixed.
 * The reference differentiates the same loss by autograd with detached resampling indices
 * (tests/diff_bpf.py:186-237, :35-56, :230-231); here a taped forward run stores, per tick, the
 * first child slot of every parent (systematic ancestors are non-decreasing, so a parent's
 * children are a contiguous run of slots) and a checkpoint of the particles every
 * checkpoint_every ticks; the backward pass recomputes each segment's particles from its
 * checkpoint, the child lists and the counter-based PCG32 noise, and runs the adjoint
 *   lambda_t,j = W_t,j dlogp(y_t|h)/dh (h_t,j) + rho * sum_{children i of j} lambda_t+1,i
 * backward through it, accumulating the parameter adjoints (including the stationary initial
 * draw) in FP64. Tapes resample every tick (ess_threshold 0, the reference's diff_bpf choice). */
typedef struct GpuBpfGrad GpuBpfGrad;

/* Tape for up to max_ticks ticks of n_particles (checkpoint_every 0 = 16). NULL on error.
 * Device memory: gpu_bpf_grad_tape_bytes() (about 4 * n_particles * max_ticks bytes). */
GpuBpfGrad* gpu_bpf_grad_create(int n_particles, int max_ticks, int checkpoint_every);
void        gpu_bpf_grad_destroy(GpuBpfGrad* grad);
size_t      gpu_bpf_grad_tape_bytes(int n_particles, int max_ticks, int checkpoint_every);
void*       gpu_bpf_grad_stream(GpuBpfGrad* grad);                 /* cudaStream_t of the tape */
int         gpu_bpf_grad_checkpoint_every(GpuBpfGrad* grad);
/* Taped forward run from a fresh start (as gpu_bpf_create + reset(seed) + n_ticks steps;
 * nu_state and nu_obs as in gpu_bpf_create):
 * y_dev[n_ticks] in, loglik_dev[0] = FP64 total log-likelihood out. Enqueued on the tape's
 * stream. ess_threshold must be 0 (BPF_ERR_UNSUPPORTED otherwise). */
int gpu_bpf_grad_forward(GpuBpfGrad* grad, float mu, float rho, float sigma_z, float nu_state, float nu_obs,
                         int seed, float ess_threshold, const float* y_dev, int n_ticks, double* loglik_dev);
/* Adjoint of the last taped run: grad_dev[3] = d loglik / d(mu, rho, sigma_z), FP64. */
int gpu_bpf_grad_backward(GpuBpfGrad* grad, double* grad_dev);
/* FP64 re-run of the taped run's noise and ancestors at (mu, rho, sigma_z) with forward-mode
 * tangents: out_dev[4] = {loglik, d/dmu, d/drho, d/dsigma_z}; per_tick_dev[4*n_ticks] (or NULL)
 * the same per tick. For finite-difference checks under common random numbers. */
int gpu_bpf_grad_replay(GpuBpfGrad* grad, double mu, double rho, double sigma_z, double* out_dev,
                        double* per_tick_dev);
/* Testing aids (wait for the tape's stream): the taped run's first n records, and the first
 * child slot of every parent after tick `tick`'s resampling (host arrays). */
int gpu_bpf_grad_get_records(GpuBpfGrad* grad, BpfTickRecord* out, int n);
int gpu_bpf_grad_get_children(GpuBpfGrad* grad, int tick, int32_t* first_child);

/* ---- SMC^2 over the SV parameters (addition) ---------------------------------
 * Online Bayesian learning of theta = (mu, rho, sigma_z) by SMC^2: n_theta theta-particles, each
 * with an inner bootstrap filter of n_particles (<= 16384) run as one resumable batch; outer
 * weights are the inner log-likelihood increments; when the outer ESS falls below the
 * threshold the theta-particles are resampled and rejuvenated by particle marginal
 * Metropolis-Hastings moves whose proposals are scored by fresh inner filters over the whole
 * history. The outer loop of the reference's smc2_cuda_update
 * (smc2/smc2_rbpf_batch.cu:1329-1502, host API smc2/smc2_rbpf_batch.cuh:461-489) on this build's
 * SV model, with the reference's correlated-noise (CPMMH) moves as an option
 * (gpu_bpf_smc2_set_cpmmh_rho); the reference's regime-switching RBPF inner model is not part
 * of it. Prior: mu ~ N(mu_mean, mu_sd^2), rho ~ U(rho_lo, rho_hi), sigma_z ~ U(sigma_lo,
 * sigma_hi) (NULL = N(-1, 0.5^2), U(0.85, 0.995), U(0.05, 0.4)). Deterministic given the seed. */
typedef struct {
    float mu_mean, mu_sd, rho_lo, rho_hi, sigma_lo, sigma_hi;
} BpfSmc2Prior;
typedef struct GpuBpfSmc2 GpuBpfSmc2;

/* ~ smc2_cuda_alloc + smc2_cuda_set_seed + smc2_cuda_init_from_prior. max_ticks bounds the
 * observation history kept on the device. NULL on error. */
GpuBpfSmc2* gpu_bpf_smc2_create(int n_theta, int n_particles, int max_ticks, const BpfSmc2Prior* prior,
                                unsigned long long seed);
void        gpu_bpf_smc2_destroy(GpuBpfSmc2* smc2);                              /* ~ smc2_cuda_free */
/* Rejuvenation: PMMH moves per resampling (default 1), outer ESS threshold as a fraction of
 * n_theta (default 0.5), random-walk scale relative to 2.38^2/3 times the theta covariance (1). */
int         gpu_bpf_smc2_set_moves(GpuBpfSmc2* smc2, int n_moves, float outer_ess_threshold,
                                   float proposal_scale);
/* ~ smc2_cuda_update: one observation; returns the outer ESS after it (NaN on error). Waits. */
float       gpu_bpf_smc2_update(GpuBpfSmc2* smc2, float y);
float       gpu_bpf_smc2_get_outer_ess(GpuBpfSmc2* smc2);                        /* ~ smc2_cuda_get_outer_ess */
/* ~ smc2_cuda_get_theta_mean / _std: weighted posterior mean and std of (mu, rho, sigma_z). */
int         gpu_bpf_smc2_get_theta(GpuBpfSmc2* smc2, float* mean3, float* std3);
/* theta[3*n_theta] (mu, rho, sigma_z per particle), outer log-weights and inner total
 * log-likelihoods (each may be NULL). */
int         gpu_bpf_smc2_get_particles(GpuBpfSmc2* smc2, float* theta, double* logw, double* loglik);
int         gpu_bpf_smc2_stats(GpuBpfSmc2* smc2, int* n_rejuvenations, long long* n_proposed,
                               long long* n_accepted);
/* ~ smc2_cuda_set_cpmmh_rho (smc2/smc2_rbpf_batch.cu:1238-1240): correlated-noise PMMH moves.
 * rho in (0, 1] keeps every theta-particle's auxiliary noise (its inner filter's normals and
 * resampling normals, as in gpu_bpf_batch_run_correlated) on the device and scores each proposal
 * with noise rho * current + sqrt(1 - rho^2) * fresh; accepted proposals' noise becomes current,
 * outer resampling copies it with the filter. rho = 0 (the default) scores proposals with fresh
 * inner filters. Switching between 0 and > 0 is allowed only before the first update; the noise
 * takes 8 * n_theta * max_ticks * (n_particles + 8) bytes; n_particles must be at most 4096. The
 * reference's default is 0.99. */
int         gpu_bpf_smc2_set_cpmmh_rho(GpuBpfSmc2* smc2, float rho);
/* The last PMMH move (host arrays, each may be NULL): proposed and current theta [3*n_theta]
 * (as the inner filters use them), the proposals' and the current inner log-likelihoods
 * [n_theta] and the acceptance flags [n_theta]. BPF_ERR_STATE before the first move. */
int         gpu_bpf_smc2_get_last_move(GpuBpfSmc2* smc2, float* theta_prop, float* theta_cur,
                                       double* loglik_prop, double* loglik_cur, int* accepted);
/* The last update (host arrays, each may be NULL): the forward tick's inner log-likelihood
 * increments [n_theta] (the outer log-weights' increments), whether the theta-particles were
 * resampled, and then their outer ancestors [n_theta]. BPF_ERR_STATE before the first update. */
int         gpu_bpf_smc2_get_last_update(GpuBpfSmc2* smc2, double* dll, int* resampled, int* ancestors);
/* Theta-particle j's current auxiliary noise for ticks 0..n_ticks-1 (n_ticks at most the ticks
 * seen; layout of gpu_bpf_batch_run_correlated's areas) into the host array out. Needs
 * rho > 0. */
int         gpu_bpf_smc2_get_noise(GpuBpfSmc2* smc2, int j, int n_ticks, float* out);

/* Allocation fault injection (addition; testing aid). Every device and pinned
 * allocation of the library goes through one set of wrappers. After
 * gpu_bpf_debug_fail_alloc(k) the next k allocations succeed and the one after
 * them fails as an out-of-memory allocation would (once; k < 0 disarms), so the
 * error path of any create function can be exercised on the host without a GPU
 * fault. gpu_bpf_debug_alloc_count: allocations attempted since the library was
 * loaded; gpu_bpf_debug_live_allocs: allocations not yet freed. */
int       gpu_bpf_debug_fail_alloc(long long k);
long long gpu_bpf_debug_alloc_count(void);
long long gpu_bpf_debug_live_allocs(void);

/* Number of kernel launches this library has issued (all filters). */
long long gpu_bpf_launch_count(void);

/* Device-side PCG32 probes: raw output of draw t for slots 0..n-1 and the
 * normal the filter derives from it (writes host arrays). */
int gpu_bpf_debug_pcg32(int seed, int n, int t, uint32_t* out);
int gpu_bpf_debug_normals(int seed, int n, int t, float* out);

#ifdef __cplusplus
}
#endif

#endif /* GPU_BPF_H */
