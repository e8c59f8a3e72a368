/*
 * pasta_b200.h -- C ABI of the B200 (sm_100a) implementation of PASTA's
 * per-particle model-evaluation and chi2 hot path.
 *
 * Every entry point returns an int status: 0 on success, a negative
 * PASTA_E_* code on failure, with a message from pasta_last_error()
 * (thread-local).  All array arguments are caller-owned HOST pointers; the
 * library copies them to the device and back.  Handles own device memory
 * until destroyed.  No torch or C++ types cross this boundary.
 *
 * Reference interface that each entry point replaces is cited as
 * file:line in SimonVanSchuylenbergh/PASTA (Rust + PyO3).
 */
#ifndef PASTA_B200_H
#define PASTA_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PASTA_B200_ABI_VERSION 1

/* wavelength grid kinds (interpolate.rs:672-679) */
enum { PASTA_WL_LINSPACE = 0, PASTA_WL_LOGSPACE = 1, PASTA_WL_NONUNIFORM = 2 };
/* dispersion kinds (lib.rs:655-662) */
enum { PASTA_DISP_NONE = 0, PASTA_DISP_FIXED = 1, PASTA_DISP_VARIABLE = 2 };
/* continuum fitter kinds (lib.rs:800-807) */
enum { PASTA_CONT_CHUNK = 0, PASTA_CONT_LINEAR = 1, PASTA_CONT_FIXED = 2, PASTA_CONT_CONSTANT = 3 };
/* fit execution forms */
enum { PASTA_FIT_BATCHED = 0, PASTA_FIT_PLAIN = 1 };

/* error codes */
enum {
  PASTA_OK = 0,
  PASTA_E_ARG = -1,            /* invalid argument / length mismatch      */
  PASTA_E_CUDA = -2,           /* CUDA runtime error                      */
  PASTA_E_NOMEM = -3,          /* device memory or HBM budget exhausted   */
  PASTA_E_OUT_OF_GRID = -10,   /* label outside the grid (interpolate.rs:425-430) */
  PASTA_E_NEIGHBORS = -11,     /* neighbour search failed (interpolate.rs:105-159, cubic.rs:155) */
  PASTA_E_VSINI = -12,         /* vsini < 0 (convolve_rv.rs:489-491)      */
  PASTA_E_KERNEL_WIDTH = -13,  /* rotation kernel > 2048 (convolve_rv.rs:512-519) */
  PASTA_E_RV_RANGE = -14,      /* shifted window leaves the synthetic grid (convolve_rv.rs:549-567) */
  PASTA_E_RESAMPLE = -15,      /* resampling reads one pixel past the grid (convolve_rv.rs:572) */
  PASTA_E_BOUNDS = -16,        /* PSO particle outside the bounds (particleswarm.rs:267-275) */
  PASTA_E_CLAMP = -17,         /* clamp limits invalid (bounds.rs:13-16)  */
  PASTA_E_CONTINUUM = -18,     /* continuum fitter cannot run on this spectrum */
  PASTA_E_NAN = -19,           /* NaN label                                */
  PASTA_E_UNSUPPORTED = -20,   /* e.g. rotation on a non-uniform grid (convolve_rv.rs:506) */
  PASTA_E_INTERNAL = -99
};

typedef struct pasta_grid pasta_grid;
typedef struct pasta_dispersion pasta_dispersion;
typedef struct pasta_continuum pasta_continuum;
typedef struct pasta_server pasta_server;

typedef struct {
  int32_t num_particles;
  int32_t max_iters;
  double inertia_factor, cognitive_factor, social_factor, delta;
  double vsini_lo, vsini_hi, rv_lo, rv_hi;
  /* per-parameter constraint: 0 none, 1 fixed at a, 2 range [a, b] (lib.rs:817-835) */
  int32_t ckind[5];
  double ca[5], cb[5];
} pasta_pso_settings;

typedef struct {
  double label[5]; /* teff, m, logg, vsini, rv */
  double chi2;
  double time;     /* seconds from submission to result */
  int32_t iterations;
  int32_t status;  /* 0 ok, else PASTA_E_* of the failing particle */
  int32_t n_params;
  int32_t _pad;
} pasta_fit_result;

/* ------------------------------------------------------------ library */
int pasta_abi_version(void);
const char *pasta_last_error(void);
/* Select the CUDA device used by handles created afterwards on this thread. */
int pasta_set_device(int device);
/* Number of launches of this library's kernels since load (all threads). */
int64_t pasta_kernel_launch_count(void);
/* Linear-model continua (LinearModelFitter, continuum_fitting.rs:44-107)
 * with at most 64 design columns run on the tensor cores (tcgen05, f32
 * accuracy by split tf32 operands); 0 selects the CUDA-core path instead,
 * for the calls and batches started afterwards (no counterpart in the
 * reference; the environment variable PASTA_LINEAR_TC=0 sets the default). */
int pasta_set_linear_tensor_cores(int on);
/* Interpolation (GridInterpolator::interpolate, interpolate.rs:930-983) of
 * 16 or more evaluations of one star that share their 64 neighbour rows (a
 * contracted swarm) runs as one matrix product on the tensor cores (tcgen05,
 * rows staged by TMA, f32 accuracy from exact bf16 byte planes and three-part
 * bf16 weights); 0 keeps every evaluation on the CUDA cores, for the calls
 * and batches started afterwards (no counterpart in the reference; the
 * environment variable PASTA_INTERP_TC=0 sets the default). */
int pasta_set_interp_tensor_cores(int on);

/* ----------------------------------------------------------- the grid
 * Replaces InMemFetcher::new / from_tar_zstd + GridInterpolator::new
 * (model_fetchers.rs:136-226, interpolate.rs:905) and the PyO3
 * constructors InMemInterpolator/OnDiskInterpolator/CachedInterpolator
 * (lib.rs:1875-1931).  labels: n x (teff, m, logg) in any order; spectra:
 * n x n_px uint16, row i for labels[i]; maxima: the includes_factor f32
 * maxima (model_fetchers.rs:53-63) or NULL.  The grid is uploaded once and
 * stays resident in HBM.  Creation also measures, on this device, up to
 * which combined broadening width (rotation taps + 2 x instrument half
 * width) a direct convolution beats the FFT blocks; the environment
 * variable PASTA_DIRECT_MAX_TAPS fixes that width instead (0: FFT only). */
int pasta_grid_create(const double *labels, const uint16_t *spectra,
                      const float *maxima, int64_t n_models, int64_t n_px,
                      int wl_kind, double wl_a, double wl_b,
                      const double *wl_values, pasta_grid **out);
int pasta_grid_destroy(pasta_grid *g);
/* the measured direct/FFT crossover in taps (no counterpart in the
 * reference); set: 0..512, for the batches and fits started afterwards */
int pasta_grid_direct_max(const pasta_grid *g, int32_t *taps);
int pasta_grid_set_direct_max(pasta_grid *g, int32_t taps);
/* the measured group size (evaluations of one star sharing their 64
 * neighbour rows) from which the interpolation runs on the tensor cores, 65
 * = never (no counterpart in the reference); set: 8..65, for the batches and
 * fits started afterwards; PASTA_INTERP_TC_MIN fixes it at grid creation */
int pasta_grid_tc_min(const pasta_grid *g, int32_t *members);
int pasta_grid_set_tc_min(pasta_grid *g, int32_t members);
/* sizes: n_teff, n_m, n_logg, n_px, n_models (lib.rs:1436-1461) */
int pasta_grid_shape(const pasta_grid *g, int64_t *out5);
int pasta_grid_axis(const pasta_grid *g, int axis, double *out);
int pasta_grid_logg_limits(const pasta_grid *g, int64_t *lo, int64_t *hi);
int pasta_grid_cumulative_size(const pasta_grid *g, int64_t *out);
/* Grid::clamp_1d (interpolate.rs:625-628, lib.rs:1377-1382) */
int pasta_grid_clamp_1d(const pasta_grid *g, double teff, double m,
                        double logg, int index, double *out);
/* Grid::is_teff_logg_between_bounds (interpolate.rs:351-369, lib.rs:1463) */
int pasta_grid_is_teff_logg_between_bounds(const pasta_grid *g, double teff,
                                           double logg, int *out);
/* neighbour columns (-1 = missing) and f32 weights of the 4x4x4 cube plus
 * the flat factors (lib.rs:1388-1433, cubic.rs:159-243) */
int pasta_grid_coefficients(const pasta_grid *g, double teff, double m,
                            double logg, int64_t *cols64, float *w64,
                            double *teff16, double *logg16, double *m4);

/* GridInterpolator::interpolate (interpolate.rs:930-983, lib.rs:1111):
 * tml L x 3, out L x n_px float, status[L]. */
int pasta_interpolate(const pasta_grid *g, const double *tml, int64_t L,
                      float *out, int32_t *status);

/* ----------------------------------------------------- dispersions
 * NoConvolutionDispersion / FixedResolutionDispersion /
 * VariableResolutionDispersion (lib.rs:763-797; convolve_rv.rs:72-431).
 * The synthetic wavelength grid is passed like WlGrid (lib.rs:636-648).
 * disp: per observed pixel Gaussian sigma in Angstrom (variable kind). */
int pasta_dispersion_create(int synth_kind, double synth_a, double synth_b,
                            int64_t synth_n, const double *synth_values,
                            int kind, const double *wl_obs, int64_t n_obs,
                            double resolution, const float *disp,
                            pasta_dispersion **out);
int pasta_dispersion_destroy(pasta_dispersion *d);
/* PyWavelengthDispersion.convolve (lib.rs:671-680): in/out n = synth n */
int pasta_dispersion_convolve(const pasta_dispersion *d, const float *in,
                              int64_t n, float *out);
/* The arithmetic of PyWavelengthDispersion.convolve_and_resample_directory
 * (lib.rs:686-755) for M grid spectra at once: each row of in [M x n_in]
 * (dequantised flux on the input wavelength grid in_kind/in_a/in_b, which
 * has the dispersion's synth length) is convolved with the dispersion's
 * instrument profile and resampled at RV 0 to its observed wavelengths,
 * out [M x n_obs] (shift_and_resample, convolve_rv.rs:532-604).  Linspace
 * and Logspace input grids; a non-uniform one is PASTA_E_UNSUPPORTED. */
int pasta_dispersion_convolve_resample(const pasta_dispersion *d, int in_kind,
                                       double in_a, double in_b, int64_t n_in,
                                       const float *in, int64_t M, float *out);
/* kernel width (odd) and, if out != NULL, the kernels width x n_synth
 * row-major as get_kernels returns them (lib.rs:1043-1060) */
int pasta_dispersion_kernels(const pasta_dispersion *d, int64_t *width,
                             float *out);

/* ------------------------------------------------------ continuum
 * ChunkContinuumFitter / LinearModelContinuumFitter / FixedContinuum /
 * ConstantContinuum (lib.rs:945-983; continuum_fitting.rs:44-505).
 * design: n x k row-major f32. */
int pasta_continuum_create(int kind, const double *wl, int64_t n,
                           int n_chunks, int p_order, double overlap,
                           const float *design, int k,
                           const float *continuum, int ignore_first_and_last,
                           pasta_continuum **out);
int pasta_continuum_destroy(pasta_continuum *c);
int pasta_continuum_nparams(const pasta_continuum *c);
/* ContinuumFitter::fit_continuum (continuum_fitting.rs:13-17; lib.rs:862) */
int pasta_continuum_fit(const pasta_continuum *c, const float *model,
                        const float *flux, const float *var, int64_t n,
                        float *params, double *chi2);
/* ContinuumFitter::build_continuum (lib.rs:927-939); out has n values
 * (1 for the constant fitter) */
int pasta_continuum_build(const pasta_continuum *c, const float *params,
                          int64_t n_params, float *out);

/* ------------------------------------------------------ model / chi2
 * Interpolator::produce_model (interpolate.rs:1068-1090; lib.rs:993-1011,
 * 1064-1089): labels L x 5, out L x n_obs. */
int pasta_produce_model(const pasta_grid *g, const pasta_dispersion *d,
                        const double *labels, int64_t L, float *out,
                        int32_t *status);
/* interpolate_and_convolve (interpolate.rs:1030-1047; lib.rs:1141):
 * labels L x 4 (teff, m, logg, vsini), out L x n_synth. */
int pasta_interpolate_and_convolve(const pasta_grid *g,
                                   const pasta_dispersion *d,
                                   const double *labels, int64_t L,
                                   float *out, int32_t *status);
/* SingleFitter::chi2 via CostFunction::cost (fitting.rs:313-326, 460-478;
 * lib.rs:1603-1627): out[L] chi2 (NaN where status != 0). */
int pasta_chi2(const pasta_grid *g, const pasta_dispersion *d,
               const pasta_continuum *c, const float *flux, const float *var,
               int64_t n, const double *labels, int64_t L, double *out,
               int32_t *status);

/* InMemInterpolator.ccf (lib.rs:1340-1371): the model at (teff, m, logg),
 * interpolated once, shifted to each velocity vs[i] and resampled onto the
 * dispersion's wavelengths (shift_and_resample, convolve_rv.rs:532-604; no
 * broadening), dotted with flux (n = the dispersion's length).  out[V]; the
 * dot products are summed in FP64 on the device and rounded to f32 (the
 * reference sums in f32).  Status per velocity; NaN where it is non-zero. */
int pasta_ccf(const pasta_grid *g, const pasta_dispersion *d, const double *vs,
              int64_t V, double teff, double m, double logg, const float *flux,
              int64_t n, float *out, int32_t *status);

/* chi2 of S spectra, each with its own dispersion, continuum fitter, pixel
 * count and label (labels S x 5), in one batched device pass: the batched
 * form of InMemInterpolator.chi2_bulk (lib.rs:1297-1338), which evaluates
 * one spectrum per call there.  out[S] (NaN where status != 0). */
int pasta_chi2_many(const pasta_grid *g, int64_t S, const pasta_dispersion *const *d,
                    const pasta_continuum *const *c, const float *const *flux,
                    const float *const *var, const int64_t *n, const double *labels,
                    double *out, int32_t *status);

/* pasta_chi2 for callers that cannot allocate device memory: a host
 * framework that gives the GPU's whole memory to its own pool, a real-time
 * loop that may not call cudaMalloc (which can synchronise the device), a
 * service whose footprint is fixed after start-up.  No counterpart in the
 * reference.  flux, var (n floats), labels (L x 5 doubles), out (L doubles)
 * and status (L int32) are DEVICE buffers the caller owns; the work is
 * queued on `stream` (a cudaStream_t; NULL = the legacy default stream) and
 * is complete when that stream reaches it.  The evaluation workspace is a
 * 32 MiB static device array inside the library, held by every GPU that
 * loads it until exit and shared by all calls: L is limited to what fits
 * (about 180 labels for a 20,000-pixel grid, 50 for 80,000 pixels) and larger
 * L is rejected with PASTA_E_ARG; calls whose work overlaps on the GPU race
 * on the array.  The first call on a device sets up the array's address and
 * should come before any stream capture.  Nothing is allocated: no
 * cudaMalloc, cudaFree or allocating library routine.  L == 0 returns
 * PASTA_OK with nothing queued.  A CUDA error already pending in the calling
 * thread is reported (PASTA_E_CUDA) and left pending; a stream of another
 * device than the grid's is rejected (PASTA_E_ARG).  The calling thread's
 * current device is the same after the call as before.  Every evaluation
 * takes the FFT broadening path (blocks sized for the widest 2,048-tap
 * rotation kernel), so narrow kernels cost more than in pasta_chi2 and
 * their chi2 carries the FFT path's roundoff. */
int pasta_chi2_noalloc(const pasta_grid *g, const pasta_dispersion *d,
                       const pasta_continuum *c, const float *flux,
                       const float *var, int64_t n, const double *labels,
                       int64_t L, double *out, int32_t *status, void *stream);

/* ------------------------------------------------------------- fit
 * SingleFitter::fit / fit_bulk (fitting.rs:399-458; lib.rs:1478-1540) with
 * the particle swarm of particleswarm.rs:111-307.  S stars share the
 * dispersion and continuum fitter; flux/var are S x n.  seeds[S] select the
 * counter-based draw stream.  mode PASTA_FIT_BATCHED runs every star's
 * swarm on the device in one launch sequence per iteration captured in a
 * CUDA graph; PASTA_FIT_PLAIN runs one star at a time with the swarm update
 * on the host (the comparison baseline).  params: S x nparams floats.
 * trace (optional): (max_iters + 1) x num_particles x 6 doubles for star 0
 * (position, cost) after initialisation and after every iteration. */
int pasta_fit(const pasta_grid *g, const pasta_dispersion *d,
              const pasta_continuum *c, const pasta_pso_settings *settings,
              const float *flux, const float *var, int64_t n, int64_t S,
              const uint64_t *seeds, int mode, pasta_fit_result *results,
              float *params, double *trace);

/* Batched fit of S stars with their own dispersion, continuum fitter,
 * settings and pixel count (ragged batches: every star its own observed
 * wavelength grid).  params[i] receives pasta_continuum_nparams(c[i]) floats
 * (or is NULL). */
int pasta_fit_many(const pasta_grid *g, int64_t S,
                   const pasta_dispersion *const *d,
                   const pasta_continuum *const *c,
                   const pasta_pso_settings *settings,
                   const float *const *flux, const float *const *var,
                   const int64_t *n, const uint64_t *seeds, int mode,
                   pasta_fit_result *results, float *const *params);

/* SingleFitter::compute_uncertainty / compute_uncertainty_bulk
 * (fitting.rs:480-568, lib.rs:1545-1600): for each of S spectra (flux, var
 * [S x n], one dispersion and continuum fitter) and its best-fit label
 * (labels [S x 5]), the distances below and above each label where chi2
 * reaches chi2_best * (1 + sqrt(2 / n_eff)), n_eff = 4 spec_res (l_last -
 * l_first) / (l_first + l_last), found by Brent's method (tol 1e-3 in units
 * of the search radius).  search_radius [5] or NULL for (2000, 0.3, 0.3,
 * 40, 40); as in the reference the Teff radius is multiplied by Teff and the
 * vsini radius is max(vsini * r, 100).  out [S x 5 x 2] (label-major,
 * below then above) and bound_status [S x 5 x 2] (0 = found, else the
 * PASTA_E_* that stopped the search, out = NaN); star_status [S] is the
 * status of chi2 at the given label (non-zero fails all its bounds, where
 * the reference returns an error). */
int pasta_compute_uncertainty(const pasta_grid *g, const pasta_dispersion *d,
                              const pasta_continuum *c, int64_t S,
                              const float *flux, const float *var, int64_t n,
                              double spec_res, const double *labels,
                              const double *search_radius, double *out,
                              int32_t *bound_status, int32_t *star_status);

/* Step-wise batched fit (what pasta_fit_many runs): create uploads the
 * stars and places the swarms, step advances every swarm by `steps` PSO
 * steps (the first step evaluates the initial swarm) and reports the device
 * time between CUDA events on the library's stream, finish runs the final
 * refit and returns results.  profile_step runs one step stage by stage and
 * writes 12 doubles: stage times in ms (swarm update, prep, rotation
 * spectra, interpolation, fused broadening, unfused rotation + instrument
 * profile, resampling + chi2, best update), then the step's interpolated
 * pixels, evaluations, observed pixels and broadening blocks.  info: stars, particles, evaluations per
 * step, iterations, steps done, kernels per captured step.  No counterpart
 * in the reference (its fit runs to completion inside argmin's Executor). */
typedef struct pasta_batch pasta_batch;
int pasta_batch_create(const pasta_grid *g, int64_t S,
                       const pasta_dispersion *const *d,
                       const pasta_continuum *const *c,
                       const pasta_pso_settings *settings,
                       const float *const *flux, const float *const *var,
                       const int64_t *n, const uint64_t *seeds,
                       pasta_batch **out);
int pasta_batch_step(pasta_batch *b, int steps, double *device_ms);
int pasta_batch_profile_step(pasta_batch *b, double *out12);
int pasta_batch_info(const pasta_batch *b, int64_t *out6);
int pasta_batch_finish(pasta_batch *b, pasta_fit_result *results,
                       float *const *params);
int pasta_batch_destroy(pasta_batch *b);

/* ------------------------------------------------------- serving
 * Continuous batching: requests are admitted into device slots as slots and
 * HBM budget free up, every admitted star advances one PSO iteration per
 * device step, finished stars leave and new ones join without draining.
 * Each request carries its own dispersion and continuum fitter.  No
 * counterpart in the reference (its fit calls block one star at a time).
 * hbm_budget_bytes caps the device memory the running requests hold (their
 * spectra, swarm state and the evaluation workspace of their particles);
 * 0 = the 40% of the device's memory the evaluation workspace may take (or
 * PASTA_WORKSPACE_BYTES).  A request waits in the queue while admitting it
 * would exceed the budget and other requests are running. */
int pasta_server_create(const pasta_grid *g, int max_slots,
                        int64_t hbm_budget_bytes, pasta_server **out);
/* the server's HBM budget and the bytes its running requests hold */
int pasta_server_memory(const pasta_server *s, int64_t *budget, int64_t *used);
int pasta_server_submit(pasta_server *s, const pasta_dispersion *d,
                        const pasta_continuum *c,
                        const pasta_pso_settings *settings, const float *flux,
                        const float *var, int64_t n, uint64_t seed,
                        int64_t *request_id);
/* advance the device loop by one step: one PSO step of every occupied slot
 * (finished swarms are refitted in the same step), admission of queued
 * requests into free slots (while the step runs on the device; the new
 * slots join the next step, except that an idle server admits first) and
 * retirement of the finished requests; returns the number of active slots
 * after the step */
int pasta_server_step(pasta_server *s);
/* collect up to max finished results (non-blocking) */
int pasta_server_poll(pasta_server *s, int64_t *ids, pasta_fit_result *results,
                      float *params, int64_t params_stride, int max,
                      int *n_out);
int pasta_server_pending(const pasta_server *s, int64_t *queued,
                         int64_t *active, int64_t *done);
int pasta_server_destroy(pasta_server *s);
/* `steps` server steps back to back (admitting queued requests as slots
 * free up), timed between CUDA events on the library's stream (host work
 * between the launches is inside the interval). */
int pasta_server_run(pasta_server *s, int steps, double *device_ms);
/* out7: chi2 evaluations run, steps run, particles per slot, and the host
 * microseconds spent in steps before the device loop is launched
 * (admissions), waiting for it, after it (retirements), and of those in
 * the final refits. */
int pasta_server_stats(const pasta_server *s, int64_t *out7);

/* ---------------------------------------------------------- binaries
 * A binary label is star 1 (teff, m, logg, vsini, rv), star 2 (the same)
 * and the light ratio: 11 doubles.  cont_grid is the interpolator of the
 * unnormalised models that supplies each star's continuum; it must have the
 * same number of pixels as g (the reference indexes both with the same
 * synthetic pixel). */

/* Interpolator::interpolate_linear (interpolate.rs:985-1028; lib.rs:1127):
 * labels L x 3 (teff, m, logg), out L x n_synth. */
int pasta_interpolate_linear(const pasta_grid *g, const double *tml,
                             int64_t L, float *out, int32_t *status);
/* Interpolator::produce_binary_model_norm (interpolate.rs:822-893,
 * convolve_rv.rs:606-700; lib.rs:1019-1041): labels L x 11, out L x n_obs. */
int pasta_binary_model(const pasta_grid *g, const pasta_grid *cont_grid,
                       const pasta_dispersion *d, const double *labels,
                       int64_t L, float *out, int32_t *status);
/* BinaryFitter::chi2 via BinaryCostFunction::cost (fitting.rs:584-600,
 * 699-717; lib.rs:1673-1698): out[L] chi2 (NaN where status != 0). */
int pasta_binary_chi2(const pasta_grid *g, const pasta_grid *cont_grid,
                      const pasta_dispersion *d, const pasta_continuum *c,
                      const float *flux, const float *var, int64_t n,
                      const double *labels, int64_t L, double *out,
                      int32_t *status);

typedef struct {
  int32_t num_particles;
  int32_t max_iters;
  double inertia_factor, cognitive_factor, social_factor, delta;
  double vsini_lo, vsini_hi, rv_lo, rv_hi;
  /* per-parameter constraint over the 11 binary parameters:
   * 0 none, 1 fixed at a, 2 range [a, b] (lib.rs:817-835) */
  int32_t ckind[11];
  double ca[11], cb[11];
} pasta_binary_settings;

typedef struct {
  double label1[5], label2[5];
  double light_ratio;
  double chi2;
  double time;     /* seconds */
  int32_t iterations;
  int32_t status;  /* 0 ok, else PASTA_E_* of the failing particle */
  int32_t n_params;
  int32_t _pad;
} pasta_binary_result;

/* BinaryFitter::fit (fitting.rs:633-697; lib.rs:1636-1671): particle swarm
 * over the 11 parameters with the light ratio in (0, 1), on the draw stream
 * of `seed` (the single-star phases, dimensions 0..10).  Every particle of
 * an iteration is evaluated in one batch on the device.  params receives
 * pasta_continuum_nparams(c) floats (or is NULL); trace (or NULL) receives
 * (max_iters + 1) x num_particles x 12 doubles (position, cost). */
int pasta_binary_fit(const pasta_grid *g, const pasta_grid *cont_grid,
                     const pasta_dispersion *d, const pasta_continuum *c,
                     const pasta_binary_settings *settings,
                     const float *flux, const float *var, int64_t n,
                     uint64_t seed, pasta_binary_result *result,
                     float *params, double *trace);

#ifdef __cplusplus
}
#endif
#endif
