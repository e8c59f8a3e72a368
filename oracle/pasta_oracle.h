/*
 * pasta_oracle.h -- CPU oracle for the PASTA per-particle hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path
 * and the timed CPU baseline.  The product (pasta_b200) never links, loads or
 * calls it; only tests/, __graft_entry__.smoke() and bench.py's CPU legs do.
 *
 * It restates the reference's Rust algorithm (SimonVanSchuylenbergh/PASTA,
 * the src/ directory) in C++ in two precisions:
 *   OP_F32 : "FP32 mirror" -- the reference's dtypes and operation order,
 *            including its quirks (tail pixels scaled by an extra 1/65535,
 *            the resampling index rounded to f32 before the weight is formed,
 *            the per-fitter chi2 normalisations).  Where the reference calls a
 *            third-party numeric routine the mirror substitutes its own:
 *            realfft/rustfft -> own radix-2 real FFT of 2048 with the same
 *            overlap-add blocking; nalgebra f32 SVD least squares -> f32
 *            Householder QR least squares.  Those substitutions match the
 *            reference to roundoff, not bitwise.
 *   OP_F64 : the same algorithm and the same discrete choices (quirks kept)
 *            with all arithmetic in double; convolutions are direct sums and
 *            least squares is a double Householder QR.
 *
 * Parity status: UNPINNED by reference outputs.  The reference is Rust (no
 * cargo/rustc here), ships no tests, fixtures or golden vectors, and its
 * benchmark data is not public.  The oracle is pinned by analytic
 * known-answer tests (tests/test_oracle_kat.py) and by committed fixtures
 * it generated itself (tests/golden/).
 *
 * PSO draws: the reference's RNG is unseeded (StdRng::from_entropy).  Both
 * this oracle and the CUDA path consume one counter-based stream
 * (pasta_draw_u01: SplitMix64 finaliser over (seed, phase, a, b, c)), so a
 * seeded fit is replayable exactly.
 */
#ifndef PASTA_ORACLE_H
#define PASTA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OP_F32 = 0, OP_F64 = 1 };
enum { OWL_LINSPACE = 0, OWL_LOGSPACE = 1, OWL_NONUNIFORM = 2 };
enum { ODISP_NONE = 0, ODISP_FIXED = 1, ODISP_VARIABLE = 2 };
enum { OCONT_CHUNK = 0, OCONT_LINEAR = 1, OCONT_FIXED = 2, OCONT_CONSTANT = 3 };

typedef struct OGrid OGrid;
typedef struct ODisp ODisp;
typedef struct OCont OCont;

const char *or_last_error(void);

/* Grid: labels n x (teff, m, logg); spectra n x npx uint16, row i belongs to
 * labels[i]; factors[i] is the includes_factor f32 maximum read from the
 * file's first four bytes (model_fetchers.rs:53-63), or NULL (scale 1/65535). */
OGrid *or_grid_create(const double *labels, const uint16_t *spectra,
                      const float *factors, int64_t n_models, int64_t npx,
                      int wl_kind, double wl_a, double wl_b,
                      const double *wl_values);
void or_grid_free(OGrid *g);
/* axis sizes and geometry (for tests of the host logic) */
int or_grid_axes(const OGrid *g, int *n_teff, int *n_m, int *n_logg);
int or_grid_axis_values(const OGrid *g, int axis, double *out);
int or_grid_logg_limits(const OGrid *g, int *lo, int *hi);
/* 64 column indices (-1 for a missing neighbour) and weights for a label */
int or_local_grid(const OGrid *g, double teff, double m, double logg,
                  int64_t *cols, double *weights64);
int or_is_within_bounds(const OGrid *g, double teff, double m, double logg);
int or_limits_at(const OGrid *g, const double *tml, int index, double *lo,
                 double *hi);

/* interpolate(teff, m, logg) -> npx values */
int or_interpolate(const OGrid *g, int prec, double teff, double m,
                   double logg, double *out);
/* rotation kernel (convolve_rv.rs:438) */
int or_rotation_kernel(double vsini, double dvelo, double *out, int cap);
/* convolve_rotation on an arbitrary input of the grid's length */
int or_convolve_rotation(const OGrid *g, int prec, const double *in,
                         double vsini, double *out);

/* Dispersions. fixed: resolution > 0; variable: disp[n_obs] (sigma in A). */
ODisp *or_disp_create(const OGrid *g, int kind, const double *wl_obs,
                      int64_t n_obs, double resolution, const float *disp);
void or_disp_free(ODisp *d);
int or_disp_convolve(const ODisp *d, int prec, const double *in, double *out);
int or_disp_kernel_width(const ODisp *d);

int or_produce_model(const OGrid *g, const ODisp *d, int prec,
                     const double *label5, double *out_obs);

/* Continuum fitters (continuum_fitting.rs). design is n x k row-major. */
OCont *or_cont_create(int kind, const double *wl, int64_t n, int n_chunks,
                      int p_order, double overlap, const float *design, int k,
                      const float *continuum, int ignore_first_and_last);
void or_cont_free(OCont *c);
int or_cont_nparams(const OCont *c);
int or_cont_chunk_bounds(const OCont *c, int64_t *startstop);
int or_fit_continuum(const OCont *c, int prec, const float *flux,
                     const float *var, const double *model, int64_t n,
                     double *params, double *chi2);
int or_build_continuum(const OCont *c, int prec, const double *params,
                       double *out);

/* cost (fitting.rs:313) for L labels; status per label (0 ok) */
int or_chi2(const OGrid *g, const ODisp *d, const OCont *c, int prec,
            const float *flux, const float *var, int64_t n,
            const double *labels, int64_t L, double *out, int *status,
            int nthreads);

/* PSO fit (fitting.rs:399 + particleswarm.rs). */
typedef struct {
  int num_particles;
  int max_iters;
  double inertia, cognitive, social, delta;
  double vsini_lo, vsini_hi, rv_lo, rv_hi;
  /* constraints per parameter: kind 0 none, 1 fixed(a), 2 range(a, b) */
  int ckind[5];
  double ca[5], cb[5];
} OPsoSettings;

typedef struct {
  double label[5];
  double chi2;
  int iterations;
  int status;
  int n_params;
  double params[512];
} OFitResult;

/* Fit S stars that share grid/dispersion/continuum.  flux/var are S x n.
 * Star s uses seed seeds[s].  Threads over stars (fit_bulk) when
 * threads_over_stars, else over particles (fit with parallelize=true).
 * trace (optional, may be NULL): (max_iters+1) x P x 6 per star 0 (position,
 * cost) after init (sorted) and after every iteration. */
int or_fit(const OGrid *g, const ODisp *d, const OCont *c, int prec,
           const OPsoSettings *st, const float *flux, const float *var,
           int64_t n, int64_t S, const uint64_t *seeds, int nthreads,
           int threads_over_stars, OFitResult *out, double *trace);

/* ------------------------------------------------------------- binaries */
/* 8 column indices and f64 weights of the linear interpolation
 * (interpolate.rs:536-600, cubic.rs:246-270) */
int or_local_grid_linear(const OGrid *g, double teff, double m, double logg,
                         int64_t *cols, double *w);
/* interpolate_linear(teff, m, logg) -> npx values (interpolate.rs:985) */
int or_interpolate_linear(const OGrid *g, int prec, double teff, double m,
                          double logg, double *out);
/* produce_binary_model_norm (interpolate.rs:868): lab = star 1 [5],
 * star 2 [5], light ratio; gc is the continuum grid; out [n_obs] */
int or_binary_model(const OGrid *g, const OGrid *gc, const ODisp *d, int prec,
                    const double *lab, double *out);
/* BinaryCostFunction::cost (fitting.rs:584) for L labels [L x 11] */
int or_binary_chi2(const OGrid *g, const OGrid *gc, const ODisp *d,
                   const OCont *c, int prec, const float *flux,
                   const float *var, int64_t n, const double *labels,
                   int64_t L, double *out, int *status, int nthreads);

typedef struct {
  int num_particles;
  int max_iters;
  double inertia, cognitive, social, delta;
  double vsini_lo, vsini_hi, rv_lo, rv_hi;
  int ckind[11];
  double ca[11], cb[11];
} OBinarySettings;

typedef struct {
  double label1[5], label2[5];
  double light_ratio;
  double chi2;
  int iterations;
  int status;
  int n_params;
  double params[512];
} OBinaryResult;

/* BinaryFitter::fit (fitting.rs:633-697); particles threaded over
 * nthreads.  trace (optional): (max_iters+1) x P x 12 (position, cost). */
int or_binary_fit(const OGrid *g, const OGrid *gc, const ODisp *d,
                  const OCont *c, int prec, const OBinarySettings *st,
                  const float *flux, const float *var, int64_t n,
                  uint64_t seed, int nthreads, OBinaryResult *out,
                  double *trace);

/* the shared PSO draw stream */
double or_draw_u01(uint64_t seed, uint64_t phase, uint64_t a, uint64_t b,
                   uint64_t c);

#ifdef __cplusplus
}
#endif
#endif
