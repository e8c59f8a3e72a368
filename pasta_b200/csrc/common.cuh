// common.cuh -- types and __host__ __device__ helpers shared by the host
// engine and the sm_100a kernels of pasta_b200.
//
// Grid geometry, cubic coefficients, bounds and the draw stream restate the
// reference's algorithm (SimonVanSchuylenbergh/PASTA, src/interpolate.rs,
// src/cubic.rs, src/bounds.rs, src/particleswarm.rs) in code that runs both
// on the host (set-up, the plain path) and inside the kernels.
#pragma once
#include <stdint.h>

#include <cmath>

#ifdef __CUDACC__
#define PB_HD __host__ __device__ __forceinline__
#else
#define PB_HD inline
#endif

namespace pb {

constexpr double C_KMS = 299792.0;  // convolve_rv.rs:440, 547
constexpr int FFTN = 2048;          // convolve_rv.rs:433 (FFTSIZE)
constexpr int MAX_CHUNKS = 32;
constexpr int MAX_P1 = 16;          // polynomial order + 1
constexpr int MAX_LIN_K = 128;      // linear-model columns
constexpr int MAX_PARTICLES = 1024;
// the fused broadening kernel needs this many outputs per 2048-point block
constexpr int MIN_FUSED_OUTPUTS = 128;
// direct (non-FFT) broadening: outputs per tile, and the widest combined
// kernel (rotation taps + 2 x instrument half width) it takes
constexpr int DIRECT_TILE = 2048;
constexpr int DIRECT_MAX_TAPS = 512;

// Legendre recurrence in f32 with explicit rounding, evaluated identically
// by the host (Gram matrices) and the device (moments, continuum):
// P0 = 1, P1 = x, P(k+1) = fma(A_k x, P_k, -(C_k P(k-1))), A_k = (2k+1)/(k+1),
// C_k = k/(k+1) rounded to f32.
PB_HD float leg_a(int k) { return (float)((double)(2 * k + 1) / (double)(k + 1)); }
PB_HD float leg_c(int k) { return (float)((double)k / (double)(k + 1)); }
PB_HD float leg_step(float a, float c, float x, float pk, float pkm1) {
#ifdef __CUDA_ARCH__
  return __fmaf_rn(__fmul_rn(a, x), pk, -__fmul_rn(c, pkm1));
#else
  return std::fmaf(a * x, pk, -(c * pkm1));
#endif
}

// status codes (mirror include/pasta_b200.h)
enum : int {
  S_OK = 0,
  S_OUT_OF_GRID = -10,
  S_NEIGHBORS = -11,
  S_VSINI = -12,
  S_KERNEL_WIDTH = -13,
  S_RV_RANGE = -14,
  S_RESAMPLE = -15,
  S_BOUNDS = -16,
  S_CLAMP = -17,
  S_CONTINUUM = -18,
  S_NAN = -19,
  S_UNSUPPORTED = -20,
  S_INACTIVE = 1,  // slot without work this step (not an error)
};

enum { WL_LIN = 0, WL_LOG = 1, WL_NONUNI = 2 };
enum { DISP_NONE = 0, DISP_FIXED = 1, DISP_PIXEL = 2 };
enum { CONT_CHUNK = 0, CONT_LINEAR = 1, CONT_FIXED = 2, CONT_CONSTANT = 3 };

// ------------------------------------------------------------ device data
struct GridGeom {
  const double *tv, *mv, *lv;  // axis values
  const int *llo, *lhi;        // per-teff logg index limits
  const int64_t *cum;          // per-teff cumulative (teff, logg) count
  int nt, nm, nl;
};

struct DevGrid {
  GridGeom g;
  const uint16_t *spectra;  // [n_cols][stride] model-major (one row per model)
  const float *factor;      // [n_cols] f32 scale: max/65535 or 1/65535
  int64_t stride;           // row stride in uint16 (multiple of 64)
  int npx;
  int tail_start;           // npx - npx % 128 (interpolate.rs:969)
  int wl_kind;
  double wl_a, wl_b;        // Linspace (first, step) / Logspace (log10 first, step)
  const double *wl_vals;    // NonUniform values (device)
  double synth_first, synth_last;  // WlGrid::get_first_and_last
  double dvelo;             // rotation pixel velocity step (convolve_rv.rs:499-507), 0 if unsupported
};

// A star (or slot): observed spectrum + its dispersion and continuum tables.
struct DevStar {
  int n_obs;
  int disp_kind;     // DISP_*
  int gw;            // Gaussian width (odd) for DISP_FIXED / DISP_PIXEL
  int cont_kind;     // CONT_*
  int n_chunks, p1;  // chunk fitter
  int k_lin;         // linear model columns
  int ignore;        // fixed continuum ignore_first_and_last
  int cont_bad;      // continuum fitter cannot evaluate chi2 on this spectrum
  int obs_sorted;    // observed float indices never decrease (the resampling index is monotone)
  const float *flux, *var;
  const double *fidx;   // float index of every observed pixel in the synth grid
  const double *wl_obs; // observed wavelengths (NonUniform synth grids)
  double wl_first, wl_last;   // first/last observed wavelength (range check)
  double wl_min, wl_max;      // extreme observed wavelengths (windows on NonUniform grids)
  double fidx_min, fidx_max;  // extreme float indices (windows on uniform grids)
  const float *gk;      // DISP_FIXED: [gw]; DISP_PIXEL: [npx][gw]
  const float2 *gspec;  // DISP_FIXED: 2048-point spectrum of gk (1025 bins), else null
  const int *cstart, *cstop;  // chunk bounds
  const float *xa, *xb, *fac; // per observed pixel: coordinate in lower/upper chunk, blend factor
  const double *chol;   // per chunk: p1 x p1 lower Cholesky factor of the Legendre Gram (row-major)
  const float *q;       // linear: k x n_obs orthonormal basis (each basis vector contiguous)
  const float *qt;      // linear: the same basis pixel-major, kp columns (zero padded), for the tensor cores
  int kp;               // linear: basis columns padded to a multiple of 16 (0: no tensor-core path)
  const float *cont;    // fixed continuum
};

// Per-evaluation record written by the preparation kernel.
struct EvalPrep {
  int status;
  int star;
  int m;          // rotation kernel width (odd); 1 = identity
  int nblk;       // blocks of the broadening kernel (fused) or of the rotation FFT (unfused)
  int hg;         // instrument-profile half width (0: no instrument profile)
  int fused;      // 1: rotation and instrument profile in one kernel (k_broaden)
  int final_in_b; // 1: the broadened spectrum ends in buffer B, else in A
  int epi;        // 1: k_broaden resamples to the observed pixels itself (no synth row)
  int mobs_in_b;  // model at the observed pixels: 1 = row of B, 0 = row of A
  int direct;     // 1: broadened by direct convolution (k_direct) into B instead of the FFT kernels
  int ndt;        // direct tiles of (DIRECT_TILE - 2 hg) & ~3 outputs over [o_lo & ~3, o_hi)
  int o_lo, o_hi; // synth pixels the resampler reads [o_lo, o_hi)
  int g_lo, g_hi; // rotation outputs the Gaussian reads [g_lo, g_hi)
  int i_lo, i_hi; // interpolated pixels needed [i_lo, i_hi) (multiples of 8)
  double shift_log;    // Logspace: log10(1 - rv/c) / step
  double shift_factor; // 1 - rv/c
  double lin_offset;   // Linspace: (start / step) * (shift_factor - 1)
  double vsini;
  int cols[64];
  float w[64];
};

struct PsoParams {
  int P;
  int max_iters;
  double inertia, cognitive, social;
  double vs_lo, vs_hi, rv_lo, rv_hi;
  int ckind[5];
  double ca[5], cb[5];
  double mn[5], mx[5];  // constrained outer limits
};

// ------------------------------------------------------------ geometry
// Range::get_right_index (interpolate.rs:73-75): lower bound + exact match.
PB_HD int lower_bound(const double *v, int n, double x, bool &found) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (v[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  found = lo < n && v[lo] == x;
  return lo;
}

// Range::find_neighbors (interpolate.rs:105-159); -1 encodes None.
PB_HD int find_neighbors(const double *v, int n, double x, int left, int right, int out[4]) {
  bool found;
  int i = lower_bound(v, n, x, found);
  if (found) {
    if (i < left || i > right) return S_NEIGHBORS;
    if (i == left) { out[0] = -1; out[1] = i; out[2] = i + 1; out[3] = i + 2; }
    else if (i == right) { out[0] = i - 2; out[1] = i - 1; out[2] = i; out[3] = -1; }
    else if (i == right - 1) { out[0] = i - 2; out[1] = i - 1; out[2] = i; out[3] = i + 1; }
    else { out[0] = i - 1; out[1] = i; out[2] = i + 1; out[3] = i + 2; }
  } else {
    if (i <= left || i > right) return S_NEIGHBORS;
    if (i == left + 1) { out[0] = -1; out[1] = i - 1; out[2] = i; out[3] = i + 1; }
    else if (i == right) { out[0] = i - 2; out[1] = i - 1; out[2] = i; out[3] = -1; }
    else { out[0] = i - 2; out[1] = i - 1; out[2] = i; out[3] = i + 1; }
  }
  return S_OK;
}

// Grid::is_teff_logg_between_bounds (interpolate.rs:351-369)
PB_HD bool teff_logg_ok(const GridGeom &G, double t, double lg) {
  bool f;
  int i = lower_bound(G.tv, G.nt, t, f);
  if (f) return lg >= G.lv[G.llo[i]] && lg <= G.lv[G.lhi[i]];
  if (i == 0 || i == G.nt) return false;
  return lg >= G.lv[G.llo[i - 1]] && lg <= G.lv[G.lhi[i - 1]] && lg >= G.lv[G.llo[i]] &&
         lg <= G.lv[G.lhi[i]];
}
PB_HD bool m_ok(const GridGeom &G, double m) { return m >= G.mv[0] && m <= G.mv[G.nm - 1]; }

// Grid::get_logg_index_limits_at (interpolate.rs:378-398)
PB_HD int logg_index_limits_at(const GridGeom &G, double t, int &lo, int &hi) {
  bool f;
  int i = lower_bound(G.tv, G.nt, t, f);
  if (f) {
    if (i == G.nt - 1) { lo = G.llo[i]; hi = G.lhi[i]; return S_OK; }
    lo = G.llo[i] > G.llo[i + 1] ? G.llo[i] : G.llo[i + 1];
    hi = G.lhi[i] < G.lhi[i + 1] ? G.lhi[i] : G.lhi[i + 1];
    return S_OK;
  }
  if (i == 0 || i == G.nt) return S_OUT_OF_GRID;
  lo = G.llo[i - 1] > G.llo[i] ? G.llo[i - 1] : G.llo[i];
  hi = G.lhi[i - 1] < G.lhi[i] ? G.lhi[i - 1] : G.lhi[i];
  return S_OK;
}

// Grid::get_teff_index_limits_at (interpolate.rs:402-421)
PB_HD int teff_index_limits_at(const GridGeom &G, double lg, int &lo, int &hi) {
  lo = -1;
  hi = -1;
  for (int i = 0; i < G.nt; i++) {
    if (lg >= G.lv[G.llo[i]] && lg <= G.lv[G.lhi[i]]) {
      if (lo < 0) lo = i;
      hi = i;
    }
  }
  return lo < 0 ? S_OUT_OF_GRID : S_OK;
}

// cubic.rs:12-27
PB_HD void factors_quadratic(double x, double x0, double x1, double x2, bool start, double o[4]) {
  double xsq = x * x;
  double d0 = x0 * x0 - x0 * x1 - x0 * x2 + x1 * x2;
  double d1 = -x1 * x1 + x0 * x1 - x0 * x2 + x1 * x2;
  double d2 = x2 * x2 + x0 * x1 - x0 * x2 - x1 * x2;
  double f0 = (xsq - (x1 + x2) * x + x1 * x2) / d0;
  double f1 = (-xsq + (x0 + x2) * x - x0 * x2) / d1;
  double f2 = (xsq - (x0 + x1) * x + x0 * x1) / d2;
  if (start) { o[0] = 0.0; o[1] = f0; o[2] = f1; o[3] = f2; }
  else { o[0] = f0; o[1] = f1; o[2] = f2; o[3] = 0.0; }
}
// cubic.rs:29-60
PB_HD void factors_cubic(double x, double x0, double x1, double x2, double x3, double o[4]) {
  double xsq = x * x, xcu = xsq * x;
  double d0 = x0 * x0 * x0 - x0 * x0 * x1 - x0 * x0 * x2 - x0 * x0 * x3 + x0 * x1 * x2 +
              x0 * x1 * x3 + x0 * x2 * x3 - x1 * x2 * x3;
  double d1 = -x1 * x1 * x1 + x1 * x1 * x0 + x1 * x1 * x2 + x1 * x1 * x3 - x0 * x1 * x2 -
              x0 * x1 * x3 + x0 * x2 * x3 - x1 * x2 * x3;
  double d2 = x2 * x2 * x2 - x2 * x2 * x0 - x2 * x2 * x1 - x2 * x2 * x3 + x0 * x1 * x2 -
              x0 * x1 * x3 + x0 * x2 * x3 + x1 * x2 * x3;
  double d3 = -x3 * x3 * x3 + x3 * x3 * x0 + x3 * x3 * x1 + x3 * x3 * x2 + x0 * x1 * x2 -
              x0 * x1 * x3 - x0 * x2 * x3 - x1 * x2 * x3;
  o[0] = (xcu - (x1 + x2 + x3) * xsq + (x1 * x2 + x1 * x3 + x2 * x3) * x - (x1 * x2 * x3)) / d0;
  o[1] = (-xcu + (x0 + x2 + x3) * xsq - (x0 * x2 + x0 * x3 + x2 * x3) * x + (x0 * x2 * x3)) / d1;
  o[2] = (xcu - (x0 + x1 + x3) * xsq + (x0 * x1 + x0 * x3 + x1 * x3) * x - (x0 * x1 * x3)) / d2;
  o[3] = (-xcu + (x0 + x1 + x2) * xsq - (x0 * x1 + x0 * x2 + x1 * x2) * x + (x0 * x1 * x2)) / d3;
}
// cubic.rs:68-91 + 143-157 (mask bit i set = neighbour i present)
PB_HD int coeffs_from_neighbors(double x, int mask, const double val[4], double o[4]) {
  if (mask == 15) {
    double x0 = val[0], x1 = val[1], x2 = val[2], x3 = val[3];
    factors_cubic((x - x0) / (x3 - x0), 0.0, (x1 - x0) / (x3 - x0), (x2 - x0) / (x3 - x0), 1.0, o);
  } else if (mask == 7) {
    double x0 = val[0], x1 = val[1], x2 = val[2];
    factors_quadratic((x - x0) / (x2 - x0), 0.0, (x1 - x0) / (x2 - x0), 1.0, false, o);
  } else if (mask == 14) {
    double x0 = val[1], x1 = val[2], x2 = val[3];
    factors_quadratic((x - x0) / (x2 - x0), 0.0, (x1 - x0) / (x2 - x0), 1.0, true, o);
  } else if (mask == 0) {
    o[0] = o[1] = o[2] = o[3] = 0.0;
  } else {
    return S_NEIGHBORS;
  }
  return S_OK;
}

// Grid::get_local_grid + calculate_interpolation_coefficients
// (interpolate.rs:424-533, 934-949; cubic.rs:159-243).  Writes the 64
// column indices (-1 = missing) and f32 weights in the reference's order:
// teff neighbour c (outer), logg neighbour r, [M/H] neighbour k (inner).
PB_HD int local_grid(const GridGeom &G, double t, double m, double lg, int cols[64], float w[64],
                     double *ft_out = nullptr, double *fl_out = nullptr, double *fm_out = nullptr) {
  if (t != t || m != m || lg != lg) return S_NAN;
  if (!teff_logg_ok(G, t, lg)) return S_OUT_OF_GRID;
  if (!m_ok(G, m)) return S_OUT_OF_GRID;
  int tlo, thi, llo, lhi;
  int st = teff_index_limits_at(G, lg, tlo, thi);
  if (st) return st;
  st = logg_index_limits_at(G, t, llo, lhi);
  if (st) return st;
  int tn[4], mn[4], ln[4];
  if (find_neighbors(G.tv, G.nt, t, tlo, thi, tn)) return S_NEIGHBORS;
  if (find_neighbors(G.mv, G.nm, m, 0, G.nm - 1, mn)) return S_NEIGHBORS;
  if (find_neighbors(G.lv, G.nl, lg, llo, lhi, ln)) return S_NEIGHBORS;
  int ok = 0;  // bit r*4+c
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++)
      if (tn[c] >= 0 && ln[r] >= 0 && ln[r] >= G.llo[tn[c]] && ln[r] <= G.lhi[tn[c]]) ok |= 1 << (r * 4 + c);
  double tv[4], lv[4], mv[4];
  int mmask = 0;
  for (int i = 0; i < 4; i++) {
    tv[i] = tn[i] >= 0 ? G.tv[tn[i]] : 0.0;
    lv[i] = ln[i] >= 0 ? G.lv[ln[i]] : 0.0;
    mv[i] = mn[i] >= 0 ? G.mv[mn[i]] : 0.0;
    if (mn[i] >= 0) mmask |= 1 << i;
  }
  double ft[16], fl[16], fm[4], o[4];
  for (int r = 0; r < 4; r++) {  // teff factors along logg row r
    int mask = (ok >> (r * 4)) & 15;
    if (coeffs_from_neighbors(t, mask, tv, o)) return S_NEIGHBORS;
    for (int c = 0; c < 4; c++) ft[r * 4 + c] = o[c];
  }
  for (int c = 0; c < 4; c++) {  // logg factors down teff column c
    int mask = 0;
    for (int r = 0; r < 4; r++) if (ok & (1 << (r * 4 + c))) mask |= 1 << r;
    if (coeffs_from_neighbors(lg, mask, lv, o)) return S_NEIGHBORS;
    for (int r = 0; r < 4; r++) fl[r * 4 + c] = o[r];
  }
  if (coeffs_from_neighbors(m, mmask, mv, fm)) return S_NEIGHBORS;
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++) {
      double a = ft[r * 4 + c] * fl[r * 4 + c];
      bool pres = (ok >> (r * 4 + c)) & 1;
      for (int k = 0; k < 4; k++) {
        int idx = (c * 4 + r) * 4 + k;
        w[idx] = (float)(a * fm[k]);
        if (pres && mn[k] >= 0) {
          int i = tn[c];
          cols[idx] = (int)((G.cum[i] + ln[r] - G.llo[i]) * (int64_t)G.nm + mn[k]);
        } else {
          cols[idx] = -1;
        }
      }
    }
  if (ft_out) for (int i = 0; i < 16; i++) ft_out[i] = ft[i];
  if (fl_out) for (int i = 0; i < 16; i++) fl_out[i] = fl[i];
  if (fm_out) for (int i = 0; i < 4; i++) fm_out[i] = fm[i];
  return S_OK;
}

// Range::find_neighbors_linear (interpolate.rs:161-213): the two grid
// points around x.  A grid point at the right limit takes its left partner
// (none at index 0, where the reference's usize subtraction panics).
PB_HD int find_neighbors_linear(const double *v, int n, double x, int left, int right, int out[2]) {
  bool found;
  int i = lower_bound(v, n, x, found);
  if (found) {
    if (i < left || i > right) return S_NEIGHBORS;
    if (i == right) {
      if (i == 0) return S_NEIGHBORS;
      out[0] = i - 1; out[1] = i;
    } else {
      out[0] = i; out[1] = i + 1;
    }
  } else {
    if (i <= left || i > right) return S_NEIGHBORS;
    out[0] = i - 1; out[1] = i;
  }
  return S_OK;
}

// Grid::get_local_grid_linear + calculate_interpolation_coefficients_linear
// (interpolate.rs:536-600; cubic.rs:6-10, 246-270): the 8 corners of the
// cube around the label, teff outer, logg middle, [M/H] inner, with f32
// weights (a * b * c).  A corner whose logg index lies outside its teff's
// logg limits has no model: S_NEIGHBORS (the reference would read a
// neighbouring column there).
PB_HD int local_grid_linear(const GridGeom &G, double t, double m, double lg, int cols[8], float w[8]) {
  if (t != t || m != m || lg != lg) return S_NAN;
  if (!teff_logg_ok(G, t, lg)) return S_OUT_OF_GRID;
  if (!m_ok(G, m)) return S_OUT_OF_GRID;
  int tlo, thi, llo, lhi;
  int st = teff_index_limits_at(G, lg, tlo, thi);
  if (st) return st;
  st = logg_index_limits_at(G, t, llo, lhi);
  if (st) return st;
  int tn[2], mn[2], ln[2];
  if (find_neighbors_linear(G.tv, G.nt, t, tlo, thi, tn)) return S_NEIGHBORS;
  if (find_neighbors_linear(G.mv, G.nm, m, 0, G.nm - 1, mn)) return S_NEIGHBORS;
  if (find_neighbors_linear(G.lv, G.nl, lg, llo, lhi, ln)) return S_NEIGHBORS;
  double ft[2], fl[2], fm[2];
  ft[0] = (t - G.tv[tn[1]]) / (G.tv[tn[0]] - G.tv[tn[1]]);
  ft[1] = (t - G.tv[tn[0]]) / (G.tv[tn[1]] - G.tv[tn[0]]);
  fl[0] = (lg - G.lv[ln[1]]) / (G.lv[ln[0]] - G.lv[ln[1]]);
  fl[1] = (lg - G.lv[ln[0]]) / (G.lv[ln[1]] - G.lv[ln[0]]);
  fm[0] = (m - G.mv[mn[1]]) / (G.mv[mn[0]] - G.mv[mn[1]]);
  fm[1] = (m - G.mv[mn[0]]) / (G.mv[mn[1]] - G.mv[mn[0]]);
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) {
      const int i = tn[a];
      if (ln[b] < G.llo[i] || ln[b] > G.lhi[i]) return S_NEIGHBORS;
      for (int c = 0; c < 2; c++) {
        const int idx = (a * 2 + b) * 2 + c;
        w[idx] = (float)(ft[a] * fl[b] * fm[c]);
        cols[idx] = (int)((G.cum[i] + ln[b] - G.llo[i]) * (int64_t)G.nm + mn[c]);
      }
    }
  return S_OK;
}

// Grid::get_limits_at (interpolate.rs:647-664)
PB_HD int grid_limits_at(const GridGeom &G, const double *p, int index, double &lo, double &hi) {
  int a, b, st;
  if (index == 0) {
    st = teff_index_limits_at(G, p[2], a, b);
    if (st) return st;
    lo = G.tv[a]; hi = G.tv[b];
  } else if (index == 1) {
    lo = G.mv[0]; hi = G.mv[G.nm - 1];
  } else {
    st = logg_index_limits_at(G, p[0], a, b);
    if (st) return st;
    lo = G.lv[a]; hi = G.lv[b];
  }
  return S_OK;
}

// ConstrainedPSOBounds<SingleBounds>::get_limits_at (bounds.rs:112-115, 168-176)
PB_HD int pso_limits_at(const GridGeom &G, const PsoParams &S, const double *p, int i, double &lo, double &hi) {
  if (i == 3) { lo = S.vs_lo; hi = S.vs_hi; }
  else if (i == 4) { lo = S.rv_lo; hi = S.rv_hi; }
  else {
    int st = grid_limits_at(G, p, i, lo, hi);
    if (st) return st;
  }
  if (S.ckind[i] == 1) { lo = S.ca[i]; hi = S.ca[i]; }
  else if (S.ckind[i] == 2) { lo = lo > S.ca[i] ? lo : S.ca[i]; hi = hi < S.cb[i] ? hi : S.cb[i]; }
  return S_OK;
}

// PSOBounds::clamp_1d (bounds.rs:13-16); f64::clamp panics on lo > hi.
PB_HD int pso_clamp_1d(const GridGeom &G, const PsoParams &S, const double *p, int i, double &out) {
  double lo, hi;
  int st = pso_limits_at(G, S, p, i, lo, hi);
  if (st) return st;
  if (!(lo <= hi)) return S_CLAMP;
  double x = p[i];
  out = x < lo ? lo : (x > hi ? hi : x);
  return S_OK;
}

// ConstrainedPSOBounds::is_within_bounds (bounds.rs:117-129, 178-185)
PB_HD bool pso_within(const GridGeom &G, const PsoParams &S, const double *p) {
  if (!(m_ok(G, p[1]) && teff_logg_ok(G, p[0], p[2]))) return false;
  if (!(p[3] >= S.vs_lo && p[3] <= S.vs_hi && p[4] >= S.rv_lo && p[4] <= S.rv_hi)) return false;
  for (int i = 0; i < 5; i++) {
    if (S.ckind[i] == 1) {
      double d = p[i] - S.ca[i];
      if (!((d < 0 ? -d : d) <= 2.220446049250313e-16)) return false;
    } else if (S.ckind[i] == 2) {
      if (!(p[i] >= S.ca[i] && p[i] <= S.cb[i])) return false;
    }
  }
  return true;
}

// ------------------------------------------------------------ draws
// Counter-based stream shared with the oracle: SplitMix64 finaliser
// (Steele, Lea & Flood 2014) over (seed, phase, a, b, c).
PB_HD uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
PB_HD double draw_u01(uint64_t seed, uint64_t phase, uint64_t a, uint64_t b, uint64_t c) {
  uint64_t h = mix64(seed);
  h = mix64(h ^ ((phase << 56) | (a & 0x00FFFFFFFFFFFFFFull)));
  h = mix64(h ^ ((b << 32) | (c & 0xFFFFFFFFull)));
  return (double)(h >> 11) * 1.1102230246251565e-16;  // 2^-53
}
// random_uniform (particleswarm.rs:153-161) with gen_range(lo..hi) = u*(hi-lo)+lo
PB_HD double uniform_between(double a, double b, double u) {
  if (a == b) return a;
  double lo = a < b ? a : b, hi = a < b ? b : a;
#ifdef __CUDA_ARCH__
  return __dadd_rn(__dmul_rn(u, __dsub_rn(hi, lo)), lo);
#else
  return u * (hi - lo) + lo;
#endif
}
enum { PH_INIT_POS = 1, PH_INIT_VEL = 2, PH_ITER = 3 };

// ------------------------------------------------------------ rotation
// Width of the rotation kernel (convolve_rv.rs:438-449); 0 when vsini <= 0.
PB_HD int rotation_width(double vsini, double dvelo) {
  const double eps = 0.6;
  double vrot = vsini / C_KMS;
  double q = 4.0 * (eps - 1.0) / (3.141592653589793 * eps);
  double wdt = 2.0 * vrot / dvelo * sqrt(1.0 + q * q);
  if (!(wdt < 1e8)) return 1 << 30;
  double c = ceil(wdt);
  long long nme = (c > 0 ? (long long)c : 0) + 2;
  if (nme < 1) nme = 1;
  return (int)(nme + 1 - nme % 2);
}

}  // namespace pb
