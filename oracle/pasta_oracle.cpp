// pasta_oracle.cpp -- CPU oracle for the PASTA per-particle hot path.
//
// TEST INFRASTRUCTURE ONLY (see pasta_oracle.h): the checker for the CUDA
// path and the timed CPU baseline.  Never linked into the product.
//
// Each function names the reference function it restates
// (SimonVanSchuylenbergh/PASTA, paths relative to the project root).
// Parity status: unpinned by reference outputs; pinned by analytic
// known-answer tests.
#include "pasta_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;
struct OErr : std::runtime_error {
  using std::runtime_error::runtime_error;
};
[[noreturn]] void fail(const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  throw OErr(buf);
}

constexpr double C_KMS = 299792.0;  // convolve_rv.rs:440, 547
constexpr int FFTSIZE = 2048;       // convolve_rv.rs:433

// ---------------------------------------------------------------- geometry
// interpolate.rs:66-250 (Range)
struct Range {
  std::vector<double> v;
  int n() const { return (int)v.size(); }
  // binary_search_by(partial_cmp): found -> (true, i), else (false, insertion)
  std::pair<bool, int> search(double x) const {
    if (std::isnan(x)) fail("NaN label");
    int i = (int)(std::lower_bound(v.begin(), v.end(), x) - v.begin());
    if (i < n() && v[i] == x) return {true, i};
    return {false, i};
  }
  // interpolate.rs:105-159
  void find_neighbors(double x, int left, int right, int out[4]) const {
    auto r = search(x);
    int i = r.second;
    if (r.first) {
      if (i < left) fail("Index %d out of left bound, x=%g", i, x);
      if (i > right) fail("Index %d out of right bound, x=%g", i, x);
      if (i == left) { out[0] = -1; out[1] = i; out[2] = i + 1; out[3] = i + 2; }
      else if (i == right) { out[0] = i - 2; out[1] = i - 1; out[2] = i; out[3] = -1; }
      else if (i == right - 1) { out[0] = i - 2; out[1] = i - 1; out[2] = i; out[3] = i + 1; }
      else { out[0] = i - 1; out[1] = i; out[2] = i + 1; out[3] = i + 2; }
    } else {
      if (i <= left) fail("Index %d out of left bound, x=%g", i, x);
      if (i > right) fail("Index %d out of right bound, x=%g", i, x);
      if (i == left + 1) { out[0] = -1; out[1] = i - 1; out[2] = i; out[3] = i + 1; }
      else if (i == right) { out[0] = i - 2; out[1] = i - 1; out[2] = i; out[3] = -1; }
      else { out[0] = i - 2; out[1] = i - 1; out[2] = i; out[3] = i + 1; }
    }
  }
};

struct WlGrid {  // interpolate.rs:672-744
  int kind = OWL_LOGSPACE;
  double a = 0, b = 0;
  int64_t n = 0;
  std::vector<double> vals;
  std::pair<double, double> first_last() const {
    if (kind == OWL_LINSPACE) return {a, a + b * (double)n};
    if (kind == OWL_LOGSPACE) return {std::pow(10.0, a), std::pow(10.0, a + b * (double)n)};
    return {vals[0], vals[vals.size() - 1]};
  }
  double float_index(double wl) const {
    if (kind == OWL_LINSPACE) return (wl - a) / b;
    if (kind == OWL_LOGSPACE) return (std::log10(wl) - a) / b;
    auto it = std::lower_bound(vals.begin(), vals.end(), wl);
    int64_t i = it - vals.begin();
    if (i < (int64_t)vals.size() && vals[i] == wl) return (double)i;
    if (i == 0) return 0.0;
    if (i == (int64_t)vals.size()) return (double)vals.size() - 1.0;
    double left = vals[i - 1], right = vals[i];
    return (wl - left) / (right - left) + (double)i - 1.0;
  }
  double at(int64_t i) const {
    if (kind == OWL_LINSPACE) return a + b * (double)i;
    if (kind == OWL_LOGSPACE) return std::pow(10.0, a + b * (double)i);
    return vals[i];
  }
};

}  // namespace

struct OGrid {
  Range teff, m, logg;
  std::vector<std::pair<int, int>> logg_limits;
  std::vector<int64_t> cum;
  std::vector<uint16_t> spectra;  // columns in list_gridpoints order
  std::vector<float> factors;     // per column, f32 max/65535 (model_fetchers.rs:62)
  std::vector<double> factors64;  // per column, the same scale formed in double
  int64_t npx = 0;
  WlGrid wl;

  int64_t column(int i, int j, int k) const {  // model_fetchers.rs:233-236
    return (cum[i] + k - logg_limits[i].first) * (int64_t)m.n() + j;
  }
  // interpolate.rs:351-369
  bool teff_logg_ok(double t, double lg) const {
    auto r = teff.search(t);
    if (r.first) {
      auto b = logg_limits[r.second];
      return lg >= logg.v[b.first] && lg <= logg.v[b.second];
    }
    int i = r.second;
    if (i == 0 || i == teff.n()) return false;
    auto l = logg_limits[i - 1], rr = logg_limits[i];
    return lg >= logg.v[l.first] && lg <= logg.v[l.second] &&
           lg >= logg.v[rr.first] && lg <= logg.v[rr.second];
  }
  bool m_ok(double x) const { return x >= m.v.front() && x <= m.v.back(); }
  // interpolate.rs:378-398
  std::pair<int, int> logg_index_limits_at(double t) const {
    auto r = teff.search(t);
    if (r.first) {
      int i = r.second;
      if (i == teff.n() - 1) return logg_limits[i];
      auto l = logg_limits[i], rr = logg_limits[i + 1];
      return {std::max(l.first, rr.first), std::min(l.second, rr.second)};
    }
    int i = r.second;
    if (i == 0 || i == teff.n()) fail("Teff out of bounds");
    auto l = logg_limits[i - 1], rr = logg_limits[i];
    return {std::max(l.first, rr.first), std::min(l.second, rr.second)};
  }
  // interpolate.rs:402-421
  std::pair<int, int> teff_index_limits_at(double lg) const {
    int lo = -1, hi = -1;
    for (int i = 0; i < teff.n(); i++) {
      auto b = logg_limits[i];
      if (lg >= logg.v[b.first] && lg <= logg.v[b.second]) {
        if (lo < 0) lo = i;
        hi = i;
      }
    }
    if (lo < 0) fail("No teff bounds at logg=%g", lg);
    return {lo, hi};
  }
  // interpolate.rs:647-664
  std::pair<double, double> limits_at(const double *p, int index) const {
    if (index == 0) {
      auto l = teff_index_limits_at(p[2]);
      return {teff.v[l.first], teff.v[l.second]};
    }
    if (index == 1) return {m.v.front(), m.v.back()};
    if (index == 2) {
      auto l = logg_index_limits_at(p[0]);
      return {logg.v[l.first], logg.v[l.second]};
    }
    fail("Index out of bounds %d", index);
  }
  bool within(const double *p) const { return m_ok(p[1]) && teff_logg_ok(p[0], p[2]); }
};

namespace {

// cubic.rs:12-27
void factors_quadratic(double x, double x0, double x1, double x2, bool start, double out[4]) {
  double xsq = x * x;
  double d0 = x0 * x0 - x0 * x1 - x0 * x2 + x1 * x2;
  double d1 = -x1 * x1 + x0 * x1 - x0 * x2 + x1 * x2;
  double d2 = x2 * x2 + x0 * x1 - x0 * x2 - x1 * x2;
  double f0 = (xsq - (x1 + x2) * x + x1 * x2) / d0;
  double f1 = (-xsq + (x0 + x2) * x - x0 * x2) / d1;
  double f2 = (xsq - (x0 + x1) * x + x0 * x1) / d2;
  if (start) { out[0] = 0; out[1] = f0; out[2] = f1; out[3] = f2; }
  else { out[0] = f0; out[1] = f1; out[2] = f2; out[3] = 0; }
}
// cubic.rs:29-60
void factors_cubic(double x, double x0, double x1, double x2, double x3, double out[4]) {
  double xsq = x * x, xcu = xsq * x;
  double d0 = x0 * x0 * x0 - x0 * x0 * x1 - x0 * x0 * x2 - x0 * x0 * x3 + x0 * x1 * x2 +
              x0 * x1 * x3 + x0 * x2 * x3 - x1 * x2 * x3;
  double d1 = -x1 * x1 * x1 + x1 * x1 * x0 + x1 * x1 * x2 + x1 * x1 * x3 - x0 * x1 * x2 -
              x0 * x1 * x3 + x0 * x2 * x3 - x1 * x2 * x3;
  double d2 = x2 * x2 * x2 - x2 * x2 * x0 - x2 * x2 * x1 - x2 * x2 * x3 + x0 * x1 * x2 -
              x0 * x1 * x3 + x0 * x2 * x3 + x1 * x2 * x3;
  double d3 = -x3 * x3 * x3 + x3 * x3 * x0 + x3 * x3 * x1 + x3 * x3 * x2 + x0 * x1 * x2 -
              x0 * x1 * x3 - x0 * x2 * x3 - x1 * x2 * x3;
  out[0] = (xcu - (x1 + x2 + x3) * xsq + (x1 * x2 + x1 * x3 + x2 * x3) * x - (x1 * x2 * x3)) / d0;
  out[1] = (-xcu + (x0 + x2 + x3) * xsq - (x0 * x2 + x0 * x3 + x2 * x3) * x + (x0 * x2 * x3)) / d1;
  out[2] = (xcu - (x0 + x1 + x3) * xsq + (x0 * x1 + x0 * x3 + x1 * x3) * x - (x0 * x1 * x3)) / d2;
  out[3] = (-xcu + (x0 + x1 + x2) * xsq - (x0 * x1 + x0 * x2 + x1 * x2) * x + (x0 * x1 * x2)) / d3;
}
// cubic.rs:68-91 + 143-157; present[i] false = None
void coeffs_from_neighbors(double x, const bool present[4], const double val[4], double out[4]) {
  bool p0 = present[0], p1 = present[1], p2 = present[2], p3 = present[3];
  if (p0 && p1 && p2 && p3) {
    double x0 = val[0], x1 = val[1], x2 = val[2], x3 = val[3];
    factors_cubic((x - x0) / (x3 - x0), 0.0, (x1 - x0) / (x3 - x0), (x2 - x0) / (x3 - x0), 1.0, out);
  } else if (p0 && p1 && p2 && !p3) {
    double x0 = val[0], x1 = val[1], x2 = val[2];
    factors_quadratic((x - x0) / (x2 - x0), 0.0, (x1 - x0) / (x2 - x0), 1.0, false, out);
  } else if (!p0 && p1 && p2 && p3) {
    double x0 = val[1], x1 = val[2], x2 = val[3];
    factors_quadratic((x - x0) / (x2 - x0), 0.0, (x1 - x0) / (x2 - x0), 1.0, true, out);
  } else if (!p0 && !p1 && !p2 && !p3) {
    out[0] = out[1] = out[2] = out[3] = 0.0;
  } else {
    fail("Not enough neighbors: %g", x);
  }
}

// interpolate.rs:424-533 + cubic.rs:159-243.  cols[64]: -1 for None.
// w64 holds the f64 products (a*b) before the f32 cast of cubic.rs:241.
void local_grid(const OGrid &g, double t, double mm, double lg, int64_t cols[64], double w64[64]) {
  if (!g.teff_logg_ok(t, lg)) fail("Teff, logg out of bounds (%g, %g)", t, lg);
  if (!g.m_ok(mm)) fail("M out of bounds (%g)", mm);
  auto tl = g.teff_index_limits_at(lg);
  auto ll = g.logg_index_limits_at(t);
  int tn[4], mn[4], ln[4];
  g.teff.find_neighbors(t, tl.first, tl.second, tn);
  g.m.find_neighbors(mm, 0, g.m.n() - 1, mn);
  g.logg.find_neighbors(lg, ll.first, ll.second, ln);
  // idx[r][c]: logg neighbour r (row), teff neighbour c (column)
  bool ok[4][4];
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++) {
      ok[r][c] = false;
      if (tn[c] >= 0 && ln[r] >= 0) {
        auto lim = g.logg_limits[tn[c]];
        ok[r][c] = ln[r] >= lim.first && ln[r] <= lim.second;
      }
    }
  double tv[4], lv[4], mv[4];
  bool mp[4];
  for (int i = 0; i < 4; i++) {
    tv[i] = tn[i] >= 0 ? g.teff.v[tn[i]] : 0.0;
    lv[i] = ln[i] >= 0 ? g.logg.v[ln[i]] : 0.0;
    mv[i] = mn[i] >= 0 ? g.m.v[mn[i]] : 0.0;
    mp[i] = mn[i] >= 0;
  }
  double ft[4][4], fl[4][4], fm[4];
  for (int r = 0; r < 4; r++) {  // map_rows: teff factors along each logg row
    bool pres[4];
    for (int c = 0; c < 4; c++) pres[c] = ok[r][c];
    double o[4];
    coeffs_from_neighbors(t, pres, tv, o);
    for (int c = 0; c < 4; c++) ft[r][c] = o[c];
  }
  for (int c = 0; c < 4; c++) {  // map_columns: logg factors down each teff column
    bool pres[4];
    for (int r = 0; r < 4; r++) pres[r] = ok[r][c];
    double o[4];
    coeffs_from_neighbors(lg, pres, lv, o);
    for (int r = 0; r < 4; r++) fl[r][c] = o[r];
  }
  coeffs_from_neighbors(mm, mp, mv, fm);
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++)
      for (int k = 0; k < 4; k++) {
        int idx = (c * 4 + r) * 4 + k;
        double a = ft[r][c] * fl[r][c];
        w64[idx] = a * fm[k];
        cols[idx] = (ok[r][c] && mn[k] >= 0) ? g.column(tn[c], mn[k], ln[r]) : -1;
      }
}

// interpolate.rs:930-983
template <class T>
std::vector<T> interpolate(const OGrid &g, double t, double mm, double lg) {
  int64_t cols[64];
  double w64[64];
  local_grid(g, t, mm, lg, cols, w64);
  const int64_t n = g.npx;
  std::vector<T> out(n, T(0));
  T w[64], fac[64];
  const uint16_t *col[64];
  for (int j = 0; j < 64; j++) {
    if (std::is_same<T, float>::value) w[j] = (T)(float)w64[j];
    else w[j] = (T)w64[j];
    if (cols[j] >= 0) {
      col[j] = &g.spectra[(size_t)cols[j] * n];
      fac[j] = std::is_same<T, float>::value ? (T)g.factors[cols[j]] : (T)g.factors64[cols[j]];
    } else {
      col[j] = nullptr;
      fac[j] = std::is_same<T, float>::value ? (T)(1.0f / 65535.0f) : (T)(1.0 / 65535.0);
    }
  }
  const int64_t nb = n / 128 * 128;
  for (int64_t s = 0; s < nb; s += 128) {
    T acc[128];
    for (int i = 0; i < 128; i++) acc[i] = T(0);
    for (int j = 0; j < 64; j++) {
      const T wj = w[j], fj = fac[j];
      const uint16_t *cj = col[j];
      for (int i = 0; i < 128; i++) {
        T x = cj ? (T)cj[s + i] : T(0);
        T mval = x * fj;
        T prod = wj * mval;
        acc[i] = acc[i] + prod;
      }
    }
    for (int i = 0; i < 128; i++) out[s + i] = acc[i];
  }
  // tail: scaled by an extra 1/65535 (interpolate.rs:978)
  for (int64_t i = nb; i < n; i++) {
    T acc = T(0);
    for (int j = 0; j < 64; j++) {
      T x = col[j] ? (T)col[j][i] : T(0);
      T mval = x / T(65535.0) * fac[j];
      acc = acc + w[j] * mval;
    }
    out[i] = acc;
  }
  return out;
}

// Range::find_neighbors_linear (interpolate.rs:161-213): the two grid points
// around x.  A grid point at the right limit takes its left partner; a right
// limit at index 0 has none (the reference's usize subtraction panics).
void find_neighbors_linear(const Range &r, double x, int left, int right, int out[2]) {
  auto s = r.search(x);
  int i = s.second;
  if (s.first) {
    if (i < left) fail("Index %d out of left bound, x=%g", i, x);
    if (i > right) fail("Index %d out of right bound, x=%g", i, x);
    if (i == right) {
      if (i == 0) fail("no left neighbour for x=%g", x);
      out[0] = i - 1; out[1] = i;
    } else {
      out[0] = i; out[1] = i + 1;
    }
  } else {
    if (i <= left) fail("Index %d out of left bound, x=%g", i, x);
    if (i > right) fail("Index %d out of right bound, x=%g", i, x);
    out[0] = i - 1; out[1] = i;
  }
}

// Grid::get_local_grid_linear (interpolate.rs:536-600) and
// calculate_interpolation_coefficients_linear (cubic.rs:6-10, 246-270):
// the 2 x 2 x 2 cube around the label, teff outer, logg middle, [M/H] inner,
// weights (a * b * c) in f64 before the f32 cast.  A (teff, logg) corner
// outside that teff's logg limits has no model; the reference would read a
// neighbouring column there, the oracle stops.
void local_grid_linear(const OGrid &g, double t, double mm, double lg, int64_t cols[8], double w64[8]) {
  if (t != t || mm != mm || lg != lg) fail("NaN label");
  if (!g.teff_logg_ok(t, lg)) fail("Teff, logg out of bounds (%g, %g)", t, lg);
  if (!g.m_ok(mm)) fail("M out of bounds (%g)", mm);
  auto tl = g.teff_index_limits_at(lg);
  auto ll = g.logg_index_limits_at(t);
  int tn[2], mn[2], ln[2];
  find_neighbors_linear(g.teff, t, tl.first, tl.second, tn);
  find_neighbors_linear(g.m, mm, 0, g.m.n() - 1, mn);
  find_neighbors_linear(g.logg, lg, ll.first, ll.second, ln);
  auto lin = [](double x, double x0, double x1, double f[2]) {  // cubic.rs:6-10
    f[0] = (x - x1) / (x0 - x1);
    f[1] = (x - x0) / (x1 - x0);
  };
  double ft[2], fl[2], fm[2];
  lin(t, g.teff.v[tn[0]], g.teff.v[tn[1]], ft);
  lin(lg, g.logg.v[ln[0]], g.logg.v[ln[1]], fl);
  lin(mm, g.m.v[mn[0]], g.m.v[mn[1]], fm);
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++) {
      auto lim = g.logg_limits[tn[a]];
      if (ln[b] < lim.first || ln[b] > lim.second)
        fail("no model at teff index %d, logg index %d", tn[a], ln[b]);
      for (int c = 0; c < 2; c++) {
        const int idx = (a * 2 + b) * 2 + c;
        w64[idx] = ft[a] * fl[b] * fm[c];
        cols[idx] = g.column(tn[a], mn[c], ln[b]);
      }
    }
}

// GridInterpolator::interpolate_linear (interpolate.rs:985-1028): every
// pixel (the batched part and the tail alike) is u16 / 65535 * factor,
// summed over the 8 corners in order.
template <class T>
std::vector<T> interpolate_linear(const OGrid &g, double t, double mm, double lg) {
  int64_t cols[8];
  double w64[8];
  local_grid_linear(g, t, mm, lg, cols, w64);
  const int64_t n = g.npx;
  const bool f32 = std::is_same<T, float>::value;
  T w[8], fac[8];
  const uint16_t *col[8];
  for (int j = 0; j < 8; j++) {
    w[j] = f32 ? (T)(float)w64[j] : (T)w64[j];
    fac[j] = f32 ? (T)g.factors[cols[j]] : (T)g.factors64[cols[j]];
    col[j] = &g.spectra[(size_t)cols[j] * n];
  }
  std::vector<T> out(n);
  for (int64_t i = 0; i < n; i++) {
    T acc = T(0);
    for (int j = 0; j < 8; j++) {
      T mval = (T)col[j][i] / T(65535.0) * fac[j];
      acc = acc + mval * w[j];
    }
    out[i] = acc;
  }
  return out;
}

// ------------------------------------------------------------------ FFT
// Own radix-2 real FFT of 2048 (stand-in for realfft/rustfft).
struct Fft2048 {
  float wr[1024], wi[1024];  // W_2048^k, k < 1024
  int rev[1024];
  Fft2048() {
    for (int k = 0; k < 1024; k++) {
      double ang = -2.0 * M_PI * (double)k / 2048.0;
      wr[k] = (float)std::cos(ang);
      wi[k] = (float)std::sin(ang);
    }
    for (int i = 0; i < 1024; i++) {
      int r = 0;
      for (int b = 0; b < 10; b++) if (i & (1 << b)) r |= 1 << (9 - b);
      rev[i] = r;
    }
  }
  // complex 1024-point FFT in place; sign -1 forward, +1 inverse (unnormalised)
  void cfft(float *re, float *im, int sign) const {
    for (int i = 0; i < 1024; i++) {
      int j = rev[i];
      if (j > i) { std::swap(re[i], re[j]); std::swap(im[i], im[j]); }
    }
    for (int len = 2; len <= 1024; len <<= 1) {
      int half = len >> 1, stride = 2048 / len;
      for (int i = 0; i < 1024; i += len)
        for (int j = 0; j < half; j++) {
          float cr = wr[j * stride], ci = sign < 0 ? wi[j * stride] : -wi[j * stride];
          float ar = re[i + j + half], ai = im[i + j + half];
          float vr = ar * cr - ai * ci, vi = ar * ci + ai * cr;
          float ur = re[i + j], ui = im[i + j];
          re[i + j] = ur + vr; im[i + j] = ui + vi;
          re[i + j + half] = ur - vr; im[i + j + half] = ui - vi;
        }
    }
  }
  // real x[2048] -> X[0..1024] (1025 bins)
  void rfft(const float *x, float *Xr, float *Xi) const {
    float zr[1024], zi[1024];
    for (int k = 0; k < 1024; k++) { zr[k] = x[2 * k]; zi[k] = x[2 * k + 1]; }
    cfft(zr, zi, -1);
    for (int k = 0; k <= 1024; k++) {
      int k1 = k & 1023, k2 = (1024 - k) & 1023;
      float ar = zr[k1], ai = zi[k1], br = zr[k2], bi = -zi[k2];  // conj(Z[N/2-k])
      float er = 0.5f * (ar + br), ei = 0.5f * (ai + bi);
      float dr = 0.5f * (ar - br), di = 0.5f * (ai - bi);
      float orr = di, oi = -dr;  // -i * d
      float cr = wr[k & 1023], ci = wi[k & 1023];
      if (k == 1024) { cr = -1.0f; ci = 0.0f; }
      Xr[k] = er + (orr * cr - oi * ci);
      Xi[k] = ei + (orr * ci + oi * cr);
    }
  }
  // X[0..1024] -> 2048 * x (unnormalised inverse, like realfft)
  void irfft(const float *Xr, const float *Xi, float *x) const {
    float zr[1024], zi[1024];
    for (int k = 0; k < 1024; k++) {
      // X[k + N/2] = conj(X[N/2 - k])
      float ar = Xr[k], ai = Xi[k], br = Xr[1024 - k], bi = -Xi[1024 - k];
      float er = ar + br, ei = ai + bi;
      float dr = ar - br, di = ai - bi;
      float cr = wr[k], ci = -wi[k];  // W^{-k}
      float orr = dr * cr - di * ci, oi = dr * ci + di * cr;
      zr[k] = er - oi; zi[k] = ei + orr;  // e + i*o
    }
    cfft(zr, zi, +1);
    for (int k = 0; k < 1024; k++) { x[2 * k] = zr[k]; x[2 * k + 1] = zi[k]; }
  }
};
const Fft2048 &fft() { static Fft2048 f; return f; }

// convolve_rv.rs:121-157 (f32, FFT overlap-add)
std::vector<float> oa_convolve(const std::vector<float> &in, const std::vector<float> &kernel) {
  const int n = FFTSIZE;
  const int64_t m = (int64_t)kernel.size();
  const int64_t step = n - (m - 1);
  const int64_t l = (int64_t)in.size();
  const int64_t nx = (l + step - 1) / step * step;
  float pad[2048], Hr[1025], Hi[1025], Xr[1025], Xi[1025], r[2048];
  std::memset(pad, 0, sizeof pad);
  for (int64_t i = 0; i < m; i++) pad[i] = kernel[i];
  fft().rfft(pad, Hr, Hi);
  std::vector<float> y(nx + m - 1, 0.0f);
  for (int64_t pos = 0; pos < nx; pos += step) {
    int64_t len = pos + step < l ? step : l - pos;
    std::memset(pad, 0, sizeof pad);
    for (int64_t i = 0; i < len; i++) pad[i] = in[pos + i];
    fft().rfft(pad, Xr, Xi);
    for (int k = 0; k <= 1024; k++) {
      float ar = Xr[k], ai = Xi[k];
      Xr[k] = ar * Hr[k] - ai * Hi[k];
      Xi[k] = ar * Hi[k] + ai * Hr[k];
    }
    fft().irfft(Xr, Xi, r);
    for (int i = 0; i < n; i++) y[pos + i] = y[pos + i] + r[i] / (float)n;
  }
  return y;
}

// Iterative radix-2 complex FFT in double (unnormalised; sign -1 forward,
// +1 inverse) of size n = 2^k, twiddles from std::cos / std::sin per size.
struct FftD {
  int n = 0;
  std::vector<double> wr, wi;
  std::vector<int> rev;
  explicit FftD(int n_) : n(n_), wr(n_ / 2), wi(n_ / 2), rev(n_) {
    int bits = 0;
    while ((1 << bits) < n) bits++;
    for (int k = 0; k < n / 2; k++) {
      const double ang = -2.0 * M_PI * (double)k / (double)n;
      wr[k] = std::cos(ang);
      wi[k] = std::sin(ang);
    }
    for (int i = 0; i < n; i++) {
      int r = 0;
      for (int b = 0; b < bits; b++)
        if (i & (1 << b)) r |= 1 << (bits - 1 - b);
      rev[i] = r;
    }
  }
  void run(double *re, double *im, int sign) const {
    for (int i = 0; i < n; i++) {
      const int j = rev[i];
      if (j > i) {
        std::swap(re[i], re[j]);
        std::swap(im[i], im[j]);
      }
    }
    for (int len = 2; len <= n; len <<= 1) {
      const int half = len >> 1, stride = n / len;
      for (int i = 0; i < n; i += len)
        for (int j = 0; j < half; j++) {
          const double cr = wr[j * stride], ci = sign < 0 ? wi[j * stride] : -wi[j * stride];
          const double ar = re[i + j + half], ai = im[i + j + half];
          const double vr = ar * cr - ai * ci, vi = ar * ci + ai * cr;
          const double ur = re[i + j], ui = im[i + j];
          re[i + j] = ur + vr;
          im[i + j] = ui + vi;
          re[i + j + half] = ur - vr;
          im[i + j + half] = ui - vi;
        }
    }
  }
};

// Linear convolution in double by overlap-save FFT blocks (two real blocks
// per complex transform): full-convolution entries [off, off + cnt).  The
// FP64 mode uses it for wide kernels, where it agrees with the direct sum to
// ~1e-15 relative and is much faster; it is the same linear convolution.
std::vector<double> fft_convolve64(const std::vector<double> &in, const std::vector<double> &h, int64_t off,
                                   int64_t cnt) {
  const int64_t l = (int64_t)in.size(), m = (int64_t)h.size();
  int n = 1024;
  while (n < 4 * m) n <<= 1;
  const FftD F(n);
  const int64_t V = n - (m - 1);
  std::vector<double> hr(n, 0.0), hi(n, 0.0), xr(n), xi(n);
  for (int64_t k = 0; k < m; k++) hr[k] = h[k];
  F.run(hr.data(), hi.data(), -1);
  std::vector<double> y(cnt, 0.0);
  for (int64_t j0 = off; j0 < off + cnt; j0 += 2 * V) {
    const int64_t j1 = j0 + V;
    for (int t = 0; t < n; t++) {
      const int64_t a = j0 - (m - 1) + t, b = j1 - (m - 1) + t;
      xr[t] = (a >= 0 && a < l) ? in[a] : 0.0;
      xi[t] = (b >= 0 && b < l) ? in[b] : 0.0;
    }
    F.run(xr.data(), xi.data(), -1);
    for (int k = 0; k < n; k++) {
      const double ar = xr[k], ai = xi[k];
      xr[k] = ar * hr[k] - ai * hi[k];
      xi[k] = ar * hi[k] + ai * hr[k];
    }
    F.run(xr.data(), xi.data(), +1);
    for (int64_t t = m - 1; t < n; t++) {
      const int64_t u0 = j0 + t - (m - 1) - off, u1 = j1 + t - (m - 1) - off;
      if (u0 >= 0 && u0 < cnt && j0 + t - (m - 1) < j1) y[u0] = xr[t] / n;
      if (u1 >= 0 && u1 < cnt) y[u1] = xi[t] / n;
    }
  }
  return y;
}

// linear convolution in double: full-convolution entries [off, off+cnt)
// (direct sums for narrow kernels, FFT blocks in double for wide ones)
std::vector<double> direct_convolve(const std::vector<double> &in, const std::vector<double> &h,
                                    int64_t off, int64_t cnt) {
  const int64_t l = (int64_t)in.size(), m = (int64_t)h.size();
  if (m > 48 && cnt > 4096) return fft_convolve64(in, h, off, cnt);
  std::vector<double> y(cnt, 0.0);
  for (int64_t t = 0; t < cnt; t++) {
    int64_t j = off + t;
    double acc = 0.0;
    int64_t k0 = std::max<int64_t>(0, j - (l - 1)), k1 = std::min<int64_t>(m - 1, j);
    for (int64_t k = k0; k <= k1; k++) acc += h[k] * in[j - k];
    y[t] = acc;
  }
  return y;
}

// convolve_rv.rs:438-475; returns f64 values and the f32 kernel normalised in f32
void rotation_kernel(double vsini, double dvelo, std::vector<float> &k32, std::vector<double> &k64) {
  const double epsilon = 0.6;
  const double vrot = vsini / C_KMS;
  double q = 4.0 * (epsilon - 1.0) / (M_PI * epsilon);
  double wdt = 2.0 * vrot / dvelo * std::sqrt(1.0 + std::pow(q, 2.0));
  double cw = std::ceil(wdt);
  size_t nme = (cw > 0 ? (size_t)cw : 0) + 2;
  if (nme < 1) nme = 1;
  if (!(wdt < 1e9)) fail("rotation kernel too wide");
  size_t n = nme + 1 - nme % 2;
  std::vector<double> velo(n);
  for (size_t i = 0; i < n; i++) velo[i] = (double)i * dvelo;
  double mid = velo[n - 1] / 2.0;
  for (auto &v : velo) v -= mid;
  k32.assign(n, 0.0f);
  k64.assign(n, 0.0);
  for (size_t i = 0; i < n; i++) {
    double r = velo[i] / vrot;
    double y = 1.0 - r * r;
    if (y > 0.0) {
      double val = (2.0 * (1.0 - epsilon) * std::sqrt(y) + M_PI * epsilon / 2.0 * y) /
                   (M_PI * vrot * (1.0 - epsilon / 3.0));
      k32[i] = (float)val;
      k64[i] = val;
    }
  }
  float s32 = 0.0f;
  for (float v : k32) s32 = s32 + v;
  for (auto &v : k32) v = v / s32;
  double s64 = 0.0;
  for (double v : k64) s64 += v;
  for (auto &v : k64) v /= s64;
}

double grid_dvelo(const WlGrid &wl) {  // convolve_rv.rs:499-507
  if (wl.kind == OWL_LINSPACE) {
    double avg = (wl.a + wl.a + wl.b * (double)wl.n) / 2.0;
    return wl.b / avg;
  }
  if (wl.kind == OWL_LOGSPACE) return M_LN10 * wl.b;
  fail("Non-equidistant wavelength grid not supported");
}

// convolve_rv.rs:484-529
template <class T>
std::vector<T> convolve_rotation(const OGrid &g, const std::vector<T> &in, double vsini) {
  if (vsini < 0.0) fail("vsini must be positive");
  if ((int64_t)in.size() != g.wl.n) fail("Length of model and wavelength grid don't match");
  double dvelo = grid_dvelo(g.wl);
  std::vector<float> k32;
  std::vector<double> k64;
  rotation_kernel(vsini, dvelo, k32, k64);
  if (vsini == 0.0 || k32.size() <= 2) return in;
  if (k32.size() > (size_t)FFTSIZE) fail("Kernel size is larger than FFTSIZE. Kernel size: %zu, vsini: %g", k32.size(), vsini);
  const int64_t start = (int64_t)k32.size() / 2, N = (int64_t)in.size();
  std::vector<T> out(N);
  if (std::is_same<T, float>::value) {
    std::vector<float> inf(in.begin(), in.end());
    auto y = oa_convolve(inf, k32);
    for (int64_t i = 0; i < N; i++) out[i] = (T)y[start + i];
  } else {
    std::vector<double> ind(in.begin(), in.end());
    auto y = direct_convolve(ind, k64, start, N);
    for (int64_t i = 0; i < N; i++) out[i] = (T)y[i];
  }
  return out;
}

// convolve_rv.rs:107-118
void make_gaussian32(float *arr, int n, float sigma) {
  int mid = (n - 1) / 2;
  for (int i = 0; i < n; i++) {
    float x = ((float)i - (float)mid) / sigma;
    arr[i] = std::exp(-0.5f * x * x);
  }
  float s = 0.0f;
  for (int i = 0; i < n; i++) s = s + arr[i];
  for (int i = 0; i < n; i++) arr[i] = arr[i] / s;
}
void make_gaussian64(double *arr, int n, double sigma) {
  int mid = (n - 1) / 2;
  for (int i = 0; i < n; i++) {
    double x = ((double)i - (double)mid) / sigma;
    arr[i] = std::exp(-0.5 * x * x);
  }
  double s = 0.0;
  for (int i = 0; i < n; i++) s += arr[i];
  for (int i = 0; i < n; i++) arr[i] /= s;
}

int odd_width(double six_sigma) {  // ceil as usize, made odd
  double c = std::ceil(six_sigma);
  size_t nme = c > 0 ? (size_t)c : 0;
  return (int)(nme + 1 - nme % 2);
}

}  // namespace

struct ODisp {
  int kind = ODISP_NONE;
  std::vector<double> wl;     // observed wavelengths
  std::vector<double> fidx;   // float_indices_in_synth_grid
  // fixed-resolution log grid: one kernel
  std::vector<float> gk32;
  std::vector<double> gk64;
  int half = 0;               // (kernel width - 1) / 2
  // per-pixel kernels (variable / fixed non-log): width x nsynth, column-major
  std::vector<float> pk32;
  std::vector<double> pk64;
  int width = 0;
  bool per_pixel = false;
  const OGrid *g = nullptr;
};

namespace {

// convolve_rv.rs:303-331
std::vector<float> resample_observed_to_synth(const std::vector<double> &wl_obs, const WlGrid &wl, const float *y) {
  std::vector<float> out(wl.n);
  size_t j = 0;
  const size_t L = wl_obs.size();
  for (int64_t i = 0; i < wl.n; i++) {
    double x = wl.at(i);
    while (j < L - 1 && wl_obs[j + 1] < x) j++;
    if (j == L - 1) out[i] = y[j];
    else {
      float w = (float)((x - wl_obs[j]) / (wl_obs[j + 1] - wl_obs[j]));
      out[i] = (1.0f - w) * y[j] + w * y[j + 1];
    }
  }
  return out;
}

void build_per_pixel(ODisp &d, const std::vector<float> &sig32, const std::vector<double> &sig64) {
  float largest = sig32[0];
  for (float s : sig32) if (s > largest || std::isnan(largest)) largest = s;
  int w = odd_width((double)(largest * 6.0f));
  d.width = w;
  d.half = (w - 1) / 2;
  d.per_pixel = true;
  const int64_t N = (int64_t)sig32.size();
  d.pk32.assign((size_t)w * N, 0.0f);
  d.pk64.assign((size_t)w * N, 0.0);
  for (int64_t i = 0; i < N; i++) {
    make_gaussian32(&d.pk32[(size_t)i * w], w, sig32[i]);
    make_gaussian64(&d.pk64[(size_t)i * w], w, sig64[i]);
  }
}

// convolve_rv.rs:213-233 / 414-430
template <class T>
std::vector<T> convolve_per_pixel(const ODisp &d, const std::vector<T> &in) {
  const int64_t N = (int64_t)in.size();
  if (N != d.g->wl.n) fail("flux_arr and wavelength grid don't match");
  const int n = d.half, w = d.width;
  std::vector<T> out(N);
  for (int64_t i = 0; i < N; i++) {
    if (i < n || i >= N - n) { out[i] = in[i]; continue; }
    T acc = T(0);
    for (int t = 0; t < w; t++) {
      T kv = std::is_same<T, float>::value ? (T)d.pk32[(size_t)i * w + t] : (T)d.pk64[(size_t)i * w + t];
      acc = acc + kv * in[i - n + t];
    }
    out[i] = acc;
  }
  return out;
}

template <class T>
std::vector<T> disp_convolve(const ODisp &d, const std::vector<T> &in) {
  if (d.kind == ODISP_NONE) return in;
  if (d.per_pixel) return convolve_per_pixel(d, in);
  const int64_t N = (int64_t)in.size();
  std::vector<T> out(N);
  if (std::is_same<T, float>::value) {  // convolve_rv.rs:207-210
    std::vector<float> inf(in.begin(), in.end());
    auto y = oa_convolve(inf, d.gk32);
    for (int64_t i = 0; i < N; i++) out[i] = (T)y[d.half + i];
  } else {
    std::vector<double> ind(in.begin(), in.end());
    auto y = direct_convolve(ind, d.gk64, d.half, N);
    for (int64_t i = 0; i < N; i++) out[i] = (T)y[i];
  }
  return out;
}

// convolve_rv.rs:532-604
template <class T>
std::vector<T> shift_and_resample(const OGrid &g, const std::vector<T> &in, const ODisp &d, double rv) {
  const int64_t N = g.wl.n;
  if ((int64_t)in.size() != N) fail("Length of input_array and wavelength grid don't match");
  const double shift = 1.0 - rv / C_KMS;
  auto fl = g.wl.first_last();
  const double first_src = d.wl[0] * shift;
  if (first_src < fl.first) fail("Observed wavelength is smaller than synthetic wavelength (RV=%g, %.1f < %.1f)", rv, first_src, fl.first);
  const double last_src = d.wl[d.wl.size() - 1] * shift;
  if (last_src > fl.second) fail("Observed wavelength is larger than synthetic wavelength (RV=%g, %.1f > %.1f)", rv, last_src, fl.second);
  const int64_t L = (int64_t)d.wl.size();
  std::vector<T> out(L);
  auto resample = [&](double index) -> T {
    double fl_ = std::floor(index);
    int64_t j = fl_ > 0 ? (int64_t)fl_ : 0;  // `as usize` saturates at 0
    if (j + 1 >= N) fail("resampling index %lld out of range (%lld)", (long long)(j + 1), (long long)N);
    T w = (T)(float)index - (T)(float)j;
    return (T(1) - w) * in[j] + w * in[j + 1];
  };
  if (g.wl.kind == OWL_LINSPACE) {
    double offset = (g.wl.a / g.wl.b) * (shift - 1.0);
    for (int64_t i = 0; i < L; i++) out[i] = resample(shift * d.fidx[i] + offset);
  } else if (g.wl.kind == OWL_LOGSPACE) {
    double shift_log = std::log10(shift) / g.wl.b;
    for (int64_t i = 0; i < L; i++) out[i] = resample(d.fidx[i] + shift_log);
  } else {
    for (int64_t i = 0; i < L; i++) out[i] = resample(g.wl.float_index(d.wl[i] * shift));
  }
  return out;
}

template <class T>
std::vector<T> produce_model(const OGrid &g, const ODisp &d, const double *lab) {
  auto interp = interpolate<T>(g, lab[0], lab[1], lab[2]);
  auto rot = convolve_rotation<T>(g, interp, lab[3]);
  auto conv = disp_convolve<T>(d, rot);
  return shift_and_resample<T>(g, conv, d, lab[4]);
}

// ---------------------------------------------------------------- binary
// DVector::mean: sum in order, times 1 / n
template <class T>
T row_mean(const std::vector<T> &v) {
  T s = T(0);
  for (T x : v) s = s + x;
  return s * (T(1) / (T)v.size());
}

// Interpolator::produce_binary_model_norm (interpolate.rs:868-893):
// produce_binary_components (822-866) -- each star's normalised model
// broadened on the synthetic grid, its continuum linearly interpolated in
// the continuum grid, lr = light_ratio * mean(c1) / mean(c2) -- then
// shift_resample_and_add_binary_components (convolve_rv.rs:606-700):
// per observed pixel (n1 c1 + lr n2 c2) / (c1 + lr c2), each factor
// resampled at its star's RV.  lab = (star 1 [5], star 2 [5], light ratio).
// The FP32 mirror casts the light ratio to f32 as the reference does
// (fitting.rs:596); the FP64 mode keeps it in double.
template <class T>
std::vector<T> binary_model(const OGrid &g, const OGrid &gc, const ODisp &d, const double *lab) {
  const bool f32 = std::is_same<T, float>::value;
  auto norm = [&](const double *p) {
    auto interp = interpolate<T>(g, p[0], p[1], p[2]);
    auto rot = convolve_rotation<T>(g, interp, p[3]);
    return disp_convolve<T>(d, rot);
  };
  auto n1 = norm(lab);
  auto c1 = interpolate_linear<T>(gc, lab[0], lab[1], lab[2]);
  auto n2 = norm(lab + 5);
  auto c2 = interpolate_linear<T>(gc, lab[5], lab[6], lab[7]);
  const T lr0 = f32 ? (T)(float)lab[10] : (T)lab[10];
  const T lr = lr0 * row_mean(c1) / row_mean(c2);

  const int64_t N = g.wl.n;
  if ((int64_t)n1.size() != N) fail("Length of input_array and wavelength grid don't match");
  const double rv1 = lab[4], rv2 = lab[9];
  if (rv1 != rv1 || rv2 != rv2) fail("NaN RV");
  const double sf1 = 1.0 - rv1 / C_KMS, sf2 = 1.0 - rv2 / C_KMS;
  auto fl = g.wl.first_last();
  const double first_src = d.wl[0] * std::min(sf1, sf2);
  if (first_src < fl.first) fail("Observed wavelength is smaller than synthetic wavelength (%.1f < %.1f)", first_src, fl.first);
  const double last_src = d.wl[d.wl.size() - 1] * std::max(sf1, sf2);
  if (last_src > fl.second) fail("Observed wavelength is larger than synthetic wavelength (%.1f > %.1f)", last_src, fl.second);
  const int64_t NC = (int64_t)c1.size();
  auto at = [&](double index, const std::vector<T> &a, const std::vector<T> &c, T &av, T &cv) {
    const double f = std::floor(index);
    const int64_t j = f > 0 ? (int64_t)f : 0;  // `as usize` saturates at 0
    if (j + 1 >= N || j + 1 >= NC) fail("resampling index %lld out of range (%lld)", (long long)(j + 1), (long long)N);
    const T w = (T)(float)index - (T)(float)j;
    av = (T(1) - w) * a[j] + w * a[j + 1];
    cv = (T(1) - w) * c[j] + w * c[j + 1];
  };
  const int64_t L = (int64_t)d.wl.size();
  std::vector<T> out(L);
  for (int64_t i = 0; i < L; i++) {
    double i1, i2;
    if (g.wl.kind == OWL_LINSPACE) {
      i1 = sf1 * d.fidx[i] + (g.wl.a / g.wl.b) * (sf1 - 1.0);
      i2 = sf2 * d.fidx[i] + (g.wl.a / g.wl.b) * (sf2 - 1.0);
    } else if (g.wl.kind == OWL_LOGSPACE) {
      i1 = d.fidx[i] + std::log10(sf1) / g.wl.b;
      i2 = d.fidx[i] + std::log10(sf2) / g.wl.b;
    } else {
      i1 = g.wl.float_index(d.wl[i] * sf1);
      i2 = g.wl.float_index(d.wl[i] * sf2);
    }
    T a1, k1, a2, k2;
    at(i1, n1, c1, a1, k1);
    at(i2, n2, c2, a2, k2);
    out[i] = (a1 * k1 + lr * a2 * k2) / (k1 + lr * k2);
  }
  return out;
}

// ------------------------------------------------------- least squares
// Householder QR of an m x n column-major matrix, precomputed once per
// design (stand-in for nalgebra's SVD::new); solve() applies Q^T and
// back-substitutes (stand-in for SVD::solve).
template <class T>
struct QR {
  int64_t m = 0;
  int n = 0;
  std::vector<T> a;     // column-major, Householder vectors below diag
  std::vector<T> beta;  // 2 / (v^T v)
  std::vector<T> rdiag;
  void factor(const std::vector<T> &A, int64_t rows, int cols) {
    m = rows; n = cols; a = A; beta.assign(n, T(0)); rdiag.assign(n, T(0));
    for (int k = 0; k < n; k++) {
      T *ck = &a[(size_t)k * m];
      T nrm = T(0);
      for (int64_t i = k; i < m; i++) nrm = nrm + ck[i] * ck[i];
      nrm = std::sqrt(nrm);
      if (nrm == T(0)) { rdiag[k] = T(0); beta[k] = T(0); continue; }
      T alpha = ck[k] > T(0) ? -nrm : nrm;
      ck[k] = ck[k] - alpha;
      T vv = T(0);
      for (int64_t i = k; i < m; i++) vv = vv + ck[i] * ck[i];
      beta[k] = vv > T(0) ? T(2) / vv : T(0);
      for (int j = k + 1; j < n; j++) {
        T *cj = &a[(size_t)j * m];
        T s = T(0);
        for (int64_t i = k; i < m; i++) s = s + ck[i] * cj[i];
        s = s * beta[k];
        for (int64_t i = k; i < m; i++) cj[i] = cj[i] - s * ck[i];
      }
      rdiag[k] = alpha;
    }
  }
  std::vector<T> solve(const T *b) const {
    std::vector<T> y(b, b + m);
    for (int k = 0; k < n; k++) {
      const T *ck = &a[(size_t)k * m];
      T s = T(0);
      for (int64_t i = k; i < m; i++) s = s + ck[i] * y[i];
      s = s * beta[k];
      for (int64_t i = k; i < m; i++) y[i] = y[i] - s * ck[i];
    }
    std::vector<T> x(n, T(0));
    for (int k = n - 1; k >= 0; k--) {
      if (rdiag[k] == T(0)) { x[k] = T(0); continue; }
      T s = y[k];
      for (int j = k + 1; j < n; j++) s = s - a[(size_t)j * m + k] * x[j];
      x[k] = s / rdiag[k];
    }
    return x;
  }
};

template <class F>
F map_range(F x, F fl, F fh, F tl, F th, bool clamp) {  // continuum_fitting.rs:109-116
  F v = (x - fl) / (fh - fl) * (th - tl) + tl;
  if (clamp) v = std::min(std::max(v, tl), th);
  return v;
}
float poly_blend32(float x) {  // continuum_fitting.rs:119-123
  float xc = std::min(std::max(x, 0.0f), 1.0f);
  float s = std::sin(xc * (float)M_PI / 2.0f);
  return s * s;
}
double poly_blend64(double x) {
  double xc = std::min(std::max(x, 0.0), 1.0);
  double s = std::sin(xc * M_PI / 2.0);
  return s * s;
}
double powi(double x, int e) {  // binary exponentiation, as f64::powi lowers to
  double r = 1.0;
  while (true) {
    if (e & 1) r *= x;
    e >>= 1;
    if (e == 0) break;
    x *= x;
  }
  return r;
}

}  // namespace

struct OCont {
  int kind = OCONT_CHUNK;
  int64_t n = 0;
  // chunk
  int n_chunks = 0, p = 0;
  std::vector<double> wl;
  std::vector<int64_t> start, stop;
  std::vector<std::vector<float>> dm32;   // per chunk, row-major len x (p+1)
  std::vector<std::vector<double>> dm64;
  std::vector<QR<float>> qr32;
  std::vector<QR<double>> qr64;
  std::vector<std::vector<float>> fac32;  // factor_arrays
  std::vector<std::vector<double>> fac64;
  // linear
  int k = 0;
  std::vector<float> d32;  // row-major n x k
  std::vector<double> d64;
  QR<float> lqr32;
  QR<double> lqr64;
  // fixed
  std::vector<float> cont;
  int ignore = 0;
};

namespace {

// continuum_fitting.rs:140-214
void chunk_setup(OCont &c) {
  const auto &wl = c.wl;
  const int nc = c.n_chunks, p = c.p;
  c.dm32.resize(nc); c.dm64.resize(nc); c.qr32.resize(nc); c.qr64.resize(nc);
  for (int ch = 0; ch < nc; ch++) {
    int64_t s = c.start[ch], e = c.stop[ch], len = e - s;
    if (len <= 0) fail("empty chunk %d", ch);
    std::vector<float> col32((size_t)len * (p + 1));
    std::vector<double> col64((size_t)len * (p + 1));
    c.dm32[ch].assign((size_t)len * (p + 1), 0.0f);
    c.dm64[ch].assign((size_t)len * (p + 1), 0.0);
    for (int64_t i = 0; i < len; i++) {
      double x = map_range(wl[s + i], wl[s], wl[e - 1], -1.0, 1.0, false);
      for (int k = 0; k <= p; k++) {
        double v = powi(x, k);
        c.dm32[ch][(size_t)i * (p + 1) + k] = (float)v;
        c.dm64[ch][(size_t)i * (p + 1) + k] = v;
        col32[(size_t)k * len + i] = (float)v;
        col64[(size_t)k * len + i] = v;
      }
    }
    c.qr32[ch].factor(col32, len, p + 1);
    c.qr64[ch].factor(col64, len, p + 1);
  }
  c.fac32.resize(nc > 0 ? nc - 1 : 0);
  c.fac64.resize(nc > 0 ? nc - 1 : 0);
  for (int ch = 0; ch + 1 < nc; ch++) {
    int64_t e = c.stop[ch], sn = c.start[ch + 1];
    if (e < sn) fail("chunks %d and %d do not overlap", ch, ch + 1);
    for (int64_t i = sn; i < e; i++) {
      float v32 = poly_blend32(map_range((float)wl[i], (float)wl[sn], (float)wl[e - 1], 1.0f, 0.0f, false));
      double v64 = poly_blend64(map_range(wl[i], wl[sn], wl[e - 1], 1.0, 0.0, false));
      c.fac32[ch].push_back(v32);
      c.fac64[ch].push_back(v64);
    }
  }
}

template <class T> const std::vector<T> &dmv(const OCont &c, int ch);
template <> const std::vector<float> &dmv<float>(const OCont &c, int ch) { return c.dm32[ch]; }
template <> const std::vector<double> &dmv<double>(const OCont &c, int ch) { return c.dm64[ch]; }
template <class T> const std::vector<T> &facv(const OCont &c, int ch);
template <> const std::vector<float> &facv<float>(const OCont &c, int ch) { return c.fac32[ch]; }
template <> const std::vector<double> &facv<double>(const OCont &c, int ch) { return c.fac64[ch]; }
template <class T> const QR<T> &qrv(const OCont &c, int ch);
template <> const QR<float> &qrv<float>(const OCont &c, int ch) { return c.qr32[ch]; }
template <> const QR<double> &qrv<double>(const OCont &c, int ch) { return c.qr64[ch]; }

template <class T>
T dot_row(const std::vector<T> &dm, int p1, int64_t row, const std::vector<T> &pc) {
  T acc = T(0);
  for (int k = 0; k < p1; k++) acc = acc + dm[(size_t)row * p1 + k] * pc[k];
  return acc;
}

// continuum_fitting.rs:382-396 (+ 216-226, 280-360)
template <class T>
void chunk_fit(const OCont &c, const float *flux, const float *var, const std::vector<T> &model,
               std::vector<double> &params, double &chi2) {
  const int64_t N = c.n;
  const int nc = c.n_chunks, p1 = c.p + 1;
  std::vector<T> y(N);
  for (int64_t i = 0; i < N; i++) y[i] = (T)flux[i] / model[i];
  std::vector<std::vector<T>> pf(nc);
  for (int ch = 0; ch < nc; ch++) pf[ch] = qrv<T>(c, ch).solve(&y[c.start[ch]]);
  params.clear();
  for (int ch = 0; ch < nc; ch++) for (int k = 0; k < p1; k++) params.push_back((double)pf[ch][k]);
  if (N < 100) fail("spectrum too short for chi2 (%lld)", (long long)N);
  if (nc < 2) fail("chunk fitter needs at least 2 chunks");
  T total = T(0);
  {
    int64_t sn = c.start[1];
    if (sn < 50) fail("second chunk starts before pixel 50");
    T s = T(0);
    for (int64_t i = 50; i < sn; i++) {
      T r = (T)flux[i] - dot_row(dmv<T>(c, 0), p1, i - c.start[0], pf[0]) * model[i];
      s = s + r * r / (T)var[i];
    }
    total = total + s;
  }
  for (int ch = 1; ch < nc; ch++) {
    int64_t st = c.start[ch], sp = c.stop[ch - 1], stp = c.start[ch - 1];
    int64_t sn = ch == nc - 1 ? N - 50 : c.start[ch + 1];
    const auto &fac = facv<T>(c, ch - 1);
    T s = T(0);
    for (int64_t i = st; i < sp; i++) {
      T prev = dot_row(dmv<T>(c, ch - 1), p1, i - stp, pf[ch - 1]);
      T cur = dot_row(dmv<T>(c, ch), p1, i - st, pf[ch]);
      T f = fac[i - st];
      T pp = prev * f + cur * (T(1) - f);
      T r = (T)flux[i] - pp * model[i];
      s = s + r * r / (T)var[i];
    }
    total = total + s;
    if (sn < sp) fail("chunk %d: next chunk starts inside the previous overlap", ch);
    s = T(0);
    for (int64_t i = sp; i < sn; i++) {
      T r = (T)flux[i] - dot_row(dmv<T>(c, ch), p1, i - st, pf[ch]) * model[i];
      s = s + r * r / (T)var[i];
    }
    total = total + s;
  }
  chi2 = (double)total / (double)(N - 100);
}

// continuum_fitting.rs:228-278 (params are monomial coefficients per chunk)
template <class T>
std::vector<T> chunk_build(const OCont &c, const double *params) {
  const int64_t N = c.n;
  const int nc = c.n_chunks, p1 = c.p + 1;
  std::vector<std::vector<T>> pf(nc, std::vector<T>(p1));
  for (int ch = 0; ch < nc; ch++) for (int k = 0; k < p1; k++) pf[ch][k] = (T)params[ch * p1 + k];
  std::vector<T> cont(N, T(0));
  for (int64_t i = c.start[0]; i < c.stop[0]; i++) cont[i] = dot_row(dmv<T>(c, 0), p1, i - c.start[0], pf[0]);
  for (int ch = 1; ch < nc; ch++) {
    int64_t st = c.start[ch], e = c.stop[ch], sp = c.stop[ch - 1];
    for (int64_t i = st; i < e; i++) {
      T f;
      if (std::is_same<T, float>::value)
        f = (T)poly_blend32(map_range((float)c.wl[i], (float)c.wl[sp - 1], (float)c.wl[st], 0.0f, 1.0f, false));
      else
        f = (T)poly_blend64(map_range(c.wl[i], c.wl[sp - 1], c.wl[st], 0.0, 1.0, false));
      T pv = dot_row(dmv<T>(c, ch), p1, i - st, pf[ch]);
      cont[i] = cont[i] * f + pv * (T(1) - f);
    }
  }
  return cont;
}

// continuum_fitting.rs:68-95
template <class T>
void linear_fit(const OCont &c, const float *flux, const float *var, const std::vector<T> &model,
                std::vector<double> &params, double &chi2) {
  const int64_t N = c.n;
  const int k = c.k;
  if ((int64_t)(c.d32.size() / (size_t)(k > 0 ? k : 1)) != N) fail("design matrix rows do not match the spectrum");
  std::vector<T> b(N);
  for (int64_t i = 0; i < N; i++) b[i] = (T)flux[i] / model[i];
  std::vector<T> sol;
  if (std::is_same<T, float>::value) { auto s = c.lqr32.solve((const float *)b.data()); sol.assign(s.begin(), s.end()); }
  else { auto s = c.lqr64.solve((const double *)b.data()); sol.assign(s.begin(), s.end()); }
  params.assign(sol.begin(), sol.end());
  if (N < 100) fail("spectrum too short for chi2");
  T s = T(0);
  for (int64_t i = 50; i < N - 50; i++) {
    T mdl = T(0);
    for (int j = 0; j < k; j++) {
      T dv = std::is_same<T, float>::value ? (T)c.d32[(size_t)i * k + j] : (T)c.d64[(size_t)i * k + j];
      mdl = mdl + dv * sol[j];
    }
    T r = mdl - b[i];
    s = s + r / (T)var[i] * r;
  }
  chi2 = (double)s / (double)N;
}

template <class T>
void fit_continuum(const OCont &c, const float *flux, const float *var, const std::vector<T> &model,
                   std::vector<double> &params, double &chi2) {
  const int64_t N = c.n;
  if ((int64_t)model.size() != N) fail("Length of observed and synthetic spectrum are different");
  if (c.kind == OCONT_CHUNK) return chunk_fit<T>(c, flux, var, model, params, chi2);
  if (c.kind == OCONT_LINEAR) return linear_fit<T>(c, flux, var, model, params, chi2);
  if (c.kind == OCONT_FIXED) {  // continuum_fitting.rs:441-474
    const int64_t ig = c.ignore;
    if (N - 2 * ig <= 0) fail("ignore_first_and_last too large");
    T s = T(0);
    for (int64_t i = ig; i < N - ig; i++) {
      T r = (T)flux[i] - model[i] * (T)c.cont[i];
      s = s + r / (T)var[i] * r;
    }
    params.assign(1, 0.0);
    chi2 = (double)s / (double)(N - 2 * ig);
    return;
  }
  // ConstantContinuum continuum_fitting.rs:484-500
  T sum = T(0);
  for (int64_t i = 0; i < N; i++) sum = sum + (T)flux[i] / model[i];
  T mean = sum / (T)N;
  T s = T(0);
  for (int64_t i = 0; i < N; i++) {
    T r = (T)flux[i] - model[i] * mean;
    s = s + r / (T)var[i] * r;
  }
  params.assign(1, (double)mean);
  chi2 = (double)s / (double)N;
}

template <class T>
double cost(const OGrid &g, const ODisp &d, const OCont &c, const float *flux, const float *var, const double *lab) {
  auto mdl = produce_model<T>(g, d, lab);
  std::vector<double> params;
  double chi2;
  fit_continuum<T>(c, flux, var, mdl, params, chi2);
  return chi2;
}

// ------------------------------------------------------------------ PSO
uint64_t mix64(uint64_t z) {  // SplitMix64 finaliser (Steele, Lea, Flood 2014)
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double draw_u01(uint64_t seed, uint64_t phase, uint64_t a, uint64_t b, uint64_t c) {
  uint64_t h = mix64(seed);
  h = mix64(h ^ ((phase << 56) | (a & 0x00FFFFFFFFFFFFFFull)));
  h = mix64(h ^ ((b << 32) | (c & 0xFFFFFFFFull)));
  return (double)(h >> 11) * 0x1.0p-53;
}
// particleswarm.rs:153-161 with gen_range(lo..hi) = u * (hi - lo) + lo
double uniform_between(double a, double b, double u) {
  if (a == b) return a;
  double lo = a < b ? a : b, hi = a < b ? b : a;
  return u * (hi - lo) + lo;
}

struct Bounds {  // bounds.rs:69-186 (SingleBounds wrapped in ConstrainedPSOBounds)
  const OGrid *g;
  const OPsoSettings *st;
  void outer(double mn[5], double mx[5]) const {
    mn[0] = g->teff.v.front(); mx[0] = g->teff.v.back();
    mn[1] = g->m.v.front(); mx[1] = g->m.v.back();
    mn[2] = g->logg.v.front(); mx[2] = g->logg.v.back();
    mn[3] = st->vsini_lo; mx[3] = st->vsini_hi;
    mn[4] = st->rv_lo; mx[4] = st->rv_hi;
    for (int i = 0; i < 5; i++) {
      if (st->ckind[i] == 1) { mn[i] = st->ca[i]; mx[i] = st->ca[i]; }
      else if (st->ckind[i] == 2) { mn[i] = std::max(mn[i], st->ca[i]); mx[i] = std::min(mx[i], st->cb[i]); }
    }
  }
  std::pair<double, double> limits_at(const double *p, int i) const {
    std::pair<double, double> l;
    if (i == 3) l = {st->vsini_lo, st->vsini_hi};
    else if (i == 4) l = {st->rv_lo, st->rv_hi};
    else l = g->limits_at(p, i);
    if (st->ckind[i] == 1) return {st->ca[i], st->ca[i]};
    if (st->ckind[i] == 2) return {std::max(l.first, st->ca[i]), std::min(l.second, st->cb[i])};
    return l;
  }
  double clamp_1d(const double *p, int i) const {
    auto l = limits_at(p, i);
    if (!(l.first <= l.second)) fail("clamp limits invalid (%g > %g) in dim %d", l.first, l.second, i);
    return std::min(std::max(p[i], l.first), l.second);
  }
  bool within(const double *p) const {
    if (!g->within(p)) return false;
    if (!(p[3] >= st->vsini_lo && p[3] <= st->vsini_hi && p[4] >= st->rv_lo && p[4] <= st->rv_hi)) return false;
    for (int i = 0; i < 5; i++) {
      if (st->ckind[i] == 1 && !(std::fabs(p[i] - st->ca[i]) <= 2.220446049250313e-16)) return false;
      if (st->ckind[i] == 2 && !(p[i] >= st->ca[i] && p[i] <= st->cb[i])) return false;
    }
    return true;
  }
};

struct Particle {
  double x[5], v[5], bx[5];
  double cost, bcost;
};

template <class T>
void bulk_cost(const OGrid &g, const ODisp &d, const OCont &c, const float *flux, const float *var,
               std::vector<Particle> &ps, int nthreads, bool parallel) {
  const int P = (int)ps.size();
  std::vector<std::string> errs(P);
  std::vector<int> bad(P, 0);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1) if (parallel)
  for (int i = 0; i < P; i++) {
    try {
      ps[i].cost = cost<T>(g, d, c, flux, var, ps[i].x);
    } catch (const std::exception &e) {
      bad[i] = 1;
      errs[i] = e.what();
    }
  }
  for (int i = 0; i < P; i++) if (bad[i]) fail("particle %d: %s", i, errs[i].c_str());
}

// fitting.rs:399-458 + particleswarm.rs:111-307
template <class T>
void fit_one(const OGrid &g, const ODisp &d, const OCont &c, const OPsoSettings &st, const float *flux,
             const float *var, uint64_t seed, int nthreads, bool parallel, OFitResult &res, double *trace) {
  Bounds B{&g, &st};
  const int P = st.num_particles;
  if (P <= 0) fail("num_particles must be positive");
  double mn[5], mx[5];
  B.outer(mn, mx);
  std::vector<Particle> ps(P);
  // bounds.rs:21-35: rejection sampling
  uint64_t cand = 0;
  for (int p = 0; p < P;) {
    if (cand > 10000000ull) fail("could not place particles within bounds");
    double x[5];
    for (int dd = 0; dd < 5; dd++) {
      x[dd] = mn[dd] == mx[dd] ? mn[dd] : uniform_between(mn[dd], mx[dd], draw_u01(seed, 1, cand, 0, dd));
    }
    cand++;
    if (B.within(x)) { std::memcpy(ps[p].x, x, sizeof x); p++; }
  }
  // particleswarm.rs:137-150: velocities in (-width, width)
  for (int p = 0; p < P; p++)
    for (int dd = 0; dd < 5; dd++) {
      double w = mx[dd] - mn[dd];
      ps[p].v[dd] = (-w == w) ? -w : uniform_between(-w, w, draw_u01(seed, 2, p, 0, dd));
    }
  bulk_cost<T>(g, d, c, flux, var, ps, nthreads, parallel);
  for (auto &q : ps) { std::memcpy(q.bx, q.x, sizeof q.x); q.bcost = q.cost; }
  std::stable_sort(ps.begin(), ps.end(), [](const Particle &a, const Particle &b) {
    return a.cost < b.cost;  // NaN compares false both ways = Equal
  });
  double gx[5];
  std::memcpy(gx, ps[0].x, sizeof gx);
  double gcost = ps[0].cost;
  auto dump = [&](int it) {
    if (!trace) return;
    double *t = trace + (size_t)it * P * 6;
    for (int p = 0; p < P; p++) { for (int dd = 0; dd < 5; dd++) t[p * 6 + dd] = ps[p].x[dd]; t[p * 6 + 5] = ps[p].cost; }
  };
  dump(0);
  for (int it = 0; it < st.max_iters; it++) {
    for (int p = 0; p < P; p++) {
      Particle &q = ps[p];
      for (int dd = 0; dd < 5; dd++) {
        double momentum = q.v[dd] * st.inertia;
        double to_opt = q.bx[dd] - q.x[dd];
        double pull = (to_opt == 0.0 ? 0.0 : uniform_between(0.0, to_opt, draw_u01(seed, 3, it, p, 2 * dd))) * st.cognitive;
        double to_g = gx[dd] - q.x[dd];
        double pullg = (to_g == 0.0 ? 0.0 : uniform_between(0.0, to_g, draw_u01(seed, 3, it, p, 2 * dd + 1))) * st.social;
        q.v[dd] = momentum + pull + pullg;
        double nx[5];
        std::memcpy(nx, q.x, sizeof nx);
        nx[dd] += q.v[dd];
        q.x[dd] = B.clamp_1d(nx, dd);
        if (!B.within(q.x)) fail("Particle %d is not within bounds", p);
      }
    }
    bulk_cost<T>(g, d, c, flux, var, ps, nthreads, parallel);
    for (auto &q : ps) {
      if (q.cost < q.bcost) {
        std::memcpy(q.bx, q.x, sizeof q.x);
        q.bcost = q.cost;
        if (q.cost < gcost) { std::memcpy(gx, q.x, sizeof gx); gcost = q.cost; }
      }
    }
    dump(it + 1);
  }
  std::memcpy(res.label, gx, sizeof gx);
  res.chi2 = gcost;
  res.iterations = st.max_iters;
  auto mdl = produce_model<T>(g, d, gx);
  std::vector<double> params;
  double chi2;
  fit_continuum<T>(c, flux, var, mdl, params, chi2);
  res.n_params = (int)std::min<size_t>(params.size(), 512);
  for (int i = 0; i < res.n_params; i++) res.params[i] = params[i];
}

// BinaryCostFunction::cost (fitting.rs:584-600)
template <class T>
double binary_cost(const OGrid &g, const OGrid &gc, const ODisp &d, const OCont &c, const float *flux,
                   const float *var, const double *lab) {
  auto mdl = binary_model<T>(g, gc, d, lab);
  std::vector<double> params;
  double chi2;
  fit_continuum<T>(c, flux, var, mdl, params, chi2);
  return chi2;
}

// BinaryBounds (bounds.rs:188-275) wrapped in ConstrainedPSOBounds
// (bounds.rs:69-130): star 1 at 0..5, star 2 at 5..10, light ratio at 10
// with the range (0, 1) BinaryFitter::fit gives it (fitting.rs:649-655).
struct BinaryBoundsO {
  const OGrid *g;
  const OBinarySettings *st;
  static constexpr double lr_lo = 0.0, lr_hi = 1.0;
  std::pair<double, double> raw(const double *p, int i) const {
    if (i == 3 || i == 8) return {st->vsini_lo, st->vsini_hi};
    if (i == 4 || i == 9) return {st->rv_lo, st->rv_hi};
    if (i == 10) return {lr_lo, lr_hi};
    return i < 5 ? g->limits_at(p, i) : g->limits_at(p + 5, i - 5);
  }
  std::pair<double, double> constrain(int i, std::pair<double, double> l) const {
    if (st->ckind[i] == 1) return {st->ca[i], st->ca[i]};
    if (st->ckind[i] == 2) return {std::max(l.first, st->ca[i]), std::min(l.second, st->cb[i])};
    return l;
  }
  void outer(double mn[11], double mx[11]) const {
    for (int k = 0; k < 2; k++) {
      mn[5 * k + 0] = g->teff.v.front(); mx[5 * k + 0] = g->teff.v.back();
      mn[5 * k + 1] = g->m.v.front(); mx[5 * k + 1] = g->m.v.back();
      mn[5 * k + 2] = g->logg.v.front(); mx[5 * k + 2] = g->logg.v.back();
      mn[5 * k + 3] = st->vsini_lo; mx[5 * k + 3] = st->vsini_hi;
      mn[5 * k + 4] = st->rv_lo; mx[5 * k + 4] = st->rv_hi;
    }
    mn[10] = lr_lo; mx[10] = lr_hi;
    for (int i = 0; i < 11; i++) {
      auto l = constrain(i, {mn[i], mx[i]});
      mn[i] = l.first; mx[i] = l.second;
    }
  }
  double clamp_1d(const double *p, int i) const {
    auto l = constrain(i, raw(p, i));
    if (!(l.first <= l.second)) fail("clamp limits invalid (%g > %g) in dim %d", l.first, l.second, i);
    return std::min(std::max(p[i], l.first), l.second);
  }
  bool within(const double *p) const {
    if (!g->within(p) || !g->within(p + 5)) return false;
    for (int k = 0; k < 2; k++) {
      const double vs = p[5 * k + 3], rv = p[5 * k + 4];
      if (!(vs >= st->vsini_lo && vs <= st->vsini_hi && rv >= st->rv_lo && rv <= st->rv_hi)) return false;
    }
    if (!(p[10] >= lr_lo && p[10] <= lr_hi)) return false;
    for (int i = 0; i < 11; i++) {
      if (st->ckind[i] == 1 && !(std::fabs(p[i] - st->ca[i]) <= 2.220446049250313e-16)) return false;
      if (st->ckind[i] == 2 && !(p[i] >= st->ca[i] && p[i] <= st->cb[i])) return false;
    }
    return true;
  }
};

// BinaryFitter::fit (fitting.rs:633-697) with the particle swarm of
// particleswarm.rs:111-307 over 11 dimensions, on the shared draw stream
// (the same phases and counters as the single-star fit, dimension d < 11).
template <class T>
void fit_binary(const OGrid &g, const OGrid &gc, const ODisp &d, const OCont &c, const OBinarySettings &st,
                const float *flux, const float *var, uint64_t seed, int nthreads, OBinaryResult &res,
                double *trace) {
  constexpr int D = 11;
  BinaryBoundsO B{&g, &st};
  const int P = st.num_particles;
  if (P <= 0) fail("num_particles must be positive");
  double mn[D], mx[D];
  B.outer(mn, mx);
  struct Pt {
    double x[D], v[D], bx[D];
    double cost, bcost;
  };
  std::vector<Pt> ps(P);
  uint64_t cand = 0;
  for (int p = 0; p < P;) {  // bounds.rs:21-35
    if (cand > 10000000ull) fail("could not place particles within bounds");
    double x[D];
    for (int k = 0; k < D; k++)
      x[k] = mn[k] == mx[k] ? mn[k] : uniform_between(mn[k], mx[k], draw_u01(seed, 1, cand, 0, k));
    cand++;
    if (B.within(x)) { std::memcpy(ps[p].x, x, sizeof x); p++; }
  }
  for (int p = 0; p < P; p++)
    for (int k = 0; k < D; k++) {
      double w = mx[k] - mn[k];
      ps[p].v[k] = (-w == w) ? -w : uniform_between(-w, w, draw_u01(seed, 2, p, 0, k));
    }
  auto evaluate = [&]() {
    std::vector<std::string> errs(P);
    std::vector<int> bad(P, 0);
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
    for (int i = 0; i < P; i++) {
      try {
        ps[i].cost = binary_cost<T>(g, gc, d, c, flux, var, ps[i].x);
      } catch (const std::exception &e) {
        bad[i] = 1;
        errs[i] = e.what();
      }
    }
    for (int i = 0; i < P; i++) if (bad[i]) fail("particle %d: %s", i, errs[i].c_str());
  };
  evaluate();
  for (auto &q : ps) { std::memcpy(q.bx, q.x, sizeof q.x); q.bcost = q.cost; }
  std::stable_sort(ps.begin(), ps.end(), [](const Pt &a, const Pt &b) { return a.cost < b.cost; });
  double gx[D];
  std::memcpy(gx, ps[0].x, sizeof gx);
  double gcost = ps[0].cost;
  auto dump = [&](int it) {
    if (!trace) return;
    double *t = trace + (size_t)it * P * (D + 1);
    for (int p = 0; p < P; p++) {
      for (int k = 0; k < D; k++) t[p * (D + 1) + k] = ps[p].x[k];
      t[p * (D + 1) + D] = ps[p].cost;
    }
  };
  dump(0);
  for (int it = 0; it < st.max_iters; it++) {
    for (int p = 0; p < P; p++) {
      Pt &q = ps[p];
      for (int k = 0; k < D; k++) {
        double momentum = q.v[k] * st.inertia;
        double to_opt = q.bx[k] - q.x[k];
        double pull = (to_opt == 0.0 ? 0.0 : uniform_between(0.0, to_opt, draw_u01(seed, 3, it, p, 2 * k))) * st.cognitive;
        double to_g = gx[k] - q.x[k];
        double pullg = (to_g == 0.0 ? 0.0 : uniform_between(0.0, to_g, draw_u01(seed, 3, it, p, 2 * k + 1))) * st.social;
        q.v[k] = momentum + pull + pullg;
        double nx[D];
        std::memcpy(nx, q.x, sizeof nx);
        nx[k] += q.v[k];
        q.x[k] = B.clamp_1d(nx, k);
        if (!B.within(q.x)) fail("Particle %d is not within bounds", p);
      }
    }
    evaluate();
    for (auto &q : ps) {
      if (q.cost < q.bcost) {
        std::memcpy(q.bx, q.x, sizeof q.x);
        q.bcost = q.cost;
        if (q.cost < gcost) { std::memcpy(gx, q.x, sizeof gx); gcost = q.cost; }
      }
    }
    dump(it + 1);
  }
  std::memcpy(res.label1, gx, 5 * sizeof(double));
  std::memcpy(res.label2, gx + 5, 5 * sizeof(double));
  res.light_ratio = gx[10];
  res.chi2 = gcost;
  res.iterations = st.max_iters;
  auto mdl = binary_model<T>(g, gc, d, gx);
  std::vector<double> params;
  double chi2;
  fit_continuum<T>(c, flux, var, mdl, params, chi2);
  res.n_params = (int)std::min<size_t>(params.size(), 512);
  for (int i = 0; i < res.n_params; i++) res.params[i] = params[i];
}

template <class F>
int guard(F &&f) {
  try {
    f();
    return 0;
  } catch (const std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

}  // namespace

// ================================================================== C API
extern "C" {

const char *or_last_error(void) { return g_err.c_str(); }

double or_draw_u01(uint64_t seed, uint64_t phase, uint64_t a, uint64_t b, uint64_t c) {
  return draw_u01(seed, phase, a, b, c);
}

// interpolate.rs:267-331 (Grid::new) + model_fetchers.rs:136-166 (column order)
OGrid *or_grid_create(const double *labels, const uint16_t *spectra, const float *factors, int64_t n_models,
                      int64_t npx, int wl_kind, double wl_a, double wl_b, const double *wl_values) {
  OGrid *g = new OGrid();
  int rc = guard([&] {
    std::vector<double> t, m, l;
    auto ins = [](std::vector<double> &v, double x) {
      if (std::find(v.begin(), v.end(), x) == v.end()) v.insert(std::lower_bound(v.begin(), v.end(), x), x);
    };
    for (int64_t i = 0; i < n_models; i++) { ins(t, labels[3 * i]); ins(m, labels[3 * i + 1]); ins(l, labels[3 * i + 2]); }
    g->teff.v = t; g->m.v = m; g->logg.v = l;
    g->logg_limits.assign(t.size(), {(int)l.size() - 1, 0});
    for (int64_t i = 0; i < n_models; i++) {
      int ti = g->teff.search(labels[3 * i]).second, li = g->logg.search(labels[3 * i + 2]).second;
      auto &lim = g->logg_limits[ti];
      if (li < lim.first) lim.first = li;
      if (li > lim.second) lim.second = li;
    }
    for (auto &lim : g->logg_limits) if (lim.first > lim.second) fail("Invalid logg limits");
    g->cum.resize(t.size());
    int64_t acc = 0;
    for (size_t i = 0; i < t.size(); i++) { g->cum[i] = acc; acc += g->logg_limits[i].second - g->logg_limits[i].first + 1; }
    const int64_t ncols = acc * (int64_t)m.size();
    g->npx = npx;
    g->spectra.assign((size_t)ncols * npx, 0);
    g->factors.assign(ncols, 1.0f / 65535.0f);
    g->factors64.assign(ncols, 1.0 / 65535.0);
    std::vector<char> seen(ncols, 0);
    for (int64_t i = 0; i < n_models; i++) {
      int ti = g->teff.search(labels[3 * i]).second, mi = g->m.search(labels[3 * i + 1]).second,
          li = g->logg.search(labels[3 * i + 2]).second;
      int64_t col = g->column(ti, mi, li);
      seen[col] = 1;
      std::memcpy(&g->spectra[(size_t)col * npx], spectra + (size_t)i * npx, npx * sizeof(uint16_t));
      if (factors) {
        if (factors[i] < 0.0f) fail("Negative factor: %g", (double)factors[i]);
        g->factors[col] = factors[i] / 65535.0f;
        g->factors64[col] = (double)factors[i] / 65535.0;
      }
    }
    for (int64_t cidx = 0; cidx < ncols; cidx++) if (!seen[cidx]) fail("grid model missing at column %lld", (long long)cidx);
    g->wl.kind = wl_kind; g->wl.a = wl_a; g->wl.b = wl_b; g->wl.n = npx;
    if (wl_kind == OWL_NONUNIFORM) g->wl.vals.assign(wl_values, wl_values + npx);
  });
  if (rc) { delete g; return nullptr; }
  return g;
}
void or_grid_free(OGrid *g) { delete g; }
int or_grid_axes(const OGrid *g, int *nt, int *nm, int *nl) { *nt = g->teff.n(); *nm = g->m.n(); *nl = g->logg.n(); return 0; }
int or_grid_axis_values(const OGrid *g, int axis, double *out) {
  const auto &v = axis == 0 ? g->teff.v : axis == 1 ? g->m.v : g->logg.v;
  std::copy(v.begin(), v.end(), out);
  return 0;
}
int or_grid_logg_limits(const OGrid *g, int *lo, int *hi) {
  for (size_t i = 0; i < g->logg_limits.size(); i++) { lo[i] = g->logg_limits[i].first; hi[i] = g->logg_limits[i].second; }
  return 0;
}
int or_local_grid(const OGrid *g, double t, double m, double l, int64_t *cols, double *w) {
  return guard([&] { local_grid(*g, t, m, l, cols, w); });
}
int or_is_within_bounds(const OGrid *g, double t, double m, double l) {
  double p[3] = {t, m, l};
  return g->within(p) ? 1 : 0;
}
int or_limits_at(const OGrid *g, const double *tml, int index, double *lo, double *hi) {
  return guard([&] { auto r = g->limits_at(tml, index); *lo = r.first; *hi = r.second; });
}
int or_interpolate(const OGrid *g, int prec, double t, double m, double l, double *out) {
  return guard([&] {
    if (prec == OP_F32) { auto v = interpolate<float>(*g, t, m, l); std::copy(v.begin(), v.end(), out); }
    else { auto v = interpolate<double>(*g, t, m, l); std::copy(v.begin(), v.end(), out); }
  });
}
int or_rotation_kernel(double vsini, double dvelo, double *out, int cap) {
  int n = 0;
  int rc = guard([&] {
    std::vector<float> k32; std::vector<double> k64;
    rotation_kernel(vsini, dvelo, k32, k64);
    n = (int)k32.size();
    for (int i = 0; i < n && i < cap; i++) out[i] = k32[i];
  });
  return rc ? rc : n;
}
int or_convolve_rotation(const OGrid *g, int prec, const double *in, double vsini, double *out) {
  return guard([&] {
    if (prec == OP_F32) { std::vector<float> x(in, in + g->npx); auto v = convolve_rotation<float>(*g, x, vsini); std::copy(v.begin(), v.end(), out); }
    else { std::vector<double> x(in, in + g->npx); auto v = convolve_rotation<double>(*g, x, vsini); std::copy(v.begin(), v.end(), out); }
  });
}

// lib.rs:763-797 + convolve_rv.rs:77-86, 169-196, 244-287, 350-402
ODisp *or_disp_create(const OGrid *g, int kind, const double *wl_obs, int64_t n_obs, double resolution, const float *disp) {
  ODisp *d = new ODisp();
  int rc = guard([&] {
    d->g = g;
    d->kind = kind;
    d->wl.assign(wl_obs, wl_obs + n_obs);
    d->fidx.resize(n_obs);
    for (int64_t i = 0; i < n_obs; i++) d->fidx[i] = g->wl.float_index(wl_obs[i]);
    const WlGrid &w = g->wl;
    if (kind == ODISP_FIXED) {
      if (resolution <= 0.0) fail("Resolution must be positive");
      if (w.kind == OWL_LOGSPACE) {
        double sigma = 1.0 / (M_LN10 * 2.355 * resolution * w.b);
        int n = odd_width(6.0 * sigma);
        d->gk32.assign(n, 0.0f); d->gk64.assign(n, 0.0);
        make_gaussian32(d->gk32.data(), n, (float)sigma);
        make_gaussian64(d->gk64.data(), n, sigma);
        d->half = (n - 1) / 2;
        d->width = n;
      } else {
        std::vector<float> s32(w.n); std::vector<double> s64(w.n);
        for (int64_t i = 0; i < w.n; i++) {
          if (w.kind == OWL_LINSPACE) { double v = w.at(i) / (resolution * w.b * 2.355); s32[i] = (float)v; s64[i] = v; }
          else if (i == 0 || i == w.n - 1) { s32[i] = 2.0f; s64[i] = 2.0; }
          else { double st = (w.vals[i + 1] - w.vals[i - 1]) / 2.0; double v = w.vals[i] / (resolution * st * 2.355); s32[i] = (float)v; s64[i] = v; }
        }
        build_per_pixel(*d, s32, s64);
      }
    } else if (kind == ODISP_VARIABLE) {
      auto dr = resample_observed_to_synth(d->wl, w, disp);
      std::vector<float> s32(w.n); std::vector<double> s64(w.n);
      for (int64_t i = 0; i < w.n; i++) {
        if (w.kind == OWL_LOGSPACE) { float den = (float)(w.b * M_LN10 * w.at(i)); s32[i] = dr[i] / den; s64[i] = (double)dr[i] / (w.b * M_LN10 * w.at(i)); }
        else if (w.kind == OWL_LINSPACE) { s32[i] = dr[i] / (float)w.b; s64[i] = (double)dr[i] / w.b; }
        else if (i == 0 || i == w.n - 1) { s32[i] = 2.0f; s64[i] = 2.0; }
        else { double st = (w.vals[i + 1] - w.vals[i - 1]) / 2.0; s32[i] = dr[i] / (float)st; s64[i] = (double)dr[i] / st; }
      }
      build_per_pixel(*d, s32, s64);
    }
  });
  if (rc) { delete d; return nullptr; }
  return d;
}
void or_disp_free(ODisp *d) { delete d; }
int or_disp_kernel_width(const ODisp *d) { return d->width; }
int or_disp_convolve(const ODisp *d, int prec, const double *in, double *out) {
  return guard([&] {
    if (prec == OP_F32) { std::vector<float> x(in, in + d->g->npx); auto v = disp_convolve<float>(*d, x); std::copy(v.begin(), v.end(), out); }
    else { std::vector<double> x(in, in + d->g->npx); auto v = disp_convolve<double>(*d, x); std::copy(v.begin(), v.end(), out); }
  });
}
int or_produce_model(const OGrid *g, const ODisp *d, int prec, const double *lab, double *out) {
  return guard([&] {
    if (prec == OP_F32) { auto v = produce_model<float>(*g, *d, lab); std::copy(v.begin(), v.end(), out); }
    else { auto v = produce_model<double>(*g, *d, lab); std::copy(v.begin(), v.end(), out); }
  });
}

// lib.rs:945-983
OCont *or_cont_create(int kind, const double *wl, int64_t n, int n_chunks, int p_order, double overlap,
                      const float *design, int k, const float *continuum, int ignore) {
  OCont *c = new OCont();
  int rc = guard([&] {
    c->kind = kind;
    c->n = n;
    if (kind == OCONT_CHUNK) {
      if (n_chunks < 1 || p_order < 0) fail("invalid chunk settings");
      c->n_chunks = n_chunks; c->p = p_order;
      c->wl.assign(wl, wl + n);
      c->start.resize(n_chunks); c->stop.resize(n_chunks);
      for (int i = 0; i < n_chunks; i++) {  // continuum_fitting.rs:144-165
        double s = map_range((double)i - overlap, 0.0, (double)n_chunks, wl[0], wl[n - 1], true);
        double e = map_range((double)i + 1.0 + overlap, 0.0, (double)n_chunks, wl[0], wl[n - 1], true);
        int64_t a = -1, b = -1;
        for (int64_t j = 0; j < n; j++) if (wl[j] > s) { a = j; break; }
        for (int64_t j = n - 1; j >= 0; j--) if (wl[j] < e) { b = j; break; }
        if (a < 0 || b < 0) fail("chunk %d has no pixels", i);
        c->start[i] = a; c->stop[i] = b + 1;
      }
      c->start[0] = 0;
      c->stop[n_chunks - 1] = n;
      chunk_setup(*c);
    } else if (kind == OCONT_LINEAR) {
      c->k = k;
      c->d32.assign(design, design + (size_t)n * k);
      c->d64.assign(c->d32.begin(), c->d32.end());
      std::vector<float> col32((size_t)n * k);
      std::vector<double> col64((size_t)n * k);
      for (int64_t i = 0; i < n; i++) for (int j = 0; j < k; j++) { col32[(size_t)j * n + i] = design[(size_t)i * k + j]; col64[(size_t)j * n + i] = design[(size_t)i * k + j]; }
      c->lqr32.factor(col32, n, k);
      c->lqr64.factor(col64, n, k);
    } else if (kind == OCONT_FIXED) {
      c->cont.assign(continuum, continuum + n);
      c->ignore = ignore;
    }
  });
  if (rc) { delete c; return nullptr; }
  return c;
}
void or_cont_free(OCont *c) { delete c; }
int or_cont_nparams(const OCont *c) {
  if (c->kind == OCONT_CHUNK) return c->n_chunks * (c->p + 1);
  if (c->kind == OCONT_LINEAR) return c->k;
  return 1;
}
int or_cont_chunk_bounds(const OCont *c, int64_t *ss) {
  for (int i = 0; i < c->n_chunks; i++) { ss[2 * i] = c->start[i]; ss[2 * i + 1] = c->stop[i]; }
  return c->n_chunks;
}
int or_fit_continuum(const OCont *c, int prec, const float *flux, const float *var, const double *model, int64_t n,
                     double *params, double *chi2) {
  return guard([&] {
    std::vector<double> pv;
    if (prec == OP_F32) { std::vector<float> m(model, model + n); fit_continuum<float>(*c, flux, var, m, pv, *chi2); }
    else { std::vector<double> m(model, model + n); fit_continuum<double>(*c, flux, var, m, pv, *chi2); }
    std::copy(pv.begin(), pv.end(), params);
  });
}
int or_build_continuum(const OCont *c, int prec, const double *params, double *out) {
  return guard([&] {
    if (c->kind == OCONT_CHUNK) {
      if (prec == OP_F32) { auto v = chunk_build<float>(*c, params); std::copy(v.begin(), v.end(), out); }
      else { auto v = chunk_build<double>(*c, params); std::copy(v.begin(), v.end(), out); }
    } else if (c->kind == OCONT_LINEAR) {
      for (int64_t i = 0; i < c->n; i++) {
        if (prec == OP_F32) { float a = 0.0f; for (int j = 0; j < c->k; j++) a = a + c->d32[(size_t)i * c->k + j] * (float)params[j]; out[i] = a; }
        else { double a = 0.0; for (int j = 0; j < c->k; j++) a += c->d64[(size_t)i * c->k + j] * params[j]; out[i] = a; }
      }
    } else if (c->kind == OCONT_FIXED) {
      for (int64_t i = 0; i < c->n; i++) out[i] = c->cont[i];
    } else {
      out[0] = params[0];
    }
  });
}
int or_chi2(const OGrid *g, const ODisp *d, const OCont *c, int prec, const float *flux, const float *var, int64_t n,
            const double *labels, int64_t L, double *out, int *status, int nthreads) {
  if (n != (int64_t)d->wl.size()) { g_err = "Observed spectrum and target dispersion must have the same length"; return -1; }
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (int64_t i = 0; i < L; i++) {
    try {
      out[i] = prec == OP_F32 ? cost<float>(*g, *d, *c, flux, var, labels + 5 * i)
                              : cost<double>(*g, *d, *c, flux, var, labels + 5 * i);
      status[i] = 0;
    } catch (const std::exception &e) {
      out[i] = NAN;
      status[i] = -1;
    }
  }
  return 0;
}
int or_fit(const OGrid *g, const ODisp *d, const OCont *c, int prec, const OPsoSettings *st, const float *flux,
           const float *var, int64_t n, int64_t S, const uint64_t *seeds, int nthreads, int over_stars,
           OFitResult *out, double *trace) {
  if (n != (int64_t)d->wl.size()) { g_err = "Observed spectrum and target dispersion must have the same length"; return -1; }
  std::vector<std::string> errs(S);
  int any = 0;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1) if (over_stars)
  for (int64_t s = 0; s < S; s++) {
    std::memset(&out[s], 0, sizeof(OFitResult));
    try {
      if (prec == OP_F32)
        fit_one<float>(*g, *d, *c, *st, flux + (size_t)s * n, var + (size_t)s * n, seeds[s], nthreads, !over_stars, out[s], s == 0 ? trace : nullptr);
      else
        fit_one<double>(*g, *d, *c, *st, flux + (size_t)s * n, var + (size_t)s * n, seeds[s], nthreads, !over_stars, out[s], s == 0 ? trace : nullptr);
      out[s].status = 0;
    } catch (const std::exception &e) {
      out[s].status = -1;
      errs[s] = e.what();
#pragma omp atomic write
      any = 1;
    }
  }
  if (any) for (int64_t s = 0; s < S; s++) if (out[s].status) { g_err = errs[s]; break; }
  return any ? -1 : 0;
}

int or_local_grid_linear(const OGrid *g, double t, double m, double l, int64_t *cols, double *w) {
  return guard([&] { local_grid_linear(*g, t, m, l, cols, w); });
}
int or_interpolate_linear(const OGrid *g, int prec, double t, double m, double l, double *out) {
  return guard([&] {
    if (prec == OP_F32) { auto v = interpolate_linear<float>(*g, t, m, l); std::copy(v.begin(), v.end(), out); }
    else { auto v = interpolate_linear<double>(*g, t, m, l); std::copy(v.begin(), v.end(), out); }
  });
}
int or_binary_model(const OGrid *g, const OGrid *gc, const ODisp *d, int prec, const double *lab, double *out) {
  return guard([&] {
    if (prec == OP_F32) { auto v = binary_model<float>(*g, *gc, *d, lab); std::copy(v.begin(), v.end(), out); }
    else { auto v = binary_model<double>(*g, *gc, *d, lab); std::copy(v.begin(), v.end(), out); }
  });
}
int or_binary_chi2(const OGrid *g, const OGrid *gc, const ODisp *d, const OCont *c, int prec, const float *flux,
                   const float *var, int64_t n, const double *labels, int64_t L, double *out, int *status,
                   int nthreads) {
  if (n != (int64_t)d->wl.size()) { g_err = "Observed spectrum and target dispersion must have the same length"; return -1; }
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1)
  for (int64_t i = 0; i < L; i++) {
    try {
      out[i] = prec == OP_F32 ? binary_cost<float>(*g, *gc, *d, *c, flux, var, labels + 11 * i)
                              : binary_cost<double>(*g, *gc, *d, *c, flux, var, labels + 11 * i);
      status[i] = 0;
    } catch (const std::exception &e) {
      out[i] = NAN;
      status[i] = -1;
    }
  }
  return 0;
}
int or_binary_fit(const OGrid *g, const OGrid *gc, const ODisp *d, const OCont *c, int prec,
                  const OBinarySettings *st, const float *flux, const float *var, int64_t n, uint64_t seed,
                  int nthreads, OBinaryResult *out, double *trace) {
  if (n != (int64_t)d->wl.size()) { g_err = "Observed spectrum and target dispersion must have the same length"; return -1; }
  std::memset(out, 0, sizeof(OBinaryResult));
  int rc = guard([&] {
    if (prec == OP_F32) fit_binary<float>(*g, *gc, *d, *c, *st, flux, var, seed, nthreads, *out, trace);
    else fit_binary<double>(*g, *gc, *d, *c, *st, flux, var, seed, nthreads, *out, trace);
  });
  out->status = rc;
  return rc;
}

}  // extern "C"
