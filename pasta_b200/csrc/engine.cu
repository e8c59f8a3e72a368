// engine.cu -- host engine and C ABI of pasta_b200.
//
// Owns device memory for grids, dispersions, continuum fitters and
// evaluation workspaces; runs the evaluation pipeline
//   prep -> rotation spectra -> interpolation -> rotation FFT ->
//   instrument profile -> resampling + continuum + chi2
// over batches of (star, label) evaluations; drives the particle swarm
// either fully on the device (batched form, one CUDA graph per PSO step)
// or with the swarm on the host one star at a time (plain form).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <limits>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <array>
#include <vector>

#include "../../include/pasta_b200.h"
#include "common.cuh"
#include "kernels.h"

using namespace pb;

namespace {

thread_local std::string g_last_error;

struct PErr : std::runtime_error {
  int code;
  PErr(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] void fail(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  throw PErr(code, buf);
}
#define CK(call)                                                                                 \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) fail(PASTA_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

template <class F>
int guard(F &&f) {
  try {
    f();
    return PASTA_OK;
  } catch (const PErr &e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::bad_alloc &) {
    g_last_error = "host allocation failed";
    return PASTA_E_NOMEM;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return PASTA_E_INTERNAL;
  }
}

const char *status_message(int s) {
  switch (s) {
    case S_OUT_OF_GRID: return "label outside the grid";
    case S_NEIGHBORS: return "not enough grid neighbours for cubic interpolation";
    case S_VSINI: return "vsini must be positive";
    case S_KERNEL_WIDTH: return "rotation kernel is larger than FFTSIZE (2048)";
    case S_RV_RANGE: return "shifted observed wavelengths leave the synthetic grid";
    case S_RESAMPLE: return "resampling index out of range";
    case S_BOUNDS: return "particle is not within bounds";
    case S_CLAMP: return "clamp limits are invalid";
    case S_CONTINUUM: return "continuum fitter cannot evaluate chi2 on this spectrum";
    case S_NAN: return "NaN label";
    case S_UNSUPPORTED: return "non-equidistant wavelength grid not supported";
    default: return "error";
  }
}

// ---------------------------------------------------------------- memory
template <class T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    release();
    if (count == 0) return;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      fail(PASTA_E_NOMEM, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
    }
    n = count;
  }
  void upload(const T *h, size_t count) {
    alloc(count);
    if (count) CK(cudaMemcpy(p, h, count * sizeof(T), cudaMemcpyHostToDevice));
  }
  void upload(const std::vector<T> &v) { upload(v.data(), v.size()); }
};

// page-locked host buffer: copies from and to it are asynchronous and can
// be captured in a CUDA graph
template <class T>
struct HostBuf {
  T *p = nullptr;
  HostBuf() = default;
  HostBuf(const HostBuf &) = delete;
  HostBuf &operator=(const HostBuf &) = delete;
  ~HostBuf() {
    if (p) cudaFreeHost(p);
  }
  void alloc(size_t count) {
    if (p) cudaFreeHost(p);
    p = nullptr;
    if (count == 0) return;
    cudaError_t e = cudaMallocHost(&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      fail(PASTA_E_NOMEM, "cudaMallocHost of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
    }
  }
};

// an instantiated CUDA graph, destroyed with its owner
struct GraphHold {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  GraphHold() = default;
  GraphHold(const GraphHold &) = delete;
  GraphHold &operator=(const GraphHold &) = delete;
  ~GraphHold() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

struct Ctx {
  int dev = 0;
  cudaStream_t stream = nullptr;
  DBuf<float2> tw;  // W_2048^k
};
std::mutex g_ctx_mu;
std::map<int, std::unique_ptr<Ctx>> g_ctx;
thread_local int g_dev = -1;

Ctx &ctx() {
  if (g_dev < 0) {
    int d;
    CK(cudaGetDevice(&d));
    g_dev = d;
  }
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  auto &c = g_ctx[g_dev];
  if (!c) {
    c.reset(new Ctx());
    c->dev = g_dev;
    CK(cudaSetDevice(g_dev));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    std::vector<float2> t(FFTN);
    for (int k = 0; k < FFTN; k++) {
      double a = -2.0 * M_PI * (double)k / (double)FFTN;
      t[k] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    c->tw.upload(t);
  }
  CK(cudaSetDevice(c->dev));
  return *c;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// =================================================================== grid
// slots of the table that merges evaluations alone in their segment: a power
// of two, at least twice the evaluations (at most half full)
int merge_table_slots(int64_t evals) {
  int64_t n = 1024;
  while (n < 2 * evals) n *= 2;
  return (int)n;
}

struct Workspace {
  int64_t cap = 0, stride = 0;
  int bnd_stride = 0;
  int64_t gen = 0;  // bumped on every reallocation (captured graphs compare it)
  DBuf<float> A, B;
  DBuf<float2> H, HG;
  DBuf<EvalPrep> prep;
  DBuf<int> bnd;       // first observed pixel per broadening block
  DBuf<GroupRec> grec; // interpolation groups, at each segment's first evaluation
  DBuf<int> gcount;    // groups per segment
  DBuf<TcGroup> tcrec; // tensor-core interpolation groups, at each segment's first evaluation
  DBuf<int> tccount;   // tensor-core groups per segment
  DBuf<int> tclist;    // indices of all tensor-core groups, and their count [1]
  DBuf<int> tclist_count;
  DBuf<double> cpart;  // chunk chi2 partials [cap][MAX_CHUNKS]
  DBuf<int> dlist;     // evaluations on the direct broadening path [cap], and their count [1]
  DBuf<double> zpart;  // tensor-core linear continua: partial coefficients [cap][LIN_MAX_SLICES][64]
  DBuf<int> dcount;
  // merging of evaluations alone in their segment (EvalBatch::mkey)
  int mtab = 0;
  DBuf<unsigned long long> mkey;
  DBuf<int> mcnt, mmem, mslot, erec, mrcount;
  DBuf<GroupRec> mrec;
  void ensure(int64_t want, int64_t str, int bstr) {
    if (want <= cap && str == stride && bstr == bnd_stride) return;
    A.release(); B.release(); H.release(); HG.release(); prep.release();
    bnd.release(); cpart.release(); grec.release(); gcount.release();
    tcrec.release(); tccount.release(); tclist.release(); tclist_count.release();
    dlist.release(); dcount.release(); zpart.release();
    mkey.release(); mcnt.release(); mmem.release(); mslot.release(); erec.release(); mrec.release(); mrcount.release();
    cap = 0;
    A.alloc((size_t)want * str);
    B.alloc((size_t)want * str);
    H.alloc((size_t)want * 1025);
    HG.alloc((size_t)want * 1025);
    prep.alloc((size_t)want);
    bnd.alloc((size_t)want * bstr);
    grec.alloc((size_t)(want + SEG - 1) / SEG * SEG);
    gcount.alloc((size_t)want);
    tcrec.alloc((size_t)want);
    tccount.alloc((size_t)want);
    tclist.alloc((size_t)want);
    tclist_count.alloc(1);
    cpart.alloc((size_t)want * MAX_CHUNKS);
    dlist.alloc((size_t)want);
    zpart.alloc((size_t)want * LIN_MAX_SLICES * 64);
    dcount.alloc(1);
    mtab = merge_table_slots(want);
    mkey.alloc((size_t)mtab);
    mcnt.alloc((size_t)mtab);
    mmem.alloc((size_t)mtab * MERGE_CAP);
    mslot.alloc((size_t)mtab + 1);
    erec.alloc((size_t)want);
    mrec.alloc((size_t)(want + 1) / 2);
    mrcount.alloc(1);
    cap = want;
    stride = str;
    bnd_stride = bstr;
    gen++;
  }
};

// bytes of workspace one evaluation takes with rows of `stride` floats
int64_t workspace_bytes_per_eval(int64_t stride, int bnd_stride) {
  return stride * 8 + 2 * 1025 * 8 + (int64_t)sizeof(EvalPrep) + (int64_t)sizeof(GroupRec) + (int64_t)sizeof(TcGroup) +
         8 + (int64_t)bnd_stride * 4 +
         (int64_t)MAX_CHUNKS * 8 + 4 + (int64_t)LIN_MAX_SLICES * 64 * 8 +
         // merge table (up to 4 slots per evaluation), own-record index, merged records
         4 * (8 + 4 + 4 * MERGE_CAP + 4) + 4 + (int64_t)sizeof(GroupRec) / 2;
}

struct pasta_grid {
  int dev = 0;
  DevGrid d{};
  GridGeom hg{};
  std::vector<double> tv, mv, lv, wl_vals;
  std::vector<int> llo, lhi;
  std::vector<int64_t> cum;
  int64_t n_cols = 0, npx = 0, stride = 0;
  int wl_kind = WL_LOG;
  double wl_a = 0, wl_b = 0;
  DBuf<uint16_t> spectra;
  DBuf<float> factor;
  DBuf<double> dtv, dmv, dlv, dwl;
  DBuf<int> dllo, dlhi;
  DBuf<int64_t> dcum;
  std::mutex mu;
  Workspace ws;
  int direct_max = 0;  // combined kernels of at most this many taps are broadened directly (measured)
  alignas(64) CUtensorMap tmap;  // TMA view of the resident rows (tensor-core interpolation)
  bool has_tmap = false;
  int tc_min = 16;  // members from which a shared-row group is interpolated on the tensor cores (measured)
};

namespace {

int64_t workspace_cap(const pasta_grid *g, int64_t want, int64_t stride) {
  // per evaluation: two spectrum rows + rotation half spectrum + prep record
  // + block bounds + chunk coefficients and partial sums
  const int64_t per = workspace_bytes_per_eval(stride, bnd_stride_for((int)g->npx));
  // default: up to 40% of the device's memory for evaluation workspaces
  int64_t budget = 24ll << 30;
  size_t fr = 0, tot = 0;
  const bool have = cudaMemGetInfo(&fr, &tot) == cudaSuccess;
  if (have) budget = (int64_t)(0.4 * (double)tot);
  if (const char *e = getenv("PASTA_WORKSPACE_BYTES")) budget = atoll(e);
  if (have) {
    const int64_t avail = (int64_t)fr - (2ll << 30) +
                          (int64_t)g->ws.cap * workspace_bytes_per_eval(g->ws.stride, g->ws.bnd_stride);
    if (avail < budget) budget = avail;
  }
  int64_t cap = std::max<int64_t>(1, budget / per);
  return std::min<int64_t>(cap, std::max<int64_t>(want, 1));
}

}  // namespace

// ============================================================ dispersion
struct pasta_dispersion {
  int kind = PASTA_DISP_NONE, dev_kind = DISP_NONE;
  int synth_kind = WL_LOG;
  double synth_a = 0, synth_b = 0;
  int64_t synth_n = 0;
  std::vector<double> synth_vals, wl, fidx;
  double wl_first = 0, wl_last = 0, wl_min = 0, wl_max = 0, fidx_min = 0, fidx_max = 0;
  int sorted = 0;  // observed wavelengths and float indices never decrease
  int gw = 0;
  std::vector<float> gk;  // fixed: [gw]; per pixel: [synth_n][gw]
  DBuf<double> dfidx, dwl;
  DBuf<float> dgk;
  DBuf<float2> dgspec;  // fixed kernel: 2048-point spectrum (1025 bins)
};

namespace {
// Spectrum of a short real kernel zero-padded to 2048 points, in double
// (radix-2, iterative), returned as 1025 f32 bins.
std::vector<float2> kernel_spectrum(const std::vector<float> &k) {
  const int n = FFTN;
  std::vector<double> re(n, 0.0), im(n, 0.0);
  for (size_t i = 0; i < k.size() && i < (size_t)n; i++) re[i] = k[i];
  for (int i = 1, j = 0; i < n; i++) {  // bit reversal
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) { std::swap(re[i], re[j]); std::swap(im[i], im[j]); }
  }
  for (int len = 2; len <= n; len <<= 1) {
    const double ang = -2.0 * M_PI / len;
    for (int i = 0; i < n; i += len)
      for (int j = 0; j < len / 2; j++) {
        const double wr = std::cos(ang * j), wi = std::sin(ang * j);
        const double ar = re[i + j + len / 2], ai = im[i + j + len / 2];
        const double vr = ar * wr - ai * wi, vi = ar * wi + ai * wr;
        re[i + j + len / 2] = re[i + j] - vr;
        im[i + j + len / 2] = im[i + j] - vi;
        re[i + j] += vr;
        im[i + j] += vi;
      }
  }
  std::vector<float2> out(n / 2 + 1);
  for (int i = 0; i <= n / 2; i++) out[i] = make_float2((float)re[i], (float)im[i]);
  return out;
}
}  // namespace

namespace {

// WlGrid helpers (interpolate.rs:681-743)
double wl_at(int kind, double a, double b, const std::vector<double> &v, int64_t i) {
  if (kind == WL_LIN) return a + b * (double)i;
  if (kind == WL_LOG) return std::pow(10.0, a + b * (double)i);
  return v[i];
}
double wl_float_index(int kind, double a, double b, const std::vector<double> &v, double wl) {
  if (kind == WL_LIN) return (wl - a) / b;
  if (kind == WL_LOG) return (std::log10(wl) - a) / b;
  auto it = std::lower_bound(v.begin(), v.end(), wl);
  int64_t i = it - v.begin();
  if (i < (int64_t)v.size() && v[i] == wl) return (double)i;
  if (i == 0) return 0.0;
  if (i == (int64_t)v.size()) return (double)v.size() - 1.0;
  return (wl - v[i - 1]) / (v[i] - v[i - 1]) + (double)i - 1.0;
}

// convolve_rv.rs:107-118 (f32)
void make_gaussian(float *arr, int n, float sigma) {
  int mid = (n - 1) / 2;
  for (int i = 0; i < n; i++) {
    float x = ((float)i - (float)mid) / sigma;
    arr[i] = std::exp(-0.5f * x * x);
  }
  float s = 0.0f;
  for (int i = 0; i < n; i++) s = s + arr[i];
  for (int i = 0; i < n; i++) arr[i] = arr[i] / s;
}
int odd_width(double six_sigma) {
  double c = std::ceil(six_sigma);
  int64_t nme = c > 0 ? (int64_t)c : 0;
  return (int)(nme + 1 - nme % 2);
}

void disp_per_pixel(pasta_dispersion *d, const std::vector<float> &sig) {
  float largest = sig[0];
  for (float s : sig) if (s > largest) largest = s;
  int w = odd_width((double)(largest * 6.0f));
  if (w > 2 * 255 + 1) fail(PASTA_E_UNSUPPORTED, "instrument kernel of %d taps exceeds the supported 511", w);
  d->gw = w;
  d->dev_kind = DISP_PIXEL;
  d->gk.assign((size_t)w * sig.size(), 0.0f);
  for (size_t i = 0; i < sig.size(); i++) make_gaussian(&d->gk[i * w], w, sig[i]);
}

}  // namespace

// ============================================================= continuum
struct pasta_continuum {
  int kind = PASTA_CONT_CHUNK;
  int64_t n = 0;
  int bad = 0;
  std::string bad_msg;
  // chunk
  int nc = 0, p1 = 0;
  std::vector<int> cstart, cstop;
  std::vector<float> xa, xb, fac;
  std::vector<double> chol;  // nc x p1 x p1
  // linear
  int k = 0;
  std::vector<float> qcol;  // k x n column-major
  std::vector<double> R;    // k x k upper (row-major)
  int kp = 0;               // k padded to a multiple of 16 for the tensor-core path (0: k > 64)
  std::vector<float> qt;    // n x kp pixel-major copy of the basis (zero padded)
  // fixed
  std::vector<float> cont;
  int ignore = 0;
  DBuf<int> dcs, dce;
  DBuf<float> dxa, dxb, dfac, dq, dqt, dcont;
  DBuf<double> dchol;
};

namespace {

template <class F>
F map_range(F x, F fl, F fh, F tl, F th, bool clamp) {  // continuum_fitting.rs:109-116
  F v = (x - fl) / (fh - fl) * (th - tl) + tl;
  if (clamp) v = std::min(std::max(v, tl), th);
  return v;
}
float poly_blend(float x) {  // continuum_fitting.rs:119-123
  float xc = std::min(std::max(x, 0.0f), 1.0f);
  float s = std::sin(xc * (float)M_PI / 2.0f);
  return s * s;
}
// Legendre values at x exactly as the device evaluates them (f32 recurrence
// with explicit rounding, common.cuh), widened to double for the Gram.
void legendre_host(float x, int p1, double *P) {
  float p[MAX_P1];
  p[0] = 1.0f;
  if (p1 > 1) p[1] = x;
  for (int k = 1; k + 1 < p1; k++) p[k + 1] = leg_step(leg_a(k), leg_c(k), x, p[k], p[k - 1]);
  for (int k = 0; k < p1; k++) P[k] = (double)p[k];
}
// monomial coefficients of P_0..P_{p1-1}: T[k][j]
std::vector<double> legendre_to_monomial(int p1) {
  std::vector<double> T((size_t)p1 * p1, 0.0);
  T[0] = 1.0;
  if (p1 > 1) T[(size_t)1 * p1 + 1] = 1.0;
  for (int k = 1; k + 1 < p1; k++) {
    const double a = (double)(2 * k + 1) / (double)(k + 1), c = (double)k / (double)(k + 1);
    for (int j = 0; j < p1; j++) {
      double v = -c * T[(size_t)(k - 1) * p1 + j];
      if (j > 0) v += a * T[(size_t)k * p1 + j - 1];
      T[(size_t)(k + 1) * p1 + j] = v;
    }
  }
  return T;
}

// ChunkFitter::new (continuum_fitting.rs:140-214) plus the Legendre Gram
// Cholesky factors used by the device solve.
void chunk_setup(pasta_continuum *c, const double *wl, int n_chunks, int p_order, double overlap) {
  const int64_t n = c->n;
  if (n_chunks < 1) fail(PASTA_E_ARG, "n_chunks must be >= 1");
  if (n_chunks > MAX_CHUNKS) fail(PASTA_E_UNSUPPORTED, "at most %d chunks are supported", MAX_CHUNKS);
  if (p_order < 0 || p_order + 1 > MAX_P1) fail(PASTA_E_UNSUPPORTED, "polynomial order must be 0..%d", MAX_P1 - 1);
  if (n < 2) fail(PASTA_E_ARG, "wavelength array too short");
  c->nc = n_chunks;
  c->p1 = p_order + 1;
  c->cstart.resize(n_chunks);
  c->cstop.resize(n_chunks);
  for (int i = 0; i < n_chunks; i++) {
    double s = map_range((double)i - overlap, 0.0, (double)n_chunks, wl[0], wl[n - 1], true);
    double e = map_range((double)i + 1.0 + overlap, 0.0, (double)n_chunks, wl[0], wl[n - 1], true);
    int64_t a = -1, b = -1;
    for (int64_t j = 0; j < n; j++) if (wl[j] > s) { a = j; break; }
    for (int64_t j = n - 1; j >= 0; j--) if (wl[j] < e) { b = j; break; }
    if (a < 0 || b < 0) fail(PASTA_E_ARG, "chunk %d has no pixels", i);
    c->cstart[i] = (int)a;
    c->cstop[i] = (int)(b + 1);
  }
  c->cstart[0] = 0;
  c->cstop[n_chunks - 1] = (int)n;
  const int nc = n_chunks, p1 = c->p1;
  for (int i = 0; i < nc; i++)
    if (c->cstop[i] - c->cstart[i] < 2) fail(PASTA_E_ARG, "chunk %d is empty", i);
  c->xa.assign(n, 0.0f);
  c->xb.assign(n, 0.0f);
  c->fac.assign(n, 0.0f);
  for (int ch = 0; ch < nc; ch++) {
    const int s = c->cstart[ch], e = c->cstop[ch];
    for (int i = s; i < e; i++) {
      float x = (float)map_range(wl[i], wl[s], wl[e - 1], -1.0, 1.0, false);
      if (ch > 0 && i < c->cstop[ch - 1]) c->xb[i] = x;  // overlap with the previous chunk
      else c->xa[i] = x;
    }
  }
  for (int ch = 0; ch + 1 < nc; ch++) {  // factor_arrays (continuum_fitting.rs:184-200)
    const int e = c->cstop[ch], sn = c->cstart[ch + 1];
    for (int i = sn; i < e; i++)
      c->fac[i] = poly_blend(map_range((float)wl[i], (float)wl[sn], (float)wl[e - 1], 1.0f, 0.0f, false));
  }
  // Legendre Gram per chunk, FP64 Cholesky
  c->chol.assign((size_t)nc * p1 * p1, 0.0);
  std::vector<double> G((size_t)p1 * p1), P(p1);
  for (int ch = 0; ch < nc && !c->bad; ch++) {
    std::fill(G.begin(), G.end(), 0.0);
    for (int i = c->cstart[ch]; i < c->cstop[ch]; i++) {
      const float xf = (ch > 0 && i < c->cstop[ch - 1]) ? c->xb[i] : c->xa[i];
      legendre_host(xf, p1, P.data());
      for (int a = 0; a < p1; a++)
        for (int b = 0; b <= a; b++) G[(size_t)a * p1 + b] += P[a] * P[b];
    }
    double *L = &c->chol[(size_t)ch * p1 * p1];
    for (int a = 0; a < p1; a++) {
      for (int b = 0; b <= a; b++) {
        double s = G[(size_t)a * p1 + b];
        for (int k = 0; k < b; k++) s -= L[a * p1 + k] * L[b * p1 + k];
        if (a == b) {
          if (!(s > 1e-12 * std::max(1.0, G[(size_t)a * p1 + a]))) {
            c->bad = 1;
            c->bad_msg = "chunk polynomial basis is rank deficient";
            s = 1.0;
          }
          L[a * p1 + a] = std::sqrt(s);
        } else {
          L[a * p1 + b] = s / L[b * p1 + b];
        }
      }
    }
  }
  // the reference's chi2 loops panic on these layouts (continuum_fitting.rs:301-357)
  if (!c->bad) {
    if (nc < 2) { c->bad = 1; c->bad_msg = "chunk fitter needs at least 2 chunks"; }
    else if (n < 100) { c->bad = 1; c->bad_msg = "spectrum shorter than 100 pixels"; }
    else if (c->cstart[1] < 50) { c->bad = 1; c->bad_msg = "second chunk starts before pixel 50"; }
    else {
      for (int ch = 1; ch < nc; ch++) {
        const int nx = ch == nc - 1 ? (int)n - 50 : c->cstart[ch + 1];
        if (c->cstop[ch - 1] < c->cstart[ch] || nx < c->cstop[ch - 1]) {
          c->bad = 1;
          c->bad_msg = "chunk overlaps are inconsistent";
          break;
        }
      }
    }
  }
}

// LinearModelFitter::new (continuum_fitting.rs:53-56): thin Householder QR
// in double of the design matrix; Q (f32) spans the same column space.
void linear_setup(pasta_continuum *c, const float *design, int k) {
  const int64_t n = c->n;
  if (k < 1 || k > MAX_LIN_K) fail(PASTA_E_UNSUPPORTED, "design matrix must have 1..%d columns", MAX_LIN_K);
  if (n < k) fail(PASTA_E_ARG, "design matrix has fewer rows than columns");
  c->k = k;
  std::vector<double> A((size_t)n * k);  // column-major
  for (int64_t i = 0; i < n; i++)
    for (int j = 0; j < k; j++) A[(size_t)j * n + i] = design[(size_t)i * k + j];
  std::vector<double> beta(k, 0.0);
  c->R.assign((size_t)k * k, 0.0);
  for (int j = 0; j < k; j++) {
    double *cj = &A[(size_t)j * n];
    double nrm = 0.0;
    for (int64_t i = j; i < n; i++) nrm += cj[i] * cj[i];
    nrm = std::sqrt(nrm);
    double alpha = cj[j] > 0 ? -nrm : nrm;
    if (nrm == 0.0) { beta[j] = 0.0; c->R[(size_t)j * k + j] = 0.0; continue; }
    cj[j] -= alpha;
    double vv = 0.0;
    for (int64_t i = j; i < n; i++) vv += cj[i] * cj[i];
    beta[j] = 2.0 / vv;
    for (int l = j + 1; l < k; l++) {
      double *cl = &A[(size_t)l * n];
      double s = 0.0;
      for (int64_t i = j; i < n; i++) s += cj[i] * cl[i];
      s *= beta[j];
      for (int64_t i = j; i < n; i++) cl[i] -= s * cj[i];
    }
    c->R[(size_t)j * k + j] = alpha;
    for (int l = j + 1; l < k; l++) c->R[(size_t)j * k + l] = A[(size_t)l * n + j];
  }
  double rmax = 0.0;
  for (int j = 0; j < k; j++) rmax = std::max(rmax, std::fabs(c->R[(size_t)j * k + j]));
  for (int j = 0; j < k; j++)
    if (!(std::fabs(c->R[(size_t)j * k + j]) > 1e-10 * rmax)) {
      c->bad = 1;
      c->bad_msg = "design matrix is rank deficient";
    }
  // explicit Q: apply the reflectors to the first k unit vectors
  c->qcol.assign((size_t)k * n, 0.0f);
  std::vector<double> q(n);
  for (int col = 0; col < k; col++) {
    std::fill(q.begin(), q.end(), 0.0);
    q[col] = 1.0;
    for (int j = k - 1; j >= 0; j--) {
      if (beta[j] == 0.0) continue;
      const double *v = &A[(size_t)j * n];
      double s = 0.0;
      for (int64_t i = j; i < n; i++) s += v[i] * q[i];
      s *= beta[j];
      for (int64_t i = j; i < n; i++) q[i] -= s * v[i];
    }
    for (int64_t i = 0; i < n; i++) c->qcol[(size_t)col * n + i] = (float)q[i];
  }
  // pixel-major copy for the tensor-core products (at most 64 columns)
  c->kp = k <= 64 ? (k + 15) / 16 * 16 : 0;
  if (c->kp) {
    c->qt.assign((size_t)n * c->kp, 0.0f);
    for (int col = 0; col < k; col++)
      for (int64_t i = 0; i < n; i++) c->qt[(size_t)i * c->kp + col] = c->qcol[(size_t)col * n + i];
  }
}

// Host result of a continuum solve -> the reference's parameter vector.
std::vector<float> params_from_device(const pasta_continuum *c, const double *p) {
  std::vector<float> out;
  if (c->kind == PASTA_CONT_CHUNK) {
    const int p1 = c->p1;
    auto T = legendre_to_monomial(p1);
    for (int ch = 0; ch < c->nc; ch++)
      for (int j = 0; j < p1; j++) {
        double s = 0.0;
        for (int k = 0; k < p1; k++) s += p[ch * p1 + k] * T[(size_t)k * p1 + j];
        out.push_back((float)s);
      }
  } else if (c->kind == PASTA_CONT_LINEAR) {
    const int k = c->k;
    std::vector<double> x(k);
    for (int j = k - 1; j >= 0; j--) {
      double s = p[j];
      for (int l = j + 1; l < k; l++) s -= c->R[(size_t)j * k + l] * x[l];
      x[j] = s / c->R[(size_t)j * k + j];
    }
    for (double v : x) out.push_back((float)v);
  } else {
    out.push_back((float)p[0]);
  }
  return out;
}

int cont_nparams(const pasta_continuum *c) {
  if (c->kind == PASTA_CONT_CHUNK) return c->nc * c->p1;
  if (c->kind == PASTA_CONT_LINEAR) return c->k;
  return 1;
}
int device_param_stride(const pasta_continuum *c) {
  if (c->kind == PASTA_CONT_CHUNK) return c->nc * c->p1;
  if (c->kind == PASTA_CONT_LINEAR) return c->k;
  return 1;
}

// Assemble a device star from its dispersion, continuum and observed data.
DevStar make_star(const pasta_dispersion *d, const pasta_continuum *c, const float *dflux, const float *dvar,
                  int64_t n) {
  DevStar s{};
  s.n_obs = (int)n;
  s.disp_kind = d ? d->dev_kind : DISP_NONE;
  s.gw = d ? d->gw : 0;
  s.flux = dflux;
  s.var = dvar;
  if (d) {
    s.fidx = d->dfidx.p;
    s.wl_obs = d->dwl.p;
    s.wl_first = d->wl_first; s.wl_last = d->wl_last;
    s.wl_min = d->wl_min; s.wl_max = d->wl_max;
    s.fidx_min = d->fidx_min; s.fidx_max = d->fidx_max;
    s.obs_sorted = d->sorted;
    s.gk = d->dgk.p;
    s.gspec = d->dgspec.p;
  }
  if (c) {
    s.cont_kind = c->kind;
    s.cont_bad = c->bad;
    s.n_chunks = c->nc;
    s.p1 = c->p1;
    s.k_lin = c->k;
    s.ignore = c->ignore;
    s.cstart = c->dcs.p;
    s.cstop = c->dce.p;
    s.xa = c->dxa.p; s.xb = c->dxb.p; s.fac = c->dfac.p;
    s.chol = c->dchol.p;
    s.q = c->dq.p;
    s.qt = c->dqt.p;
    s.kp = c->dqt.p ? c->kp : 0;
    s.cont = c->dcont.p;
  } else {
    s.cont_kind = CONT_CONSTANT;
  }
  return s;
}

void check_disp_grid(const pasta_grid *g, const pasta_dispersion *d) {
  if (!d) return;
  if (d->synth_n != g->npx)
    fail(PASTA_E_ARG, "Length of model and wavelength grid don't match. model: %lld, synth_wl: %lld",
         (long long)g->npx, (long long)d->synth_n);
}

// ============================================================ pipeline
struct EvalArgs {
  const DevStar *stars = nullptr;
  const double *labels = nullptr;
  const int *eval_star = nullptr;
  const int *eval_active = nullptr;
  int64_t E = 0;
  double *cost = nullptr;
  int *status = nullptr;
  double *params = nullptr;
  int param_stride = 0;
  int need_chi2 = 0;
  int full_window = 0;
  int max_m = 1;
  int max_hg = 0;                // widest instrument half width among the stars
  uint32_t chunk_p1_mask = 0;    // chunk continua present, by coefficient count
  int max_chunks = 0;            // most chunks of those continua
  int other_cont = 0;            // linear / fixed / constant continua present
  int64_t max_nobs = 0;          // longest observed spectrum
  float *out_obs = nullptr;
  int64_t out_stride = 0;
  float *out_synth = nullptr;
  const float *given = nullptr;  // model given at observed pixels
  int64_t given_stride = 0;      // floats between the given rows of consecutive evaluations
  int lin_group = 0;             // consecutive evaluations sharing a star (tensor-core linear continua), or 0
  int star_len = 0;              // consecutive evaluations per star (interpolation segments); 0: one star
  uint32_t lin_kp_mask = 0;      // tensor-core bases present (bit kp / 16)
};

// continuum kinds and instrument widths of the stars a batch can touch
void star_kinds(const std::vector<DevStar> &h, EvalArgs &a) {
  for (const auto &st : h) {
    if (st.cont_kind == CONT_CHUNK) {
      a.chunk_p1_mask |= 1u << st.p1;
      a.max_chunks = std::max(a.max_chunks, st.n_chunks);
    } else {
      a.other_cont = 1;
    }
    a.max_nobs = std::max<int64_t>(a.max_nobs, st.n_obs);
    if (st.disp_kind != DISP_NONE) a.max_hg = std::max(a.max_hg, (st.gw - 1) / 2);
    if (st.cont_kind == CONT_LINEAR && st.kp > 0) a.lin_kp_mask |= 1u << (st.kp / 16);
  }
}

// pixel slices per group of the tensor-core linear continua: enough CTAs
// for two waves of two per SM, at most LIN_MAX_SLICES
void set_lin_slices(pasta_grid *g, EvalBatch &b) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  b.lin_zpart = g->ws.zpart.p;
  if (b.lin_group <= 0) {
    b.lin_slices = 1;
    return;
  }
  const int groups = (b.E + b.lin_group - 1) / b.lin_group;
  b.lin_slices = std::max(1, std::min(LIN_MAX_SLICES, (4 * sms + groups - 1) / groups));
}

// tensor-core linear continua: on unless PASTA_LINEAR_TC=0 or
// pasta_set_linear_tensor_cores(0) selects the CUDA-core path
std::atomic<int> g_linear_tc{-1};
bool linear_tc_enabled() {
  int v = g_linear_tc.load();
  if (v < 0) {
    const char *e = getenv("PASTA_LINEAR_TC");
    v = (e && e[0] == '0') ? 0 : 1;
    int expect = -1;
    g_linear_tc.compare_exchange_strong(expect, v);
    v = g_linear_tc.load();
  }
  return v != 0;
}

// tensor-core interpolation of shared-row groups: on unless
// PASTA_INTERP_TC=0 or pasta_set_interp_tensor_cores(0) selects the CUDA cores
std::atomic<int> g_interp_tc{-1};
bool interp_tc_enabled() {
  int v = g_interp_tc.load();
  if (v < 0) {
    const char *e = getenv("PASTA_INTERP_TC");
    v = (e && e[0] == '0') ? 0 : 1;
    int expect = -1;
    g_interp_tc.compare_exchange_strong(expect, v);
    v = g_interp_tc.load();
  }
  return v != 0;
}

// evaluations alone in their segment merged across segments: on unless
// PASTA_INTERP_MERGE=0
bool interp_merge_enabled() {
  const char *e = getenv("PASTA_INTERP_MERGE");
  return !(e && e[0] == '0');
}

int width_upper_bound(const pasta_grid *g, double vsini_hi) {
  if (g->d.dvelo <= 0.0 || !(vsini_hi > 0.0)) return 1;
  int w = rotation_width(vsini_hi, g->d.dvelo);
  return std::min(w, FFTN);
}

// The batch of evaluations [off, off + cnt) of a in the grid's workspace.
EvalBatch make_batch(pasta_grid *g, const EvalArgs &a, int64_t off, int64_t cnt) {
  if (a.max_nobs > g->ws.stride) fail(PASTA_E_INTERNAL, "workspace rows are shorter than the observed spectrum");
  EvalBatch b{};
  b.E = (int)cnt;
  b.labels = a.labels ? a.labels + 5 * off : nullptr;
  b.eval_star = a.eval_star + off;
  b.eval_active = a.eval_active ? a.eval_active + off : nullptr;
  b.stars = a.stars;
  b.prep = g->ws.prep.p;
  b.H = g->ws.H.p;
  b.HG = g->ws.HG.p;
  b.bufA = g->ws.A.p;
  b.bufB = g->ws.B.p;
  b.stride = g->ws.stride;
  b.cost = a.cost ? a.cost + off : nullptr;
  b.status = a.status ? a.status + off : nullptr;
  b.params = a.params ? a.params + (size_t)off * a.param_stride : nullptr;
  b.param_stride = a.param_stride;
  b.need_chi2 = a.need_chi2;
  b.chunk_p1_mask = a.chunk_p1_mask;
  b.max_chunks = a.max_chunks;
  b.other_cont = a.other_cont;
  // chi2 batches resample inside the broadening kernel unless a synth row is wanted
  b.obs_epi = a.need_chi2 && !a.out_obs && !a.out_synth && !a.full_window ? 1 : 0;
  b.bnd = g->ws.bnd.p;
  b.grec = g->ws.grec.p;
  b.gcount = g->ws.gcount.p;
  // segments start at star boundaries; a sub-batch that starts inside a star
  // is cut in plain chunks of SEG
  b.seg_len = a.star_len > 0 && off % a.star_len == 0 ? a.star_len : 0;
  const bool tc = interp_tc_enabled() && g->has_tmap;
  b.tcrec = tc ? g->ws.tcrec.p : nullptr;
  b.tccount = g->ws.tccount.p;
  b.tclist = g->ws.tclist.p;
  b.tclist_count = g->ws.tclist_count.p;
  b.tmap = tc ? &g->tmap : nullptr;
  b.tc_min = g->tc_min;
  if (interp_merge_enabled()) {
    b.mkey = g->ws.mkey.p;
    b.mcnt = g->ws.mcnt.p;
    b.mmem = g->ws.mmem.p;
    b.mslot = g->ws.mslot.p;
    b.mtab = g->ws.mtab;
    b.erec = g->ws.erec.p;
    b.mrec = g->ws.mrec.p;
    b.mrcount = g->ws.mrcount.p;
  }
  b.bnd_stride = g->ws.bnd_stride;
  b.cpart = g->ws.cpart.p;
  b.given = a.given ? a.given + (size_t)off * a.given_stride : nullptr;
  b.given_stride = a.given_stride;
  b.direct_max = g->direct_max;
  b.max_dtiles = (int)((g->npx + DIRECT_TILE - DIRECT_MAX_TAPS - 1) / (DIRECT_TILE - DIRECT_MAX_TAPS));
  b.direct_list = g->ws.dlist.p;
  b.direct_count = g->ws.dcount.p;
  // groups must start at star boundaries: sub-batches that begin inside a
  // group take the CUDA-core path
  const bool lin = linear_tc_enabled() && a.lin_group > 0 && a.lin_group <= 128 && off % a.lin_group == 0;
  b.lin_group = lin ? a.lin_group : 0;
  b.lin_kp_mask = lin ? a.lin_kp_mask : 0u;
  set_lin_slices(g, b);
  return b;
}

// Launch the evaluation pipeline for a.E evaluations, in workspace-sized
// sub-batches.  Capturable in a CUDA graph (no allocation, no sync).
void run_evals(pasta_grid *g, const EvalArgs &a, cudaStream_t s) {
  Ctx &C = ctx();
  const int64_t cap = g->ws.cap;
  int max_pairs, max_pairs_unfused, may_unfuse;
  pipeline_pairs((int)g->npx, a.max_m, a.max_hg, &max_pairs, &max_pairs_unfused, &may_unfuse);
  PipelineOpts o;
  o.full_window = a.full_window;
  o.rot = a.max_m > 1;
  o.may_unfuse = may_unfuse;
  for (int64_t off = 0; off < a.E; off += cap) {
    const int64_t cnt = std::min(cap, a.E - off);
    EvalBatch b = make_batch(g, a, off, cnt);
    b.max_pairs = max_pairs;
    b.max_pairs_unfused = max_pairs_unfused;
    if (a.given) {
      launch_chi2(g->d, b, s);
      continue;
    }
    launch_pipeline(g->d, b, C.tw.p, o, s);
    if (a.out_obs) launch_resample_out(g->d, b, a.out_obs + (size_t)off * a.out_stride, a.out_stride, s);
    if (a.out_synth) launch_copy_broadened(g->d, b, a.out_synth + (size_t)off * g->npx, s);
  }
  CK(cudaGetLastError());
}

// Workspace for E evaluations (or as many as fit) whose rows hold both a
// synth spectrum and an observed spectrum of max_nobs pixels.
void ensure_workspace(pasta_grid *g, int64_t E, int64_t max_nobs) {
  const int64_t need = std::max<int64_t>(g->stride, (max_nobs + 63) / 64 * 64);
  const int64_t stride = std::max(need, g->ws.stride);  // rows never shrink
  const int bstr = bnd_stride_for((int)g->npx);
  // enough already (no device-memory query on this path: it runs every step)
  if (g->ws.cap >= std::max<int64_t>(E, 1) && g->ws.stride == stride && g->ws.bnd_stride == bstr) return;
  const int64_t want = workspace_cap(g, E, stride);
  if (g->ws.cap >= want && g->ws.stride == stride && g->ws.bnd_stride == bstr) return;
  g->ws.ensure(want, stride, bstr);
}

// ================================================================= swarm
PsoParams make_pso_params(const pasta_grid *g, const pasta_pso_settings &st) {
  if (st.num_particles < 1 || st.num_particles > MAX_PARTICLES)
    fail(PASTA_E_ARG, "num_particles must be in 1..%d", MAX_PARTICLES);
  if (st.max_iters < 0) fail(PASTA_E_ARG, "max_iters must be >= 0");
  if (st.social_factor < 0.0) fail(PASTA_E_ARG, "`ParticleSwarm`: social factor must be >=0.");
  if (st.delta < 0.0) fail(PASTA_E_ARG, "`ParticleSwarm`: delta must be >=0.");
  PsoParams P{};
  P.P = st.num_particles;
  P.max_iters = st.max_iters;
  P.inertia = st.inertia_factor;
  P.cognitive = st.cognitive_factor;
  P.social = st.social_factor;
  P.vs_lo = st.vsini_lo; P.vs_hi = st.vsini_hi;
  P.rv_lo = st.rv_lo; P.rv_hi = st.rv_hi;
  double mn[5] = {g->tv.front(), g->mv.front(), g->lv.front(), st.vsini_lo, st.rv_lo};
  double mx[5] = {g->tv.back(), g->mv.back(), g->lv.back(), st.vsini_hi, st.rv_hi};
  for (int i = 0; i < 5; i++) {
    P.ckind[i] = st.ckind[i];
    P.ca[i] = st.ca[i];
    P.cb[i] = st.cb[i];
    if (st.ckind[i] == 1) { mn[i] = st.ca[i]; mx[i] = st.ca[i]; }
    else if (st.ckind[i] == 2) { mn[i] = std::max(mn[i], st.ca[i]); mx[i] = std::min(mx[i], st.cb[i]); }
    P.mn[i] = mn[i];
    P.mx[i] = mx[i];
  }
  return P;
}

// bounds.rs:21-35 + particleswarm.rs:137-150 on the shared draw stream.
int init_swarm_host(const pasta_grid *g, const PsoParams &S, uint64_t seed, double *x, double *v) {
  uint64_t cand = 0;
  for (int p = 0; p < S.P;) {
    if (cand > 20000000ull) return S_BOUNDS;
    double t[5];
    for (int d = 0; d < 5; d++)
      t[d] = S.mn[d] == S.mx[d] ? S.mn[d] : uniform_between(S.mn[d], S.mx[d], draw_u01(seed, PH_INIT_POS, cand, 0, d));
    cand++;
    if (pso_within(g->hg, S, t)) {
      for (int d = 0; d < 5; d++) x[p * 5 + d] = t[d];
      p++;
    }
  }
  for (int p = 0; p < S.P; p++)
    for (int d = 0; d < 5; d++) {
      const double w = S.mx[d] - S.mn[d];
      v[p * 5 + d] = (-w == w) ? -w : uniform_between(-w, w, draw_u01(seed, PH_INIT_VEL, p, 0, d));
    }
  return S_OK;
}

struct StarInput {
  const pasta_dispersion *d;
  const pasta_continuum *c;
  const pasta_pso_settings *st;
  const float *flux, *var;
  int64_t n;
  uint64_t seed;
};

// Upload the observed data of S stars (concatenated) and build DevStars.
struct StarSet {
  DBuf<float> flux, var;
  DBuf<DevStar> dstars;
  std::vector<DevStar> h;
  void build(const std::vector<StarInput> &in) {
    int64_t tot = 0;
    for (auto &s : in) tot += s.n;
    std::vector<float> f(tot), v(tot);
    std::vector<int64_t> off(in.size());
    int64_t o = 0;
    for (size_t i = 0; i < in.size(); i++) {
      off[i] = o;
      std::memcpy(&f[o], in[i].flux, in[i].n * sizeof(float));
      std::memcpy(&v[o], in[i].var, in[i].n * sizeof(float));
      o += in[i].n;
    }
    flux.upload(f);
    var.upload(v);
    h.resize(in.size());
    for (size_t i = 0; i < in.size(); i++) h[i] = make_star(in[i].d, in[i].c, flux.p + off[i], var.p + off[i], in[i].n);
    dstars.upload(h);
  }
};

void validate_star(const pasta_grid *g, const StarInput &s) {
  check_disp_grid(g, s.d);
  if (s.n != (int64_t)s.d->wl.size()) fail(PASTA_E_ARG, "Observed spectrum and target dispersion must have the same length");
  if (s.c && s.c->kind != PASTA_CONT_CONSTANT && s.c->n != s.n)
    fail(PASTA_E_ARG, "Length of observed and continuum spectrum are different %lld, %lld", (long long)s.n, (long long)s.c->n);
}

struct SwarmBuffers {
  int S = 0, Pmax = 0;
  DBuf<double> x, v, bx, cost, bcost, gx, gcost, labels, ecost;
  DBuf<int> iter, status, done, active, eval_active, eval_star, estatus;
  DBuf<uint64_t> seed;
  DBuf<PsoParams> params;
  Swarm view() {
    Swarm w;
    w.S = S; w.Pmax = Pmax;
    w.x = x.p; w.v = v.p; w.bx = bx.p; w.cost = cost.p; w.bcost = bcost.p;
    w.gx = gx.p; w.gcost = gcost.p; w.iter = iter.p; w.status = status.p; w.done = done.p;
    w.active = active.p; w.seed = seed.p; w.params = params.p; w.labels = labels.p;
    w.eval_active = eval_active.p;
    w.refit = nullptr;
    return w;
  }
  void alloc(int S_, int Pmax_) {
    S = S_; Pmax = Pmax_;
    const size_t E = (size_t)S * Pmax;
    x.alloc(E * 5); v.alloc(E * 5); bx.alloc(E * 5); cost.alloc(E); bcost.alloc(E);
    gx.alloc((size_t)S * 5); gcost.alloc(S); labels.alloc(E * 5); ecost.alloc(E);
    iter.alloc(S); status.alloc(S); done.alloc(S); active.alloc(S);
    eval_active.alloc(E); eval_star.alloc(E); estatus.alloc(E);
    seed.alloc(S); params.alloc(S);
    std::vector<int> es(E);
    for (size_t e = 0; e < E; e++) es[e] = (int)(e / Pmax);
    CK(cudaMemcpy(eval_star.p, es.data(), E * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemset(eval_active.p, 0, E * sizeof(int)));
    CK(cudaMemset(x.p, 0, E * 5 * sizeof(double)));
    CK(cudaMemset(v.p, 0, E * 5 * sizeof(double)));
    CK(cudaMemset(labels.p, 0, E * 5 * sizeof(double)));
  }
};

// Final refit at the best labels (fitting.rs:436-440) -> continuum params.
// Device buffers of a final refit, kept by callers that refit often (the
// server retires a few stars every step) so that no step allocates.
struct RefitScratch {
  DBuf<double> lab, cost, par;
  DBuf<int> es, ea, st;
  void ensure(int S, int pstride) {
    if (cost.n < (size_t)S) {
      lab.alloc((size_t)S * 5);
      cost.alloc(S);
      es.alloc(S);
      ea.alloc(S);
      st.alloc(S);
    }
    if (par.n < (size_t)S * pstride) par.alloc((size_t)S * pstride);
  }
};

void final_refit(pasta_grid *g, StarSet &ss, const std::vector<StarInput> &in, const std::vector<double> &best,
                 const std::vector<int> &ok, std::vector<std::vector<float>> &params, cudaStream_t s,
                 RefitScratch *scratch = nullptr, const DevStar *dstars = nullptr) {
  const int S = (int)in.size();
  int pstride = 1, max_m = 1;
  for (auto &x : in) {
    pstride = std::max(pstride, device_param_stride(x.c));
    double vhi = x.st->vsini_hi;
    if (x.st->ckind[3] == 1) vhi = x.st->ca[3];
    max_m = std::max(max_m, width_upper_bound(g, vhi));
  }
  RefitScratch local;
  RefitScratch &R = scratch ? *scratch : local;
  R.ensure(S, pstride);
  std::vector<int> star(S);
  for (int i = 0; i < S; i++) star[i] = i;
  CK(cudaMemcpyAsync(R.lab.p, best.data(), (size_t)S * 5 * sizeof(double), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(R.es.p, star.data(), (size_t)S * sizeof(int), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(R.ea.p, ok.data(), (size_t)S * sizeof(int), cudaMemcpyHostToDevice, s));
  DBuf<double> &lab = R.lab, &cost = R.cost, &par = R.par;
  DBuf<int> &es = R.es, &ea = R.ea, &st = R.st;
  EvalArgs a;
  a.stars = dstars ? dstars : ss.dstars.p;
  a.labels = lab.p;
  a.eval_star = es.p;
  a.eval_active = ea.p;
  a.E = S;
  a.cost = cost.p;
  a.status = st.p;
  a.params = par.p;
  a.param_stride = pstride;
  a.need_chi2 = 1;
  a.max_m = max_m;
  star_kinds(ss.h, a);
  a.lin_group = 1;  // one evaluation per star
  a.star_len = 1;
  ensure_workspace(g, S, a.max_nobs);
  run_evals(g, a, s);
  std::vector<double> hp((size_t)S * pstride);
  CK(cudaMemcpyAsync(hp.data(), par.p, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  params.assign(S, {});
  for (int i = 0; i < S; i++)
    if (ok[i]) params[i] = params_from_device(in[i].c, &hp[(size_t)i * pstride]);
}

// Batched form: all stars' swarms on the device, one CUDA graph per PSO
// step (position update -> evaluation pipeline -> best update).
struct Batch {
  pasta_grid *g = nullptr;
  std::vector<StarInput> in;
  std::vector<pasta_pso_settings> settings;
  std::vector<PsoParams> pp;
  StarSet ss;
  SwarmBuffers W;
  EvalArgs a;
  Swarm sw{};
  int S = 0, Pmax = 0, iters = 0, max_m = 1, steps_done = 0;
  int kernels_per_step = 0;
  double t0 = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev[12] = {};
  ~Batch() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto &e : ev)
      if (e) cudaEventDestroy(e);
  }
  void step_eager(cudaStream_t s) {
    launch_pso_update(g->d, sw, s);
    run_evals(g, a, s);
    launch_pso_best(sw, W.ecost.p, W.estatus.p, s);
  }
};

void batch_init(Batch &B, pasta_grid *g, const std::vector<StarInput> &in) {
  Ctx &C = ctx();
  cudaStream_t s = C.stream;
  B.t0 = now_s();
  B.g = g;
  B.in = in;
  B.S = (int)in.size();
  B.settings.resize(B.S);
  for (int i = 0; i < B.S; i++) {
    B.settings[i] = *in[i].st;
    B.in[i].st = &B.settings[i];
  }
  B.pp.resize(B.S);
  for (int i = 0; i < B.S; i++) {
    B.pp[i] = make_pso_params(g, B.settings[i]);
    B.Pmax = std::max(B.Pmax, B.pp[i].P);
    B.iters = std::max(B.iters, B.pp[i].max_iters);
    B.max_m = std::max(B.max_m, width_upper_bound(g, B.pp[i].mx[3]));
  }
  const int S = B.S, Pmax = B.Pmax;
  B.ss.build(in);
  SwarmBuffers &W = B.W;
  W.alloc(S, Pmax);
  const size_t E = (size_t)S * Pmax;
  std::vector<double> hx(E * 5, 0.0), hv(E * 5, 0.0);
  std::vector<int> status(S, 0), done(S, 0), active(S, 1), iter(S, -1);
  std::vector<uint64_t> seeds(S);
  for (int i = 0; i < S; i++) {
    seeds[i] = in[i].seed;
    int st = init_swarm_host(g, B.pp[i], in[i].seed, &hx[(size_t)i * Pmax * 5], &hv[(size_t)i * Pmax * 5]);
    if (st) { status[i] = st; done[i] = 1; }
  }
  CK(cudaMemcpy(W.x.p, hx.data(), E * 5 * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(W.v.p, hv.data(), E * 5 * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(W.status.p, status.data(), S * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(W.done.p, done.data(), S * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(W.active.p, active.data(), S * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(W.iter.p, iter.data(), S * sizeof(int), cudaMemcpyHostToDevice));
  W.seed.upload(seeds);
  W.params.upload(B.pp);
  B.sw = W.view();
  EvalArgs &a = B.a;
  a.stars = B.ss.dstars.p;
  a.labels = W.labels.p;
  a.eval_star = W.eval_star.p;
  a.eval_active = W.eval_active.p;
  a.E = (int64_t)E;
  a.cost = W.ecost.p;
  a.status = W.estatus.p;
  a.need_chi2 = 1;
  a.max_m = B.max_m;
  star_kinds(B.ss.h, a);
  a.lin_group = B.Pmax <= 128 ? B.Pmax : 0;  // star s owns evaluations [s Pmax, (s + 1) Pmax)
  a.star_len = B.Pmax;
  ensure_workspace(g, (int64_t)E, a.max_nobs);
  for (auto &e : B.ev) CK(cudaEventCreate(&e));
  if (!getenv("PASTA_NO_GRAPH")) {
    const int64_t k0 = kernel_launches();
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    B.step_eager(s);
    CK(cudaStreamEndCapture(s, &B.graph));
    CK(cudaGraphInstantiate(&B.exec, B.graph, 0));
    B.kernels_per_step = (int)(kernel_launches() - k0);
  }
}

// Launch n PSO steps; returns the device time between CUDA events recorded
// on the launching stream around them.
double batch_steps(Batch &B, int n, double *trace) {
  Ctx &C = ctx();
  cudaStream_t s = C.stream;
  std::vector<double> tx, tc;
  const int Ptr = B.pp.empty() ? 0 : B.pp[0].P;
  CK(cudaEventRecord(B.ev[0], s));
  for (int k = 0; k < n; k++) {
    if (B.exec) CK(cudaGraphLaunch(B.exec, s));
    else B.step_eager(s);
    const int it = B.steps_done++;
    if (trace && it <= B.pp[0].max_iters) {
      tx.resize((size_t)B.Pmax * 5);
      tc.resize(B.Pmax);
      CK(cudaMemcpyAsync(tx.data(), B.W.x.p, tx.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(tc.data(), B.W.cost.p, tc.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      for (int p = 0; p < Ptr; p++) {
        double *t = trace + ((size_t)it * Ptr + p) * 6;
        for (int d = 0; d < 5; d++) t[d] = tx[(size_t)p * 5 + d];
        t[5] = tc[p];
      }
    }
  }
  CK(cudaEventRecord(B.ev[1], s));
  CK(cudaEventSynchronize(B.ev[1]));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, B.ev[0], B.ev[1]));
  return ms;
}

// One step launched stage by stage with events between the stages:
// out[0] swarm update, [1] prep, [2] rotation spectra, [3] interpolation,
// [4] fused broadening (block bounds + k_broaden), [5] unfused rotation and
// instrument profile, [6] resampling left over + chi2, [7] best update,
// [8] interpolated pixels (sum of windows), [9] evaluations, [10] sum of
// observed pixels, [11] broadening blocks.
void batch_profile_step(Batch &B, double *out) {
  Ctx &C = ctx();
  cudaStream_t s = C.stream;
  pasta_grid *g = B.g;
  const EvalArgs &a = B.a;
  if (a.E > g->ws.cap) fail(PASTA_E_UNSUPPORTED, "profiled step needs the batch in one workspace");
  EvalBatch b = make_batch(g, a, 0, a.E);
  int may_unfuse;
  pipeline_pairs((int)g->npx, a.max_m, a.max_hg, &b.max_pairs, &b.max_pairs_unfused, &may_unfuse);
  CK(cudaEventRecord(B.ev[0], s));
  launch_pso_update(g->d, B.sw, s);
  CK(cudaEventRecord(B.ev[1], s));
  launch_prep(g->d, b, s);
  CK(cudaEventRecord(B.ev[2], s));
  if (a.max_m > 1) launch_rotker(g->d, b, C.tw.p, s);
  CK(cudaEventRecord(B.ev[3], s));
  launch_group(g->d, b, s);
  launch_interp_tc(g->d, b, s);
  launch_interp(g->d, b, s);
  CK(cudaEventRecord(B.ev[4], s));
  launch_obs_bounds(g->d, b, s);
  launch_broaden(g->d, b, C.tw.p, s);
  CK(cudaEventRecord(B.ev[5], s));
  launch_direct(g->d, b, s);
  if (may_unfuse) {
    launch_rot(g->d, b, C.tw.p, s);
    launch_gauss(g->d, b, s);
  }
  CK(cudaEventRecord(B.ev[6], s));
  launch_resample_obs(g->d, b, s);
  launch_chi2(g->d, b, s);
  CK(cudaEventRecord(B.ev[7], s));
  launch_pso_best(B.sw, B.W.ecost.p, B.W.estatus.p, s);
  CK(cudaEventRecord(B.ev[8], s));
  CK(cudaGetLastError());
  CK(cudaEventSynchronize(B.ev[8]));
  for (int i = 0; i < 8; i++) {
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, B.ev[i], B.ev[i + 1]));
    out[i] = ms;
  }
  B.steps_done++;
  std::vector<EvalPrep> hp(a.E);
  CK(cudaMemcpy(hp.data(), g->ws.prep.p, a.E * sizeof(EvalPrep), cudaMemcpyDeviceToHost));
  double px = 0, ev = 0, obs = 0, blk = 0;
  std::vector<DevStar> hs = B.ss.h;
  for (const auto &P : hp) {
    if (P.status) continue;
    px += P.i_hi - P.i_lo;
    ev += 1;
    obs += hs[P.star].n_obs;
    blk += P.nblk;
  }
  out[8] = px;
  out[9] = ev;
  out[10] = obs;
  out[11] = blk;
}

void batch_finish(Batch &B, pasta_fit_result *res, std::vector<std::vector<float>> &params) {
  Ctx &C = ctx();
  cudaStream_t s = C.stream;
  const int S = B.S;
  std::vector<double> gx((size_t)S * 5), gc(S);
  std::vector<int> status(S);
  CK(cudaMemcpyAsync(gx.data(), B.W.gx.p, gx.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(gc.data(), B.W.gcost.p, gc.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(status.data(), B.W.status.p, S * sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  std::vector<int> ok(S);
  for (int i = 0; i < S; i++) ok[i] = status[i] == 0 ? 1 : 0;
  final_refit(B.g, B.ss, B.in, gx, ok, params, s);
  const double dt = now_s() - B.t0;
  for (int i = 0; i < S; i++) {
    pasta_fit_result &r = res[i];
    std::memset(&r, 0, sizeof r);
    for (int d = 0; d < 5; d++) r.label[d] = gx[(size_t)i * 5 + d];
    r.chi2 = gc[i];
    r.iterations = B.pp[i].max_iters;
    r.status = status[i];
    r.time = dt;
    r.n_params = (int)params[i].size();
  }
}

void fit_batched(pasta_grid *g, const std::vector<StarInput> &in, pasta_fit_result *res,
                 std::vector<std::vector<float>> &params, double *trace) {
  Batch B;
  batch_init(B, g, in);
  batch_steps(B, B.iters + 1, trace);
  batch_finish(B, res, params);
}

// Plain form: one star at a time, the swarm on the host, one launch per
// stage per iteration with a device->host round trip of the costs.
void fit_plain(pasta_grid *g, const std::vector<StarInput> &in, pasta_fit_result *res,
               std::vector<std::vector<float>> &params, double *trace) {
  Ctx &C = ctx();
  cudaStream_t s = C.stream;
  const int S = (int)in.size();
  params.assign(S, {});
  for (int si = 0; si < S; si++) {
    const double t0 = now_s();
    const StarInput &X = in[si];
    PsoParams pp = make_pso_params(g, *X.st);
    const int P = pp.P;
    StarSet ss;
    ss.build({X});
    std::vector<double> x((size_t)P * 5), v((size_t)P * 5), bx, cost(P), bcost(P), gxv(5);
    double gcost = 0;
    int status = init_swarm_host(g, pp, X.seed, x.data(), v.data());
    DBuf<double> dl, dc;
    DBuf<int> de, ds;
    dl.alloc((size_t)P * 5);
    dc.alloc(P);
    ds.alloc(P);
    de.upload(std::vector<int>(P, 0));
    EvalArgs a;
    a.stars = ss.dstars.p;
    a.labels = dl.p;
    a.eval_star = de.p;
    a.E = P;
    a.cost = dc.p;
    a.status = ds.p;
    a.need_chi2 = 1;
    a.max_m = width_upper_bound(g, pp.mx[3]);
    star_kinds(ss.h, a);
    a.lin_group = 128;  // the particles of the one star
    ensure_workspace(g, P, a.max_nobs);
    std::vector<int> est(P);
    auto evaluate = [&]() -> int {
      CK(cudaMemcpyAsync(dl.p, x.data(), x.size() * sizeof(double), cudaMemcpyHostToDevice, s));
      run_evals(g, a, s);
      CK(cudaMemcpyAsync(cost.data(), dc.p, P * sizeof(double), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(est.data(), ds.p, P * sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      for (int p = 0; p < P; p++)
        if (est[p]) return est[p];
      return 0;
    };
    auto dump = [&](int it) {
      if (!trace || si != 0) return;
      for (int p = 0; p < P; p++) {
        double *t = trace + ((size_t)it * P + p) * 6;
        for (int d = 0; d < 5; d++) t[d] = x[(size_t)p * 5 + d];
        t[5] = cost[p];
      }
    };
    if (!status) status = evaluate();
    if (!status) {  // sort by cost (stable), NaN last
      std::vector<int> idx(P);
      for (int p = 0; p < P; p++) idx[p] = p;
      auto key = [&](int p) { return cost[p] != cost[p] ? INFINITY : cost[p]; };
      std::stable_sort(idx.begin(), idx.end(), [&](int a_, int b_) { return key(a_) < key(b_); });
      std::vector<double> x2(x.size()), v2(v.size()), c2(P);
      for (int r = 0; r < P; r++) {
        for (int d = 0; d < 5; d++) { x2[(size_t)r * 5 + d] = x[(size_t)idx[r] * 5 + d]; v2[(size_t)r * 5 + d] = v[(size_t)idx[r] * 5 + d]; }
        c2[r] = cost[idx[r]];
      }
      x = x2; v = v2; cost = c2;
      bx = x; bcost = cost;
      for (int d = 0; d < 5; d++) gxv[d] = x[d];
      gcost = cost[0];
      dump(0);
    }
    for (int it = 0; it < pp.max_iters && !status; it++) {
      for (int p = 0; p < P && !status; p++) {
        for (int d = 0; d < 5; d++) {
          const double momentum = v[p * 5 + d] * pp.inertia;
          const double to_opt = bx[p * 5 + d] - x[p * 5 + d];
          const double pull = (to_opt == 0.0 ? 0.0 : uniform_between(0.0, to_opt, draw_u01(X.seed, PH_ITER, it, p, 2 * d))) * pp.cognitive;
          const double to_g = gxv[d] - x[p * 5 + d];
          const double pullg = (to_g == 0.0 ? 0.0 : uniform_between(0.0, to_g, draw_u01(X.seed, PH_ITER, it, p, 2 * d + 1))) * pp.social;
          v[p * 5 + d] = momentum + pull + pullg;
          double nx[5];
          for (int k = 0; k < 5; k++) nx[k] = x[p * 5 + k];
          nx[d] += v[p * 5 + d];
          double c;
          int st = pso_clamp_1d(g->hg, pp, nx, d, c);
          if (st) { status = st; break; }
          x[p * 5 + d] = c;
          if (!pso_within(g->hg, pp, &x[p * 5])) { status = S_BOUNDS; break; }
        }
      }
      if (status) break;
      status = evaluate();
      if (status) break;
      for (int p = 0; p < P; p++) {
        if (cost[p] < bcost[p]) {
          for (int d = 0; d < 5; d++) bx[p * 5 + d] = x[p * 5 + d];
          bcost[p] = cost[p];
          if (cost[p] < gcost) {
            for (int d = 0; d < 5; d++) gxv[d] = x[p * 5 + d];
            gcost = cost[p];
          }
        }
      }
      dump(it + 1);
    }
    std::vector<std::vector<float>> pr;
    final_refit(g, ss, {X}, gxv, {status == 0 ? 1 : 0}, pr, s);
    params[si] = pr[0];
    pasta_fit_result &r = res[si];
    std::memset(&r, 0, sizeof r);
    for (int d = 0; d < 5; d++) r.label[d] = gxv[d];
    r.chi2 = gcost;
    r.iterations = pp.max_iters;
    r.status = status;
    r.time = now_s() - t0;
    r.n_params = (int)params[si].size();
  }
}

}  // namespace

// ================================================================ serving
// continuum parameters per slot of the in-graph refit: the most any
// continuum fitter has (chunks x coefficients, or linear-model columns)
constexpr int SERVER_REFIT_STRIDE = MAX_CHUNKS * MAX_P1 > MAX_LIN_K ? MAX_CHUNKS * MAX_P1 : MAX_LIN_K;

struct pasta_server {
  pasta_grid *g = nullptr;
  int slots = 0, Pmax = 0;
  int64_t budget = 0, used = 0;
  struct Req {
    int64_t id;
    const pasta_dispersion *d;
    const pasta_continuum *c;
    pasta_pso_settings st;
    std::vector<float> flux, var;
    double t_submit;
    uint64_t seed;
    int64_t bytes;
  };
  std::deque<Req> queue;
  std::vector<std::unique_ptr<Req>> slot_req;
  std::vector<std::unique_ptr<DBuf<float>>> slot_flux, slot_var;
  std::vector<DevStar> hstars;
  DBuf<DevStar> dstars;
  SwarmBuffers W;
  std::vector<PsoParams> pp;
  struct Done {
    int64_t id;
    pasta_fit_result r;
    std::vector<float> params;
  };
  std::deque<Done> done;
  int64_t next_id = 1;
  int64_t evals_total = 0, steps_total = 0;  // evaluations and steps run so far
  int64_t graph_kernels = 0;                  // kernels in the captured step
  double t_before = 0, t_step = 0, t_after = 0;  // host seconds: admission, graph run, retirement
  double t_refit = 0;                              // of which reading the refits back
  // in-graph final refit: per slot the finished flag, identity star index,
  // chi2, status and continuum parameters
  DBuf<int> rf_flag, rf_star, rf_status;
  DBuf<double> rf_cost, rf_params;
  int max_m = 1, graph_max_m = 0;
  int64_t graph_gen = -1;
  uint32_t graph_mask = 0;  // continuum kinds / instrument width the captured step covers
  int graph_other = 0, graph_hg = 0, graph_chunks = 0;
  uint32_t graph_lin = 0;   // tensor-core linear bases the captured step covers
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  std::mutex mu;
  ~pasta_server() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
  }
};

// ================================================================= C ABI
extern "C" {

int pasta_abi_version(void) { return PASTA_B200_ABI_VERSION; }
int pasta_set_interp_tensor_cores(int on) {
  g_interp_tc.store(on ? 1 : 0);
  return PASTA_OK;
}

int pasta_set_linear_tensor_cores(int on) {
  g_linear_tc.store(on ? 1 : 0);
  return PASTA_OK;
}
const char *pasta_last_error(void) { return g_last_error.c_str(); }
int64_t pasta_kernel_launch_count(void) { return kernel_launches(); }

int pasta_set_device(int device) {
  return guard([&] {
    CK(cudaSetDevice(device));
    g_dev = device;
    ctx();
  });
}

// interpolate.rs:267-331 (Grid::new) + model_fetchers.rs:136-166 (column order)
namespace {

// Autotuner of the broadening path: the crossover between the direct and the
// FFT broadening on this device.  For rotation widths on a ladder, the
// pipeline runs 256 or more evaluations of one grid label over the whole
// synthetic grid with either path, timed with CUDA events (best of 3 after a warm-up);
// direct_max is the widest kernel up to which the direct path won at every
// rung.  PASTA_DIRECT_MAX_TAPS fixes the value instead (0: FFT only);
// PASTA_TUNE_VERBOSE prints the measured ladder.
void tune_direct(pasta_grid *g) {
  g->direct_max = 0;
  if (const char *ev = getenv("PASTA_DIRECT_MAX_TAPS")) {
    g->direct_max = std::max(0, std::min(DIRECT_MAX_TAPS, atoi(ev)));
    return;
  }
  if (g->wl_kind == WL_NONUNI || !(g->d.dvelo > 0.0)) return;
  Ctx &C = ctx();
  cudaStream_t s = C.stream;
  // at least ~15M window pixels per run (256 evaluations at 80,000 px, 768
  // at 20,000), so that small grids are timed on throughput rather than on
  // launch latency, where both paths tie and the comparison is noise
  const int E = std::max(256, std::min(2048, (int)(20000000LL / std::max<int64_t>(g->npx, 1)) / 256 * 256));
  const int ti = (int)g->tv.size() / 2;
  const double t = g->tv[ti], mh = g->mv[g->mv.size() / 2], lg = g->lv[(g->llo[ti] + g->lhi[ti]) / 2];
  DevStar st = make_star(nullptr, nullptr, nullptr, nullptr, 0);
  st.disp_kind = DISP_NONE;
  DBuf<DevStar> ds;
  ds.upload(&st, 1);
  DBuf<double> dl;
  dl.alloc((size_t)E * 5);
  DBuf<int> de;
  de.upload(std::vector<int>(E, 0));
  ensure_workspace(g, E, 0);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int ladder[] = {17, 33, 65, 97, 129, 193, 257, 385, 511};
  int best = 0;
  std::vector<double> lab((size_t)E * 5);
  for (int w : ladder) {
    double lo = 0.0, hi = 1e5;  // the largest vsini whose kernel has at most w taps
    for (int it = 0; it < 80; it++) {
      const double mid = 0.5 * (lo + hi);
      if (rotation_width(mid, g->d.dvelo) <= w) lo = mid;
      else hi = mid;
    }
    const int mw = rotation_width(lo, g->d.dvelo);
    if (mw < 3 || mw > w) continue;
    for (int i = 0; i < E; i++) {
      double *q = &lab[(size_t)i * 5];
      q[0] = t; q[1] = mh; q[2] = lg; q[3] = lo; q[4] = 0.0;
    }
    CK(cudaMemcpy(dl.p, lab.data(), lab.size() * sizeof(double), cudaMemcpyHostToDevice));
    EvalArgs a;
    a.stars = ds.p;
    a.labels = dl.p;
    a.eval_star = de.p;
    a.E = E;
    a.full_window = 1;
    a.max_m = mw;
    star_kinds({st}, a);
    float tm[2];
    for (int mode = 0; mode < 2; mode++) {
      g->direct_max = mode ? DIRECT_MAX_TAPS : 0;
      run_evals(g, a, s);
      float bt = 1e30f;
      for (int rep = 0; rep < 3; rep++) {
        CK(cudaEventRecord(e0, s));
        run_evals(g, a, s);
        CK(cudaEventRecord(e1, s));
        CK(cudaEventSynchronize(e1));
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        bt = std::min(bt, ms);
      }
      tm[mode] = bt;
    }
    if (getenv("PASTA_TUNE_VERBOSE"))
      fprintf(stderr, "pasta_b200 tune: %lld px, rotation %d taps: FFT %.4f ms, direct %.4f ms (%d evaluations)\n",
              (long long)g->npx, mw, tm[0], tm[1], E);
    if (tm[1] < tm[0]) best = mw;
    else break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  g->direct_max = best;
}

// The group size from which the tensor-core interpolation beats the CUDA
// cores on this device and grid: 16 segments of 64 evaluations, each split
// into groups of gs evaluations in distinct grid cubes, interpolated with
// the tensor-core path on and off (CUDA events, best of 3 after a warm-up),
// for gs on a ladder; the smallest gs at which the tensor cores win, and
// every larger gs on the ladder, sets the threshold (SEG + 1: never).
void tune_interp_tc(pasta_grid *g) {
  g->tc_min = 16;
  if (const char *ev = getenv("PASTA_INTERP_TC_MIN")) {
    g->tc_min = std::max(TC_MIN_MEMBERS, std::min(SEG + 1, atoi(ev)));
    return;
  }
  if (!g->has_tmap) return;
  // label centres of distinct cubes (neighbour columns) around the grid's middle
  std::vector<std::array<double, 3>> cubes;
  std::vector<std::vector<int>> seen;
  const int nt = (int)g->tv.size(), nm = (int)g->mv.size();
  for (int i = 0; i + 1 < nt && cubes.size() < 64; i++)
    for (int j = 0; j + 1 < nm && cubes.size() < 64; j++) {
      const int ti = (nt / 2 + i) % (nt - 1), mj = (nm / 2 + j) % (nm - 1);
      const double t = 0.5 * (g->tv[ti] + g->tv[ti + 1]), mh = 0.5 * (g->mv[mj] + g->mv[mj + 1]);
      const int lo = std::max(g->llo[ti], g->llo[ti + 1]), hi = std::min(g->lhi[ti], g->lhi[ti + 1]);
      if (hi <= lo) continue;
      const double lg = 0.5 * (g->lv[(lo + hi) / 2] + g->lv[(lo + hi) / 2 + 1]);
      int cols[64];
      float w[64];
      if (local_grid(g->hg, t, mh, lg, cols, w) != 0) continue;
      std::vector<int> c(cols, cols + 64);
      if (std::find(seen.begin(), seen.end(), c) != seen.end()) continue;
      seen.push_back(c);
      cubes.push_back({t, mh, lg});
    }
  if (cubes.size() < 8) return;
  Ctx &C = ctx();
  cudaStream_t s = C.stream;
  const int E = 16 * SEG;
  DevStar st = make_star(nullptr, nullptr, nullptr, nullptr, 0);
  st.disp_kind = DISP_NONE;
  DBuf<DevStar> ds;
  ds.upload(&st, 1);
  DBuf<double> dl;
  dl.alloc((size_t)E * 5);
  DBuf<int> de;
  de.upload(std::vector<int>(E, 0));
  ensure_workspace(g, E, 0);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const double dt = 0.05 * (g->tv[1] - g->tv[0]), dm = 0.05 * (g->mv[1] - g->mv[0]);
  const int ladder[] = {8, 12, 16, 24, 32, 48, 64};
  int best = SEG + 1;
  std::vector<double> lab((size_t)E * 5);
  for (int gs : ladder) {
    const int ng = SEG / gs;
    for (int e = 0; e < E; e++) {
      const int q = e / SEG, u = e % SEG, gi = std::min(u / gs, ng);
      const auto &c = cubes[(size_t)(q * (ng + 1) + gi) % cubes.size()];
      double *x = &lab[(size_t)e * 5];
      x[0] = c[0] + dt * ((u % gs) % 7 - 3) / 3.0;
      x[1] = c[1] + dm * ((u % gs) % 5 - 2) / 2.0;
      x[2] = c[2];
      x[3] = 0.0;
      x[4] = 0.0;
    }
    CK(cudaMemcpy(dl.p, lab.data(), lab.size() * sizeof(double), cudaMemcpyHostToDevice));
    EvalArgs a;
    a.stars = ds.p;
    a.labels = dl.p;
    a.eval_star = de.p;
    a.E = E;
    a.full_window = 1;
    a.max_m = 1;
    star_kinds({st}, a);
    float tm[2];
    for (int mode = 0; mode < 2; mode++) {
      g->tc_min = mode ? gs : SEG + 1;
      run_evals(g, a, s);
      float bt = 1e30f;
      for (int rep = 0; rep < 3; rep++) {
        CK(cudaEventRecord(e0, s));
        run_evals(g, a, s);
        CK(cudaEventRecord(e1, s));
        CK(cudaEventSynchronize(e1));
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        bt = std::min(bt, ms);
      }
      tm[mode] = bt;
    }
    if (getenv("PASTA_TUNE_VERBOSE"))
      fprintf(stderr, "pasta_b200 tune: %lld px, groups of %d: CUDA cores %.4f ms, tensor cores %.4f ms\n",
              (long long)g->npx, gs, tm[0], tm[1]);
    if (tm[1] < tm[0]) {
      if (best > SEG) best = gs;
    } else {
      best = SEG + 1;  // the tensor cores must win from the threshold on
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  g->tc_min = best;
}

}  // namespace

int pasta_grid_create(const double *labels, const uint16_t *spectra, const float *maxima, int64_t n_models,
                      int64_t n_px, int wl_kind, double wl_a, double wl_b, const double *wl_values,
                      pasta_grid **out) {
  return guard([&] {
    if (!labels || !spectra || !out || n_models < 1 || n_px < 2) fail(PASTA_E_ARG, "invalid grid arguments");
    if (wl_kind < 0 || wl_kind > 2) fail(PASTA_E_ARG, "invalid wavelength grid kind");
    Ctx &C = ctx();
    std::unique_ptr<pasta_grid> g(new pasta_grid());
    g->dev = C.dev;
    auto ins = [](std::vector<double> &v, double x) {
      if (std::find(v.begin(), v.end(), x) == v.end()) v.insert(std::lower_bound(v.begin(), v.end(), x), x);
    };
    for (int64_t i = 0; i < n_models; i++) {
      for (int k = 0; k < 3; k++)
        if (labels[3 * i + k] != labels[3 * i + k]) fail(PASTA_E_ARG, "NaN grid label");
      ins(g->tv, labels[3 * i]);
      ins(g->mv, labels[3 * i + 1]);
      ins(g->lv, labels[3 * i + 2]);
    }
    const int nt = (int)g->tv.size(), nm = (int)g->mv.size(), nl = (int)g->lv.size();
    g->llo.assign(nt, nl - 1);
    g->lhi.assign(nt, 0);
    auto idx = [](const std::vector<double> &v, double x) {
      return (int)(std::lower_bound(v.begin(), v.end(), x) - v.begin());
    };
    for (int64_t i = 0; i < n_models; i++) {
      int ti = idx(g->tv, labels[3 * i]), li = idx(g->lv, labels[3 * i + 2]);
      g->llo[ti] = std::min(g->llo[ti], li);
      g->lhi[ti] = std::max(g->lhi[ti], li);
    }
    for (int i = 0; i < nt; i++)
      if (g->llo[i] > g->lhi[i]) fail(PASTA_E_ARG, "Invalid logg limits");
    g->cum.resize(nt);
    int64_t acc = 0;
    for (int i = 0; i < nt; i++) { g->cum[i] = acc; acc += g->lhi[i] - g->llo[i] + 1; }
    g->n_cols = acc * nm;
    if (g->n_cols != n_models)
      fail(PASTA_E_ARG, "grid is incomplete: %lld models given, %lld gridpoints expected", (long long)n_models,
           (long long)g->n_cols);
    g->npx = n_px;
    g->stride = (n_px + 63) / 64 * 64;
    g->hg = GridGeom{g->tv.data(), g->mv.data(), g->lv.data(), g->llo.data(), g->lhi.data(), g->cum.data(), nt, nm, nl};
    // place each model at its column; rows padded to `stride` with zeros
    std::vector<int64_t> col(n_models);
    std::vector<char> seen(g->n_cols, 0);
    std::vector<float> fac(g->n_cols, 1.0f / 65535.0f);
    for (int64_t i = 0; i < n_models; i++) {
      int ti = idx(g->tv, labels[3 * i]), mi = idx(g->mv, labels[3 * i + 1]), li = idx(g->lv, labels[3 * i + 2]);
      int64_t c = (g->cum[ti] + li - g->llo[ti]) * (int64_t)nm + mi;
      if (seen[c]) fail(PASTA_E_ARG, "duplicate grid model (%g, %g, %g)", labels[3 * i], labels[3 * i + 1], labels[3 * i + 2]);
      seen[c] = 1;
      col[i] = c;
      if (maxima) {
        if (maxima[i] < 0.0f) fail(PASTA_E_ARG, "Negative factor: %g", (double)maxima[i]);
        fac[c] = maxima[i] / 65535.0f;
      }
    }
    g->spectra.alloc((size_t)g->n_cols * g->stride);
    CK(cudaMemset(g->spectra.p, 0, (size_t)g->n_cols * g->stride * sizeof(uint16_t)));
    bool in_order = true;
    for (int64_t i = 0; i < n_models; i++) in_order &= col[i] == i;
    if (in_order) {
      CK(cudaMemcpy2D(g->spectra.p, g->stride * sizeof(uint16_t), spectra, n_px * sizeof(uint16_t),
                      n_px * sizeof(uint16_t), n_models, cudaMemcpyHostToDevice));
    } else {
      for (int64_t i = 0; i < n_models; i++)
        CK(cudaMemcpy(g->spectra.p + (size_t)col[i] * g->stride, spectra + (size_t)i * n_px, n_px * sizeof(uint16_t),
                      cudaMemcpyHostToDevice));
    }
    g->factor.upload(fac);
    g->has_tmap = make_grid_tensor_map(g->spectra.p, g->n_cols, g->stride, &g->tmap);
    g->dtv.upload(g->tv); g->dmv.upload(g->mv); g->dlv.upload(g->lv);
    g->dllo.upload(g->llo); g->dlhi.upload(g->lhi); g->dcum.upload(g->cum);
    g->wl_kind = wl_kind;
    g->wl_a = wl_a;
    g->wl_b = wl_b;
    if (wl_kind == WL_NONUNI) {
      if (!wl_values) fail(PASTA_E_ARG, "non-uniform grid needs wavelength values");
      g->wl_vals.assign(wl_values, wl_values + n_px);
      g->dwl.upload(g->wl_vals);
    }
    DevGrid &d = g->d;
    d.g = GridGeom{g->dtv.p, g->dmv.p, g->dlv.p, g->dllo.p, g->dlhi.p, g->dcum.p, nt, nm, nl};
    d.spectra = g->spectra.p;
    d.factor = g->factor.p;
    d.stride = g->stride;
    d.npx = (int)n_px;
    d.tail_start = (int)(n_px - n_px % 128);
    d.wl_kind = wl_kind;
    d.wl_a = wl_a;
    d.wl_b = wl_b;
    d.wl_vals = g->dwl.p;
    if (wl_kind == WL_LIN) { d.synth_first = wl_a; d.synth_last = wl_a + wl_b * (double)n_px; }
    else if (wl_kind == WL_LOG) { d.synth_first = std::pow(10.0, wl_a); d.synth_last = std::pow(10.0, wl_a + wl_b * (double)n_px); }
    else { d.synth_first = wl_values[0]; d.synth_last = wl_values[n_px - 1]; }
    if (wl_kind == WL_LIN) d.dvelo = wl_b / ((wl_a + wl_a + wl_b * (double)n_px) / 2.0);
    else if (wl_kind == WL_LOG) d.dvelo = M_LN10 * wl_b;
    else d.dvelo = 0.0;
    tune_direct(g.get());
    tune_interp_tc(g.get());
    *out = g.release();
  });
}

int pasta_grid_tc_min(const pasta_grid *g, int32_t *out) {
  return guard([&] {
    if (!g || !out) fail(PASTA_E_ARG, "grid and output required");
    *out = g->tc_min;
  });
}
int pasta_grid_set_tc_min(pasta_grid *g, int32_t members) {
  return guard([&] {
    if (!g) fail(PASTA_E_ARG, "grid required");
    if (members < TC_MIN_MEMBERS || members > SEG + 1) fail(PASTA_E_ARG, "members must be in [%d, %d]", TC_MIN_MEMBERS, SEG + 1);
    g->tc_min = members;
  });
}

int pasta_grid_direct_max(const pasta_grid *g, int32_t *out) {
  return guard([&] { *out = g->direct_max; });
}
int pasta_grid_set_direct_max(pasta_grid *g, int32_t taps) {
  return guard([&] {
    if (taps < 0 || taps > DIRECT_MAX_TAPS) fail(PASTA_E_ARG, "direct_max must be in 0..%d", DIRECT_MAX_TAPS);
    std::lock_guard<std::mutex> lk(g->mu);
    g->direct_max = taps;
  });
}

int pasta_grid_destroy(pasta_grid *g) {
  return guard([&] {
    if (!g) return;
    CK(cudaSetDevice(g->dev));
    CK(cudaDeviceSynchronize());
    delete g;
  });
}

int pasta_grid_shape(const pasta_grid *g, int64_t *o) {
  return guard([&] {
    o[0] = (int64_t)g->tv.size(); o[1] = (int64_t)g->mv.size(); o[2] = (int64_t)g->lv.size();
    o[3] = g->npx; o[4] = g->n_cols;
  });
}
int pasta_grid_axis(const pasta_grid *g, int axis, double *out) {
  return guard([&] {
    const auto &v = axis == 0 ? g->tv : axis == 1 ? g->mv : g->lv;
    std::copy(v.begin(), v.end(), out);
  });
}
int pasta_grid_logg_limits(const pasta_grid *g, int64_t *lo, int64_t *hi) {
  return guard([&] {
    for (size_t i = 0; i < g->llo.size(); i++) { lo[i] = g->llo[i]; hi[i] = g->lhi[i]; }
  });
}
int pasta_grid_cumulative_size(const pasta_grid *g, int64_t *out) {
  return guard([&] { std::copy(g->cum.begin(), g->cum.end(), out); });
}
int pasta_grid_clamp_1d(const pasta_grid *g, double t, double m, double lg, int index, double *out) {
  return guard([&] {
    if (index < 0 || index > 2) fail(PASTA_E_ARG, "Index out of bounds %d", index);
    double p[3] = {t, m, lg}, lo, hi;
    int st = grid_limits_at(g->hg, p, index, lo, hi);
    if (st) fail(PASTA_E_OUT_OF_GRID, index == 0 ? "Cannot clamp teff at logg=%g" : "Cannot clamp logg at Teff=%g",
                 index == 0 ? lg : t);
    if (!(lo <= hi)) fail(PASTA_E_CLAMP, "clamp limits invalid");
    double x = p[index];
    *out = x < lo ? lo : (x > hi ? hi : x);
  });
}
int pasta_grid_is_teff_logg_between_bounds(const pasta_grid *g, double t, double lg, int *out) {
  return guard([&] { *out = teff_logg_ok(g->hg, t, lg) ? 1 : 0; });
}
int pasta_grid_coefficients(const pasta_grid *g, double t, double m, double lg, int64_t *cols64, float *w64,
                            double *t16, double *l16, double *m4) {
  return guard([&] {
    int cols[64];
    float w[64];
    double ft[16], fl[16], fm[4];
    int st = local_grid(g->hg, t, m, lg, cols, w, ft, fl, fm);
    if (st) fail(st == S_NAN ? PASTA_E_NAN : st == S_OUT_OF_GRID ? PASTA_E_OUT_OF_GRID : PASTA_E_NEIGHBORS,
                 "%s (%g, %g, %g)", status_message(st), t, m, lg);
    for (int i = 0; i < 64; i++) {
      if (cols64) cols64[i] = cols[i];
      if (w64) w64[i] = w[i];
    }
    if (t16) std::copy(ft, ft + 16, t16);
    if (l16) std::copy(fl, fl + 16, l16);
    if (m4) std::copy(fm, fm + 4, m4);
  });
}

// -------------------------------------------------------- dispersions
int pasta_dispersion_create(int synth_kind, double synth_a, double synth_b, int64_t synth_n,
                            const double *synth_values, int kind, const double *wl_obs, int64_t n_obs,
                            double resolution, const float *disp, pasta_dispersion **out) {
  return guard([&] {
    if (!wl_obs || n_obs < 1 || !out) fail(PASTA_E_ARG, "invalid dispersion arguments");
    ctx();
    std::unique_ptr<pasta_dispersion> d(new pasta_dispersion());
    d->kind = kind;
    d->synth_kind = synth_kind;
    d->synth_a = synth_a;
    d->synth_b = synth_b;
    d->synth_n = synth_n;
    if (synth_kind == WL_NONUNI) d->synth_vals.assign(synth_values, synth_values + synth_n);
    d->wl.assign(wl_obs, wl_obs + n_obs);
    d->fidx.resize(n_obs);
    for (int64_t i = 0; i < n_obs; i++)
      d->fidx[i] = wl_float_index(synth_kind, synth_a, synth_b, d->synth_vals, wl_obs[i]);
    d->wl_first = d->wl.front();
    d->wl_last = d->wl.back();
    d->wl_min = *std::min_element(d->wl.begin(), d->wl.end());
    d->wl_max = *std::max_element(d->wl.begin(), d->wl.end());
    d->fidx_min = *std::min_element(d->fidx.begin(), d->fidx.end());
    d->fidx_max = *std::max_element(d->fidx.begin(), d->fidx.end());
    d->sorted = std::is_sorted(d->fidx.begin(), d->fidx.end()) && std::is_sorted(d->wl.begin(), d->wl.end());
    const auto &vals = d->synth_vals;
    if (kind == PASTA_DISP_NONE) {
      d->dev_kind = DISP_NONE;
    } else if (kind == PASTA_DISP_FIXED) {
      if (resolution <= 0.0) fail(PASTA_E_ARG, "Resolution must be positive");
      if (synth_kind == WL_LOG) {  // convolve_rv.rs:169-196
        double sigma = 1.0 / (M_LN10 * 2.355 * resolution * synth_b);
        int n = odd_width(6.0 * sigma);
        if (n > 2 * 255 + 1) fail(PASTA_E_UNSUPPORTED, "instrument kernel of %d taps exceeds the supported 511", n);
        d->gk.assign(n, 0.0f);
        make_gaussian(d->gk.data(), n, (float)sigma);
        d->gw = n;
        d->dev_kind = DISP_FIXED;
      } else {  // convolve_rv.rs:244-287
        std::vector<float> sig(synth_n);
        for (int64_t i = 0; i < synth_n; i++) {
          if (synth_kind == WL_LIN) sig[i] = (float)(wl_at(synth_kind, synth_a, synth_b, vals, i) / (resolution * synth_b * 2.355));
          else if (i == 0 || i == synth_n - 1) sig[i] = 2.0f;
          else sig[i] = (float)(vals[i] / (resolution * ((vals[i + 1] - vals[i - 1]) / 2.0) * 2.355));
        }
        disp_per_pixel(d.get(), sig);
      }
    } else if (kind == PASTA_DISP_VARIABLE) {  // convolve_rv.rs:350-402
      if (!disp) fail(PASTA_E_ARG, "variable dispersion needs disp values");
      const size_t L = d->wl.size();
      std::vector<float> dr(synth_n);
      size_t j = 0;
      for (int64_t i = 0; i < synth_n; i++) {  // resample_observed_to_synth (convolve_rv.rs:303-331)
        double x = wl_at(synth_kind, synth_a, synth_b, vals, i);
        while (j < L - 1 && d->wl[j + 1] < x) j++;
        if (j == L - 1) dr[i] = disp[j];
        else {
          float w = (float)((x - d->wl[j]) / (d->wl[j + 1] - d->wl[j]));
          dr[i] = (1.0f - w) * disp[j] + w * disp[j + 1];
        }
      }
      std::vector<float> sig(synth_n);
      for (int64_t i = 0; i < synth_n; i++) {
        if (synth_kind == WL_LOG) sig[i] = dr[i] / (float)(synth_b * M_LN10 * wl_at(synth_kind, synth_a, synth_b, vals, i));
        else if (synth_kind == WL_LIN) sig[i] = dr[i] / (float)synth_b;
        else if (i == 0 || i == synth_n - 1) sig[i] = 2.0f;
        else sig[i] = dr[i] / (float)((vals[i + 1] - vals[i - 1]) / 2.0);
      }
      disp_per_pixel(d.get(), sig);
    } else {
      fail(PASTA_E_ARG, "invalid dispersion kind %d", kind);
    }
    d->dfidx.upload(d->fidx);
    d->dwl.upload(d->wl);
    if (!d->gk.empty()) d->dgk.upload(d->gk);
    if (d->dev_kind == DISP_FIXED) d->dgspec.upload(kernel_spectrum(d->gk));
    *out = d.release();
  });
}
int pasta_dispersion_destroy(pasta_dispersion *d) {
  return guard([&] { delete d; });
}
int pasta_dispersion_kernels(const pasta_dispersion *d, int64_t *width, float *out) {
  return guard([&] {
    *width = d->gw;
    if (out && d->dev_kind == DISP_PIXEL) {  // width x n_synth row-major
      for (int64_t i = 0; i < d->synth_n; i++)
        for (int t = 0; t < d->gw; t++) out[(size_t)t * d->synth_n + i] = d->gk[(size_t)i * d->gw + t];
    } else if (out && d->dev_kind == DISP_FIXED) {
      std::copy(d->gk.begin(), d->gk.end(), out);
    }
  });
}

// --------------------------------------------------------- continuum
int pasta_continuum_create(int kind, const double *wl, int64_t n, int n_chunks, int p_order, double overlap,
                           const float *design, int k, const float *continuum, int ignore,
                           pasta_continuum **out) {
  return guard([&] {
    if (!out) fail(PASTA_E_ARG, "null output");
    ctx();
    std::unique_ptr<pasta_continuum> c(new pasta_continuum());
    c->kind = kind;
    c->n = n;
    if (kind == PASTA_CONT_CHUNK) {
      if (!wl) fail(PASTA_E_ARG, "chunk fitter needs wavelengths");
      chunk_setup(c.get(), wl, n_chunks, p_order, overlap);
      c->dcs.upload(c->cstart);
      c->dce.upload(c->cstop);
      c->dxa.upload(c->xa);
      c->dxb.upload(c->xb);
      c->dfac.upload(c->fac);
      c->dchol.upload(c->chol);
    } else if (kind == PASTA_CONT_LINEAR) {
      if (!design) fail(PASTA_E_ARG, "linear fitter needs a design matrix");
      linear_setup(c.get(), design, k);
      c->dq.upload(c->qcol);
      if (c->kp) c->dqt.upload(c->qt);
    } else if (kind == PASTA_CONT_FIXED) {
      if (!continuum) fail(PASTA_E_ARG, "fixed continuum needs values");
      c->cont.assign(continuum, continuum + n);
      c->ignore = ignore;
      if (n - 2 * (int64_t)ignore <= 0) { c->bad = 1; c->bad_msg = "ignore_first_and_last too large"; }
      c->dcont.upload(c->cont);
    } else if (kind != PASTA_CONT_CONSTANT) {
      fail(PASTA_E_ARG, "invalid continuum kind %d", kind);
    }
    *out = c.release();
  });
}
int pasta_continuum_destroy(pasta_continuum *c) {
  return guard([&] { delete c; });
}
int pasta_continuum_nparams(const pasta_continuum *c) { return cont_nparams(c); }

// ContinuumFitter::fit_continuum on a given model (lib.rs:862-874)
int pasta_continuum_fit(const pasta_continuum *c, const float *model, const float *flux, const float *var, int64_t n,
                        float *params, double *chi2) {
  return guard([&] {
    if (c->kind != PASTA_CONT_CONSTANT && n != c->n)
      fail(PASTA_E_ARG, "Length of observed and synthetic spectrum are different %lld, %lld", (long long)n, (long long)c->n);
    if (c->bad) fail(PASTA_E_CONTINUUM, "%s", c->bad_msg.c_str());
    Ctx &C = ctx();
    cudaStream_t s = C.stream;
    DBuf<float> dm, df, dv;
    dm.upload(model, n);
    df.upload(flux, n);
    dv.upload(var, n);
    DevStar st = make_star(nullptr, c, df.p, dv.p, n);
    DBuf<DevStar> ds;
    ds.upload(&st, 1);
    EvalPrep ep{};
    DBuf<EvalPrep> dp;
    dp.upload(&ep, 1);
    DBuf<double> dc, dpar;
    DBuf<int> dst;
    dc.alloc(1);
    dst.alloc(1);
    const int ps = device_param_stride(c);
    dpar.alloc(ps);
    EvalBatch b{};
    b.E = 1;
    b.stars = ds.p;
    b.prep = dp.p;
    b.cost = dc.p;
    b.status = dst.p;
    b.params = dpar.p;
    b.param_stride = ps;
    b.chunk_p1_mask = st.cont_kind == CONT_CHUNK ? 1u << st.p1 : 0u;
    b.max_chunks = st.cont_kind == CONT_CHUNK ? st.n_chunks : 0;
    b.other_cont = st.cont_kind == CONT_CHUNK ? 0 : 1;
    DBuf<double> dpart;
    dpart.alloc(MAX_CHUNKS);
    b.cpart = dpart.p;
    b.given = dm.p;
    DevGrid G{};
    launch_chi2(G, b, s);
    CK(cudaGetLastError());
    double hc;
    int hs;
    std::vector<double> hp(ps);
    CK(cudaMemcpyAsync(&hc, dc.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&hs, dst.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hp.data(), dpar.p, ps * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (hs) fail(PASTA_E_CONTINUUM, "%s", status_message(hs));
    auto pv = params_from_device(c, hp.data());
    if (params) std::copy(pv.begin(), pv.end(), params);
    *chi2 = hc;
  });
}

// ContinuumFitter::build_continuum (lib.rs:927-939)
int pasta_continuum_build(const pasta_continuum *c, const float *params, int64_t np, float *out) {
  return guard([&] {
    if (np != cont_nparams(c))
      fail(PASTA_E_ARG, "Incorrect number of continuum parameters: %lld, expected: %d", (long long)np, cont_nparams(c));
    if (c->kind == PASTA_CONT_CONSTANT) { out[0] = params[0]; return; }
    if (c->kind == PASTA_CONT_FIXED) { std::copy(c->cont.begin(), c->cont.end(), out); return; }
    Ctx &C = ctx();
    cudaStream_t s = C.stream;
    if (c->kind == PASTA_CONT_LINEAR) {  // D * params with D = Q R
      const int k = c->k;
      std::vector<double> z(k, 0.0);
      for (int j = 0; j < k; j++)
        for (int l = j; l < k; l++) z[j] += c->R[(size_t)j * k + l] * (double)params[l];
      for (int64_t i = 0; i < c->n; i++) {
        double s2 = 0.0;
        for (int j = 0; j < k; j++) s2 += (double)c->qcol[(size_t)j * c->n + i] * z[j];
        out[i] = (float)s2;
      }
      return;
    }
    // chunk: monomial -> Legendre coefficients, then the device blend
    const int p1 = c->p1;
    auto T = legendre_to_monomial(p1);
    std::vector<double> coef((size_t)c->nc * MAX_P1, 0.0);
    for (int ch = 0; ch < c->nc; ch++) {
      // solve T^T l = a (upper triangular in the column index)
      std::vector<double> a(p1), l(p1);
      for (int j = 0; j < p1; j++) a[j] = params[ch * p1 + j];
      for (int k = p1 - 1; k >= 0; k--) {
        double s2 = a[k];
        for (int kk = k + 1; kk < p1; kk++) s2 -= T[(size_t)kk * p1 + k] * l[kk];
        l[k] = s2 / T[(size_t)k * p1 + k];
      }
      for (int k = 0; k < p1; k++) coef[(size_t)ch * MAX_P1 + k] = l[k];
    }
    DevStar st = make_star(nullptr, c, nullptr, nullptr, c->n);
    DBuf<DevStar> ds;
    ds.upload(&st, 1);
    DBuf<double> dcoef;
    dcoef.upload(coef);
    DBuf<float> dout;
    dout.alloc(c->n);
    launch_build_chunk(ds.p, dcoef.p, (int)c->n, dout.p, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, dout.p, c->n * sizeof(float), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  });
}

// ----------------------------------------------------- model / chi2
static int run_label_batch(const pasta_grid *gc, const pasta_dispersion *d, const pasta_continuum *c,
                           const float *flux, const float *var, int64_t n, const double *labels, int ncols,
                           int64_t L, float *out_obs, float *out_synth, double *out_chi2, int32_t *status,
                           int full_window, int no_rotation, const float *dot_with = nullptr) {
  return guard([&] {
    pasta_grid *g = const_cast<pasta_grid *>(gc);
    if (L < 0) fail(PASTA_E_ARG, "negative label count");
    if (L == 0) return;
    check_disp_grid(g, d);
    if (d && c && c->kind != PASTA_CONT_CONSTANT && c->n != (int64_t)d->wl.size())
      fail(PASTA_E_ARG, "continuum fitter and dispersion have different lengths");
    if (c && flux && n != (int64_t)d->wl.size())
      fail(PASTA_E_ARG, "Observed spectrum and target dispersion must have the same length");
    Ctx &C = ctx();
    cudaStream_t s = C.stream;
    std::lock_guard<std::mutex> lk(g->mu);
    std::vector<double> lab((size_t)L * 5, 0.0);
    double vmax = 0.0;
    for (int64_t i = 0; i < L; i++) {
      for (int k = 0; k < ncols; k++) lab[(size_t)i * 5 + k] = labels[(size_t)i * ncols + k];
      if (no_rotation) lab[(size_t)i * 5 + 3] = 0.0;
      double v = lab[(size_t)i * 5 + 3];
      if (v > vmax) vmax = v;
    }
    DBuf<float> df, dv;
    const int64_t nobs = d ? (int64_t)d->wl.size() : 0;
    if (flux) { df.upload(flux, n); dv.upload(var, n); }
    DevStar st = make_star(d, c, df.p, dv.p, nobs);
    if (!d) { st.disp_kind = DISP_NONE; }
    DBuf<DevStar> ds;
    ds.upload(&st, 1);
    DBuf<double> dl, dc;
    DBuf<int> de, dst;
    dl.upload(lab);
    de.upload(std::vector<int>(L, 0));
    dc.alloc(L);
    dst.alloc(L);
    DBuf<float> dout;
    EvalArgs a;
    a.stars = ds.p;
    a.labels = dl.p;
    a.eval_star = de.p;
    a.E = L;
    a.cost = dc.p;
    a.status = dst.p;
    a.need_chi2 = out_chi2 ? 1 : 0;
    a.full_window = full_window;
    a.max_m = width_upper_bound(g, vmax);
    star_kinds({st}, a);
    a.lin_group = 128;  // every evaluation belongs to the one star
    if (out_obs) { dout.alloc((size_t)L * nobs); a.out_obs = dout.p; a.out_stride = nobs; }
    if (out_synth) { dout.alloc((size_t)L * g->npx); a.out_synth = dout.p; }
    ensure_workspace(g, L, a.max_nobs);
    run_evals(g, a, s);
    std::vector<int> hst(L, 0);
    CK(cudaMemcpyAsync(hst.data(), dst.p, L * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (out_chi2) {
      std::vector<double> hc(L);
      CK(cudaMemcpyAsync(hc.data(), dc.p, L * sizeof(double), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      for (int64_t i = 0; i < L; i++) out_chi2[i] = hst[i] ? NAN : hc[i];
    }
    CK(cudaStreamSynchronize(s));
    if (status)
      for (int64_t i = 0; i < L; i++) status[i] = hst[i];
    if (out_obs && dot_with) {  // the models stay on the device: out_obs receives L dot products
      DBuf<float> dx, dd;
      dx.upload(dot_with, nobs);
      dd.alloc(L);
      launch_dot_rows(dout.p, nobs, (int)nobs, dx.p, dst.p, dd.p, (int)L, s);
      CK(cudaMemcpyAsync(out_obs, dd.p, (size_t)L * sizeof(float), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
    } else if (out_obs) {
      CK(cudaMemcpyAsync(out_obs, dout.p, (size_t)L * nobs * sizeof(float), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      for (int64_t i = 0; i < L; i++)
        if (hst[i]) std::fill(out_obs + i * nobs, out_obs + (i + 1) * nobs, NAN);
    }
    if (out_synth) {
      CK(cudaMemcpyAsync(out_synth, dout.p, (size_t)L * g->npx * sizeof(float), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      for (int64_t i = 0; i < L; i++)
        if (hst[i]) std::fill(out_synth + i * g->npx, out_synth + (i + 1) * g->npx, NAN);
    }
  });
}

int pasta_interpolate(const pasta_grid *g, const double *tml, int64_t L, float *out, int32_t *status) {
  return run_label_batch(g, nullptr, nullptr, nullptr, nullptr, 0, tml, 3, L, nullptr, out, nullptr, status, 1, 1);
}
int pasta_interpolate_and_convolve(const pasta_grid *g, const pasta_dispersion *d, const double *labels, int64_t L,
                                   float *out, int32_t *status) {
  return run_label_batch(g, d, nullptr, nullptr, nullptr, 0, labels, 4, L, nullptr, out, nullptr, status, 1, 0);
}
int pasta_produce_model(const pasta_grid *g, const pasta_dispersion *d, const double *labels, int64_t L, float *out,
                        int32_t *status) {
  if (!d) { g_last_error = "dispersion required"; return PASTA_E_ARG; }
  return run_label_batch(g, d, nullptr, nullptr, nullptr, 0, labels, 5, L, out, nullptr, nullptr, status, 0, 0);
}
int pasta_ccf(const pasta_grid *g, const pasta_dispersion *d, const double *vs, int64_t V, double teff, double m,
              double logg, const float *flux, int64_t n, float *out, int32_t *status) {
  if (!d || !flux || !out || (V > 0 && !vs)) { g_last_error = "dispersion, velocities, flux and output required"; return PASTA_E_ARG; }
  if (n != (int64_t)d->wl.size()) { g_last_error = "Dispersion and observed flux must have the same length."; return PASTA_E_ARG; }
  // no broadening: the dispersion's wavelengths only (the reference resamples the unbroadened model)
  if (d->kind != PASTA_DISP_NONE) { g_last_error = "ccf needs a no-convolution dispersion on the observed wavelengths"; return PASTA_E_ARG; }
  std::vector<double> lab((size_t)std::max<int64_t>(V, 0) * 5);
  for (int64_t i = 0; i < V; i++) {
    lab[(size_t)i * 5 + 0] = teff;
    lab[(size_t)i * 5 + 1] = m;
    lab[(size_t)i * 5 + 2] = logg;
    lab[(size_t)i * 5 + 3] = 0.0;
    lab[(size_t)i * 5 + 4] = vs[i];
  }
  return run_label_batch(g, d, nullptr, nullptr, nullptr, 0, lab.data(), 5, V, out, nullptr, nullptr, status, 0, 0, flux);
}
int pasta_chi2(const pasta_grid *g, const pasta_dispersion *d, const pasta_continuum *c, const float *flux,
               const float *var, int64_t n, const double *labels, int64_t L, double *out, int32_t *status) {
  if (!d || !c || !flux || !var) { g_last_error = "dispersion, continuum and data required"; return PASTA_E_ARG; }
  return run_label_batch(g, d, c, flux, var, n, labels, 5, L, nullptr, nullptr, out, status, 0, 0);
}

int pasta_chi2_many(const pasta_grid *g, int64_t S, const pasta_dispersion *const *d, const pasta_continuum *const *c,
                    const float *const *flux, const float *const *var, const int64_t *n, const double *labels,
                    double *out, int32_t *status) {
  return guard([&] {
    if (S < 0 || (S > 0 && (!d || !c || !flux || !var || !n || !labels || !out)))
      fail(PASTA_E_ARG, "dispersions, continua, spectra, labels and outputs are required");
    if (S == 0) return;
    std::vector<StarInput> in(S);
    double vmax = 0.0;
    for (int64_t i = 0; i < S; i++) {
      if (!d[i] || !c[i] || !flux[i] || !var[i]) fail(PASTA_E_ARG, "spectrum %lld: missing input", (long long)i);
      in[i] = StarInput{d[i], c[i], nullptr, flux[i], var[i], n[i], 0};
      validate_star(g, in[i]);
      if (labels[5 * i + 3] > vmax) vmax = labels[5 * i + 3];
    }
    pasta_grid *gg = const_cast<pasta_grid *>(g);
    std::lock_guard<std::mutex> lk(gg->mu);
    Ctx &C = ctx();
    cudaStream_t s = C.stream;
    StarSet ss;
    ss.build(in);
    std::vector<int> star(S);
    for (int64_t i = 0; i < S; i++) star[i] = (int)i;
    DBuf<double> lab, cost;
    DBuf<int> es, st;
    lab.upload(labels, (size_t)S * 5);
    es.upload(star);
    cost.alloc(S);
    st.alloc(S);
    EvalArgs a;
    a.stars = ss.dstars.p;
    a.labels = lab.p;
    a.eval_star = es.p;
    a.E = S;
    a.cost = cost.p;
    a.status = st.p;
    a.need_chi2 = 1;
    a.max_m = width_upper_bound(g, vmax);
    star_kinds(ss.h, a);
    a.lin_group = 1;  // one evaluation per star
    a.star_len = 1;
    ensure_workspace(gg, S, a.max_nobs);
    run_evals(gg, a, s);
    std::vector<int> hs(S);
    CK(cudaMemcpyAsync(out, cost.p, (size_t)S * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hs.data(), st.p, (size_t)S * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int64_t i = 0; i < S; i++) {
      if (status) status[i] = hs[i];
      if (hs[i]) out[i] = std::numeric_limits<double>::quiet_NaN();
    }
  });
}

int pasta_dispersion_convolve(const pasta_dispersion *d, const float *in, int64_t n, float *out) {
  return guard([&] {
    if (n != d->synth_n)
      fail(PASTA_E_ARG, "flux_arr and wavelength grid don't match. flux_arr: %lld, synth_wl: %lld", (long long)n,
           (long long)d->synth_n);
    Ctx &C = ctx();
    cudaStream_t s = C.stream;
    DBuf<float> di, dout;
    di.upload(in, n);
    dout.alloc(n);
    DevStar st = make_star(d, nullptr, nullptr, nullptr, 0);
    DBuf<DevStar> ds;
    ds.upload(&st, 1);
    DevGrid G{};
    G.npx = (int)n;
    launch_gauss_standalone(G, ds.p, di.p, dout.p, s);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, dout.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  });
}

int pasta_dispersion_convolve_resample(const pasta_dispersion *d, int in_kind, double in_a, double in_b,
                                       int64_t n_in, const float *in, int64_t M, float *out) {
  return guard([&] {
    if (!d || !in || !out || M < 0) fail(PASTA_E_ARG, "dispersion, input and output are required");
    if (M == 0) return;
    if (n_in != d->synth_n)
      fail(PASTA_E_ARG, "flux_arr and wavelength grid don't match. flux_arr: %lld, synth_wl: %lld", (long long)n_in,
           (long long)d->synth_n);
    if (in_kind != WL_LOG && in_kind != WL_LIN)
      fail(PASTA_E_UNSUPPORTED, "resampling from a non-uniform input wavelength grid is not supported");
    // the range checks of shift_and_resample at RV 0 (convolve_rv.rs:548-567);
    // WlGrid::get_first_and_last ends one step past the last pixel (interpolate.rs:695-698)
    const double first = in_kind == WL_LOG ? std::pow(10.0, in_a) : in_a;
    const double last = in_kind == WL_LOG ? std::pow(10.0, in_a + in_b * (double)n_in) : in_a + in_b * (double)n_in;
    if (d->wl.front() < first)
      fail(PASTA_E_RV_RANGE, "Observed wavelength is smaller than synthetic wavelength (RV=0, %.1f < %.1f)",
           d->wl.front(), first);
    if (d->wl.back() > last)
      fail(PASTA_E_RV_RANGE, "Observed wavelength is larger than synthetic wavelength (RV=0, %.1f > %.1f)",
           d->wl.back(), last);
    // the reference reads pixel floor(index) + 1 (an index panic past the end)
    if (std::floor(d->fidx_max) + 1.0 >= (double)n_in) fail(PASTA_E_RESAMPLE, "resampling index out of range");
    Ctx &C = ctx();
    cudaStream_t s = C.stream;
    DevStar st = make_star(d, nullptr, nullptr, nullptr, (int64_t)d->wl.size());
    DBuf<DevStar> ds;
    ds.upload(&st, 1);
    const int64_t nobs = (int64_t)d->wl.size();
    // spectra per launch: device buffers of about 1 GB
    const int64_t per = (2 * n_in + nobs) * (int64_t)sizeof(float);
    const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(M, (1ll << 30) / per));
    DBuf<float> di, dc, dout;
    di.alloc((size_t)chunk * n_in);
    dc.alloc((size_t)chunk * n_in);
    dout.alloc((size_t)chunk * nobs);
    for (int64_t m0 = 0; m0 < M; m0 += chunk) {
      const int64_t k = std::min(chunk, M - m0);
      CK(cudaMemcpyAsync(di.p, in + (size_t)m0 * n_in, (size_t)k * n_in * sizeof(float), cudaMemcpyHostToDevice, s));
      launch_gauss_batch((int)n_in, ds.p, di.p, dc.p, (int)k, s);
      launch_resample_rows((int)n_in, in_kind, ds.p, (int)nobs, dc.p, dout.p, (int)k, s);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(out + (size_t)m0 * nobs, dout.p, (size_t)k * nobs * sizeof(float), cudaMemcpyDeviceToHost,
                         s));
      CK(cudaStreamSynchronize(s));
    }
  });
}

// ============================================================= binaries
namespace {

// Device buffers for binary labels: up to cap labels of an observed
// spectrum of nobs pixels on a grid with `tiles` continuum tiles.
struct BinaryScratch {
  int64_t cap = 0, nobs = 0;
  int tiles = 0;
  DBuf<double> labels;  // [cap][11]
  DBuf<double> comp;    // [2 cap][5]
  DBuf<int> star0;      // [2 cap] all zero: every component belongs to star 0
  DBuf<LinRec> lin;     // [2 cap]
  DBuf<double> part;    // [2 cap][tiles]
  DBuf<EvalPrep> cprep; // [cap]
  DBuf<float> model;    // [cap][nobs]
  DBuf<double> cost;    // [cap]
  DBuf<int> status;     // [cap]
  void ensure(int64_t L, int t, int64_t n) {
    if (L <= cap && t == tiles && n == nobs) return;
    labels.alloc((size_t)L * 11);
    comp.alloc((size_t)L * 10);
    star0.alloc((size_t)L * 2);
    CK(cudaMemset(star0.p, 0, (size_t)L * 2 * sizeof(int)));
    lin.alloc((size_t)L * 2);
    part.alloc((size_t)L * 2 * t);
    cprep.alloc((size_t)L);
    CK(cudaMemset(cprep.p, 0, (size_t)L * sizeof(EvalPrep)));
    model.alloc((size_t)L * n);
    cost.alloc((size_t)L);
    status.alloc((size_t)L);
    cap = L;
    tiles = t;
    nobs = n;
  }
};

void check_binary_grids(const pasta_grid *g, const pasta_grid *gc) {
  if (!gc) fail(PASTA_E_ARG, "a continuum interpolator is required");
  if (gc->npx != g->npx)
    fail(PASTA_E_ARG, "continuum grid has %lld pixels and the model grid %lld: they must be equal",
         (long long)gc->npx, (long long)g->npx);
  if (gc->dev != g->dev) fail(PASTA_E_ARG, "the continuum grid lives on another device");
}

// The L binary labels in bs.labels (device): the components through the
// regular pipeline on the whole synthetic grid, the continua, the combined
// model at the observed pixels (bs.model, status in bs.cprep) and, when
// chi2, the continuum fit (bs.cost, bs.status; params when given).  Runs in
// sub-batches of half the workspace (two components per label);
// asynchronous on s, no allocation.
void run_binary(pasta_grid *g, const pasta_grid *gc, const DevStar *dstar, const DevStar &hstar,
                BinaryScratch &bs, int64_t L, double vs_max, bool chi2, double *dparams, int param_stride,
                cudaStream_t s) {
  EvalArgs a;
  a.stars = dstar;
  a.eval_star = bs.star0.p;
  a.need_chi2 = 0;
  a.full_window = 1;
  a.max_m = width_upper_bound(g, vs_max);
  star_kinds({hstar}, a);
  const int64_t capL = std::min<int64_t>(g->ws.cap / 2, bs.cap);
  if (capL < 1) fail(PASTA_E_NOMEM, "the evaluation workspace holds fewer than two evaluations");
  const int64_t nobs = hstar.n_obs;
  for (int64_t off = 0; off < L; off += capL) {
    const int64_t cnt = std::min(capL, L - off);
    BinaryBatch bb{};
    bb.L = (int)cnt;
    bb.labels = bs.labels.p + (size_t)off * 11;
    bb.comp_labels = bs.comp.p;
    bb.lin = bs.lin.p;
    bb.part = bs.part.p;
    bb.lin_tiles = bs.tiles;
    bb.cprep = bs.cprep.p + off;
    bb.model = bs.model.p + (size_t)off * nobs;
    bb.model_stride = nobs;
    launch_binary_split(gc->d, bb, s);
    a.labels = bs.comp.p;
    a.E = 2 * cnt;
    run_evals(g, a, s);  // 2 cnt <= workspace capacity: rows [0, 2 cnt)
    const EvalBatch comp = make_batch(g, a, 0, 2 * cnt);
    launch_interp_linear(gc->d, comp, bb, s);
    launch_binary_combine(g->d, (int)gc->npx, comp, bb, (int)nobs, s);
    if (chi2) {
      EvalBatch cb{};
      cb.E = (int)cnt;
      cb.stars = dstar;
      cb.prep = bb.cprep;
      cb.cost = bs.cost.p + off;
      cb.status = bs.status.p + off;
      cb.params = dparams ? dparams + (size_t)off * param_stride : nullptr;
      cb.param_stride = param_stride;
      cb.need_chi2 = 1;
      cb.chunk_p1_mask = a.chunk_p1_mask;
      cb.max_chunks = a.max_chunks;
      cb.other_cont = a.other_cont;
      cb.lin_group = linear_tc_enabled() ? 128 : 0;  // every label belongs to the one star
      cb.lin_kp_mask = a.lin_kp_mask;
      set_lin_slices(g, cb);
      cb.cpart = g->ws.cpart.p;
      cb.given = bb.model;
      cb.given_stride = nobs;
      launch_chi2(g->d, cb, s);
    }
  }
  CK(cudaGetLastError());
}

double max_binary_vsini(const double *labels, int64_t L) {
  double v = 0.0;
  for (int64_t i = 0; i < L; i++)
    for (int k : {3, 8}) {
      const double x = labels[(size_t)i * 11 + k];
      if (x > v) v = x;
    }
  return v;
}

// statuses of the L labels whose combination ran (model entry point)
std::vector<int> binary_status(const BinaryScratch &bs, int64_t L, cudaStream_t s) {
  std::vector<EvalPrep> hp((size_t)L);
  CK(cudaMemcpyAsync(hp.data(), bs.cprep.p, (size_t)L * sizeof(EvalPrep), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  std::vector<int> st((size_t)L);
  for (int64_t i = 0; i < L; i++) st[i] = hp[i].status;
  return st;
}

}  // namespace

int pasta_interpolate_linear(const pasta_grid *gc_, const double *tml, int64_t L, float *out, int32_t *status) {
  return guard([&] {
    pasta_grid *g = const_cast<pasta_grid *>(gc_);
    if (L < 0) fail(PASTA_E_ARG, "negative label count");
    if (L == 0) return;
    Ctx &C = ctx();
    cudaStream_t s = C.stream;
    const int64_t npx = g->npx, str = (npx + 63) / 64 * 64;
    const int tiles = linear_tiles((int)npx);
    DBuf<double> dl;
    DBuf<LinRec> lin;
    DBuf<double> part;
    DBuf<float> dout;
    dl.upload(tml, (size_t)L * 3);
    lin.alloc((size_t)L);
    part.alloc((size_t)L * tiles);
    dout.alloc((size_t)L * str);
    launch_linear_prep(g->d, dl.p, (int)L, lin.p, s);
    launch_interp_linear_rows(g->d, lin.p, (int)L, dout.p, str, part.p, s);
    CK(cudaGetLastError());
    std::vector<LinRec> hl((size_t)L);
    CK(cudaMemcpyAsync(hl.data(), lin.p, (size_t)L * sizeof(LinRec), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpy2DAsync(out, npx * sizeof(float), dout.p, str * sizeof(float), npx * sizeof(float), (size_t)L,
                         cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int64_t i = 0; i < L; i++) {
      if (status) status[i] = hl[i].status;
      if (hl[i].status) std::fill(out + i * npx, out + (i + 1) * npx, NAN);
    }
  });
}

int pasta_binary_model(const pasta_grid *g_, const pasta_grid *cg, const pasta_dispersion *d, const double *labels,
                       int64_t L, float *out, int32_t *status) {
  return guard([&] {
    pasta_grid *g = const_cast<pasta_grid *>(g_);
    if (!d) fail(PASTA_E_ARG, "dispersion required");
    if (L < 0) fail(PASTA_E_ARG, "negative label count");
    if (L == 0) return;
    check_disp_grid(g, d);
    check_binary_grids(g, cg);
    Ctx &C = ctx();
    cudaStream_t s = C.stream;
    std::lock_guard<std::mutex> lk(g->mu);
    const int64_t nobs = (int64_t)d->wl.size();
    DevStar st = make_star(d, nullptr, nullptr, nullptr, nobs);
    DBuf<DevStar> ds;
    ds.upload(&st, 1);
    ensure_workspace(g, 2 * L, nobs);
    BinaryScratch bs;
    bs.ensure(L, linear_tiles((int)g->npx), nobs);
    CK(cudaMemcpyAsync(bs.labels.p, labels, (size_t)L * 11 * sizeof(double), cudaMemcpyHostToDevice, s));
    run_binary(g, cg, ds.p, st, bs, L, max_binary_vsini(labels, L), false, nullptr, 0, s);
    CK(cudaMemcpyAsync(out, bs.model.p, (size_t)L * nobs * sizeof(float), cudaMemcpyDeviceToHost, s));
    const std::vector<int> hs = binary_status(bs, L, s);
    for (int64_t i = 0; i < L; i++) {
      if (status) status[i] = hs[i];
      if (hs[i]) std::fill(out + i * nobs, out + (i + 1) * nobs, NAN);
    }
  });
}

int pasta_binary_chi2(const pasta_grid *g_, const pasta_grid *cg, const pasta_dispersion *d,
                      const pasta_continuum *c, const float *flux, const float *var, int64_t n,
                      const double *labels, int64_t L, double *out, int32_t *status) {
  return guard([&] {
    pasta_grid *g = const_cast<pasta_grid *>(g_);
    if (!d || !c || !flux || !var) fail(PASTA_E_ARG, "dispersion, continuum and data required");
    if (L < 0) fail(PASTA_E_ARG, "negative label count");
    if (L == 0) return;
    check_disp_grid(g, d);
    check_binary_grids(g, cg);
    if (n != (int64_t)d->wl.size()) fail(PASTA_E_ARG, "Observed spectrum and target dispersion must have the same length");
    if (c->kind != PASTA_CONT_CONSTANT && c->n != n)
      fail(PASTA_E_ARG, "continuum fitter and dispersion have different lengths");
    Ctx &C = ctx();
    cudaStream_t s = C.stream;
    std::lock_guard<std::mutex> lk(g->mu);
    DBuf<float> df, dv;
    df.upload(flux, n);
    dv.upload(var, n);
    DevStar st = make_star(d, c, df.p, dv.p, n);
    DBuf<DevStar> ds;
    ds.upload(&st, 1);
    ensure_workspace(g, 2 * L, n);
    BinaryScratch bs;
    bs.ensure(L, linear_tiles((int)g->npx), n);
    CK(cudaMemcpyAsync(bs.labels.p, labels, (size_t)L * 11 * sizeof(double), cudaMemcpyHostToDevice, s));
    run_binary(g, cg, ds.p, st, bs, L, max_binary_vsini(labels, L), true, nullptr, 0, s);
    std::vector<double> hc((size_t)L);
    std::vector<int> hs((size_t)L);
    CK(cudaMemcpyAsync(hc.data(), bs.cost.p, (size_t)L * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(hs.data(), bs.status.p, (size_t)L * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int64_t i = 0; i < L; i++) {
      out[i] = hs[i] ? NAN : hc[i];
      if (status) status[i] = hs[i];
    }
  });
}

namespace {

// BinaryBounds (bounds.rs:188-275) inside ConstrainedPSOBounds
// (bounds.rs:69-130): star 1 at 0..5, star 2 at 5..10, the light ratio at
// 10 in (0, 1) as BinaryFitter::fit sets it (fitting.rs:649-655).
struct BinaryBoundsH {
  const GridGeom *G = nullptr;
  pasta_binary_settings S{};
  double mn[11], mx[11];
  void constrain(int i, double &lo, double &hi) const {
    if (S.ckind[i] == 1) { lo = S.ca[i]; hi = S.ca[i]; }
    else if (S.ckind[i] == 2) { lo = std::max(lo, S.ca[i]); hi = std::min(hi, S.cb[i]); }
  }
  void init(const pasta_grid *g, const pasta_binary_settings &st) {
    G = &g->hg;
    S = st;
    for (int k = 0; k < 2; k++) {
      mn[5 * k] = g->tv.front(); mx[5 * k] = g->tv.back();
      mn[5 * k + 1] = g->mv.front(); mx[5 * k + 1] = g->mv.back();
      mn[5 * k + 2] = g->lv.front(); mx[5 * k + 2] = g->lv.back();
      mn[5 * k + 3] = st.vsini_lo; mx[5 * k + 3] = st.vsini_hi;
      mn[5 * k + 4] = st.rv_lo; mx[5 * k + 4] = st.rv_hi;
    }
    mn[10] = 0.0; mx[10] = 1.0;
    for (int i = 0; i < 11; i++) constrain(i, mn[i], mx[i]);
  }
  int limits_at(const double *p, int i, double &lo, double &hi) const {
    if (i == 3 || i == 8) { lo = S.vsini_lo; hi = S.vsini_hi; }
    else if (i == 4 || i == 9) { lo = S.rv_lo; hi = S.rv_hi; }
    else if (i == 10) { lo = 0.0; hi = 1.0; }
    else {
      const int st = grid_limits_at(*G, i < 5 ? p : p + 5, i < 5 ? i : i - 5, lo, hi);
      if (st) return st;
    }
    constrain(i, lo, hi);
    return S_OK;
  }
  int clamp_1d(const double *p, int i, double &out) const {  // bounds.rs:13-16
    double lo, hi;
    const int st = limits_at(p, i, lo, hi);
    if (st) return st;
    if (!(lo <= hi)) return S_CLAMP;
    out = p[i] < lo ? lo : (p[i] > hi ? hi : p[i]);
    return S_OK;
  }
  bool within(const double *p) const {
    for (int k = 0; k < 2; k++) {
      const double *q = p + 5 * k;
      if (!(m_ok(*G, q[1]) && teff_logg_ok(*G, q[0], q[2]))) return false;
      if (!(q[3] >= S.vsini_lo && q[3] <= S.vsini_hi && q[4] >= S.rv_lo && q[4] <= S.rv_hi)) return false;
    }
    if (!(p[10] >= 0.0 && p[10] <= 1.0)) return false;
    for (int i = 0; i < 11; i++) {
      if (S.ckind[i] == 1 && !(std::fabs(p[i] - S.ca[i]) <= 2.220446049250313e-16)) return false;
      if (S.ckind[i] == 2 && !(p[i] >= S.ca[i] && p[i] <= S.cb[i])) return false;
    }
    return true;
  }
};

}  // namespace

// BinaryFitter::fit: the swarm runs on the host (11-dimensional positions on
// the draw stream of the single-star fit), every iteration's particles are
// evaluated as one batch on the device.
int pasta_binary_fit(const pasta_grid *g_, const pasta_grid *cg, const pasta_dispersion *d,
                     const pasta_continuum *c, const pasta_binary_settings *settings, const float *flux,
                     const float *var, int64_t n, uint64_t seed, pasta_binary_result *res, float *params,
                     double *trace) {
  return guard([&] {
    pasta_grid *g = const_cast<pasta_grid *>(g_);
    if (!d || !c || !settings || !flux || !var || !res) fail(PASTA_E_ARG, "dispersion, continuum, settings and data required");
    const pasta_binary_settings &st = *settings;
    if (st.num_particles < 1 || st.num_particles > MAX_PARTICLES)
      fail(PASTA_E_ARG, "num_particles must be in 1..%d", MAX_PARTICLES);
    if (st.max_iters < 0) fail(PASTA_E_ARG, "max_iters must be >= 0");
    if (st.social_factor < 0.0) fail(PASTA_E_ARG, "`ParticleSwarm`: social factor must be >=0.");
    if (st.delta < 0.0) fail(PASTA_E_ARG, "`ParticleSwarm`: delta must be >=0.");
    check_disp_grid(g, d);
    check_binary_grids(g, cg);
    if (n != (int64_t)d->wl.size()) fail(PASTA_E_ARG, "Observed spectrum and target dispersion must have the same length");
    if (c->kind != PASTA_CONT_CONSTANT && c->n != n)
      fail(PASTA_E_ARG, "continuum fitter and dispersion have different lengths");
    const double t0 = now_s();
    Ctx &C = ctx();
    cudaStream_t s = C.stream;
    std::lock_guard<std::mutex> lk(g->mu);
    constexpr int D = 11;
    const int P = st.num_particles;
    BinaryBoundsH B;
    B.init(g, st);
    DBuf<float> df, dv;
    df.upload(flux, n);
    dv.upload(var, n);
    DevStar hstar = make_star(d, c, df.p, dv.p, n);
    DBuf<DevStar> ds;
    ds.upload(&hstar, 1);
    ensure_workspace(g, 2 * (int64_t)P, n);
    BinaryScratch bs;
    bs.ensure(P, linear_tiles((int)g->npx), n);
    const double vs_max = std::max(B.mx[3], B.mx[8]);
    std::vector<double> x((size_t)P * D), v((size_t)P * D), bx, cost(P), bcost, gx(D);
    std::vector<int> est(P);
    double gcost = 0.0;
    int status = S_OK;
    // bounds.rs:21-35 (rejection sampling) and particleswarm.rs:137-150
    uint64_t cand = 0;
    for (int p = 0; p < P && !status;) {
      if (cand > 20000000ull) { status = S_BOUNDS; break; }
      double t[D];
      for (int k = 0; k < D; k++)
        t[k] = B.mn[k] == B.mx[k] ? B.mn[k] : uniform_between(B.mn[k], B.mx[k], draw_u01(seed, PH_INIT_POS, cand, 0, k));
      cand++;
      if (B.within(t)) {
        std::copy(t, t + D, &x[(size_t)p * D]);
        p++;
      }
    }
    for (int p = 0; p < P; p++)
      for (int k = 0; k < D; k++) {
        const double w = B.mx[k] - B.mn[k];
        v[(size_t)p * D + k] = (-w == w) ? -w : uniform_between(-w, w, draw_u01(seed, PH_INIT_VEL, p, 0, k));
      }
    // One evaluation of the swarm: positions in, costs and statuses out,
    // through page-locked buffers.  The sequence is the same every
    // iteration, so it is captured once as a CUDA graph and replayed (one
    // launch per iteration instead of a dozen kernels and three copies).
    HostBuf<double> hx, hcost;
    HostBuf<int> hest;
    hx.alloc((size_t)P * D);
    hcost.alloc(P);
    hest.alloc(P);
    auto enqueue = [&]() {
      CK(cudaMemcpyAsync(bs.labels.p, hx.p, (size_t)P * D * sizeof(double), cudaMemcpyHostToDevice, s));
      run_binary(g, cg, ds.p, hstar, bs, P, vs_max, true, nullptr, 0, s);
      CK(cudaMemcpyAsync(hcost.p, bs.cost.p, P * sizeof(double), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(hest.p, bs.status.p, P * sizeof(int), cudaMemcpyDeviceToHost, s));
    };
    GraphHold gh;
    bool try_graph = !getenv("PASTA_NO_GRAPH");
    auto evaluate = [&]() -> int {
      std::copy(x.begin(), x.end(), hx.p);
      if (try_graph) {
        try_graph = false;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        try {
          enqueue();
        } catch (...) {
          cudaGraph_t dead = nullptr;
          cudaStreamEndCapture(s, &dead);  // leave capture mode before the error propagates
          if (dead) cudaGraphDestroy(dead);
          cudaGetLastError();
          throw;
        }
        CK(cudaStreamEndCapture(s, &gh.graph));
        CK(cudaGraphInstantiate(&gh.exec, gh.graph, 0));
      }
      if (gh.exec) CK(cudaGraphLaunch(gh.exec, s));
      else enqueue();
      CK(cudaStreamSynchronize(s));
      std::copy(hcost.p, hcost.p + P, cost.begin());
      std::copy(hest.p, hest.p + P, est.begin());
      for (int p = 0; p < P; p++)
        if (est[p]) return est[p];
      return S_OK;
    };
    auto dump = [&](int it) {
      if (!trace) return;
      for (int p = 0; p < P; p++) {
        double *t = trace + ((size_t)it * P + p) * (D + 1);
        for (int k = 0; k < D; k++) t[k] = x[(size_t)p * D + k];
        t[D] = cost[p];
      }
    };
    if (!status) status = evaluate();
    if (!status) {  // particleswarm.rs:111-134: sorted by cost once (stable, NaN last)
      std::vector<int> idx(P);
      for (int p = 0; p < P; p++) idx[p] = p;
      auto key = [&](int p) { return cost[p] != cost[p] ? INFINITY : cost[p]; };
      std::stable_sort(idx.begin(), idx.end(), [&](int a_, int b_) { return key(a_) < key(b_); });
      std::vector<double> x2(x.size()), v2(v.size()), c2(P);
      for (int r = 0; r < P; r++) {
        for (int k = 0; k < D; k++) {
          x2[(size_t)r * D + k] = x[(size_t)idx[r] * D + k];
          v2[(size_t)r * D + k] = v[(size_t)idx[r] * D + k];
        }
        c2[r] = cost[idx[r]];
      }
      x = x2; v = v2; cost = c2;
      bx = x; bcost = cost;
      std::copy(x.begin(), x.begin() + D, gx.begin());
      gcost = cost[0];
      dump(0);
    }
    for (int it = 0; it < st.max_iters && !status; it++) {  // particleswarm.rs:219-307
      for (int p = 0; p < P && !status; p++) {
        double *xp = &x[(size_t)p * D], *vp = &v[(size_t)p * D];
        const double *bp = &bx[(size_t)p * D];
        for (int k = 0; k < D; k++) {
          const double momentum = vp[k] * st.inertia_factor;
          const double to_opt = bp[k] - xp[k];
          const double pull = (to_opt == 0.0 ? 0.0 : uniform_between(0.0, to_opt, draw_u01(seed, PH_ITER, it, p, 2 * k))) * st.cognitive_factor;
          const double to_g = gx[k] - xp[k];
          const double pullg = (to_g == 0.0 ? 0.0 : uniform_between(0.0, to_g, draw_u01(seed, PH_ITER, it, p, 2 * k + 1))) * st.social_factor;
          vp[k] = momentum + pull + pullg;
          double nx[D];
          std::copy(xp, xp + D, nx);
          nx[k] += vp[k];
          double cl;
          const int cs = B.clamp_1d(nx, k, cl);
          if (cs) { status = cs; break; }
          xp[k] = cl;
          if (!B.within(xp)) { status = S_BOUNDS; break; }
        }
      }
      if (status) break;
      status = evaluate();
      if (status) break;
      for (int p = 0; p < P; p++) {
        if (cost[p] < bcost[p]) {
          std::copy(&x[(size_t)p * D], &x[(size_t)p * D] + D, &bx[(size_t)p * D]);
          bcost[p] = cost[p];
          if (cost[p] < gcost) {
            std::copy(&x[(size_t)p * D], &x[(size_t)p * D] + D, gx.begin());
            gcost = cost[p];
          }
        }
      }
      dump(it + 1);
    }
    // continuum parameters at the best position (fitting.rs:674-686)
    std::vector<float> pv;
    if (!status) {
      const int ps = device_param_stride(c);
      DBuf<double> dpar;
      dpar.alloc(ps);
      CK(cudaMemcpyAsync(bs.labels.p, gx.data(), D * sizeof(double), cudaMemcpyHostToDevice, s));
      run_binary(g, cg, ds.p, hstar, bs, 1, std::max(gx[3], gx[8]), true, dpar.p, ps, s);
      std::vector<double> hp(ps);
      int hs = 0;
      CK(cudaMemcpyAsync(hp.data(), dpar.p, ps * sizeof(double), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(&hs, bs.status.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      if (hs) status = hs;
      else pv = params_from_device(c, hp.data());
    }
    std::memset(res, 0, sizeof *res);
    for (int k = 0; k < 5; k++) {
      res->label1[k] = gx[k];
      res->label2[k] = gx[5 + k];
    }
    res->light_ratio = gx[10];
    res->chi2 = gcost;
    res->iterations = st.max_iters;
    res->status = status;
    res->n_params = (int)pv.size();
    res->time = now_s() - t0;
    if (params) std::copy(pv.begin(), pv.end(), params);
  });
}

// ------------------------------------------------------------- fit
static int fit_common(const pasta_grid *gc, std::vector<StarInput> &in, int mode, pasta_fit_result *results,
                      float *const *params, double *trace) {
  return guard([&] {
    pasta_grid *g = const_cast<pasta_grid *>(gc);
    if (in.empty()) return;
    for (auto &s : in) validate_star(g, s);
    std::lock_guard<std::mutex> lk(g->mu);
    std::vector<std::vector<float>> pv;
    if (mode == PASTA_FIT_PLAIN) fit_plain(g, in, results, pv, trace);
    else fit_batched(g, in, results, pv, trace);
    for (size_t i = 0; i < in.size(); i++)
      if (params && params[i]) std::copy(pv[i].begin(), pv[i].end(), params[i]);
  });
}

int pasta_fit(const pasta_grid *g, const pasta_dispersion *d, const pasta_continuum *c,
              const pasta_pso_settings *settings, const float *flux, const float *var, int64_t n, int64_t S,
              const uint64_t *seeds, int mode, pasta_fit_result *results, float *params, double *trace) {
  std::vector<StarInput> in(S);
  std::vector<float *> pp(S);
  const int np = c ? cont_nparams(c) : 1;
  for (int64_t i = 0; i < S; i++) {
    in[i] = StarInput{d, c, settings, flux + (size_t)i * n, var + (size_t)i * n, n, seeds[i]};
    pp[i] = params ? params + (size_t)i * np : nullptr;
  }
  return fit_common(g, in, mode, results, pp.data(), trace);
}

int pasta_fit_many(const pasta_grid *g, int64_t S, const pasta_dispersion *const *d, const pasta_continuum *const *c,
                   const pasta_pso_settings *settings, const float *const *flux, const float *const *var,
                   const int64_t *n, const uint64_t *seeds, int mode, pasta_fit_result *results,
                   float *const *params) {
  std::vector<StarInput> in(S);
  for (int64_t i = 0; i < S; i++) in[i] = StarInput{d[i], c[i], &settings[i], flux[i], var[i], n[i], seeds[i]};
  return fit_common(g, in, mode, results, params, nullptr);
}

// ---------------------------------------------------------- uncertainty
namespace {

// Brent's zero finder (R. P. Brent, "Algorithms for Minimization without
// Derivatives", 1973, ch. 4; the same iteration as Numerical Recipes'
// zbrent): bisection, secant and inverse quadratic interpolation with the
// bracket [b, c] kept around the root.  SingleFitter::compute_uncertainty
// runs it through argmin's BrentRoot with tol = 1e-3 (fitting.rs:536-541).
// The search is a state machine so that one batched chi2 launch serves the
// pending evaluation of every open search.
struct BrentSearch {
  double a = 0, b = 0, c = 0, d = 0, e = 0, fa = 0, fb = 0, fc = 0, tol = 1e-3;
  int state = 0;  // 0: f(a), f(b) pending; 1: f(b) pending; 2: converged; 3: failed
  int status = 0; // failure code
  int iters = 0;
  // after fb is known: either converge or move b and ask for f(b)
  void advance() {
    if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) {
      c = a;
      fc = fa;
      d = b - a;
      e = d;
    }
    if (std::fabs(fc) < std::fabs(fb)) {
      a = b; b = c; c = a;
      fa = fb; fb = fc; fc = fa;
    }
    const double tol1 = 2.0 * std::numeric_limits<double>::epsilon() * std::fabs(b) + 0.5 * tol;
    const double xm = 0.5 * (c - b);
    if (std::fabs(xm) <= tol1 || fb == 0.0) {
      state = 2;
      return;
    }
    if (++iters > 500) {
      state = 3;
      status = PASTA_E_INTERNAL;
      return;
    }
    if (std::fabs(e) >= tol1 && std::fabs(fa) > std::fabs(fb)) {
      const double s = fb / fa;
      double p, q;
      if (a == c) {
        p = 2.0 * xm * s;
        q = 1.0 - s;
      } else {
        const double qq = fa / fc, r = fb / fc;
        p = s * (2.0 * xm * qq * (qq - r) - (b - a) * (r - 1.0));
        q = (qq - 1.0) * (r - 1.0) * (s - 1.0);
      }
      if (p > 0.0) q = -q;
      p = std::fabs(p);
      const double min1 = 3.0 * xm * q - std::fabs(tol1 * q), min2 = std::fabs(e * q);
      if (2.0 * p < std::min(min1, min2)) {
        e = d;
        d = p / q;
      } else {
        d = xm;
        e = d;
      }
    } else {
      d = xm;
      e = d;
    }
    a = b;
    fa = fb;
    b += std::fabs(d) > tol1 ? d : std::copysign(tol1, xm);
    state = 1;
  }
};

}  // namespace

// SingleFitter::compute_uncertainty (fitting.rs:480-568) for S spectra on
// one dispersion and continuum fitter (compute_uncertainty_bulk,
// lib.rs:1570-1600): per label i and side, the distance from `labels` to
// where chi2 crosses chi2_best * (1 + sqrt(2 / n)), n = 4 R (l_last -
// l_first) / (l_first + l_last), searched in units of the search radius
// within the SingleBounds(grid, (0, 1e4), (-1e3, 1e3)) clamp.  All open
// searches of all spectra evaluate together in one batched chi2 per round.
int pasta_compute_uncertainty(const pasta_grid *gc, const pasta_dispersion *d, const pasta_continuum *c, int64_t S,
                              const float *flux, const float *var, int64_t n, double spec_res, const double *labels,
                              const double *search_radius, double *out, int32_t *bound_status,
                              int32_t *star_status) {
  return guard([&] {
    pasta_grid *g = const_cast<pasta_grid *>(gc);
    if (!d || !c || !flux || !var || !labels || !out || !bound_status || !star_status)
      fail(PASTA_E_ARG, "dispersion, continuum, data, labels and outputs are required");
    if (S < 0) fail(PASTA_E_ARG, "negative spectrum count");
    if (S == 0) return;
    check_disp_grid(g, d);
    if (n != (int64_t)d->wl.size()) fail(PASTA_E_ARG, "Observed spectrum and target dispersion must have the same length");
    if (c->kind != PASTA_CONT_CONSTANT && c->n != n)
      fail(PASTA_E_ARG, "Length of observed and continuum spectrum are different %lld, %lld", (long long)n,
           (long long)c->n);
    double sr0[5] = {2000.0, 0.3, 0.3, 40.0, 40.0};
    if (search_radius) std::copy(search_radius, search_radius + 5, sr0);
    Ctx &C = ctx();
    cudaStream_t s = C.stream;
    std::lock_guard<std::mutex> lk(g->mu);
    // one device star per spectrum
    std::vector<StarInput> in(S);
    for (int64_t i = 0; i < S; i++) in[i] = StarInput{d, c, nullptr, flux + (size_t)i * n, var + (size_t)i * n, n, 0};
    StarSet ss;
    ss.build(in);
    EvalArgs a;
    a.stars = ss.dstars.p;
    a.need_chi2 = 1;
    star_kinds(ss.h, a);
    // the evaluation buffers hold the largest round: two points per search
    const int64_t Emax = S * 20;
    DBuf<double> dl, dc;
    DBuf<int> de, dst;
    dl.alloc((size_t)Emax * 5);
    dc.alloc(Emax);
    de.alloc(Emax);
    dst.alloc(Emax);
    ensure_workspace(g, std::min<int64_t>(Emax, 1 << 16), a.max_nobs);
    std::vector<double> hl;
    std::vector<int> hs;
    std::vector<double> hc;
    std::vector<int> hst;
    // chi2 of the labels in hl (5 per point) for the stars in hs
    auto evaluate = [&]() {
      const int64_t E = (int64_t)hs.size();
      hc.assign(E, 0.0);
      hst.assign(E, 0);
      if (E == 0) return;
      double vmax = 0.0;
      for (int64_t k = 0; k < E; k++) vmax = std::max(vmax, hl[(size_t)k * 5 + 3]);
      CK(cudaMemcpyAsync(dl.p, hl.data(), (size_t)E * 5 * sizeof(double), cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(de.p, hs.data(), (size_t)E * sizeof(int), cudaMemcpyHostToDevice, s));
      a.labels = dl.p;
      a.eval_star = de.p;
      a.E = E;
      a.cost = dc.p;
      a.status = dst.p;
      a.max_m = width_upper_bound(g, vmax);
      run_evals(g, a, s);
      CK(cudaMemcpyAsync(hc.data(), dc.p, (size_t)E * sizeof(double), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(hst.data(), dst.p, (size_t)E * sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
    };
    // best chi2 at the given labels (an error there fails the whole spectrum)
    hl.assign(labels, labels + (size_t)S * 5);
    hs.resize(S);
    for (int64_t i = 0; i < S; i++) hs[i] = (int)i;
    evaluate();
    const double l0 = d->wl.front(), l1 = d->wl.back();
    const double neff = 4.0 * spec_res * (l1 - l0) / (l0 + l1);
    std::vector<double> target(S), radius((size_t)S * 5);
    for (int64_t i = 0; i < S; i++) {
      star_status[i] = hst[i];
      target[i] = hc[i] * (1.0 + std::sqrt(2.0 / neff));
      const double *L = labels + (size_t)i * 5;
      double *r = &radius[(size_t)i * 5];
      for (int k = 0; k < 5; k++) r[k] = sr0[k];
      r[0] *= L[0];
      r[3] = std::max(L[3] * r[3], 100.0);
    }
    // bounds of every search; outer limits SingleBounds(grid, (0, 1e4), (-1e3, 1e3))
    PsoParams lim{};
    lim.vs_lo = 0.0; lim.vs_hi = 1e4;
    lim.rv_lo = -1e3; lim.rv_hi = 1e3;
    const int64_t NS = S * 10;  // search q = (spectrum, label, side): q = (i * 5 + k) * 2 + right
    std::vector<BrentSearch> bs(NS);
    for (int64_t q = 0; q < NS; q++) {
      const int64_t i = q / 10;
      const int k = (int)(q / 2 % 5), right = (int)(q % 2);
      BrentSearch &B = bs[q];
      if (star_status[i]) {
        B.state = 3;
        B.status = star_status[i];
        continue;
      }
      double bl[5];
      std::copy(labels + (size_t)i * 5, labels + (size_t)i * 5 + 5, bl);
      const double r = radius[(size_t)i * 5 + k];
      bl[k] += right ? r : -r;
      double bound;
      const int st = pso_clamp_1d(g->hg, lim, bl, k, bound);
      if (st) {
        B.state = 3;
        B.status = st;
        continue;
      }
      const double resc = (bound - labels[(size_t)i * 5 + k]) / r;
      if (right) { B.a = 0.0; B.b = std::min(resc, 1.0); }
      else { B.a = resc; B.b = 0.0; }
    }
    // rounds: every open search contributes its pending points
    std::vector<int64_t> owner;
    std::vector<int> which;
    for (int round = 0; round < 1000; round++) {
      hl.clear(); hs.clear(); owner.clear(); which.clear();
      auto push = [&](int64_t q, double param, int w) {
        const int64_t i = q / 10;
        const int k = (int)(q / 2 % 5);
        for (int t = 0; t < 5; t++) hl.push_back(labels[(size_t)i * 5 + t]);
        hl[hl.size() - 5 + k] += param * radius[(size_t)i * 5 + k];
        hs.push_back((int)i);
        owner.push_back(q);
        which.push_back(w);
      };
      for (int64_t q = 0; q < NS; q++) {
        if (bs[q].state == 0) { push(q, bs[q].a, 0); push(q, bs[q].b, 1); }
        else if (bs[q].state == 1) push(q, bs[q].b, 1);
      }
      if (hs.empty()) break;
      evaluate();
      for (size_t t = 0; t < owner.size(); t++) {
        BrentSearch &B = bs[owner[t]];
        if (B.state == 3) continue;
        if (hst[t]) {
          B.state = 3;
          B.status = hst[t];
          continue;
        }
        const double f = hc[t] - target[owner[t] / 10];
        if (which[t] == 0) B.fa = f;
        else B.fb = f;
      }
      for (int64_t q = 0; q < NS; q++) {
        BrentSearch &B = bs[q];
        if (B.state == 0) {
          if (B.fa * B.fb > 0.0) {  // argmin: f(min) and f(max) must have different signs
            B.state = 3;
            B.status = PASTA_E_ARG;
            continue;
          }
          B.c = B.b;
          B.fc = B.fb;
          B.d = B.b - B.a;
          B.e = B.d;
          B.advance();
        } else if (B.state == 1) {
          B.advance();
        }
      }
    }
    for (int64_t q = 0; q < NS; q++) {
      const int64_t i = q / 10;
      const int k = (int)(q / 2 % 5), right = (int)(q % 2);
      const BrentSearch &B = bs[q];
      const bool ok = B.state == 2;
      const double r = radius[(size_t)i * 5 + k];
      out[q] = ok ? (right ? B.b * r : -B.b * r) : NAN;
      bound_status[q] = ok ? 0 : (B.status ? B.status : PASTA_E_INTERNAL);
    }
  });
}

// ----------------------------------------------------- batch sessions
struct pasta_batch {
  Batch B;
};

int pasta_batch_create(const pasta_grid *gc, int64_t S, const pasta_dispersion *const *d,
                       const pasta_continuum *const *c, const pasta_pso_settings *settings, const float *const *flux,
                       const float *const *var, const int64_t *n, const uint64_t *seeds, pasta_batch **out) {
  return guard([&] {
    pasta_grid *g = const_cast<pasta_grid *>(gc);
    if (S < 1 || !out) fail(PASTA_E_ARG, "invalid batch arguments");
    std::vector<StarInput> in(S);
    for (int64_t i = 0; i < S; i++) in[i] = StarInput{d[i], c[i], &settings[i], flux[i], var[i], n[i], seeds[i]};
    for (auto &s : in) validate_star(g, s);
    std::lock_guard<std::mutex> lk(g->mu);
    std::unique_ptr<pasta_batch> b(new pasta_batch());
    batch_init(b->B, g, in);
    *out = b.release();
  });
}

int pasta_batch_step(pasta_batch *b, int steps, double *device_ms) {
  return guard([&] {
    std::lock_guard<std::mutex> lk(b->B.g->mu);
    double ms = batch_steps(b->B, steps, nullptr);
    if (device_ms) *device_ms = ms;
  });
}

int pasta_batch_profile_step(pasta_batch *b, double *out12) {
  return guard([&] {
    std::lock_guard<std::mutex> lk(b->B.g->mu);
    batch_profile_step(b->B, out12);
  });
}

int pasta_batch_info(const pasta_batch *b, int64_t *out6) {
  return guard([&] {
    const Batch &B = b->B;
    out6[0] = B.S;
    out6[1] = B.Pmax;
    out6[2] = (int64_t)B.S * B.Pmax;
    out6[3] = B.iters;
    out6[4] = B.steps_done;
    out6[5] = B.kernels_per_step;
  });
}

int pasta_batch_finish(pasta_batch *b, pasta_fit_result *results, float *const *params) {
  return guard([&] {
    std::lock_guard<std::mutex> lk(b->B.g->mu);
    std::vector<std::vector<float>> pv;
    batch_finish(b->B, results, pv);
    for (int i = 0; i < b->B.S; i++)
      if (params && params[i]) std::copy(pv[i].begin(), pv[i].end(), params[i]);
  });
}

int pasta_batch_destroy(pasta_batch *b) {
  return guard([&] { delete b; });
}

// ------------------------------------------------------------ serving
int pasta_server_create(const pasta_grid *gc, int max_slots, int64_t hbm_budget_bytes, pasta_server **out) {
  return guard([&] {
    if (max_slots < 1) fail(PASTA_E_ARG, "max_slots must be >= 1");
    ctx();
    std::unique_ptr<pasta_server> sv(new pasta_server());
    sv->g = const_cast<pasta_grid *>(gc);
    sv->slots = max_slots;
    if (hbm_budget_bytes > 0) {
      sv->budget = hbm_budget_bytes;
    } else {
      // default: the device memory the evaluation workspace may take (40% of
      // the device, or PASTA_WORKSPACE_BYTES), so the admitted requests'
      // evaluations fit one workspace and a step is never split in sub-batches
      size_t fr = 0, tot = 0;
      CK(cudaMemGetInfo(&fr, &tot));
      sv->budget = (int64_t)(0.4 * (double)tot);
      if (const char *e = getenv("PASTA_WORKSPACE_BYTES")) sv->budget = atoll(e);
    }
    sv->slot_req.resize(max_slots);
    sv->slot_flux.resize(max_slots);
    sv->slot_var.resize(max_slots);
    sv->hstars.assign(max_slots, DevStar{});
    sv->pp.assign(max_slots, PsoParams{});
    *out = sv.release();
  });
}

int pasta_server_submit(pasta_server *sv, const pasta_dispersion *d, const pasta_continuum *c,
                        const pasta_pso_settings *settings, const float *flux, const float *var, int64_t n,
                        uint64_t seed, int64_t *request_id) {
  return guard([&] {
    StarInput si{d, c, settings, flux, var, n, seed};
    validate_star(sv->g, si);
    make_pso_params(sv->g, *settings);
    std::lock_guard<std::mutex> lk(sv->mu);
    pasta_server::Req r;
    r.id = sv->next_id++;
    r.d = d;
    r.c = c;
    r.st = *settings;
    r.flux.assign(flux, flux + n);
    r.var.assign(var, var + n);
    r.t_submit = now_s();
    r.seed = seed;
    // device memory the request holds while it runs: its spectrum and swarm
    // state, and the evaluation workspace of its particles
    const int64_t stride = std::max<int64_t>(sv->g->stride, (n + 63) / 64 * 64);
    r.bytes = n * 8 + (int64_t)settings->num_particles *
                          (200 + workspace_bytes_per_eval(stride, bnd_stride_for((int)sv->g->npx)));
    sv->queue.push_back(std::move(r));
    if (request_id) *request_id = sv->queue.back().id;
  });
}

namespace {

void server_rebuild(pasta_server *sv, int Pmax) {
  // (re)allocate slot swarm arrays for a larger particle count; only when empty
  sv->Pmax = Pmax;
  sv->W.alloc(sv->slots, Pmax);
  std::vector<int> ident(sv->slots);
  for (int i = 0; i < sv->slots; i++) ident[i] = i;
  sv->rf_star.upload(ident);
  sv->rf_flag.alloc(sv->slots);
  CK(cudaMemset(sv->rf_flag.p, 0, sv->slots * sizeof(int)));
  sv->rf_status.alloc(sv->slots);
  sv->rf_cost.alloc(sv->slots);
  sv->rf_params.alloc((size_t)sv->slots * SERVER_REFIT_STRIDE);
  std::vector<int> z(sv->slots, 0), done1(sv->slots, 1), im(sv->slots, -1);
  CK(cudaMemcpy(sv->W.active.p, z.data(), z.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sv->W.done.p, done1.data(), z.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sv->W.status.p, z.data(), z.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(sv->W.iter.p, im.data(), z.size() * sizeof(int), cudaMemcpyHostToDevice));
  sv->pp.assign(sv->slots, PsoParams{});
  sv->W.params.upload(sv->pp);
  sv->dstars.upload(sv->hstars);
  if (sv->exec) { cudaGraphExecDestroy(sv->exec); sv->exec = nullptr; }
  if (sv->graph) { cudaGraphDestroy(sv->graph); sv->graph = nullptr; }
}

}  // namespace

int pasta_server_step(pasta_server *sv) {
  int active_after = 0;
  int rc = guard([&] {
    const double t0 = now_s();
    std::lock_guard<std::mutex> lk(sv->mu);
    pasta_grid *g = sv->g;
    std::lock_guard<std::mutex> lg(g->mu);
    Ctx &C = ctx();
    cudaStream_t s = C.stream;
    bool any_active = false;
    for (int i = 0; i < sv->slots; i++) any_active |= (bool)sv->slot_req[i];
    // grow the particle capacity when the device loop is idle
    int needP = sv->Pmax;
    for (auto &r : sv->queue) needP = std::max(needP, r.st.num_particles);
    if (needP != sv->Pmax && !any_active) server_rebuild(sv, needP);
    // admit queued requests into free slots within the HBM budget: the
    // slot state is uploaded on the stream (pageable sources are staged
    // when the copies are issued)
    std::vector<int> admitted;
    auto admit = [&]() {
      for (int i = 0; i < sv->slots && !sv->queue.empty(); i++) {
        if (sv->slot_req[i]) continue;
        auto &r = sv->queue.front();
        if (r.st.num_particles > sv->Pmax) break;
        // a request that alone exceeds the budget still runs when nothing else does
        if (sv->used + r.bytes > sv->budget && sv->used > 0) break;
        std::unique_ptr<pasta_server::Req> rp(new pasta_server::Req(std::move(r)));
        sv->queue.pop_front();
        sv->used += rp->bytes;
        // the slot's spectrum buffers are kept between requests and grow only
        // for a longer spectrum (no allocation or free in the steady state)
        const size_t nobs = rp->flux.size();
        if (!sv->slot_flux[i] || sv->slot_flux[i]->n < nobs) {
          sv->slot_flux[i].reset(new DBuf<float>());
          sv->slot_var[i].reset(new DBuf<float>());
          sv->slot_flux[i]->alloc(nobs);
          sv->slot_var[i]->alloc(nobs);
        }
        CK(cudaMemcpyAsync(sv->slot_flux[i]->p, rp->flux.data(), nobs * sizeof(float), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(sv->slot_var[i]->p, rp->var.data(), nobs * sizeof(float), cudaMemcpyHostToDevice, s));
        sv->hstars[i] = make_star(rp->d, rp->c, sv->slot_flux[i]->p, sv->slot_var[i]->p, (int64_t)nobs);
        PsoParams P = make_pso_params(g, rp->st);
        sv->pp[i] = P;
        sv->max_m = std::max(sv->max_m, width_upper_bound(g, P.mx[3]));
        std::vector<double> x((size_t)sv->Pmax * 5, 0.0), v((size_t)sv->Pmax * 5, 0.0);
        int st = init_swarm_host(g, P, rp->seed, x.data(), v.data());
        const size_t base = (size_t)i * sv->Pmax * 5;
        CK(cudaMemcpyAsync(sv->W.x.p + base, x.data(), x.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(sv->W.v.p + base, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        int one = 1, zero = 0, m1 = -1, done0 = st ? 1 : 0;
        uint64_t sd = rp->seed;
        CK(cudaMemcpyAsync(sv->W.active.p + i, &one, sizeof(int), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(sv->W.done.p + i, &done0, sizeof(int), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(sv->W.status.p + i, st ? &st : &zero, sizeof(int), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(sv->W.iter.p + i, &m1, sizeof(int), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(sv->W.seed.p + i, &sd, sizeof(uint64_t), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(sv->W.params.p + i, &P, sizeof(PsoParams), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(sv->dstars.p + i, &sv->hstars[i], sizeof(DevStar), cudaMemcpyHostToDevice, s));
        // pageable sources are staged when the copies are issued; the step's
        // launches follow on the same stream
        sv->slot_req[i] = std::move(rp);
        admitted.push_back(i);
      }
    };
    // an idle server admits before its launch; a busy one after it, so the
    // host work overlaps the step on the device and the new slots join the
    // next step
    if (!any_active) admit();
    bool any = false;
    for (int i = 0; i < sv->slots; i++) any |= (bool)sv->slot_req[i];
    if (!any) return;
    const int64_t E = (int64_t)sv->slots * sv->Pmax;
    Swarm sw = sv->W.view();
    sw.refit = sv->rf_flag.p;
    EvalArgs a;
    a.stars = sv->dstars.p;
    a.labels = sv->W.labels.p;
    a.eval_star = sv->W.eval_star.p;
    a.eval_active = sv->W.eval_active.p;
    a.E = E;
    a.cost = sv->W.ecost.p;
    a.status = sv->W.estatus.p;
    a.need_chi2 = 1;
    a.max_m = sv->max_m;
    {
      std::vector<DevStar> occ;
      for (int i = 0; i < sv->slots; i++)
        if (sv->slot_req[i]) occ.push_back(sv->hstars[i]);
      star_kinds(occ, a);
      a.chunk_p1_mask |= sv->graph_mask;  // keep what the captured graph already covers
      if (sv->graph_other) a.other_cont = 1;
      a.max_hg = std::max(a.max_hg, sv->graph_hg);
      a.max_chunks = std::max(a.max_chunks, sv->graph_chunks);
      a.lin_kp_mask |= sv->graph_lin;
      a.lin_group = sv->Pmax <= 128 ? sv->Pmax : 0;
      a.star_len = sv->Pmax;
    }
    ensure_workspace(g, E, a.max_nobs);
    const bool grown = sv->graph_max_m < sv->max_m || (a.chunk_p1_mask & ~sv->graph_mask) ||
                       (a.other_cont && !sv->graph_other) || a.max_hg > sv->graph_hg ||
                       a.max_chunks > sv->graph_chunks || (a.lin_kp_mask & ~sv->graph_lin);
    if (sv->exec && (grown || sv->graph_gen != g->ws.gen)) {
      // a wider kernel or a new continuum kind was admitted, or the workspace moved
      cudaGraphExecDestroy(sv->exec);
      cudaGraphDestroy(sv->graph);
      sv->exec = nullptr;
      sv->graph = nullptr;
    }
    if (!sv->exec) {
      sv->graph_max_m = sv->max_m;
      sv->graph_gen = g->ws.gen;
      sv->graph_mask = a.chunk_p1_mask;
      sv->graph_other = a.other_cont;
      sv->graph_hg = a.max_hg;
      sv->graph_chunks = a.max_chunks;
      sv->graph_lin = a.lin_kp_mask;
      const int64_t k0 = kernel_launches();
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      launch_pso_update(g->d, sw, s);
      run_evals(g, a, s);
      launch_pso_best(sw, sv->W.ecost.p, sv->W.estatus.p, s);
      // final refit (fitting.rs:436-440) of the swarms that finished in this
      // step: chi2 at the best label with the continuum parameters written
      EvalArgs r = a;
      r.labels = sv->W.gx.p;
      r.eval_star = sv->rf_star.p;
      r.eval_active = sv->rf_flag.p;
      r.E = sv->slots;
      r.cost = sv->rf_cost.p;
      r.status = sv->rf_status.p;
      r.params = sv->rf_params.p;
      r.param_stride = SERVER_REFIT_STRIDE;
      run_evals(g, r, s);
      CK(cudaStreamEndCapture(s, &sv->graph));
      sv->graph_kernels = kernel_launches() - k0;
      count_launch(-(int)sv->graph_kernels);  // counted again at every replay
      CK(cudaGraphInstantiate(&sv->exec, sv->graph, 0));
    }
    const double t1 = now_s();
    CK(cudaGraphLaunch(sv->exec, s));
    count_launch((int)sv->graph_kernels);
    for (int i = 0; i < sv->slots; i++)
      if (sv->slot_req[i]) sv->evals_total += sv->slot_req[i]->st.num_particles;
    sv->steps_total++;
    if (any_active) admit();
    // the step's flags and every slot's best (small) in one wait
    std::vector<int> done(sv->slots), status(sv->slots);
    std::vector<double> gx((size_t)sv->slots * 5), gc(sv->slots);
    CK(cudaMemcpyAsync(done.data(), sv->W.done.p, sv->slots * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(status.data(), sv->W.status.p, sv->slots * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(gx.data(), sv->W.gx.p, gx.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(gc.data(), sv->W.gcost.p, gc.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    const double t2 = now_s();
    sv->t_before += t1 - t0;
    sv->t_step += t2 - t1;
    // retire finished requests: final refit for their params, free the slot
    std::vector<int> fin;
    for (int i = 0; i < sv->slots; i++)
      if (sv->slot_req[i] && done[i]) fin.push_back(i);
    if (!fin.empty()) {
      // the step's graph refitted every swarm that finished successfully
      // (chi2 at its best label with the continuum parameters written)
      const double tr0 = now_s();
      std::vector<std::vector<double>> rows(fin.size());
      std::vector<int> rst(fin.size(), 0);
      for (size_t q = 0; q < fin.size(); q++) {
        const int i = fin[q];
        if (status[i] != 0) continue;
        rows[q].resize(device_param_stride(sv->slot_req[i]->c));
        CK(cudaMemcpyAsync(rows[q].data(), sv->rf_params.p + (size_t)i * SERVER_REFIT_STRIDE,
                           rows[q].size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&rst[q], sv->rf_status.p + i, sizeof(int), cudaMemcpyDeviceToHost, s));
      }
      CK(cudaStreamSynchronize(s));
      sv->t_refit += now_s() - tr0;
      const double tnow = now_s();
      for (size_t q = 0; q < fin.size(); q++) {
        const int i = fin[q];
        auto &r = *sv->slot_req[i];
        pasta_server::Done dn;
        dn.id = r.id;
        std::memset(&dn.r, 0, sizeof dn.r);
        for (int d = 0; d < 5; d++) dn.r.label[d] = gx[(size_t)i * 5 + d];
        dn.r.chi2 = gc[i];
        dn.r.iterations = r.st.max_iters;
        dn.r.status = status[i];
        dn.r.time = tnow - r.t_submit;
        if (status[i] == 0 && rst[q] == 0) dn.params = params_from_device(r.c, rows[q].data());
        dn.r.n_params = (int)dn.params.size();
        sv->done.push_back(std::move(dn));
        sv->used -= r.bytes;
        sv->slot_req[i].reset();
        int zero = 0;
        CK(cudaMemcpyAsync(sv->W.active.p + i, &zero, sizeof(int), cudaMemcpyHostToDevice, s));
      }
    }
    for (int i = 0; i < sv->slots; i++) active_after += sv->slot_req[i] ? 1 : 0;
    sv->t_after += now_s() - t2;
  });
  return rc ? rc : active_after;
}

// `steps` server steps back to back, with the time between CUDA events on
// the library's stream around them (host work between the launches, such as
// admissions and retirements, is inside the interval).
int pasta_server_run(pasta_server *sv, int steps, double *device_ms) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = guard([&] {
    if (steps < 0) fail(PASTA_E_ARG, "steps must be >= 0");
    cudaStream_t s = ctx().stream;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, s));
  });
  if (rc) return rc;
  for (int k = 0; k < steps && !rc; k++) {
    const int r = pasta_server_step(sv);
    if (r < 0) rc = r;
  }
  const int rc2 = guard([&] {
    cudaStream_t s = ctx().stream;
    CK(cudaEventRecord(e1, s));
    CK(cudaEventSynchronize(e1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    if (device_ms) *device_ms = ms;
  });
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc ? rc : rc2;
}

int pasta_server_stats(const pasta_server *sv, int64_t *out7) {
  return guard([&] {
    if (!out7) fail(PASTA_E_ARG, "output required");
    int64_t *out6 = out7;
    out6[0] = sv->evals_total;
    out6[1] = sv->steps_total;
    out6[2] = sv->Pmax;
    out6[3] = (int64_t)(sv->t_before * 1e6);
    out6[4] = (int64_t)(sv->t_step * 1e6);
    out6[5] = (int64_t)(sv->t_after * 1e6);
    out6[6] = (int64_t)(sv->t_refit * 1e6);
  });
}

int pasta_server_poll(pasta_server *sv, int64_t *ids, pasta_fit_result *results, float *params, int64_t pstride,
                      int max, int *n_out) {
  return guard([&] {
    std::lock_guard<std::mutex> lk(sv->mu);
    int k = 0;
    while (k < max && !sv->done.empty()) {
      auto &d = sv->done.front();
      if (ids) ids[k] = d.id;
      if (results) results[k] = d.r;
      if (params) std::copy(d.params.begin(), d.params.begin() + std::min<int64_t>(pstride, d.params.size()),
                            params + (size_t)k * pstride);
      sv->done.pop_front();
      k++;
    }
    *n_out = k;
  });
}

int pasta_server_memory(const pasta_server *sv, int64_t *budget, int64_t *used) {
  return guard([&] {
    pasta_server *s = const_cast<pasta_server *>(sv);
    std::lock_guard<std::mutex> lk(s->mu);
    if (budget) *budget = s->budget;
    if (used) *used = s->used;
  });
}

int pasta_server_pending(const pasta_server *sv, int64_t *queued, int64_t *active, int64_t *done) {
  return guard([&] {
    pasta_server *s = const_cast<pasta_server *>(sv);
    std::lock_guard<std::mutex> lk(s->mu);
    int64_t a = 0;
    for (auto &r : s->slot_req) a += r ? 1 : 0;
    if (queued) *queued = (int64_t)s->queue.size();
    if (active) *active = a;
    if (done) *done = (int64_t)s->done.size();
  });
}

int pasta_server_destroy(pasta_server *sv) {
  return guard([&] {
    if (!sv) return;
    ctx();
    CK(cudaDeviceSynchronize());
    delete sv;
  });
}

}  // extern "C"

// ------------------------------------------------------------------------
// Read-only views of the handles for the allocation-free entry point
// (noalloc.cu): the grid's device description and one assembled star.
// Nothing is allocated or copied.
namespace pb {
int internal_eval_view(const pasta_grid *g, const pasta_dispersion *d, const pasta_continuum *c, const float *flux,
                       const float *var, int64_t n, DevGrid *grid, int64_t *stride, DevStar *star, int *device,
                       std::string *err) {
  try {
    if (!g || !d || !c) fail(PASTA_E_ARG, "grid, dispersion and continuum handles are required");
    StarInput si{d, c, nullptr, flux, var, n, 0};
    validate_star(g, si);
    *grid = g->d;
    *stride = g->stride;
    *star = make_star(d, c, flux, var, n);
    *device = g->dev;
    return PASTA_OK;
  } catch (const PErr &e) {
    *err = e.what();
    return e.code;
  }
}
}  // namespace pb

namespace pb {
// lets noalloc.cu report through pasta_last_error()
void internal_set_last_error(const std::string &msg) { g_last_error = msg; }
}  // namespace pb
