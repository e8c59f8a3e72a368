// kernels.cu -- the bandwidth and FFT kernels of the per-particle hot path.
//
// Buffer protocol per evaluation e (rows of `stride` floats):
//   k_interp writes the interpolated spectrum to A.
//   k_rot writes the rotation-broadened spectrum to B (skipped when the
//     rotation is the identity; then A holds it).
//   k_gauss writes the instrument-broadened spectrum to the other buffer.
//   k_chi2 / k_resample_out read the final buffer (final_row()).
#include <cuda_runtime.h>

#include "common.cuh"
#include "fft.cuh"
#include "kernels.h"

namespace pb {

__device__ __forceinline__ const float *rot_row(const EvalBatch &b, const EvalPrep &P, int e) {
  return (P.m > 1 ? b.bufB : b.bufA) + (size_t)e * b.stride;
}
__device__ __forceinline__ const float *final_row(const EvalBatch &b, const EvalPrep &P, int disp_kind, int e) {
  const bool rot_in_b = P.m > 1;
  const bool in_b = disp_kind == DISP_NONE ? rot_in_b : !rot_in_b;
  return (in_b ? b.bufB : b.bufA) + (size_t)e * b.stride;
}

// ---------------------------------------------------------------- interp
// flux[px] = sum_n w_n * (u16_n[px] * factor_n) over the 64 neighbours
// (interpolate.rs:954-981), 8 pixels per thread from one 128-bit load per
// neighbour.  Grid: x = evaluation, y = 2048-pixel tile, so CTAs that run
// together read the same tile of the resident grid (particles of one star
// share neighbours, which then hit in L2).
constexpr int IT_T = 256, IT_TILE = IT_T * 8;

__global__ void __launch_bounds__(IT_T) k_interp(DevGrid G, EvalBatch b) {
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  if (P.status) return;
  const int t0 = blockIdx.y * IT_TILE;
  const int ilo = P.i_lo, ihi = P.i_hi;
  if (t0 >= ihi || t0 + IT_TILE <= ilo) return;
  __shared__ const uint16_t *rows[64];
  __shared__ float ws[64], fs[64];
  if (threadIdx.x < 64) {
    const int c = P.cols[threadIdx.x];
    rows[threadIdx.x] = c >= 0 ? G.spectra + (size_t)c * G.stride : nullptr;
    ws[threadIdx.x] = P.w[threadIdx.x];
    fs[threadIdx.x] = c >= 0 ? G.factor[c] : 0.0f;
  }
  __syncthreads();
  const int px = t0 + threadIdx.x * 8;
  if (px < ilo || px >= ihi) return;
  float acc[8];
#pragma unroll
  for (int k = 0; k < 8; k++) acc[k] = 0.0f;
  const bool tail = px + 8 > G.tail_start;
#pragma unroll 8
  for (int n = 0; n < 64; n++) {
    const uint16_t *r = rows[n];
    if (r == nullptr) continue;
    const uint4 q = __ldg(reinterpret_cast<const uint4 *>(r + px));
    const float wn = ws[n], fn = fs[n];
    const uint32_t u[4] = {q.x, q.y, q.z, q.w};
    if (!tail) {
#pragma unroll
      for (int k = 0; k < 4; k++) {
        acc[2 * k] = fmaf(wn, __fmul_rn((float)(u[k] & 0xFFFFu), fn), acc[2 * k]);
        acc[2 * k + 1] = fmaf(wn, __fmul_rn((float)(u[k] >> 16), fn), acc[2 * k + 1]);
      }
    } else {
      // the last npx % 128 pixels carry an extra 1/65535 (interpolate.rs:978)
#pragma unroll
      for (int k = 0; k < 8; k++) {
        const float x = (float)((u[k >> 1] >> (16 * (k & 1))) & 0xFFFFu);
        const float v = px + k >= G.tail_start ? __fmul_rn(__fdiv_rn(x, 65535.0f), fn) : __fmul_rn(x, fn);
        acc[k] = fmaf(wn, v, acc[k]);
      }
    }
  }
  float4 *out = reinterpret_cast<float4 *>(b.bufA + (size_t)e * b.stride + px);
  out[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
  out[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
}

void launch_interp(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0) return;
  dim3 grid(b.E, (G.npx + IT_TILE - 1) / IT_TILE);
  k_interp<<<grid, IT_T, 0, s>>>(G, b);
  count_launch();
}

// ------------------------------------------------------------ rotation
// Overlap-save convolution with the rotation kernel (the reference uses
// overlap-add, convolve_rv.rs:121-157; both are the same linear
// convolution).  Two real blocks of one evaluation ride in the real and
// imaginary parts of one complex 2048-point FFT; the kernel is real, so the
// two products separate again after the inverse transform.  Block b of an
// evaluation produces rotation outputs [g_lo + b V, g_lo + (b+1) V) with
// V = 2048 - (m - 1).  Persistent CTAs walk (evaluation, block pair) items.
__global__ void __launch_bounds__(FFT_T) k_rot(DevGrid G, EvalBatch b, const float2 *__restrict__ tw) {
  __shared__ float re[FFT_SM], im[FFT_SM];
  const long long total = (long long)b.E * b.max_pairs;
  for (long long item = blockIdx.x; item < total; item += gridDim.x) {
    const int e = (int)(item / b.max_pairs), pair = (int)(item % b.max_pairs);
    const EvalPrep &P = b.prep[e];
    const int m = P.m, nblk = P.nblk;
    if (P.status || m <= 1 || 2 * pair >= nblk) continue;
    const int V = FFTN - (m - 1), hw = (m - 1) / 2;
    const int s0 = P.g_lo + 2 * pair * V, s1 = s0 + V;
    const bool has1 = 2 * pair + 1 < nblk;
    const int ilo = P.i_lo, ihi = P.i_hi, ghi = P.g_hi;
    const float *x = b.bufA + (size_t)e * b.stride;
    for (int t = threadIdx.x; t < FFTN; t += FFT_T) {
      const int j0 = s0 - hw + t, j1 = s1 - hw + t;
      re[pidx(t)] = (j0 >= ilo && j0 < ihi) ? x[j0] : 0.0f;
      im[pidx(t)] = (has1 && j1 >= ilo && j1 < ihi) ? x[j1] : 0.0f;
    }
    __syncthreads();
    fft2048<false>(re, im, tw);
    const float2 *H = b.H + (size_t)e * 1025;
    for (int k = threadIdx.x; k < FFTN; k += FFT_T) {
      float2 h = k <= 1024 ? H[k] : H[FFTN - k];
      if (k > 1024) h.y = -h.y;
      const int a = pidx(k);
      const cf z = cmul(cf{re[a], im[a]}, cf{h.x, h.y});
      re[a] = z.x;
      im[a] = z.y;
    }
    __syncthreads();
    fft2048<true>(re, im, tw);
    float *y = b.bufB + (size_t)e * b.stride;
    const float sc = 1.0f / 2048.0f;
    for (int t = m - 1 + threadIdx.x; t < FFTN; t += FFT_T) {
      const int i0 = s0 + t - (m - 1);
      if (i0 < ghi) y[i0] = re[pidx(t)] * sc;
      if (has1) {
        const int i1 = s1 + t - (m - 1);
        if (i1 < ghi) y[i1] = im[pidx(t)] * sc;
      }
    }
    __syncthreads();
  }
}

static int g_num_sms = 0;
static int num_sms() {
  if (!g_num_sms) {
    int dev;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

void launch_rot(const DevGrid &G, const EvalBatch &b, const float2 *tw, cudaStream_t s) {
  if (b.E <= 0 || b.max_pairs <= 0) return;
  long long total = (long long)b.E * b.max_pairs;
  long long grid = (long long)num_sms() * 8;
  if (grid > total) grid = total;
  k_rot<<<(unsigned)grid, FFT_T, 0, s>>>(G, b, tw);
  count_launch();
}

// ----------------------------------------------------- instrument profile
// FixedTargetDispersionLogSpace: one Gaussian, output i = sum_k g[k]
// r[i + h - k] with r zero outside the grid (convolve_rv.rs:207-210).
// Per-pixel kernels (VariableTargetDispersion / FixedTargetDispersionNonLog):
// output i = kernel_i . r[i-h .. i+h], pixels within h of either end pass
// through (convolve_rv.rs:213-233, 414-430).
constexpr int GT = 256, G_TILE = 1024, G_HMAX = 256;

__device__ __forceinline__ void gauss_tile(const DevStar &st, const float *src, float *dst, int N, int t0, int t1,
                                           int glo, int ghi, float *sbuf) {
  const int w = st.gw, h = (w - 1) / 2;
  const int base = t0 - h;
  for (int j = threadIdx.x; j < (t1 - t0) + 2 * h; j += blockDim.x) {
    const int g = base + j;
    sbuf[j] = (g >= glo && g < ghi) ? src[g] : 0.0f;
  }
  __syncthreads();
  for (int i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
    float acc = 0.0f;
    if (st.disp_kind == DISP_FIXED) {
      const float *g = st.gk;
      for (int k = 0; k < w; k++) acc = fmaf(__ldg(&g[k]), sbuf[i + h - k - base], acc);
    } else {
      if (i < h || i >= N - h) {
        acc = sbuf[i - base];
      } else {
        const float *kk = st.gk + (size_t)i * w;
        for (int t = 0; t < w; t++) acc = fmaf(__ldg(&kk[t]), sbuf[i - h + t - base], acc);
      }
    }
    dst[i] = acc;
  }
}

__global__ void __launch_bounds__(GT) k_gauss(DevGrid G, EvalBatch b) {
  __shared__ float sbuf[G_TILE + 2 * G_HMAX];
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  if (P.status) return;
  const DevStar &st = b.stars[P.star];
  if (st.disp_kind == DISP_NONE) return;
  const int t0 = max(blockIdx.y * G_TILE, P.o_lo), t1 = min((int)(blockIdx.y + 1) * G_TILE, P.o_hi);
  if (t0 >= t1) return;
  const bool rot_in_b = P.m > 1;
  const float *src = (rot_in_b ? b.bufB : b.bufA) + (size_t)e * b.stride;
  float *dst = (rot_in_b ? b.bufA : b.bufB) + (size_t)e * b.stride;
  gauss_tile(st, src, dst, G.npx, t0, t1, P.g_lo, P.g_hi, sbuf);
}

void launch_gauss(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0) return;
  dim3 grid(b.E, (G.npx + G_TILE - 1) / G_TILE);
  k_gauss<<<grid, GT, 0, s>>>(G, b);
  count_launch();
}

// standalone PyWavelengthDispersion.convolve (lib.rs:671-680): in -> out, all pixels
__global__ void __launch_bounds__(GT) k_gauss_alone(int N, const DevStar *stp, const float *in, float *out) {
  __shared__ float sbuf[G_TILE + 2 * G_HMAX];
  const DevStar &st = *stp;
  const int t0 = blockIdx.x * G_TILE, t1 = min(t0 + G_TILE, N);
  if (st.disp_kind == DISP_NONE) {
    for (int i = t0 + threadIdx.x; i < t1; i += blockDim.x) out[i] = in[i];
    return;
  }
  gauss_tile(st, in, out, N, t0, t1, 0, N, sbuf);
}
void launch_gauss_standalone(const DevGrid &G, const DevStar *star, const float *in, float *out, cudaStream_t s) {
  k_gauss_alone<<<(G.npx + G_TILE - 1) / G_TILE, GT, 0, s>>>(G.npx, star, in, out);
  count_launch();
}

// ------------------------------------------------------------ resampling
// shift_and_resample (convolve_rv.rs:569-603): index in double, weight from
// the f32-rounded index minus the f32 floor, linear interpolation in f32.
struct Resampler {
  const float *s;
  int N, kind;
  double shift_log, shift_factor, lin_offset;
  const double *fidx, *wl_obs, *wl_vals;
  const float *given;  // model given directly at the observed pixels
  __device__ __forceinline__ float operator()(int i) const {
    if (given) return given[i];
    double idx;
    if (kind == WL_LOG) idx = fidx[i] + shift_log;
    else if (kind == WL_LIN) idx = __dadd_rn(__dmul_rn(shift_factor, fidx[i]), lin_offset);
    else {
      const double wl = __dmul_rn(wl_obs[i], shift_factor);
      bool f;
      int k = lower_bound(wl_vals, N, wl, f);
      if (f) idx = (double)k;
      else if (k == 0) idx = 0.0;
      else if (k == N) idx = (double)N - 1.0;
      else idx = __dadd_rn(__dadd_rn(__ddiv_rn(wl - wl_vals[k - 1], wl_vals[k] - wl_vals[k - 1]), (double)k), -1.0);
    }
    const double fl = floor(idx);
    int j = fl > 0 ? (int)fl : 0;
    if (j > N - 2) j = N - 2;  // the preparation kernel rejected j + 1 >= N already
    const float w = (float)idx - (float)j;
    return __fadd_rn(__fmul_rn(1.0f - w, s[j]), __fmul_rn(w, s[j + 1]));
  }
};

__device__ __forceinline__ Resampler make_resampler(const DevGrid &G, const DevStar &st, const EvalPrep &P,
                                                    const float *row, const float *given) {
  Resampler r;
  r.s = row;
  r.N = G.npx;
  r.kind = G.wl_kind;
  r.shift_log = P.shift_log;
  r.shift_factor = P.shift_factor;
  r.lin_offset = P.lin_offset;
  r.fidx = st.fidx;
  r.wl_obs = st.wl_obs;
  r.wl_vals = G.wl_vals;
  r.given = given;
  return r;
}

__global__ void k_resample_out(DevGrid G, EvalBatch b, float *out, int64_t out_stride) {
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  if (P.status) return;
  const DevStar &st = b.stars[P.star];
  const Resampler R = make_resampler(G, st, P, final_row(b, P, st.disp_kind, e), nullptr);
  for (int i = blockIdx.y * blockDim.x + threadIdx.x; i < st.n_obs; i += gridDim.y * blockDim.x)
    out[(size_t)e * out_stride + i] = R(i);
}
void launch_resample_out(const DevGrid &G, const EvalBatch &b, float *out, int64_t out_stride, cudaStream_t s) {
  if (b.E <= 0) return;
  dim3 grid(b.E, 16);
  k_resample_out<<<grid, 256, 0, s>>>(G, b, out, out_stride);
  count_launch();
}

__global__ void k_copy_broadened(DevGrid G, EvalBatch b, float *out) {
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  if (P.status) return;
  const DevStar &st = b.stars[P.star];
  const float *row = final_row(b, P, st.disp_kind, e);
  for (int i = blockIdx.y * blockDim.x + threadIdx.x; i < G.npx; i += gridDim.y * blockDim.x)
    out[(size_t)e * G.npx + i] = row[i];
}
void launch_copy_broadened(const DevGrid &G, const EvalBatch &b, float *out, cudaStream_t s) {
  if (b.E <= 0) return;
  dim3 grid(b.E, 16);
  k_copy_broadened<<<grid, 256, 0, s>>>(G, b, out);
  count_launch();
}

// ------------------------------------------------------------ chi2
constexpr int CT = 512, CW = CT / 32;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// block sum of n <= MAX_P1 per-thread doubles into out[0..n)
__device__ __forceinline__ void block_sum_vec(const double (&v)[MAX_P1], int n, double (*ws)[MAX_P1],
                                              double *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < MAX_P1; k++) {
    if (k < n) {
      const double s = warp_sum(v[k]);
      if (lane == 0) ws[warp][k] = s;
    }
  }
  __syncthreads();
  if (warp == 0) {
    for (int k = 0; k < n; k++) {
      double s = lane < CW ? ws[lane][k] : 0.0;
      s = warp_sum(s);
      if (lane == 0) out[k] = s;
    }
  }
  __syncthreads();
}

__device__ __forceinline__ double block_sum(double v, double (*ws)[MAX_P1]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) ws[warp][0] = v;
  __syncthreads();
  double r = 0.0;
  if (warp == 0) {
    r = lane < CW ? ws[lane][0] : 0.0;
    r = warp_sum(r);
    if (lane == 0) ws[0][1] = r;
  }
  __syncthreads();
  r = ws[0][1];
  __syncthreads();
  return r;
}

// Legendre P_0..P_{p1-1} at x (double recurrence; the host Gram uses the
// identical recurrence and coefficients).
__device__ __forceinline__ void legendre(double x, int p1, double (&P)[MAX_P1]) {
  P[0] = 1.0;
  P[1] = x;
#pragma unroll
  for (int k = 1; k < MAX_P1 - 1; k++) {
    if (k + 1 < p1) {
      const double a = (double)(2 * k + 1) / (double)(k + 1), c = (double)k / (double)(k + 1);
      P[k + 1] = a * x * P[k] - c * P[k - 1];
    }
  }
}

__device__ __forceinline__ float poly_eval(const double *coef, int p1, float xf) {
  double P[MAX_P1];
  legendre((double)xf, p1, P);
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < MAX_P1; k++)
    if (k < p1) s += coef[k] * P[k];
  return (float)s;
}

// CostFunction::cost after produce_model (fitting.rs:322-325): the
// continuum fit of observed/model and the variance-weighted chi2, one CTA
// per evaluation.
//  chunk   (continuum_fitting.rs:216-226, 280-360): per chunk the unweighted
//          least-squares polynomial of flux/model is the projection onto
//          the chunk's polynomial space; it is solved here in a Legendre
//          basis with the FP64 Cholesky factor of its Gram matrix (same
//          space as the reference's monomial SVD, far better conditioned),
//          then chi2 is summed over [50, N-50) with the sin^2 blend in the
//          overlaps and divided by N - 100.
//  linear  (continuum_fitting.rs:68-95): projection onto the design
//          matrix's column space through its orthonormal basis Q; chi2 of
//          the ratio-space residual over [50, N-50) divided by N.
//  fixed   (continuum_fitting.rs:441-474), constant (484-500).
// Moments and chi2 accumulate in FP64.
__global__ void __launch_bounds__(CT) k_chi2(DevGrid G, EvalBatch b, const float *given) {
  __shared__ double ws[CW][MAX_P1];
  __shared__ double zs[MAX_CHUNKS * MAX_P1 > MAX_LIN_K ? MAX_CHUNKS * MAX_P1 : MAX_LIN_K];
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  if (P.status) {
    if (threadIdx.x == 0) {
      b.cost[e] = __longlong_as_double(0x7FF8000000000000ll);
      b.status[e] = P.status;
    }
    return;
  }
  const DevStar &st = b.stars[P.star];
  const int N = st.n_obs;
  const Resampler R = make_resampler(G, st, P, given ? nullptr : final_row(b, P, st.disp_kind, e), given);
  const float *flux = st.flux, *var = st.var;
  double chi2 = 0.0;
  int status = 0;
  double *par = b.params ? b.params + (size_t)e * b.param_stride : nullptr;

  if (st.cont_kind == CONT_CHUNK) {
    const int nc = st.n_chunks, p1 = st.p1;
    if (st.cont_bad) status = S_CONTINUUM;
    else {
      for (int c = 0; c < nc; c++) {
        const int lo = st.cstart[c], hi = st.cstop[c], prev = c > 0 ? st.cstop[c - 1] : -1;
        double z[MAX_P1];
#pragma unroll
        for (int k = 0; k < MAX_P1; k++) z[k] = 0.0;
        for (int i = lo + threadIdx.x; i < hi; i += CT) {
          const float y = flux[i] / R(i);
          const float xf = (c > 0 && i < prev) ? st.xb[i] : st.xa[i];
          double Pk[MAX_P1];
          legendre((double)xf, p1, Pk);
          const double yd = (double)y;
#pragma unroll
          for (int k = 0; k < MAX_P1; k++)
            if (k < p1) z[k] += Pk[k] * yd;
        }
        block_sum_vec(z, p1, ws, zs + c * MAX_P1);
      }
      // per-chunk FP64 Cholesky solve G c = z
      if (threadIdx.x < nc) {
        const int c = threadIdx.x;
        const double *L = st.chol + (size_t)c * p1 * p1;
        double *z = zs + c * MAX_P1;
        double u[MAX_P1];
        for (int k = 0; k < p1; k++) {
          double s = z[k];
          for (int j = 0; j < k; j++) s -= L[k * p1 + j] * u[j];
          u[k] = s / L[k * p1 + k];
        }
        for (int k = p1 - 1; k >= 0; k--) {
          double s = u[k];
          for (int j = k + 1; j < p1; j++) s -= L[j * p1 + k] * z[j];
          z[k] = s / L[k * p1 + k];
        }
        if (par)
          for (int k = 0; k < p1; k++) par[c * p1 + k] = z[k];
      }
      __syncthreads();
      double acc = 0.0;
      // [50, start_1): chunk 0 alone
      for (int i = 50 + threadIdx.x; i < st.cstart[1]; i += CT) {
        const float p = poly_eval(zs, p1, st.xa[i]);
        const float r = flux[i] - p * R(i);
        acc += (double)(r * r / var[i]);
      }
      for (int c = 1; c < nc; c++) {
        const int s0 = st.cstart[c], sp = st.cstop[c - 1];
        const int nx = c == nc - 1 ? N - 50 : st.cstart[c + 1];
        const double *cp = zs + (c - 1) * MAX_P1, *cc = zs + c * MAX_P1;
        for (int i = s0 + threadIdx.x; i < sp; i += CT) {  // overlap: blend previous and current
          const float pv = poly_eval(cp, p1, st.xa[i]);
          const float cu = poly_eval(cc, p1, st.xb[i]);
          const float f = st.fac[i];
          const float p = pv * f + cu * (1.0f - f);
          const float r = flux[i] - p * R(i);
          acc += (double)(r * r / var[i]);
        }
        for (int i = sp + threadIdx.x; i < nx; i += CT) {
          const float p = poly_eval(cc, p1, st.xa[i]);
          const float r = flux[i] - p * R(i);
          acc += (double)(r * r / var[i]);
        }
      }
      chi2 = block_sum(acc, ws) / (double)(N - 100);
    }
  } else if (st.cont_kind == CONT_LINEAR) {
    const int K = st.k_lin;
    for (int g0 = 0; g0 < K; g0 += MAX_P1) {
      const int nk = min(MAX_P1, K - g0);
      double z[MAX_P1];
#pragma unroll
      for (int k = 0; k < MAX_P1; k++) z[k] = 0.0;
      for (int i = threadIdx.x; i < N; i += CT) {
        const double bd = (double)(flux[i] / R(i));
#pragma unroll
        for (int k = 0; k < MAX_P1; k++)
          if (k < nk) z[k] += (double)__ldg(&st.q[(size_t)(g0 + k) * N + i]) * bd;
      }
      block_sum_vec(z, nk, ws, zs + g0);
    }
    if (par && threadIdx.x < K)
      for (int k = threadIdx.x; k < K; k += CT) par[k] = zs[k];
    double acc = 0.0;
    for (int i = 50 + threadIdx.x; i < N - 50; i += CT) {
      const float bb = flux[i] / R(i);
      double fit = 0.0;
      for (int k = 0; k < K; k++) fit += (double)__ldg(&st.q[(size_t)k * N + i]) * zs[k];
      const float r = (float)fit - bb;
      acc += (double)(r / var[i] * r);
    }
    chi2 = block_sum(acc, ws) / (double)N;
  } else if (st.cont_kind == CONT_FIXED) {
    const int ig = st.ignore;
    double acc = 0.0;
    for (int i = ig + threadIdx.x; i < N - ig; i += CT) {
      const float r = flux[i] - R(i) * st.cont[i];
      acc += (double)(r / var[i] * r);
    }
    chi2 = block_sum(acc, ws) / (double)(N - 2 * ig);
    if (par && threadIdx.x == 0) par[0] = 0.0;
  } else {
    double sum = 0.0;
    for (int i = threadIdx.x; i < N; i += CT) sum += (double)(flux[i] / R(i));
    const float mean = (float)(block_sum(sum, ws) / (double)N);
    double acc = 0.0;
    for (int i = threadIdx.x; i < N; i += CT) {
      const float r = flux[i] - R(i) * mean;
      acc += (double)(r / var[i] * r);
    }
    chi2 = block_sum(acc, ws) / (double)N;
    if (par && threadIdx.x == 0) par[0] = (double)mean;
  }
  if (threadIdx.x == 0) {
    b.cost[e] = status ? __longlong_as_double(0x7FF8000000000000ll) : chi2;
    b.status[e] = status;
  }
}

// per-evaluation status when no chi2 is computed (model / spectrum outputs)
__global__ void k_prep_status(EvalBatch b) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < b.E) b.status[e] = b.prep[e].status;
}
void launch_prep_status(const EvalBatch &b, cudaStream_t s) {
  k_prep_status<<<(b.E + 255) / 256, 256, 0, s>>>(b);
  count_launch();
}

void launch_chi2(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0) return;
  k_chi2<<<b.E, CT, 0, s>>>(G, b, nullptr);
  count_launch();
}

// ContinuumFitter::fit_continuum on a given model (lib.rs:862-874): the
// evaluations' resampled model is `given` (observed pixels).
void launch_chi2_given(const DevGrid &G, const EvalBatch &b, const float *given, cudaStream_t s) {
  if (b.E <= 0) return;
  k_chi2<<<b.E, CT, 0, s>>>(G, b, given);
  count_launch();
}

// ChunkFitter::build_continuum_from_chunks (continuum_fitting.rs:228-278)
// from Legendre coefficients: continuum = blend of the chunk polynomials.
__global__ void k_build_chunk(const DevStar *stp, const double *coef, int n, float *out) {
  const DevStar &st = *stp;
  const int nc = st.n_chunks, p1 = st.p1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c = 0;
    while (c + 1 < nc && i >= st.cstart[c + 1]) c++;
    float v;
    if (c > 0 && i < st.cstop[c - 1]) {
      const float pv = poly_eval(coef + (c - 1) * MAX_P1, p1, st.xa[i]);
      const float cu = poly_eval(coef + c * MAX_P1, p1, st.xb[i]);
      const float f = st.fac[i];
      v = pv * f + cu * (1.0f - f);
    } else {
      v = poly_eval(coef + c * MAX_P1, p1, st.xa[i]);
    }
    out[i] = v;
  }
}
void launch_build_chunk(const DevStar *star, const double *coef, int n, float *out, cudaStream_t s) {
  k_build_chunk<<<(n + 255) / 256, 256, 0, s>>>(star, coef, n, out);
  count_launch();
}

}  // namespace pb
