// kernels.cu -- the bandwidth, FFT and reduction kernels of the hot path.
//
// Buffer protocol per evaluation e (rows of `stride` floats):
//   k_interp writes the interpolated spectrum to A.
//   k_broaden (rotation FFT + instrument profile, fused) reads A, writes B.
//   Very wide kernels (m - 1 + 2 hg > 2048 - 128) take the unfused pair
//   k_rot (A -> B) and k_gauss (B -> A, or A -> B when the rotation is the
//   identity).  EvalPrep::final_in_b says where the result is.
//   k_chi2_* / k_resample_out read the final row.
#include <cuda_runtime.h>

#include "common.cuh"
#include "fft.cuh"
#include "kernels.h"

namespace pb {

__device__ __forceinline__ const float *final_row(const EvalBatch &b, const EvalPrep &P, int e) {
  return (P.final_in_b ? b.bufB : b.bufA) + (size_t)e * b.stride;
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

// ---------------------------------------------------------------- interp
// flux[px] = sum_n w_n * u16_n[px] * factor_n over the 64 neighbours
// (interpolate.rs:954-981), 8 pixels per thread from one 128-bit load per
// neighbour.  Grid: x = evaluation, y = 2048-pixel tile, so CTAs that run
// together read the same 57 MB tile slab of the resident grid, which stays
// in L2 across evaluations.  The weight and the dequantisation factor are
// folded into one f32 (w * factor); the u16 -> f32 conversion is exact
// (PRMT under the exponent of 2^23, one packed add), and the accumulation is
// one packed f32x2 FMA per two pixels.  Neighbours with weight 0 (absent or
// exactly at a node) contribute exactly 0 and are skipped.
constexpr int IT_T = 256, IT_TILE = IT_T * 8;

__global__ void __launch_bounds__(IT_T) k_interp(DevGrid G, EvalBatch b) {
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  if (P.status) return;
  const int t0 = blockIdx.y * IT_TILE;
  const int ilo = P.i_lo, ihi = P.i_hi;
  if (t0 >= ihi || t0 + IT_TILE <= ilo) return;
  // the neighbours with a non-zero weight, compacted and padded to a
  // multiple of 8 with zero-weight entries (which add exactly 0), so the
  // main loop issues its loads in branch-free groups of 8
  __shared__ const uint16_t *rows[64];
  __shared__ float ws[64], fs[64], wf[64];
  __shared__ int nnz;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    int base = 0;
    for (int h = 0; h < 2; h++) {
      const int n = h * 32 + lane;
      const int c = P.cols[n];
      const float f = c >= 0 ? G.factor[c] : 0.0f;
      const float w = c >= 0 ? P.w[n] : 0.0f;
      const bool keep = w * f != 0.0f;
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int pos = base + __popc(bal & ((1u << lane) - 1u));
        ws[pos] = w;
        fs[pos] = f;
        wf[pos] = w * f;
        rows[pos] = G.spectra + (size_t)c * G.stride;
      }
      base += __popc(bal);
    }
    const int padded = (base + 7) & ~7;
    for (int pos = base + lane; pos < padded; pos += 32) {
      ws[pos] = 0.0f;
      fs[pos] = 0.0f;
      wf[pos] = 0.0f;
      rows[pos] = G.spectra;
    }
    if (lane == 0) nnz = padded;
  }
  __syncthreads();
  const int px = t0 + threadIdx.x * 8;
  if (px < ilo || px >= ihi) return;
  float4 *out = reinterpret_cast<float4 *>(b.bufA + (size_t)e * b.stride + px);
  const int nn = nnz;
  if (px + 8 <= G.tail_start) {
    float2 acc[4];
#pragma unroll
    for (int k = 0; k < 4; k++) acc[k] = make_float2(0.0f, 0.0f);
    const float2 bias = make_float2(-8388608.0f, -8388608.0f);
#pragma unroll 8
    for (int n = 0; n < nn; n++) {
      const float w = wf[n];
      const uint4 q = __ldg(reinterpret_cast<const uint4 *>(rows[n] + px));
      const float2 w2 = make_float2(w, w);
      const uint32_t u[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int k = 0; k < 4; k++) {
        float2 v = make_float2(__int_as_float(__byte_perm(u[k], 0x4B000000u, 0x7410)),
                               __int_as_float(__byte_perm(u[k], 0x4B000000u, 0x7432)));
        v = __fadd2_rn(v, bias);
        acc[k] = __ffma2_rn(w2, v, acc[k]);
      }
    }
    out[0] = make_float4(acc[0].x, acc[0].y, acc[1].x, acc[1].y);
    out[1] = make_float4(acc[2].x, acc[2].y, acc[3].x, acc[3].y);
    return;
  }
  // last tile: the final npx % 128 pixels carry an extra 1/65535 (interpolate.rs:978)
  float acc[8];
#pragma unroll
  for (int k = 0; k < 8; k++) acc[k] = 0.0f;
  for (int n = 0; n < nn; n++) {
    const uint4 q = __ldg(reinterpret_cast<const uint4 *>(rows[n] + px));
    const float wn = ws[n], fn = fs[n];
    const uint32_t u[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const float x = (float)((u[k >> 1] >> (16 * (k & 1))) & 0xFFFFu);
      const float v = px + k >= G.tail_start ? __fmul_rn(__fdiv_rn(x, 65535.0f), fn) : __fmul_rn(x, fn);
      acc[k] = fmaf(wn, v, acc[k]);
    }
  }
  out[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
  out[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
}

void launch_interp(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0) return;
  dim3 grid(b.E, (G.npx + IT_TILE - 1) / IT_TILE);
  k_interp<<<grid, IT_T, 0, s>>>(G, b);
  count_launch();
}

// ------------------------------------------------ instrument profile (tile)
// FixedTargetDispersionLogSpace: g[i] = sum_k gk[k] r[i + h - k], r zero
// outside the grid (convolve_rv.rs:207-210).  Per-pixel kernels
// (VariableTargetDispersion / FixedTargetDispersionNonLog):
// g[i] = kernel_i . r[i-h .. i+h], pixels within h of either end pass
// through (convolve_rv.rs:213-233, 414-430).  r(t) reads the rotation
// output for synth pixel t from wherever the caller staged it.
template <class RF>
__device__ __forceinline__ float instrument(const DevStar &st, int N, int i, int h, const RF &r) {
  const int w = 2 * h + 1;
  float acc = 0.0f;
  if (st.disp_kind == DISP_FIXED) {
    const float *g = st.gk;
    for (int k = 0; k < w; k++) acc = fmaf(__ldg(&g[k]), r(i + h - k), acc);
  } else {
    if (i < h || i >= N - h) return r(i);
    const float *kk = st.gk + (size_t)i * w;
    for (int t = 0; t < w; t++) acc = fmaf(__ldg(&kk[t]), r(i - h + t), acc);
  }
  return acc;
}

// ------------------------------------------------------ fused broadening
// One work item = two blocks of one evaluation.  Block b yields the final
// outputs [o_lo + b V, o_lo + (b+1) V) with V = 2048 - (m - 1) - 2 hg: the
// rotation outputs [s - hg, s + V + hg) come from one overlap-save block of
// 2048 inputs (the reference uses overlap-add, convolve_rv.rs:121-157; both
// are the same linear convolution), and the instrument profile is then
// applied from shared memory.  The two real blocks ride in the real and
// imaginary parts of one complex FFT (the kernel is real, so the two
// products separate after the inverse).  Rotation outputs outside [0, N)
// are zero, like the reference's cropped segment.  With the identity
// rotation the FFT is skipped.
__global__ void __launch_bounds__(FFT_T, 4) k_broaden(DevGrid G, EvalBatch b, const float2 *__restrict__ tw) {
  __shared__ float re[FFT_SM], im[FFT_SM];
  __shared__ float gks[2 * 255 + 1];  // the fixed instrument kernel of the current item
  const long long total = (long long)b.E * b.max_pairs;
  const int N = G.npx;
  for (long long item = blockIdx.x; item < total; item += gridDim.x) {
    const int e = (int)(item / b.max_pairs), pair = (int)(item % b.max_pairs);
    const EvalPrep &P = b.prep[e];
    const int m = P.m, nblk = P.nblk, hg = P.hg;
    if (P.status || !P.fused || 2 * pair >= nblk) continue;
    const DevStar &st = b.stars[P.star];
    const int hw = (m - 1) / 2;
    const int V = FFTN - (m - 1) - 2 * hg;
    const int s0 = P.o_lo + 2 * pair * V, s1 = s0 + V;
    const bool has1 = 2 * pair + 1 < nblk;
    const int ilo = P.i_lo, ihi = P.i_hi, ohi = P.o_hi;
    const float *x = b.bufA + (size_t)e * b.stride;
    // input t of a block is synth pixel (s - hg - hw + t) for the rotation,
    // (s - hg + t) for the identity
    const int shift = m > 1 ? hg + hw : hg;
    for (int t = threadIdx.x; t < FFTN; t += FFT_T) {
      const int j0 = s0 - shift + t, j1 = s1 - shift + t;
      re[pidx(t)] = (j0 >= ilo && j0 < ihi) ? x[j0] : 0.0f;
      im[pidx(t)] = (has1 && j1 >= ilo && j1 < ihi) ? x[j1] : 0.0f;
    }
    const bool fixedk = hg > 0 && st.disp_kind == DISP_FIXED;
    const int gw = 2 * hg + 1;
    if (fixedk)
      for (int t = threadIdx.x; t < gw; t += FFT_T) gks[t] = st.gk[t];
    __syncthreads();
    int base = 0;  // data index of rotation output (s - hg)
    // Away from the grid ends the Gaussian acts on rotation outputs that are
    // all inside [0, N), where rotation-then-Gaussian equals one convolution
    // with the combined kernel: multiply the spectra and skip the taps.
    const int e_last = min((has1 ? s1 : s0) + V, ohi);
    const bool fold = fixedk && m > 1 && st.gspec != nullptr && s0 - hg >= 0 && e_last + hg <= N;
    if (m > 1) {
      fft2048<false>(re, im, tw);
      const float2 *H = b.H + (size_t)e * 1025;
      for (int k = threadIdx.x; k < FFTN; k += FFT_T) {
        float2 h = k <= 1024 ? H[k] : H[FFTN - k];
        if (k > 1024) h.y = -h.y;
        cf hk{h.x, h.y};
        if (fold) {
          float2 g = k <= 1024 ? st.gspec[k] : st.gspec[FFTN - k];
          if (k > 1024) g.y = -g.y;
          hk = cmul(hk, cf{g.x, g.y});
        }
        const int a = pidx(k);
        const cf z = cmul(cf{re[a], im[a]}, hk);
        re[a] = z.x;
        im[a] = z.y;
      }
      __syncthreads();
      fft2048<true>(re, im, tw);
      base = m - 1;
      const float sc = 1.0f / 2048.0f;
      if (fold) {  // output i sits at base + 2 hg + (i - s)
        float *y = b.bufB + (size_t)e * b.stride;
        for (int u = threadIdx.x; u < V; u += FFT_T) {
          const int i0 = s0 + u, i1 = s1 + u;
          if (i0 < ohi) y[i0] = re[pidx(base + 2 * hg + u)] * sc;
          if (has1 && i1 < ohi) y[i1] = im[pidx(base + 2 * hg + u)] * sc;
        }
        __syncthreads();
        continue;
      }
      for (int t = base + threadIdx.x; t < FFTN; t += FFT_T) {
        const int i0 = s0 - hg + (t - base), i1 = s1 - hg + (t - base);
        re[pidx(t)] = (i0 >= 0 && i0 < N) ? re[pidx(t)] * sc : 0.0f;
        im[pidx(t)] = (i1 >= 0 && i1 < N) ? im[pidx(t)] * sc : 0.0f;
      }
      __syncthreads();
    }
    float *y = b.bufB + (size_t)e * b.stride;
    for (int u = threadIdx.x; u < V; u += FFT_T) {
      const int i0 = s0 + u, i1 = s1 + u;
      float v0, v1;
      if (hg == 0) {
        v0 = re[pidx(base + u)];
        v1 = im[pidx(base + u)];
      } else if (fixedk) {  // g[i] = sum_k gk[k] r[i + hg - k]; r[i] sits at base + (i - s + hg)
        float a0 = 0.0f, a1 = 0.0f;
        for (int k = 0; k < gw; k++) {
          const float g = gks[k];
          const int t = pidx(base + u + 2 * hg - k);
          a0 = fmaf(g, re[t], a0);
          a1 = fmaf(g, im[t], a1);
        }
        v0 = a0;
        v1 = a1;
      } else {
        v0 = instrument(st, N, i0, hg, [&](int i) { return re[pidx(base + i - (s0 - hg))]; });
        v1 = has1 ? instrument(st, N, i1, hg, [&](int i) { return im[pidx(base + i - (s1 - hg))]; }) : 0.0f;
      }
      if (i0 < ohi) y[i0] = v0;
      if (has1 && i1 < ohi) y[i1] = v1;
    }
    __syncthreads();
  }
}

void launch_broaden(const DevGrid &G, const EvalBatch &b, const float2 *tw, cudaStream_t s) {
  if (b.E <= 0 || b.max_pairs <= 0) return;
  const long long total = (long long)b.E * b.max_pairs;
  long long grid = (long long)num_sms() * 4;  // persistent: the CTAs that fit at once (64 regs x 256)
  if (grid > total) grid = total;
  k_broaden<<<(unsigned)grid, FFT_T, 0, s>>>(G, b, tw);
  count_launch();
}

// ------------------------------------------- unfused rotation (wide kernels)
// Overlap-save with the rotation kernel alone: block b produces rotation
// outputs [g_lo + b V, g_lo + (b+1) V), V = 2048 - (m - 1), into B.
__global__ void __launch_bounds__(FFT_T, 3) k_rot(DevGrid G, EvalBatch b, const float2 *__restrict__ tw) {
  __shared__ float re[FFT_SM], im[FFT_SM];
  const long long total = (long long)b.E * b.max_pairs_unfused;
  for (long long item = blockIdx.x; item < total; item += gridDim.x) {
    const int e = (int)(item / b.max_pairs_unfused), pair = (int)(item % b.max_pairs_unfused);
    const EvalPrep &P = b.prep[e];
    const int m = P.m, nblk = P.nblk;
    if (P.status || P.fused || m <= 1 || 2 * pair >= nblk) continue;
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

void launch_rot(const DevGrid &G, const EvalBatch &b, const float2 *tw, cudaStream_t s) {
  if (b.E <= 0 || b.max_pairs_unfused <= 0) return;
  const long long total = (long long)b.E * b.max_pairs_unfused;
  long long grid = (long long)num_sms() * 6;
  if (grid > total) grid = total;
  k_rot<<<(unsigned)grid, FFT_T, 0, s>>>(G, b, tw);
  count_launch();
}

// unfused instrument profile: src = rotation output, dst = the other buffer
constexpr int GT = 256, G_TILE = 4096, G_HMAX = 256;

__global__ void __launch_bounds__(GT) k_gauss(DevGrid G, EvalBatch b) {
  __shared__ float sbuf[G_TILE + 2 * G_HMAX];
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  if (P.status || P.fused || P.hg == 0) return;
  const DevStar &st = b.stars[P.star];
  const int t0 = max((int)blockIdx.y * G_TILE, P.o_lo), t1 = min((int)(blockIdx.y + 1) * G_TILE, P.o_hi);
  if (t0 >= t1) return;
  const bool rot_in_b = P.m > 1;
  const float *src = (rot_in_b ? b.bufB : b.bufA) + (size_t)e * b.stride;
  float *dst = (rot_in_b ? b.bufA : b.bufB) + (size_t)e * b.stride;
  const int h = P.hg, base = t0 - h;
  for (int j = threadIdx.x; j < (t1 - t0) + 2 * h; j += blockDim.x) {
    const int g = base + j;
    sbuf[j] = (g >= P.g_lo && g < P.g_hi) ? src[g] : 0.0f;
  }
  __syncthreads();
  for (int i = t0 + threadIdx.x; i < t1; i += blockDim.x)
    dst[i] = instrument(st, G.npx, i, h, [&](int t) { return sbuf[t - base]; });
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
  const int h = (st.gw - 1) / 2, base = t0 - h;
  for (int j = threadIdx.x; j < (t1 - t0) + 2 * h; j += blockDim.x) {
    const int g = base + j;
    sbuf[j] = (g >= 0 && g < N) ? in[g] : 0.0f;
  }
  __syncthreads();
  for (int i = t0 + threadIdx.x; i < t1; i += blockDim.x)
    out[i] = instrument(st, N, i, h, [&](int t) { return sbuf[t - base]; });
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
  const Resampler R = make_resampler(G, st, P, final_row(b, P, e), nullptr);
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
  const float *row = final_row(b, P, e);
  for (int i = blockIdx.y * blockDim.x + threadIdx.x; i < G.npx; i += gridDim.y * blockDim.x)
    out[(size_t)e * G.npx + i] = row[i];
}
void launch_copy_broadened(const DevGrid &G, const EvalBatch &b, float *out, cudaStream_t s) {
  if (b.E <= 0) return;
  dim3 grid(b.E, 16);
  k_copy_broadened<<<grid, 256, 0, s>>>(G, b, out);
  count_launch();
}

// ------------------------------------------------------------------ chi2
constexpr int CT = 256, CW = CT / 32;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// block sum of K per-thread doubles into out[0..K)
template <int K>
__device__ __forceinline__ void block_sum_vec(const double (&v)[K], double (*ws)[MAX_P1], double *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) {
    const double s = warp_sum(v[k]);
    if (lane == 0) ws[warp][k] = s;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) {
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

// Legendre P_0..P_{K-1} at x (f32, the host Gram uses the same recurrence)
template <int K>
__device__ __forceinline__ void legendre(float x, float (&P)[K]) {
  P[0] = 1.0f;
  if (K > 1) P[1] = x;
#pragma unroll
  for (int k = 1; k + 1 < K; k++) P[k + 1] = leg_step(leg_a(k), leg_c(k), x, P[k], P[k - 1]);
}

template <int K>
__device__ __forceinline__ float poly_eval(const float *coef, float x) {
  float P[K];
  legendre<K>(x, P);
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < K; k++) s = fmaf(coef[k], P[k], s);
  return s;
}

__device__ __forceinline__ void write_result(const EvalBatch &b, int e, double chi2, int status) {
  if (threadIdx.x == 0) {
    b.cost[e] = status ? __longlong_as_double(0x7FF8000000000000ll) : chi2;
    b.status[e] = status;
  }
}

// ChunkFitter::fit_continuum (continuum_fitting.rs:382-396): per chunk the
// unweighted least-squares polynomial of flux/model (216-226) is the
// projection onto the chunk's polynomial space; it is solved here in a
// Legendre basis with the FP64 Cholesky factor of its Gram matrix (the same
// space as the reference's monomial SVD, far better conditioned).  chi2 is
// summed over [50, N-50) with the sin^2 blend in the overlaps and divided
// by N - 100 (280-360).  Moments and chi2 accumulate in FP64.  One CTA per
// evaluation; K = polynomial order + 1 (one instantiation per order present).
template <int K>
__global__ void __launch_bounds__(CT, 4) k_chi2_chunk(DevGrid G, EvalBatch b, const float *given) {
  __shared__ double ws[CW][MAX_P1];
  __shared__ double zs[MAX_CHUNKS * K];
  __shared__ float cf32[MAX_CHUNKS * K];
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  const DevStar &st = b.stars[P.star];
  if (st.cont_kind != CONT_CHUNK || st.p1 != K) return;
  if (P.status) {
    write_result(b, e, 0.0, P.status);
    return;
  }
  if (st.cont_bad) {
    write_result(b, e, 0.0, S_CONTINUUM);
    return;
  }
  const int N = st.n_obs, nc = st.n_chunks;
  const Resampler R = make_resampler(G, st, P, given ? nullptr : final_row(b, P, e), given);
  const float *flux = st.flux, *var = st.var;
  for (int c = 0; c < nc; c++) {
    const int lo = st.cstart[c], hi = st.cstop[c], prev = c > 0 ? st.cstop[c - 1] : -1;
    double z[K];
#pragma unroll
    for (int k = 0; k < K; k++) z[k] = 0.0;
#pragma unroll 4
    for (int i = lo + threadIdx.x; i < hi; i += CT) {
      const double y = (double)(flux[i] / R(i));
      const float xf = (c > 0 && i < prev) ? st.xb[i] : st.xa[i];
      float Pk[K];
      legendre<K>(xf, Pk);
#pragma unroll
      for (int k = 0; k < K; k++) z[k] = fma((double)Pk[k], y, z[k]);
    }
    block_sum_vec<K>(z, ws, zs + c * K);
  }
  // per-chunk FP64 Cholesky solve G c = z
  if (threadIdx.x < nc) {
    const int c = threadIdx.x;
    const double *L = st.chol + (size_t)c * K * K;
    double *z = zs + c * K;
    double u[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      double s = z[k];
#pragma unroll
      for (int j = 0; j < k; j++) s -= L[k * K + j] * u[j];
      u[k] = s / L[k * K + k];
    }
#pragma unroll
    for (int k = K - 1; k >= 0; k--) {
      double s = u[k];
#pragma unroll
      for (int j = k + 1; j < K; j++) s -= L[j * K + k] * z[j];
      z[k] = s / L[k * K + k];
      cf32[c * K + k] = (float)z[k];
    }
    if (b.params)
      for (int k = 0; k < K; k++) b.params[(size_t)e * b.param_stride + c * K + k] = z[k];
  }
  __syncthreads();
  double acc = 0.0;
  for (int i = 50 + threadIdx.x; i < st.cstart[1]; i += CT) {  // [50, start_1): chunk 0 alone
    const float p = poly_eval<K>(cf32, st.xa[i]);
    const float r = flux[i] - p * R(i);
    acc += (double)(r * r / var[i]);
  }
  for (int c = 1; c < nc; c++) {
    const int s0 = st.cstart[c], sp = st.cstop[c - 1];
    const int nx = c == nc - 1 ? N - 50 : st.cstart[c + 1];
    const float *cp = cf32 + (c - 1) * K, *cc = cf32 + c * K;
#pragma unroll 2
    for (int i = s0 + threadIdx.x; i < sp; i += CT) {  // overlap: blend previous and current
      const float pv = poly_eval<K>(cp, st.xa[i]);
      const float cu = poly_eval<K>(cc, st.xb[i]);
      const float f = st.fac[i];
      const float p = pv * f + cu * (1.0f - f);
      const float r = flux[i] - p * R(i);
      acc += (double)(r * r / var[i]);
    }
#pragma unroll 4
    for (int i = sp + threadIdx.x; i < nx; i += CT) {
      const float p = poly_eval<K>(cc, st.xa[i]);
      const float r = flux[i] - p * R(i);
      acc += (double)(r * r / var[i]);
    }
  }
  const double chi2 = block_sum(acc, ws) / (double)(N - 100);
  write_result(b, e, chi2, 0);
}

// LinearModelFitter (continuum_fitting.rs:68-95): projection onto the design
// matrix's column space through its orthonormal basis Q; chi2 of the
// ratio-space residual over [50, N-50) divided by N.  FixedContinuum
// (441-474) and ConstantContinuum (484-500) too.
__global__ void __launch_bounds__(CT) k_chi2_other(DevGrid G, EvalBatch b, const float *given) {
  __shared__ double ws[CW][MAX_P1];
  __shared__ double zs[MAX_LIN_K];
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  const DevStar &st = b.stars[P.star];
  if (st.cont_kind == CONT_CHUNK) return;
  if (P.status) {
    write_result(b, e, 0.0, P.status);
    return;
  }
  if (st.cont_bad) {
    write_result(b, e, 0.0, S_CONTINUUM);
    return;
  }
  const int N = st.n_obs;
  const Resampler R = make_resampler(G, st, P, given ? nullptr : final_row(b, P, e), given);
  const float *flux = st.flux, *var = st.var;
  double chi2 = 0.0;
  double *par = b.params ? b.params + (size_t)e * b.param_stride : nullptr;
  if (st.cont_kind == CONT_LINEAR) {
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
          if (k < nk) z[k] = fma((double)__ldg(&st.q[(size_t)(g0 + k) * N + i]), bd, z[k]);
      }
      block_sum_vec<MAX_P1>(z, ws, zs + g0);
    }
    if (par)
      for (int k = threadIdx.x; k < K; k += CT) par[k] = zs[k];
    double acc = 0.0;
    for (int i = 50 + threadIdx.x; i < N - 50; i += CT) {
      const float bb = flux[i] / R(i);
      double fit = 0.0;
      for (int k = 0; k < K; k++) fit = fma((double)__ldg(&st.q[(size_t)k * N + i]), zs[k], fit);
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
  write_result(b, e, chi2, 0);
}

template <int K>
static void launch_chunk(const DevGrid &G, const EvalBatch &b, const float *given, cudaStream_t s) {
  k_chi2_chunk<K><<<b.E, CT, 0, s>>>(G, b, given);
  count_launch();
}

static void launch_chi2_impl(const DevGrid &G, const EvalBatch &b, const float *given, cudaStream_t s) {
  if (b.E <= 0) return;
  const uint32_t m = b.chunk_p1_mask;
  if (m & (1u << 1)) launch_chunk<1>(G, b, given, s);
  if (m & (1u << 2)) launch_chunk<2>(G, b, given, s);
  if (m & (1u << 3)) launch_chunk<3>(G, b, given, s);
  if (m & (1u << 4)) launch_chunk<4>(G, b, given, s);
  if (m & (1u << 5)) launch_chunk<5>(G, b, given, s);
  if (m & (1u << 6)) launch_chunk<6>(G, b, given, s);
  if (m & (1u << 7)) launch_chunk<7>(G, b, given, s);
  if (m & (1u << 8)) launch_chunk<8>(G, b, given, s);
  if (m & (1u << 9)) launch_chunk<9>(G, b, given, s);
  if (m & (1u << 10)) launch_chunk<10>(G, b, given, s);
  if (m & (1u << 11)) launch_chunk<11>(G, b, given, s);
  if (m & (1u << 12)) launch_chunk<12>(G, b, given, s);
  if (m & (1u << 13)) launch_chunk<13>(G, b, given, s);
  if (m & (1u << 14)) launch_chunk<14>(G, b, given, s);
  if (m & (1u << 15)) launch_chunk<15>(G, b, given, s);
  if (m & (1u << 16)) launch_chunk<16>(G, b, given, s);
  if (b.other_cont) {
    k_chi2_other<<<b.E, CT, 0, s>>>(G, b, given);
    count_launch();
  }
}

void launch_chi2(const DevGrid &G, const EvalBatch &b, cudaStream_t s) { launch_chi2_impl(G, b, nullptr, s); }

// ContinuumFitter::fit_continuum on a given model (lib.rs:862-874): the
// evaluations' resampled model is `given` (observed pixels).
void launch_chi2_given(const DevGrid &G, const EvalBatch &b, const float *given, cudaStream_t s) {
  launch_chi2_impl(G, b, given, s);
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

// ChunkFitter::build_continuum_from_chunks (continuum_fitting.rs:228-278)
// from Legendre coefficients: continuum = blend of the chunk polynomials.
template <int K>
__device__ float build_one(const DevStar &st, const double *coef, int i) {
  const int nc = st.n_chunks;
  int c = 0;
  while (c + 1 < nc && i >= st.cstart[c + 1]) c++;
  float cp[K], cc[K];
  for (int k = 0; k < K; k++) cc[k] = (float)coef[c * MAX_P1 + k];
  if (c > 0 && i < st.cstop[c - 1]) {
    for (int k = 0; k < K; k++) cp[k] = (float)coef[(c - 1) * MAX_P1 + k];
    const float pv = poly_eval<K>(cp, st.xa[i]);
    const float cu = poly_eval<K>(cc, st.xb[i]);
    const float f = st.fac[i];
    return pv * f + cu * (1.0f - f);
  }
  return poly_eval<K>(cc, st.xa[i]);
}

__global__ void k_build_chunk(const DevStar *stp, const double *coef, int n, float *out) {
  const DevStar &st = *stp;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float v;
    switch (st.p1) {
      case 1: v = build_one<1>(st, coef, i); break;
      case 2: v = build_one<2>(st, coef, i); break;
      case 3: v = build_one<3>(st, coef, i); break;
      case 4: v = build_one<4>(st, coef, i); break;
      case 5: v = build_one<5>(st, coef, i); break;
      case 6: v = build_one<6>(st, coef, i); break;
      case 7: v = build_one<7>(st, coef, i); break;
      case 8: v = build_one<8>(st, coef, i); break;
      case 9: v = build_one<9>(st, coef, i); break;
      case 10: v = build_one<10>(st, coef, i); break;
      case 11: v = build_one<11>(st, coef, i); break;
      case 12: v = build_one<12>(st, coef, i); break;
      case 13: v = build_one<13>(st, coef, i); break;
      case 14: v = build_one<14>(st, coef, i); break;
      case 15: v = build_one<15>(st, coef, i); break;
      default: v = build_one<16>(st, coef, i); break;
    }
    out[i] = v;
  }
}
void launch_build_chunk(const DevStar *star, const double *coef, int n, float *out, cudaStream_t s) {
  k_build_chunk<<<(n + 255) / 256, 256, 0, s>>>(star, coef, n, out);
  count_launch();
}

void pipeline_pairs(int npx, int max_m, int max_hg, int *max_pairs, int *max_pairs_unfused, int *may_unfuse) {
  const int wide = (max_m - 1) + 2 * max_hg;
  *may_unfuse = wide > FFTN - MIN_FUSED_OUTPUTS ? 1 : 0;
  if (max_m <= 1 && max_hg == 0) {
    *max_pairs = 0;
  } else {
    const int V = *may_unfuse ? MIN_FUSED_OUTPUTS : FFTN - wide;
    const int nblk = (npx + V - 1) / V;
    *max_pairs = (nblk + 1) / 2;
  }
  if (*may_unfuse && max_m > 1) {
    const int V = FFTN - (max_m - 1);
    const int nblk = (npx + V - 1) / V;
    *max_pairs_unfused = (nblk + 1) / 2;
  } else {
    *max_pairs_unfused = 0;
  }
}

void launch_pipeline(const DevGrid &G, const EvalBatch &b, const float2 *tw, const PipelineOpts &o, cudaStream_t s) {
  if (o.full_window) launch_prep_full(G, b, s);
  else launch_prep(G, b, s);
  if (o.rot) launch_rotker(G, b, tw, s);
  launch_interp(G, b, s);
  launch_broaden(G, b, tw, s);
  if (o.may_unfuse) {
    launch_rot(G, b, tw, s);
    launch_gauss(G, b, s);
  }
  if (b.need_chi2) launch_chi2(G, b, s);
  else if (b.status) launch_prep_status(b, s);
}

}  // namespace pb
