// binary.cu -- the model of a binary system and its chi2 inputs.
//
// Interpolator::produce_binary_model_norm (interpolate.rs:822-893) and
// shift_resample_and_add_binary_components (convolve_rv.rs:606-700) for a
// batch of L binary labels (star 1 [5], star 2 [5], light ratio):
//   k_binary_split    each label's two stars become component evaluations
//                     (star 1 of every label, then star 2) for the regular
//                     interpolate -> rotate -> instrument pipeline on the
//                     whole synthetic grid, and each component gets the
//                     8 corners of its continuum's linear interpolation;
//   k_interp_linear   the continuum row of every component
//                     (interpolate.rs:985-1028) in the workspace buffer its
//                     broadened row is not in, plus its partial sums;
//   k_binary_combine  the light ratio lr = light_ratio mean(c1) / mean(c2)
//                     and, per observed pixel, (n1 c1 + lr n2 c2) / (c1 + lr c2)
//                     with each factor resampled at its star's RV.
// The continuum fitter then runs on that model like on any given model.
//
// Built with -fmad=false and explicit rounding intrinsics: every f32 and f64
// expression is evaluated as written, as in the reference.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace pb {

namespace {

constexpr int LIN_T = 256;              // threads per continuum tile
constexpr int LIN_PX = 8;               // pixels per thread (one 16-byte load per corner)
constexpr int LIN_TILE = LIN_T * LIN_PX;

__device__ __forceinline__ float lerp_ref(float w, float a, float b) {  // convolve_rv.rs:629-631
  return __fadd_rn(__fmul_rn(1.0f - w, a), __fmul_rn(w, b));
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace

int linear_tiles(int npx) { return (npx + LIN_TILE - 1) / LIN_TILE; }

__device__ __forceinline__ void make_lin_rec(const DevGrid &Gc, double t, double m, double lg, LinRec &R) {
  int cols[8];
  float w[8];
  const int st = local_grid_linear(Gc.g, t, m, lg, cols, w);
  R.status = st;
  for (int j = 0; j < 8; j++) {
    R.cols[j] = st ? 0 : cols[j];
    R.w[j] = st ? 0.0f : w[j];
    R.f[j] = st ? 0.0f : Gc.factor[cols[j]];
  }
}

// One thread per component r of 2L: star c = r / L of label l = r % L.
__global__ void k_binary_split(DevGrid Gc, BinaryBatch bb) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= 2 * bb.L) return;
  const int c = r < bb.L ? 0 : 1, l = r - c * bb.L;
  const double *p = bb.labels + 11 * (size_t)l + 5 * c;
  double *q = bb.comp_labels + 5 * (size_t)r;
  q[0] = p[0]; q[1] = p[1]; q[2] = p[2]; q[3] = p[3];
  q[4] = 0.0;  // shifted later, per observed pixel
  make_lin_rec(Gc, p[0], p[1], p[2], bb.lin[r]);
}
void launch_binary_split(const DevGrid &Gc, const BinaryBatch &bb, cudaStream_t s) {
  if (bb.L <= 0) return;
  k_binary_split<<<(2 * bb.L + 127) / 128, 128, 0, s>>>(Gc, bb);
  count_launch();
}

// corners of L labels (teff, m, logg) of the interpolate_linear entry point
__global__ void k_linear_prep(DevGrid Gc, const double *tml, int L, LinRec *lin) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= L) return;
  make_lin_rec(Gc, tml[3 * (size_t)r], tml[3 * (size_t)r + 1], tml[3 * (size_t)r + 2], lin[r]);
}
void launch_linear_prep(const DevGrid &Gc, const double *tml, int L, LinRec *lin, cudaStream_t s) {
  if (L <= 0) return;
  k_linear_prep<<<(L + 127) / 128, 128, 0, s>>>(Gc, tml, L, lin);
  count_launch();
}

// GridInterpolator::interpolate_linear (interpolate.rs:985-1028): pixel i of
// row r is sum_j (u16_j[i] / 65535 * factor_j) * w_j over the corners in
// order.  Grid x = row (rows that share corners run together and share them
// through L2), y = tile of LIN_TILE pixels.  Row r goes to A + r * stride,
// or, with prep (binary components), to the workspace buffer that does not
// hold the component's broadened row; the tile's sum (f64, fixed order) to
// part[r][tile].
__global__ void __launch_bounds__(LIN_T) k_interp_linear(DevGrid Gc, const LinRec *lin, const EvalPrep *prep,
                                                         float *A, float *B, int64_t stride, double *part_base,
                                                         int tiles) {
  __shared__ double red[LIN_T / 32];
  const int r = blockIdx.x, tile = blockIdx.y;
  const LinRec &R = lin[r];
  double *part = part_base + (size_t)r * tiles + tile;
  if (R.status || (prep && prep[r].status)) {
    if (threadIdx.x == 0) *part = 0.0;
    return;
  }
  const int N = Gc.npx;
  const int p0 = tile * LIN_TILE + threadIdx.x * LIN_PX;
  float acc[LIN_PX];
#pragma unroll
  for (int k = 0; k < LIN_PX; k++) acc[k] = 0.0f;
  double sum = 0.0;
  if (p0 < N) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const uint4 q = __ldg(reinterpret_cast<const uint4 *>(Gc.spectra + (size_t)R.cols[j] * Gc.stride + p0));
      const unsigned u[4] = {q.x, q.y, q.z, q.w};
      const float f = R.f[j], w = R.w[j];
#pragma unroll
      for (int k = 0; k < LIN_PX; k++) {
        const float x = (float)((u[k >> 1] >> (16 * (k & 1))) & 0xFFFFu);
        acc[k] = __fadd_rn(acc[k], __fmul_rn(__fmul_rn(__fdiv_rn(x, 65535.0f), f), w));
      }
    }
    float *out = (prep && !prep[r].final_in_b ? B : A) + (size_t)r * stride + p0;
    if (p0 + LIN_PX <= N) {
      reinterpret_cast<float4 *>(out)[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
      reinterpret_cast<float4 *>(out)[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
#pragma unroll
      for (int k = 0; k < LIN_PX; k++) sum += (double)acc[k];
    } else {
      for (int k = 0; k < N - p0; k++) {
        out[k] = acc[k];
        sum += (double)acc[k];
      }
    }
  }
  sum = warp_sum_d(sum);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < LIN_T / 32; i++) t += red[i];
    *part = t;
  }
}
void launch_interp_linear(const DevGrid &Gc, const EvalBatch &comp, const BinaryBatch &bb, cudaStream_t s) {
  if (bb.L <= 0) return;
  k_interp_linear<<<dim3(2 * bb.L, bb.lin_tiles), LIN_T, 0, s>>>(Gc, bb.lin, comp.prep, comp.bufA, comp.bufB,
                                                                comp.stride, bb.part, bb.lin_tiles);
  count_launch();
}
void launch_interp_linear_rows(const DevGrid &Gc, const LinRec *lin, int R, float *out, int64_t stride,
                               double *part, cudaStream_t s) {
  if (R <= 0) return;
  const int tiles = linear_tiles(Gc.npx);
  k_interp_linear<<<dim3(R, tiles), LIN_T, 0, s>>>(Gc, lin, nullptr, out, out, stride, part, tiles);
  count_launch();
}

// produce_binary_components' light ratio (interpolate.rs:858) and
// shift_resample_and_add_binary_components (convolve_rv.rs:606-700).  Grid
// x = label, y = slices of the observed pixels.  The status follows the
// reference's order: star 1's model, its continuum, star 2's model, its
// continuum, then the RV range checks on the extreme shift factors and the
// last resampled pixel of either star (uniform grids: the index grows with
// the observed float index).
__global__ void __launch_bounds__(256) k_binary_combine(DevGrid G, int Nc, EvalBatch comp, BinaryBatch bb) {
  __shared__ float s_lr;
  const int l = blockIdx.x, L = bb.L;
  const int e1 = l, e2 = L + l;
  const EvalPrep &P1 = comp.prep[e1], &P2 = comp.prep[e2];
  const DevStar &st = comp.stars[P1.star];
  const double *lab = bb.labels + 11 * (size_t)l;
  int status = P1.status;
  if (!status) status = bb.lin[e1].status;
  if (!status) status = P2.status;
  if (!status) status = bb.lin[e2].status;
  const double rv1 = lab[4], rv2 = lab[9];
  const double sf1 = __dsub_rn(1.0, __ddiv_rn(rv1, C_KMS)), sf2 = __dsub_rn(1.0, __ddiv_rn(rv2, C_KMS));
  double sl1 = 0.0, sl2 = 0.0, of1 = 0.0, of2 = 0.0;
  const bool logk = G.wl_kind == WL_LOG;
  if (!status) {
    if (rv1 != rv1 || rv2 != rv2) {
      status = S_NAN;
    } else {
      const double smin = sf1 < sf2 ? sf1 : sf2, smax = sf1 < sf2 ? sf2 : sf1;
      if (__dmul_rn(st.wl_first, smin) < G.synth_first) status = S_RV_RANGE;
      else if (__dmul_rn(st.wl_last, smax) > G.synth_last) status = S_RV_RANGE;
      else {
        if (logk) {
          sl1 = __ddiv_rn(log10(sf1), G.wl_b);
          sl2 = __ddiv_rn(log10(sf2), G.wl_b);
        } else {
          const double ab = __ddiv_rn(G.wl_a, G.wl_b);
          of1 = __dmul_rn(ab, __dsub_rn(sf1, 1.0));
          of2 = __dmul_rn(ab, __dsub_rn(sf2, 1.0));
        }
        const double h1 = logk ? __dadd_rn(st.fidx_max, sl1) : __dadd_rn(__dmul_rn(sf1, st.fidx_max), of1);
        const double h2 = logk ? __dadd_rn(st.fidx_max, sl2) : __dadd_rn(__dmul_rn(sf2, st.fidx_max), of2);
        const double f1 = floor(h1), f2 = floor(h2);
        const long long j1 = f1 > 0 ? (long long)f1 : 0, j2 = f2 > 0 ? (long long)f2 : 0;
        if (j1 + 1 >= G.npx || j2 + 1 >= G.npx) status = S_RESAMPLE;
      }
    }
  }
  if (blockIdx.y == 0 && threadIdx.x == 0) {
    bb.cprep[l].status = status;
    bb.cprep[l].star = P1.star;
  }
  if (status) return;
  if (threadIdx.x == 0) {  // DVector::mean = sum * (1 / n), the sums taken in f64
    const double *a = bb.part + (size_t)e1 * bb.lin_tiles, *b = bb.part + (size_t)e2 * bb.lin_tiles;
    double s1 = 0.0, s2 = 0.0;
    for (int t = 0; t < bb.lin_tiles; t++) {
      s1 += a[t];
      s2 += b[t];
    }
    const float inv = __fdiv_rn(1.0f, (float)Nc);
    const float m1 = __fmul_rn((float)s1, inv), m2 = __fmul_rn((float)s2, inv);
    s_lr = __fdiv_rn(__fmul_rn((float)lab[10], m1), m2);
  }
  __syncthreads();
  const float lr = s_lr;
  const size_t o1 = (size_t)e1 * comp.stride, o2 = (size_t)e2 * comp.stride;
  const float *n1 = (P1.final_in_b ? comp.bufB : comp.bufA) + o1, *c1 = (P1.final_in_b ? comp.bufA : comp.bufB) + o1;
  const float *n2 = (P2.final_in_b ? comp.bufB : comp.bufA) + o2, *c2 = (P2.final_in_b ? comp.bufA : comp.bufB) + o2;
  float *out = bb.model + (size_t)l * bb.model_stride;
  for (int i = blockIdx.y * blockDim.x + threadIdx.x; i < st.n_obs; i += gridDim.y * blockDim.x) {
    const double fx = st.fidx[i];
    const double x1 = logk ? __dadd_rn(fx, sl1) : __dadd_rn(__dmul_rn(sf1, fx), of1);
    const double x2 = logk ? __dadd_rn(fx, sl2) : __dadd_rn(__dmul_rn(sf2, fx), of2);
    const double g1 = floor(x1), g2 = floor(x2);
    const int j1 = g1 > 0 ? (int)g1 : 0, j2 = g2 > 0 ? (int)g2 : 0;
    const float w1 = __fsub_rn((float)x1, (float)j1), w2 = __fsub_rn((float)x2, (float)j2);
    const float a1 = lerp_ref(w1, n1[j1], n1[j1 + 1]), k1 = lerp_ref(w1, c1[j1], c1[j1 + 1]);
    const float a2 = lerp_ref(w2, n2[j2], n2[j2 + 1]), k2 = lerp_ref(w2, c2[j2], c2[j2 + 1]);
    const float num = __fadd_rn(__fmul_rn(a1, k1), __fmul_rn(__fmul_rn(lr, a2), k2));
    const float den = __fadd_rn(k1, __fmul_rn(lr, k2));
    out[i] = __fdiv_rn(num, den);
  }
}
void launch_binary_combine(const DevGrid &G, int Nc, const EvalBatch &comp, const BinaryBatch &bb, int n_obs,
                           cudaStream_t s) {
  if (bb.L <= 0) return;
  const int ys = std::max(1, std::min(16, (n_obs + 2047) / 2048));
  k_binary_combine<<<dim3(bb.L, ys), 256, 0, s>>>(G, Nc, comp, bb);
  count_launch();
}

}  // namespace pb
