// prep.cu -- per-evaluation preparation, rotation-kernel spectra and the
// particle-swarm kernels.  Built with -fmad=false: every double expression
// here is evaluated exactly as written, like the reference's Rust, so the
// integer outcomes (neighbour choice, kernel width, windows, clamps) match
// the host and the oracle bit for bit.
#include <atomic>

#include "common.cuh"
#include "fft.cuh"
#include "kernels.h"

namespace pb {

static std::atomic<int64_t> g_launches{0};
int64_t kernel_launches() { return g_launches.load(); }
void count_launch(int n) { g_launches += n; }

// WlGrid::get_float_index_of_wl for NonUniform grids (interpolate.rs:709-727)
__device__ double float_index_nonuni(const double *v, int n, double wl) {
  bool f;
  int i = lower_bound(v, n, wl, f);
  if (f) return (double)i;
  if (i == 0) return 0.0;
  if (i == n) return (double)n - 1.0;
  double left = v[i - 1], right = v[i];
  return (wl - left) / (right - left) + (double)i - 1.0;
}

__device__ __forceinline__ double index_of(const DevGrid &G, const DevStar &st, const EvalPrep &P, double fx,
                                           double wl) {
  if (G.wl_kind == WL_LOG) return fx + P.shift_log;
  if (G.wl_kind == WL_LIN) return P.shift_factor * fx + P.lin_offset;
  return float_index_nonuni(G.wl_vals, G.npx, wl * P.shift_factor);
}

// One thread per evaluation: neighbours + weights (interpolate.rs:930-949),
// rotation width and its error checks (convolve_rv.rs:484-519), the RV
// range checks (convolve_rv.rs:547-567) and the pixel windows every later
// stage works on.
__global__ void k_prep(DevGrid G, EvalBatch b, int full_window) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= b.E) return;
  EvalPrep &P = b.prep[e];
  const int s = b.eval_star[e];
  P.star = s;
  if (b.eval_active && !b.eval_active[e]) {
    P.status = S_INACTIVE;
    return;
  }
  const double *L = b.labels + 5 * (size_t)e;
  const DevStar &st = b.stars[s];
  const int N = G.npx;
  int status = local_grid(G.g, L[0], L[1], L[2], P.cols, P.w);
  const double vsini = L[3], rv = L[4];
  P.vsini = vsini;
  int m = 1;
  if (!status) {
    if (vsini != vsini || rv != rv) status = S_NAN;
    else if (vsini < 0.0) status = S_VSINI;
    else if (G.wl_kind == WL_NONUNI) status = S_UNSUPPORTED;
    else {
      int w = rotation_width(vsini, G.dvelo);
      if (vsini == 0.0 || w <= 2) m = 1;
      else if (w > FFTN) status = S_KERNEL_WIDTH;
      else m = w;
    }
  }
  P.m = m;
  int o_lo = 0, o_hi = N;
  const double shift = 1.0 - rv / C_KMS;
  P.shift_factor = shift;
  P.shift_log = 0.0;
  P.lin_offset = 0.0;
  if (!status && !full_window) {
    if (st.wl_first * shift < G.synth_first) status = S_RV_RANGE;
    else if (st.wl_last * shift > G.synth_last) status = S_RV_RANGE;
    else {
      if (G.wl_kind == WL_LOG) P.shift_log = log10(shift) / G.wl_b;
      else if (G.wl_kind == WL_LIN) P.lin_offset = (G.wl_a / G.wl_b) * (shift - 1.0);
      double lo_idx, hi_idx;
      if (G.wl_kind == WL_NONUNI) {
        lo_idx = float_index_nonuni(G.wl_vals, N, st.wl_min * shift);
        hi_idx = float_index_nonuni(G.wl_vals, N, st.wl_max * shift);
      } else {
        lo_idx = index_of(G, st, P, st.fidx_min, 0.0);
        hi_idx = index_of(G, st, P, st.fidx_max, 0.0);
      }
      double fl = floor(lo_idx), fh = floor(hi_idx);
      long long jl = fl > 0 ? (long long)fl : 0, jh = fh > 0 ? (long long)fh : 0;
      if (jh + 1 >= N) status = S_RESAMPLE;
      o_lo = (int)jl;
      o_hi = (int)(jh + 2 < N ? jh + 2 : N);
    }
  }
  const int hg = st.disp_kind == DISP_NONE ? 0 : (st.gw - 1) / 2;
  int g_lo = o_lo - hg, g_hi = o_hi + hg;
  g_lo = g_lo < 0 ? 0 : g_lo;
  g_hi = g_hi > N ? N : g_hi;
  const int hw = (m - 1) / 2;
  int i_lo = g_lo - hw, i_hi = g_hi + hw;
  i_lo = i_lo < 0 ? 0 : i_lo;
  i_hi = i_hi > N ? N : i_hi;
  i_lo &= ~7;
  i_hi = (i_hi + 7) & ~7;
  P.o_lo = o_lo; P.o_hi = o_hi;
  P.g_lo = g_lo; P.g_hi = g_hi;
  P.i_lo = i_lo; P.i_hi = i_hi;
  P.hg = hg;
  // fused: each 2048-point block yields Vf final outputs; the rotation halo
  // (m - 1) and the instrument halo (2 hg) both come out of the block.
  // Blocks advance by Vf - 1, so the block that owns synth pixel j (the
  // first Vf - 1 of its outputs) also holds j + 1, the resampler's partner.
  const int Vf = FFTN - (m - 1) - 2 * hg;
  const bool work = m > 1 || hg > 0;
  P.epi = 0;
  if (Vf >= MIN_FUSED_OUTPUTS) {
    P.fused = 1;
    const int span = o_hi - 1 - o_lo > 1 ? o_hi - 1 - o_lo : 1;
    P.nblk = work ? (span + Vf - 2) / (Vf - 1) : 0;
    P.final_in_b = work ? 1 : 0;
    P.epi = work && b.obs_epi && st.obs_sorted && !full_window ? 1 : 0;
  } else {  // very wide kernels: rotation FFT into B, instrument profile into A
    P.fused = 0;
    const int V = FFTN - (m - 1);
    P.nblk = m > 1 ? (g_hi - g_lo + V - 1) / V : 0;
    P.final_in_b = hg > 0 ? (m > 1 ? 0 : 1) : (m > 1 ? 1 : 0);
  }
  // narrow combined kernels: direct convolution (k_direct) into B, resampled
  // afterwards by k_resample_obs; the FFT kernels skip these evaluations
  P.direct = 0;
  P.ndt = 0;
  const int taps = m + 2 * hg;
  if (work && P.fused && b.direct_max > 0 && b.direct_list && taps <= b.direct_max && taps <= DIRECT_MAX_TAPS) {
    P.direct = 1;
    P.nblk = 0;
    P.final_in_b = 1;
    P.epi = 0;
    const int td = (DIRECT_TILE - 2 * hg) & ~3;  // final outputs per direct tile
    P.ndt = (o_hi - (o_lo & ~3) + td - 1) / td;  // tiles start at o_lo rounded down to 4
    b.direct_list[atomicAdd(b.direct_count, 1)] = e;
  }
  // the model at the observed pixels goes where no live data is: B when
  // k_broaden resamples (it reads A), else the buffer without the synth row
  P.mobs_in_b = P.epi ? 1 : (P.final_in_b ? 0 : 1);
  P.status = status;
}

// One CTA per evaluation: the limb-darkened rotation profile
// (convolve_rv.rs:438-475), normalised by its f32 sum, zero padded to 2048
// and transformed; the 1025-bin half spectrum goes to H.
__global__ void __launch_bounds__(FFT_T) k_rotker(DevGrid G, EvalBatch b, const float2 *__restrict__ tw) {
  __shared__ float2 c[FFT_SM];
  __shared__ float red[FFT_T];
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  if (P.status || P.m <= 1) return;
  const int m = P.m;
  const double eps = 0.6, pi = 3.141592653589793;
  const double vrot = P.vsini / C_KMS;
  const double dvelo = G.dvelo;
  const double mid = ((double)(m - 1) * dvelo) / 2.0;
  const double den = pi * vrot * (1.0 - eps / 3.0);
  float local = 0.0f;
  for (int t = threadIdx.x; t < FFTN; t += FFT_T) {
    float val = 0.0f;
    if (t < m) {
      double v = (double)t * dvelo - mid;
      double r = v / vrot;
      double y = 1.0 - r * r;
      if (y > 0.0) val = (float)((2.0 * (1.0 - eps) * sqrt(y) + pi * eps / 2.0 * y) / den);
    }
    c[pidx(t)] = make_float2(val, 0.0f);
    local += val;
  }
  red[threadIdx.x] = local;
  __syncthreads();
  for (int o = FFT_T / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  const float total = red[0];
  for (int t = threadIdx.x; t < m; t += FFT_T) c[pidx(t)].x = c[pidx(t)].x / total;
  __syncthreads();
  if (P.direct) {  // the direct path takes the taps themselves (first m floats of H)
    float *taps = reinterpret_cast<float *>(b.H + (size_t)e * 1025);
    for (int t = threadIdx.x; t < m; t += FFT_T) taps[t] = c[pidx(t)].x;
    return;
  }
  fft2048<false>(c, tw);
  float2 *H = b.H + (size_t)e * 1025;
  for (int k = threadIdx.x; k <= 1024; k += FFT_T) H[k] = c[pidx(k)];
  // rotation x instrument spectrum for the blocks of the broadening kernel
  // that apply both as one convolution
  const DevStar &st = b.stars[P.star];
  if (b.HG && st.gspec) {
    float2 *HG = b.HG + (size_t)e * 1025;
    for (int k = threadIdx.x; k <= 1024; k += FFT_T) {
      const float2 g = st.gspec[k];
      const float2 x = c[pidx(k)];
      const cf z = cmul(cf{x.x, x.y}, cf{g.x, g.y});
      HG[k] = make_float2(z.x, z.y);
    }
  }
}

void launch_prep(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0) return;
  if (b.direct_max > 0 && b.direct_count) cudaMemsetAsync(b.direct_count, 0, sizeof(int), s);
  k_prep<<<(b.E + 127) / 128, 128, 0, s>>>(G, b, 0);
  count_launch();
}
void launch_prep_full(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0) return;
  if (b.direct_max > 0 && b.direct_count) cudaMemsetAsync(b.direct_count, 0, sizeof(int), s);
  k_prep<<<(b.E + 127) / 128, 128, 0, s>>>(G, b, 1);
  count_launch();
}
void launch_rotker(const DevGrid &G, const EvalBatch &b, const float2 *tw, cudaStream_t s) {
  if (b.E <= 0) return;
  k_rotker<<<b.E, FFT_T, 0, s>>>(G, b, tw);
  count_launch();
}

// ------------------------------------------------------------------ swarm
// Block-wide minimum of (key, index) with ties to the lower index.
template <int MAXT>
__device__ void block_argmin(double key, int idx, bool valid, double &out_key, int &out_idx, double *skey,
                             int *sidx) {
  const int t = threadIdx.x;
  skey[t] = valid ? key : __longlong_as_double(0x7FF0000000000000ll);
  sidx[t] = valid ? idx : 0x7FFFFFFF;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (t < o) {
      double k2 = skey[t + o];
      int i2 = sidx[t + o];
      if (k2 < skey[t] || (k2 == skey[t] && i2 < sidx[t])) {
        skey[t] = k2;
        sidx[t] = i2;
      }
    }
    __syncthreads();
  }
  out_key = skey[0];
  out_idx = sidx[0];
  __syncthreads();
}

__device__ int block_min_int(int v, int *sm) {
  const int t = threadIdx.x;
  sm[t] = v;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (t < o && sm[t + o] < sm[t]) sm[t] = sm[t + o];
    __syncthreads();
  }
  int r = sm[0];
  __syncthreads();
  return r;
}

// ParticleSwarm::next_iter position/velocity update (particleswarm.rs:234-278)
// for every active star; one CTA per star, one thread per particle (in the
// population's cost-sorted order).  Stars still waiting for their initial
// evaluation just publish their host-placed positions.
__global__ void __launch_bounds__(MAX_PARTICLES) k_pso_update(DevGrid G, Swarm W) {
  __shared__ int sm[MAX_PARTICLES];
  const int s = blockIdx.x, p = threadIdx.x;
  const PsoParams &S = W.params[s];
  const bool star_ok = W.active[s] && !W.done[s] && W.status[s] == 0;
  const bool mine = star_ok && p < S.P;
  const size_t e = (size_t)s * W.Pmax + p;
  const int it = W.iter[s];
  int err = 0;
  double xx[5];
  if (mine) {
    for (int d = 0; d < 5; d++) xx[d] = W.x[e * 5 + d];
    if (it >= 0) {
      double vv[5];
      for (int d = 0; d < 5; d++) vv[d] = W.v[e * 5 + d];
      const uint64_t seed = W.seed[s];
      for (int d = 0; d < 5; d++) {
        const double momentum = vv[d] * S.inertia;
        const double to_opt = W.bx[e * 5 + d] - xx[d];
        const double pull =
            (to_opt == 0.0 ? 0.0 : uniform_between(0.0, to_opt, draw_u01(seed, PH_ITER, it, p, 2 * d))) *
            S.cognitive;
        const double to_g = W.gx[(size_t)s * 5 + d] - xx[d];
        const double pullg =
            (to_g == 0.0 ? 0.0 : uniform_between(0.0, to_g, draw_u01(seed, PH_ITER, it, p, 2 * d + 1))) *
            S.social;
        vv[d] = momentum + pull + pullg;
        double nx[5];
        for (int k = 0; k < 5; k++) nx[k] = xx[k];
        nx[d] += vv[d];
        double c;
        int st = pso_clamp_1d(G.g, S, nx, d, c);
        if (st) { err = st; break; }
        xx[d] = c;
        if (!pso_within(G.g, S, xx)) { err = S_BOUNDS; break; }
      }
      if (!err) {
        for (int d = 0; d < 5; d++) {
          W.x[e * 5 + d] = xx[d];
          W.v[e * 5 + d] = vv[d];
        }
      }
    }
  }
  // the reference aborts at the first failing particle in population order
  const int first = block_min_int(err ? p : 0x7FFFFFFF, sm);
  if (first != 0x7FFFFFFF && p == first) {
    W.status[s] = err;
    W.done[s] = 1;
  }
  if (p < W.Pmax) {
    const bool go = mine && first == 0x7FFFFFFF;
    W.eval_active[e] = go ? 1 : 0;
    if (go)
      for (int d = 0; d < 5; d++) W.labels[e * 5 + d] = xx[d];
  }
}

// After the evaluations: initial sort (particleswarm.rs:117-131, init
// 186-215) or personal/global best update (particleswarm.rs:283-298).
__global__ void __launch_bounds__(MAX_PARTICLES) k_pso_best(Swarm W, const double *cost, const int *est) {
  __shared__ double skey[MAX_PARTICLES];
  __shared__ int sidx[MAX_PARTICLES];
  const int s = blockIdx.x, p = threadIdx.x;
  if (W.refit && p == 0) W.refit[s] = 0;
  if (!(W.active[s] && !W.done[s] && W.status[s] == 0)) return;
  const PsoParams &S = W.params[s];
  const int P = S.P;
  const bool mine = p < P;
  const size_t e = (size_t)s * W.Pmax + p;
  const double c = mine ? cost[e] : 0.0;
  const int es = mine ? est[e] : 0;
  const int first = block_min_int(es != 0 ? p : 0x7FFFFFFF, sidx);
  if (first != 0x7FFFFFFF) {  // one failing particle fails the fit (particleswarm.rs:117, 281)
    if (p == first) {
      W.status[s] = es;
      W.done[s] = 1;
    }
    return;
  }
  const int it = W.iter[s];
  if (it < 0) {
    // stable sort by cost; NaN sorts last
    const double key = (c != c) ? __longlong_as_double(0x7FF0000000000000ll) : c;
    skey[p] = mine ? key : 0.0;
    __syncthreads();
    int rank = 0;
    if (mine) {
      for (int q = 0; q < P; q++) {
        const double kq = skey[q];
        rank += (kq < key || (kq == key && q < p)) ? 1 : 0;
      }
    }
    double xx[5], vv[5];
    if (mine)
      for (int d = 0; d < 5; d++) { xx[d] = W.x[e * 5 + d]; vv[d] = W.v[e * 5 + d]; }
    __syncthreads();
    if (mine) {
      const size_t r = (size_t)s * W.Pmax + rank;
      for (int d = 0; d < 5; d++) {
        W.x[r * 5 + d] = xx[d];
        W.v[r * 5 + d] = vv[d];
        W.bx[r * 5 + d] = xx[d];
      }
      W.cost[r] = c;
      W.bcost[r] = c;
      if (rank == 0) {
        for (int d = 0; d < 5; d++) W.gx[(size_t)s * 5 + d] = xx[d];
        W.gcost[s] = c;
      }
    }
    __syncthreads();
    if (p == 0) {
      W.iter[s] = 0;
      if (S.max_iters <= 0) {
        W.done[s] = 1;
        if (W.refit) W.refit[s] = 1;
      }
    }
    return;
  }
  const double g0 = W.gcost[s];
  bool cand = false;
  if (mine) {
    W.cost[e] = c;
    if (c < W.bcost[e]) {
      for (int d = 0; d < 5; d++) W.bx[e * 5 + d] = W.x[e * 5 + d];
      W.bcost[e] = c;
      cand = c < g0;
    }
  }
  double bk;
  int bi;
  block_argmin<MAX_PARTICLES>(c, p, cand, bk, bi, skey, sidx);
  if (bi != 0x7FFFFFFF && p == bi) {
    for (int d = 0; d < 5; d++) W.gx[(size_t)s * 5 + d] = W.x[e * 5 + d];
    W.gcost[s] = c;
  }
  if (p == 0) {
    W.iter[s] = it + 1;
    if (it + 1 >= S.max_iters) {
      W.done[s] = 1;
      if (W.refit) W.refit[s] = 1;
    }
  }
}

static int pso_threads(int Pmax) {
  int t = 32;
  while (t < Pmax) t <<= 1;
  return t;
}

void launch_pso_update(const DevGrid &G, const Swarm &w, cudaStream_t s) {
  k_pso_update<<<w.S, pso_threads(w.Pmax), 0, s>>>(G, w);
  count_launch();
}
void launch_pso_best(const Swarm &w, const double *cost, const int *status, cudaStream_t s) {
  k_pso_best<<<w.S, pso_threads(w.Pmax), 0, s>>>(w, cost, status);
  count_launch();
}

}  // namespace pb
