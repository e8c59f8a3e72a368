// lintc.cu -- the linear-model continuum fit on the 5th-generation tensor
// cores (tcgen05, accumulators in tensor memory).
//
// LinearModelFitter (continuum_fitting.rs:44-107): b = flux / model, the
// unweighted least-squares solution in the design matrix's column space and
// chi2 = sum over [50, N - 50) of (fit - b)^2 / var, divided by N.  With Q an
// orthonormal basis of that space (host QR), the coefficients are z = Q^T b
// and the fit is Q z.  For the evaluations of one star (up to 128, the
// particles of a swarm) these are two dense products:
//   GEMM1  Z^T [128 x KP]  = B^T [128 x N] . Q [N x KP]      (B = flux / model per evaluation)
//   GEMM2  F^T [128 x 32]  = Z^T [128 x KP] . Q^T [KP x 32]  per tile of 32 pixels,
// and the residual sum is the epilogue of GEMM2.  Each group's pixels are
// split into slices (more when there are fewer groups) worked by separate
// CTAs; the slices' partial coefficients and residual sums are added in
// slice order, so the result does not depend on scheduling.  Both run as
// tcgen05.mma kind::tf32 with M = 128 from shared-memory operands in the
// canonical K-major layout (8-row x 16-byte core matrices, no swizzle).  To
// keep f32 accuracy each operand is split into a tf32 head and an exact
// remainder and every product is formed as hi.hi + hi.lo + lo.hi (three MMAs
// into one accumulator).  Each k-step (8 elements of the reduction) has
// its own tensor-memory accumulator, so a tensor-core sum never runs over
// more than those three MMAs; the k-steps are added in f64 registers.
// Every wait on the MMA completion barrier is bounded; a wait that runs out
// marks the group's evaluations with an internal error, and the CTA still
// frees its tensor memory.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "kernels.h"

namespace pb {

namespace {

constexpr int LT_T = 256;   // threads: evaluation row p = t & 127, column half h = t >> 7
constexpr int LT_M = 128;   // evaluations per group (MMA M)
constexpr int LT_TK = 32;   // pixels per GEMM1 stage
constexpr int LT_TN = 32;   // pixels per GEMM2 tile (MMA N)
// tensor memory: one accumulator region per k-step (GEMM1: 4 regions of 64
// columns; GEMM2: up to 8 regions of 32 columns), summed in f64 on read-back
constexpr uint32_t LT_TMEM_COLS = 256;
constexpr int S_MMA_TIMEOUT = -99;      // PASTA_E_INTERNAL
// partial coefficient of a slice whose barrier wait ran out (never a real value)
constexpr double LT_FAILED = -1e300;

// shared-memory map (bytes)
constexpr int G1_AH = 0, G1_AL = 16384, G1_BH = 32768, G1_BL = 40960;  // B^T stage 128 x 32, Q stage 64 x 32
constexpr int G2_AH = 0, G2_AL = 32768;                                // Z^T 128 x 64
constexpr int G2_BH = 65536, G2_BL = 81920;                            // Q^T tile 32 x 64
constexpr int LT_MISC = 98304;                                         // barrier, tensor-memory slot, flags
constexpr int LT_RED = LT_MISC + 64;                                   // 128 doubles: half-1 residual sums
constexpr int LT_RFAIL = LT_RED + LT_M * 8;                            // 128 ints: half-1 failure flags
constexpr int LT_ROWS = LT_RFAIL + LT_M * 4;                           // 128 model-row pointers (null: no row)
constexpr int LT_VAR = LT_ROWS + LT_M * 8;                             // GEMM2: the tile's 32 variances
constexpr int LT_SMEM = LT_VAR + LT_TN * 4;
// GEMM2: the ratio tile flux/model of 128 evaluations x 32 pixels, rows
// 0-63 and 64-127 in the unused halves of the two Q^T tile buffers, each
// row's 32 values XOR-swizzled by the row (conflict-free column reads)
constexpr int G2_Y0 = G2_BH + 8192, G2_Y1 = G2_BL + 8192;
static_assert(G2_Y1 + 8192 <= LT_MISC, "ratio tile");

// byte offset of element (row, k) in a K-major tile with kt elements per
// row: core matrix (row / 8, k / 4) of 8 rows x 16 bytes, row-group stride
// kt / 4 core matrices
__device__ __forceinline__ int kmaj(int row, int k, int kt) {
  return ((((row >> 3) * (kt >> 2) + (k >> 2)) << 3) + (row & 7)) * 16 + (k & 3) * 4;
}

// shared-memory matrix descriptor: start address, leading byte offset 128
// (the next 16-byte column of core matrices along K), stride byte offset
// between 8-row groups, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, int kt) {
  const uint64_t sbo = (uint64_t)((kt >> 2) * 128);
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) | ((sbo >> 4) << 32) | (1ull << 46);
}
// instruction descriptor: f32 accumulator, tf32 A and B, both K-major
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D (tensor memory) = A . B^T (+ D when acc != 0); no output lane disabled
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  const uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(m0), "r"(m1), "r"(m2), "r"(m3));
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar)
               : "memory");
}
// bounded wait for phase `parity` of the barrier (about a second at most)
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > 2000000000ll) return false;
  }
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// eight consecutive f32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

// tf32 head (x rounded to 10 mantissa bits, nearest) and the exact remainder
__device__ __forceinline__ void split_tf32(float x, float &hi, float &lo) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  hi = __uint_as_float(r);
  lo = x - hi;
}
__device__ __forceinline__ void store_split4(unsigned char *sm, int off_hi, int off_lo, float4 v) {
  float4 h, l;
  split_tf32(v.x, h.x, l.x);
  split_tf32(v.y, h.y, l.y);
  split_tf32(v.z, h.z, l.z);
  split_tf32(v.w, h.w, l.w);
  *reinterpret_cast<float4 *>(sm + off_hi) = h;
  *reinterpret_cast<float4 *>(sm + off_lo) = l;
}

__device__ __forceinline__ const float *lt_model_row(const EvalBatch &b, const EvalPrep &P, int e) {
  if (b.given) return b.given + (size_t)e * b.given_stride;
  return (P.mobs_in_b ? b.bufB : b.bufA) + (size_t)e * b.stride;
}

// flux / model of the 16 (row, pixel) elements of a 128 x 32 stage this
// thread loads: warp w takes rows 16 w .. 16 w + 15, and one warp
// instruction covers 8 rows x 4 consecutive pixels (lane = 4 row + pixel),
// so a row's pixels are read in 16-byte pieces by neighbouring lanes and the
// K-major shared-memory stores of one instruction hit 32 distinct banks.
// Element j: row 16 w + 8 (j >> 3) + (lane >> 2), pixel 4 (j & 7) + (lane & 3).
// Rows without a model (null) and pixels at or past x1 give 0.
__device__ __forceinline__ void load_ratio_tile(const float *const *rows, const float *flux, int i0, int x1,
                                                float (&y)[16]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int rr = lane >> 2, kk = lane & 3;
  float fx[8];
#pragma unroll
  for (int pg = 0; pg < 8; pg++) {
    const int i = i0 + 4 * pg + kk;
    fx[pg] = i < x1 ? flux[i] : 0.0f;
  }
#pragma unroll
  for (int rg = 0; rg < 2; rg++) {
    const float *row = rows[16 * w + 8 * rg + rr];
#pragma unroll
    for (int pg = 0; pg < 8; pg++) {
      const int i = i0 + 4 * pg + kk;
      y[8 * rg + pg] = (row && i < x1) ? fx[pg] / row[i] : 0.0f;
    }
  }
}
__device__ __forceinline__ int ratio_row(int j) { return 16 * (threadIdx.x >> 5) + 8 * (j >> 3) + ((threadIdx.x & 31) >> 2); }
__device__ __forceinline__ int ratio_px(int j) { return 4 * (j & 7) + (threadIdx.x & 3); }

}  // namespace

// One CTA per (group of b.lin_group consecutive evaluations of one star whose
// continuum is a linear model with a tensor-core basis, pixel slice): the
// slices spread a group over the GPU when there are few groups.
// MODE 0: GEMM1 over the slice -> f64 partial coefficients lin_zpart[e][slice].
// MODE 1: the coefficients (partials summed in slice order), GEMM2 and the
//         residual sum over the slice -> cpart[e][slice].
template <int KP, int MODE>
__global__ void __launch_bounds__(LT_T) k_linear_tc(EvalBatch b) {
  static_assert(KP % 16 == 0 && KP >= 16 && KP <= 64, "basis columns");
  extern __shared__ __align__(1024) unsigned char sm[];
  const int t = threadIdx.x, p = t & (LT_M - 1), h = t >> 7, w = t >> 5;
  const int LG = b.lin_group;
  const int e0 = blockIdx.x * LG;
  // the group's star: the first member's (all members share it by construction)
  const int star = b.prep[e0].star;
  const DevStar &st = b.stars[star];
  if (st.cont_kind != CONT_LINEAR || st.kp != KP) return;
  const int N = st.n_obs, K = st.k_lin;
  const int S = gridDim.y, sl = blockIdx.y;
  const int per = ((N + S - 1) / S + LT_TK - 1) / LT_TK * LT_TK;
  const int x0 = min(N, sl * per), x1 = min(N, x0 + per);
  const int e = e0 + p;
  const bool member = p < LG && e < b.E;
  const EvalPrep *P = member ? &b.prep[e] : nullptr;
  const bool live = member && P->status == 0 && P->star == star && !st.cont_bad;
  const float *mod = live ? lt_model_row(b, *P, e) : nullptr;
  const float *flux = st.flux, *var = st.var, *q = st.q, *qt = st.qt;
  constexpr int HALF = KP / 2;
  double *zp = b.lin_zpart + ((size_t)e * LIN_MAX_SLICES) * 64;

  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
  const uint32_t mbar = sbase + LT_MISC;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + LT_MISC + 8);
  int *err = reinterpret_cast<int *>(sm + LT_MISC + 16);
  double *red = reinterpret_cast<double *>(sm + LT_RED);
  const float **rows = reinterpret_cast<const float **>(sm + LT_ROWS);
  if (t < LT_M) rows[t] = mod;  // t = p, h = 0
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mbar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    *err = 0;
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sbase + LT_MISC + 8),
                 "r"(LT_TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t lane_off = (uint32_t)((w & 3) * 32) << 16;
  uint32_t phase = 0;
  bool ok = true;
  double z[HALF];
#pragma unroll
  for (int c = 0; c < HALF; c++) z[c] = 0.0;

  if (MODE == 0) {
    // ---------------------------------------------- GEMM1: Z^T = B^T Q over the slice
    // Each k-step of a 32-pixel stage goes to its own accumulator (3 MMAs)
    // and the four are read back and added into the f64 coefficients.  The
    // next stage's operands are loaded into registers while the MMAs run.
    const uint32_t id1 = idesc_tf32(LT_M, KP);
    const int r = t >> 2, kq = 8 * (t & 3);  // Q stage: basis row r, pixels kq .. kq + 8
    float av[16], qv[8];
    auto load_stage = [&](int i0) {
      load_ratio_tile(rows, flux, i0, x1, av);
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const int i = i0 + kq + j;
        qv[j] = (r < K && i < x1) ? q[(size_t)r * N + i] : 0.0f;
      }
    };
    if (x0 < x1) load_stage(x0);
    for (int i0 = x0; i0 < x1 && ok; i0 += LT_TK) {
#pragma unroll
      for (int j = 0; j < 16; j++) {
        float hi, lo;
        split_tf32(av[j], hi, lo);
        const int o = kmaj(ratio_row(j), ratio_px(j), LT_TK);
        *reinterpret_cast<float *>(sm + G1_AH + o) = hi;
        *reinterpret_cast<float *>(sm + G1_AL + o) = lo;
      }
      if (r < KP) {
#pragma unroll
        for (int g = 0; g < 2; g++)
          store_split4(sm, G1_BH + kmaj(r, kq + 4 * g, LT_TK), G1_BL + kmaj(r, kq + 4 * g, LT_TK),
                       make_float4(qv[4 * g], qv[4 * g + 1], qv[4 * g + 2], qv[4 * g + 3]));
      }
      proxy_fence();
      __syncthreads();
      if (t == 0) {
        tc_fence_after();
#pragma unroll
        for (int s = 0; s < LT_TK / 8; s++) {
          const uint32_t off = (uint32_t)(s * 256);
          const uint64_t ah = smem_desc(sbase + G1_AH + off, LT_TK), al = smem_desc(sbase + G1_AL + off, LT_TK);
          const uint64_t bh = smem_desc(sbase + G1_BH + off, LT_TK), bl = smem_desc(sbase + G1_BL + off, LT_TK);
          const uint32_t d = tmem + (uint32_t)(s * 64);
          mma_tf32(d, ah, bh, id1, 0u);
          mma_tf32(d, ah, bl, id1, 1u);
          mma_tf32(d, al, bh, id1, 1u);
        }
        mma_commit(mbar);
      }
      if (i0 + LT_TK < x1) load_stage(i0 + LT_TK);  // in flight while the MMAs run
      if (!mbar_wait(mbar, phase)) atomicOr(err, 1);
      phase ^= 1u;
      __syncthreads();
      ok = *err == 0;
      if (!ok) break;
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < LT_TK / 8; ks++)
#pragma unroll
        for (int c = 0; c < HALF; c += 8) {
          float v[8];
          tmem_ld8(tmem + lane_off + (uint32_t)(ks * 64 + h * HALF + c), v);
#pragma unroll
          for (int j = 0; j < 8; j++) z[c + j] += (double)v[j];
        }
      tc_fence_before();
    }
    if (live) {
#pragma unroll
      for (int c = 0; c < HALF; c++) zp[(size_t)sl * 64 + h * HALF + c] = ok ? z[c] : LT_FAILED;
    }
  } else {
    // ---------------------------------------------- GEMM2 + residual epilogue over the slice
    bool zfail = false;
    if (live) {  // slot 0 holds the slices' partial coefficients added in slice order (k_linear_zsum)
#pragma unroll
      for (int c = 0; c < HALF; c++) {
        const double v = zp[h * HALF + c];
        zfail |= v == LT_FAILED;
        z[c] = v;
      }
      if (b.params && sl == 0) {
        double *par = b.params + (size_t)e * b.param_stride;
#pragma unroll
        for (int c = 0; c < HALF; c++)
          if (h * HALF + c < K) par[h * HALF + c] = z[c];
      }
    }
#pragma unroll
    for (int c = 0; c < HALF; c += 4) {
      const int k = h * HALF + c;
      float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (live) v = make_float4((float)z[c], (float)z[c + 1], (float)z[c + 2], (float)z[c + 3]);
      store_split4(sm, G2_AH + kmaj(p, k, KP), G2_AL + kmaj(p, k, KP), v);
    }
    double acc = 0.0;
    const uint32_t id2 = idesc_tf32(LT_M, LT_TN);
    const int r = t >> 3, kq = 8 * (t & 7);  // Q^T tile: pixel row r (of 32), basis columns kq .. kq + 8
    float4 qv[2];
    auto load_tile = [&](int i0) {
      const int i = i0 + r;
#pragma unroll
      for (int g = 0; g < 2; g++)
        qv[g] = (i < x1 && kq + 4 * g < KP) ? *reinterpret_cast<const float4 *>(qt + (size_t)i * KP + kq + 4 * g)
                                            : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    };
    // ratio tile element (row, pixel) in shared memory
    auto yslot = [&](int row, int k) -> float * {
      return reinterpret_cast<float *>(sm + (row < 64 ? G2_Y0 : G2_Y1)) + (row & 63) * 32 + (k ^ (row & 31));
    };
    float *svar = reinterpret_cast<float *>(sm + LT_VAR);
    float yv[16];  // this thread's part of the next ratio tile (coalesced loads)
    if (x0 < x1) {
      load_tile(x0);
      load_ratio_tile(rows, flux, x0, x1, yv);
    }
    for (int i0 = x0; i0 < x1 && ok; i0 += LT_TN) {
      if (i0 > x0) __syncthreads();  // every thread is done with the previous ratio tile
#pragma unroll
      for (int j = 0; j < 16; j++) *yslot(ratio_row(j), ratio_px(j)) = yv[j];
      if (t < LT_TN) svar[t] = i0 + t < x1 ? var[i0 + t] : 1.0f;
#pragma unroll
      for (int g = 0; g < 2; g++)
        if (kq + 4 * g < KP) store_split4(sm, G2_BH + kmaj(r, kq + 4 * g, KP), G2_BL + kmaj(r, kq + 4 * g, KP), qv[g]);
      proxy_fence();
      __syncthreads();
      if (t == 0) {
        tc_fence_after();
#pragma unroll
        for (int s = 0; s < KP / 8; s++) {
          const uint32_t off = (uint32_t)(s * 256);
          const uint64_t ah = smem_desc(sbase + G2_AH + off, KP), al = smem_desc(sbase + G2_AL + off, KP);
          const uint64_t bh = smem_desc(sbase + G2_BH + off, KP), bl = smem_desc(sbase + G2_BL + off, KP);
          const uint32_t d = tmem + (uint32_t)(s * LT_TN);
          mma_tf32(d, ah, bh, id2, 0u);
          mma_tf32(d, ah, bl, id2, 1u);
          mma_tf32(d, al, bh, id2, 1u);
        }
        mma_commit(mbar);
      }
      // while the MMAs run: the next tile's basis and ratios
      if (i0 + LT_TN < x1) {
        load_tile(i0 + LT_TN);
        load_ratio_tile(rows, flux, i0 + LT_TN, x1, yv);
      }
      if (!mbar_wait(mbar, phase)) atomicOr(err, 1);
      phase ^= 1u;
      __syncthreads();
      ok = *err == 0;
      if (!ok) break;
      tc_fence_after();
      // fit of row p at pixels i0 + 16 h + j: the k-step regions added in f64
#pragma unroll
      for (int c = 0; c < 16; c += 8) {
        double f[8];
#pragma unroll
        for (int j = 0; j < 8; j++) f[j] = 0.0;
#pragma unroll
        for (int ks = 0; ks < KP / 8; ks++) {
          float v[8];
          tmem_ld8(tmem + lane_off + (uint32_t)(ks * LT_TN + 16 * h + c), v);
#pragma unroll
          for (int j = 0; j < 8; j++) f[j] += (double)v[j];
        }
        if (live) {
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const int i = i0 + 16 * h + c + j;
            if (i >= 50 && i < N - 50 && i < x1) {
              const float rr = (float)f[j] - *yslot(p, 16 * h + c + j);
              acc += (double)(rr / svar[16 * h + c + j] * rr);
            }
          }
        }
      }
      tc_fence_before();
    }
    int *rfail = reinterpret_cast<int *>(sm + LT_RFAIL);
    if (h == 1) {
      red[p] = acc;
      rfail[p] = zfail ? 1 : 0;
    }
    __syncthreads();
    // a residual sum is never negative: -1 marks a failed slice (a NaN sum stays a NaN chi2, as in the reference)
    if (h == 0 && live) b.cpart[(size_t)e * MAX_CHUNKS + sl] = (ok && !zfail && !rfail[p]) ? acc + red[p] : -1.0;
  }
  // ------------------------------------------------ tensor memory
  tc_fence_before();
  __syncthreads();
  if (w == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(LT_TMEM_COLS) : "memory");
  }
}

// The slices' partial coefficients of every evaluation added in slice order
// into slot 0 (one thread per evaluation and basis column; a failed slice
// fails the sum), so that each residual-pass CTA reads 64 values instead of
// 64 per slice.
__global__ void k_linear_zsum(EvalBatch b, int kp) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)b.E * 64) return;
  const int e = (int)(i >> 6), c = (int)(i & 63);
  const DevStar &st = b.stars[b.prep[(e / b.lin_group) * b.lin_group].star];  // the group's star
  if (st.cont_kind != CONT_LINEAR || st.kp != kp) return;
  double *zp = b.lin_zpart + (size_t)e * LIN_MAX_SLICES * 64 + c;
  double acc = 0.0;
  bool fail = false;
  for (int s = 0; s < b.lin_slices; s++) {
    const double v = zp[(size_t)s * 64];
    fail |= v == LT_FAILED;
    acc += v;
  }
  zp[0] = fail ? LT_FAILED : acc;
}

// chi2 = the slices' residual sums in slice order / N, and the statuses, of
// the evaluations of tensor-core linear continua
__global__ void k_linear_final(EvalBatch b) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= b.E) return;
  const int LG = b.lin_group;
  const int star = b.prep[(e / LG) * LG].star;
  const DevStar &st = b.stars[star];
  if (st.cont_kind != CONT_LINEAR || st.kp == 0) return;
  const EvalPrep &P = b.prep[e];
  int s = P.status;
  if (!s && P.star != star) s = S_MMA_TIMEOUT;
  if (!s && st.cont_bad) s = S_CONTINUUM;
  double chi2 = 0.0;
  if (!s) {
    for (int k = 0; k < b.lin_slices; k++) {
      const double v = b.cpart[(size_t)e * MAX_CHUNKS + k];
      if (v < 0.0) s = S_MMA_TIMEOUT;  // a residual sum is never negative: a slice's barrier wait ran out
      chi2 += v;
    }
    chi2 /= (double)st.n_obs;
  }
  b.cost[e] = s ? __longlong_as_double(0x7FF8000000000000ll) : chi2;
  b.status[e] = s;
}

template <int KP>
static void launch_kp(const EvalBatch &b, dim3 grid, cudaStream_t s) {
  cudaFuncSetAttribute(k_linear_tc<KP, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, LT_SMEM);
  cudaFuncSetAttribute(k_linear_tc<KP, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, LT_SMEM);
  k_linear_tc<KP, 0><<<grid, LT_T, LT_SMEM, s>>>(b);
  if (grid.y > 1) {
    k_linear_zsum<<<(unsigned)(((long long)b.E * 64 + 255) / 256), 256, 0, s>>>(b, KP);
    count_launch();
  }
  k_linear_tc<KP, 1><<<grid, LT_T, LT_SMEM, s>>>(b);
  count_launch(2);
}

void launch_linear_tc(const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0 || b.lin_group <= 0 || b.lin_group > LT_M || !b.lin_kp_mask) return;
  const int groups = (b.E + b.lin_group - 1) / b.lin_group;
  const dim3 grid(groups, b.lin_slices);
  if (b.lin_kp_mask & (1u << 1)) launch_kp<16>(b, grid, s);
  if (b.lin_kp_mask & (1u << 2)) launch_kp<32>(b, grid, s);
  if (b.lin_kp_mask & (1u << 3)) launch_kp<48>(b, grid, s);
  if (b.lin_kp_mask & (1u << 4)) launch_kp<64>(b, grid, s);
  k_linear_final<<<(b.E + 255) / 256, 256, 0, s>>>(b);
  count_launch();
}

}  // namespace pb
