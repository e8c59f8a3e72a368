// fft.cuh -- shared-memory complex FFT of 2048 points for one 256-thread CTA.
//
// Stockham autosort (Govindaraju et al., "High performance discrete Fourier
// transforms on graphics processors", SC 2008) with radices 8, 8, 8, 4.
// Data live in shared memory as 2048 interleaved complex values (float2,
// one 64-bit access each) whose index is XOR-swizzled within each 16-value
// row (bits 0-3 ^= bits 3-6): a 64-bit warp access is served as two
// half-warps, and every stage's strided reads and scattered writes, and the
// linear accesses, then touch 16 distinct 8-byte bank pairs per half-warp.
// Twiddles W_2048^k = exp(-2 pi i k / 2048) come from a table the host
// computed in double.  Forward is unnormalised; the inverse is unnormalised
// too (caller scales by 1/2048, like convolve_rv.rs:153-154).
#pragma once
#include <cuda_runtime.h>

namespace pb {

constexpr int FFT_T = 256;
constexpr int FFT_SM = 2048;
__device__ __forceinline__ int pidx(int i) { return i ^ ((i >> 3) & 15); }

struct cf {
  float x, y;
};
__device__ __forceinline__ cf cmul(cf a, cf b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
// complex add / subtract as one packed f32x2 instruction each (a - b as
// b * (-1) + a: the product is exact, so this rounds like a - b)
__device__ __forceinline__ cf cadd(cf a, cf b) {
  const float2 r = __fadd2_rn(make_float2(a.x, a.y), make_float2(b.x, b.y));
  return {r.x, r.y};
}
__device__ __forceinline__ cf csub(cf a, cf b) {
  const float2 r = __ffma2_rn(make_float2(b.x, b.y), make_float2(-1.0f, -1.0f), make_float2(a.x, a.y));
  return {r.x, r.y};
}
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ cf rot90(cf a) {
  return INV ? cf{-a.y, a.x} : cf{a.y, -a.x};
}

template <bool INV>
__device__ __forceinline__ void dft4(cf &v0, cf &v1, cf &v2, cf &v3) {
  cf t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), t3 = rot90<INV>(csub(v1, v3));
  v0 = cadd(t0, t2);
  v2 = csub(t0, t2);
  v1 = cadd(t1, t3);
  v3 = csub(t1, t3);
}

template <bool INV>
__device__ __forceinline__ void dft8(cf v[8]) {
  cf e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  cf o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<INV>(e0, e1, e2, e3);
  dft4<INV>(o0, o1, o2, o3);
  const float c = 0.70710678118654752f;
  o1 = cmul(o1, cf{c, INV ? c : -c});
  o2 = rot90<INV>(o2);
  o3 = cmul(o3, cf{-c, INV ? c : -c});
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

// One Stockham stage of radix R at sub-transform length NS.  With MID all
// reads of the stage happen before a barrier, all writes after it, so the
// transform runs in place; without it the stage must read and write
// different buffers (ping-pong) and only the closing barrier remains.  The
// caller must __syncthreads() after filling the input.
// ld(i, a) returns input element i (a = its swizzled shared-memory slot),
// st(i, a, v, s) stores output element i, the thread's s-th output of the
// stage (a compile-time constant after unrolling); SmemLoad / SmemStore use the
// swizzled re/im arrays, other functors may read a staging buffer or write
// outputs elsewhere.
//
// Slot arithmetic: the swizzle only mixes bits 3-6 into bits 0-3, so
// pidx(j + c) = pidx(j) + c for every multiple c of 256, and the writes of
// the four stages of fft2048 reduce to one XOR with a per-thread base:
//   NS = 1:   pidx(8j + r)           = (8j ^ (j & 15)) ^ r
//   NS = 8:   pidx(d + 8r)           = (d ^ (j & 8)) ^ 9r
//   NS = 64:  pidx(d + 64r)          = (d ^ ((j >> 3) & 7)) ^ (64r ^ 8(r & 1))
//   NS = 512: pidx(j + 512r)         = pidx(j) + 512r
// with d the first output index of the thread's butterfly.  The identities
// and the absence of bank conflicts hold for every thread and r of these
// stages (checked exhaustively).
template <int R, int NS, bool INV, class LD, class ST, bool MID = true>
__device__ __forceinline__ void fft_pass(const float2 *__restrict__ tw, const LD &ld, const ST &st) {
  static_assert((R == 8 && (NS == 1 || NS == 8 || NS == 64)) || (R == 4 && NS == 512), "fft2048 stage");
  constexpr int N = 2048, J = N / R, PER = J / FFT_T, STEP = N / (NS * R);
  const int t = threadIdx.x;
  const int p0 = pidx(t);
  cf v[PER][R];
#pragma unroll
  for (int q = 0; q < PER; q++) {
    const int j = t + q * FFT_T;
#pragma unroll
    for (int r = 0; r < R; r++) v[q][r] = ld(j + r * J, p0 + q * FFT_T + r * J);
    if constexpr (NS > 1) {
      // twiddles W^(jm r STEP): W^1, W^2, W^4 from the table, the others by
      // at most two multiplications (jm = 0 multiplies by exactly 1)
      const int k1 = (j & (NS - 1)) * STEP;
      const float2 t1 = __ldg(&tw[k1]), t2 = __ldg(&tw[2 * k1]);
      const cf w1{t1.x, INV ? -t1.y : t1.y}, w2{t2.x, INV ? -t2.y : t2.y};
      v[q][1] = cmul(v[q][1], w1);
      v[q][2] = cmul(v[q][2], w2);
      const cf w3 = cmul(w1, w2);
      v[q][3] = cmul(v[q][3], w3);
      if constexpr (R == 8) {
        const float2 t4 = __ldg(&tw[4 * k1]);
        const cf w4{t4.x, INV ? -t4.y : t4.y};
        v[q][4] = cmul(v[q][4], w4);
        v[q][5] = cmul(v[q][5], cmul(w4, w1));
        v[q][6] = cmul(v[q][6], cmul(w4, w2));
        v[q][7] = cmul(v[q][7], cmul(w4, w3));
      }
    }
  }
  if constexpr (MID) __syncthreads();
#pragma unroll
  for (int q = 0; q < PER; q++) {
    const int j = t + q * FFT_T;
    if constexpr (R == 8) dft8<INV>(v[q]);
    else dft4<INV>(v[q][0], v[q][1], v[q][2], v[q][3]);
    const int d = (j / NS) * NS * R + (j & (NS - 1));
#pragma unroll
    for (int r = 0; r < R; r++) {
      int a;
      if constexpr (NS == 1) a = (d ^ (j & 15)) ^ r;
      else if constexpr (NS == 8) a = (d ^ (j & 8)) ^ (9 * r);
      else if constexpr (NS == 64) a = (d ^ ((j >> 3) & 7)) ^ (64 * r ^ 8 * (r & 1));
      else a = p0 + q * FFT_T + r * NS;
      st(d + r * NS, a, v[q][r], q * R + r);
    }
  }
  __syncthreads();
}

struct SmemLoad {
  const float2 *c;
  __device__ __forceinline__ cf operator()(int, int a) const {
    const float2 v = c[a];
    return cf{v.x, v.y};
  }
};
struct SmemStore {
  float2 *c;
  __device__ __forceinline__ void operator()(int, int a, cf v, int) const { c[a] = make_float2(v.x, v.y); }
};

template <int R, int NS, bool INV>
__device__ __forceinline__ void fft_stage(float2 *c, const float2 *__restrict__ tw) {
  fft_pass<R, NS, INV>(tw, SmemLoad{c}, SmemStore{c});
}
// one stage from buffer src to buffer dst (no barrier between reads and writes)
template <int R, int NS, bool INV>
__device__ __forceinline__ void fft_stage_pp(const float2 *src, float2 *dst, const float2 *__restrict__ tw) {
  fft_pass<R, NS, INV, SmemLoad, SmemStore, false>(tw, SmemLoad{src}, SmemStore{dst});
}

// ------------------------------------------------------------------------
// 2048-point FFT of one 128-thread group, 2048 = 16 x 16 x 8 ("four-step"
// decomposition, n = 128 n1 + 8 n2 + n3, k = k1 + 16 k2 + 256 k3):
//   pass 1  thread t = 8 n2 + n3: DFT-16 over n1, times W_2048^(t k1)
//   pass 2  thread t = 8 k1 + n3: DFT-16 over n2, times W_128^(n3 k2)
//   pass 3  thread t: for c = t and t + 128 (c = k1 + 16 k2), DFT-8 over n3,
//           giving X[c + 256 k3]
// Each thread keeps 16 values in registers through a pass; the passes
// exchange through shared memory twice.  The inverse runs the same passes
// backwards (DFT-8, DFT-16, DFT-16 with conjugate twiddles), starting from
// the spectrum where the forward transform left it, so a spectrum product
// between them needs no reordering: a round trip costs four exchanges.
// Exchange 1 rows are padded to F2_XP values and exchange 2 is XOR-swizzled
// so that every access of a half-warp (64-bit values) touches 16 distinct
// bank pairs.  Twiddles come from per-CTA tables built from the host's
// double-precision table.
constexpr int F2_T = 128;
constexpr int F2_XP = 136;
constexpr int F2_S1 = 16 * F2_XP;  // complex values of exchange buffer 1
constexpr int F2_S2 = 2048;        // complex values of exchange buffer 2
__device__ __forceinline__ int f2_a2(int c, int n3) { return 8 * c + (n3 ^ ((c >> 1) & 7)); }

// a * w (FWD) or a * conj(w) (INV)
template <bool INV>
__device__ __forceinline__ cf cmul_tw(cf a, float2 w) {
  return INV ? cf{a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y} : cf{a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x};
}

// DFT-16 of v (natural order in and out) as 4 x 4: n = 4a + b, k = c + 4d
template <bool INV>
__device__ __forceinline__ void dft16(cf v[16]) {
  const float c1 = 0.92387953251128674f, s1 = 0.38268343236508977f, h = 0.70710678118654752f;
#pragma unroll
  for (int b = 0; b < 4; b++) dft4<INV>(v[b], v[4 + b], v[8 + b], v[12 + b]);
  // y[b][c] sits in v[4c + b]; times W16^(bc)
  const float sg = INV ? 1.0f : -1.0f;
  v[5] = cmul(v[5], cf{c1, sg * s1});     // b1 c1: W^1
  v[6] = cmul(v[6], cf{h, sg * h});       // b2 c1: W^2
  v[7] = cmul(v[7], cf{s1, sg * c1});     // b3 c1: W^3
  v[9] = cmul(v[9], cf{h, sg * h});       // b1 c2: W^2
  v[10] = rot90<INV>(v[10]);              // b2 c2: W^4
  v[11] = cmul(v[11], cf{-h, sg * h});    // b3 c2: W^6
  v[13] = cmul(v[13], cf{s1, sg * c1});   // b1 c3: W^3
  v[14] = cmul(v[14], cf{-h, sg * h});    // b2 c3: W^6
  v[15] = cmul(v[15], cf{-c1, -sg * s1}); // b3 c3: W^9
#pragma unroll
  for (int c = 0; c < 4; c++) dft4<INV>(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
  // X[c + 4d] sits in v[4c + d]: transpose the 4 x 4 index
  cf t[16];
#pragma unroll
  for (int i = 0; i < 16; i++) t[i] = v[i];
#pragma unroll
  for (int c = 0; c < 4; c++)
#pragma unroll
    for (int d = 0; d < 4; d++) v[c + 4 * d] = t[4 * c + d];
}

template <bool INV>
__device__ __forceinline__ void fft2048(float2 *c, const float2 *__restrict__ tw) {
  fft_stage<8, 1, INV>(c, tw);
  fft_stage<8, 8, INV>(c, tw);
  fft_stage<8, 64, INV>(c, tw);
  fft_stage<4, 512, INV>(c, tw);
}

}  // namespace pb
