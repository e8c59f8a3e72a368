// interp_tc.cu -- cubic interpolation of evaluations that share their 64
// neighbour rows, on the 5th-generation tensor cores.
//
// GridInterpolator::interpolate (interpolate.rs:930-983) computes, per
// pixel, flux = sum_n w_n * (u16_n * factor_n) over the 64 neighbour models.
// A particle swarm contracts into one grid cube within a few dozen
// iterations; from then on its particles share the 64 rows and differ only
// in their weights, so the swarm's interpolation is one matrix product per
// tile of 128 pixels:
//   D [128 pixels x members] = A [128 pixels x 128] . B [128 x members]
// with A[p][k] = 256 * hi_k(p) and A[p][64 + k] = lo_k(p), the two bytes of
// row k's u16 value at pixel p (exact in bf16), and B[k][n] = B[64 + k][n]
// = weight_n,k x factor_k, split into three bf16 parts whose sum is the f32
// value (8 + 8 + 8 significant bits).  Every product is exact in the f32
// accumulator; the three parts are three MMA chains into one tensor-memory
// accumulator.  A member's result depends only on its own weights (each
// accumulator column is computed on its own), so it does not depend on the
// other members of the group.
//
// Rows are staged by TMA (cp.async.bulk.tensor, one 128-pixel box per row,
// from the grid resident in this GPU's memory; no multicast), converted to
// the bf16 byte planes by the CTA's threads, multiplied by tcgen05.mma
// (kind::f16, M = 128, N = members rounded up to 16, one thread issues),
// and read back from tensor memory by tcgen05.ld for the stores; the tiles
// of an item run as a software pipeline (see k_interp_tc).
// The last npx % 128 pixels carry the reference's extra 1/65535
// (interpolate.rs:978) and are computed on the CUDA cores.
//
// Every wait on an mbarrier is bounded (about a second); a wait that runs
// out marks the group's evaluations with an internal error and the CTA still
// frees its tensor memory.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "kernels.h"

namespace pb {

namespace {

constexpr int TT = 256;      // threads: pixel t & 127 of a tile, rows / columns half t >> 7
constexpr int TPX = 128;     // pixels per tile (MMA M)
constexpr int TK = 128;      // reduction: 64 neighbours x {256 x high byte, low byte}
constexpr int TSLAB = 16;    // tiles per item
constexpr int TMEM_COLS = 128;  // two accumulators of up to 64 columns
constexpr int S_TC_TIMEOUT = -99;  // PASTA_E_INTERNAL

// shared memory (bytes): three weight parts [64 members][128] bf16 (K-major),
// two staging tiles [64 rows][128 pixels] u16, two A tiles [128 pixels][128]
// bf16 (K-major), barriers and flags, the members' windows and indices
constexpr int SB_B = 0;
constexpr int SB_STG = SB_B + 3 * 64 * TK * 2;
constexpr int SB_A = SB_STG + 2 * 64 * TPX * 2;
constexpr int SB_MISC = SB_A + 2 * TPX * TK * 2;
constexpr int SB_WIN = SB_MISC + 64;
constexpr int SB_TOTAL = SB_WIN + 3 * SEG * 4;

// byte offset of element (row, k) of a K-major bf16 tile with TK elements
// per row: core matrices of 8 rows x 16 bytes (8 elements), K-adjacent core
// matrices 128 bytes apart, 8-row groups TK / 8 core matrices apart
__device__ __forceinline__ int kmaj16(int row, int k) {
  return ((((row >> 3) * (TK >> 3) + (k >> 3)) << 3) + (row & 7)) * 16 + (k & 7) * 2;
}
// shared-memory matrix descriptor of such a tile (no swizzle, version 1)
__device__ __forceinline__ uint64_t desc16(uint32_t saddr) {
  const uint64_t lbo = 128, sbo = (TK >> 3) * 128;
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((lbo >> 4) << 16) | ((sbo >> 4) << 32) | (1ull << 46);
}
// instruction descriptor: f32 accumulator, bf16 A and B, both K-major
__device__ __forceinline__ uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar)
               : "memory");
}
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

// TMA: one box of 128 pixels of grid row y starting at pixel x
__device__ __forceinline__ void tma_row(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}
__device__ __forceinline__ void mbar_expect(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(bytes) : "memory");
}

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

// bf16 bits of x (round to nearest even), as the low 16 bits
__device__ __forceinline__ uint32_t bf16_bits(float x) {
  uint32_t r;
  asm("{\n\t.reg .b16 h;\n\tcvt.rn.bf16.f32 h, %1;\n\tmov.b32 %0, {h, h};\n\t}" : "=r"(r) : "f"(x));
  return r & 0xFFFFu;
}
__device__ __forceinline__ float bf16_val(uint32_t bits) { return __uint_as_float(bits << 16); }

// TMA of tile i's 64 rows (pixels lo + 128 i ...) into staging buffer i & 1,
// issued by the 32 lanes of one warp (two rows each) after lane 0 has set
// the barrier's expected bytes
__device__ __forceinline__ void issue_tile(const TcGroup &R, const CUtensorMap *map, uint32_t sbase, uint32_t full0,
                                           uint32_t full1, int lo, int i, int lane) {
  const uint32_t fb = (i & 1) ? full1 : full0;
  const uint32_t dst = sbase + SB_STG + (uint32_t)((i & 1) * 64 * TPX * 2);
  if (lane == 0) mbar_expect(fb, 64 * TPX * 2);
  __syncwarp();
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int k = lane + 32 * h;
    const int c = R.col[k] >= 0 ? R.col[k] : 0;  // a missing row has weight 0
    tma_row(dst + (uint32_t)(k * TPX * 2), map, lo + i * TPX, c, fb);
  }
}

}  // namespace

// Persistent CTAs over the items (tensor-core group, slab of TSLAB tiles)
// of the groups k_group listed; tensor memory is allocated once per CTA and
// the barriers' phases run on across items.  Within an item the tiles are
// pipelined: tile i is converted into A buffer i & 1 while the product of
// tile i - 1 runs, its product is issued into accumulator i & 1, and the
// accumulator of tile i - 1 is read back and stored while it runs; the rows
// of tile i + 2 stream in by TMA meanwhile.
__global__ void __launch_bounds__(TT, 1) k_interp_tc(DevGrid G, EvalBatch b, const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int t = threadIdx.x, w = t >> 5, lane = t & 31, p = t & (TPX - 1), half = t >> 7;
  const int slabs = (G.npx + TSLAB * TPX - 1) / (TSLAB * TPX);
  const int nitems = *b.tclist_count * slabs;
  if ((int)blockIdx.x >= nitems) return;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
  const uint32_t full0 = sbase + SB_MISC, full1 = full0 + 8, mma0 = full0 + 16, mma1 = full0 + 24;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + SB_MISC + 32);
  int *err = reinterpret_cast<int *>(sm + SB_MISC + 36);
  int *wlo = reinterpret_cast<int *>(sm + SB_WIN), *whi = wlo + SEG, *wmem = whi + SEG;
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(full0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(full1) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mma0) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mma1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    *err = 0;
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sbase + SB_MISC + 32),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  uint32_t uf0 = 0u, uf1 = 0u, um0 = 0u, um1 = 0u;  // completed phases of each barrier
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const TcGroup &R = b.tcrec[b.tclist[item / slabs]];
    const int nm = R.nmem;
    // this item's pixels: tiles over [lo, tc_hi) of the group's window, the
    // tail after tail_start on the CUDA cores
    const int slab0 = (item % slabs) * TSLAB * TPX;
    const int lo = max(R.lo & ~(TPX - 1), slab0), hi = min(R.hi, slab0 + TSLAB * TPX);
    if (lo >= hi) continue;
    if (*err) {  // a wait ran out earlier in this CTA: fail this group as well
      if (t < nm) b.prep[R.member[t]].status = S_TC_TIMEOUT;
      continue;
    }
    const int tc_hi = min(hi, G.tail_start);
    const int ntiles = tc_hi > lo ? (tc_hi - lo + TPX - 1) / TPX : 0;
    const int NP = (nm + 15) & ~15;
    // the members' windows and indices, and the weights: B_j[n][k] = B_j[n][64 + k]
    if (t < SEG) {
      const int e = t < nm ? R.member[t] : -1;
      wlo[t] = e >= 0 ? b.prep[e].i_lo : 0;
      whi[t] = e >= 0 ? b.prep[e].i_hi : 0;
      wmem[t] = e;
    }
    for (int i = t; i < 64 * 64; i += TT) {
      const int n = i >> 6, k = i & 63;
      float wf = 0.0f;
      if (n < nm && R.col[k] >= 0) wf = b.prep[R.member[n]].w[k] * R.f[k];
      const uint32_t h0 = bf16_bits(wf);
      const float r1 = wf - bf16_val(h0);
      const uint32_t h1 = bf16_bits(r1);
      const uint32_t h2 = bf16_bits(r1 - bf16_val(h1));
      unsigned short *b0 = reinterpret_cast<unsigned short *>(sm + SB_B);
      unsigned short *b1 = b0 + 64 * TK, *b2 = b1 + 64 * TK;
      const int o0 = kmaj16(n, k) >> 1, o1 = kmaj16(n, 64 + k) >> 1;
      b0[o0] = b0[o1] = (unsigned short)h0;
      b1[o0] = b1[o1] = (unsigned short)h1;
      b2[o0] = b2[o1] = (unsigned short)h2;
    }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t idesc = idesc_bf16(TPX, NP);
    if (w == 0) {
      if (ntiles > 0) issue_tile(R, &tmap, sbase, full0, full1, lo, 0, lane);
      if (ntiles > 1) issue_tile(R, &tmap, sbase, full0, full1, lo, 1, lane);
    }
    // read back the accumulator of tile j and store its members' pixels:
    // warp w holds pixels 32 (w & 3) .. + 31, columns [half NP/2, (half + 1) NP/2)
    auto epilogue = [&](int j) {
      const int sb = j & 1;
      if (!mbar_wait(sb ? mma1 : mma0, (sb ? um1 : um0) & 1u)) atomicOr(err, 1);
      if (sb) um1++;
      else um0++;
      tc_fence_after();
      const int px = lo + j * TPX + 32 * (w & 3) + lane;
      const uint32_t taddr = tmem + ((uint32_t)(32 * (w & 3)) << 16) + (uint32_t)(sb * 64);
      const int c_lo = half * (NP >> 1), c_hi = c_lo + (NP >> 1);
      for (int c0 = c_lo; c0 < c_hi; c0 += 8) {
        float v[8];
        tmem_ld8(taddr + (uint32_t)c0, v);
#pragma unroll
        for (int q = 0; q < 8; q++) {
          const int n = c0 + q;
          if (n < nm && px >= wlo[n] && px < whi[n] && px < tc_hi) b.bufA[(size_t)wmem[n] * b.stride + px] = v[q];
        }
      }
      tc_fence_before();
    };
    for (int i = 0; i < ntiles; i++) {
      const int sb = i & 1;
      // rows of tile i staged
      if (!mbar_wait(sb ? full1 : full0, (sb ? uf1 : uf0) & 1u)) atomicOr(err, 1);
      if (sb) uf1++;
      else uf0++;
      // convert: pixel p, rows [32 half, 32 half + 32) -> A[p][k] = 256 x high
      // byte, A[p][64 + k] = low byte (A buffer sb: its product two tiles ago
      // was waited for by that tile's read-back)
      {
        const unsigned short *stg = reinterpret_cast<const unsigned short *>(sm + SB_STG + sb * 64 * TPX * 2);
        unsigned char *A = sm + SB_A + sb * TPX * TK * 2;
#pragma unroll
        for (int k8 = 32 * half; k8 < 32 * half + 32; k8 += 8) {
          uint32_t h[4], l[4];
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const uint32_t u0 = stg[(k8 + 2 * q) * TPX + p], u1 = stg[(k8 + 2 * q + 1) * TPX + p];
            // exact floats of the byte planes (below 2^23): f = bits(0x4B000000 | x) - 2^23
            const float2 fh = __fadd2_rn(make_float2(__uint_as_float(0x4B000000u | (u0 & 0xFF00u)),
                                                     __uint_as_float(0x4B000000u | (u1 & 0xFF00u))),
                                         make_float2(-8388608.0f, -8388608.0f));
            const float2 fl = __fadd2_rn(make_float2(__uint_as_float(0x4B000000u | (u0 & 0xFFu)),
                                                     __uint_as_float(0x4B000000u | (u1 & 0xFFu))),
                                         make_float2(-8388608.0f, -8388608.0f));
            // at most 8 significant bits: the bf16 value is the top half of the f32
            h[q] = __byte_perm(__float_as_uint(fh.x), __float_as_uint(fh.y), 0x7632);
            l[q] = __byte_perm(__float_as_uint(fl.x), __float_as_uint(fl.y), 0x7632);
          }
          *reinterpret_cast<uint4 *>(A + kmaj16(p, k8)) = make_uint4(h[0], h[1], h[2], h[3]);
          *reinterpret_cast<uint4 *>(A + kmaj16(p, 64 + k8)) = make_uint4(l[0], l[1], l[2], l[3]);
        }
      }
      proxy_fence();
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      if (*err) break;
      if (w == 0) {
        // the staging buffer is free again: tile i + 2 streams in
        if (i + 2 < ntiles) issue_tile(R, &tmap, sbase, full0, full1, lo, i + 2, lane);
        if (lane == 0) {
          const uint64_t da = desc16(sbase + SB_A + (uint32_t)(sb * TPX * TK * 2));
#pragma unroll
          for (int j = 0; j < 3; j++) {
            const uint64_t db = desc16(sbase + SB_B + (uint32_t)(j * 64 * TK * 2));
#pragma unroll
            for (int ks = 0; ks < TK / 16; ks++)
              mma_bf16(tmem + (uint32_t)(sb * 64), da + (uint64_t)((ks * 256) >> 4), db + (uint64_t)((ks * 256) >> 4),
                       idesc, (j | ks) ? 1u : 0u);
          }
          mma_commit(sb ? mma1 : mma0);
        }
        __syncwarp();
      }
      if (i > 0) epilogue(i - 1);
    }
    bool ok = *err == 0;
    if (ok && ntiles > 0) epilogue(ntiles - 1);
    __syncthreads();
    ok = *err == 0;
    // tail pixels [tail_start, hi): the reference's extra 1/65535 (interpolate.rs:978)
    if (ok && hi > G.tail_start) {
      const int t0 = max(lo, G.tail_start);
      const int npx = hi - t0;
      for (int i = t; i < npx * nm; i += TT) {
        const int n = i / npx, px = t0 + i % npx;
        if (px < wlo[n] || px >= whi[n]) continue;
        const EvalPrep &P = b.prep[wmem[n]];
        float acc = 0.0f;
        for (int k = 0; k < 64; k++) {
          const int c = R.col[k];
          if (c < 0) continue;
          const float x = (float)G.spectra[(size_t)c * G.stride + px];
          acc = fmaf(P.w[k], __fmul_rn(__fdiv_rn(x, 65535.0f), R.f[k]), acc);
        }
        b.bufA[(size_t)wmem[n] * b.stride + px] = acc;
      }
    }
    if (!ok && t < nm) b.prep[R.member[t]].status = S_TC_TIMEOUT;
    __syncthreads();  // the windows and weights are rewritten for the next item
  }
  // a tile whose barrier wait ran out may still have copies or products in
  // flight: wait for them once more (bounded) before freeing tensor memory
  if (*err && t == 0) {
    mbar_wait(full0, uf0 & 1u);
    mbar_wait(full1, uf1 & 1u);
    mbar_wait(mma0, um0 & 1u);
    mbar_wait(mma1, um1 & 1u);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (w == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS));
}

void launch_interp_tc(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0 || !b.tcrec || !b.tmap) return;
  static int per_sm[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  int fit = 1;
  if (dev >= 0 && dev < 64) {
    if (!per_sm[dev]) {
      cudaFuncSetAttribute(k_interp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, SB_TOTAL);
      int n = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_interp_tc, TT, SB_TOTAL) != cudaSuccess || n < 1) n = 1;
      per_sm[dev] = n;
    }
    fit = per_sm[dev];
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // persistent: the CTAs that fit at once; each takes items in grid strides
  k_interp_tc<<<sms * fit, TT, SB_TOTAL, s>>>(G, b, *reinterpret_cast<const CUtensorMap *>(b.tmap));
  count_launch();
}

// The grid as a 2D uint16 tensor [rows][stride] for TMA, box 128 x 1.
bool make_grid_tensor_map(const uint16_t *spectra, int64_t rows, int64_t stride, void *out) {
  typedef CUresult (*EncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                               const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                               CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      return false;
    fn = reinterpret_cast<EncodeFn>(p);
  }
  const cuuint64_t dims[2] = {(cuuint64_t)stride, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)stride * 2};
  const cuuint32_t box[2] = {(cuuint32_t)TPX, 1};
  const cuuint32_t estr[2] = {1, 1};
  return fn(reinterpret_cast<CUtensorMap *>(out), CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, (void *)spectra, dims, strides,
            box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace pb
