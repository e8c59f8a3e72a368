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
// other members of the group.  B is stored once for the 64 rows; the MMAs
// of both byte planes read it.
//
// One persistent CTA per SM, its warps specialised and handing tiles on
// through mbarriers, so that staging, conversion, products and stores of
// different tiles overlap:
//   warp 0      TMA producer: the 64 rows of a tile (16 tile::gather4
//               loads of four 128-pixel rows each, from the grid resident in
//               this GPU's own memory, each CTA loading for itself) into a ring of NSTG staging
//               buffers;
//   warp 1      one thread issues the 24 tcgen05.mma of a tile (kind::f16,
//               M = 128, N = members rounded up to 16) into one of ND
//               tensor-memory accumulators;
//   warps 2-9   converters: staging -> the bf16 byte planes of A (a ring of
//               NA buffers), and each item's B (two buffers, so the next
//               item's weights are written while the last tiles of the
//               current one multiply);
//   warps 10-13 epilogue: tcgen05.ld of an accumulator (warp w reads lanes
//               32 (w % 4) .. + 31), release, then the members' stores.
// The last npx % 128 pixels carry the reference's extra 1/65535
// (interpolate.rs:978) and are computed on the CUDA cores by the epilogue
// warps.
//
// Every wait on an mbarrier is bounded (about a second); a wait that runs
// out marks the CTA's groups with an internal error, the other roles stop at
// their next wait or tile, outstanding copies and products are waited for
// (bounded) and the CTA still frees its tensor memory.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "kernels.h"

namespace pb {

namespace {

constexpr int TPX = 128;           // pixels per tile (MMA M)
constexpr int TK = 128;            // A's reduction: 64 rows x {256 x high byte, low byte}
constexpr int BK = 64;             // B's reduction: the 64 rows, read by both planes' MMAs
constexpr int NSTG = 4;            // staging ring (raw rows)
constexpr int NA = 2;              // A ring
constexpr int ND = 4;              // accumulators in tensor memory
constexpr int DCOLS = 64;          // columns of an accumulator (members)
constexpr int TMEM_COLS = ND * DCOLS;
constexpr int TSLAB = 64;          // tiles per item
constexpr int S_TC_TIMEOUT = -99;  // PASTA_E_INTERNAL

// warp roles
constexpr int W_TMA = 0, W_MMA = 1, W_CV = 2, N_CV = 8, W_EP = W_CV + N_CV, N_EP = 4;
constexpr int TT = 32 * (W_EP + N_EP);  // 448 threads
constexpr int CVT = 32 * N_CV;          // converter threads

// shared memory (bytes): staging ring [64 rows][128 pixels] u16, A ring
// [128 pixels][128] bf16 (K-major), two B buffers of three parts
// [64 members][64] bf16 (K-major), barriers, flags, the epilogue's member table
constexpr int SZ_STG = 64 * TPX * 2;
constexpr int SZ_A = TPX * TK * 2;
constexpr int SZ_BP = 64 * BK * 2;
constexpr int SB_STG = 0;
constexpr int SB_A = SB_STG + NSTG * SZ_STG;
constexpr int SB_B = SB_A + NA * SZ_A;
constexpr int SB_BAR = SB_B + 2 * 3 * SZ_BP;
// barrier indices
constexpr int B_SFULL = 0, B_SEMPTY = B_SFULL + NSTG, B_AFULL = B_SEMPTY + NSTG, B_AEMPTY = B_AFULL + NA,
              B_DFULL = B_AEMPTY + NA, B_DEMPTY = B_DFULL + ND, B_BFULL = B_DEMPTY + ND, B_BEMPTY = B_BFULL + 2,
              B_DRAIN = B_BEMPTY + 2, NBAR = B_DRAIN + 1;
constexpr int SB_MISC = SB_BAR + NBAR * 8;  // tensor-memory address, error flag
constexpr int SB_EPI = (SB_MISC + 16 + 15) & ~15;  // per member: row pointer (8 B), window lo, hi
constexpr int SB_TOTAL = SB_EPI + 64 * 16;
static_assert(SB_A % 1024 == 0 && SB_B % 1024 == 0 && SB_BAR % 8 == 0, "shared layout");
static_assert(SB_TOTAL <= 227 * 1024, "shared memory of one CTA");

// byte offset of element (row, k) of a K-major bf16 tile with KX elements
// per row: core matrices of 8 rows x 16 bytes (8 elements), K-adjacent core
// matrices 128 bytes apart, 8-row groups KX / 8 core matrices apart
template <int KX>
__device__ __forceinline__ int kmaj16(int row, int k) {
  return ((((row >> 3) * (KX >> 3) + (k >> 3)) << 3) + (row & 7)) * 16 + (k & 7) * 2;
}
// shared-memory matrix descriptor of such a tile (no swizzle, version 1)
template <int KX>
__device__ __forceinline__ uint64_t desc16(uint32_t saddr) {
  const uint64_t lbo = 128, sbo = (KX >> 3) * 128;
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
__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(mbar) : "memory");
}
// wait for the completion of the barrier's phase with the given parity;
// false after about a second (2e9 clocks)
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
// a wait by all lanes of a warp; false for every lane when any lane's wait
// ran out or another role has stopped (the flag is set on a timeout)
__device__ __forceinline__ bool warp_wait(uint32_t mbar, uint32_t parity, volatile int *err) {
  const bool ok = mbar_wait(mbar, parity);
  if (!ok) *err = 1;
  return __all_sync(0xffffffffu, ok) && !__any_sync(0xffffffffu, *err != 0);
}
__device__ __forceinline__ bool warp_stop(volatile int *err) { return __any_sync(0xffffffffu, *err != 0); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// named barrier of the epilogue warps
__device__ __forceinline__ void ep_sync() { asm volatile("bar.sync 1, %0;\n" ::"n"(32 * N_EP) : "memory"); }
// the same barrier, returning to every epilogue thread whether any of them passed true
__device__ __forceinline__ bool ep_any(bool pred) {
  int r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.b32 p, %1, 0;\n\tbar.red.or.pred q, 1, %2, p;\n\tselp.s32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((int)pred), "n"(32 * N_EP)
      : "memory");
  return r != 0;
}

// TMA gather of four rows (one 128-pixel box each) into four consecutive boxes
__device__ __forceinline__ void tma_gather4(uint32_t dst, const CUtensorMap *map, int x, const int (&y)[4], uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n" ::
          "r"(dst), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y[0]), "r"(y[1]), "r"(y[2]), "r"(y[3]), "r"(mbar)
      : "memory");
}
__device__ __forceinline__ void mbar_expect(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(mbar), "r"(bytes) : "memory");
}

// eight consecutive f32 columns of this thread's tensor-memory lane (no wait)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}
// store v to p when ok, as one predicated instruction (no branch).  No
// memory clobber: the interpolated rows are not read in this kernel, so the
// loads of the next row pointers may move above these stores.
__device__ __forceinline__ void st_if(float *p, float v, bool ok) {
  asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.global.f32 [%0], %1;\n\t}\n" ::"l"(p), "f"(v),
               "r"((int)ok));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// bf16 bits of x (round to nearest even), as the low 16 bits
__device__ __forceinline__ uint32_t bf16_bits(float x) {
  uint32_t r;
  asm("{\n\t.reg .b16 h;\n\tcvt.rn.bf16.f32 h, %1;\n\tmov.b32 %0, {h, h};\n\t}" : "=r"(r) : "f"(x));
  return r & 0xFFFFu;
}
__device__ __forceinline__ float bf16_val(uint32_t bits) { return __uint_as_float(bits << 16); }

// An item: tiles of one tensor-core group over one slab of TSLAB tiles.
// Every role derives the same items, in the same order, from the group list.
struct TcItem {
  const TcGroup *R;
  int nm, NP;       // members, MMA N (members rounded up to 16)
  int lo, hi;       // pixels [lo, hi) of this item; lo a multiple of 128
  int tc_hi;        // tiles cover [lo, tc_hi); [max(lo, tail_start), hi) is the tail
  int ntiles;
};
__device__ __forceinline__ bool tc_item(const DevGrid &G, const EvalBatch &b, int item, int slabs, TcItem &I) {
  I.R = &b.tcrec[b.tclist[item / slabs]];
  I.nm = I.R->nmem;
  I.NP = (I.nm + 15) & ~15;
  const int slab0 = (item % slabs) * TSLAB * TPX;
  I.lo = max(I.R->lo & ~(TPX - 1), slab0);
  I.hi = min(I.R->hi, slab0 + TSLAB * TPX);
  I.tc_hi = min(I.hi, G.tail_start);
  I.ntiles = I.tc_hi > I.lo ? (I.tc_hi - I.lo + TPX - 1) / TPX : 0;
  return I.lo < I.hi;
}

}  // namespace

// Persistent CTAs over the items (tensor-core group, slab of TSLAB tiles)
// of the groups k_group listed, item = blockIdx.x, blockIdx.x + gridDim.x,
// ...; tensor memory is allocated once per CTA and every ring's phases run
// on across items.  Ring slot of the g-th use (g counted over the CTA's
// tiles): g % size; its full barrier completes for the (g / size)-th time
// (parity (g / size) & 1), and a producer's (g / size)-th reuse (>= 1) of a
// slot waits for the consumers' release of the previous use.
__global__ void __launch_bounds__(TT, 1) k_interp_tc(DevGrid G, EvalBatch b, const __grid_constant__ CUtensorMap tmap) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const int t = threadIdx.x, w = t >> 5, lane = t & 31;
  const int slabs = (G.npx + TSLAB * TPX - 1) / (TSLAB * TPX);
  const int nitems = *b.tclist_count * slabs;
  if ((int)blockIdx.x >= nitems) return;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
  auto bar = [&](int i) { return sbase + SB_BAR + 8u * (uint32_t)i; };
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + SB_MISC);
  volatile int *err = reinterpret_cast<volatile int *>(sm + SB_MISC + 4);
  if (t == 0) {
    for (int i = 0; i < NSTG; i++) {
      mbar_init(bar(B_SFULL + i), 1);
      mbar_init(bar(B_SEMPTY + i), N_CV);
    }
    for (int i = 0; i < NA; i++) {
      mbar_init(bar(B_AFULL + i), N_CV);
      mbar_init(bar(B_AEMPTY + i), 1);
    }
    for (int i = 0; i < ND; i++) {
      mbar_init(bar(B_DFULL + i), 1);
      mbar_init(bar(B_DEMPTY + i), N_EP);
    }
    for (int i = 0; i < 2; i++) {
      mbar_init(bar(B_BFULL + i), N_CV);
      mbar_init(bar(B_BEMPTY + i), 1);
    }
    mbar_init(bar(B_DRAIN), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    *err = 0;
  }
  if (w == W_TMA) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sbase + SB_MISC),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  if (w == W_TMA) {
    // ---------------------------------------------------------- producer
    long long g = 0;  // tiles issued
    bool stop = false;
    for (int item = blockIdx.x; item < nitems && !stop; item += gridDim.x) {
      TcItem I;
      if (!tc_item(G, b, item, slabs, I)) continue;
      // the rows of this group (a missing row has weight 0: row 0 stands in);
      // lane l < 16 gathers rows 4l .. 4l + 3
      const int k0 = 4 * (lane & 15);
      int rr[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int c = I.R->col[k0 + j];
        rr[j] = c >= 0 ? c : 0;
      }
      for (int i = 0; i < I.ntiles; i++, g++) {
        const int s = (int)(g % NSTG);
        const long long u = g / NSTG;
        stop = u >= 1 ? !warp_wait(bar(B_SEMPTY + s), (uint32_t)((u - 1) & 1), err) : warp_stop(err);
        if (stop) break;
        if (lane == 0) mbar_expect(bar(B_SFULL + s), SZ_STG);
        __syncwarp();
        const uint32_t dst = sbase + SB_STG + (uint32_t)(s * SZ_STG);
        const int x = I.lo + i * TPX;
        if (lane < 16) tma_gather4(dst + (uint32_t)(k0 * TPX * 2), &tmap, x, rr, bar(B_SFULL + s));
      }
    }
    // every issued copy has landed before the CTA leaves (bounded)
    if (lane == 0)
      for (long long q = g - 1; q >= 0 && q >= g - NSTG; q--) mbar_wait(bar(B_SFULL + (int)(q % NSTG)), (uint32_t)((q / NSTG) & 1));
    __syncwarp();
  } else if (w == W_MMA) {
    // ------------------------------------------------------------- MMA
    if (lane == 0) {
      long long g = 0;   // tiles multiplied
      long long it = 0;  // items
      for (int item = blockIdx.x; item < nitems && !*err; item += gridDim.x) {
        TcItem I;
        if (!tc_item(G, b, item, slabs, I)) continue;
        const int bb = (int)(it & 1);
        if (!mbar_wait(bar(B_BFULL + bb), (uint32_t)((it >> 1) & 1))) *err = 1;
        tc_fence_after();
        const uint32_t idesc = idesc_bf16(TPX, I.NP);
        for (int i = 0; i < I.ntiles && !*err; i++, g++) {
          const int a = (int)(g % NA), d = (int)(g % ND);
          if (!mbar_wait(bar(B_AFULL + a), (uint32_t)((g / NA) & 1))) *err = 1;
          if (g >= ND && !mbar_wait(bar(B_DEMPTY + d), (uint32_t)((g / ND - 1) & 1))) *err = 1;
          if (*err) break;
          tc_fence_after();
          const uint64_t da = desc16<TK>(sbase + SB_A + (uint32_t)(a * SZ_A));
          const uint32_t td = tmem + (uint32_t)(d * DCOLS);
#pragma unroll
          for (int j = 0; j < 3; j++) {
            const uint64_t db = desc16<BK>(sbase + SB_B + (uint32_t)((bb * 3 + j) * SZ_BP));
#pragma unroll
            for (int ks = 0; ks < TK / 16; ks++)
              mma_bf16(td, da + (uint64_t)((ks * 256) >> 4), db + (uint64_t)(((ks & 3) * 256) >> 4), idesc,
                       (j | ks) ? 1u : 0u);
          }
          mma_commit(bar(B_AEMPTY + a));  // A slot free once these products have read it
          mma_commit(bar(B_DFULL + d));   // accumulator ready
        }
        mma_commit(bar(B_BEMPTY + bb));  // this item's weights are free
        it++;
      }
      // every product has completed before tensor memory is freed (bounded)
      mma_commit(bar(B_DRAIN));
      mbar_wait(bar(B_DRAIN), 0u);
    }
    __syncwarp();
  } else if (w < W_EP) {
    // ------------------------------------------------------ converters
    const int c = t - 32 * W_CV;  // 0 .. CVT - 1
    const int p = c & (TPX - 1), half = c >> 7;
    long long g = 0, it = 0;
    bool stop = false;
    for (int item = blockIdx.x; item < nitems && !stop; item += gridDim.x) {
      TcItem I;
      if (!tc_item(G, b, item, slabs, I)) continue;
      // this item's weights: B_j[n][k] = part j of weight_n,k x factor_k
      const int bb = (int)(it & 1);
      stop = it >= 2 ? !warp_wait(bar(B_BEMPTY + bb), (uint32_t)(((it >> 1) - 1) & 1), err) : warp_stop(err);
      if (stop) break;
      {
        unsigned short *b0 = reinterpret_cast<unsigned short *>(sm + SB_B + bb * 3 * SZ_BP);
        unsigned short *b1 = b0 + SZ_BP / 2, *b2 = b1 + SZ_BP / 2;
        for (int i = c; i < 64 * BK; i += CVT) {
          const int n = i >> 6, k = i & 63;
          const int col = I.R->col[k];
          float wf = 0.0f;
          if (n < I.nm && col >= 0) wf = b.prep[I.R->member[n]].w[k] * I.R->f[k];
          const uint32_t h0 = bf16_bits(wf);
          const float r1 = wf - bf16_val(h0);
          const uint32_t h1 = bf16_bits(r1);
          const uint32_t h2 = bf16_bits(r1 - bf16_val(h1));
          const int o = kmaj16<BK>(n, k) >> 1;
          b0[o] = (unsigned short)h0;
          b1[o] = (unsigned short)h1;
          b2[o] = (unsigned short)h2;
        }
        proxy_fence();
        __syncwarp();
        if (lane == 0) mbar_arrive(bar(B_BFULL + bb));
      }
      it++;
      for (int i = 0; i < I.ntiles; i++, g++) {
        const int s = (int)(g % NSTG), a = (int)(g % NA);
        stop = !warp_wait(bar(B_SFULL + s), (uint32_t)((g / NSTG) & 1), err);
        if (stop) break;
        // pixel p, rows [32 half, 32 half + 32) of the staged tile
        const unsigned short *stg = reinterpret_cast<const unsigned short *>(sm + SB_STG + s * SZ_STG);
        uint32_t u[32];
#pragma unroll
        for (int k = 0; k < 32; k++) u[k] = stg[(32 * half + k) * TPX + p];
        __syncwarp();
        if (lane == 0) mbar_arrive(bar(B_SEMPTY + s));
        // A slot a: its products two tiles ago have completed
        stop = g >= NA ? !warp_wait(bar(B_AEMPTY + a), (uint32_t)((g / NA - 1) & 1), err) : false;
        if (stop) break;
        unsigned char *A = sm + SB_A + a * SZ_A;
#pragma unroll
        for (int k8 = 0; k8 < 32; k8 += 8) {
          uint32_t h[4], l[4];
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const uint32_t u0 = u[k8 + 2 * q], u1 = u[k8 + 2 * q + 1];
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
          const int k = 32 * half + k8;
          *reinterpret_cast<uint4 *>(A + kmaj16<TK>(p, k)) = make_uint4(h[0], h[1], h[2], h[3]);
          *reinterpret_cast<uint4 *>(A + kmaj16<TK>(p, 64 + k)) = make_uint4(l[0], l[1], l[2], l[3]);
        }
        proxy_fence();
        __syncwarp();
        if (lane == 0) mbar_arrive(bar(B_AFULL + a));
      }
    }
  } else {
    // -------------------------------------------------------- epilogue
    const int e = t - 32 * W_EP;  // 0 .. 127
    const int q = w & 3;          // tensor-memory lanes 32 q .. 32 q + 31
    float **rowp = reinterpret_cast<float **>(sm + SB_EPI);
    int *wlo = reinterpret_cast<int *>(sm + SB_EPI + 64 * 8), *whi = wlo + 64;
    long long g = 0;
    bool stop = false;  // uniform within a warp; made uniform over the epilogue warps at each item
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
      TcItem I;
      if (!tc_item(G, b, item, slabs, I)) continue;
      // the previous item's table is no longer read; stop together
      if (ep_any(stop || *err != 0)) break;
      if (e < 64) {
        const int m = e < I.nm ? I.R->member[e] : -1;
        rowp[e] = m >= 0 ? b.bufA + (size_t)m * b.stride : b.bufA;
        wlo[e] = m >= 0 ? b.prep[m].i_lo : 0;
        whi[e] = m >= 0 ? b.prep[m].i_hi : 0;
      }
      ep_sync();
      // pixels inside every member's window need no per-member test
      int all_lo = 0, all_hi = 1 << 30;
      for (int n = 0; n < I.nm; n++) {
        all_lo = max(all_lo, wlo[n]);
        all_hi = min(all_hi, whi[n]);
      }
      all_hi = min(all_hi, I.tc_hi);
      // after a stop the tiles are passed over without waits (the count stays
      // in step) until the next item's vote
      for (int i = 0; i < I.ntiles; i++, g++) {
        const int d = (int)(g % ND);
        if (!stop) stop = !warp_wait(bar(B_DFULL + d), (uint32_t)((g / ND) & 1), err);
        if (stop) continue;
        tc_fence_after();
        float v[DCOLS];
        const uint32_t taddr = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(d * DCOLS);
#pragma unroll
        for (int c0 = 0; c0 < DCOLS; c0 += 8)
          if (c0 < I.NP) tmem_ld8(taddr + (uint32_t)c0, v + c0);
        tmem_wait_ld();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(bar(B_DEMPTY + d));
        // straight-line predicated stores, 8 columns per (uniform) step; a
        // warp whose pixels all lie inside every member's window tests only
        // the member count
        const int px = I.lo + i * TPX + 32 * q + lane;
        if (__all_sync(0xffffffffu, px >= all_lo && px < all_hi)) {
#pragma unroll
          for (int c0 = 0; c0 < DCOLS; c0 += 8)
            if (c0 < I.NP) {
#pragma unroll
              for (int j = 0; j < 8; j++) st_if(rowp[c0 + j] + px, v[c0 + j], c0 + j < I.nm);
            }
        } else {
#pragma unroll
          for (int c0 = 0; c0 < DCOLS; c0 += 8)
            if (c0 < I.NP) {
#pragma unroll
              for (int j = 0; j < 8; j++) {
                const int n = c0 + j;
                st_if(rowp[n] + px, v[n], n < I.nm && px >= wlo[n] && px < whi[n] && px < I.tc_hi);
              }
            }
        }
      }
      // tail pixels [tail_start, hi): the reference's extra 1/65535 (interpolate.rs:978)
      if (!stop && I.hi > G.tail_start) {
        const int t0 = max(I.lo, G.tail_start);
        const int npx = I.hi - t0;
        for (int j = e; j < npx * I.nm; j += 32 * N_EP) {
          const int n = j / npx, px = t0 + j % npx;
          if (px < wlo[n] || px >= whi[n]) continue;
          const EvalPrep &P = b.prep[I.R->member[n]];
          float acc = 0.0f;
          for (int k = 0; k < 64; k++) {
            const int col = I.R->col[k];
            if (col < 0) continue;
            const float x = (float)G.spectra[(size_t)col * G.stride + px];
            acc = fmaf(P.w[k], __fmul_rn(__fdiv_rn(x, 65535.0f), I.R->f[k]), acc);
          }
          rowp[n][px] = acc;
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (*err) {  // every group this CTA took part in fails
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
      const TcGroup &R = b.tcrec[b.tclist[item / slabs]];
      for (int n = t; n < R.nmem; n += TT) b.prep[R.member[n]].status = S_TC_TIMEOUT;
    }
  }
  if (w == W_TMA) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TMEM_COLS));
}

void launch_interp_tc(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0 || !b.tcrec || !b.tmap) return;
  static bool attr[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !attr[dev]) {
    cudaFuncSetAttribute(k_interp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, SB_TOTAL);
    attr[dev] = true;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // persistent: one CTA per SM; each takes items in grid strides
  k_interp_tc<<<sms, TT, SB_TOTAL, s>>>(G, b, *reinterpret_cast<const CUtensorMap *>(b.tmap));
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
