// kernels.cu -- the bandwidth, FFT and reduction kernels of the hot path.
//
// Buffer protocol per evaluation e (rows of `stride` floats):
//   k_interp writes the interpolated spectrum to A.
//   k_broaden (rotation FFT + instrument profile, fused) reads A and writes
//   the broadened synth row to B, or in chi2 batches the model resampled
//   to the observed pixels (EvalPrep::epi).
//   Very wide kernels (m - 1 + 2 hg > 2048 - 128) take the unfused pair
//   k_rot (A -> B) and k_gauss (B -> A, or A -> B when the rotation is the
//   identity).  EvalPrep::final_in_b says where the synth row is.
//   k_resample_obs resamples the synth rows k_broaden did not, into the
//   other buffer (EvalPrep::mobs_in_b); the chi2 kernels read that model.
//   k_resample_out / k_copy_broadened serve the model entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

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
// (interpolate.rs:954-981).  Particles of one star soon sit in the same grid
// cube and then read the same 64 rows, so evaluations are grouped first:
// k_group finds, among SEG consecutive evaluations, those with identical
// neighbour columns and records each group's rows once.  k_interp then
// converts every row tile once per group and applies each member's weights
// to it: the reads and the u16 -> f32 conversions are shared, each member
// keeps its own accumulators, and each member's sum runs over its rows in
// reference order (rows another member needs add exactly 0), so the result
// is the same as interpolating every evaluation alone.

__device__ __forceinline__ unsigned long long cols_hash(const int *c) {
  unsigned long long h = 1469598103934665603ull;  // FNV-1a over the 64 indices
  for (int n = 0; n < 64; n++) h = (h ^ (unsigned)c[n]) * 1099511628211ull;
  return h;
}

// Segment s of a batch: [start, start + len), a chunk of at most SEG
// evaluations of one star (EvalBatch::seg_len), len <= 0 when empty.
__device__ __forceinline__ void seg_range(const EvalBatch &b, int s, int &start, int &len) {
  const int L = b.seg_len > 0 ? b.seg_len : b.E;
  const int spb = (L + SEG - 1) / SEG;
  const int j = s / spb, q = s - j * spb;
  start = j * L + q * SEG;
  len = min(min(SEG, L - q * SEG), b.E - start);
}
int num_segments(const EvalBatch &b) {
  if (b.E <= 0) return 0;
  const int L = b.seg_len > 0 ? b.seg_len : b.E;
  return (b.E + L - 1) / L * ((L + SEG - 1) / SEG);
}

// One CTA per segment: slice 0 (SEG threads) finds the groups, then
// GROUP_SLICES slices of SEG threads write the group records, one group per
// slice at a time (thread t of a slice handles neighbour row t).  Columns
// shared by TC_MIN_MEMBERS or more evaluations form tensor-core groups
// (with the tensor-core path on); the others form groups of up to GROUP_MAX.
constexpr int GROUP_SLICES = 4;
__global__ void __launch_bounds__(SEG *GROUP_SLICES) k_group(DevGrid G, EvalBatch b) {
  __shared__ unsigned long long hs[SEG];
  __shared__ int ok[SEG], lead[SEG], gid[SEG], slot[SEG], open_g[SEG], fill[SEG], cnt_l[SEG], tcg[SEG];
  __shared__ int ng, ntc;
  __shared__ int cnt[GROUP_SLICES][2];
  __shared__ int mem[GROUP_SLICES][GROUP_MAX];
  const int s = blockIdx.x, tid = threadIdx.x, t = tid % SEG, sl = tid / SEG;
  int start, len;
  seg_range(b, s, start, len);
  if (len <= 0) {
    if (tid == 0) {
      b.gcount[s] = 0;
      if (b.tccount) b.tccount[s] = 0;
    }
    return;
  }
  const int e = start + t;
  if (sl == 0) {
    const bool v = t < len && b.prep[e].status == 0;
    ok[t] = v;
    hs[t] = v ? cols_hash(b.prep[e].cols) : 0ull;
    cnt_l[t] = 0;
    tcg[t] = -1;
  }
  __syncthreads();
  if (sl == 0) {  // leader: the first earlier evaluation with the same columns
    int L = ok[t] ? t : -1;
    if (ok[t]) {
      const int *c = b.prep[e].cols;
      for (int u = 0; u < t; u++) {
        if (!ok[u] || hs[u] != hs[t]) continue;
        const int *cu = b.prep[start + u].cols;
        bool same = true;
        for (int n = 0; n < 64 && same; n++) same = cu[n] == c[n];
        if (same) {
          L = u;
          break;
        }
      }
      atomicAdd(&cnt_l[L], 1);
    }
    lead[t] = L;
    open_g[t] = -1;
    fill[t] = 0;
  }
  __syncthreads();
  if (tid == 0) {
    // tensor-core groups, in leader order
    int nt = 0;
    if (b.tcrec)
      for (int u = 0; u < SEG; u++)
        if (ok[u] && lead[u] == u && cnt_l[u] >= max(b.tc_min, TC_MIN_MEMBERS) && nt < TC_MAX_GROUPS) tcg[u] = nt++;
    ntc = nt;
    if (b.tccount) b.tccount[s] = nt;
    if (nt > 0) {
      const int at = atomicAdd(b.tclist_count, nt);
      for (int k = 0; k < nt; k++) b.tclist[at + k] = start + k;
    }
    // the other evaluations in groups of at most GROUP_MAX, in evaluation order
    int n = 0;
    for (int u = 0; u < SEG; u++) {
      gid[u] = -1;
      if (!ok[u] || tcg[lead[u]] >= 0) continue;
      const int l = lead[u];
      if (open_g[l] < 0 || fill[l] == GROUP_MAX) {
        open_g[l] = n++;
        fill[l] = 0;
      }
      gid[u] = open_g[l];
      slot[u] = fill[l]++;
    }
    ng = n;
    b.gcount[s] = n;
  }
  __syncthreads();
  if (sl == 0 && b.mkey && ok[t] && tcg[lead[t]] < 0 && cnt_l[lead[t]] == 1) {
    // alone in its segment: offer it to the batch-wide table of column sets
    const unsigned long long key = hs[t] | 1ull;
    unsigned slot = (unsigned)(key ^ (key >> 31)) & (unsigned)(b.mtab - 1);
    for (int probe = 0; probe < b.mtab; probe++) {  // the table is at most half full
      const unsigned long long old = atomicCAS(&b.mkey[slot], 0ull, key);
      if (old == 0ull || old == key) break;
      slot = (slot + 1) & (unsigned)(b.mtab - 1);
    }
    const int r = atomicAdd(&b.mcnt[slot], 1);
    if (r < MERGE_CAP) b.mmem[(size_t)slot * MERGE_CAP + r] = e;
    if (r == 1) b.mslot[1 + atomicAdd(&b.mslot[0], 1)] = (int)slot;
    b.erec[e] = start + gid[t];
  }
  // tensor-core group records: slice sl writes groups sl, sl + GROUP_SLICES,
  // ... (thread t: row t, member t)
  for (int tg = sl; tg < ntc; tg += GROUP_SLICES) {
    int l = -1;
    for (int u = 0; u < SEG; u++)
      if (ok[u] && lead[u] == u && tcg[u] == tg) l = u;
    TcGroup &T = b.tcrec[start + tg];
    const int c = b.prep[start + l].cols[t];
    T.col[t] = c;
    T.f[t] = c >= 0 ? G.factor[c] : 0.0f;
    // members in evaluation order: the rank of t among the group's members
    const bool mine = ok[t] && lead[t] == l;
    const unsigned bal = __ballot_sync(0xffffffffu, mine);
    const int lane = t & 31;
    if (lane == 0) cnt[sl][t >> 5] = __popc(bal);
    asm volatile("bar.sync %0, %1;" ::"r"(1 + sl), "r"(SEG) : "memory");  // this slice's two warps
    if (mine) T.member[__popc(bal & ((1u << lane) - 1u)) + ((t >> 5) ? cnt[sl][0] : 0)] = e;
    if (t == 0) {
      int lo = 1 << 30, hi = 0;
      for (int u = 0; u < SEG; u++)
        if (ok[u] && lead[u] == l) {
          lo = min(lo, b.prep[start + u].i_lo);
          hi = max(hi, b.prep[start + u].i_hi);
        }
      T.nmem = cnt_l[l];
      T.lo = lo;
      T.hi = hi;
    }
    asm volatile("bar.sync %0, %1;" ::"r"(1 + sl), "r"(SEG) : "memory");  // cnt[sl] is reused
  }
  __syncthreads();
  const int lane = tid & 31, wsl = t >> 5;  // warp within the slice
  for (int base = 0; base < ng; base += GROUP_SLICES) {
    const int g = base + sl;
    const bool act = g < ng;
    if (t < GROUP_MAX) mem[sl][t] = -1;
    __syncthreads();
    if (act && gid[t] == g) mem[sl][slot[t]] = e;
    __syncthreads();
    GroupRec &R = b.grec[(size_t)start + (act ? g : 0)];
    int c = -1, nm = 0;
    float f = 0.0f, w[GROUP_MAX], wf[GROUP_MAX];
    unsigned bal = 0u;
    bool keep = false;
    if (act) {
      for (int m = 0; m < GROUP_MAX; m++) nm += mem[sl][m] >= 0;
      // row t of the group: kept when any member weighs it
      c = b.prep[mem[sl][0]].cols[t];
      f = c >= 0 ? G.factor[c] : 0.0f;
#pragma unroll
      for (int m = 0; m < GROUP_MAX; m++) {
        w[m] = (mem[sl][m] >= 0 && c >= 0) ? b.prep[mem[sl][m]].w[t] : 0.0f;
        wf[m] = w[m] * f;
        keep |= wf[m] != 0.0f;
      }
      bal = __ballot_sync(0xffffffffu, keep);
      if (lane == 0) cnt[sl][wsl] = __popc(bal);
    }
    __syncthreads();
    if (act) {
      const int pos = __popc(bal & ((1u << lane) - 1u)) + (wsl ? cnt[sl][0] : 0);
      if (keep) {
        R.wf[pos][0] = make_float4(wf[0], wf[1], wf[2], wf[3]);
        R.wf[pos][1] = make_float4(wf[4], wf[5], wf[6], wf[7]);
        R.w[pos][0] = make_float4(w[0], w[1], w[2], w[3]);
        R.w[pos][1] = make_float4(w[4], w[5], w[6], w[7]);
        R.col[pos] = c;
        R.f[pos] = f;
      }
      const int kept = cnt[sl][0] + cnt[sl][1];
      const int padded = (kept + 7) & ~7;
      if (t >= kept && t < padded) {  // zero-weight padding rows (add exactly 0)
        const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        R.wf[t][0] = R.wf[t][1] = R.w[t][0] = R.w[t][1] = z4;
        R.col[t] = 0;
        R.f[t] = 0.0f;
      }
      if (t < GROUP_MAX) R.member[t] = mem[sl][t];
      if (t == 0) {
        R.nmem = nm;
        R.nn = padded;
      }
    }
    __syncthreads();
  }
}

// One 64-thread CTA per listed table slot (two or more evaluations alone in
// their segments chose it): the evaluations whose columns equal the first
// one's (a hash collision leaves the others alone) become group records of
// up to GROUP_MAX members like k_group's (rows any member weighs, in
// reference order), and their own single-member records are switched off
// (nmem 0).
__global__ void __launch_bounds__(SEG) k_merge(DevGrid G, EvalBatch b) {
  __shared__ int mem[MERGE_CAP];
  __shared__ int nmem_s, cnt[2];
  const int t = threadIdx.x, lane = t & 31, wv = t >> 5;
  static_assert(MERGE_CAP == SEG, "one thread per listed evaluation");
  const int nlist = b.mslot[0];
  for (int j = blockIdx.x; j < nlist; j += gridDim.x) {
    const int slot = b.mslot[1 + j];
    const int nc = min(b.mcnt[slot], MERGE_CAP);
    int e = -1;
    if (t < nc) {
      e = b.mmem[(size_t)slot * MERGE_CAP + t];
      const int *c0 = b.prep[b.mmem[(size_t)slot * MERGE_CAP]].cols, *c = b.prep[e].cols;
      bool same = true;
      for (int n = 0; n < 64 && same; n++) same = c[n] == c0[n];
      if (!same) e = -1;
    }
    // compact the matching evaluations, keeping their order
    const unsigned bm = __ballot_sync(0xffffffffu, e >= 0);
    if (lane == 0) cnt[wv] = __popc(bm);
    __syncthreads();
    if (e >= 0) mem[__popc(bm & ((1u << lane) - 1u)) + (wv ? cnt[0] : 0)] = e;
    if (t == 0) nmem_s = cnt[0] + cnt[1];
    __syncthreads();
    const int nt = nmem_s;
    if (nt >= 2) {
      for (int g0 = 0; g0 < nt; g0 += GROUP_MAX) {
        const int nm = min(GROUP_MAX, nt - g0);
        __shared__ int rec;
        if (t == 0) rec = atomicAdd(b.mrcount, 1);
        __syncthreads();
        GroupRec &R = b.mrec[rec];
        // row t of the group: kept when any member weighs it
        const int c = b.prep[mem[g0]].cols[t];
        const float f = c >= 0 ? G.factor[c] : 0.0f;
        float w[GROUP_MAX], wf[GROUP_MAX];
        bool keep = false;
#pragma unroll
        for (int m = 0; m < GROUP_MAX; m++) {
          w[m] = (m < nm && c >= 0) ? b.prep[mem[g0 + m]].w[t] : 0.0f;
          wf[m] = w[m] * f;
          keep |= wf[m] != 0.0f;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        __syncthreads();  // cnt is reused
        if (lane == 0) cnt[wv] = __popc(bal);
        __syncthreads();
        const int pos = __popc(bal & ((1u << lane) - 1u)) + (wv ? cnt[0] : 0);
        if (keep) {
          R.wf[pos][0] = make_float4(wf[0], wf[1], wf[2], wf[3]);
          R.wf[pos][1] = make_float4(wf[4], wf[5], wf[6], wf[7]);
          R.w[pos][0] = make_float4(w[0], w[1], w[2], w[3]);
          R.w[pos][1] = make_float4(w[4], w[5], w[6], w[7]);
          R.col[pos] = c;
          R.f[pos] = f;
        }
        const int kept = cnt[0] + cnt[1];
        const int padded = (kept + 7) & ~7;
        if (t >= kept && t < padded) {  // zero-weight padding rows (add exactly 0)
          const float4 z4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          R.wf[t][0] = R.wf[t][1] = R.w[t][0] = R.w[t][1] = z4;
          R.col[t] = 0;
          R.f[t] = 0.0f;
        }
        if (t < GROUP_MAX) R.member[t] = t < nm ? mem[g0 + t] : -1;
        if (t == 0) {
          R.nmem = nm;
          R.nn = padded;
        }
        if (t < nm) b.grec[b.erec[mem[g0 + t]]].nmem = 0;  // interpolated here instead
        __syncthreads();
      }
    }
    __syncthreads();
  }
}

void launch_group(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0) return;
  if (b.tcrec) cudaMemsetAsync(b.tclist_count, 0, sizeof(int), s);
  if (b.mkey) {
    cudaMemsetAsync(b.mkey, 0, (size_t)b.mtab * sizeof(unsigned long long), s);
    cudaMemsetAsync(b.mcnt, 0, (size_t)b.mtab * sizeof(int), s);
    cudaMemsetAsync(b.mslot, 0, sizeof(int), s);
    cudaMemsetAsync(b.mrcount, 0, sizeof(int), s);
  }
  k_group<<<num_segments(b), SEG * GROUP_SLICES, 0, s>>>(G, b);
  count_launch();
  if (b.mkey) {
    k_merge<<<num_sms() * 8, SEG, 0, s>>>(G, b);
    count_launch();
  }
}

constexpr int IT_T = 256, IT_PX = 4, IT_TILE = IT_T * IT_PX;

// member m's weight (x factor when wf) of compacted row n
__device__ __forceinline__ float grp_w(const float4 (&v)[2], int m) {
  const float4 q = v[m >> 2];
  const int k = m & 3;
  return k == 0 ? q.x : k == 1 ? q.y : k == 2 ? q.z : q.w;
}

// the NM members of a group on this thread's 4 pixels (one 64-bit load per row)
template <int NM>
__device__ __forceinline__ void interp_members(const DevGrid &G, const EvalBatch &b, const GroupRec &R, int px) {
  // member m's window holds px (re-evaluated at the stores, so that the
  // members' indices need no registers across the row loop)
  auto inside = [&](int m) {
    const EvalPrep &P = b.prep[R.member[m]];
    return px >= P.i_lo && px < P.i_hi;
  };
  bool any = false;
#pragma unroll
  for (int m = 0; m < NM; m++) any |= inside(m);
  if (!any) return;
  const int nn = R.nn;
  if (px + IT_PX <= G.tail_start) {
    float2 acc[NM][2];
#pragma unroll
    for (int m = 0; m < NM; m++) acc[m][0] = acc[m][1] = make_float2(0.0f, 0.0f);
    const float2 bias = make_float2(-8388608.0f, -8388608.0f);
    constexpr int UNR = NM > 4 ? 4 : NM > 2 ? 8 : 16;  // row loads in flight per thread (with their weights in registers)
#pragma unroll UNR
    for (int n = 0; n < nn; n++) {
      const uint2 q = __ldg(reinterpret_cast<const uint2 *>(G.spectra + (size_t)R.col[n] * G.stride + px));
      float ws[8];
      const float4 w0 = R.wf[n][0];
      ws[0] = w0.x; ws[1] = w0.y; ws[2] = w0.z; ws[3] = w0.w;
      if (NM > 4) {
        const float4 w1 = R.wf[n][1];
        ws[4] = w1.x; ws[5] = w1.y; ws[6] = w1.z; ws[7] = w1.w;
      }
      const uint32_t u[2] = {q.x, q.y};
#pragma unroll
      for (int k = 0; k < 2; k++) {
        float2 v = make_float2(__int_as_float(__byte_perm(u[k], 0x4B000000u, 0x7410)),
                               __int_as_float(__byte_perm(u[k], 0x4B000000u, 0x7432)));
        v = __fadd2_rn(v, bias);  // exact u16 -> f32
#pragma unroll
        for (int m = 0; m < NM; m++) acc[m][k] = __ffma2_rn(make_float2(ws[m], ws[m]), v, acc[m][k]);
      }
    }
#pragma unroll
    for (int m = 0; m < NM; m++) {
      if (!inside(m)) continue;
      *reinterpret_cast<float4 *>(b.bufA + (size_t)R.member[m] * b.stride + px) =
          make_float4(acc[m][0].x, acc[m][0].y, acc[m][1].x, acc[m][1].y);
    }
    return;
  }
  // last tile: the final npx % 128 pixels carry an extra 1/65535 (interpolate.rs:978)
#pragma unroll
  for (int m = 0; m < NM; m++) {
    if (!inside(m)) continue;
    float acc[IT_PX];
#pragma unroll
    for (int k = 0; k < IT_PX; k++) acc[k] = 0.0f;
    for (int n = 0; n < nn; n++) {
      const uint2 q = __ldg(reinterpret_cast<const uint2 *>(G.spectra + (size_t)R.col[n] * G.stride + px));
      const float wn = grp_w(R.w[n], m), fn = R.f[n];
      const uint32_t u[2] = {q.x, q.y};
#pragma unroll
      for (int k = 0; k < IT_PX; k++) {
        const float x = (float)((u[k >> 1] >> (16 * (k & 1))) & 0xFFFFu);
        const float v = px + k >= G.tail_start ? __fmul_rn(__fdiv_rn(x, 65535.0f), fn) : __fmul_rn(x, fn);
        acc[k] = fmaf(wn, v, acc[k]);
      }
    }
    *reinterpret_cast<float4 *>(b.bufA + (size_t)R.member[m] * b.stride + px) =
        make_float4(acc[0], acc[1], acc[2], acc[3]);
  }
}

// one group record on this thread's pixels (nmem 0: a record switched off)
__device__ __forceinline__ void interp_group(const DevGrid &G, const EvalBatch &b, const GroupRec &R, int px) {
  switch (R.nmem) {
    case 0: break;
    case 1: interp_members<1>(G, b, R, px); break;
    case 2: interp_members<2>(G, b, R, px); break;
    case 3: interp_members<3>(G, b, R, px); break;
    case 4: interp_members<4>(G, b, R, px); break;
    case 5: interp_members<5>(G, b, R, px); break;
    case 6: interp_members<6>(G, b, R, px); break;
    case 7: interp_members<7>(G, b, R, px); break;
    default: interp_members<8>(G, b, R, px); break;
  }
}

// Grid: x = segment, y = tile of IT_TILE pixels, so CTAs that run together read
// the same tile slab of the resident grid (57 MB for 13,860 x 80,000), which
// stays in L2; z = slice of the segment's groups (groups z, z + Z, ...), more
// than one only for batches too small to fill the GPU otherwise.  Groups have
// disjoint members, so the slicing does not change any result.
__global__ void __launch_bounds__(IT_T, 3) k_interp(DevGrid G, EvalBatch b) {
  __shared__ GroupRec R;
  const int s = blockIdx.x;
  const int px = blockIdx.y * IT_TILE + threadIdx.x * IT_PX;
  const int ng = b.gcount[s];
  int start, len;
  seg_range(b, s, start, len);
  for (int g = blockIdx.z; g < ng; g += gridDim.z) {
    const float4 *src = reinterpret_cast<const float4 *>(b.grec + (size_t)start + g);
    float4 *dst = reinterpret_cast<float4 *>(&R);
    for (int i = threadIdx.x; i < (int)(sizeof(GroupRec) / 16); i += IT_T) dst[i] = src[i];
    __syncthreads();
    interp_group(G, b, R, px);
    __syncthreads();
  }
}

// Groups merged across segments (k_merge), in work items (record, tile)
// taken tile by tile, so that CTAs that run together read the same tile
// slab of the grid; their number is known on the device only.
__global__ void __launch_bounds__(IT_T, 3) k_interp_merged(DevGrid G, EvalBatch b) {
  __shared__ GroupRec R;
  const int nrec = *b.mrcount;
  const long long work = (long long)nrec * ((G.npx + IT_TILE - 1) / IT_TILE);
  for (long long w = blockIdx.x; w < work; w += gridDim.x) {
    const int tile = (int)(w / nrec), rec = (int)(w - (long long)tile * nrec);
    const float4 *src = reinterpret_cast<const float4 *>(b.mrec + rec);
    float4 *dst = reinterpret_cast<float4 *>(&R);
    for (int i = threadIdx.x; i < (int)(sizeof(GroupRec) / 16); i += IT_T) dst[i] = src[i];
    __syncthreads();
    interp_group(G, b, R, tile * IT_TILE + threadIdx.x * IT_PX);
    __syncthreads();
  }
}

void launch_interp(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0) return;
  const int segs = num_segments(b), tiles = (G.npx + IT_TILE - 1) / IT_TILE;
  const int want = num_sms() * 6;  // two waves of the 3 CTAs an SM holds
  const int z = segs * tiles >= want ? 1 : std::min(SEG, (want + segs * tiles - 1) / (segs * tiles));
  dim3 grid(segs, tiles, z);
  k_interp<<<grid, IT_T, 0, s>>>(G, b);
  count_launch();
  if (b.mkey) {
    k_interp_merged<<<num_sms() * 6, IT_T, 0, s>>>(G, b);
    count_launch();
  }
}

// ------------------------------------------------------------ resampling
// shift_and_resample (convolve_rv.rs:569-603): index in double, weight from
// the f32-rounded index minus the f32 floor, linear interpolation in f32.
struct ResPos {
  int j;    // left synth pixel
  float w;  // weight of pixel j + 1
};
__device__ __forceinline__ float resample_value(float w, float sj, float sj1) {
  return __fadd_rn(__fmul_rn(1.0f - w, sj), __fmul_rn(w, sj1));
}
struct Resampler {
  const float *s;
  int N, kind;
  double shift_log, shift_factor, lin_offset;
  const double *fidx, *wl_obs, *wl_vals;
  const float *given;  // model given directly at the observed pixels
  // j never decreases with i when the float indices do not
  __device__ __forceinline__ ResPos pos(int i) const {
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
    return from_index(idx);
  }
  __device__ __forceinline__ ResPos from_index(double idx) const {
    const double fl = floor(idx);
    int j = fl > 0 ? (int)fl : 0;
    if (j > N - 2) j = N - 2;  // the preparation kernel rejected j + 1 >= N already
    return ResPos{j, (float)idx - (float)j};
  }
  // position from an already loaded float index (uniform grids)
  __device__ __forceinline__ ResPos pos_from_fidx(double fx) const {
    return from_index(kind == WL_LOG ? fx + shift_log : __dadd_rn(__dmul_rn(shift_factor, fx), lin_offset));
  }
  __device__ __forceinline__ float operator()(int i) const {
    if (given) return given[i];
    const ResPos q = pos(i);
    return resample_value(q.w, s[q.j], s[q.j + 1]);
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
// Asynchronous 16-byte global -> shared copies (cp.async): the next tile's
// input streams in while the current one is worked.  A copy with ok ==
// false reads nothing and fills zeros.
__device__ __forceinline__ void cp_async16(float *smem, const float *gmem, bool ok) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int n = ok ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Bulk prefetch of floats [lo, hi) of a row into L2 (one instruction, issued
// by one thread; a hint, nothing waits for it).  The row must start on a
// 16-byte boundary and hold hi rounded up to 4 floats.
__device__ __forceinline__ void prefetch_row_l2(const float *row, int lo, int hi) {
  lo &= ~3;
  hi = (hi + 3) & ~3;
  if (hi <= lo) return;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(row + lo), "r"((unsigned)(hi - lo) * 4u)
               : "memory");
}

struct BroadenItem {
  int e, pair, m, hg, V, s0, s1, j0, j1;
  bool has1;
};

// the work item (evaluation e, block pair), or false when it has nothing to do
__device__ __forceinline__ bool broaden_item(const EvalBatch &b, int e, int pair, BroadenItem &w) {
  w.e = e;
  w.pair = pair;
  const EvalPrep &P = b.prep[e];
  if (P.status || !P.fused || 2 * pair >= P.nblk) return false;
  w.m = P.m;
  w.hg = P.hg;
  w.V = FFTN - (w.m - 1) - 2 * w.hg;
  w.s0 = P.o_lo + 2 * pair * (w.V - 1);
  w.s1 = w.s0 + (w.V - 1);
  w.has1 = 2 * pair + 1 < P.nblk;
  // input t of a block is synth pixel (s - hg - hw + t) for the rotation,
  // (s - hg + t) for the identity
  const int shift = w.m > 1 ? w.hg + (w.m - 1) / 2 : w.hg;
  w.j0 = w.s0 - shift;
  w.j1 = w.s1 - shift;
  return true;
}

// The items of a CTA (item = e * max_pairs + pair) come in runs of ic
// consecutive items (mostly neighbouring block pairs of one evaluation, so
// their metadata and the overlap of their inputs are still in cache): run r
// of the CTA is items [ic R, ic R + ic) with R = blockIdx.x + r gridDim.x.
struct ItemCursor {
  int e, pair, k, ic, mp, E;
  long long run;
  __device__ __forceinline__ void set_run() {
    const long long item = run * ic;
    e = (int)(item / mp);
    pair = (int)(item % mp);
    k = 0;
  }
  __device__ __forceinline__ void init(const EvalBatch &b, int run_len) {
    mp = b.max_pairs;
    E = b.E;
    ic = run_len;
    run = blockIdx.x;
    set_run();
  }
  __device__ __forceinline__ void advance() {
    if (++k < ic) {
      if (++pair >= mp) {
        pair = 0;
        e++;
      }
    } else {
      run += gridDim.x;
      set_run();
    }
  }
  __device__ __forceinline__ bool done() const { return e >= E; }
  // move to the first item with work at or after the current one
  __device__ __forceinline__ void settle(const EvalBatch &b) {
    BroadenItem w;
    while (!done() && !broaden_item(b, e, pair, w)) advance();
  }
};

// The 2 x 16 inputs of this thread for item w: block input j = 128 n1 + t
// is synth pixel j0 + j of the interpolated row (zero outside [i_lo, i_hi)).
// Interior item pairs (both blocks inside the window, the common case) load
// without per-element bounds tests.
__device__ __forceinline__ void broaden_inputs(const EvalBatch &b, const BroadenItem &w, const EvalPrep &P,
                                               float (&x0)[16], float (&x1)[16]) {
  const float *row = b.bufA + (size_t)w.e * b.stride;
  const int ilo = P.i_lo, ihi = P.i_hi;
  if (w.has1 && w.j0 >= ilo && w.j1 + FFTN <= ihi) {
    const float *r0 = row + w.j0 + (int)threadIdx.x, *r1 = row + w.j1 + (int)threadIdx.x;
#pragma unroll
    for (int n1 = 0; n1 < 16; n1++) {
      x0[n1] = __ldg(r0 + 128 * n1);
      x1[n1] = __ldg(r1 + 128 * n1);
    }
    return;
  }
#pragma unroll
  for (int n1 = 0; n1 < 16; n1++) {
    const int g0 = w.j0 + 128 * n1 + (int)threadIdx.x, g1 = w.j1 + 128 * n1 + (int)threadIdx.x;
    x0[n1] = (g0 >= ilo && g0 < ihi) ? __ldg(row + g0) : 0.0f;
    x1[n1] = (w.has1 && g1 >= ilo && g1 < ihi) ? __ldg(row + g1) : 0.0f;
  }
}

constexpr int BT = F2_T;      // threads of k_broaden
constexpr int BR_RUN = 8;     // longest run of consecutive items a CTA takes
// dynamic shared memory (bytes): exchange buffers 1 and 2 (buffer 2 also
// holds the rotation outputs, buffer 1 the outputs of the instrument taps),
// twiddles of pass 2, the fixed instrument taps
constexpr int BR_S1 = 0, BR_S2 = BR_S1 + F2_S1 * 8, BR_T2 = BR_S2 + F2_S2 * 8, BR_GK = BR_T2 + 16 * 8 * 8,
              BR_SMEM = BR_GK + 512 * 4;

// Resampling of an item's observed pixels [q0, q2) (the left synth pixel of
// [q0, q1) in block 0, of [q1, q2) in block 1) from the final outputs in
// shared memory, with the wavelength kind fixed at compile time.  The float
// indices come from the star's table (a star's particles share it; the
// item prefetched its range into L1 before the transforms); each thread
// issues the loads of EU pixels before their arithmetic.
template <int KIND>
__device__ __forceinline__ void resample_item(const Resampler &R, float *y, const float *ob0,
                                              const float *ob1, int q0, int q1, int q2, int s0, int s1, int V) {
  constexpr int EU = 8;
  for (int i0 = q0 + (int)threadIdx.x; i0 < q2; i0 += EU * BT) {
    double fx[EU];
#pragma unroll
    for (int r = 0; r < EU; r++) {
      const int i = min(i0 + r * BT, q2 - 1);
      fx[r] = KIND == WL_NONUNI ? 0.0 : __ldg(&R.fidx[i]);
    }
#pragma unroll
    for (int r = 0; r < EU; r++) {
      const int i = i0 + r * BT;
      if (i < q2) {
        ResPos q;
        if (KIND == WL_LOG) q = R.from_index(fx[r] + R.shift_log);
        else if (KIND == WL_LIN) q = R.from_index(__dadd_rn(__dmul_rn(R.shift_factor, fx[r]), R.lin_offset));
        else q = R.pos(i);
        const bool k1 = i >= q1;
        const float *o = k1 ? ob1 : ob0;
        const int u = min(max(q.j - (k1 ? s1 : s0), 0), V - 2);  // in range by construction of bnd
        y[i] = resample_value(q.w, o[u], o[u + 1]);
      }
    }
  }
}

// the pass-1 twiddle W_2048^(t k1) of this thread from W^t, W^2t, W^4t and
// W^8t (table values, computed in double on the host) by at most three
// products
__device__ __forceinline__ cf tw_pass1(int k1, const cf &w1, const cf &w2, const cf &w4, const cf &w8) {
  cf r = (k1 & 1) ? w1 : cf{1.0f, 0.0f};
  if (k1 & 2) r = (k1 & 1) ? cmul(r, w2) : w2;
  if (k1 & 4) r = (k1 & 3) ? cmul(r, w4) : w4;
  if (k1 & 8) r = (k1 & 7) ? cmul(r, w8) : w8;
  return r;
}

// One work item = two overlap-save blocks of one evaluation.  Block k yields
// V = 2048 - (m - 1) - 2 hg final outputs starting at s_k = o_lo + k (V - 1):
// the rotation outputs [s - hg, s + V + hg) come from one overlap-save block
// of 2048 inputs (the reference uses overlap-add, convolve_rv.rs:121-157;
// both are the same linear convolution), and the instrument profile is then
// applied from shared memory.  Block k owns synth pixels [s_k, s_k + V - 1);
// its last output is the partner j + 1 of its last owned pixel j.  The two
// real blocks ride in the real and imaginary parts of one complex FFT (the
// kernel is real, so the two products separate after the inverse).  Rotation
// outputs outside [0, N) are zero, like the reference's cropped segment.
// With the identity rotation the FFT is skipped.  Away from the grid ends
// the instrument Gaussian acts on rotation outputs that are all inside
// [0, N), where rotation-then-Gaussian is one convolution with the combined
// kernel: the spectra are multiplied (H x G) and the taps are skipped.
//
// Epilogue: either the owned synth pixels go to row B, or (chi2 batches,
// EvalPrep::epi) the block resamples the observed pixels whose left synth
// pixel it owns (EvalBatch::bnd lists them per block) from shared memory and
// writes the model at the observed pixels to row B; the synth row never
// reaches memory.  An item's float indices are prefetched into L1 before its
// transforms; a CTA takes runs of consecutive items (ItemCursor).
__global__ void __launch_bounds__(BT, 5) k_broaden(DevGrid G, EvalBatch b, const float2 *__restrict__ tw, int run_len) {
  extern __shared__ __align__(16) unsigned char br_smem[];
  float2 *S1 = reinterpret_cast<float2 *>(br_smem + BR_S1);
  float2 *S2 = reinterpret_cast<float2 *>(br_smem + BR_S2);
  float2 *T2 = reinterpret_cast<float2 *>(br_smem + BR_T2);
  float *gks = reinterpret_cast<float *>(br_smem + BR_GK);
  const int t = threadIdx.x, N = G.npx;
  // twiddles: T2[k2][n3] = W_128^(n3 k2) in shared memory; W_2048^(t k1)
  // from the four powers of two of W^t in registers
  for (int i = t; i < 16 * 8; i += BT) T2[i] = __ldg(&tw[(16 * (i & 7) * (i >> 3)) & (FFTN - 1)]);
  cf tw1, tw2, tw4, tw8;
  {
    const float2 a = __ldg(&tw[t]), c = __ldg(&tw[2 * t]), d = __ldg(&tw[4 * t]), f = __ldg(&tw[8 * t]);
    tw1 = cf{a.x, a.y};
    tw2 = cf{c.x, c.y};
    tw4 = cf{d.x, d.y};
    tw8 = cf{f.x, f.y};
  }
  ItemCursor cur;
  cur.init(b, run_len);
  cur.settle(b);
  const int k1p = t >> 3, n3p = t & 7;  // pass-2 role of this thread
  int gk_star = -1;                       // star whose instrument taps are in gks
  while (!cur.done()) {
    ItemCursor nxt = cur;
    nxt.advance();
    nxt.settle(b);
    BroadenItem w;
    broaden_item(b, cur.e, cur.pair, w);
    const int e = w.e, pair = w.pair, m = w.m, hg = w.hg, V = w.V, s0 = w.s0, s1 = w.s1;
    const bool has1 = w.has1;
    const EvalPrep &P = b.prep[e];
    const int nblk = P.nblk, ohi = P.o_hi;
    const DevStar &st = b.stars[P.star];
    const bool fixedk = hg > 0 && st.disp_kind == DISP_FIXED;
    const int gw = 2 * hg + 1;
    int q0 = 0, q1 = 0, q2 = 0;
    if (P.epi) {
      const int *bd = b.bnd + (size_t)e * b.bnd_stride + 2 * pair;
      q0 = bd[0];
      q1 = bd[1];
      q2 = has1 ? bd[2] : q1;
    }
    __syncthreads();  // the last item's epilogue is done with the shared buffers
    // this item's inputs and instrument taps
    float in0[16], in1[16];
    broaden_inputs(b, w, P, in0, in1);
    if (P.epi && G.wl_kind != WL_NONUNI) {  // the float indices the resampling reads: into L1 meanwhile
      const double *fq = st.fidx + q0;
      for (int l = t; l * 16 < q2 - q0; l += BT) asm volatile("prefetch.global.L1 [%0];" ::"l"(fq + 16 * l));
    }
    const int e_last = min((has1 ? s1 : s0) + V, ohi);
    const bool fold = fixedk && m > 1 && st.gspec != nullptr && b.HG != nullptr && s0 - hg >= 0 && e_last + hg <= N;
    if (fixedk && !fold && P.star != gk_star) {  // the taps are applied from shared memory (edge blocks)
      for (int k = t; k < gw; k += BT) gks[k] = __ldg(&st.gk[k]);
      gk_star = P.star;
    }
    const float sc = 1.0f / 2048.0f;
    float *ob0, *ob1;  // final outputs u in [0, V) of the two blocks
    if (m > 1) {
      cf v[16];
#pragma unroll
      for (int n1 = 0; n1 < 16; n1++) v[n1] = cf{in0[n1], in1[n1]};
      // pass 1: DFT-16 over n1, twiddle, exchange 1
      dft16<false>(v);
#pragma unroll
      for (int k1 = 0; k1 < 16; k1++) {
        const cf z = k1 ? cmul(v[k1], tw_pass1(k1, tw1, tw2, tw4, tw8)) : v[k1];
        S1[k1 * F2_XP + t] = make_float2(z.x, z.y);
      }
      __syncthreads();
      // pass 2: DFT-16 over n2, twiddle, exchange 2
#pragma unroll
      for (int n2 = 0; n2 < 16; n2++) {
        const float2 z = S1[k1p * F2_XP + 8 * n2 + n3p];
        v[n2] = cf{z.x, z.y};
      }
      dft16<false>(v);
#pragma unroll
      for (int k2 = 0; k2 < 16; k2++) {
        const cf z = k2 ? cmul_tw<false>(v[k2], T2[k2 * 8 + n3p]) : v[k2];
        S2[f2_a2(k1p + 16 * k2, n3p)] = make_float2(z.x, z.y);
      }
      __syncthreads();
      // pass 3 (DFT-8 over n3), the spectrum product, and the inverse DFT-8
      // over k3, for c = t and t + 128; each thread rewrites the slots it read
      const float2 *H = (fold ? b.HG : b.H) + (size_t)e * 1025;
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int c = t + 128 * h;
        cf u[8];
        float2 hk[8];
        // bins k = c + 256 k3 (c < 256): k < 1024 below k3 = 4, k > 1024
        // above it (conjugate of bin 2048 - k); k3 = 4 is bin 1024 for c = 0
#pragma unroll
        for (int k3 = 0; k3 < 8; k3++) {
          const int k = c + 256 * k3;
          if (k3 < 4) {
            hk[k3] = __ldg(&H[k]);
          } else if (k3 > 4) {
            hk[k3] = __ldg(&H[FFTN - k]);
            hk[k3].y = -hk[k3].y;
          } else {
            hk[k3] = __ldg(&H[c == 0 ? 1024 : FFTN - k]);
            if (c != 0) hk[k3].y = -hk[k3].y;
          }
        }
#pragma unroll
        for (int n3 = 0; n3 < 8; n3++) {
          const float2 z = S2[f2_a2(c, n3)];
          u[n3] = cf{z.x, z.y};
        }
        dft8<false>(u);
#pragma unroll
        for (int k3 = 0; k3 < 8; k3++) u[k3] = cmul(u[k3], cf{hk[k3].x, hk[k3].y});
        dft8<true>(u);
#pragma unroll
        for (int n3 = 0; n3 < 8; n3++) S2[f2_a2(c, n3)] = make_float2(u[n3].x, u[n3].y);
      }
      __syncthreads();
      // inverse pass 2: conjugate twiddle, DFT-16 over k2, exchange 1
#pragma unroll
      for (int k2 = 0; k2 < 16; k2++) {
        const float2 z = S2[f2_a2(k1p + 16 * k2, n3p)];
        v[k2] = k2 ? cmul_tw<true>(cf{z.x, z.y}, T2[k2 * 8 + n3p]) : cf{z.x, z.y};
      }
      dft16<true>(v);
#pragma unroll
      for (int n2 = 0; n2 < 16; n2++) S1[k1p * F2_XP + 8 * n2 + n3p] = make_float2(v[n2].x, v[n2].y);
      __syncthreads();
      // inverse pass 1: conjugate twiddle, DFT-16 over k1 -> 2048 x output 128 n1 + t
#pragma unroll
      for (int k1 = 0; k1 < 16; k1++) {
        const float2 z = S1[k1 * F2_XP + t];
        v[k1] = k1 ? cmul_tw<true>(cf{z.x, z.y}, [&] {
          const cf q = tw_pass1(k1, tw1, tw2, tw4, tw8);
          return make_float2(q.x, q.y);
        }()) : cf{z.x, z.y};
      }
      dft16<true>(v);
      // FFT index i = 128 n1 + t holds rotation output (s - hg) + (i - (m - 1))
      const int base = m - 1;
      if (fold) {  // final output u = i - base - 2 hg
        ob0 = reinterpret_cast<float *>(S2);
        ob1 = ob0 + 2048;
#pragma unroll
        for (int n1 = 0; n1 < 16; n1++) {
          const int u = 128 * n1 + t - base - 2 * hg;  // at most 2047 - base - 2 hg = V - 1
          if (u >= 0) {
            ob0[u] = v[n1].x * sc;
            ob1[u] = v[n1].y * sc;
          }
        }
      } else {  // rotation outputs r = i - base, zero outside the grid
        const int r0 = s0 - hg, r1 = s1 - hg;
#pragma unroll
        for (int n1 = 0; n1 < 16; n1++) {
          const int r = 128 * n1 + t - base;
          if (r >= 0) {
            const int i0 = r0 + r, i1 = r1 + r;
            S2[r] = make_float2((i0 >= 0 && i0 < N) ? v[n1].x * sc : 0.0f, (i1 >= 0 && i1 < N) ? v[n1].y * sc : 0.0f);
          }
        }
      }
    } else {  // identity rotation: the inputs are the rotation outputs r = j
#pragma unroll
      for (int n1 = 0; n1 < 16; n1++) S2[128 * n1 + t] = make_float2(in0[n1], in1[n1]);
    }
    __syncthreads();
    if (!fold) {  // instrument taps from the rotation outputs in S2 into buffer 1
      ob0 = reinterpret_cast<float *>(S1);
      ob1 = ob0 + 2048;
      for (int u = t; u < V; u += BT) {
        const int i0 = s0 + u, i1 = s1 + u;
        float v0, v1;
        if (hg == 0) {
          const float2 x = S2[u];
          v0 = x.x;
          v1 = x.y;
        } else if (fixedk) {  // g[i] = sum_k gk[k] r[i + hg - k]; r[i] sits at i - s + hg
          float a0 = 0.0f, a1 = 0.0f;
          for (int k = 0; k < gw; k++) {
            const float g = gks[k];
            const float2 x = S2[u + 2 * hg - k];
            a0 = fmaf(g, x.x, a0);
            a1 = fmaf(g, x.y, a1);
          }
          v0 = a0;
          v1 = a1;
        } else {
          v0 = instrument(st, N, i0, hg, [&](int i) { return S2[i - (s0 - hg)].x; });
          v1 = has1 ? instrument(st, N, i1, hg, [&](int i) { return S2[i - (s1 - hg)].y; }) : 0.0f;
        }
        ob0[u] = v0;
        ob1[u] = v1;
      }
      __syncthreads();
    }
    float *y = b.bufB + (size_t)e * b.stride;
    if (P.epi) {
      // observed pixels [q0, q2) have their left synth pixel in this item's
      // blocks; the boundary between them is q1
      const Resampler R = make_resampler(G, st, P, nullptr, nullptr);
      if (R.kind == WL_LOG) resample_item<WL_LOG>(R, y, ob0, ob1, q0, q1, q2, s0, s1, V);
      else if (R.kind == WL_LIN) resample_item<WL_LIN>(R, y, ob0, ob1, q0, q1, q2, s0, s1, V);
      else resample_item<WL_NONUNI>(R, y, ob0, ob1, q0, q1, q2, s0, s1, V);
    } else {
      // owned pixels; the last block also writes its final output
      const int n0 = 2 * pair + 1 == nblk ? V : V - 1, n1 = 2 * pair + 2 == nblk ? V : V - 1;
      for (int u = t; u < V; u += BT) {
        const int i0 = s0 + u, i1 = s1 + u;
        if (u < n0 && i0 < ohi) y[i0] = ob0[u];
        if (has1 && u < n1 && i1 < ohi) y[i1] = ob1[u];
      }
    }
    cur = nxt;
  }
}

void launch_broaden(const DevGrid &G, const EvalBatch &b, const float2 *tw, cudaStream_t s) {
  if (b.E <= 0 || b.max_pairs <= 0) return;
  const size_t smem = BR_SMEM;
  static int per_sm[64] = {};  // resident CTAs per SM, per device
  int dev = 0;
  cudaGetDevice(&dev);
  int fit = 5;
  if (dev >= 0 && dev < 64) {
    if (!per_sm[dev]) {
      cudaFuncSetAttribute(k_broaden, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      int n = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_broaden, BT, smem) != cudaSuccess || n < 1) n = 1;
      per_sm[dev] = n;
    }
    fit = per_sm[dev];
  }
  const long long total = (long long)b.E * b.max_pairs;
  long long grid = (long long)num_sms() * fit;  // persistent: the CTAs that fit at once
  if (grid > total) grid = total;
  // runs of up to BR_RUN consecutive items, as long as every CTA still gets
  // 16 runs or more (small batches keep single items spread over all CTAs)
  int run_len = (int)std::min<long long>(BR_RUN, std::max<long long>(1, total / (grid * 16)));
  if (const char *rl = getenv("PASTA_BR_RUN")) run_len = std::max(1, atoi(rl));
  k_broaden<<<(unsigned)grid, BT, smem, s>>>(G, b, tw, run_len);
  count_launch();
}

// ----------------------------------------------- direct broadening (narrow)
// Evaluations whose combined kernel (m rotation taps + 2 hg instrument taps)
// is narrow are convolved directly: per tile of DIRECT_TILE - 2 hg final
// outputs [t0, t0 + n) the DIRECT_TILE rotation outputs [t0 - hg, t0 + n + hg) (zero outside the
// grid, like the reference's cropped segment) and then the instrument
// profile, both from shared memory, into B.  The result is the same linear
// convolution the FFT path computes (convolve_rv.rs:121-157, 207-210,
// 414-430, 484-529), to f32 roundoff.
constexpr int DT_T = 256;
constexpr int DT_X = DIRECT_TILE + DIRECT_MAX_TAPS + 32;  // staged input / rotation output (floats)
constexpr int DT_HALF = DT_X / 2;                          // 1296 = 16 mod 32 (see dchunk)
constexpr int DT_K = DIRECT_MAX_TAPS + 32;                // zero-padded taps
static_assert(DT_X % 8 == 0 && DT_HALF % 32 == 16, "direct tile layout");

// Rows of the direct path sit in shared memory chunk-interleaved: float4
// chunk c (elements 4c..4c+3) at (c & 1) * DT_HALF + (c >> 1) * 4.  The
// chunks 2t + q that the threads t of a warp read together are then
// consecutive 16-byte words (no bank conflicts), and so are the chunks 2t,
// 2t + 1 each thread writes.
__device__ __forceinline__ int dchunk(int c) { return ((c & 1) ? DT_HALF : 0) + ((c >> 1) << 2); }
__device__ __forceinline__ int dperm(int i) { return dchunk(i >> 2) + (i & 3); }

// out(v) = sum_{j=-h..h} k[h + j] x(D + v - j), v in [0, n), n <= 8 DT_T: the
// eight consecutive outputs v0 = 8t.. of thread t.  x (chunk-interleaved) is
// readable (finite) over [0, n + 2h + 16); D - h is 0..3; kp holds k[0..2h]
// at offset zp = 12 + the amount that makes 2h + (D - h) + zp a multiple of
// 4, zeros around it, so every window of 12 taps is three aligned float4
// reads and taps outside the kernel are exact zeros.  Each chunk of 4 inputs
// costs 2 shared-memory reads (the input, one new tap float4) for 32 FMAs.
__device__ __forceinline__ int direct_zp(int h, int pl) { return 12 + ((4 - ((2 * h + pl) & 3)) & 3); }

__device__ __forceinline__ void conv_step(const float4 a, const float4 lo, float4 &mid, float4 &hi, float (&acc)[8]) {
  const float T[12] = {lo.x, lo.y, lo.z, lo.w, mid.x, mid.y, mid.z, mid.w, hi.x, hi.y, hi.z, hi.w};
  const float av[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
  for (int c = 0; c < 8; c++)
#pragma unroll
    for (int r = 0; r < 4; r++) acc[c] = fmaf(T[4 + c - r], av[r], acc[c]);
  hi = mid;
  mid = lo;
}

template <class Store>
__device__ __forceinline__ void conv_blocked(const float *__restrict__ x, int D, int h, const float *__restrict__ kp,
                                             int n, const Store &st) {
  const int v0 = 8 * threadIdx.x;
  if (v0 >= n) return;
  const int pl = D - h;
  const int z0 = 2 * h + pl + direct_zp(h, pl);  // multiple of 4
  const int Q = (pl + 7 + 2 * h) / 4 + 1;
  const float4 *xe = reinterpret_cast<const float4 *>(x) + threadIdx.x;            // chunks 2t, 2t + 2, ...
  const float4 *xo = reinterpret_cast<const float4 *>(x + DT_HALF) + threadIdx.x;  // chunks 2t + 1, ...
  const float4 *k4 = reinterpret_cast<const float4 *>(kp) + z0 / 4;
  float acc[8];
#pragma unroll
  for (int c = 0; c < 8; c++) acc[c] = 0.0f;
  // chunk q: inputs x(v0 + 4q + r), taps kp[z0 - 4q - 4 + i], i = 4 + c - r in 1..10
  float4 hi = k4[1], mid = k4[0];
  int q = 0;
  for (; q + 1 < Q; q += 2) {
    conv_step(xe[q >> 1], k4[-q - 1], mid, hi, acc);
    conv_step(xo[q >> 1], k4[-q - 2], mid, hi, acc);
  }
  if (q < Q) conv_step(xe[q >> 1], k4[-q - 1], mid, hi, acc);
  st(v0, acc);
}

// taps k[0..2h] (or the single tap 1 when taps == null) into kp with the
// padding of conv_blocked for this D - h
__device__ __forceinline__ void direct_taps(float *kp, const float *taps, int h, int pl) {
  const int zp = direct_zp(h, pl);
  for (int t = threadIdx.x; t < DT_K; t += DT_T) {
    const int u = t - zp;
    kp[t] = (u >= 0 && u <= 2 * h) ? (taps ? taps[u] : 1.0f) : 0.0f;
  }
}

// final outputs per direct tile of an evaluation: a multiple of 4, so the
// input alignment (and with it the padding of the rotation taps) is the same
// for every tile of the evaluation; tiles start at o_lo rounded down to 4,
// so the outputs are 16-byte aligned in the row
__device__ __forceinline__ int direct_td(int hg) { return (DIRECT_TILE - 2 * hg) & ~3; }

struct DirectTile {
  int e, tile, m, hw, hg, t0, n, p0, nr, pl, x0;
};
__device__ __forceinline__ bool direct_tile(const EvalBatch &b, int e, int tile, DirectTile &d) {
  const EvalPrep &P = b.prep[e];
  if (P.status || !P.direct || tile >= P.ndt) return false;
  d.e = e;
  d.tile = tile;
  d.m = P.m;
  d.hw = (d.m - 1) / 2;
  d.hg = P.hg;
  const int td = direct_td(d.hg);
  d.t0 = (P.o_lo & ~3) + tile * td;
  d.n = min(td, P.o_hi - d.t0);
  d.p0 = d.t0 - d.hg;  // rotation outputs [p0, p0 + nr)
  d.nr = d.n + 2 * d.hg;
  d.pl = (((d.p0 - d.hw) % 4) + 4) % 4;
  d.x0 = d.p0 - d.hw - d.pl;  // inputs staged from x0, a multiple of 4
  return true;
}
__device__ __forceinline__ void direct_stage(const EvalBatch &b, const DirectTile &d, float *xs) {
  const EvalPrep &P = b.prep[d.e];
  const float *row = b.bufA + (size_t)d.e * b.stride;
  const int nx = (d.nr + 2 * d.hw + 16 + 3) & ~3;
  for (int c = threadIdx.x; c < nx / 4; c += DT_T) {
    const int g = d.x0 + 4 * c;
    const bool ok = g >= P.i_lo && g + 4 <= P.i_hi;
    cp_async16(xs + dchunk(c), ok ? row + g : row + P.i_lo, ok);
  }
}
// the next item with work at or after i in steps of gridDim.x, or false;
// item i is tile i % max_dtiles of the listed evaluation i / max_dtiles
__device__ __forceinline__ bool direct_next(const EvalBatch &b, long long &i, long long total, DirectTile &d) {
  for (; i < total; i += gridDim.x)
    if (direct_tile(b, b.direct_list[i / b.max_dtiles], (int)(i % b.max_dtiles), d)) return true;
  return false;
}

// CTAs take the tiles of the evaluations k_prep listed in grid strides, so
// those tiles (often all particles of a few stars) spread over the whole GPU;
// the next item's input is copied in (cp.async) while the current one is
// convolved.
__global__ void __launch_bounds__(DT_T) k_direct(DevGrid G, EvalBatch b) {
  __shared__ __align__(16) float xs[2][DT_X];
  __shared__ __align__(16) float rs[DT_X];
  __shared__ __align__(16) float kr[DT_K];
  __shared__ __align__(16) float kg[DT_K];
  const int N = G.npx;
  const long long total = (long long)*b.direct_count * b.max_dtiles;
  long long ic = blockIdx.x;
  DirectTile cur, nxt;
  bool have = direct_next(b, ic, total, cur);
  if (have) direct_stage(b, cur, xs[0]);
  cp_async_commit();
  int buf = 0, taps_e = -1;
  while (have) {
    long long in = ic + gridDim.x;
    const bool more = direct_next(b, in, total, nxt);
    if (more) direct_stage(b, nxt, xs[buf ^ 1]);
    cp_async_commit();
    const EvalPrep &P = b.prep[cur.e];
    const DevStar &st = b.stars[P.star];
    const bool fixedk = st.disp_kind == DISP_FIXED && cur.hg > 0;
    if (cur.e != taps_e) {
      direct_taps(kr, cur.m > 1 ? reinterpret_cast<const float *>(b.H + (size_t)cur.e * 1025) : nullptr,
                  cur.m > 1 ? cur.hw : 0, cur.pl);
      direct_taps(kg, fixedk ? st.gk : nullptr, fixedk ? cur.hg : 0, 0);
      taps_e = cur.e;
    }
    const int p0 = cur.p0, nr = cur.nr, n = cur.n, hg = cur.hg;
    for (int t = nr + threadIdx.x; t < nr + 16; t += DT_T) rs[dperm(t)] = 0.0f;
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // this item's input (the next may be in flight)
    __syncthreads();
    const float *x = xs[buf];
    if (cur.m > 1) {
      conv_blocked(x, cur.hw + cur.pl, cur.hw, kr, nr, [&](int v0, float (&acc)[8]) {
#pragma unroll
        for (int c = 0; c < 8; c++) {  // zero outside the grid and past the tile
          const int v = v0 + c, p = p0 + v;
          if (!(v < nr && p >= 0 && p < N)) acc[c] = 0.0f;
        }
        float4 *r4 = reinterpret_cast<float4 *>(rs);
        r4[dchunk(v0 >> 2) >> 2] = make_float4(acc[0], acc[1], acc[2], acc[3]);
        r4[dchunk((v0 >> 2) + 1) >> 2] = make_float4(acc[4], acc[5], acc[6], acc[7]);
      });
    } else {  // identity rotation: the staged input itself (zero outside the grid)
      for (int v = threadIdx.x; v < nr; v += DT_T) {
        const int p = p0 + v;
        rs[dperm(v)] = (p >= 0 && p < N) ? x[dperm(v + cur.pl)] : 0.0f;
      }
    }
    __syncthreads();
    float *y = b.bufB + (size_t)cur.e * b.stride + cur.t0;  // 16-byte aligned
    if (hg == 0 || fixedk) {
      conv_blocked(rs, fixedk ? hg : 0, fixedk ? hg : 0, kg, n, [&](int v0, float (&acc)[8]) {
        if (v0 + 8 <= n) {
          reinterpret_cast<float4 *>(y + v0)[0] = make_float4(acc[0], acc[1], acc[2], acc[3]);
          reinterpret_cast<float4 *>(y + v0)[1] = make_float4(acc[4], acc[5], acc[6], acc[7]);
        } else {
#pragma unroll
          for (int c = 0; c < 8; c++)
            if (v0 + c < n) y[v0 + c] = acc[c];
        }
      });
    } else {  // per-pixel instrument kernels (edge pixels pass through)
      for (int v = threadIdx.x; v < n; v += DT_T)
        y[v] = instrument(st, N, cur.t0 + v, hg, [&](int i) { return rs[dperm(i - p0)]; });
    }
    __syncthreads();  // rs and this buffer are rewritten for the item after next
    buf ^= 1;
    have = more;
    ic = in;
    cur = nxt;
  }
  cp_async_wait_all();
}

void launch_direct(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0 || b.direct_max <= 0 || b.max_dtiles <= 0 || !b.direct_list) return;
  static int per_sm[64] = {};  // resident CTAs per SM, per device
  int dev = 0;
  cudaGetDevice(&dev);
  int fit = 4;
  if (dev >= 0 && dev < 64) {
    if (!per_sm[dev]) {
      int n = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_direct, DT_T, 0) != cudaSuccess || n < 1) n = 1;
      per_sm[dev] = n;
    }
    fit = per_sm[dev];
  }
  const long long total = (long long)b.E * b.max_dtiles;
  long long grid = (long long)num_sms() * fit;
  if (grid > total) grid = total;
  k_direct<<<(unsigned)grid, DT_T, 0, s>>>(G, b);
  count_launch();
}

// First observed pixel of every fused broadening block: bnd[k] = the
// smallest i whose left synth pixel is >= s_k (binary search on the
// monotone resampling index); bnd[0] = 0, bnd[nblk] = n_obs.
__global__ void k_obs_bounds(DevGrid G, EvalBatch b) {
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  if (P.status || !P.epi) return;
  const int k = blockIdx.y * blockDim.x + threadIdx.x, nblk = P.nblk;
  if (k > nblk) return;
  const DevStar &st = b.stars[P.star];
  int *bd = b.bnd + (size_t)e * b.bnd_stride;
  if (k == 0 || k == nblk) {
    bd[k] = k == 0 ? 0 : st.n_obs;
    return;
  }
  const int target = P.o_lo + k * (FFTN - (P.m - 1) - 2 * P.hg - 1);
  const Resampler R = make_resampler(G, st, P, nullptr, nullptr);
  int lo = 0, hi = st.n_obs;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (R.pos(mid).j < target) lo = mid + 1;
    else hi = mid;
  }
  bd[k] = lo;
}

void launch_obs_bounds(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0 || b.max_pairs <= 0 || !b.obs_epi) return;
  dim3 grid(b.E, (2 * b.max_pairs + 1 + 63) / 64);
  k_obs_bounds<<<grid, 64, 0, s>>>(G, b);
  count_launch();
}

// ------------------------------------------- unfused rotation (wide kernels)
// Overlap-save with the rotation kernel alone: block b produces rotation
// outputs [g_lo + b V, g_lo + (b+1) V), V = 2048 - (m - 1), into B.
__global__ void __launch_bounds__(FFT_T, 3) k_rot(DevGrid G, EvalBatch b, const float2 *__restrict__ tw) {
  __shared__ float2 c[FFT_SM];
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
      c[pidx(t)] = make_float2((j0 >= ilo && j0 < ihi) ? x[j0] : 0.0f, (has1 && j1 >= ilo && j1 < ihi) ? x[j1] : 0.0f);
    }
    __syncthreads();
    fft2048<false>(c, tw);
    const float2 *H = b.H + (size_t)e * 1025;
    for (int k = threadIdx.x; k < FFTN; k += FFT_T) {
      float2 h = k <= 1024 ? H[k] : H[FFTN - k];
      if (k > 1024) h.y = -h.y;
      const int a = pidx(k);
      const float2 v = c[a];
      const cf z = cmul(cf{v.x, v.y}, cf{h.x, h.y});
      c[a] = make_float2(z.x, z.y);
    }
    __syncthreads();
    fft2048<true>(c, tw);
    float *y = b.bufB + (size_t)e * b.stride;
    const float sc = 1.0f / 2048.0f;
    for (int t = m - 1 + threadIdx.x; t < FFTN; t += FFT_T) {
      const int i0 = s0 + t - (m - 1);
      if (i0 < ghi) y[i0] = c[pidx(t)].x * sc;
      if (has1) {
        const int i1 = s1 + t - (m - 1);
        if (i1 < ghi) y[i1] = c[pidx(t)].y * sc;
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
// tile blockIdx.x of one spectrum: in -> out, all pixels
__device__ __forceinline__ void k_gauss_alone_body(int N, const DevStar &st, const float *in, float *out) {
  __shared__ float sbuf[G_TILE + 2 * G_HMAX];
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
__global__ void __launch_bounds__(GT) k_gauss_alone(int N, const DevStar *stp, const float *in, float *out) {
  k_gauss_alone_body(N, *stp, in, out);
}
// M spectra of N pixels at once: grid y = spectrum
__global__ void __launch_bounds__(GT) k_gauss_batch(int N, const DevStar *stp, const float *in, float *out) {
  const size_t off = (size_t)blockIdx.y * N;
  k_gauss_alone_body(N, *stp, in + off, out + off);
}
void launch_gauss_batch(int N, const DevStar *star, const float *in, float *out, int M, cudaStream_t s) {
  if (M <= 0 || N <= 0) return;
  k_gauss_batch<<<dim3((N + G_TILE - 1) / G_TILE, M), GT, 0, s>>>(N, star, in, out);
  count_launch();
}

// shift_and_resample at RV 0 (convolve_rv.rs:532-604) of M rows of N synth
// pixels to the star's observed pixels: out [M][n_obs]
__global__ void k_resample_rows(int N, int kind, const DevStar *stp, const float *in, float *out) {
  const DevStar &st = *stp;
  Resampler R;
  R.s = in + (size_t)blockIdx.y * N;
  R.N = N;
  R.kind = kind;
  R.shift_log = 0.0;
  R.shift_factor = 1.0;
  R.lin_offset = 0.0;
  R.fidx = st.fidx;
  R.wl_obs = st.wl_obs;
  R.wl_vals = nullptr;
  R.given = nullptr;
  float *o = out + (size_t)blockIdx.y * st.n_obs;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < st.n_obs; i += gridDim.x * blockDim.x) o[i] = R(i);
}
void launch_resample_rows(int N, int kind, const DevStar *star, int n_obs, const float *in, float *out, int M,
                          cudaStream_t s) {
  if (M <= 0 || n_obs <= 0) return;
  k_resample_rows<<<dim3((n_obs + 255) / 256, M), 256, 0, s>>>(N, kind, star, in, out);
  count_launch();
}

void launch_gauss_standalone(const DevGrid &G, const DevStar *star, const float *in, float *out, cudaStream_t s) {
  k_gauss_alone<<<(G.npx + G_TILE - 1) / G_TILE, GT, 0, s>>>(G.npx, star, in, out);
  count_launch();
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
// pixels per lane whose loads the chunk kernels issue together: 8 up to
// degree 5 (the Legendre values of 8 pixels fit the 64 registers of 4 CTAs
// per SM), 4 above
template <int K>
__host__ __device__ constexpr int chunk_cu() {
  return K <= 6 ? 8 : 4;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Dot product of each row with x (InMemInterpolator.ccf, lib.rs:1340-1371):
// one CTA per row, FP64 sums, rounded to f32 once; NaN for a failed row.
__global__ void __launch_bounds__(256) k_dot_rows(const float *rows, int64_t stride, int n, const float *x,
                                                   const int *status, float *out) {
  __shared__ double ws[8];
  const int r = blockIdx.x, t = threadIdx.x;
  const bool ok = status[r] == 0;
  double acc = 0.0;
  if (ok) {
    const float *row = rows + (size_t)r * stride;
    for (int i = t; i < n; i += 256) acc = fma((double)row[i], (double)x[i], acc);
  }
  acc = warp_sum(acc);
  if ((t & 31) == 0) ws[t >> 5] = acc;
  __syncthreads();
  if (t == 0) {
    double tot = 0.0;
    for (int k = 0; k < 8; k++) tot += ws[k];
    out[r] = ok ? (float)tot : __int_as_float(0x7fc00000);
  }
}
void launch_dot_rows(const float *rows, int64_t stride, int n, const float *x, const int *status, float *out, int L,
                     cudaStream_t s) {
  if (L <= 0) return;
  k_dot_rows<<<L, 256, 0, s>>>(rows, stride, n, x, status, out);
  count_launch();
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

// model at the observed pixels of evaluation e
__device__ __forceinline__ const float *model_row(const EvalBatch &b, const EvalPrep &P, int e) {
  if (b.given) return b.given + (size_t)e * b.given_stride;
  return (P.mobs_in_b ? b.bufB : b.bufA) + (size_t)e * b.stride;
}

// Evaluations that k_broaden did not resample: the model at the observed
// pixels from the final synth row, into the buffer the synth row is not in.
__global__ void k_resample_obs(DevGrid G, EvalBatch b) {
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  if (P.status || P.epi) return;
  const DevStar &st = b.stars[P.star];
  const Resampler R = make_resampler(G, st, P, final_row(b, P, e), nullptr);
  float *out = (P.mobs_in_b ? b.bufB : b.bufA) + (size_t)e * b.stride;
  for (int i = blockIdx.y * blockDim.x + threadIdx.x; i < st.n_obs; i += gridDim.y * blockDim.x) out[i] = R(i);
}
void launch_resample_obs(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0) return;
  dim3 grid(b.E, 8);
  k_resample_obs<<<grid, 256, 0, s>>>(G, b);
  count_launch();
}

// ChunkFitter::fit_continuum (continuum_fitting.rs:382-396), one warp per
// (evaluation, chunk): the unweighted least-squares polynomial of
// flux/model over the chunk (216-226) is the projection onto the chunk's
// polynomial space; it is solved here in a Legendre basis with the FP64
// Cholesky factor of its Gram matrix (the same space as the reference's
// monomial SVD, far better conditioned).  A lane sums the products
// P_k(x) y of its CU pixels in f32 and adds that partial to its running
// FP64 moment: one f32 -> f64 conversion per moment per CU pixels instead of
// one per pixel (the conversions share the narrow XU pipe with the
// division's reciprocal), and a short FP64 dependency chain.
// K = polynomial order + 1 (one instantiation per order present).  A warp
// walks the whole chunk (no block barriers), so the loads of many chunks
// are in flight per SM.
// Moments of chunk c walked by one warp; lane 0 then solves G a = z with the
// chunk's FP64 Cholesky factor, leaving the Legendre coefficients in a[0..K)
// (and the reference's parameters in b.params when requested).
template <int K>
__device__ __forceinline__ void chunk_solve_warp(const EvalBatch &b, const DevStar &st, const float *mod, int e,
                                                 int c, int lane, double *a) {
  const float *flux = st.flux;
  const int lo = st.cstart[c], hi = st.cstop[c], prev = c > 0 ? st.cstop[c - 1] : -1;
  if (lane == 0 && !b.given) prefetch_row_l2(mod, lo, hi);  // the walk below then reads from L2
  constexpr int CU = chunk_cu<K>();
  double z[K];
#pragma unroll
  for (int k = 0; k < K; k++) z[k] = 0.0;
  // pixels [a0, a1) with chunk coordinates xs (the upper-chunk coordinate
  // below the previous chunk's stop); loads of CU pixels are issued before
  // any arithmetic on them
  auto walk = [&](int a0, int a1, const float *__restrict__ xs) {
    for (int i0 = a0 + lane; i0 < a1; i0 += 32 * CU) {
      float fl[CU], md[CU], xf[CU];
#pragma unroll
      for (int u = 0; u < CU; u++) {
        const int i = min(i0 + 32 * u, a1 - 1);
        fl[u] = flux[i];
        md[u] = mod[i];
        xf[u] = xs[i];
      }
      float zp[K];
#pragma unroll
      for (int k = 0; k < K; k++) zp[k] = 0.0f;
#pragma unroll
      for (int u = 0; u < CU; u++) {
        if (i0 + 32 * u < a1) {
          // flux / model as x * rcp(y) (at most 2 ulp; the moments are sums
          // of thousands of such terms, accumulated in FP64)
          const float y = __fdividef(fl[u], md[u]);
          float Pk[K];
          legendre<K>(xf[u], Pk);
#pragma unroll
          for (int k = 0; k < K; k++) zp[k] = fmaf(Pk[k], y, zp[k]);
        }
      }
#pragma unroll
      for (int k = 0; k < K; k++) z[k] += (double)zp[k];
    }
  };
  const int split = c > 0 ? min(max(prev, lo), hi) : lo;
  walk(lo, split, st.xb);
  walk(split, hi, st.xa);
#pragma unroll
  for (int k = 0; k < K; k++) {
    const double t = warp_sum(z[k]);
    if (lane == 0) a[k] = t;
  }
  if (lane == 0) {  // FP64 Cholesky solve G a = z, in place
    const double *L = st.chol + (size_t)c * K * K;
    for (int k = 0; k < K; k++) {
      double t = a[k];
      for (int j = 0; j < k; j++) t -= L[k * K + j] * a[j];
      a[k] = t / L[k * K + k];
    }
    for (int k = K - 1; k >= 0; k--) {
      double t = a[k];
      for (int j = k + 1; j < K; j++) t -= L[j * K + k] * a[j];
      a[k] = t / L[k * K + k];
    }
    if (b.params) {
      double *par = b.params + (size_t)e * b.param_stride + c * K;
      for (int k = 0; k < K; k++) par[k] = a[k];
    }
  }
}

// Monomial coefficients of the Legendre polynomials, T[k][j] = coefficient
// of x^j in P_k, from (k + 1) P_{k+1} = (2k + 1) x P_k - k P_{k-1} (dyadic
// rationals, exact in double up to degree 15).
struct LegMono {
  double c[MAX_P1][MAX_P1];
};
constexpr LegMono make_leg_mono() {
  LegMono t{};
  t.c[0][0] = 1.0;
  t.c[1][1] = 1.0;
  for (int k = 1; k + 1 < MAX_P1; k++)
    for (int j = 0; j < MAX_P1; j++)
      t.c[k + 1][j] = ((2 * k + 1) * (j > 0 ? t.c[k][j - 1] : 0.0) - k * t.c[k - 1][j]) / (k + 1);
  return t;
}
__constant__ LegMono c_leg_mono = make_leg_mono();

// the chunk polynomial sum_k a_k P_k(x) as monomial coefficients (FP64),
// rounded to f32 for Horner evaluation
template <int K>
__device__ __forceinline__ void legendre_to_monomial(const double *a, float *m) {
  for (int j = 0; j < K; j++) {
    double s = 0.0;
    for (int k = j; k < K; k++) s = fma(a[k], c_leg_mono.c[k][j], s);
    m[j] = (float)s;
  }
}

template <int K>
__device__ __forceinline__ float horner(const float (&a)[K], float x) {
  float p = a[K - 1];
#pragma unroll
  for (int j = K - 2; j >= 0; j--) p = fmaf(p, x, a[j]);
  return p;
}

// chi2 section of chunk c (continuum_fitting.rs:280-360) walked by one
// warp: chunk 0 alone on [50, start_1); chunk c >= 1 blended with chunk
// c - 1 (sin^2 factor) on [start_c, stop_{c-1}), then alone up to
// start_{c+1} (N - 50 for the last).  A lane adds the terms of the pixels
// it loads together in f32 and those partials in FP64; the warp's sum is
// returned to lane 0.
template <int K>
__device__ __forceinline__ double chunk_resid_warp(const DevStar &st, const float *mod, int c, int lane,
                                                   const float (&cc)[K], const float (&cp)[K]) {
  const int N = st.n_obs, nc = st.n_chunks;
  const float *flux = st.flux, *var = st.var;
  double acc = 0.0;
  constexpr int CU = chunk_cu<K>();
  // [lo, hi) with chunk c alone; loads of CU pixels before their arithmetic
  auto alone = [&](int lo, int hi) {
    for (int i0 = lo + lane; i0 < hi; i0 += 32 * CU) {
      float fl[CU], md[CU], vr[CU], xa[CU];
#pragma unroll
      for (int u = 0; u < CU; u++) {
        const int i = min(i0 + 32 * u, hi - 1);
        fl[u] = flux[i];
        md[u] = mod[i];
        vr[u] = var[i];
        xa[u] = st.xa[i];
      }
      float part = 0.0f;  // the lane's CU terms in f32, then one FP64 add
#pragma unroll
      for (int u = 0; u < CU; u++) {
        if (i0 + 32 * u < hi) {
          const float p = horner<K>(cc, xa[u]);
          const float r = fl[u] - p * md[u];
          part += __fdividef(r * r, vr[u]);
        }
      }
      acc += (double)part;
    }
  };
  if (c == 0) {
    alone(50, st.cstart[1]);
  } else {
    const int s0 = st.cstart[c], sp = st.cstop[c - 1];
    const int nx = c == nc - 1 ? N - 50 : st.cstart[c + 1];
    for (int i0 = s0 + lane; i0 < sp; i0 += 32 * 2) {  // overlap: blend previous and current
      float fl[2], md[2], vr[2], xa[2], xb[2], fc[2];
#pragma unroll
      for (int u = 0; u < 2; u++) {
        const int i = min(i0 + 32 * u, sp - 1);
        fl[u] = flux[i];
        md[u] = mod[i];
        vr[u] = var[i];
        xa[u] = st.xa[i];
        xb[u] = st.xb[i];
        fc[u] = st.fac[i];
      }
      float part = 0.0f;
#pragma unroll
      for (int u = 0; u < 2; u++) {
        if (i0 + 32 * u < sp) {
          const float pv = horner<K>(cp, xa[u]);
          const float cu = horner<K>(cc, xb[u]);
          const float p = pv * fc[u] + cu * (1.0f - fc[u]);
          const float r = fl[u] - p * md[u];
          part += __fdividef(r * r, vr[u]);
        }
      }
      acc += (double)part;
    }
    alone(sp, nx);
  }
  return warp_sum(acc);
}

// ChunkFitter::fit_continuum + compute_chi2_from_chunks
// (continuum_fitting.rs:216-226, 280-360, 382-396) for one evaluation per
// CTA: warp w takes chunks w, w + 8, ...  First every chunk's moments and
// FP64 solve: the unweighted least-squares polynomial of flux/model over
// the chunk is the projection onto the chunk's polynomial space, solved here
// in a Legendre basis with the Cholesky factor of its Gram matrix (the same
// space as the reference's monomial SVD, far better conditioned).  After a
// CTA barrier every chunk section's chi2 from the coefficients in shared
// memory, reading the model row a second time while it is still in L2;
// then the sections added in chunk order in FP64 / (N - 100).  Errors give
// NaN with the evaluation's status.  K = polynomial order + 1 (one
// instantiation per order present; other orders return at once).
template <int K>
__global__ void __launch_bounds__(CT, K <= 8 ? 4 : 2) k_chunk_fit(EvalBatch b) {
  __shared__ double zs[MAX_CHUNKS][MAX_P1];
  __shared__ float cfs[MAX_CHUNKS][MAX_P1];
  __shared__ double part[MAX_CHUNKS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  const DevStar &st = b.stars[P.star];
  if (st.cont_kind != CONT_CHUNK || st.p1 != K) return;
  int status = P.status;
  if (!status && st.cont_bad) status = S_CONTINUUM;
  if (status) {
    write_result(b, e, 0.0, status);
    return;
  }
  const float *mod = model_row(b, P, e);
  const int nc = st.n_chunks;
  for (int c = warp; c < nc; c += CW) {
    chunk_solve_warp<K>(b, st, mod, e, c, lane, zs[c]);
    if (lane == 0) legendre_to_monomial<K>(zs[c], cfs[c]);
  }
  __syncthreads();
  for (int c = warp; c < nc; c += CW) {
    float cc[K], cp[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
      cc[k] = cfs[c][k];
      cp[k] = c > 0 ? cfs[c - 1][k] : 0.0f;
    }
    const double acc = chunk_resid_warp<K>(st, mod, c, lane, cc, cp);
    if (lane == 0) part[c] = acc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double chi2 = 0.0;
    for (int c = 0; c < nc; c++) chi2 += part[c];
    write_result(b, e, chi2 / (double)(st.n_obs - 100), 0);
  }
}

// LinearModelFitter (continuum_fitting.rs:68-95): projection onto the design
// matrix's column space through its orthonormal basis Q; chi2 of the
// ratio-space residual over [50, N-50) divided by N.  FixedContinuum
// (441-474) and ConstantContinuum (484-500) too.  One CTA per evaluation.
__global__ void __launch_bounds__(CT) k_chi2_other(DevGrid G, EvalBatch b) {
  __shared__ double ws[CW][MAX_P1];
  __shared__ double zs[MAX_LIN_K];
  const int e = blockIdx.x;
  const EvalPrep &P = b.prep[e];
  const DevStar &st = b.stars[P.star];
  if (st.cont_kind == CONT_CHUNK) return;
  if (st.cont_kind == CONT_LINEAR && st.kp > 0 && b.lin_group > 0) return;  // k_linear_tc
  if (P.status) {
    write_result(b, e, 0.0, P.status);
    return;
  }
  if (st.cont_bad) {
    write_result(b, e, 0.0, S_CONTINUUM);
    return;
  }
  const int N = st.n_obs;
  const float *mod = model_row(b, P, e);
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
        const double bd = (double)(flux[i] / mod[i]);
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
      const float bb = flux[i] / mod[i];
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
      const float r = flux[i] - mod[i] * st.cont[i];
      acc += (double)(r / var[i] * r);
    }
    chi2 = block_sum(acc, ws) / (double)(N - 2 * ig);
    if (par && threadIdx.x == 0) par[0] = 0.0;
  } else {
    double sum = 0.0;
    for (int i = threadIdx.x; i < N; i += CT) sum += (double)(flux[i] / mod[i]);
    const float mean = (float)(block_sum(sum, ws) / (double)N);
    double acc = 0.0;
    for (int i = threadIdx.x; i < N; i += CT) {
      const float r = flux[i] - mod[i] * mean;
      acc += (double)(r / var[i] * r);
    }
    chi2 = block_sum(acc, ws) / (double)N;
    if (par && threadIdx.x == 0) par[0] = (double)mean;
  }
  write_result(b, e, chi2, 0);
}

template <int K>
static void launch_chunk(const EvalBatch &b, cudaStream_t s) {
  k_chunk_fit<K><<<b.E, CT, 0, s>>>(b);
  count_launch();
}

// chi2 of every evaluation from the model at its observed pixels
// (model_row: resampled by k_broaden / k_resample_obs, or given)
void launch_chi2(const DevGrid &G, const EvalBatch &b, cudaStream_t s) {
  if (b.E <= 0) return;
  const uint32_t m = b.chunk_p1_mask;
  if (m && b.max_chunks > 0) {
    if (m & (1u << 1)) launch_chunk<1>(b, s);
    if (m & (1u << 2)) launch_chunk<2>(b, s);
    if (m & (1u << 3)) launch_chunk<3>(b, s);
    if (m & (1u << 4)) launch_chunk<4>(b, s);
    if (m & (1u << 5)) launch_chunk<5>(b, s);
    if (m & (1u << 6)) launch_chunk<6>(b, s);
    if (m & (1u << 7)) launch_chunk<7>(b, s);
    if (m & (1u << 8)) launch_chunk<8>(b, s);
    if (m & (1u << 9)) launch_chunk<9>(b, s);
    if (m & (1u << 10)) launch_chunk<10>(b, s);
    if (m & (1u << 11)) launch_chunk<11>(b, s);
    if (m & (1u << 12)) launch_chunk<12>(b, s);
    if (m & (1u << 13)) launch_chunk<13>(b, s);
    if (m & (1u << 14)) launch_chunk<14>(b, s);
    if (m & (1u << 15)) launch_chunk<15>(b, s);
    if (m & (1u << 16)) launch_chunk<16>(b, s);
  }
  if (b.other_cont) {
    if (b.lin_group > 0) launch_linear_tc(b, s);
    k_chi2_other<<<b.E, CT, 0, s>>>(G, b);
    count_launch();
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
    const int V = (*may_unfuse ? MIN_FUSED_OUTPUTS : FFTN - wide) - 1;  // block advance
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
  launch_group(G, b, s);
  launch_interp_tc(G, b, s);
  launch_interp(G, b, s);
  launch_obs_bounds(G, b, s);
  launch_broaden(G, b, tw, s);
  launch_direct(G, b, s);
  if (o.may_unfuse) {
    launch_rot(G, b, tw, s);
    launch_gauss(G, b, s);
  }
  if (b.need_chi2) {
    launch_resample_obs(G, b, s);
    launch_chi2(G, b, s);
  } else if (b.status) {
    launch_prep_status(b, s);
  }
}

}  // namespace pb
