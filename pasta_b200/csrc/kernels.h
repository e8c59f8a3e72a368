// kernels.h -- launch wrappers of the pasta_b200 sm_100a kernels.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace pb {

// Evaluations that share all 64 neighbour rows (same grid cube), up to
// GROUP_MAX per group, found among SEG consecutive evaluations (the
// particles of one star in the batched engine), with the rows they use in
// reference order (zero-weight rows of every member dropped, padded to a
// multiple of 8 with zero weights).
constexpr int GROUP_MAX = 8, SEG = 64;
constexpr int MERGE_CAP = 64;  // evaluations one merge-table slot takes (in groups of GROUP_MAX)
struct __align__(16) GroupRec {
  float4 wf[64][2];       // per member (8) weight x dequantisation factor (0: padding / not a member)
  float4 w[64][2];        // per member weight (the exact tail path)
  int col[64];            // grid row of compacted neighbour n
  float f[64];            // its dequantisation factor
  int member[GROUP_MAX];  // evaluation indices (-1: unused)
  int nmem, nn;           // members, compacted rows
  int pad[2];
};

// Evaluations with identical neighbour columns, EvalBatch::tc_min or more
// of them in one segment (at least TC_MIN_MEMBERS), are interpolated
// together on the tensor cores (interp_tc.cu): the group's rows are staged
// by TMA and its members' weights are the columns of one matrix product.
constexpr int TC_MIN_MEMBERS = 8, TC_MAX_GROUPS = SEG / TC_MIN_MEMBERS;
struct __align__(16) TcGroup {
  int member[SEG];  // evaluation indices, ascending (first nmem valid)
  int col[64];      // the shared neighbour columns (-1: missing)
  float f[64];      // their dequantisation factors (0 for missing)
  int nmem;
  int lo, hi;       // union of the members' interpolation windows [i_lo, i_hi)
  int pad;
};

constexpr int LIN_MAX_SLICES = 32;  // at most MAX_CHUNKS: the slices' residual sums use EvalBatch::cpart

// Per-launch description of one batch of evaluations.
struct EvalBatch {
  int E;                     // evaluations in this batch
  const double *labels;      // [E][5]
  const int *eval_star;      // [E] index into stars
  const int *eval_active;    // [E] or null: 0 = skip
  const DevStar *stars;
  EvalPrep *prep;            // [E]
  float2 *H;                 // [E][1025] rotation kernel half-spectra
  float2 *HG;                // [E][1025] the same times the fixed instrument spectrum (or null)
  float *bufA, *bufB;        // [E][stride] spectra workspaces
  int64_t stride;            // floats per evaluation row
  double *cost;              // [E]
  int *status;               // [E]
  double *params;            // [E][param_stride] or null
  int param_stride;
  int max_pairs;             // fused broadening: max ceil(nblk/2) over the batch
  int max_pairs_unfused;     // unfused rotation FFT: max ceil(nblk/2) (0: none can occur)
  int need_chi2;
  uint32_t chunk_p1_mask;    // bit p1 set: a chunk continuum with p1 coefficients is present
  int other_cont;            // a linear / fixed / constant continuum is present
  int max_chunks;            // most chunks of any chunk continuum in the batch
  int obs_epi;               // chi2 batches: resample inside k_broaden, synth rows are not kept
  int *bnd;                  // [E][bnd_stride] first observed pixel of every broadening block
  int bnd_stride;
  double *cpart;             // [E][MAX_CHUNKS] chi2 partial sums per chunk section
  // Segments: the evaluations of each star (seg_len consecutive ones; 0:
  // the whole batch is one star) in chunks of at most SEG from the star's
  // first evaluation, so a star's groups do not depend on the rest of the
  // batch.  A segment's records sit at its first evaluation's index.
  int seg_len;
  GroupRec *grec;            // [E] groups of each segment, in order
  int *gcount;               // [segments] groups per segment
  TcGroup *tcrec;            // [E] tensor-core groups of each segment (null: none)
  int *tclist;               // [E] indices into tcrec of all tensor-core groups, in any order
  int *tclist_count;         // [1] their number (zeroed before k_group)
  int tc_min;                // members a tensor-core group needs (TC_MIN_MEMBERS .. SEG; larger: none)
  int *tccount;              // [segments]
  // Evaluations that end up alone in their segment (spread swarms: the early
  // iterations of a fit) are merged across segments with the others that
  // have the same neighbour columns, in groups of up to GROUP_MAX, when mkey
  // is set (null: off).  Merging changes no result: every member keeps its
  // own accumulators and row order.
  unsigned long long *mkey;  // [mtab] hash of the columns per table slot (0: empty); zeroed before k_group
  int *mcnt;                 // [mtab] evaluations that chose each slot; zeroed before k_group
  int *mmem;                 // [mtab][MERGE_CAP] the first MERGE_CAP of them
  int *mslot;                // [1 + mtab] number of slots with two or more evaluations, then the slots
  int mtab;                  // table slots (a power of two, at least 2 E)
  int *erec;                 // [E] record index of the evaluation's own (alone) group
  GroupRec *mrec;            // [(E + 1) / 2] merged group records (at most half the evaluations)
  int *mrcount;              // [1] their number
  const void *tmap;          // host pointer to the grid's TMA tensor map (null: no tensor-core path)
  const float *given;        // model given at the observed pixels (continuum utilities) or null
  int64_t given_stride;      // floats between the given rows of consecutive evaluations
  int direct_max;            // combined kernels of at most this many taps are convolved directly (0: never)
  int max_dtiles;            // direct tiles per evaluation at most (at least DIRECT_TILE - DIRECT_MAX_TAPS outputs each)
  int *direct_list;          // [E] evaluations k_prep routed to the direct path (in any order)
  int *direct_count;         // [1] their number (zeroed before k_prep)
  int lin_group;             // linear continua on the tensor cores: groups of this many consecutive
                             // evaluations share a star (0: the CUDA-core path)
  uint32_t lin_kp_mask;      // bit kp / 16: a linear continuum with a kp-column tensor-core basis is present
  int lin_slices;            // pixel slices per group (1..LIN_MAX_SLICES)
  double *lin_zpart;         // [E][LIN_MAX_SLICES][64] partial coefficients of the slices
};

// int entries per evaluation of EvalBatch::bnd for a grid of npx pixels
inline int bnd_stride_for(int npx) { return npx / (MIN_FUSED_OUTPUTS - 1) + 3; }

// Everything from the preparation to chi2 (or to the outputs) for one batch.
struct PipelineOpts {
  int full_window = 0;       // every synthetic pixel, no resampling (interpolate entry points)
  int rot = 1;               // some evaluation may rotate (launch the rotation spectra)
  int may_unfuse = 0;        // some evaluation may need the unfused path
};
void launch_pipeline(const DevGrid &G, const EvalBatch &b, const float2 *twiddle, const PipelineOpts &o,
                     cudaStream_t s);
// pair counts for a batch whose widest rotation is max_m taps and widest
// instrument half width max_hg
void pipeline_pairs(int npx, int max_m, int max_hg, int *max_pairs, int *max_pairs_unfused, int *may_unfuse);

void launch_prep(const DevGrid &G, const EvalBatch &b, cudaStream_t s);
// same, for entry points that need every synthetic pixel and no resampling
void launch_prep_full(const DevGrid &G, const EvalBatch &b, cudaStream_t s);
void launch_rotker(const DevGrid &G, const EvalBatch &b, const float2 *twiddle, cudaStream_t s);
// groups of evaluations sharing their neighbour rows (after the preparation)
void launch_group(const DevGrid &G, const EvalBatch &b, cudaStream_t s);
void launch_interp(const DevGrid &G, const EvalBatch &b, cudaStream_t s);
// tensor-core interpolation of the groups k_group marked (interp_tc.cu)
void launch_interp_tc(const DevGrid &G, const EvalBatch &b, cudaStream_t s);
// segments of a batch (see EvalBatch::seg_len)
int num_segments(const EvalBatch &b);
// the grid's TMA tensor map: uint16 [rows][stride], box 128 pixels x 1 row
// (host side; out points to a CUtensorMap); false when the driver lacks it
bool make_grid_tensor_map(const uint16_t *spectra, int64_t rows, int64_t stride, void *out);
// first observed pixel of every fused broadening block (chi2 batches)
void launch_obs_bounds(const DevGrid &G, const EvalBatch &b, cudaStream_t s);
void launch_broaden(const DevGrid &G, const EvalBatch &b, const float2 *twiddle, cudaStream_t s);
// direct convolution of the evaluations k_prep routed to it (EvalPrep::direct)
void launch_direct(const DevGrid &G, const EvalBatch &b, cudaStream_t s);
void launch_rot(const DevGrid &G, const EvalBatch &b, const float2 *twiddle, cudaStream_t s);
void launch_gauss(const DevGrid &G, const EvalBatch &b, cudaStream_t s);
// model at the observed pixels for the evaluations k_broaden did not resample
void launch_resample_obs(const DevGrid &G, const EvalBatch &b, cudaStream_t s);
// chi2 from the model at the observed pixels (b.given when set)
void launch_chi2(const DevGrid &G, const EvalBatch &b, cudaStream_t s);
// linear-model continua on the tensor cores, every basis width present (lintc.cu)
void launch_linear_tc(const EvalBatch &b, cudaStream_t s);
// copy the preparation status to b.status (batches without chi2)
void launch_prep_status(const EvalBatch &b, cudaStream_t s);
// model at the observed pixels: out [E][out_stride]
// out[r] = rows[r] . x (n values, FP64 sums), NaN where status[r] != 0
void launch_dot_rows(const float *rows, int64_t stride, int n, const float *x, const int *status, float *out, int L,
                     cudaStream_t s);
void launch_resample_out(const DevGrid &G, const EvalBatch &b, float *out, int64_t out_stride,
                         cudaStream_t s);
// broadened synth spectrum (before resampling): out [E][npx]
void launch_copy_broadened(const DevGrid &G, const EvalBatch &b, float *out, cudaStream_t s);
void launch_build_chunk(const DevStar *star, const double *coef, int n, float *out, cudaStream_t s);
void launch_gauss_standalone(const DevGrid &G, const DevStar *star, const float *in, float *out,
                             cudaStream_t s);
// instrument profile of M spectra of N pixels: in, out [M][N]
void launch_gauss_batch(int N, const DevStar *star, const float *in, float *out, int M, cudaStream_t s);
// resampling at RV 0 of M rows of N synth pixels (grid kind WL_*) to the star's n_obs observed pixels
void launch_resample_rows(int N, int kind, const DevStar *star, int n_obs, const float *in, float *out, int M,
                          cudaStream_t s);

// ---------------------------------------------------------------- binaries
// Linear interpolation corners of one component's continuum
// (interpolate.rs:536-600): 8 grid rows, their f32 weights and factors.
struct LinRec {
  int cols[8];
  float w[8];
  float f[8];
  int status;
};
// L binary labels (star 1 [5], star 2 [5], light ratio) evaluated as 2L
// component evaluations: star 1 of every label, then star 2 of every label.
struct BinaryBatch {
  int L;
  const double *labels;   // [L][11]
  double *comp_labels;    // [2L][5] (RV 0: the shift is applied per observed pixel)
  LinRec *lin;            // [2L]
  double *part;           // [2L][lin_tiles] partial sums of the continuum rows
  int lin_tiles;
  EvalPrep *cprep;        // [L] status and star of every label for the continuum fit
  float *model;           // [L][model_stride] binary model at the observed pixels
  int64_t model_stride;
};
int linear_tiles(int npx);
// component labels and continuum corners (Gc: the continuum grid)
void launch_binary_split(const DevGrid &Gc, const BinaryBatch &bb, cudaStream_t s);
// continuum rows into the workspace buffer without the broadened row
void launch_interp_linear(const DevGrid &Gc, const EvalBatch &comp, const BinaryBatch &bb, cudaStream_t s);
// interpolate_linear entry point: corners of L labels [L][3], then R rows into
// out [R][stride] with the per-tile sums part [R][linear_tiles(npx)]
void launch_linear_prep(const DevGrid &Gc, const double *tml, int L, LinRec *lin, cudaStream_t s);
void launch_interp_linear_rows(const DevGrid &Gc, const LinRec *lin, int R, float *out, int64_t stride,
                               double *part, cudaStream_t s);
// light ratio, shift, resampling and sum of the two stars (Nc continuum pixels)
void launch_binary_combine(const DevGrid &G, int Nc, const EvalBatch &comp, const BinaryBatch &bb, int n_obs,
                           cudaStream_t s);

// swarm state of S stars x Pmax particles (structure of arrays)
struct Swarm {
  int S, Pmax;
  double *x, *v, *bx;        // [S][Pmax][5]
  double *cost, *bcost;      // [S][Pmax]
  double *gx, *gcost;        // [S][5], [S]
  int *iter, *status, *done; // [S]
  int *active;               // [S] slot in use
  uint64_t *seed;            // [S]
  PsoParams *params;         // [S]
  double *labels;            // [S*Pmax][5] evaluation labels
  int *eval_active;          // [S*Pmax]
  int *refit;                // [S] or null: 1 for a swarm that finished successfully in this step
};
// positions for this step (update, or publish host-placed initial positions)
void launch_pso_update(const DevGrid &G, const Swarm &w, cudaStream_t s);
// after evaluation: initial sort or best update, iteration counter, done flags
void launch_pso_best(const Swarm &w, const double *cost, const int *status, cudaStream_t s);

int64_t kernel_launches();
void count_launch(int n = 1);

}  // namespace pb
