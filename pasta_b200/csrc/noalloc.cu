// noalloc.cu -- chi2 of a batch of labels without allocating device memory.
//
// Some callers of this library cannot call cudaMalloc.  A host framework may
// hand the whole of the GPU's memory to its own pool allocator at start-up.
// A real-time loop may not take the driver's allocation path (cudaMalloc can
// synchronise the device) between frames.  A multi-tenant service may have
// its footprint fixed once the process is up.  For them pasta_chi2_noalloc
// evaluates chi2 exactly like pasta_chi2.  The inputs and outputs are device
// buffers the caller already owns.  The evaluation workspace lives in the
// file-scope array g_noalloc_scratch below.
//
// The array is NOALLOC_SCRATCH_BYTES (32 MiB).  Every GPU that loads the
// library holds it until the process exits.  All calls share it and it keeps
// the last call's contents.  No part of it has to start at zero: every stage
// writes the rows it later reads.  Calls whose work overlaps on the GPU race
// on the array, so a caller serialises its calls (one stream, or
// synchronisation between streams).
//
// Set-up: the first call on a device, with that device current, resolves
// the array's device address with cudaGetSymbolAddress and copies the FFT
// twiddle table into g_noalloc_twiddle.  That first call should therefore
// come before any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/pasta_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace pb {
int internal_eval_view(const pasta_grid *g, const pasta_dispersion *d, const pasta_continuum *c, const float *flux,
                       const float *var, int64_t n, DevGrid *grid, int64_t *stride, DevStar *star, int *device,
                       std::string *err);
void internal_set_last_error(const std::string &msg);
}

using namespace pb;

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = 32u << 20;
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) float2 g_noalloc_twiddle[FFTN];

struct DeviceSetup {
  bool ready = false;
  unsigned char *scratch = nullptr;
  float2 *twiddle = nullptr;
};
std::mutex g_setup_mu;
DeviceSetup g_setup[MAX_DEVICES];

// errors are reported through pasta_last_error()
struct ErrSink {
  ErrSink &operator=(const std::string &m) {
    internal_set_last_error(m);
    return *this;
  }
  ErrSink &operator=(const char *m) { return *this = std::string(m); }
} g_noalloc_err;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// bytes of scratch one label needs: prep record, rotation half spectra
// (alone and times the instrument spectrum),
// eval->star index, the two spectrum rows, the broadening block bounds and
// the partial chi2 sums
size_t per_label_bytes(int64_t stride, int bnd_stride) {
  return align256(sizeof(EvalPrep)) + 2 * align256(1025 * sizeof(float2)) + align256(sizeof(int)) +
         2 * align256((size_t)stride * sizeof(float)) + align256((size_t)bnd_stride * sizeof(int)) +
         align256((size_t)MAX_CHUNKS * sizeof(double)) +
         align256(sizeof(GroupRec)) + align256(sizeof(int));
}

int setup_device(int dev, DeviceSetup **out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (dev < 0 || dev >= MAX_DEVICES) {
    g_noalloc_err = "device index out of range";
    return PASTA_E_ARG;
  }
  DeviceSetup &s = g_setup[dev];
  if (!s.ready) {
    cudaError_t e = cudaGetSymbolAddress((void **)&s.scratch, g_noalloc_scratch);
    if (e != cudaSuccess) {
      g_noalloc_err = std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") + cudaGetErrorString(e);
      return PASTA_E_CUDA;
    }
    e = cudaGetSymbolAddress((void **)&s.twiddle, g_noalloc_twiddle);
    if (e != cudaSuccess) {
      g_noalloc_err = std::string("cudaGetSymbolAddress(g_noalloc_twiddle) failed: ") + cudaGetErrorString(e);
      return PASTA_E_CUDA;
    }
    float2 tw[FFTN];
    for (int k = 0; k < FFTN; k++) {
      const double a = -2.0 * M_PI * (double)k / (double)FFTN;
      tw[k] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    e = cudaMemcpyToSymbol(g_noalloc_twiddle, tw, sizeof tw);
    if (e != cudaSuccess) {
      g_noalloc_err = std::string("twiddle upload failed: ") + cudaGetErrorString(e);
      return PASTA_E_CUDA;
    }
    s.ready = true;
  }
  *out = &s;
  return PASTA_OK;
}

// writes the star descriptor and the all-zero eval->star map into scratch
__global__ void k_noalloc_init(DevStar st, DevStar *dst, int *eval_star, int L) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *dst = st;
  if (i < L) eval_star[i] = 0;
}

}  // namespace

// chi2 of L labels (like pasta_chi2) with every buffer supplied by the caller:
// flux, var [n] f32, labels [L x 5] f64, out [L] f64, status [L] int32 are
// device pointers; stream is a cudaStream_t (NULL: the legacy default stream).
// Asynchronous: results are valid once the stream has reached this work.
// Restores the calling thread's current device on every return path, so a
// framework that works on another device finds its device unchanged.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

extern "C" int pasta_chi2_noalloc(const pasta_grid *g, const pasta_dispersion *d, const pasta_continuum *c,
                                  const float *flux, const float *var, int64_t n, const double *labels, int64_t L,
                                  double *out, int32_t *status, void *stream) {
  DeviceGuard keep_device;
  // an error left by the caller's own earlier work stays the caller's: it is
  // reported, not consumed, and nothing is launched
  if (cudaError_t pend = cudaPeekAtLastError(); pend != cudaSuccess) {
    g_noalloc_err = std::string("a CUDA error was already pending before this call: ") + cudaGetErrorString(pend);
    return PASTA_E_CUDA;
  }
  DevGrid G;
  DevStar star;
  int64_t stride = 0;
  int dev = 0;
  std::string err;
  int rc = internal_eval_view(g, d, c, flux, var, n, &G, &stride, &star, &dev, &err);
  if (rc) {
    g_noalloc_err = err;
    return rc;
  }
  if (!flux || !var || !labels || !out || !status) {
    g_noalloc_err = "flux, var, labels, out and status must be device pointers";
    return PASTA_E_ARG;
  }
  if (L < 0) {
    g_noalloc_err = "the label count must not be negative";
    return PASTA_E_ARG;
  }
  if (L == 0) return PASTA_OK;  // nothing to evaluate, like pasta_chi2
  stride = std::max<int64_t>(stride, (n + 63) / 64 * 64);  // rows also hold the model at the observed pixels
  const int bstr = bnd_stride_for(G.npx);
  // the star record, and the group slots of a partly filled last segment
  const size_t fixed = align256(sizeof(DevStar)) + align256((size_t)(SEG - 1) * sizeof(GroupRec)) + 256;
  const size_t per = per_label_bytes(stride, bstr);
  const int64_t max_labels = NOALLOC_SCRATCH_BYTES > fixed ? (int64_t)((NOALLOC_SCRATCH_BYTES - fixed) / per) : 0;
  if (L > max_labels) {
    char buf[256];
    snprintf(buf, sizeof buf,
             "%lld labels exceed the allocation-free scratch (%zu bytes): at most %lld labels for a grid of %lld "
             "pixels",
             (long long)L, NOALLOC_SCRATCH_BYTES, (long long)max_labels, (long long)G.npx);
    g_noalloc_err = buf;
    return PASTA_E_ARG;
  }
  cudaError_t e = cudaSetDevice(dev);
  if (e != cudaSuccess) {
    g_noalloc_err = std::string("cudaSetDevice failed: ") + cudaGetErrorString(e);
    return PASTA_E_CUDA;
  }
  if (stream) {
    int sdev = -1;
    if (cudaStreamGetDevice((cudaStream_t)stream, &sdev) == cudaSuccess && sdev != dev) {
      g_noalloc_err = "the stream belongs to another device than the grid";
      return PASTA_E_ARG;
    }
  }
  DeviceSetup *S = nullptr;
  rc = setup_device(dev, &S);
  if (rc) return rc;
  // carve the scratch
  unsigned char *p = S->scratch;
  DevStar *dstar = (DevStar *)p;
  p += fixed;
  EvalPrep *prep = (EvalPrep *)p;
  p += align256(sizeof(EvalPrep) * (size_t)L);
  float2 *H = (float2 *)p;
  p += align256(1025 * sizeof(float2) * (size_t)L);
  float2 *HG = (float2 *)p;
  p += align256(1025 * sizeof(float2) * (size_t)L);
  int *eval_star = (int *)p;
  p += align256(sizeof(int) * (size_t)L);
  float *A = (float *)p;
  p += align256((size_t)stride * sizeof(float) * (size_t)L);
  float *B = (float *)p;
  p += align256((size_t)stride * sizeof(float) * (size_t)L);
  int *bnd = (int *)p;
  p += align256((size_t)bstr * sizeof(int) * (size_t)L);
  double *cpart = (double *)p;
  p += align256((size_t)MAX_CHUNKS * sizeof(double) * (size_t)L);
  // SEG group slots per segment of SEG labels: L rounded up to SEG
  const int64_t Lseg = (L + SEG - 1) / SEG * SEG;
  GroupRec *grec = (GroupRec *)p;
  p += align256(sizeof(GroupRec) * (size_t)Lseg);
  int *gcount = (int *)p;
  cudaStream_t s = (cudaStream_t)stream;
  k_noalloc_init<<<(unsigned)((L + 255) / 256), 256, 0, s>>>(star, dstar, eval_star, (int)L);
  EvalBatch b{};
  b.E = (int)L;
  b.labels = labels;
  b.eval_star = eval_star;
  b.stars = dstar;
  b.prep = prep;
  b.H = H;
  b.HG = HG;
  b.bufA = A;
  b.bufB = B;
  b.stride = stride;
  b.cost = out;
  b.status = status;
  // labels live on the device, so the blocks are sized for the widest
  // rotation kernel the reference accepts (2048 taps); work items beyond an
  // evaluation's own blocks return at once
  const int hg = star.disp_kind == DISP_NONE ? 0 : (star.gw - 1) / 2;
  PipelineOpts o;
  pipeline_pairs(G.npx, FFTN, hg, &b.max_pairs, &b.max_pairs_unfused, &o.may_unfuse);
  b.need_chi2 = 1;
  b.chunk_p1_mask = star.cont_kind == CONT_CHUNK ? 1u << star.p1 : 0u;
  b.max_chunks = star.cont_kind == CONT_CHUNK ? star.n_chunks : 0;
  b.other_cont = star.cont_kind == CONT_CHUNK ? 0 : 1;
  b.obs_epi = 1;
  b.bnd = bnd;
  b.bnd_stride = bstr;
  b.cpart = cpart;
  b.grec = grec;
  b.gcount = gcount;
  launch_pipeline(G, b, S->twiddle, o, s);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_noalloc_err = std::string("kernel launch failed: ") + cudaGetErrorString(e);
    return PASTA_E_CUDA;
  }
  return PASTA_OK;
}
