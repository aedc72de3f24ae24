// Internal declarations shared by the libcctconv translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "cct_conv.h"

namespace cct {

// Geometry of one ConvolveOp, resolved from a cct_conv_desc.  Coordinates are
// "post-sampling" (the up-sampled input grid when sampling is UP): output
// (i, j) reads input rows i*down - low_r + r and cols j*down - low_c + s.
struct ConvGeom {
  int H, W;          // input plane (pre-sampling)
  int OH, OW;        // output plane
  int R, S;          // filter plane (FilterAdjoint + UpsampleInput: the upsampled size)
  int low_r, low_c;  // low halo (ConvolveHyperKernel.scala:824-830)
  int border;        // CCT_BORDER_*
  int orient;        // CCT_CROSS_CORRELATION / CCT_CONVOLUTION
  int down, up;      // sampling steps (1 when unused)
  int mode;          // CCT_* vector mode
  int pin, pf;       // input / filter planes (>= 1)
  int pout;          // output planes
  int batch;         // logical images
  int n;             // planes per image (frame modes)
  int groups;        // filters per image: pf / n (frame modes)
  int terms;         // planes summed per output plane (n for *_REDUCE, else 1)
  uint32_t flags;
  int fr, fs;        // filter plane as stored (R = fr * fup, S = fs * fup)
  int fup;           // FilterAdjoint + UpsampleInput: the gradient's upsampling step, else 1
};

// Plane mixing of ConvolveHyperKernel (ConvolveHyperKernel.scala:124-199,
// 319-340): input and filter plane of term t of output plane o.
__host__ __device__ inline void plane_pair(const ConvGeom &g, int o, int t,
                                           int *ip, int *fp) {
  switch (g.mode) {
    case CCT_PLANE_BY_PLANE:
      *ip = g.pin == 1 ? 0 : o;
      *fp = g.pf == 1 ? 0 : o;
      break;
    case CCT_PROJECT_FRAME: {
      int b = o / g.pf, p = o - b * g.pf;
      *ip = b * g.n + p % g.n;
      *fp = p;
      break;
    }
    case CCT_PROJECT_FRAME_BLOCK_REDUCE_SUM: {
      int b = o / g.groups, k = o - b * g.groups;
      *ip = b * g.n + t;
      *fp = k * g.n + t;
      break;
    }
    case CCT_BACK_PROJECT_FRAME: {
      int b = o / g.pf, w = o - b * g.pf;
      *ip = b * g.n + w % g.n;
      *fp = g.groups * (w % g.n) + w / g.n;
      break;
    }
    case CCT_BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM: {
      int b = o / g.groups, l = o - b * g.groups;
      *ip = b * g.n + t;
      *fp = t * g.groups + l;
      break;
    }
    case CCT_FILTER_ADJOINT: {  // out B*w + b, w = l*C + c (ConvolveHyperKernel.scala:187, 333, 575-590)
      int b = o % g.batch, w = o / g.batch;
      *ip = b * g.n + w % g.n;
      *fp = b * g.groups + w / g.n;
      break;
    }
    default: {  // CCT_FILTER_ADJOINT_BLOCK_REDUCE_SUM: out w, term t = image t of the batch
      *ip = t * g.n + o % g.n;
      *fp = t * g.groups + o / g.n;
      break;
    }
  }
}

// Validate a descriptor and resolve its geometry (the rules of
// cct_conv_output_shape).  Returns CCT_OK or CCT_EINVAL.
int resolve_geom(const cct_conv_desc *desc, ConvGeom *g);

// Error reporting (thread-local message, returned status).
int set_error(int status, const char *fmt, ...);
int check_cuda(cudaError_t e, const char *what);
void count_launches(uint64_t n);
void set_launch_capture(bool on);

// Kernel families (each returns CCT_OK or an error status).
int launch_direct(const ConvGeom &g, const float *x, const float *f, float *y,
                  cudaStream_t stream);
bool direct_tma_supported(const ConvGeom &g, const float *x);
int launch_direct_tma(const ConvGeom &g, const float *x, const float *f, float *y,
                      cudaStream_t stream, unsigned *err);
// Per-device error word passed to kernels with bounded waits: a statically
// allocated device word whose address is looked up on first use on the
// current device (nothing is allocated).  nullptr if the lookup fails.
unsigned *device_error_word();
// FilterAdjoint with small results (fa_f32.cu): BorderValid, no sampling,
// result width <= 8.  The block-reduced form needs fa_workspace_bytes() of
// plan workspace.
bool fa_f32_supported(const ConvGeom &g);
size_t fa_workspace_bytes(const ConvGeom &g);
int launch_fa_f32(const ConvGeom &g, const float *x, const float *f, float *y, float *work, cudaStream_t st);
// FilterAdjointBlockReduceSum on the tensor cores (fa_tc.cu), split BF16:
// the shapes fa_f32 takes; workspace for the per-split partial sums.
bool fa_tc_supported(const ConvGeom &g);
size_t fa_tc_workspace_bytes(const ConvGeom &g, int sms);
int launch_fa_tc(const ConvGeom &g, const float *x, const float *f, float *y, float *work, unsigned *err,
                 cudaStream_t st);
bool frame_f32_supported(const ConvGeom &g);
int launch_frame_f32(const ConvGeom &g, const float *x, const float *f,
                     float *y, cudaStream_t stream);
// Launch with programmatic stream serialisation: the kernel may be scheduled
// while the previous kernel in the stream runs, and must call
// grid_dependency_wait() (sm100_util.cuh) before it touches global memory
// that earlier work reads or writes.
template <typename... Params, typename... Args>
int launch_pdl(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
               const char *what, Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return check_cuda(cudaLaunchKernelEx(&cfg, kernel, static_cast<Args &&>(args)...), what);
}

// Checkpoint records (record.cu): one layer = a descriptor and, for a
// constant filter, its values.
struct RecordLayer {
  cct_conv_desc desc;
  std::vector<float> filter;
};
int record_encode(int kind, int64_t time, const std::vector<RecordLayer> &layers, std::vector<uint32_t> *out);
int record_decode(const uint32_t *words, size_t n, int *kind, int64_t *time, std::vector<RecordLayer> *layers);
int record_store(const std::vector<uint32_t> &words, uint32_t *out, size_t capacity, size_t *n_words);
int record_plan_layer(const cct_conv_plan *p, RecordLayer *out);
// Plan internals the records need (cct_conv.cu): the descriptor, the device
// copy of the constant filter (null if none) with its element count, and the
// plan's device; the filter element count a plan takes.
int plan_record_parts(const cct_conv_plan *p, cct_conv_desc *desc, const float **dev_filter, size_t *elems,
                      int *device);
int plan_filter_elems(const cct_conv_plan *p, size_t *elems);
int launch_scalar_matrix(int rows, int cols, const float *x, const float *mats, int L, int size, int border,
                         float *y, cudaStream_t stream);
int launch_separable(int rows, int cols, int planes, const float *x,
                     const float *rf, int rlen, const float *cf, int clen,
                     int border, int orient, float *tmp, float *y,
                     cudaStream_t stream);

}  // namespace cct
