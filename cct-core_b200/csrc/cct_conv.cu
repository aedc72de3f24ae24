// C-ABI of libcctconv: descriptor validation, plans, dispatch, memory helpers.
//
// The descriptor rules restate ConvolveHyperKernel.outputFieldType
// (hyperkernels/ConvolveHyperKernel.scala:1297-1450) and the legality checks of
// DynamicConvolutionGenerator.convolveDirectly
// (generator/DynamicConvolutionGenerator.scala:484-539).
#include <atomic>
#include <map>
#include <mutex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "cct_internal.h"
#include "bank_tc.h"
#include "fft_conv.h"
#include "frame_tc.h"

namespace cct {

static thread_local char g_err[512] = "no error";
static std::atomic<uint64_t> g_launches{0};

int set_error(int status, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return status;
}

int check_cuda(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return CCT_OK;
  const int status = e == cudaErrorMemoryAllocation ? CCT_ENOMEM : CCT_ECUDA;
  return set_error(status, "%s: %s", what, cudaGetErrorString(e));
}

// Launches issued while this thread captures a CUDA graph are not counted
// (nothing runs); each replay of the graph counts its kernel nodes instead.
static thread_local bool t_capturing = false;
void count_launches(uint64_t n) {
  if (!t_capturing) g_launches.fetch_add(n, std::memory_order_relaxed);
}
void set_launch_capture(bool on) { t_capturing = on; }

// The device error word: one statically allocated word per device (module
// data, zero at load), so neither a plan nor the allocation-free entry point
// allocates it.  Its name is a host-side stand-in: the device address is
// looked up once per device, with that device current, and cached for the
// life of the CUDA context (cudaDeviceReset invalidates it).
static __device__ unsigned g_dev_err_word;
static std::mutex g_err_mu;
static unsigned *g_err_word[64];

unsigned *device_error_word() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(g_err_mu);
  if (!g_err_word[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_dev_err_word) != cudaSuccess) return nullptr;
    g_err_word[dev] = static_cast<unsigned *>(p);
  }
  return g_err_word[dev];
}

// Resolve and validate a descriptor.  Returns CCT_OK or CCT_EINVAL with the
// reference's error text.
static int resolve(const cct_conv_desc *d, ConvGeom *g) {
  if (!d) return set_error(CCT_EINVAL, "null descriptor");
  if (d->struct_size != (int32_t)sizeof(cct_conv_desc))
    return set_error(CCT_EINVAL, "descriptor struct_size %d != %d", d->struct_size,
                     (int)sizeof(cct_conv_desc));
  if (d->image_rows < 1 || d->image_cols < 1 || d->filter_rows < 1 || d->filter_cols < 1)
    return set_error(CCT_EINVAL, "field and filter sizes must be positive");
  if (d->image_planes < 0 || d->filter_planes < 0)
    return set_error(CCT_EINVAL, "plane counts must be >= 0");
  if (d->border < CCT_BORDER_ZERO || d->border > CCT_BORDER_FULL)
    return set_error(CCT_EINVAL, "bad border policy %d", d->border);
  if (d->orientation != CCT_CROSS_CORRELATION && d->orientation != CCT_CONVOLUTION)
    return set_error(CCT_EINVAL, "bad filter orientation %d", d->orientation);
  if (d->vector_mode < CCT_PLANE_BY_PLANE || d->vector_mode > CCT_FILTER_ADJOINT_BLOCK_REDUCE_SUM)
    return set_error(CCT_EINVAL, "bad vector mode %d", d->vector_mode);
  if (d->precision != CCT_PREC_FP32 && d->precision != CCT_PREC_BF16X3 && d->precision != CCT_PREC_BF16X6)
    return set_error(CCT_EINVAL, "bad precision %d", d->precision);
  if (d->algo < CCT_ALGO_AUTO || d->algo > CCT_ALGO_FFT)
    return set_error(CCT_EINVAL, "bad algorithm %d", d->algo);
  if (d->flags & ~CCT_FLAG_RELU) return set_error(CCT_EINVAL, "unknown flags 0x%x", d->flags);

  int sampling = d->sampling;
  if (sampling < CCT_SAMPLE_NONE || sampling > CCT_SAMPLE_UP)
    return set_error(CCT_EINVAL, "bad sampling policy %d", sampling);
  if (sampling != CCT_SAMPLE_NONE && d->step < 1)
    return set_error(CCT_EINVAL, "sampling step must be >= 1");
  // CogFunctionAPI.scala:1139-1143: Upsample(1) / Downsample(1) are NoSampling.
  if (sampling != CCT_SAMPLE_NONE && d->step == 1) sampling = CCT_SAMPLE_NONE;
  const int step = sampling == CCT_SAMPLE_NONE ? 1 : d->step;

  const int R = d->filter_rows, S = d->filter_cols;
  if (d->border != CCT_BORDER_VALID && d->border != CCT_BORDER_FULL && (R % 2 == 0 || S % 2 == 0))
    return set_error(CCT_EINVAL, "filter must be of odd shape for border policy %d", d->border);
  if (sampling == CCT_SAMPLE_DOWN) {
    int cr = 0, cc = 0;
    if (d->border == CCT_BORDER_VALID) { cr = R - 1; cc = S - 1; }
    if (d->border == CCT_BORDER_FULL) { cr = 1 - R; cc = 1 - S; }
    if ((d->image_rows - cr) % step != 0 || (d->image_cols - cc) % step != 0)
      return set_error(CCT_EINVAL,
                       "The size of the input for convolution must be divisible by the "
                       "downsampling step size after border contraction.");
  }
  if (sampling == CCT_SAMPLE_UP && d->border == CCT_BORDER_CLAMP)
    return set_error(CCT_EINVAL, "Integrated upsampling with BorderClamp convolution not supported");

  // FilterAdjoint upsamples its second operand (the gradient), not the
  // image (ConvolveHyperKernel.scala:1306-1326).
  const bool fa = d->vector_mode == CCT_FILTER_ADJOINT || d->vector_mode == CCT_FILTER_ADJOINT_BLOCK_REDUCE_SUM;
  const int fup = (fa && sampling == CCT_SAMPLE_UP) ? step : 1;
  const int Re = R * fup, Se = S * fup;
  long long ur = d->image_rows, uc = d->image_cols;
  if (sampling == CCT_SAMPLE_UP && !fa) { ur *= step; uc *= step; }
  long long orow = ur, ocol = uc;
  if (d->border == CCT_BORDER_VALID) { orow = ur - Re + 1; ocol = uc - Se + 1; }
  if (d->border == CCT_BORDER_FULL) { orow = ur + Re - 1; ocol = uc + Se - 1; }
  if (orow < 1 || ocol < 1) return set_error(CCT_EINVAL, "BorderValid filter larger than the input");
  if (sampling == CCT_SAMPLE_DOWN) { orow = (orow + step - 1) / step; ocol = (ocol + step - 1) / step; }
  if (orow > (1 << 30) || ocol > (1 << 30)) return set_error(CCT_EINVAL, "output too large");

  const int pin = d->image_planes < 1 ? 1 : d->image_planes;
  const int pf = d->filter_planes < 1 ? 1 : d->filter_planes;
  const int batch = d->batch_size < 1 ? 1 : d->batch_size;
  int pout, n = 1, groups = 1, terms = 1;
  if (d->vector_mode == CCT_PLANE_BY_PLANE) {
    if (!(d->image_planes == 0 || d->filter_planes == 0 || d->image_planes == d->filter_planes))
      return set_error(CCT_EINVAL,
                       "plane-by-plane convolution needs a ScalarField operand or equal tensor shapes");
    pout = d->image_planes == 0 ? pf : pin;
  } else if (fa) {
    // ConvolveHyperKernel.scala:1366-1377 (checks) and 1414-1429 (output planes)
    if (pf % batch != 0)
      return set_error(CCT_EINVAL, "Filter tensorshape points %d must be a multiple of the batchSize %d", pf,
                       batch);
    if (pin % batch != 0)
      return set_error(CCT_EINVAL, "Input tensorshape points %d must be a multiple of the batchSize %d",
                       pin, batch);
    n = pin / batch;
    groups = pf / batch;
    if (d->vector_mode == CCT_FILTER_ADJOINT) {
      pout = n * groups * batch;
    } else {
      pout = n * groups;
      terms = batch;
    }
  } else {
    if (pin % batch != 0)
      return set_error(CCT_EINVAL, "Input tensorshape points %d must be a multiple of the batchSize %d",
                       pin, batch);
    n = pin / batch;
    if (pf % n != 0)
      return set_error(CCT_EINVAL, "filter tensor length %d not a multiple of per-image tensor length %d",
                       pf, n);
    groups = pf / n;
    if (d->vector_mode == CCT_PROJECT_FRAME || d->vector_mode == CCT_BACK_PROJECT_FRAME) {
      pout = pf * batch;
    } else {
      pout = batch * groups;
      terms = n;
    }
  }

  g->H = d->image_rows;
  g->W = d->image_cols;
  g->OH = (int)orow;
  g->OW = (int)ocol;
  g->R = Re;
  g->S = Se;
  g->fr = R;
  g->fs = S;
  g->fup = fup;
  g->low_r = d->border == CCT_BORDER_FULL ? Re - 1 : (d->border == CCT_BORDER_VALID ? 0 : (Re - 1) / 2);
  g->low_c = d->border == CCT_BORDER_FULL ? Se - 1 : (d->border == CCT_BORDER_VALID ? 0 : (Se - 1) / 2);
  g->border = d->border;
  g->orient = d->orientation;
  g->down = sampling == CCT_SAMPLE_DOWN ? step : 1;
  g->up = (sampling == CCT_SAMPLE_UP && !fa) ? step : 1;
  g->mode = d->vector_mode;
  g->pin = pin;
  g->pf = pf;
  g->pout = pout;
  g->batch = batch;
  g->n = n;
  g->groups = groups;
  g->terms = terms;
  g->flags = d->flags;
  return CCT_OK;
}

int resolve_geom(const cct_conv_desc *desc, ConvGeom *g) { return resolve(desc, g); }

}  // namespace cct

using namespace cct;

enum { ALGO_DIRECT = 0, ALGO_FRAME_F32 = 1, ALGO_FRAME_BF16X3 = 2, ALGO_FFT = 3, ALGO_FILTER_ADJOINT = 4,
       ALGO_FILTER_ADJOINT_BF16X3 = 5 };

struct cct_conv_plan {
  cct_conv_desc desc;
  ConvGeom g;
  int algo;
  int device;
  unsigned *err;  // device error word of `device`
  size_t x_elems, f_elems, y_elems;
  float *static_filter;  // device copy of a static filter, or null
  FrameTcChoice tc;      // tensor-core frame kernel and tile plan (ALGO_FRAME_BF16X3)
  uint8_t *packed;       // packed bf16 hi/lo filter operand (plan workspace)
  bool packed_static;    // packed holds the static filter
  FftParams fft;         // FFT plan (ALGO_FFT)
  float2 *fft_spec;      // working spectrum (plan workspace)
  float2 *fft_filter;    // filter spectrum
  float2 *fft_tw;        // twiddle tables
  bool fft_static;       // fft_filter holds the static filter's FP64 spectrum
  float *fa_work;        // per-image FilterAdjoint results before the block reduce
  // run_host staging (allocated on the first cct_conv_run_host call)
  float *d_x, *d_f, *d_y;
};

namespace cct {

int plan_record_parts(const cct_conv_plan *p, cct_conv_desc *desc, const float **dev_filter, size_t *elems,
                      int *device) {
  if (!p) return set_error(CCT_EINVAL, "null plan");
  *desc = p->desc;
  *dev_filter = p->static_filter;
  *elems = p->f_elems;
  *device = p->device;
  return CCT_OK;
}

int plan_filter_elems(const cct_conv_plan *p, size_t *elems) {
  if (!p) return set_error(CCT_EINVAL, "null plan");
  *elems = p->f_elems;
  return CCT_OK;
}

}  // namespace cct

extern "C" {

void cct_conv_desc_init(cct_conv_desc *d) {
  if (!d) return;
  memset(d, 0, sizeof(*d));
  d->struct_size = (int32_t)sizeof(cct_conv_desc);
  d->image_rows = d->image_cols = 1;
  d->filter_rows = d->filter_cols = 1;
  d->batch_size = 1;
  d->border = CCT_BORDER_ZERO;
  d->orientation = CCT_CONVOLUTION;
  d->sampling = CCT_SAMPLE_NONE;
  d->step = 1;
  d->vector_mode = CCT_PLANE_BY_PLANE;
  d->precision = CCT_PREC_FP32;
  d->algo = CCT_ALGO_AUTO;
}

int cct_conv_output_shape(const cct_conv_desc *d, int32_t *rows, int32_t *cols, int32_t *planes) {
  ConvGeom g;
  int rc = resolve(d, &g);
  if (rc) return rc;
  if (rows) *rows = g.OH;
  if (cols) *cols = g.OW;
  if (planes) *planes = g.pout;
  return CCT_OK;
}

static int current_sm100(int *dev) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    cudaGetLastError();
    return set_error(CCT_ENODEV, "no CUDA device visible");
  }
  int rc = check_cuda(cudaGetDevice(dev), "cudaGetDevice");
  if (rc) return rc;
  int major = 0;
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, *dev);
  if (major != 10) return set_error(CCT_ENODEV, "device %d is not sm_100 (major %d)", *dev, major);
  return CCT_OK;
}

// Direct vs FFT for UseFFTWhenBest.  The reference decides from a timing
// table measured offline per field and filter size
// (generator/FFTConvolutionUtils.scala:100-142, 145-236); here the two
// kernels are timed on the device itself, once per (device, field size,
// filter size, border), on one plane, and the decision is cached for the
// process.  Both paths cost the same per plane, so one plane decides for
// any plane count.  The FFT is timed with a static filter (its spectrum made
// once, as for the reference's constant filters).  The direct kernels keep
// the reference's FP32 arithmetic bit for bit, so the FFT is taken only when
// it is clearly faster: at least 1.2x when measured, never for launch-bound
// planes (direct under 5 us by the model), and without measuring where the
// modelled times differ tenfold.
static int time_plan_us(cct_conv_plan *p, const float *x, const float *f, float *y, cudaStream_t st, float *us);
static bool fft_measured_faster(const cct_conv_desc *d, const ConvGeom &g, const FftParams &fp, int dev) {
  const double direct_s = 2.0 * g.OH * g.OW * g.R * g.S / 30e12 + 3e-6;
  const double fft_s = 24.0 * fp.Fr * fp.Fc / 2e12 + 12e-6;
  if (direct_s < 5e-6) return false;
  if (direct_s > 10.0 * fft_s) return true;
  if (fft_s > 10.0 * direct_s) return false;
  static std::mutex mu;
  static std::map<std::vector<int>, bool> cache;
  const std::vector<int> key = {dev, g.H, g.W, g.R, g.S, g.border};
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  bool fft_faster = fft_s < direct_s;  // the model, should a measurement fail
  cct_conv_desc one = *d;
  one.image_planes = 0;
  one.filter_planes = 0;
  one.batch_size = 1;
  one.vector_mode = CCT_PLANE_BY_PLANE;
  one.precision = CCT_PREC_FP32;
  one.flags = 0;
  cct_conv_plan *pd = nullptr, *pf = nullptr;
  float *x = nullptr, *f = nullptr, *y = nullptr;
  cudaStream_t st = nullptr;
  float td = 0.0f, tf = 0.0f;
  one.algo = CCT_ALGO_DIRECT;
  int rc = cct_conv_plan_create(&one, &pd);
  one.algo = CCT_ALGO_FFT;
  if (!rc) rc = cct_conv_plan_create(&one, &pf);
  if (!rc) rc = check_cuda(cudaMalloc(&x, sizeof(float) * (size_t)g.H * g.W), "triage buffers");
  if (!rc) rc = check_cuda(cudaMalloc(&y, sizeof(float) * (size_t)g.OH * g.OW), "triage buffers");
  if (!rc) rc = check_cuda(cudaMalloc(&f, sizeof(float) * (size_t)g.R * g.S), "triage buffers");
  if (!rc) rc = check_cuda(cudaMemset(x, 0, sizeof(float) * (size_t)g.H * g.W), "triage buffers");
  if (!rc) rc = check_cuda(cudaMemset(f, 0, sizeof(float) * (size_t)g.R * g.S), "triage buffers");
  if (!rc) {
    std::vector<float> hf((size_t)g.R * g.S, 0.0f);
    rc = cct_conv_plan_set_static_filter(pf, hf.data());
  }
  if (!rc) rc = check_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "triage stream");
  if (!rc) rc = time_plan_us(pd, x, f, y, st, &td);
  if (!rc) rc = time_plan_us(pf, x, nullptr, y, st, &tf);
  if (!rc) fft_faster = 1.2f * tf < td;
  if (st) cudaStreamDestroy(st);
  cudaFree(x);
  cudaFree(y);
  cudaFree(f);
  cct_conv_plan_destroy(pd);
  cct_conv_plan_destroy(pf);
  if (!rc) {
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = fft_faster;
  }
  return fft_faster;
}

static int time_plan_us(cct_conv_plan *p, const float *x, const float *f, float *y, cudaStream_t st, float *us) {
  for (int i = 0; i < 2; ++i) {
    const int rc = cct_conv_run(p, x, f, y, st);
    if (rc) return rc;
  }
  cudaEvent_t a = nullptr, b = nullptr;
  int rc = check_cuda(cudaEventCreate(&a), "triage event");
  if (!rc) rc = check_cuda(cudaEventCreate(&b), "triage event");
  if (!rc) rc = check_cuda(cudaEventRecord(a, st), "triage event");
  for (int i = 0; i < 5 && !rc; ++i) rc = cct_conv_run(p, x, f, y, st);
  if (!rc) rc = check_cuda(cudaEventRecord(b, st), "triage event");
  if (!rc) rc = check_cuda(cudaEventSynchronize(b), "triage event");
  float ms = 0.0f;
  if (!rc) rc = check_cuda(cudaEventElapsedTime(&ms, a, b), "triage event");
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  *us = ms * 200.0f;  // per run, microseconds
  return rc;
}

int cct_conv_plan_create(const cct_conv_desc *d, cct_conv_plan **out) {
  if (!out) return set_error(CCT_EINVAL, "null plan output");
  *out = nullptr;
  ConvGeom g;
  int rc = resolve(d, &g);
  if (rc) return rc;
  int dev = 0;
  rc = current_sm100(&dev);
  if (rc) return rc;

  int algo;
  const bool reduce = g.mode == CCT_PROJECT_FRAME_BLOCK_REDUCE_SUM ||
                      g.mode == CCT_BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM;
  // Direct vs FFT (DynamicConvolutionGenerator.scala:109-150): the FFT takes
  // plane-by-plane convolutions without sampling under Zero/Clamp/Cyclic;
  // UseFFTAlways falls back to the direct kernels outside that, as the
  // reference does; WhenBest takes the path measured faster on this device.
  FftParams fp{};
  bool use_fft = false;
  if (d->algo != CCT_ALGO_DIRECT && fft_plan(g, &fp))
    use_fft = d->algo == CCT_ALGO_FFT || fft_measured_faster(d, g, fp, dev);
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const bool fa_reduce = g.mode == CCT_FILTER_ADJOINT_BLOCK_REDUCE_SUM;
  if (d->precision == CCT_PREC_BF16X3 && !reduce && !fa_reduce)
    return set_error(CCT_EINVAL, "BF16X3 precision applies to the BlockReduceSum modes only");
  if (d->precision == CCT_PREC_BF16X6 && !reduce)
    return set_error(CCT_EINVAL, "BF16X6 precision applies to the frame BlockReduceSum modes only");
  FrameTcChoice tc{};
  if (use_fft)
    algo = ALGO_FFT;
  else if (d->precision == CCT_PREC_BF16X3 && fa_reduce && fa_tc_supported(g))
    algo = ALGO_FILTER_ADJOINT_BF16X3;
  else if (fa_f32_supported(g))
    algo = ALGO_FILTER_ADJOINT;
  else if (d->precision != CCT_PREC_FP32 && frame_tc_choose(g, d->precision, sms, &tc))
    algo = ALGO_FRAME_BF16X3;
  else
    // the FP32 frame kernel: fused and unfused frame modes (with the reduce
    // or each input plane's result to its own output plane)
    algo = frame_f32_supported(g) ? ALGO_FRAME_F32 : ALGO_DIRECT;

  unsigned *err_word = device_error_word();
  if (!err_word) return set_error(CCT_ECUDA, "device error word: symbol address lookup failed");

  cct_conv_plan *p = new (std::nothrow) cct_conv_plan();
  if (!p) return set_error(CCT_ENOMEM, "plan allocation failed");
  p->desc = *d;
  p->g = g;
  p->algo = algo;
  p->device = dev;
  p->err = err_word;
  p->x_elems = (size_t)g.pin * g.H * g.W;
  p->f_elems = (size_t)g.pf * g.fr * g.fs;
  p->y_elems = (size_t)g.pout * g.OH * g.OW;
  p->tc = tc;
  if (algo == ALGO_FRAME_BF16X3) {
    rc = check_cuda(cudaMalloc(&p->packed, tc.pack_bytes), "cudaMalloc(packed filters)");
    if (rc) {
      delete p;
      return rc;
    }
  }
  if (algo == ALGO_FILTER_ADJOINT_BF16X3) {
    rc = check_cuda(cudaMalloc(&p->fa_work, fa_tc_workspace_bytes(g, sms)),
                    "cudaMalloc(FilterAdjoint partial sums)");
    if (rc) {
      cct_conv_plan_destroy(p);
      return rc;
    }
  }
  if (algo == ALGO_FILTER_ADJOINT && fa_workspace_bytes(g)) {
    rc = check_cuda(cudaMalloc(&p->fa_work, fa_workspace_bytes(g)), "cudaMalloc(FilterAdjoint workspace)");
    if (rc) {
      cct_conv_plan_destroy(p);
      return rc;
    }
  }
  if (algo == ALGO_FFT) {
    p->fft = fp;
    rc = check_cuda(cudaMalloc(&p->fft_spec, fp.spec_elems * sizeof(float2)), "cudaMalloc(fft spectrum)");
    if (!rc)
      rc = check_cuda(cudaMalloc(&p->fft_filter, fp.filter_elems * sizeof(float2)),
                      "cudaMalloc(fft filter spectrum)");
    if (!rc) rc = check_cuda(cudaMalloc(&p->fft_tw, fp.tw_elems * sizeof(float2)), "cudaMalloc(fft twiddles)");
    if (!rc) {
      std::vector<float> tw;
      fft_twiddles(fp, &tw);
      rc = check_cuda(cudaMemcpy(p->fft_tw, tw.data(), tw.size() * sizeof(float), cudaMemcpyHostToDevice),
                      "cudaMemcpy(fft twiddles)");
    }
    if (rc) {
      cct_conv_plan_destroy(p);
      return rc;
    }
    fft_set_tables(&p->fft, p->fft_tw);
  }
  *out = p;
  return CCT_OK;
}

int cct_conv_plan_destroy(cct_conv_plan *p) {
  if (!p) return CCT_OK;
  cudaFree(p->static_filter);
  cudaFree(p->packed);
  cudaFree(p->fft_spec);
  cudaFree(p->fft_filter);
  cudaFree(p->fft_tw);
  cudaFree(p->fa_work);
  cudaFree(p->d_x);
  cudaFree(p->d_f);
  cudaFree(p->d_y);
  delete p;
  return CCT_OK;
}

int cct_conv_plan_algo(const cct_conv_plan *p, int32_t *algo) {
  if (!p || !algo) return set_error(CCT_EINVAL, "null argument");
  *algo = p->algo;
  return CCT_OK;
}

int cct_conv_plan_set_static_filter(cct_conv_plan *p, const float *host_filter) {
  if (!p || !host_filter) return set_error(CCT_EINVAL, "null argument");
  const size_t bytes = p->f_elems * sizeof(float);
  if (!p->static_filter) {
    int rc = check_cuda(cudaMalloc(&p->static_filter, bytes), "cudaMalloc(static filter)");
    if (rc) return rc;
  }
  int rc = check_cuda(cudaMemcpy(p->static_filter, host_filter, bytes, cudaMemcpyHostToDevice),
                      "cudaMemcpy(static filter)");
  if (rc) return rc;
  if (p->algo == ALGO_FFT) {
    // the reference transforms constant filters on the host in FP64
    // (DynamicConvolutionGenerator.scala:342-350, 376-405)
    std::vector<float> spec;
    fft_static_spectrum(p->fft, host_filter, &spec);
    rc = check_cuda(cudaMemcpy(p->fft_filter, spec.data(), spec.size() * sizeof(float), cudaMemcpyHostToDevice),
                    "cudaMemcpy(static filter spectrum)");
    if (rc) return rc;
    p->fft_static = true;
  }
  if (p->algo == ALGO_FRAME_BF16X3) {
    rc = frame_tc_pack(p->tc, p->static_filter, p->packed, 0);
    if (!rc) rc = check_cuda(cudaStreamSynchronize(0), "pack static filter");
    if (rc) return rc;
    p->packed_static = true;
  }
  return CCT_OK;
}

int cct_conv_run(const cct_conv_plan *p, const float *x, const float *f, float *y, void *stream) {
  if (!p) return set_error(CCT_EINVAL, "null plan");
  if (!f) f = p->static_filter;
  if (!x || !f || !y) return set_error(CCT_EINVAL, "null image, filter or output pointer");
  cudaStream_t st = (cudaStream_t)stream;
  switch (p->algo) {
    case ALGO_FRAME_BF16X3: {
      int rc = CCT_OK;
      const bool pack = f != p->static_filter || !p->packed_static;
      if (pack) rc = frame_tc_pack(p->tc, f, p->packed, st);
      if (rc) return rc;
      return frame_tc_run(p->tc, x, y, p->packed, p->err, st, pack);
    }
    case ALGO_FRAME_F32:
      return launch_frame_f32(p->g, x, f, y, st);
    case ALGO_FILTER_ADJOINT:
      return launch_fa_f32(p->g, x, f, y, p->fa_work, st);
    case ALGO_FILTER_ADJOINT_BF16X3:
      return launch_fa_tc(p->g, x, f, y, p->fa_work, p->err, st);
    case ALGO_FFT: {
      int rc = CCT_OK;
      if (f != p->static_filter || !p->fft_static)
        rc = launch_fft_filter_spectrum(p->fft, f, p->fft_filter, st);
      if (rc) return rc;
      return launch_fft_conv(p->fft, x, p->fft_filter, p->fft_spec, y, st);
    }
    default:
      if (direct_tma_supported(p->g, x)) return launch_direct_tma(p->g, x, f, y, st, p->err);
      return launch_direct(p->g, x, f, y, st);
  }
}

int cct_conv_run_host(cct_conv_plan *p, const float *hx, const float *hf, float *hy, void *stream) {
  if (!p) return set_error(CCT_EINVAL, "null plan");
  if (!hx || !hy || (!hf && !p->static_filter))
    return set_error(CCT_EINVAL, "null host image, filter or output pointer");
  cudaStream_t st = (cudaStream_t)stream;
  int rc;
  if (!p->d_x) {
    rc = check_cuda(cudaMalloc(&p->d_x, p->x_elems * sizeof(float)), "cudaMalloc(staging)");
    if (!rc) rc = check_cuda(cudaMalloc(&p->d_f, p->f_elems * sizeof(float)), "cudaMalloc(staging)");
    if (!rc) rc = check_cuda(cudaMalloc(&p->d_y, p->y_elems * sizeof(float)), "cudaMalloc(staging)");
    if (rc) return rc;
  }
  rc = check_cuda(cudaMemcpyAsync(p->d_x, hx, p->x_elems * sizeof(float), cudaMemcpyHostToDevice, st),
                  "H2D image");
  if (rc) return rc;
  const float *df = p->static_filter;
  if (hf) {
    rc = check_cuda(cudaMemcpyAsync(p->d_f, hf, p->f_elems * sizeof(float), cudaMemcpyHostToDevice, st),
                    "H2D filter");
    if (rc) return rc;
    df = p->d_f;
  }
  rc = cct_conv_run(p, p->d_x, df, p->d_y, stream);
  if (rc) return rc;
  rc = check_cuda(cudaMemcpyAsync(hy, p->d_y, p->y_elems * sizeof(float), cudaMemcpyDeviceToHost, st),
                  "D2H output");
  if (rc) return rc;
  return check_cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize");
}

int cct_conv_separable(int32_t rows, int32_t cols, int32_t planes, const float *x, const float *rf,
                       int32_t rlen, const float *cf, int32_t clen, int32_t border, int32_t orient,
                       float *tmp, float *y, void *stream) {
  if (!x || !rf || !cf || !tmp || !y) return set_error(CCT_EINVAL, "null pointer argument");
  return launch_separable(rows, cols, planes < 1 ? 1 : planes, x, rf, rlen, cf, clen, border, orient,
                          tmp, y, (cudaStream_t)stream);
}

int cct_conv_scalar_matrix(int32_t rows, int32_t cols, const float *image, const float *matrices,
                           int32_t matrix_rows, int32_t matrix_cols, int32_t size, int32_t border,
                           int32_t orientation, int32_t sampling, int32_t step, float *out, void *stream) {
  // ScalarMatrixConvolve2DHyperKernel.apply (ScalarMatrixConvolve2DHyperKernel.scala:118-152)
  if (border == CCT_BORDER_FULL) return set_error(CCT_EINVAL, "unsupported: BorderFull");
  if (border == CCT_BORDER_VALID) return set_error(CCT_EINVAL, "unsupported: BorderValid");
  if (border != CCT_BORDER_ZERO && border != CCT_BORDER_CLAMP && border != CCT_BORDER_CYCLIC)
    return set_error(CCT_EINVAL, "bad border policy %d", border);
  // CogFunctionAPI.scala:1139-1143: step-1 sampling is NoSampling
  if (sampling != CCT_SAMPLE_NONE && !(step == 1 && (sampling == CCT_SAMPLE_DOWN || sampling == CCT_SAMPLE_UP)))
    return set_error(CCT_EINVAL, "sampling not supported yet");
  if (orientation != CCT_CROSS_CORRELATION) return set_error(CCT_EINVAL, "convolution not supported yet");
  if (rows < 1 || cols < 1 || matrix_rows < 1 || matrix_cols < 1 || size < 1)
    return set_error(CCT_EINVAL, "field, matrix field and matrix sizes must be positive");
  if (size % 2 != 1) return set_error(CCT_EINVAL, "matrix in field must have odd size");
  if (!image || !matrices || !out) return set_error(CCT_EINVAL, "null image, matrix or output pointer");
  const long long L = (long long)matrix_rows * matrix_cols;
  if (L > (1 << 24)) return set_error(CCT_ENOTSUP, "scalar-matrix convolution: too many matrices");
  return launch_scalar_matrix(rows, cols, image, matrices, (int)L, size, border, out, (cudaStream_t)stream);
}

int cct_malloc(void **ptr, size_t bytes) {
  if (!ptr) return set_error(CCT_EINVAL, "null pointer argument");
  return check_cuda(cudaMalloc(ptr, bytes), "cudaMalloc");
}
int cct_free(void *ptr) { return check_cuda(cudaFree(ptr), "cudaFree"); }
int cct_memcpy_h2d(void *dst, const void *src, size_t bytes, void *stream) {
  return check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream),
                    "cudaMemcpyAsync H2D");
}
int cct_memcpy_d2h(void *dst, const void *src, size_t bytes, void *stream) {
  return check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream),
                    "cudaMemcpyAsync D2H");
}
int cct_stream_create(void **stream) {
  if (!stream) return set_error(CCT_EINVAL, "null pointer argument");
  return check_cuda(cudaStreamCreateWithFlags((cudaStream_t *)stream, cudaStreamNonBlocking),
                    "cudaStreamCreate");
}
int cct_stream_destroy(void *stream) {
  return check_cuda(cudaStreamDestroy((cudaStream_t)stream), "cudaStreamDestroy");
}
int cct_stream_synchronize(void *stream) {
  return check_cuda(cudaStreamSynchronize((cudaStream_t)stream), "cudaStreamSynchronize");
}

int cct_device_status(void) {
  unsigned *w = device_error_word();
  if (!w) return set_error(CCT_ENODEV, "no device error word");
  unsigned v = 0;
  int rc = check_cuda(cudaMemcpy(&v, w, sizeof(v), cudaMemcpyDeviceToHost), "cudaMemcpy(status)");
  if (rc) return rc;
  if (v == 0) return CCT_OK;
  rc = check_cuda(cudaMemset(w, 0, sizeof(unsigned)), "cudaMemset(status)");
  if (rc) return rc;
  return set_error(CCT_ETIMEOUT, "a bounded wait inside a kernel gave up (status 0x%x)", v);
}

const char *cct_last_error_string(void) { return g_err; }
int cct_abi_version(void) { return CCT_ABI_VERSION; }
uint64_t cct_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

}  // extern "C"
