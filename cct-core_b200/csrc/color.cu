// Colour-field convolution (generator/DynamicConvolutionGenerator.scala:
// 89-106): a ColorField is an RGBA UNORM_INT8 image (OpenCLBuffer.scala:
// 135-136).  The reference splits it into red, green and blue scalar planes
// (ColorPlaneHyperKernel: byte / 255), convolves each with the scalar filter
// through the ordinary convolution triage, and merges the three results into
// a colour field (CreateColorFieldHyperKernel: (r, g, b, 1) written to the
// UNORM_INT8 image, i.e. saturate(v * 255) rounded half to even).
//
// Here a colour plan wraps one plane plan over the three planes (one
// launch, the filter shared) between an unpack and a pack kernel.
#include <cuda_runtime.h>

#include <new>

#include "cct_internal.h"

namespace cct {
namespace {

__global__ void color_unpack_kernel(long long n, const uchar4 *__restrict__ rgba, float *__restrict__ planes) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const uchar4 v = rgba[i];
    planes[i] = (float)v.x / 255.0f;
    planes[n + i] = (float)v.y / 255.0f;
    planes[2 * n + i] = (float)v.z / 255.0f;
  }
}

__device__ __forceinline__ unsigned char to_unorm8(float v) {
  const float s = v * 255.0f;
  // fmaxf/fminf return the number for a NaN operand, so NaN saturates to 0
  return (unsigned char)__float2uint_rn(fminf(fmaxf(s, 0.0f), 255.0f));
}

__global__ void color_pack_kernel(long long n, const float *__restrict__ planes, uchar4 *__restrict__ rgba) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    rgba[i] = make_uchar4(to_unorm8(planes[i]), to_unorm8(planes[n + i]), to_unorm8(planes[2 * n + i]), 255);
}

unsigned grid_for(long long n) {
  const long long b = (n + 255) / 256;
  return (unsigned)(b < 148LL * 16 ? (b < 1 ? 1 : b) : 148LL * 16);
}

}  // namespace
}  // namespace cct

using namespace cct;

struct cct_color_plan {
  cct_conv_plan *planes;  // the plane plan over red, green, blue
  float *in, *out;        // 3 planes each
  long long n_in, n_out;  // pixels per plane
};

extern "C" {

int cct_color_plan_create(const cct_conv_desc *desc, cct_color_plan **out) {
  if (!out) return set_error(CCT_EINVAL, "null plan output");
  *out = nullptr;
  if (!desc) return set_error(CCT_EINVAL, "null descriptor");
  if (desc->struct_size != (int32_t)sizeof(cct_conv_desc))
    return set_error(CCT_EINVAL, "descriptor struct_size %d != %d", desc->struct_size, (int)sizeof(cct_conv_desc));
  if (desc->image_planes > 1)
    return set_error(CCT_EINVAL, "colour convolution: the image is one colour field (image_planes 0 or 1)");
  if (desc->filter_planes > 1)
    return set_error(CCT_EINVAL, "colour convolution needs a scalar filter");
  if (desc->vector_mode != CCT_PLANE_BY_PLANE)
    return set_error(CCT_EINVAL, "colour convolution is plane by plane (projections need a real image input)");
  if (desc->precision != CCT_PREC_FP32) return set_error(CCT_EINVAL, "colour convolution runs in FP32");
  cct_conv_desc d = *desc;
  d.image_planes = 3;
  d.filter_planes = 0;
  int32_t orows = 0, ocols = 0;
  int rc = cct_conv_output_shape(&d, &orows, &ocols, nullptr);
  if (rc) return rc;
  cct_color_plan *p = new (std::nothrow) cct_color_plan();
  if (!p) return set_error(CCT_ENOMEM, "plan allocation failed");
  rc = cct_conv_plan_create(&d, &p->planes);
  p->n_in = (long long)d.image_rows * d.image_cols;
  p->n_out = (long long)orows * ocols;
  if (!rc) rc = check_cuda(cudaMalloc(&p->in, 3 * p->n_in * sizeof(float)), "cudaMalloc(colour planes)");
  if (!rc) rc = check_cuda(cudaMalloc(&p->out, 3 * p->n_out * sizeof(float)), "cudaMalloc(colour planes)");
  if (rc) {
    cct_color_plan_destroy(p);
    return rc;
  }
  *out = p;
  return CCT_OK;
}

int cct_color_plan_destroy(cct_color_plan *p) {
  if (!p) return CCT_OK;
  cct_conv_plan_destroy(p->planes);
  cudaFree(p->in);
  cudaFree(p->out);
  delete p;
  return CCT_OK;
}

int cct_color_plan_set_static_filter(cct_color_plan *p, const float *host_filter) {
  if (!p) return set_error(CCT_EINVAL, "null plan");
  return cct_conv_plan_set_static_filter(p->planes, host_filter);
}

int cct_color_run(const cct_color_plan *p, const uint8_t *image, const float *filter, uint8_t *out, void *stream) {
  if (!p) return set_error(CCT_EINVAL, "null plan");
  if (!image || !out) return set_error(CCT_EINVAL, "null image or output pointer");
  if ((reinterpret_cast<uintptr_t>(image) & 3) != 0 || (reinterpret_cast<uintptr_t>(out) & 3) != 0)
    return set_error(CCT_EINVAL, "colour fields must be 4-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  color_unpack_kernel<<<grid_for(p->n_in), 256, 0, st>>>(p->n_in, reinterpret_cast<const uchar4 *>(image), p->in);
  count_launches(1);
  int rc = check_cuda(cudaGetLastError(), "colour unpack launch");
  if (rc) return rc;
  rc = cct_conv_run(p->planes, p->in, filter, p->out, stream);
  if (rc) return rc;
  color_pack_kernel<<<grid_for(p->n_out), 256, 0, st>>>(p->n_out, p->out, reinterpret_cast<uchar4 *>(out));
  count_launches(1);
  return check_cuda(cudaGetLastError(), "colour pack launch");
}

}  // extern "C"
