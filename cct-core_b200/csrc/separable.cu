// Separable convolution: a rows pass then a columns pass
// (ConvolveRows2DHyperKernel.scala:66-160, ConvolveColumns2DHyperKernel.scala).
// Each output is a fused multiply-add chain from 0 over the 1-D filter taps,
// the order of the reference's `sum += localImage[..] * filter` loop.
// One thread per output; neighbouring threads share input lines through L1.
#include "cct_internal.h"
#include "tile_common.cuh"

namespace cct {
namespace {

constexpr int kThreads = 256;

// dir 0: along columns of a row (rows pass); dir 1: along rows (columns pass).
template <int DIR>
__global__ void __launch_bounds__(kThreads)
    separable_pass(int rows, int cols, int planes, const float *__restrict__ x,
                   const float *__restrict__ filt, int len, int border, int orient,
                   float *__restrict__ y) {
  __shared__ float wf[1024];
  for (int i = threadIdx.x; i < len; i += blockDim.x)
    wf[i] = filt[orient == CCT_CONVOLUTION ? len - 1 - i : i];
  __syncthreads();
  const long long total = (long long)rows * cols * planes;
  const int halo = (len - 1) / 2;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(idx % cols);
    const long long rp = idx / cols;
    const int r = (int)(rp % rows);
    const float *xp = x + (rp / rows) * (long long)rows * cols;
    float sum = 0.0f;
    if (DIR == 0) {
      const float *line = xp + (size_t)r * cols;
      for (int k = 0; k < len; ++k) {
        const int j = border_index(border, c - halo + k, cols);
        sum = __fmaf_rn(j < 0 ? 0.0f : __ldg(line + j), wf[k], sum);
      }
    } else {
      for (int k = 0; k < len; ++k) {
        const int i = border_index(border, r - halo + k, rows);
        sum = __fmaf_rn(i < 0 ? 0.0f : __ldg(xp + (size_t)i * cols + c), wf[k], sum);
      }
    }
    y[idx] = sum;
  }
}

}  // namespace

int launch_separable(int rows, int cols, int planes, const float *x, const float *rf,
                     int rlen, const float *cf, int clen, int border, int orient,
                     float *tmp, float *y, cudaStream_t st) {
  if (rows < 1 || cols < 1 || planes < 1)
    return set_error(CCT_EINVAL, "separable: field sizes must be positive");
  if (border != CCT_BORDER_ZERO && border != CCT_BORDER_CLAMP && border != CCT_BORDER_CYCLIC)
    return set_error(CCT_EINVAL, "separable: unsupported border policy %d", border);
  if (rlen < 1 || clen < 1 || rlen % 2 == 0 || clen % 2 == 0)
    return set_error(CCT_EINVAL, "separable: row and column filters must be of odd size");
  if (rlen > 1024 || clen > 1024)
    return set_error(CCT_ENOTSUP, "separable: filters longer than 1024 taps");
  if (orient != CCT_CONVOLUTION && orient != CCT_CROSS_CORRELATION)
    return set_error(CCT_EINVAL, "separable: bad orientation");
  const long long total = (long long)rows * cols * planes;
  const long long want = (total + kThreads - 1) / kThreads;
  const int blocks = (int)(want < 148LL * 64 ? want : 148LL * 64);
  separable_pass<0><<<blocks, kThreads, 0, st>>>(rows, cols, planes, x, rf, rlen, border, orient, tmp);
  separable_pass<1><<<blocks, kThreads, 0, st>>>(rows, cols, planes, tmp, cf, clen, border, orient, y);
  count_launches(2);
  return check_cuda(cudaGetLastError(), "separable launch");
}

}  // namespace cct
