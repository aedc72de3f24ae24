// Separable convolution: a rows pass then a columns pass
// (ConvolveRows2DHyperKernel.scala:66-160, ConvolveColumns2DHyperKernel.scala).
// Each output is a fused multiply-add chain from 0 over the 1-D filter taps,
// the order of the reference's `sum += localImage[..] * filter` loop.
// Short filters run both passes fused per output tile (separable_fused);
// long ones run one thread per output per pass, through a scratch field.
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

// Both passes fused per 32 x 64 output tile: the image rows the columns
// pass needs (border-mapped) are staged in shared memory with their
// border-mapped column halo, the rows pass fills an intermediate tile of
// those rows, and the columns pass reads it.  Each intermediate value is the
// same fma chain as in the two-pass form, so the result is bit-identical to
// it while the image is read and the result written once.
constexpr int kSTH = 32, kSTW = 64;

__global__ void __launch_bounds__(kThreads)
    separable_fused(int rows, int cols, int planes, const float *__restrict__ x,
                    const float *__restrict__ rf, int rlen, const float *__restrict__ cf, int clen,
                    int border, int orient, float *__restrict__ y, int tiles_x, int tiles_y) {
  extern __shared__ __align__(16) float sm[];
  const int hr = (rlen - 1) / 2, hc = (clen - 1) / 2;
  const int IR = kSTH + clen - 1, IC = kSTW + rlen - 1;  // staged image rows x columns
  float *wr = sm, *wc = sm + rlen;
  float *img = wc + clen;                // IR x IC
  float *mid = img + (size_t)IR * IC;    // IR x kSTW (rows pass)
  const bool conv = orient == CCT_CONVOLUTION;
  for (int i = threadIdx.x; i < rlen; i += blockDim.x) wr[i] = rf[conv ? rlen - 1 - i : i];
  for (int i = threadIdx.x; i < clen; i += blockDim.x) wc[i] = cf[conv ? clen - 1 - i : i];
  int bid = blockIdx.x;
  const int tx = bid % tiles_x;
  bid /= tiles_x;
  const int ty = bid % tiles_y, pl = bid / tiles_y;
  const int r0 = ty * kSTH, c0 = tx * kSTW;
  const float *xp = x + (size_t)pl * rows * cols;
  // image rows r0-hc .. r0+kSTH+hc-1, mapped by the border (the intermediate
  // field's border), columns c0-hr .. c0+kSTW+hr-1 mapped likewise; one warp
  // per staged row, lanes along it
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const bool inside_c = c0 - hr >= 0 && c0 - hr + IC <= cols;
  for (int ir = warp; ir < IR; ir += nwarps) {
    const int sr = border_index(border, r0 - hc + ir, rows);
    float *dst = img + (size_t)ir * IC;
    if (sr < 0) {
      for (int ic = lane; ic < IC; ic += 32) dst[ic] = 0.0f;
    } else if (inside_c) {
      const float *src = xp + (size_t)sr * cols + (c0 - hr);
      for (int ic = lane; ic < IC; ic += 32) dst[ic] = __ldg(src + ic);
    } else {
      const float *src = xp + (size_t)sr * cols;
      for (int ic = lane; ic < IC; ic += 32) {
        const int sc = border_index(border, c0 - hr + ic, cols);
        dst[ic] = sc >= 0 ? __ldg(src + sc) : 0.0f;
      }
    }
  }
  __syncthreads();
  // rows pass: intermediate of every staged row (zero rows stay zero: the
  // intermediate field is zero outside under BorderZero)
  for (int e = threadIdx.x; e < IR * kSTW; e += blockDim.x) {
    const int ir = e / kSTW, j = e - ir * kSTW;
    const float *line = img + (size_t)ir * IC + j;
    float sum = 0.0f;
#pragma unroll 4
    for (int k = 0; k < rlen; ++k) sum = __fmaf_rn(line[k], wr[k], sum);
    mid[e] = sum;
  }
  __syncthreads();
  // columns pass
  float *yp = y + (size_t)pl * rows * cols;
  for (int e = threadIdx.x; e < kSTH * kSTW; e += blockDim.x) {
    const int i = e / kSTW, j = e - i * kSTW;
    const int r = r0 + i, c = c0 + j;
    if (r >= rows || c >= cols) continue;
    const float *col = mid + (size_t)i * kSTW + j;
    float sum = 0.0f;
#pragma unroll 4
    for (int k = 0; k < clen; ++k) sum = __fmaf_rn(col[(size_t)k * kSTW], wc[k], sum);
    yp[(size_t)r * cols + c] = sum;
  }
}

size_t separable_fused_smem(int rlen, int clen) {
  const size_t IR = kSTH + clen - 1, IC = kSTW + rlen - 1;
  return sizeof(float) * (rlen + clen + IR * IC + IR * kSTW);
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
  const size_t fsmem = separable_fused_smem(rlen, clen);
  if (fsmem <= 96 * 1024) {
    const int tiles_x = (cols + kSTW - 1) / kSTW, tiles_y = (rows + kSTH - 1) / kSTH;
    const long long blocks = (long long)tiles_x * tiles_y * planes;
    if (blocks <= 0x7fffffffLL) {
      if (fsmem > 48 * 1024) {
        int rc = check_cuda(cudaFuncSetAttribute(separable_fused, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)fsmem),
                            "cudaFuncSetAttribute(separable)");
        if (rc) return rc;
      }
      separable_fused<<<(unsigned)blocks, kThreads, fsmem, st>>>(rows, cols, planes, x, rf, rlen, cf, clen,
                                                                 border, orient, y, tiles_x, tiles_y);
      count_launches(1);
      return check_cuda(cudaGetLastError(), "separable launch");
    }
  }
  // long filters: the two passes through the caller's scratch field
  const long long total = (long long)rows * cols * planes;
  const long long want = (total + kThreads - 1) / kThreads;
  const int blocks = (int)(want < 148LL * 64 ? want : 148LL * 64);
  separable_pass<0><<<blocks, kThreads, 0, st>>>(rows, cols, planes, x, rf, rlen, border, orient, tmp);
  separable_pass<1><<<blocks, kThreads, 0, st>>>(rows, cols, planes, tmp, cf, clen, border, orient, y);
  count_launches(2);
  return check_cuda(cudaGetLastError(), "separable launch");
}

}  // namespace cct
