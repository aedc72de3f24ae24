// Scalar field cross-correlated with every matrix of a matrix field
// (ScalarMatrixConvolve2DHyperKernel.scala:43-160), the form
// CogFunctionAPI.scala:1209-1216 selects when a ScalarField is convolved with
// a MatrixField.  Output plane p = row * matrix_cols + col holds the
// cross-correlation with the matrix at (row, col); every output is ONE fused
// multiply-add chain from 0 over the taps in row-major order (the kernel's
// `sum += inputPixel * filterElement`), with halo size / 2 and the border's
// index rule for the input tile.
//
// A CTA stages a 32 x 64 output tile's border-mapped input halo and a block
// of matrices in shared memory; thread (row i, 8-column group g) slides a
// register window along its 8 outputs of row i for each matrix in turn.
// Odd row pitch: the 32 lanes of a warp (32 rows, one column group) hit 32
// banks; the matrix taps are broadcast.  The grid spans tiles x matrix blocks
// so that a single small field still fills the GPU.
#include "cct_internal.h"
#include "tile_common.cuh"

namespace cct {
namespace {

constexpr int kThreads = 256, kTH = 32, kTW = 64, kU = 8;
constexpr int kMaxFilterFloats = 12288;  // staged matrix taps per CTA (48 KB)

struct SmTile {
  int fs, IR, ICU, IC;
  __host__ __device__ explicit SmTile(int size)
      : fs(size), IR(kTH + size - 1), ICU(kTW + size - 1), IC((kTW + size - 1) | 1) {}
};

// F > 0: size fixed at compile time (register window); F == 0: run-time size.
template <int F>
__global__ void __launch_bounds__(kThreads)
    scalar_matrix_kernel(int rows, int cols, const float *__restrict__ x, const float *__restrict__ mats,
                         int L, int size, int border, float *__restrict__ y, int tiles_x, int lb) {
  extern __shared__ float sm[];
  const SmTile t(F > 0 ? F : size);
  const int fs = t.fs, taps = fs * fs, h = fs / 2;
  float *img = sm;                       // IR x IC
  float *filt = sm + (size_t)t.IR * t.IC;  // lb matrices x taps, matrix-major
  const int tx = blockIdx.x % tiles_x, ty = blockIdx.x / tiles_x;
  const int r0 = ty * kTH, c0 = tx * kTW;
  const int p0 = blockIdx.y * lb;
  const int nl = min(lb, L - p0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;

  // border-mapped input halo: rows r0-h .., columns c0-h ..
  const bool inside_c = c0 - h >= 0 && c0 - h + t.ICU <= cols;
  for (int ir = warp; ir < t.IR; ir += nwarps) {
    const int sr = border_index(border, r0 - h + ir, rows);
    float *dst = img + (size_t)ir * t.IC;
    if (sr < 0) {
      for (int ic = lane; ic < t.ICU; ic += 32) dst[ic] = 0.0f;
    } else if (inside_c) {
      const float *src = x + (size_t)sr * cols + (c0 - h);
      for (int ic = lane; ic < t.ICU; ic += 32) dst[ic] = __ldg(src + ic);
    } else {
      const float *src = x + (size_t)sr * cols;
      for (int ic = lane; ic < t.ICU; ic += 32) {
        const int sc = border_index(border, c0 - h + ic, cols);
        dst[ic] = sc >= 0 ? __ldg(src + sc) : 0.0f;
      }
    }
  }
  // this block's matrices: the field stores tap-major, so consecutive threads
  // read consecutive matrices of one tap
  for (int e = threadIdx.x; e < nl * taps; e += blockDim.x) {
    const int tap = e / nl, q = e - tap * nl;
    filt[q * taps + tap] = __ldg(mats + (size_t)tap * L + p0 + q);
  }
  __syncthreads();

  const int i = threadIdx.x & 31, cg = threadIdx.x >> 5;  // kThreads / 32 == kTW / kU
  const int orow = r0 + i, ocol = c0 + cg * kU;
  if (orow >= rows || ocol >= cols) return;
  const size_t page = (size_t)rows * cols;
  float *yp = y + (size_t)p0 * page + (size_t)orow * cols + ocol;
  const bool full = ocol + kU <= cols;
  for (int q = 0; q < nl; ++q) {
    const float *w = filt + q * taps;
    float sum[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) sum[u] = 0.0f;
    if (F > 0) {
#pragma unroll 1
      for (int r = 0; r < (F > 0 ? F : 1); ++r) {
        const float *line = img + (size_t)(i + r) * t.IC + cg * kU;
        float win[kU + (F > 0 ? F : 1) - 1];
#pragma unroll
        for (int k = 0; k < kU + F - 1; ++k) win[k] = line[k];
#pragma unroll
        for (int c = 0; c < F; ++c) {
          const float wt = w[r * F + c];
#pragma unroll
          for (int u = 0; u < kU; ++u) sum[u] = __fmaf_rn(win[u + c], wt, sum[u]);
        }
      }
    } else {
      for (int r = 0; r < fs; ++r) {
        const float *line = img + (size_t)(i + r) * t.IC + cg * kU;
        for (int c = 0; c < fs; ++c) {
          const float wt = w[r * fs + c];
#pragma unroll
          for (int u = 0; u < kU; ++u) sum[u] = __fmaf_rn(line[u + c], wt, sum[u]);
        }
      }
    }
    float *dst = yp + (size_t)q * page;
    if (full) {
#pragma unroll
      for (int u = 0; u < kU; ++u) dst[u] = sum[u];
    } else {
#pragma unroll
      for (int u = 0; u < kU; ++u)
        if (ocol + u < cols) dst[u] = sum[u];
    }
  }
}

template <int F>
int launch_sm(int rows, int cols, const float *x, const float *mats, int L, int size, int border, float *y,
              cudaStream_t st) {
  const SmTile t(size);
  const int taps = size * size;
  const int tiles_x = (cols + kTW - 1) / kTW, tiles_y = (rows + kTH - 1) / kTH;
  const long long tiles = (long long)tiles_x * tiles_y;
  if (tiles > 0x7fffffffLL) return set_error(CCT_ENOTSUP, "scalar-matrix convolution: field too large");
  // matrices per CTA: enough CTAs to fill the GPU (about 2 per SM), at most
  // what the staging buffer holds
  const long long want_blocks = (296 + tiles - 1) / tiles;
  long long lb = (L + want_blocks - 1) / want_blocks;
  lb = std::min<long long>(lb, std::max(1, kMaxFilterFloats / taps));
  lb = std::max<long long>(lb, 1);
  const long long ly = (L + lb - 1) / lb;
  if (ly > 65535) return set_error(CCT_ENOTSUP, "scalar-matrix convolution: too many matrices");
  const size_t smem = sizeof(float) * ((size_t)t.IR * t.IC + (size_t)lb * taps);
  if (smem > 200 * 1024) return set_error(CCT_ENOTSUP, "scalar-matrix convolution: matrix size %d too large", size);
  auto kern = scalar_matrix_kernel<F>;
  if (smem > 48 * 1024) {
    int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                        "cudaFuncSetAttribute(scalar_matrix)");
    if (rc) return rc;
  }
  kern<<<dim3((unsigned)tiles, (unsigned)ly), kThreads, smem, st>>>(rows, cols, x, mats, L, size, border, y,
                                                                     tiles_x, (int)lb);
  count_launches(1);
  return check_cuda(cudaGetLastError(), "scalar_matrix launch");
}

}  // namespace

int launch_scalar_matrix(int rows, int cols, const float *x, const float *mats, int L, int size, int border,
                         float *y, cudaStream_t st) {
  switch (size) {
    case 1: return launch_sm<1>(rows, cols, x, mats, L, size, border, y, st);
    case 3: return launch_sm<3>(rows, cols, x, mats, L, size, border, y, st);
    case 5: return launch_sm<5>(rows, cols, x, mats, L, size, border, y, st);
    case 7: return launch_sm<7>(rows, cols, x, mats, L, size, border, y, st);
    case 9: return launch_sm<9>(rows, cols, x, mats, L, size, border, y, st);
    case 11: return launch_sm<11>(rows, cols, x, mats, L, size, border, y, st);
    default: return launch_sm<0>(rows, cols, x, mats, L, size, border, y, st);
  }
}

}  // namespace cct
