// Separable convolution: a rows pass then a columns pass
// (ConvolveRows2DHyperKernel.scala:66-160, ConvolveColumns2DHyperKernel.scala).
// Each output is a fused multiply-add chain from 0 over the 1-D filter taps,
// the order of the reference's `sum += localImage[..] * filter` loop.
// Short filters run both passes fused per output tile: under BorderZero on
// fields whose width is a multiple of 4 floats the halo tiles arrive by TMA
// (separable_tma), otherwise threads stage them (separable_fused_t /
// separable_fused); long filters run one thread per output per pass, through
// a scratch field.
#include <atomic>

#include "cct_internal.h"
#include "sm100_util.cuh"
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

// The same fused tile with the filter lengths fixed at compile time (1, 3,
// 5, 7 or 9): each thread slides a register window along 8 outputs of a row
// in the rows pass and down 8 outputs of a column in the columns pass, so a
// tap costs a multiply-add and not a shared-memory read.
template <int RL, int CL>
struct SepTile {
  static constexpr int hr = (RL - 1) / 2, hc = (CL - 1) / 2, U = 8;
  // Odd pitches keep both passes free of bank conflicts: in the rows pass a
  // warp's lanes walk down 32 staged rows of one 8-column block (pitch IC)
  // and write the intermediate down a column (pitch MP); in the columns pass
  // lanes walk along a row of the intermediate.
  static constexpr int IR = kSTH + CL - 1, ICU = kSTW + RL - 1, IC = ICU | 1, MP = kSTW + 1;
};

template <int RL, int CL>
__global__ void __launch_bounds__(kThreads)
    separable_fused_t(int rows, int cols, const float *__restrict__ x, const float *__restrict__ rf,
                      const float *__restrict__ cf, int border, int orient, float *__restrict__ y,
                      int tiles_x, int tiles_y, long long tiles) {
  grid_dependency_wait();  // launched with programmatic serialisation: nothing global before this
  using T = SepTile<RL, CL>;
  constexpr int IR = T::IR, IC = T::IC, MP = T::MP, U = T::U, hr = T::hr, hc = T::hc, ICU = T::ICU;
  __shared__ float img[IR * IC];
  __shared__ float mid[IR * MP];
  float wr[RL], wc[CL];
  const bool conv = orient == CCT_CONVOLUTION;
#pragma unroll
  for (int k = 0; k < RL; ++k) wr[k] = __ldg(rf + (conv ? RL - 1 - k : k));
#pragma unroll
  for (int k = 0; k < CL; ++k) wc[k] = __ldg(cf + (conv ? CL - 1 - k : k));
  int bid = blockIdx.x;
  const int tx = bid % tiles_x;
  bid /= tiles_x;
  const int ty = bid % tiles_y, pl = bid / tiles_y;
  const int r0 = ty * kSTH, c0 = tx * kSTW;
  const float *xp = x + (size_t)pl * rows * cols;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const bool inside_c = c0 - hr >= 0 && c0 - hr + ICU <= cols;
  for (int ir = warp; ir < IR; ir += nwarps) {
    const int sr = border_index(border, r0 - hc + ir, rows);
    float *dst = img + ir * IC;
    if (sr < 0) {
      for (int ic = lane; ic < ICU; ic += 32) dst[ic] = 0.0f;
    } else if (inside_c) {
      const float *src = xp + (size_t)sr * cols + (c0 - hr);
      for (int ic = lane; ic < ICU; ic += 32) dst[ic] = __ldg(src + ic);
    } else {
      const float *src = xp + (size_t)sr * cols;
      for (int ic = lane; ic < ICU; ic += 32) {
        const int sc = border_index(border, c0 - hr + ic, cols);
        dst[ic] = sc >= 0 ? __ldg(src + sc) : 0.0f;
      }
    }
  }
  __syncthreads();
  for (int item = threadIdx.x; item < IR * (kSTW / U); item += blockDim.x) {
    const int jb = item / IR, ir = item - jb * IR, j0 = jb * U;
    const float *line = img + ir * IC + j0;
    float win[U + RL - 1];
#pragma unroll
    for (int k = 0; k < U + RL - 1; ++k) win[k] = line[k];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      float sum = 0.0f;
#pragma unroll
      for (int k = 0; k < RL; ++k) sum = __fmaf_rn(win[u + k], wr[k], sum);
      mid[ir * MP + j0 + u] = sum;
    }
  }
  __syncthreads();
  float *yp = y + (size_t)pl * rows * cols;
  for (int item = threadIdx.x; item < kSTW * (kSTH / U); item += blockDim.x) {
    const int j = item % kSTW, i0 = (item / kSTW) * U;
    const int c = c0 + j;
    float win[U + CL - 1];
#pragma unroll
    for (int k = 0; k < U + CL - 1; ++k) win[k] = mid[(i0 + k) * MP + j];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      float sum = 0.0f;
#pragma unroll
      for (int k = 0; k < CL; ++k) sum = __fmaf_rn(win[u + k], wc[k], sum);
      const int r = r0 + i0 + u;
      if (r < rows && c < cols) yp[(size_t)r * cols + c] = sum;
    }
  }
}

template <int RL, int CL>
int launch_fused_t(int rows, int cols, const float *x, const float *rf, const float *cf, int border,
                   int orient, float *y, int tiles_x, int tiles_y, long long tiles, cudaStream_t st) {
  if (tiles > 0x7fffffffLL) return set_error(CCT_ENOTSUP, "separable: grid too large");
  const int rc = launch_pdl(separable_fused_t<RL, CL>, dim3((unsigned)tiles), dim3(kThreads), 0, st,
                            "separable launch", rows, cols, x, rf, cf, border, orient, y, tiles_x, tiles_y, tiles);
  if (!rc) count_launches(1);
  return rc;
}

// BorderZero with TMA staging: persistent CTAs walk 64 x 128 output tiles
// and thread 0 keeps kSepStages halo tiles in flight (3-D TMA loads
// completing on mbarriers; TMA's out-of-bounds zero fill is BorderZero, for
// the image and for the intermediate field alike).  The box's x origin is
// rounded down to a multiple of 4 floats and the kernel indexes from the
// remainder OFF.  A thread owns 4 columns x 8 rows of output: for each staged
// row it forms the 4 row-filtered values (an fma chain from 0 over the row
// taps) and feeds each to the column chains of the outputs that use that
// row, in tap order, so every output is the same fma chain of the same
// values as in the two-pass form.
constexpr int kSepTW = 64, kSepTH = 128, kSepU = 4, kSepV = 8, kSepTX = 16, kSepStages = 2;

template <int RL, int CL, int OFF>
struct SepTma {
  static constexpr int hr = (RL - 1) / 2, hc = (CL - 1) / 2;
  static constexpr int IN_ROWS = kSepTH + CL - 1;
  static constexpr int BOX_C = (kSepTW + RL - 1 + OFF + 3) & ~3;
  static constexpr int STAGE = ((IN_ROWS * BOX_C) + 31) & ~31;  // floats, 128-byte multiple
  static constexpr uint32_t BYTES = IN_ROWS * BOX_C * 4;
  static constexpr size_t SMEM = (size_t)kSepStages * STAGE * 4;
};

template <int RL, int CL, int OFF>
__global__ void __launch_bounds__(kThreads)
    separable_tma(const __grid_constant__ CUtensorMap xmap, int rows, int cols, const float *__restrict__ rf,
                  const float *__restrict__ cf, int orient, float *__restrict__ y, int tiles_x, int tiles_y,
                  int total, unsigned *err) {
  using T = SepTma<RL, CL, OFF>;
  constexpr int E = kSepU - 1 + RL;  // staged values a thread reads per row, from OFF
  constexpr int E4 = (OFF + E + 3) / 4;
  extern __shared__ __align__(128) float smem[];
  __shared__ __align__(8) uint64_t full[kSepStages];
  __shared__ int timed_out;
  const int tid = threadIdx.x;
  const int tx = tid % kSepTX, ty = tid / kSepTX;
  if (tid == 0) {
    for (int s = 0; s < kSepStages; ++s) mbar_init(&full[s], 1);
    timed_out = 0;
    fence_barrier_init();
  }
  __syncthreads();
  grid_dependency_wait();  // launched with programmatic serialisation: global memory only after this
  allow_dependent_launch();  // persistent: every CTA is resident already
  auto decode = [&](int i, int &pl, int &tyi, int &txi) {
    txi = i % tiles_x;
    const int q = i / tiles_x;
    tyi = q % tiles_y;
    pl = q / tiles_y;
  };
  auto issue = [&](int i, int s) {
    int pl, tyi, txi;
    decode(i, pl, tyi, txi);
    mbar_arrive_expect_tx(&full[s], T::BYTES);
    tma_load_3d(smem + s * T::STAGE, &xmap, &full[s], txi * kSepTW - T::hr - OFF, tyi * kSepTH - T::hc, pl);
  };
  if (tid == 0)
    for (int k = 0; k < kSepStages; ++k) {
      const int i = blockIdx.x + k * gridDim.x;
      if (i < total) issue(i, k);
    }
  float wr[RL], wc[CL];
  const bool conv = orient == CCT_CONVOLUTION;
#pragma unroll
  for (int k = 0; k < RL; ++k) wr[k] = __ldg(rf + (conv ? RL - 1 - k : k));
#pragma unroll
  for (int k = 0; k < CL; ++k) wc[k] = __ldg(cf + (conv ? CL - 1 - k : k));
  const size_t page = (size_t)rows * cols;

  int j = 0;
  for (int i = blockIdx.x; i < total; i += gridDim.x, ++j) {
    const int s = j % kSepStages;
    const uint32_t parity = (uint32_t)((j / kSepStages) & 1);
    int pl, tyi, txi;
    decode(i, pl, tyi, txi);
    if (!mbar_wait(&full[s], parity, err)) timed_out = 1;
    __syncthreads();
    if (timed_out) {
      // Give the copies still in flight a bounded chance to land, then leave.
      if (tid == 0)
        for (int k = 1; k < kSepStages; ++k) {
          const int jj = j + k;
          if (blockIdx.x + jj * gridDim.x < total)
            mbar_wait(&full[jj % kSepStages], (uint32_t)((jj / kSepStages) & 1), err);
        }
      return;
    }
    const float *base = smem + s * T::STAGE + (ty * kSepV) * T::BOX_C + tx * kSepU;
    float acc[kSepV][kSepU];
#pragma unroll
    for (int v = 0; v < kSepV; ++v)
#pragma unroll
      for (int u = 0; u < kSepU; ++u) acc[v][u] = 0.0f;
#pragma unroll
    for (int tr = 0; tr < kSepV + CL - 1; ++tr) {
      float vals[E4 * 4];
#pragma unroll
      for (int e = 0; e < E4; ++e) {
        const float4 q = *reinterpret_cast<const float4 *>(base + tr * T::BOX_C + 4 * e);
        vals[4 * e + 0] = q.x;
        vals[4 * e + 1] = q.y;
        vals[4 * e + 2] = q.z;
        vals[4 * e + 3] = q.w;
      }
      float h[kSepU];
#pragma unroll
      for (int u = 0; u < kSepU; ++u) {
        float sum = 0.0f;
#pragma unroll
        for (int k = 0; k < RL; ++k) sum = __fmaf_rn(vals[OFF + u + k], wr[k], sum);
        h[u] = sum;
      }
#pragma unroll
      for (int v = 0; v < kSepV; ++v) {
        const int k = tr - v;
        if (k >= 0 && k < CL) {
#pragma unroll
          for (int u = 0; u < kSepU; ++u) acc[v][u] = __fmaf_rn(h[u], wc[k], acc[v][u]);
        }
      }
    }
    // the field width is a multiple of 4, so a thread's 4 columns are all in
    // or all out
    const int col0 = txi * kSepTW + tx * kSepU;
    if (col0 < cols) {
      float *yp = y + (size_t)pl * page + col0;
#pragma unroll
      for (int v = 0; v < kSepV; ++v) {
        const int row = tyi * kSepTH + ty * kSepV + v;
        if (row < rows)
          *reinterpret_cast<float4 *>(yp + (size_t)row * cols) = make_float4(acc[v][0], acc[v][1], acc[v][2],
                                                                             acc[v][3]);
      }
    }
    __syncthreads();  // every thread is done with stage s
    if (tid == 0) {
      const int next = i + kSepStages * gridDim.x;
      if (next < total) {
        fence_proxy_async_smem();
        issue(next, s);
      }
    }
  }
}

template <int RL, int CL, int OFF>
int launch_tma_t(int rows, int cols, int planes, const float *x, const float *rf, const float *cf, int orient,
                 float *y, cudaStream_t st) {
  using T = SepTma<RL, CL, OFF>;
  const int tiles_x = (cols + kSepTW - 1) / kSepTW, tiles_y = (rows + kSepTH - 1) / kSepTH;
  const long long total = (long long)tiles_x * tiles_y * planes;
  if (total > 0x7fffffffLL) return set_error(CCT_ENOTSUP, "separable: grid too large");
  CUtensorMap map;
  int rc = encode_tensor_map_3d(&map, x, cols, rows, planes, T::BOX_C, T::IN_ROWS);
  if (rc) return rc;
  auto kern = separable_tma<RL, CL, OFF>;
  int dev = 0;
  rc = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  // per instance: devices whose function attributes and grid size are set
  static std::atomic<unsigned long long> ready{0};
  static int grid_cap[64];
  if (dev >= 64) return set_error(CCT_ENOTSUP, "separable: device ordinal %d", dev);
  if (!(ready.load() >> dev & 1ull)) {
    rc = check_cuda(cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)T::SMEM),
                    "cudaFuncSetAttribute(separable_tma)");
    int sms = 0, per_sm = 0;
    if (!rc) rc = check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    if (!rc)
      rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, T::SMEM),
                      "separable occupancy");
    if (rc) return rc;
    grid_cap[dev] = sms * (per_sm > 0 ? per_sm : 1);
    ready.fetch_or(1ull << dev);
  }
  const int grid = (int)(total < grid_cap[dev] ? total : grid_cap[dev]);
  const int rc2 = launch_pdl(kern, dim3(grid), dim3(kThreads), T::SMEM, st, "separable_tma launch", map, rows, cols,
                             rf, cf, orient, y, tiles_x, tiles_y, (int)total, device_error_word());
  if (!rc2) count_launches(1);
  return rc2;
}

// Row lengths 1..9 (odd) with their x-offset remainder, column lengths 1..9
// (odd); -1 if not covered, else the launch status.
int launch_tma_small(int rows, int cols, int planes, const float *x, const float *rf, int rlen, const float *cf,
                     int clen, int orient, float *y, cudaStream_t st) {
#define CCT_SEPT_C(RL, CL, OFF) \
  if (rlen == RL && clen == CL) return launch_tma_t<RL, CL, OFF>(rows, cols, planes, x, rf, cf, orient, y, st);
#define CCT_SEPT_R(RL, OFF) \
  CCT_SEPT_C(RL, 1, OFF) CCT_SEPT_C(RL, 3, OFF) CCT_SEPT_C(RL, 5, OFF) CCT_SEPT_C(RL, 7, OFF) CCT_SEPT_C(RL, 9, OFF)
  // OFF = (-(RL - 1) / 2) mod 4
  CCT_SEPT_R(1, 0) CCT_SEPT_R(3, 3) CCT_SEPT_R(5, 2) CCT_SEPT_R(7, 1) CCT_SEPT_R(9, 0)
#undef CCT_SEPT_R
#undef CCT_SEPT_C
  return -1;
}

// Compile-time lengths 1, 3, 5, 7, 9 for both filters; -1 if not covered,
// else the launch status.
int launch_fused_small(int rows, int cols, const float *x, const float *rf, int rlen, const float *cf,
                       int clen, int border, int orient, float *y, int tiles_x, int tiles_y, long long tiles,
                       cudaStream_t st) {
#define CCT_SEP_C(RL, CL)                                                                                 \
  if (rlen == RL && clen == CL)                                                                           \
    return launch_fused_t<RL, CL>(rows, cols, x, rf, cf, border, orient, y, tiles_x, tiles_y, tiles, st);
#define CCT_SEP_R(RL) CCT_SEP_C(RL, 1) CCT_SEP_C(RL, 3) CCT_SEP_C(RL, 5) CCT_SEP_C(RL, 7) CCT_SEP_C(RL, 9)
  CCT_SEP_R(1) CCT_SEP_R(3) CCT_SEP_R(5) CCT_SEP_R(7) CCT_SEP_R(9)
#undef CCT_SEP_R
#undef CCT_SEP_C
  return -1;
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
    if (border == CCT_BORDER_ZERO && (cols & 3) == 0 && (reinterpret_cast<uintptr_t>(x) & 15) == 0 &&
        (reinterpret_cast<uintptr_t>(y) & 15) == 0) {
      const int rc = launch_tma_small(rows, cols, planes, x, rf, rlen, cf, clen, orient, y, st);
      if (rc >= 0) return rc;
    }
    const int rc = launch_fused_small(rows, cols, x, rf, rlen, cf, clen, border, orient, y, tiles_x, tiles_y,
                                      blocks, st);
    if (rc >= 0) return rc;
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
