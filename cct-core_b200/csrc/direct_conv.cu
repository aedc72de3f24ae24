// Direct (stencil) field convolution: one output plane per CTA column of
// tiles, halo tile staged in shared memory, register-blocked outputs.
//
// Every output follows the summation order of the reference's generated
// OpenCL (ConvolveHyperKernel.scala:509-521 and :593-603): for each filter
// row a fused multiply-add chain over the filter columns starting from 0
// (`columnSum`), added into `rowSum`; frame reductions add `rowSum` of each
// input plane in increasing plane order.  The explicit __fmaf_rn/__fadd_rn
// keep nvcc from contracting the adds, so results are bit-identical to the
// CPU restatement of that order.
#include <algorithm>

#include "cct_internal.h"
#include "sm100_util.cuh"
#include "tile_common.cuh"

namespace cct {
namespace {

constexpr int kThreads = 256;
constexpr int kTX = 16, kTY = 16;  // thread grid of the fixed-size kernel

// Filter sizes compiled with the filter held in registers.
template <int R, int S, int DOWN, int U, int V>
__global__ void __launch_bounds__(kThreads)
    direct_fixed_kernel(ConvGeom g, const float *__restrict__ x,
                        const float *__restrict__ f, float *__restrict__ y,
                        int tiles_x, int tiles_y) {
  grid_dependency_wait();  // launched with programmatic serialisation: nothing global before this
  constexpr int TW = kTX * U, TH = kTY * V;
  constexpr int IN_COLS = (TW - 1) * DOWN + S;
  constexpr int IN_ROWS = (TH - 1) * DOWN + R;
  constexpr int PITCH = (IN_COLS + 3) & ~3;
  constexpr int E = (U - 1) * DOWN + S;  // values per tile row per thread
  constexpr int E4 = (E + 3) / 4;
  static_assert((U * DOWN) % 4 == 0, "thread column origin must be 16-byte aligned");
  __shared__ __align__(16) float tile[IN_ROWS * PITCH];

  int bid = blockIdx.x;
  const int tx_i = bid % tiles_x;
  bid /= tiles_x;
  const int ty_i = bid % tiles_y;
  const int o = bid / tiles_y;
  const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
  const int out_r0 = ty_i * TH, out_c0 = tx_i * TW;
  const int org_r = out_r0 * DOWN - g.low_r;
  const int org_c = out_c0 * DOWN - g.low_c;

  float acc[V][U];
#pragma unroll
  for (int v = 0; v < V; ++v)
#pragma unroll
    for (int u = 0; u < U; ++u) acc[v][u] = 0.0f;

  for (int t = 0; t < g.terms; ++t) {
    int ip, fp;
    plane_pair(g, o, t, &ip, &fp);
    const float *xs = x + (size_t)ip * g.H * g.W;
    const float *fs = f + (size_t)fp * (R * S);
    float w[R][S];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int s = 0; s < S; ++s)
        w[r][s] = __ldg(fs + (g.orient == CCT_CONVOLUTION
                                  ? (R - 1 - r) * S + (S - 1 - s)
                                  : r * S + s));
    if (t > 0) __syncthreads();
    load_tile(tile, PITCH, IN_ROWS, IN_COLS, xs, g, org_r, org_c);
    __syncthreads();

    float rs[V][U];
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
      for (int u = 0; u < U; ++u) rs[v][u] = 0.0f;

    const float *base = tile + (ty * V * DOWN) * PITCH + tx * U * DOWN;
#pragma unroll
    for (int tr = 0; tr < (V - 1) * DOWN + R; ++tr) {
      float vals[E4 * 4];
#pragma unroll
      for (int e = 0; e < E4; ++e) {
        const float4 q = *reinterpret_cast<const float4 *>(base + tr * PITCH + 4 * e);
        vals[4 * e + 0] = q.x;
        vals[4 * e + 1] = q.y;
        vals[4 * e + 2] = q.z;
        vals[4 * e + 3] = q.w;
      }
#pragma unroll
      for (int v = 0; v < V; ++v) {
        const int r = tr - v * DOWN;
        if (r >= 0 && r < R) {
#pragma unroll
          for (int u = 0; u < U; ++u) {
            float cs = 0.0f;
#pragma unroll
            for (int s = 0; s < S; ++s) cs = __fmaf_rn(vals[u * DOWN + s], w[r][s], cs);
            rs[v][u] = __fadd_rn(rs[v][u], cs);
          }
        }
      }
    }
#pragma unroll
    for (int v = 0; v < V; ++v)
#pragma unroll
      for (int u = 0; u < U; ++u)
        acc[v][u] = (t == 0) ? rs[v][u] : __fadd_rn(acc[v][u], rs[v][u]);
  }

  float *ys = y + (size_t)o * g.OH * g.OW;
  const bool relu = (g.flags & CCT_FLAG_RELU) != 0;
#pragma unroll
  for (int v = 0; v < V; ++v) {
    const int row = out_r0 + ty * V + v;
    if (row >= g.OH) continue;
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int col = out_c0 + tx * U + u;
      if (col < g.OW) ys[(size_t)row * g.OW + col] = relu ? fmaxf(acc[v][u], 0.0f) : acc[v][u];
    }
  }
}

// Any filter size and down-sampling step: filter staged in shared memory,
// four outputs along a row per thread.
constexpr int kGU = 4;                       // outputs per thread (columns)
constexpr int kGTW = kTX * kGU, kGTH = kTY;  // 64 x 16 output tile

__global__ void __launch_bounds__(kThreads)
    direct_generic_kernel(ConvGeom g, const float *__restrict__ x,
                          const float *__restrict__ f, float *__restrict__ y,
                          int tiles_x, int tiles_y, int in_rows, int in_cols,
                          int pitch) {
  grid_dependency_wait();  // launched with programmatic serialisation: nothing global before this
  extern __shared__ __align__(16) float smem[];
  float *tile = smem;
  float *wf = smem + in_rows * pitch;

  int bid = blockIdx.x;
  const int tx_i = bid % tiles_x;
  bid /= tiles_x;
  const int ty_i = bid % tiles_y;
  const int o = bid / tiles_y;
  const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
  const int out_r0 = ty_i * kGTH, out_c0 = tx_i * kGTW;
  const int org_r = out_r0 * g.down - g.low_r;
  const int org_c = out_c0 * g.down - g.low_c;
  const int R = g.R, S = g.S, D = g.down;

  float acc[kGU];
#pragma unroll
  for (int u = 0; u < kGU; ++u) acc[u] = 0.0f;

  for (int t = 0; t < g.terms; ++t) {
    int ip, fp;
    plane_pair(g, o, t, &ip, &fp);
    const float *xs = x + (size_t)ip * g.H * g.W;
    const float *fs = f + (size_t)fp * g.fr * g.fs;
    if (t > 0) __syncthreads();
    // Tap (r, s) of the R x S filter as applied: flipped for convolution, and
    // for an upsampled FilterAdjoint gradient the zero-inserted lattice
    // (stored taps at multiples of fup).
    for (int i = threadIdx.x; i < R * S; i += blockDim.x) {
      const int r = i / S, s = i - r * S;
      const int er = g.orient == CCT_CONVOLUTION ? R - 1 - r : r;
      const int es = g.orient == CCT_CONVOLUTION ? S - 1 - s : s;
      float v = 0.0f;
      if (er % g.fup == 0 && es % g.fup == 0) v = __ldg(fs + (er / g.fup) * g.fs + es / g.fup);
      wf[i] = v;
    }
    load_tile(tile, pitch, in_rows, in_cols, xs, g, org_r, org_c);
    __syncthreads();

    float rs[kGU];
#pragma unroll
    for (int u = 0; u < kGU; ++u) rs[u] = 0.0f;
    const float *base = tile + (ty * D) * pitch + tx * kGU * D;
    for (int r = 0; r < R; ++r) {
      const float *row = base + r * pitch;
      const float *wr = wf + r * S;
      float cs[kGU];
#pragma unroll
      for (int u = 0; u < kGU; ++u) cs[u] = 0.0f;
      for (int s = 0; s < S; ++s) {
        const float w = wr[s];
#pragma unroll
        for (int u = 0; u < kGU; ++u) cs[u] = __fmaf_rn(row[u * D + s], w, cs[u]);
      }
#pragma unroll
      for (int u = 0; u < kGU; ++u) rs[u] = __fadd_rn(rs[u], cs[u]);
    }
#pragma unroll
    for (int u = 0; u < kGU; ++u) acc[u] = (t == 0) ? rs[u] : __fadd_rn(acc[u], rs[u]);
  }

  const int row = out_r0 + ty;
  if (row < g.OH) {
    float *ys = y + (size_t)o * g.OH * g.OW + (size_t)row * g.OW;
    const bool relu = (g.flags & CCT_FLAG_RELU) != 0;
#pragma unroll
    for (int u = 0; u < kGU; ++u) {
      const int col = out_c0 + tx * kGU + u;
      if (col < g.OW) ys[col] = relu ? fmaxf(acc[u], 0.0f) : acc[u];
    }
  }
}

template <int R, int S, int DOWN, int U, int V>
int launch_fixed(const ConvGeom &g, const float *x, const float *f, float *y,
                 cudaStream_t st) {
  constexpr int TW = kTX * U, TH = kTY * V;
  const int tiles_x = (g.OW + TW - 1) / TW, tiles_y = (g.OH + TH - 1) / TH;
  const long long blocks = (long long)tiles_x * tiles_y * g.pout;
  if (blocks > 0x7fffffffLL) return set_error(CCT_ENOTSUP, "direct convolution grid too large");
  const int rc = launch_pdl(direct_fixed_kernel<R, S, DOWN, U, V>, dim3((unsigned)blocks), dim3(kThreads), 0, st,
                            "direct_fixed_kernel launch", g, x, f, y, tiles_x, tiles_y);
  if (!rc) count_launches(1);
  return rc;
}

int launch_generic(const ConvGeom &g, const float *x, const float *f, float *y,
                   cudaStream_t st) {
  const int tiles_x = (g.OW + kGTW - 1) / kGTW, tiles_y = (g.OH + kGTH - 1) / kGTH;
  const int in_rows = (kGTH - 1) * g.down + g.R;
  const int in_cols = (kGTW - 1) * g.down + g.S;
  const int pitch = (in_cols + 3) & ~3;
  const size_t smem = sizeof(float) * ((size_t)in_rows * pitch + (size_t)g.R * g.S);
  int dev = 0, max_smem = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (smem > (size_t)max_smem)
    return set_error(CCT_ENOTSUP, "filter %dx%d with step %d needs %zu bytes of shared memory (max %d)",
                     g.R, g.S, g.down, smem, max_smem);
  if (smem > 48 * 1024) {
    int rc = check_cuda(cudaFuncSetAttribute(direct_generic_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                        "cudaFuncSetAttribute");
    if (rc) return rc;
  }
  const long long blocks = (long long)tiles_x * tiles_y * g.pout;
  if (blocks > 0x7fffffffLL) return set_error(CCT_ENOTSUP, "direct convolution grid too large");
  const int rc = launch_pdl(direct_generic_kernel, dim3((unsigned)blocks), dim3(kThreads), smem, st,
                            "direct_generic_kernel launch", g, x, f, y, tiles_x, tiles_y, in_rows, in_cols, pitch);
  if (!rc) count_launches(1);
  return rc;
}

}  // namespace

int launch_direct(const ConvGeom &g, const float *x, const float *f, float *y,
                  cudaStream_t st) {
  if (g.fup != 1) return launch_generic(g, x, f, y, st);
  if (g.R == g.S && g.down == 1) {
    switch (g.R) {
      case 1: return launch_fixed<1, 1, 1, 4, 4>(g, x, f, y, st);
      case 3: return launch_fixed<3, 3, 1, 4, 4>(g, x, f, y, st);
      case 5: return launch_fixed<5, 5, 1, 4, 4>(g, x, f, y, st);
      case 7: return launch_fixed<7, 7, 1, 4, 4>(g, x, f, y, st);
      default: break;
    }
  }
  if (g.R == g.S && g.down == 2) {
    switch (g.R) {
      case 1: return launch_fixed<1, 1, 2, 2, 2>(g, x, f, y, st);
      case 3: return launch_fixed<3, 3, 2, 2, 2>(g, x, f, y, st);
      case 5: return launch_fixed<5, 5, 2, 2, 2>(g, x, f, y, st);
      case 7: return launch_fixed<7, 7, 2, 2, 2>(g, x, f, y, st);
      default: break;
    }
  }
  return launch_generic(g, x, f, y, st);
}

}  // namespace cct
