// Device helpers shared by the direct and frame convolution kernels: border
// extension and the halo-tile loaders.
#pragma once

#include "cct_internal.h"

namespace cct {

// Border extension of one coordinate in input (pre-sampling) space; -1 means
// "reads zero".  Semantics of ConvolveHyperKernel.scala:235-317: Zero/Full
// fill zeros, Clamp replicates the edge, Cyclic wraps with a non-negative
// modulus, Valid only protects the high edge.
__device__ __forceinline__ int border_index(int border, int v, int n) {
  switch (border) {
    case CCT_BORDER_CLAMP:
      return v < 0 ? 0 : (v >= n ? n - 1 : v);
    case CCT_BORDER_CYCLIC: {
      int r = v % n;
      return r < 0 ? r + n : r;
    }
    case CCT_BORDER_VALID:
      return v >= n ? n - 1 : (v < 0 ? -1 : v);
    default:
      return (v >= 0 && v < n) ? v : -1;
  }
}

// Post-sampling coordinate -> source index, or -1.  With up-sampling by `up`
// the input is zero-inserted: only multiples of `up` carry a value
// (ConvolveHyperKernel.scala:206-212, 405-436 visit exactly those taps).
__device__ __forceinline__ int source_index(int border, int p, int n, int up) {
  if (up > 1) {
    int q = p / up;
    if (p - q * up != 0) return -1;
    p = q;
  }
  return border_index(border, p, n);
}

// Synchronous halo-tile load: rows x cols post-sampling values whose top-left
// corner is (org_r, org_c), into tile[tr * pitch + tc].  One warp per row,
// lanes across columns (coalesced).  An in-bounds tile without up-sampling
// skips the border logic.
__device__ __forceinline__ void load_tile(float *tile, int pitch, int rows,
                                          int cols,
                                          const float *__restrict__ src,
                                          const ConvGeom &g, int org_r,
                                          int org_c) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  const bool interior = g.up == 1 && org_r >= 0 && org_c >= 0 &&
                        org_r + rows <= g.H && org_c + cols <= g.W;
  if (interior) {
    for (int tr = warp; tr < rows; tr += nwarps) {
      const float *s = src + (size_t)(org_r + tr) * g.W + org_c;
      float *d = tile + tr * pitch;
      for (int tc = lane; tc < cols; tc += 32) d[tc] = __ldg(s + tc);
    }
  } else {
    for (int tr = warp; tr < rows; tr += nwarps) {
      const int sr = source_index(g.border, org_r + tr, g.H, g.up);
      const float *s = src + (size_t)(sr < 0 ? 0 : sr) * g.W;
      float *d = tile + tr * pitch;
      for (int tc = lane; tc < cols; tc += 32) {
        const int sc = source_index(g.border, org_c + tc, g.W, g.up);
        d[tc] = (sr >= 0 && sc >= 0) ? __ldg(s + sc) : 0.0f;
      }
    }
  }
}

// Asynchronous (cp.async) variant of load_tile: 4-byte copies with zero fill
// (src-size 0) for positions that read zero.  The caller commits and waits.
__device__ __forceinline__ void cp_async_f32(float *dst, const float *src,
                                             bool valid) {
  const unsigned saddr = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(saddr),
               "l"(src), "r"(valid ? 4 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void load_tile_async(float *tile, int pitch,
                                                int rows, int cols,
                                                const float *__restrict__ src,
                                                const ConvGeom &g, int org_r,
                                                int org_c) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
  const bool interior = g.up == 1 && org_r >= 0 && org_c >= 0 &&
                        org_r + rows <= g.H && org_c + cols <= g.W;
  if (interior) {
    for (int tr = warp; tr < rows; tr += nwarps) {
      const float *s = src + (size_t)(org_r + tr) * g.W + org_c;
      float *d = tile + tr * pitch;
      for (int tc = lane; tc < cols; tc += 32) cp_async_f32(d + tc, s + tc, true);
    }
  } else {
    for (int tr = warp; tr < rows; tr += nwarps) {
      const int sr = source_index(g.border, org_r + tr, g.H, g.up);
      const float *s = src + (size_t)(sr < 0 ? 0 : sr) * g.W;
      float *d = tile + tr * pitch;
      for (int tc = lane; tc < cols; tc += 32) {
        const int sc = source_index(g.border, org_c + tc, g.W, g.up);
        const bool ok = sr >= 0 && sc >= 0;
        cp_async_f32(d + tc, ok ? s + sc : src, ok);
      }
    }
  }
}

}  // namespace cct
