// FilterAdjoint (weight gradient) in FP32 for small results:
//   out[B*w + b](r, s) = sum_(i,j) x[b*C + w%C](r + i, s + j) * g'[b*L + w/C](i, j)
// with BorderValid, no sampling (ConvolveHyperKernel.scala:187, 333, 575-590;
// CogFunctionAPI.scala:1480-1511), g' = g flipped for convolveFilterAdjoint.
// The block-reduced form sums the B images of each w in order.
//
// The result planes are tiny (the filter's size) and the reduction is long
// (the whole gradient plane).  Each thread owns one (input plane c, gradient
// plane l, result row r) and keeps the result row's S outputs in registers
// while it walks the gradient; the image row it needs slides through a
// register window, so each tap costs one image load and one gradient load for
// S multiply-adds.  Per output the order is the reference's: an fma chain over
// j from 0 per gradient row, row sums added in order, so the result is
// bit-identical to the FP32 oracle.
//
// fa_rows_kernel (the main path): a CTA serves one image b, kCG input planes
// and kLG gradient planes.  It streams the gradient rows i = 0.. through
// shared memory together with a ring of the OH image rows each step needs
// (cp.async, the next rows landing while the current ones are used), so
// every image row and gradient row is read from L2 once per CTA.
// fa_f32_kernel: the fallback for image rows too wide to stage; one CTA per
// (b, l) with the gradient plane in shared memory and image rows read
// through L1.
// The block-reduced form writes the per-image results to plan workspace and
// a second kernel adds them in image order.
#include "cct_internal.h"
#include "tile_common.cuh"

namespace cct {
namespace {

constexpr int kFaThreads = 256;
constexpr int kFaMaxS = 8;
constexpr int kCG = 8, kLG = 8;  // input planes x gradient planes per CTA (fa_rows_kernel)
constexpr size_t kRowsSmemMax = 96 * 1024;

// shared memory of fa_rows_kernel: a ring of OH + 1 image rows per input
// plane and two gradient rows per gradient plane, each row padded to 4 floats
__host__ __device__ inline int fa_row_pitch(int n) { return (n + 3) & ~3; }
__host__ __device__ inline size_t fa_rows_smem(const ConvGeom &g) {
  return sizeof(float) * ((size_t)kCG * (g.OH + 1) * fa_row_pitch(g.W) + (size_t)kLG * 2 * fa_row_pitch(g.S));
}

template <int S>
__global__ void __launch_bounds__(kCG * kLG * kFaMaxS)
    fa_rows_kernel(ConvGeom g, const float *__restrict__ x, const float *__restrict__ f, float *__restrict__ y,
                   int cgroups, int lgroups) {
  extern __shared__ __align__(16) float sm[];
  const int Hg = g.R, Wg = g.S, C = g.n, L = g.groups, B = g.batch, OH = g.OH;
  const int xp_pitch = fa_row_pitch(g.W), gp_pitch = fa_row_pitch(Wg), slots = OH + 1;
  float *xring = sm;                                       // [c][slot][xp_pitch]
  float *grow = sm + (size_t)kCG * slots * xp_pitch;       // [l][2][gp_pitch]
  int bid = blockIdx.x;
  const int cg = bid % cgroups;
  bid /= cgroups;
  const int lg = bid % lgroups, b = bid / lgroups;
  const int c0 = cg * kCG, l0 = lg * kLG;
  const bool conv = g.orient == CCT_CONVOLUTION;
  const int nthreads = blockDim.x;
  // thread -> (l, c, r): r fastest, so neighbouring threads share image rows
  const int r = threadIdx.x % OH, q = threadIdx.x / OH;
  const int cl = q % kCG, ll = q / kCG;
  const bool active = ll < kLG && c0 + cl < C && l0 + ll < L;

  // copies of image row `row` of every input plane of the group into its slot
  auto load_x_row = [&](int row) {
    const int slot = row % slots;
    for (int e = threadIdx.x; e < kCG * g.W; e += nthreads) {
      const int c = e / g.W, col = e - c * g.W;
      const bool ok = c0 + c < C;
      const float *src = x + ((size_t)(b * C + c0 + c) * g.H + row) * g.W + col;
      cp_async_f32(xring + ((size_t)c * slots + slot) * xp_pitch + col, ok ? src : x, ok);
    }
  };
  // gradient row i (flipped for convolution) of every gradient plane into buffer i&1
  auto load_g_row = [&](int i) {
    const int gi = conv ? Hg - 1 - i : i;
    for (int e = threadIdx.x; e < kLG * Wg; e += nthreads) {
      const int l = e / Wg, j = e - l * Wg;
      const bool ok = l0 + l < L;
      const int gj = conv ? Wg - 1 - j : j;
      const float *src = f + ((size_t)(b * L + l0 + l) * Hg + gi) * Wg + gj;
      cp_async_f32(grow + ((size_t)l * 2 + (i & 1)) * gp_pitch + j, ok ? src : f, ok);
    }
  };

  for (int row = 0; row < OH; ++row) load_x_row(row);
  load_g_row(0);
  cp_async_commit();

  float acc[S];
#pragma unroll
  for (int s = 0; s < S; ++s) acc[s] = 0.0f;
  for (int i = 0; i < Hg; ++i) {
    if (i + 1 < Hg) {  // next step's rows land while this step computes
      load_x_row(i + OH);
      load_g_row(i + 1);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    if (active) {
      const float *xr = xring + ((size_t)cl * slots + (i + r) % slots) * xp_pitch;
      const float *gr = grow + ((size_t)ll * 2 + (i & 1)) * gp_pitch;
      float win[S], col[S];
#pragma unroll
      for (int s = 0; s < S; ++s) {
        col[s] = 0.0f;
        win[s] = xr[s];
      }
      for (int j = 0; j < Wg; ++j) {
        const float w = gr[j];
#pragma unroll
        for (int s = 0; s < S; ++s) col[s] = __fmaf_rn(win[s], w, col[s]);
#pragma unroll
        for (int s = 0; s + 1 < S; ++s) win[s] = win[s + 1];
        win[S - 1] = xr[min(j + S, g.W - 1)];  // the last step's value is never used
      }
#pragma unroll
      for (int s = 0; s < S; ++s) acc[s] = __fadd_rn(acc[s], col[s]);
    }
    __syncthreads();  // the ring slot and gradient buffer are refilled next step
  }
  if (!active) return;
  float *yp = y + ((size_t)B * ((l0 + ll) * C + c0 + cl) + b) * OH * g.OW + (size_t)r * g.OW;
  const bool relu = (g.flags & CCT_FLAG_RELU) != 0;
#pragma unroll
  for (int s = 0; s < S; ++s) yp[s] = relu ? fmaxf(acc[s], 0.0f) : acc[s];
}

template <int S>
__global__ void __launch_bounds__(kFaThreads)
    fa_f32_kernel(ConvGeom g, const float *__restrict__ x, const float *__restrict__ f, float *__restrict__ y,
                  int cgroups) {
  extern __shared__ __align__(16) float gs[];
  const int Hg = g.R, Wg = g.S;  // the gradient plane is the "filter"
  const int C = g.n, L = g.groups, B = g.batch;
  int bid = blockIdx.x;
  const int cg = bid % cgroups;
  bid /= cgroups;
  const int l = bid % L, b = bid / L;
  const int per = blockDim.x / g.OH;  // input planes per CTA
  const int c = cg * per + threadIdx.x / g.OH, r = threadIdx.x % g.OH;
  const bool conv = g.orient == CCT_CONVOLUTION;
  const float *gp = f + (size_t)(b * L + l) * Hg * Wg;
  for (int i = threadIdx.x; i < Hg * Wg; i += blockDim.x)
    gs[i] = __ldg(gp + (conv ? Hg * Wg - 1 - i : i));
  __syncthreads();
  if (threadIdx.x >= per * g.OH || c >= C) return;
  const float *xp = x + (size_t)(b * C + c) * g.H * g.W + (size_t)r * g.W;
  float acc[S];
#pragma unroll
  for (int s = 0; s < S; ++s) acc[s] = 0.0f;
  for (int i = 0; i < Hg; ++i) {
    const float *xr = xp + (size_t)i * g.W;
    const float *gr = gs + i * Wg;
    float win[S], col[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      col[s] = 0.0f;
      win[s] = s < g.OW ? __ldg(xr + s) : 0.0f;
    }
    for (int j = 0; j < Wg; ++j) {
      const float w = gr[j];
#pragma unroll
      for (int s = 0; s < S; ++s) col[s] = __fmaf_rn(win[s], w, col[s]);
      // slide: win[s] = x(r + i, j + 1 + s)
#pragma unroll
      for (int s = 0; s + 1 < S; ++s) win[s] = win[s + 1];
      const int nx = j + S;
      win[S - 1] = nx < g.W ? __ldg(xr + nx) : 0.0f;
    }
#pragma unroll
    for (int s = 0; s < S; ++s) acc[s] = __fadd_rn(acc[s], col[s]);
  }
  // output plane B*w + b, w = l*C + c
  float *yp = y + ((size_t)B * (l * C + c) + b) * g.OH * g.OW + (size_t)r * g.OW;
  const bool relu = (g.flags & CCT_FLAG_RELU) != 0;
#pragma unroll
  for (int s = 0; s < S; ++s)
    if (s < g.OW) yp[s] = relu ? fmaxf(acc[s], 0.0f) : acc[s];
}

// out[w] = sum_b part[B*w + b], images in order (acc from 0).
__global__ void fa_reduce_kernel(const float *__restrict__ part, float *__restrict__ y, int B, long long planes,
                                 int plane_elems, bool relu) {
  const long long n = planes * plane_elems;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const long long w = e / plane_elems, q = e - w * plane_elems;
    const float *pp = part + (size_t)w * B * plane_elems + q;
    float acc = 0.0f;
    for (int b = 0; b < B; ++b) acc = __fadd_rn(acc, pp[(size_t)b * plane_elems]);
    y[e] = relu ? fmaxf(acc, 0.0f) : acc;
  }
}

}  // namespace

bool fa_f32_supported(const ConvGeom &g) {
  if (g.mode != CCT_FILTER_ADJOINT && g.mode != CCT_FILTER_ADJOINT_BLOCK_REDUCE_SUM) return false;
  if (g.border != CCT_BORDER_VALID || g.down != 1 || g.up != 1 || g.fup != 1) return false;
  if (g.OW > kFaMaxS || g.OH > kFaThreads) return false;
  return (size_t)g.R * g.S * sizeof(float) <= 96 * 1024;
}

size_t fa_workspace_bytes(const ConvGeom &g) {
  if (g.mode != CCT_FILTER_ADJOINT_BLOCK_REDUCE_SUM || g.batch == 1) return 0;
  return (size_t)g.batch * g.n * g.groups * g.OH * g.OW * sizeof(float);
}

int launch_fa_f32(const ConvGeom &g, const float *x, const float *f, float *y, float *work, cudaStream_t st) {
  const bool reduce = g.mode == CCT_FILTER_ADJOINT_BLOCK_REDUCE_SUM && g.batch > 1;
  float *dst = reduce ? work : y;
  if (reduce && !work) return set_error(CCT_EINVAL, "FilterAdjoint block reduce needs plan workspace");
  const int per = kFaThreads / g.OH;
  const int cgroups = (g.n + per - 1) / per;
  const size_t smem = (size_t)g.R * g.S * sizeof(float);
  const long long blocks = (long long)g.batch * g.groups * cgroups;
  if (blocks > 0x7fffffffLL) return set_error(CCT_ENOTSUP, "FilterAdjoint grid too large");
  ConvGeom q = g;
  if (reduce) q.flags &= ~CCT_FLAG_RELU;  // ReLU applies to the reduced sum
  const size_t rsmem = fa_rows_smem(g);
  if (g.OH <= kFaMaxS && rsmem <= kRowsSmemMax) {
    const int cgroups = (g.n + kCG - 1) / kCG, lgroups = (g.groups + kLG - 1) / kLG;
    const long long rblocks = (long long)g.batch * lgroups * cgroups;
    if (rblocks > 0x7fffffffLL) return set_error(CCT_ENOTSUP, "FilterAdjoint grid too large");
    const int threads = kCG * kLG * g.OH;
#define CCT_FA_ROWS_CASE(SS)                                                                            \
  case SS: {                                                                                            \
    if (rsmem > 48 * 1024) {                                                                            \
      int rc = check_cuda(cudaFuncSetAttribute(fa_rows_kernel<SS>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                               (int)rsmem),                                             \
                          "cudaFuncSetAttribute(fa rows)");                                             \
      if (rc) return rc;                                                                                \
    }                                                                                                   \
    fa_rows_kernel<SS><<<(unsigned)rblocks, threads, rsmem, st>>>(q, x, f, dst, cgroups, lgroups);      \
    break;                                                                                              \
  }
    switch (g.OW) {
      CCT_FA_ROWS_CASE(1) CCT_FA_ROWS_CASE(2) CCT_FA_ROWS_CASE(3) CCT_FA_ROWS_CASE(4)
      CCT_FA_ROWS_CASE(5) CCT_FA_ROWS_CASE(6) CCT_FA_ROWS_CASE(7) CCT_FA_ROWS_CASE(8)
      default: return set_error(CCT_ENOTSUP, "FilterAdjoint result width %d", g.OW);
    }
#undef CCT_FA_ROWS_CASE
    count_launches(1);
  } else {
#define CCT_FA_CASE(SS)                                                                               \
  case SS: {                                                                                          \
    if (smem > 48 * 1024) {                                                                           \
      int rc = check_cuda(cudaFuncSetAttribute(fa_f32_kernel<SS>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                               (int)smem),                                            \
                          "cudaFuncSetAttribute(fa)");                                                \
      if (rc) return rc;                                                                              \
    }                                                                                                 \
    fa_f32_kernel<SS><<<(unsigned)blocks, per * g.OH, smem, st>>>(q, x, f, dst, cgroups);             \
    break;                                                                                            \
  }
  switch (g.OW) {
    CCT_FA_CASE(1) CCT_FA_CASE(2) CCT_FA_CASE(3) CCT_FA_CASE(4)
    CCT_FA_CASE(5) CCT_FA_CASE(6) CCT_FA_CASE(7) CCT_FA_CASE(8)
    default: return set_error(CCT_ENOTSUP, "FilterAdjoint result width %d", g.OW);
  }
#undef CCT_FA_CASE
    count_launches(1);
  }
  if (reduce) {
    const long long planes = (long long)g.n * g.groups;
    const long long n = planes * g.OH * g.OW;
    const int rblocks = (int)std::min<long long>((n + 255) / 256, 148LL * 8);
    fa_reduce_kernel<<<rblocks, 256, 0, st>>>(work, y, g.batch, planes, g.OH * g.OW,
                                              (g.flags & CCT_FLAG_RELU) != 0);
    count_launches(1);
  }
  return check_cuda(cudaGetLastError(), "FilterAdjoint launch");
}

}  // namespace cct
