// Fused filter-bank convolution in FP32 on the CUDA cores:
//   ProjectFrameBlockReduceSum      y[b*K+k] = sum_c xcorr(x[b*N+c], f[k*N+c])
//   BackProjectFrameBlockReduceSum  y[b*L+l] = sum_n conv (x[b*N+n], f[n*L+l])
// (ConvolveHyperKernel.scala:153-199, 319-340, 574-645, fused by
// ProjectFrameTensorReduceSumOptimizer.scala:75-170).
//
// One CTA owns a 32x16 output tile of one image for a block of 16 output
// planes.  It walks the N input planes in order; each plane's halo tile and
// the 16 filters' taps for that plane are staged in shared memory with
// cp.async, double-buffered so the next plane loads while this one computes.
// A thread holds 4 adjacent outputs x 8 output planes.  Summation order per
// output matches the reference (per-row fma chain, row sum, plane sum), so
// results are bit-identical to the FP32 CPU restatement.
//
// The same kernel without the reduce (REDUCE = false) serves the unfused
// modes ProjectFrame / BackProjectFrame (CogFunctionAPI.scala:1370-1377,
// 1425-1432), whose output plane b*F + k*N + c is input plane c of image b
// correlated with one filter: each input plane's tile feeds the 16 filters
// of the block and every result (per-row fma chain, row sum) is stored to
// its own plane.
#include "cct_internal.h"
#include "sm100_util.cuh"
#include "tile_common.cuh"

namespace cct {
namespace {

constexpr int kThreads = 256;
constexpr int kU = 4;        // adjacent outputs per thread
constexpr int kKT = 8;       // output planes per thread
constexpr int kKG = 2;       // plane groups per CTA
constexpr int kKB = kKT * kKG;  // output planes per CTA
constexpr int kSX = 8, kSY = 16;  // spatial threads per group
constexpr int kTW = kSX * kU, kTH = kSY;  // 32 x 16 output tile

template <int R, int S, int DOWN>
struct FrameTile {
  static constexpr int IN_COLS = (kTW - 1) * DOWN + S;
  static constexpr int IN_ROWS = (kTH - 1) * DOWN + R;
  static constexpr int PITCH = (IN_COLS + 3) & ~3;
  static constexpr int TILE = IN_ROWS * PITCH;
  static constexpr int FILT = R * S * kKB;  // [tap][plane]
  static constexpr int STAGE = TILE + FILT;
};

template <int R, int S, int DOWN, bool REDUCE>
__global__ void __launch_bounds__(kThreads, 2)
    frame_f32_kernel(ConvGeom g, const float *__restrict__ x,
                     const float *__restrict__ f, float *__restrict__ y,
                     int tiles_x, int tiles_y, int kblocks, int tchunk) {
  grid_dependency_wait();  // launched with programmatic serialisation: nothing global before this
  using T = FrameTile<R, S, DOWN>;
  constexpr int E = (kU - 1) * DOWN + S;
  constexpr int E4 = (E + 3) / 4;
  static_assert((kU * DOWN) % 4 == 0, "16-byte aligned thread origin");
  extern __shared__ __align__(16) float smem[];

  int bid = blockIdx.x;
  const int tx_i = bid % tiles_x;
  bid /= tiles_x;
  const int ty_i = bid % tiles_y;
  bid /= tiles_y;
  const int kb = bid % kblocks;
  bid /= kblocks;
  // unfused modes: the input planes are split into chunks of tchunk, one per
  // CTA (their outputs are independent); reduced modes: one chunk of all
  const int nchunks = REDUCE ? 1 : (g.n + tchunk - 1) / tchunk;
  const int t0 = REDUCE ? 0 : (bid % nchunks) * tchunk;
  const int b = bid / nchunks;
  const int k0 = kb * kKB;
  const int kcount = min(kKB, g.groups - k0);

  const int grp = threadIdx.x / (kSX * kSY);
  const int sp = threadIdx.x % (kSX * kSY);
  const int tx = sp % kSX, ty = sp / kSX;
  const int out_r0 = ty_i * kTH, out_c0 = tx_i * kTW;
  const int org_r = out_r0 * DOWN - g.low_r;
  const int org_c = out_c0 * DOWN - g.low_c;
  const int plane = g.H * g.W;
  const bool conv = g.orient == CCT_CONVOLUTION;

  // Stage loader for input-plane term t into buffer `buf`.
  auto issue = [&](int t, int buf) {
    float *tile = smem + buf * T::STAGE;
    float *ft = tile + T::TILE;
    const int ip = b * g.n + t0 + t;
    load_tile_async(tile, T::PITCH, T::IN_ROWS, T::IN_COLS, x + (size_t)ip * plane, g, org_r, org_c);
    for (int i = threadIdx.x; i < R * S * kKB; i += kThreads) {
      const int kk = i / (R * S), tap = i - kk * (R * S);
      const int r = tap / S, s = tap - r * S;
      const int src_tap = conv ? (R - 1 - r) * S + (S - 1 - s) : tap;
      // output plane of filter k0 + kk: b*K + k (reduced) or b*F + k*N + t
      const int o = REDUCE ? b * g.groups + k0 + kk : b * g.pf + (k0 + kk) * g.n + t0 + t;
      int ipp, fp;
      plane_pair(g, o, REDUCE ? t : 0, &ipp, &fp);
      const bool ok = kk < kcount;
      cp_async_f32(ft + tap * kKB + kk, ok ? f + (size_t)fp * (R * S) + src_tap : f, ok);
    }
    cp_async_commit();
  };

  // Output planes k, k+1 advance together in packed fma.rn.f32x2 / add.rn.f32x2
  // (each lane the same RN operation as the scalar form, so the order and
  // the result per output are unchanged).
  constexpr int kP = kKT / 2;
  float2 acc[kU][kP];
#pragma unroll
  for (int u = 0; u < kU; ++u)
#pragma unroll
    for (int k = 0; k < kP; ++k) acc[u][k] = make_float2(0.0f, 0.0f);

  const int nterms = REDUCE ? g.terms : min(tchunk, g.n - t0);
  const bool relu = (g.flags & CCT_FLAG_RELU) != 0;
  const size_t opage = (size_t)g.OH * g.OW;
  const int row = out_r0 + ty;
  issue(0, 0);
  for (int t = 0; t < nterms; ++t) {
    if (t + 1 < nterms) {
      issue(t + 1, (t + 1) & 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const float *tile = smem + (t & 1) * T::STAGE;
    const float *ft = tile + T::TILE + grp * kKT;
    const float *base = tile + (ty * DOWN) * T::PITCH + tx * kU * DOWN;

    float2 rs[kU][kP];
#pragma unroll
    for (int u = 0; u < kU; ++u)
#pragma unroll
      for (int k = 0; k < kP; ++k) rs[u][k] = make_float2(0.0f, 0.0f);

#pragma unroll
    for (int r = 0; r < R; ++r) {
      float vals[E4 * 4];
#pragma unroll
      for (int e = 0; e < E4; ++e) {
        const float4 q = *reinterpret_cast<const float4 *>(base + r * T::PITCH + 4 * e);
        vals[4 * e + 0] = q.x;
        vals[4 * e + 1] = q.y;
        vals[4 * e + 2] = q.z;
        vals[4 * e + 3] = q.w;
      }
      float2 cs[kU][kP];
#pragma unroll
      for (int s = 0; s < S; ++s) {
        float2 w[kP];
#pragma unroll
        for (int k4 = 0; k4 < kKT / 4; ++k4) {
          const float4 q = *reinterpret_cast<const float4 *>(ft + (r * S + s) * kKB + 4 * k4);
          w[2 * k4 + 0] = make_float2(q.x, q.y);
          w[2 * k4 + 1] = make_float2(q.z, q.w);
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const float xv = vals[u * DOWN + s];
          const float2 x2 = make_float2(xv, xv);
#pragma unroll
          for (int k = 0; k < kP; ++k)
            cs[u][k] = __ffma2_rn(x2, w[k], s == 0 ? make_float2(0.0f, 0.0f) : cs[u][k]);
        }
      }
#pragma unroll
      for (int u = 0; u < kU; ++u)
#pragma unroll
        for (int k = 0; k < kP; ++k) rs[u][k] = __fadd2_rn(rs[u][k], cs[u][k]);
    }
    if (REDUCE) {
#pragma unroll
      for (int u = 0; u < kU; ++u)
#pragma unroll
        for (int k = 0; k < kP; ++k) acc[u][k] = (t == 0) ? rs[u][k] : __fadd2_rn(acc[u][k], rs[u][k]);
    } else if (row < g.OH) {
      // this input plane's result for each filter of the block: its own plane
      const int col0 = out_c0 + tx * kU;
      const bool vec = (g.OW & 3) == 0 && col0 + kU <= g.OW;
#pragma unroll
      for (int k = 0; k < kKT; ++k) {
        const int kk = grp * kKT + k;
        if (kk >= kcount) break;
        float *ys = y + (size_t)(b * g.pf + (k0 + kk) * g.n + t0 + t) * opage + (size_t)row * g.OW;
        float v[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
          const float a = (k & 1) ? rs[u][k >> 1].y : rs[u][k >> 1].x;
          v[u] = relu ? fmaxf(a, 0.0f) : a;
        }
        if (vec) {
          *reinterpret_cast<float4 *>(ys + col0) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
#pragma unroll
          for (int u = 0; u < kU; ++u)
            if (col0 + u < g.OW) ys[col0 + u] = v[u];
        }
      }
    }
    __syncthreads();
  }

  if constexpr (REDUCE) {
    if (row >= g.OH) return;
#pragma unroll
    for (int k = 0; k < kKT; ++k) {
      const int kk = grp * kKT + k;
      if (kk >= kcount) break;
      float *ys = y + (size_t)(b * g.groups + k0 + kk) * opage + (size_t)row * g.OW;
#pragma unroll
      for (int u = 0; u < kU; ++u) {
        const int col = out_c0 + tx * kU + u;
        const float a = (k & 1) ? acc[u][k >> 1].y : acc[u][k >> 1].x;
        if (col < g.OW) ys[col] = relu ? fmaxf(a, 0.0f) : a;
      }
    }
  }
}

template <int R, int S, int DOWN>
int launch(const ConvGeom &g, const float *x, const float *f, float *y, cudaStream_t st) {
  const bool reduce = g.mode == CCT_PROJECT_FRAME_BLOCK_REDUCE_SUM || g.mode == CCT_BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM;
  using T = FrameTile<R, S, DOWN>;
  const int tiles_x = (g.OW + kTW - 1) / kTW, tiles_y = (g.OH + kTH - 1) / kTH;
  const int kblocks = (g.groups + kKB - 1) / kKB;
  const int tchunk = reduce ? g.terms : 4;  // unfused: 4 input planes per CTA
  const int nchunks = reduce ? 1 : (g.n + tchunk - 1) / tchunk;
  const long long blocks = (long long)tiles_x * tiles_y * kblocks * nchunks * g.batch;
  if (blocks > 0x7fffffffLL) return set_error(CCT_ENOTSUP, "frame grid too large");
  const size_t smem = 2 * sizeof(float) * T::STAGE;
  static_assert(2 * sizeof(float) * T::STAGE <= 48 * 1024, "frame stages exceed the default smem limit");
  const int rc = launch_pdl(reduce ? frame_f32_kernel<R, S, DOWN, true> : frame_f32_kernel<R, S, DOWN, false>,
                            dim3((unsigned)blocks), dim3(kThreads), smem, st, "frame_f32_kernel launch", g, x, f, y,
                            tiles_x, tiles_y, kblocks, tchunk);
  if (!rc) count_launches(1);
  return rc;
}

}  // namespace

bool frame_f32_supported(const ConvGeom &g) {
  if (g.mode != CCT_PROJECT_FRAME_BLOCK_REDUCE_SUM && g.mode != CCT_BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM &&
      g.mode != CCT_PROJECT_FRAME && g.mode != CCT_BACK_PROJECT_FRAME)
    return false;
  if (g.up != 1) return false;
  if (g.R != g.S) return false;
  if (g.down != 1 && g.down != 2) return false;
  return g.R == 1 || g.R == 3 || g.R == 5 || g.R == 7 || g.R == 9;
}

int launch_frame_f32(const ConvGeom &g, const float *x, const float *f, float *y,
                     cudaStream_t st) {
#define CCT_FRAME_CASE(RR, DD) \
  if (g.R == RR && g.down == DD) return launch<RR, RR, DD>(g, x, f, y, st);
  CCT_FRAME_CASE(1, 1) CCT_FRAME_CASE(3, 1) CCT_FRAME_CASE(5, 1) CCT_FRAME_CASE(7, 1) CCT_FRAME_CASE(9, 1)
  CCT_FRAME_CASE(1, 2) CCT_FRAME_CASE(3, 2) CCT_FRAME_CASE(5, 2) CCT_FRAME_CASE(7, 2) CCT_FRAME_CASE(9, 2)
#undef CCT_FRAME_CASE
  return set_error(CCT_ENOTSUP, "frame FP32 kernel: unsupported filter %dx%d step %d", g.R, g.S,
                   g.down);
}

}  // namespace cct
