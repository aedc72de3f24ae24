// Memory-bound direct convolution with TMA halo-tile staging.
//
// Persistent CTAs walk 64x128 output tiles; thread 0 keeps kStages tiles in
// flight with 3-D TMA loads (cols, rows, plane) completing on mbarriers, so
// HBM reads overlap the stencil arithmetic.  Zero-fill borders (Zero, Full,
// and Valid, which never reads outside for kept outputs) come for free from
// TMA's out-of-bounds zero fill.  The box's x origin is rounded down to a
// multiple of 4 floats (TMA needs 16-byte aligned x) and the kernel indexes
// from the remainder OFF.  Summation order per output is the reference's
// (ConvolveHyperKernel.scala:509-521): per filter row an fma chain from 0,
// then the row sum.
#include <mutex>
#include <unordered_map>

#include "cct_internal.h"
#include "sm100_util.cuh"
#include "tile_common.cuh"

namespace cct {
namespace {

constexpr int kThreads = 256;
// 64 x 128 output tiles, a thread owning 4 columns x 8 rows: each staged row
// feeds up to 8 output rows, so the loads, tile bookkeeping and barrier per
// output are half those of 64 x 64 tiles with 4 rows per thread (0.77 of the
// copy bandwidth against 0.72); two stages of 38 KB, two CTAs per SM.
constexpr int kTW = 64, kTH = 128, kU = 4, kV = 8, kTX = 16;
constexpr int kStages = 2;
constexpr int kCtasPerSm = 2;

template <int R, int S, int OFF>
struct TmaTile {
  static constexpr int IN_ROWS = kTH + R - 1;
  static constexpr int BOX_C = (kTW + S - 1 + OFF + 3) & ~3;
  static constexpr int STAGE = ((IN_ROWS * BOX_C) + 31) & ~31;  // floats, 128-byte multiple
  static constexpr uint32_t BYTES = IN_ROWS * BOX_C * 4;
  static constexpr size_t SMEM = (size_t)kStages * STAGE * 4;
};

template <int R, int S, int OFF>
__global__ void __launch_bounds__(kThreads, kCtasPerSm)
    direct_tma_kernel(const __grid_constant__ CUtensorMap xmap, ConvGeom g,
                      const float *__restrict__ f, float *__restrict__ y, int tiles_x,
                      int tiles_y, int total, unsigned *err) {
  using T = TmaTile<R, S, OFF>;
  constexpr int E = (kU - 1) + S;
  constexpr int E4 = (OFF + E + 3) / 4;
  extern __shared__ __align__(128) float smem[];
  __shared__ __align__(8) uint64_t full[kStages];
  __shared__ int timed_out;

  const int tid = threadIdx.x;
  const int tx = tid % kTX, ty = tid / kTX;
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) mbar_init(&full[s], 1);
    timed_out = 0;
    fence_barrier_init();
  }
  __syncthreads();
  grid_dependency_wait();  // launched with programmatic serialisation: global memory only after this
  allow_dependent_launch();  // persistent: every CTA is resident already

  auto decode = [&](int i, int &o, int &tyi, int &txi) {
    txi = i % tiles_x;
    const int q = i / tiles_x;
    tyi = q % tiles_y;
    o = q / tiles_y;
  };
  auto issue = [&](int i, int s) {
    int o, tyi, txi, ip, fp;
    decode(i, o, tyi, txi);
    plane_pair(g, o, 0, &ip, &fp);
    const int org_r = tyi * kTH - g.low_r;
    const int start_c = txi * kTW - g.low_c - OFF;  // multiple of 4
    mbar_arrive_expect_tx(&full[s], T::BYTES);
    tma_load_3d(smem + s * T::STAGE, &xmap, &full[s], start_c, org_r, ip);
  };

  if (tid == 0) {
    for (int k = 0; k < kStages; ++k) {
      const int i = blockIdx.x + k * gridDim.x;
      if (i < total) issue(i, k);
    }
  }

  const bool conv = g.orient == CCT_CONVOLUTION;
  const bool relu = (g.flags & CCT_FLAG_RELU) != 0;
  const bool vec_store = (g.OW & 3) == 0;
  const size_t opage = (size_t)g.OH * g.OW;
  int cur_fp = -1;
  float w[R][S];

  int j = 0;
  for (int i = blockIdx.x; i < total; i += gridDim.x, ++j) {
    const int s = j % kStages;
    const uint32_t parity = (uint32_t)((j / kStages) & 1);
    int o, tyi, txi, ip, fp;
    decode(i, o, tyi, txi);
    plane_pair(g, o, 0, &ip, &fp);
    if (fp != cur_fp) {
      const float *fs = f + (size_t)fp * (R * S);
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int c = 0; c < S; ++c)
          w[r][c] = __ldg(fs + (conv ? (R - 1 - r) * S + (S - 1 - c) : r * S + c));
      cur_fp = fp;
    }
    if (!mbar_wait(&full[s], parity, err)) timed_out = 1;
    __syncthreads();
    if (timed_out) {
      // Give the copies still in flight a bounded chance to land, then leave.
      if (tid == 0)
        for (int k = 1; k < kStages; ++k) {
          const int jj = j + k;
          if (blockIdx.x + jj * gridDim.x < total)
            mbar_wait(&full[jj % kStages], (uint32_t)((jj / kStages) & 1), err);
        }
      return;
    }

    const float *base = smem + s * T::STAGE + (ty * kV) * T::BOX_C + tx * kU;
    float rs[kV][kU];
#pragma unroll
    for (int v = 0; v < kV; ++v)
#pragma unroll
      for (int u = 0; u < kU; ++u) rs[v][u] = 0.0f;
#pragma unroll
    for (int tr = 0; tr < kV - 1 + R; ++tr) {
      float vals[E4 * 4];
#pragma unroll
      for (int e = 0; e < E4; ++e) {
        const float4 q = *reinterpret_cast<const float4 *>(base + tr * T::BOX_C + 4 * e);
        vals[4 * e + 0] = q.x;
        vals[4 * e + 1] = q.y;
        vals[4 * e + 2] = q.z;
        vals[4 * e + 3] = q.w;
      }
#pragma unroll
      for (int v = 0; v < kV; ++v) {
        const int r = tr - v;
        if (r >= 0 && r < R) {
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            float cs = 0.0f;
#pragma unroll
            for (int c = 0; c < S; ++c) cs = __fmaf_rn(vals[OFF + u + c], w[r][c], cs);
            rs[v][u] = __fadd_rn(rs[v][u], cs);
          }
        }
      }
    }

    float *ys = y + (size_t)o * opage;
    const int col0 = txi * kTW + tx * kU;
#pragma unroll
    for (int v = 0; v < kV; ++v) {
      const int row = tyi * kTH + ty * kV + v;
      if (row >= g.OH) break;
      float out[kU];
#pragma unroll
      for (int u = 0; u < kU; ++u) out[u] = relu ? fmaxf(rs[v][u], 0.0f) : rs[v][u];
      float *dst = ys + (size_t)row * g.OW + col0;
      if (vec_store && col0 + kU <= g.OW) {
        *reinterpret_cast<float4 *>(dst) = make_float4(out[0], out[1], out[2], out[3]);
      } else {
#pragma unroll
        for (int u = 0; u < kU; ++u)
          if (col0 + u < g.OW) dst[u] = out[u];
      }
    }

    __syncthreads();  // every thread is done with stage s
    if (tid == 0) {
      const int next = i + kStages * gridDim.x;
      if (next < total) {
        fence_proxy_async_smem();
        issue(next, s);
      }
    }
  }
}

using EncodeFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                              const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                              const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn() {
  static EncodeFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeFn>(p);
  });
  return fn;
}

std::mutex g_attr_mu;
std::unordered_map<uint64_t, bool> g_attr_done;

int ensure_smem(const void *func, size_t bytes) {
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t key = reinterpret_cast<uint64_t>(func) ^ ((uint64_t)dev << 56);
  std::lock_guard<std::mutex> lk(g_attr_mu);
  if (g_attr_done.count(key)) return CCT_OK;
  int rc = check_cuda(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)bytes),
                      "cudaFuncSetAttribute(direct_tma)");
  if (!rc) g_attr_done[key] = true;
  return rc;
}

template <int R, int OFF>
int launch_tma(const ConvGeom &g, const float *x, const float *f, float *y, cudaStream_t st,
               unsigned *err) {
  using T = TmaTile<R, R, OFF>;
  CUtensorMap map;
  int rc = encode_tensor_map_3d(&map, x, g.W, g.H, g.pin, T::BOX_C, T::IN_ROWS);
  if (rc) return rc;
  const int tiles_x = (g.OW + kTW - 1) / kTW, tiles_y = (g.OH + kTH - 1) / kTH;
  const long long total = (long long)tiles_x * tiles_y * g.pout;
  if (total > 0x7fffffffLL) return set_error(CCT_ENOTSUP, "direct convolution grid too large");
  auto kern = direct_tma_kernel<R, R, OFF>;
  rc = ensure_smem((const void *)kern, T::SMEM);
  if (rc) return rc;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // persistent CTAs: as many as are resident at once (registers and shared
  // memory decide), so no CTA waits for another to finish
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, T::SMEM);
  const int grid = (int)std::min<long long>(total, (long long)std::max(per_sm, 1) * sms);
  const int rc2 = launch_pdl(kern, dim3(grid), dim3(kThreads), T::SMEM, st, "direct_tma_kernel launch", map, g, f,
                             y, tiles_x, tiles_y, (int)total, err);
  if (!rc2) count_launches(1);
  return rc2;
}

}  // namespace

int encode_tensor_map_3d(CUtensorMap *map, const float *base, uint64_t cols, uint64_t rows,
                         uint64_t planes, uint32_t box_c, uint32_t box_r) {
  return encode_tensor_map_3d_box(map, base, cols, rows, planes, box_c, box_r, 1);
}

int encode_tensor_map_3d_box(CUtensorMap *map, const float *base, uint64_t cols, uint64_t rows,
                             uint64_t planes, uint32_t box_c, uint32_t box_r, uint32_t box_z) {
  EncodeFn fn = encode_fn();
  if (!fn) return set_error(CCT_ECUDA, "cuTensorMapEncodeTiled unavailable");
  const cuuint64_t dims[3] = {cols, rows, planes};
  const cuuint64_t strides[2] = {cols * 4, cols * rows * 4};
  const cuuint32_t box[3] = {box_c, box_r, box_z};
  const cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(CCT_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return CCT_OK;
}

int encode_tensor_map_f32(CUtensorMap *map, const float *base, int rank, const uint64_t *dims,
                          const uint64_t *strides, const uint32_t *box) {
  EncodeFn fn = encode_fn();
  if (!fn) return set_error(CCT_ECUDA, "cuTensorMapEncodeTiled unavailable");
  if (rank < 1 || rank > 5) return set_error(CCT_EINVAL, "tensor map rank %d", rank);
  cuuint64_t d[5], st[4];
  cuuint32_t b[5], e[5];
  for (int i = 0; i < rank; ++i) {
    d[i] = dims[i];
    b[i] = box[i];
    e[i] = 1;
    if (i > 0) st[i - 1] = strides[i - 1];
  }
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank, (void *)base, d, st, b, e,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(CCT_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return CCT_OK;
}

bool direct_tma_supported(const ConvGeom &g, const float *x) {
  if (g.terms != 1 || g.up != 1 || g.down != 1 || g.fup != 1) return false;
  if (g.border != CCT_BORDER_ZERO && g.border != CCT_BORDER_FULL && g.border != CCT_BORDER_VALID)
    return false;
  if (g.R != g.S || (g.R != 1 && g.R != 3 && g.R != 5 && g.R != 7)) return false;
  if ((g.W & 3) != 0) return false;
  if ((reinterpret_cast<uintptr_t>(x) & 15) != 0) return false;
  return true;
}

int launch_direct_tma(const ConvGeom &g, const float *x, const float *f, float *y,
                      cudaStream_t st, unsigned *err) {
  const int off = ((g.low_c % 4) == 0) ? 0 : 4 - (g.low_c % 4);  // (-low_c) mod 4
#define CCT_TMA_CASE(RR, OO) \
  if (g.R == RR && off == OO) return launch_tma<RR, OO>(g, x, f, y, st, err);
  CCT_TMA_CASE(1, 0)
  CCT_TMA_CASE(3, 0) CCT_TMA_CASE(3, 2) CCT_TMA_CASE(3, 3)
  CCT_TMA_CASE(5, 0) CCT_TMA_CASE(5, 2)
  CCT_TMA_CASE(7, 0) CCT_TMA_CASE(7, 1) CCT_TMA_CASE(7, 2)
#undef CCT_TMA_CASE
  return set_error(CCT_ENOTSUP, "direct TMA kernel: filter %d with halo %d", g.R, g.low_c);
}

}  // namespace cct
