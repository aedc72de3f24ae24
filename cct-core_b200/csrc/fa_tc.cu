// FilterAdjointBlockReduceSum (the weight gradient) on the tcgen05 tensor
// cores in split-BF16 precision, for the shapes fa_f32 serves (BorderValid,
// no sampling, small results):
//   out[l*C + c](r, s) = sum_b sum_(i,j) x[b*C + c](r + i, s + j) * g'[b*L + l](i, j)
// (ConvolveHyperKernel.scala:187, 333, 575-590; CogFunctionAPI.scala:1480-1511;
// g' = g flipped for convolveFilterAdjoint).
//
// GEMM view: D[m][n] = sum_k A[m][k] B[n][k] with rows m = (c, r, s) of the
// result (M = C*OH*OW), columns n = l (the gradient planes) and the reduction
// k = (b, i, j) over every image's gradient pixels.  A reduction chunk is 32
// consecutive pixels j of one gradient row i of one image b:
//   A[m][jj] = x[b*C + c](r + i, s + j0 + jj)  (tensor memory, lane m)
//   B[n][jj] = g'[b*L + l](i, j0 + jj)        (shared memory, K-major)
// Both are split into bf16 hi + lo as they are built, and each chunk issues
// A_hi x [B_hi; B_lo] into [hh | small] and A_lo x B_hi into the small half,
// as the frame kernel does (the small products never meet the large sum in
// the tensor core's FP32 accumulation).
//
// The grid is (row tile, column block, reduction split): each CTA reduces a
// contiguous range of chunks into its accumulator and stores its partial
// sums; fa_tc_reduce adds the splits in split order, so the result does not
// depend on scheduling.  Within a CTA all 8 warps build every chunk (the
// next chunks' loads in flight while the current one is converted) into one
// of kStages stages and arrive on the stage's `full` barrier; one thread
// waits on it, issues the MMAs, and their commit on `empty` frees the stage.
// Every wait is bounded; on a timeout the CTA
// raises the device error word, waits (bounded) for its MMAs, frees its
// tensor memory and leaves.
#include <cuda_bf16.h>

#include <algorithm>

#include "cct_internal.h"
#include "sm100_util.cuh"

namespace cct {
namespace {

constexpr int kFaThreads = 256;
constexpr int kMT = 128;   // result rows (c, r, s) per tile = TMEM lanes
constexpr int kNT = 64;    // gradient planes per column block (max)
constexpr int kKC = 32;    // gradient pixels per reduction chunk (two MMA K-steps)
constexpr int kTmemCols = 256;
constexpr int kPF = 2;     // chunks whose loads are in flight ahead of the one being built
constexpr int kStages = 4; // A/B stages: chunks built ahead of the MMAs that read them

struct FaTcParams {
  int H, W, Hg, Wg, OH, OW, C, L, B;
  int conv;
  int M, Mpad, NT, Lpad, mtiles, nblocks, jb, nch, splits;
  const float *x, *g;
  float *part;  // [split][Lpad][Mpad]
  unsigned *err;
};

// Byte offset of (n, k) in one K-major operand image of rows x 32 bf16 (no
// swizzle): core matrix (8 rows x 8 elements, 128 bytes) at (n/8)*512 + (k/8)*128.
__device__ __forceinline__ uint32_t b_offset(int n, int k) {
  return (uint32_t)((n >> 3) * 512 + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2);
}

__global__ void __launch_bounds__(kFaThreads, 2) fa_tc_kernel(const __grid_constant__ FaTcParams p) {
  extern __shared__ __align__(1024) uint8_t smem[];  // kStages stages of [B_hi; B_lo]: 2 * NT * 32 bf16 each
  __shared__ __align__(8) uint64_t empty[kStages];
  __shared__ __align__(8) uint64_t full[kStages];
  __shared__ __align__(8) uint64_t done;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t stage_bytes = 2u * p.NT * kKC * 2;  // [B_hi; B_lo], NT x 32 bf16 each

  int bid = blockIdx.x;
  const int mt = bid % p.mtiles;
  bid /= p.mtiles;
  const int nb = bid % p.nblocks, split = bid / p.nblocks;
  const int q0 = (int)((long long)split * p.nch / p.splits), q1 = (int)((long long)(split + 1) * p.nch / p.splits);

  if (tid == 0) {
    for (int k = 0; k < kStages; ++k) {
      mbar_init(&empty[k], 1);                // the MMA commit
      mbar_init(&full[k], kFaThreads / 32);   // one arrival per warp
    }
    mbar_init(&done, 1);
    fence_barrier_init();
  }
  if (warp == 0) tmem_alloc(&tmem_slot, kTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  grid_dependency_wait();  // launched with programmatic serialisation: global memory only after this

  // this thread's A elements: row m (lane quarter warp & 3), K half warp >> 2
  const int m = (warp & 3) * 32 + lane, khalf = warp >> 2;
  const int mg = mt * kMT + m;
  const bool mvalid = mg < p.M;
  const int ohw = p.OH * p.OW;
  const int c = mvalid ? mg / ohw : 0, rs = mvalid ? mg - c * ohw : 0;
  const int r = rs / p.OW, s = rs - r * p.OW;
  // this thread's B elements: row n, K quarter
  const int n = tid >> 2, kq = (tid & 3) * 8;
  const int l = nb * kNT + n;
  const bool nvalid = n < p.NT && l < p.L;
  const float *xt = p.x + ((size_t)c * p.H + r) * p.W + s + khalf * 16;  // + b*C*H*W + i*W + j0
  const float *gt = p.g + (size_t)(nvalid ? l : 0) * p.Hg * p.Wg;         // + b*L*Hg*Wg + row*Wg
  const size_t ximg = (size_t)p.C * p.H * p.W, gimg = (size_t)p.L * p.Hg * p.Wg;

  // the next chunk to load, as (image lb, gradient row li, pixel block lj),
  // advanced one chunk per load (no divisions in the loop)
  int lj = q0 % p.jb, li = (q0 / p.jb) % p.Hg, lb = q0 / (p.jb * p.Hg);
  float ra[kPF][16], rb[kPF][8];
  auto load = [&](float (&a)[16], float (&bv)[8]) {
    const int j0 = lj * kKC;
    const float *xr = xt + lb * ximg + (size_t)li * p.W + j0;
    const int ii = p.conv ? p.Hg - 1 - li : li;
    const float *gr = gt + lb * gimg + (size_t)ii * p.Wg;
    if (j0 + kKC <= p.Wg) {
#pragma unroll
      for (int e = 0; e < 16; ++e) a[e] = mvalid ? __ldg(xr + e) : 0.0f;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int j = j0 + kq + e;
        bv[e] = nvalid ? __ldg(gr + (p.conv ? p.Wg - 1 - j : j)) : 0.0f;
      }
    } else {
#pragma unroll
      for (int e = 0; e < 16; ++e) a[e] = (mvalid && j0 + khalf * 16 + e < p.Wg) ? __ldg(xr + e) : 0.0f;
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        const int j = j0 + kq + e;
        bv[e] = (nvalid && j < p.Wg) ? __ldg(gr + (p.conv ? p.Wg - 1 - j : j)) : 0.0f;
      }
    }
    if (++lj == p.jb) {
      lj = 0;
      if (++li == p.Hg) {
        li = 0;
        ++lb;
      }
    }
  };

  const uint32_t acc = tmem;                  // [hh | small], 2 * NT columns
  const uint32_t a_col0 = tmem + 2u * kNT;    // stage st: hi words at + 32 st, lo words at + 16
  const uint32_t lane_base = (uint32_t)((warp & 3) * 32) << 16;
  const uint32_t idesc_n = idesc_bf16_f32(kMT, p.NT), idesc_2n = idesc_bf16_f32(kMT, 2 * p.NT);
  bool failed = false;
#pragma unroll
  for (int u = 0; u < kPF; ++u)
    if (q0 + u < q1) load(ra[u], rb[u]);
  for (int qb = q0; qb < q1 && !failed; qb += kPF) {
#pragma unroll
    for (int u = 0; u < kPF; ++u) {
      const int q = qb + u;
      if (q >= q1) break;
      const int t = q - q0, st = t % kStages;
      if (t >= kStages && !mbar_wait(&empty[st], ((t / kStages) - 1) & 1, p.err)) failed = true;
      // the CTA agrees on a timeout once per kStages chunks (a late stop only
      // spoils results that the device status already reports as failed)
      if (st == 0 && __syncthreads_or(failed)) {
        failed = true;
        break;
      }
      // A: this thread's 16 values of row m -> 8 hi and 8 lo words
      uint32_t hi[8], lo[8];
#pragma unroll
      for (int e = 0; e < 8; ++e) split_bf16x2(ra[u][2 * e], ra[u][2 * e + 1], hi[e], lo[e]);
      const uint32_t acol = a_col0 + 32u * st + 8u * khalf + lane_base;
      tmem_st8(acol, hi);
      tmem_st8(acol + 16, lo);
      // B: this thread's 8 values of row n -> the hi and lo images of the stage
      uint8_t *bst = smem + (size_t)st * stage_bytes;
      if (n < p.NT) {
        uint32_t bh[4], bl[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) split_bf16x2(rb[u][2 * e], rb[u][2 * e + 1], bh[e], bl[e]);
        const uint32_t off = b_offset(n, kq);
        *reinterpret_cast<uint4 *>(bst + off) = make_uint4(bh[0], bh[1], bh[2], bh[3]);
        *reinterpret_cast<uint4 *>(bst + (size_t)p.NT * kKC * 2 + off) = make_uint4(bl[0], bl[1], bl[2], bl[3]);
      }
      if (q + kPF < q1) load(ra[u], rb[u]);  // kPF chunks ahead
      // this warp's part of the chunk is in place: tensor-memory stores done,
      // shared-memory stores visible to the tensor core's (async) proxy
      tc_wait_st();
      fence_proxy_async_smem();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&full[st]);
      if (tid == 0) {
        const bool ready = mbar_wait(&full[st], (t / kStages) & 1, p.err);
        if (!ready) failed = true;
        tc_fence_after();
        if (ready) {
#pragma unroll
          for (int ks = 0; ks < kKC / 16; ++ks) {
            const uint64_t dh = smem_desc_kmajor(smem_u32(bst) + 256u * ks, 128, 512);
            const uint32_t ah = a_col0 + 32u * st + 8u * ks;
            mma_bf16_ts(acc, ah, dh, idesc_2n, (t > 0 || ks > 0) ? 1u : 0u);  // [hi*hi | hi*lo]
            mma_bf16_ts(acc + p.NT, ah + 16, dh, idesc_n, 1u);                // small half += lo*hi
          }
        }
        tc_commit(&empty[st]);  // frees the stage once the MMAs issued so far are done
      }
    }
  }
  // every MMA issued has retired before the accumulator is read or freed
  if (tid == 0) tc_commit(&done);
  if (!mbar_wait(&done, 0, p.err)) failed = true;
  tc_fence_after();
  if (__syncthreads_or(failed)) failed = true;
  if (!failed && warp < 4 && q0 < q1) {
    float *dst = p.part + ((size_t)split * p.Lpad + nb * kNT) * p.Mpad + mt * kMT + m;
    for (int c0 = 0; c0 < p.NT; c0 += 16) {
      uint32_t v[16], v2[16];
      tmem_ld16(acc + lane_base + c0, v);
      tmem_ld16(acc + lane_base + p.NT + c0, v2);
      tc_wait_ld();
#pragma unroll
      for (int k = 0; k < 16; ++k) dst[(size_t)(c0 + k) * p.Mpad] = __uint_as_float(v[k]) + __uint_as_float(v2[k]);
    }
  } else if (!failed && warp < 4) {
    // an empty chunk range (more splits than chunks) contributes zeros
    float *dst = p.part + ((size_t)split * p.Lpad + nb * kNT) * p.Mpad + mt * kMT + m;
    for (int k = 0; k < p.NT; ++k) dst[(size_t)k * p.Mpad] = 0.0f;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

// out[l*C + c](r, s) = sum over splits, in split order, of the partial sums.
__global__ void fa_tc_reduce(const __grid_constant__ FaTcParams p, float *__restrict__ y) {
  grid_dependency_wait();
  const long long total = (long long)p.L * p.M;
  for (long long o = (long long)blockIdx.x * blockDim.x + threadIdx.x; o < total;
       o += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(o / p.M), mg = (int)(o - (long long)l * p.M);
    float sum = 0.0f;
    for (int sp = 0; sp < p.splits; ++sp) sum += p.part[((size_t)sp * p.Lpad + l) * p.Mpad + mg];
    y[o] = sum;  // plane l*C + c, pixel (r, s): o = l*M + (c*OH + r)*OW + s
  }
}

FaTcParams make_params(const ConvGeom &g, int sms) {
  FaTcParams p{};
  p.Hg = g.R;
  p.Wg = g.S;
  p.OH = g.OH;
  p.OW = g.OW;
  p.H = g.H;
  p.W = g.W;
  p.C = g.n;
  p.L = g.groups;
  p.B = g.batch;
  p.conv = g.orient == CCT_CONVOLUTION;
  p.M = p.C * p.OH * p.OW;
  p.mtiles = (p.M + kMT - 1) / kMT;
  p.Mpad = p.mtiles * kMT;
  p.NT = std::min(kNT, ((p.L + 15) / 16) * 16);
  p.nblocks = (p.L + kNT - 1) / kNT;
  p.Lpad = p.nblocks * kNT;
  p.jb = (p.Wg + kKC - 1) / kKC;
  p.nch = p.B * p.Hg * p.jb;
  const int tiles = p.mtiles * p.nblocks;
  int splits = (2 * sms) / tiles;  // two CTAs per SM: one wave
  splits = std::max(1, std::min(splits, p.nch));
  p.splits = splits;
  return p;
}

}  // namespace

bool fa_tc_supported(const ConvGeom &g) {
  if (g.mode != CCT_FILTER_ADJOINT_BLOCK_REDUCE_SUM) return false;
  if (g.border != CCT_BORDER_VALID || g.down != 1 || g.up != 1 || g.fup != 1) return false;
  // the image rows r + i and columns s + j stay inside the plane by construction
  const long long M = (long long)g.n * g.OH * g.OW;
  return M >= 1 && M <= (1 << 24) && g.groups >= 1 && (long long)g.batch * g.R <= (1 << 26);
}

size_t fa_tc_workspace_bytes(const ConvGeom &g, int sms) {
  const FaTcParams p = make_params(g, sms);
  return (size_t)p.splits * p.Lpad * p.Mpad * sizeof(float);
}

int launch_fa_tc(const ConvGeom &g, const float *x, const float *f, float *y, float *work, unsigned *err,
                 cudaStream_t st) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  FaTcParams p = make_params(g, sms);
  p.x = x;
  p.g = f;
  p.part = work;
  p.err = err;
  if (!work) return set_error(CCT_EINVAL, "tensor-core FilterAdjoint needs plan workspace");
  const long long grid = (long long)p.mtiles * p.nblocks * p.splits;
  if (grid > 0x7fffffffLL) return set_error(CCT_ENOTSUP, "FilterAdjoint grid too large");
  // the stages need kStages * 2 * NT * 32 bf16 (32 KB at most); asking for 96 KB keeps
  // at most two CTAs on an SM, so their tensor memory (256 columns each)
  // always fits and no allocation waits
  const size_t smem = 96 * 1024;
  static_assert(kStages * 2u * kNT * kKC * 2 <= 96 * 1024, "FilterAdjoint stages");
  static_assert(2 * kNT + kStages * kKC <= kTmemCols, "FilterAdjoint tensor memory");
  int rc = check_cuda(cudaFuncSetAttribute(fa_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                      "cudaFuncSetAttribute(fa_tc)");
  if (rc) return rc;
  rc = launch_pdl(fa_tc_kernel, dim3((unsigned)grid), dim3(kFaThreads), smem, st, "fa_tc_kernel launch", p);
  if (rc) return rc;
  const long long total = (long long)p.L * p.M;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 8);
  rc = launch_pdl(fa_tc_reduce, dim3(blocks), dim3(256), 0, st, "fa_tc_reduce launch", p, y);
  if (rc) return rc;
  count_launches(2);
  return CCT_OK;
}

}  // namespace cct
