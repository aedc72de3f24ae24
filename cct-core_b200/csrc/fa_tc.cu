// FilterAdjointBlockReduceSum (the weight gradient) on the tcgen05 tensor
// cores in split-BF16 precision, for the shapes fa_f32 serves (BorderValid,
// no sampling):
//   out[l*C + c](r, s) = sum_b sum_(i,j) x[b*C + c](r + i, s + j) * g'[b*L + l](i, j)
// (ConvolveHyperKernel.scala:187, 333, 575-590; CogFunctionAPI.scala:1480-1511;
// g' = g flipped for convolveFilterAdjoint).  Two forms:
// - the gradient-planes form (fa_bank_kernel, below): gradient planes as the
//   MMA rows, (result row, image plane) as the columns, one accumulator per
//   result column; taken when the rows suit TMA and OH * CB <= 160;
// - the im2col form (fa_tc_kernel) for the other shapes:
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

// ---------------------------------------------------------------------------
// Gradient-planes form (fa_bank_kernel), used when the rows suit TMA (widths
// multiples of 4, 16-byte aligned fields) and a result row block fits:
// OH * CB <= 160 accumulator columns for a plane block CB of 8..64.
//
// For a result column s the reduction over gradient columns j reads image
// column j + s, so with s fixed:
//   D_s[l][(r, c)] = sum_(b, i, j) g'[b*L + l](i, j) * x[b*C + c](r + i, s + j)
// is a GEMM with rows m = gradient plane l (64 per block), columns
// n = (result row r, image plane c) and the reduction k = (b, i, j).  A
// reduction chunk is 16 gradient columns j0..j0+15 of gradient row i of image
// b.  Its B operand is the image rows i..i+OH-1 at columns j0+s..: OH
// consecutive [CB planes][16 columns] row tiles, so one stage's B is a run of
// image-row tiles that every chunk of the stage reads at its own offset, and
// the gradient (A) is converted once per chunk for two result columns (a CTA
// serves the columns s0 and s0 + 1, one accumulator each).
// Split BF16: a chunk's A1 (tensor memory) holds Gh in rows 0-63 and Gl in
// rows 64-127, A2 the same halves swapped; A1 x Xh + A2 x Xl leaves
// Gh*Xh + Gl*Xl in accumulator rows 0-63 and Gl*Xh + Gh*Xl in rows 64-127,
// added after the reduction, so the small products never meet the large sum
// in the tensor core's accumulation.  Rows of planes past L and columns of
// planes past C hold other images' data (finite values) and are never
// stored; gradient columns outside 0..Wg-1 come from TMA's zero fill.
//
// Warps 0-15 convert (fp32 staging -> A in tensor memory, B in shared
// memory), warps 16 and 17 issue the MMAs of the first and second result
// column (one issuing thread could not keep the tensor core fed: ~110
// cycles an MMA against its 80 of work), warp 18 issues the TMA loads of the
// fp32 staging: a gradient box [20 columns][5 rows][64 planes] and an image box
// [20 columns][xrows][CB planes], three stages deep (a box took ~3k cycles
// to land).  Their plane pitches are odd numbers of 16-byte units, so the
// converters' float4 reads are conflict-free.  B
// layout: [k group][row tile][8-row group][8 rows][16 B], 8-row groups
// adjacent, which the tensor core reads at its full rate.  Each CTA reduces
// a contiguous range of chunks, adds its two row halves and stores its
// partial sums; fa_bank_reduce adds them in a fixed order.
constexpr int kFbConvWarps = 16;
constexpr int kFbConvThreads = 32 * kFbConvWarps;
constexpr int kFbMmaWarp = 16;                  // and 17: one issuing thread per result column
constexpr int kFbLoadWarp = 18;
constexpr int kFbThreads = 32 * 19;
constexpr int kFbChunks = 5;                    // chunks per stage
constexpr int kFbStg = 3;                       // fp32 staging slots: a load has two stages to land
constexpr int kFbGCols = 20, kFbGRows = 5;      // gradient box (odd plane pitch in 16-byte units)
constexpr int kFbXCols = 20;                    // image box columns: s0 % 4 + 1 + 15 < 20
constexpr int kFbLB = 64;                       // gradient planes per block
constexpr int kFbMaxN = 160;                    // accumulator columns per result column
constexpr int kFbAcol = 2 * kFbMaxN;            // first A column in tensor memory
constexpr uint32_t kFbGBytes = kFbGCols * kFbGRows * kFbLB * 4;
static_assert(kFbAcol + 2 * kFbChunks * 16 <= 512, "fa_bank tensor memory");
static_assert(kFbGRows >= kFbChunks && (kFbGCols / 4 * kFbGRows) % 2 == 1, "fa_bank gradient box");

struct FaBankParams {
  int H, W, Hg, Wg, OH, OW, C, L, B;
  int CB, cb_log2, N, xrows, rows_max, cblocks, lblocks, JB, nch;
  int npairs, P, Q, NS;  // column pairs; splits of a pair, of the lone column (odd OW); max(P, Q)
  uint32_t kg_bytes, term_bytes, bop_bytes, xbox_bytes, stg_bytes;
  size_t smem;
  float *part;  // [OW][C][OH][NS][lblocks*64]
  unsigned *err;
};

struct FbStage {
  int b, jb, i, n;
};

__device__ __forceinline__ FbStage fb_stage(const FaBankParams &p, int q, int q1) {
  FbStage st;
  const int t = q / p.Hg;
  st.i = q - t * p.Hg;
  st.jb = t % p.JB;
  st.b = t / p.JB;
  st.n = min(min(kFbChunks, q1 - q), p.Hg - st.i);
  return st;
}

// B: image row tiles t < nrows; item (t, kg, c) with c fastest (a
// quarter-warp reads 8 planes: conflict-free, and writes 128 contiguous
// bytes); one 16-byte core row of each term for each result column, from
// box column 8*kg + D + sh (D = s0 % 4, uniform).
template <int D>
__device__ __forceinline__ void fb_convert_b(const FaBankParams &p, const float *xbox, uint8_t *bbase, int nitems,
                                             int nsh, int tid) {
  for (int it = tid; it < nitems; it += kFbConvThreads) {
    const int c = it & (p.CB - 1), tk = it >> p.cb_log2;
    const int kg = tk & 1, t = tk >> 1;
    const float4 *src = reinterpret_cast<const float4 *>(xbox + ((size_t)c * p.xrows + t) * kFbXCols + 8 * kg);
    float w[12];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const float4 t4 = src[v];
      w[4 * v] = t4.x;
      w[4 * v + 1] = t4.y;
      w[4 * v + 2] = t4.z;
      w[4 * v + 3] = t4.w;
    }
    uint8_t *dst = bbase + (uint32_t)kg * p.kg_bytes + ((uint32_t)t * p.CB + c) * 16;
#pragma unroll
    for (int sh = 0; sh < 2; ++sh) {
      if (sh < nsh) {
        uint32_t h[4], l[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) split_bf16x2(w[D + sh + 2 * v], w[D + sh + 2 * v + 1], h[v], l[v]);
        uint8_t *d = dst + (size_t)(2 * sh) * p.term_bytes;
        *reinterpret_cast<uint4 *>(d) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4 *>(d + p.term_bytes) = make_uint4(l[0], l[1], l[2], l[3]);
      }
    }
  }
}

template <bool CONV>
__global__ void __launch_bounds__(kFbThreads, 1)
    fa_bank_kernel(const __grid_constant__ FaBankParams p, const __grid_constant__ CUtensorMap gmap,
                   const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap omap) {
  // 3 fp32 staging slots [gradient box | image box], then 2 B operand slots
  // [result column][hi | lo][k group][row tiles]
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t fp_full[kFbStg], fp_empty[kFbStg], op_full[2], op_empty[2], done;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  // CTA: (plane block, gradient block, result-column group, split); group g
  // serves columns 2g and 2g + 1 with P splits, or (odd OW) the last column
  // alone with Q splits
  int bid = blockIdx.x;
  const int per_cl = p.npairs * p.P + p.Q;
  const int e = bid % per_cl;
  bid /= per_cl;
  const int cblk = bid % p.cblocks, lblk = bid / p.cblocks;
  const int grp = e < p.npairs * p.P ? e / p.P : p.npairs, sp = e - grp * p.P;
  const int s0 = 2 * grp, nsh = min(2, p.OW - s0);
  const int nsplit = grp < p.npairs ? p.P : p.Q;
  const int q0 = (int)((long long)sp * p.nch / nsplit), q1 = (int)((long long)(sp + 1) * p.nch / nsplit);

  if (threadIdx.x == 0) {
    for (int k = 0; k < kFbStg; ++k) {
      mbar_init(&fp_full[k], 1);              // loader expect_tx
      mbar_init(&fp_empty[k], kFbConvWarps);  // one arrival per converter warp
    }
    for (int k = 0; k < 2; ++k) {
      mbar_init(&op_full[k], kFbConvWarps);
      mbar_init(&op_empty[k], 2);             // both issuers' commits
    }
    mbar_init(&done, 2);
    abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == kFbMmaWarp) tmem_alloc(&tmem_slot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  grid_dependency_wait();  // launched with programmatic serialisation: global memory only after this
  allow_dependent_launch();
  volatile int *abort = &abort_flag;
  uint8_t *ops = smem + kFbStg * (size_t)p.stg_bytes;
  bool failed = false;

  if (warp < kFbConvWarps) {
    // ------------------------------------------------------------ converters
    const int quarter = warp & 3, par = warp >> 2;  // lane quarter, chunk phase (0-3)
    const int lloc = (quarter & 1) * 32 + lane, half = quarter >> 1;
    const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
    const int dsh = s0 & 3;  // image box column of result column s0 at gradient column j0
    int u = 0;
    for (int q = q0; q < q1; ++u) {
      const FbStage st = fb_stage(p, q, q1);
      const int slot = u & 1, sslot = u % kFbStg;
      const uint32_t ph = (uint32_t)(u >> 1) & 1;
      if (*abort || !mbar_wait(&fp_full[sslot], (uint32_t)(u / kFbStg) & 1, p.err) ||
          (u >= 2 && !mbar_wait(&op_empty[slot], ph ^ 1, p.err))) {
        failed = true;
        break;
      }
      const uint8_t *stg = smem + (size_t)sslot * p.stg_bytes;
      // A: chunks par, par + 4 of the stage, this lane's gradient plane.  The
      // box row of gradient row i + k is k (convolution: the box starts at row
      // Hg - i - 5 and column Wg - 16 - j0, read backwards: row 4 - k, column 15 - kk)
      for (int k = par; k < st.n; k += 4) {
        const float4 *src = reinterpret_cast<const float4 *>(stg) +
                            ((size_t)lloc * kFbGRows + (CONV ? kFbGRows - 1 - k : k)) * (kFbGCols / 4);
        float v[16];
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          const float4 t = src[w];
          if (CONV) {
            v[15 - 4 * w] = t.x;
            v[14 - 4 * w] = t.y;
            v[13 - 4 * w] = t.z;
            v[12 - 4 * w] = t.w;
          } else {
            v[4 * w] = t.x;
            v[4 * w + 1] = t.y;
            v[4 * w + 2] = t.z;
            v[4 * w + 3] = t.w;
          }
        }
        uint32_t hi[8], lo[8];
#pragma unroll
        for (int w = 0; w < 8; ++w) split_bf16x2(v[2 * w], v[2 * w + 1], hi[w], lo[w]);
        const uint32_t a1 = tmem + lane_base + kFbAcol + (uint32_t)(slot * kFbChunks + k) * 16;
        if (half == 0) {
          tmem_st8(a1, hi);
          tmem_st8(a1 + 8, lo);
        } else {
          tmem_st8(a1, lo);
          tmem_st8(a1 + 8, hi);
        }
      }
      const float *xbox = reinterpret_cast<const float *>(stg + kFbGBytes);
      uint8_t *opb = ops + (size_t)slot * p.bop_bytes;
      const int nitems = (st.n + p.OH - 1) * 2 * p.CB;
      switch (dsh) {
        case 0: fb_convert_b<0>(p, xbox, opb, nitems, nsh, threadIdx.x); break;
        case 1: fb_convert_b<1>(p, xbox, opb, nitems, nsh, threadIdx.x); break;
        case 2: fb_convert_b<2>(p, xbox, opb, nitems, nsh, threadIdx.x); break;
        default: fb_convert_b<3>(p, xbox, opb, nitems, nsh, threadIdx.x); break;
      }
      // the tensor core reads A (tensor memory) and B (async proxy)
      tc_wait_st();
      fence_proxy_async_smem();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) {
        mbar_arrive(&fp_empty[sslot]);
        mbar_arrive(&op_full[slot]);
      }
      q += st.n;
    }
    if (failed) *abort = 1;
    // -------------------------------------------------------------- epilogue
    // The CTA's partial sums are assembled in shared memory (idle now: every
    // load was consumed and every MMA has retired) as TMA store boxes
    // [result column][CB * OH (plane, row)][64 planes l]: the warps holding
    // rows 0-63 (Gh*Xh + Gl*Xl) and those holding rows 64-127 (the small
    // products) write two copies at once, all warps add them (float4), and
    // one thread stores each column's box.
    bool bad = failed || *abort != 0;
    if (!bad) bad = !mbar_wait(&done, 0, p.err);
    bad = named_sync_or(1, kFbConvThreads, bad);
    const int box_floats = p.CB * p.OH * kFbLB;
    float *obox = reinterpret_cast<float *>(smem);               // rows 0-63, then the sums
    float *sbox = obox + (size_t)2 * box_floats;                 // rows 64-127
    if (!bad) {
      tc_fence_after();
      float *mine = half ? sbox : obox;
      const int stride = p.OH * kFbLB;  // between planes c and c + 1 of one result row r
      for (int sh = 0; sh < nsh; ++sh) {
        for (int c0 = par * 16; c0 < p.N; c0 += 64) {
          uint32_t v[16];
          tmem_ld16(tmem + lane_base + (uint32_t)(sh * p.N + c0), v);
          tc_wait_ld();
          // columns n = c0..c0+15 = (r, c): box row c * OH + r; an empty chunk
          // range (more splits than chunks) contributes zeros
          float *o = mine + (size_t)sh * box_floats + lloc;
          if (p.CB >= 16) {  // one result row per 16 columns
            float *ob = o + ((size_t)(c0 & (p.CB - 1)) * p.OH + (c0 >> p.cb_log2)) * kFbLB;
#pragma unroll
            for (int k = 0; k < 16; ++k) ob[k * stride] = q0 < q1 ? __uint_as_float(v[k]) : 0.0f;
          } else {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
              const int n = c0 + k;
              o[((size_t)(n & (p.CB - 1)) * p.OH + (n >> p.cb_log2)) * kFbLB] = q0 < q1 ? __uint_as_float(v[k]) : 0.0f;
            }
          }
        }
      }
    }
    named_sync(1, kFbConvThreads);
    if (!bad) {
      float4 *o4 = reinterpret_cast<float4 *>(obox);
      const float4 *s4 = reinterpret_cast<const float4 *>(sbox);
      for (int i = threadIdx.x; i < nsh * box_floats / 4; i += kFbConvThreads) {
        float4 a = o4[i];
        const float4 b = s4[i];
        a.x += b.x;
        a.y += b.y;
        a.z += b.z;
        a.w += b.w;
        o4[i] = a;
      }
      fence_proxy_async_smem();  // the box is read by the async proxy (TMA store)
    }
    named_sync(1, kFbConvThreads);
    if (!bad && warp == 0) {
      if (lane == 0) {
        for (int sh = 0; sh < nsh; ++sh)
          tma_store_4d(&omap, obox + (size_t)sh * box_floats, lblk * kFbLB, sp, cblk * p.CB * p.OH, s0 + sh);
        bulk_commit_group();
        // the shared memory must stay valid until the stores have read it;
        // their global writes are part of this grid's completion, which the
        // reduce kernel's grid_dependency_wait() (and stream order) waits for
        bulk_wait_group_read0();
      }
      __syncwarp();
    }
  } else if (warp == kFbMmaWarp || warp == kFbMmaWarp + 1) {
    // ------------------------------------------------------------ MMA issuers
    // warp 16: result column s0 (accumulator at column 0), warp 17: s0 + 1
    // (at column N), if the CTA has it; both commit every stage
    const int sh = warp - kFbMmaWarp;
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(128, p.N);
      const uint64_t bt = smem_desc_kmajor(0, p.kg_bytes, 128);
      const uint32_t b_hi = (uint32_t)(bt >> 32), b_lo = (uint32_t)bt;
      // The issuing thread's own latency bounds the MMA rate, so the loop
      // keeps running 32-bit descriptor words and no per-MMA branching.
      const uint32_t ops16 = smem_u32(ops) >> 4;
      const uint32_t cb16 = (uint32_t)p.CB, term16 = p.term_bytes >> 4;  // a row tile: CB rows of 16 bytes
      const uint32_t d = tmem + (uint32_t)(sh * p.N);
      const bool mine = sh < nsh;
      uint32_t acc = 0;
      int u = 0;
      for (int q = q0; q < q1; ++u) {
        const FbStage st = fb_stage(p, q, q1);
        const int slot = u & 1;
        if (*abort || !mbar_wait(&op_full[slot], (uint32_t)(u >> 1) & 1, p.err)) {
          failed = true;
          break;
        }
        tc_fence_after();
        if (mine) {
          uint32_t a1 = tmem + kFbAcol + (uint32_t)(slot * kFbChunks) * 16;
          uint32_t bw = b_lo + ops16 + ((uint32_t)slot * p.bop_bytes >> 4) + 2u * sh * term16;
          for (int k = 0; k < st.n; ++k, a1 += 16, bw += cb16) {
            mma_bf16_ts(d, a1, desc_word(b_hi, bw), idesc, acc);
            mma_bf16_ts(d, a1 + 8, desc_word(b_hi, bw + term16), idesc, 1u);
            acc = 1u;
          }
        }
        tc_commit(&op_empty[slot]);  // frees the stage once its MMAs are done
        q += st.n;
      }
      tc_commit(&done);
      if (failed) *abort = 1;
      mbar_wait(&done, 0, p.err);  // every MMA retired before the tensor memory is freed
    }
    __syncwarp();
  } else if (warp == kFbLoadWarp) {
    // --------------------------------------------------------------- loader
    if (lane == 0) {
      int u = 0;
      for (int q = q0; q < q1; ++u) {
        const FbStage st = fb_stage(p, q, q1);
        const int sslot = u % kFbStg;
        if (*abort ||
            (u >= kFbStg && !mbar_wait(&fp_empty[sslot], ((uint32_t)(u / kFbStg) & 1) ^ 1, p.err))) {
          *abort = 1;
          break;
        }
        uint8_t *gdst = smem + (size_t)sslot * p.stg_bytes;
        const int j0 = st.jb * 16;
        mbar_arrive_expect_tx(&fp_full[sslot], kFbGBytes + p.xbox_bytes);
        tma_load_3d(gdst, &gmap, &fp_full[sslot], CONV ? p.Wg - 16 - j0 : j0, CONV ? p.Hg - st.i - kFbGRows : st.i,
                    st.b * p.L + lblk * kFbLB);
        tma_load_3d(gdst + kFbGBytes, &xmap, &fp_full[sslot], j0 + (s0 & ~3), st.i, st.b * p.C + cblk * p.CB);
        q += st.n;
      }
    }
    __syncwarp();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kFbMmaWarp) tmem_dealloc(tmem, 512);
}

// out[l*C + c](r, s) = the CTAs' partial sums for (s, c, r, l) in a fixed
// order.  A block of 128 threads serves one (s, c, r) and 64 planes, whose
// partial sums are one contiguous run [split][planes]: thread (k, quad) adds
// four planes of the splits k, k + 8, ... in split order (eight loads in
// flight), and one thread per quad adds the eight sums in lane order.
__global__ void __launch_bounds__(128) fa_bank_reduce(const __grid_constant__ FaBankParams p, float *__restrict__ y) {
  __shared__ float4 red[8][16];
  grid_dependency_wait();
  const int Lpad = p.lblocks * kFbLB, quads = Lpad / 4;
  const int quad16 = threadIdx.x & 15, k = threadIdx.x >> 4;
  const int nblk = p.OW * p.C * p.OH * p.lblocks;
  for (int bi = blockIdx.x; bi < nblk; bi += gridDim.x) {
    const int lb = bi % p.lblocks, scr = bi / p.lblocks;  // scr = (s * C + c) * OH + r
    const int s = scr / (p.C * p.OH);
    const int nsplit = s / 2 < p.npairs ? p.P : p.Q;
    const float4 *q = reinterpret_cast<const float4 *>(p.part + (size_t)scr * p.NS * Lpad) + lb * 16 + quad16;
    float4 acc = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (int base = k; base < nsplit; base += 64) {
      float4 v[8];
#pragma unroll
      for (int j = 0; j < 8; ++j)
        v[j] = base + 8 * j < nsplit ? q[(size_t)(base + 8 * j) * quads] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        acc.x += v[j].x;
        acc.y += v[j].y;
        acc.z += v[j].z;
        acc.w += v[j].w;
      }
    }
    red[k][quad16] = acc;
    __syncthreads();
    if (threadIdx.x < 16) {
      float4 t = red[0][threadIdx.x];
#pragma unroll
      for (int kk = 1; kk < 8; ++kk) {
        const float4 u = red[kk][threadIdx.x];
        t.x += u.x;
        t.y += u.y;
        t.z += u.z;
        t.w += u.w;
      }
      const int cr = scr - s * p.C * p.OH, c = cr / p.OH, r = cr - c * p.OH;
      const int l0 = lb * kFbLB + 4 * threadIdx.x;
      const size_t plane = (size_t)p.C * p.OH * p.OW;
      float *o = y + ((size_t)l0 * p.C + c) * p.OH * p.OW + (size_t)r * p.OW + s;
      if (l0 < p.L) o[0] = t.x;
      if (l0 + 1 < p.L) o[plane] = t.y;
      if (l0 + 2 < p.L) o[2 * plane] = t.z;
      if (l0 + 3 < p.L) o[3 * plane] = t.w;
    }
    __syncthreads();
  }
}

// The gradient-planes form's plan, or false when the shape does not suit it.
bool make_bank_params(const ConvGeom &g, int sms, FaBankParams *out) {
  FaBankParams p{};
  p.Hg = g.R;
  p.Wg = g.S;
  p.OH = g.OH;
  p.OW = g.OW;
  p.H = g.H;
  p.W = g.W;
  p.C = g.n;
  p.L = g.groups;
  p.B = g.batch;
  if ((p.W & 3) || (p.Wg & 3) || p.OH < 1 || p.OW < 1 || p.L < 1 || p.C < 1) return false;
  const size_t budget = 225 * 1024;
  // plane block (a power of two): the fewest blocks, then the smallest block
  bool found = false;
  int best_blocks = 0;
  for (int lg = 3; lg <= 6; ++lg) {
    const int cb = 1 << lg;
    if (cb * p.OH > kFbMaxN || (cb * p.OH) % 16) continue;
    const int rows_max = kFbChunks + p.OH - 1;
    const int xrows = rows_max | 1;  // odd: the image staging's plane pitch is an odd number of 16-byte units
    const uint32_t xbox = (uint32_t)kFbXCols * xrows * cb * 4;
    const uint32_t stg = kFbGBytes + xbox;  // gradient box + image box
    const uint32_t kgb = (uint32_t)rows_max * cb * 16;  // one k group of a term's row tiles
    const uint32_t term = 2 * kgb;
    const uint32_t bop = 4 * term;                      // two result columns x (hi, lo)
    const size_t smem = kFbStg * (size_t)stg + 2 * (size_t)bop;
    // the epilogue's boxes (two copies of two columns x N x 64 planes) reuse the staging and operands
    if (smem > budget || (size_t)4 * cb * p.OH * 64 * 4 > smem) continue;
    const int nb = (p.C + cb - 1) / cb;
    if (found && nb >= best_blocks) continue;
    found = true;
    best_blocks = nb;
    p.CB = cb;
    p.cb_log2 = lg;
    p.N = cb * p.OH;
    p.rows_max = rows_max;
    p.xrows = xrows;
    p.xbox_bytes = xbox;
    p.stg_bytes = stg;
    p.kg_bytes = kgb;
    p.term_bytes = term;
    p.bop_bytes = bop;
    p.smem = smem;
  }
  if (!found || p.xrows > 256) return false;
  p.cblocks = best_blocks;
  p.lblocks = (p.L + kFbLB - 1) / kFbLB;
  p.JB = (p.Wg + 15) / 16;
  const long long nch = (long long)p.B * p.JB * p.Hg;
  if (nch < 1 || nch > 0x3fffffffLL) return false;
  p.nch = (int)nch;
  // Splits: one wave of CTAs.  A lone column's CTA converts and stages as
  // much per chunk as a pair's for about 0.8 of its time (measured: 455
  // against 574 cycles a chunk), so it gets 0.8 as many splits and every
  // CTA has about the same work.
  const long long cl = (long long)p.cblocks * p.lblocks;
  p.npairs = p.OW / 2;
  const bool lone = (p.OW & 1) != 0;
  const long long per_cl = std::max(1LL, sms / cl);
  if (p.npairs == 0) {
    p.P = 1;
    p.Q = (int)std::min<long long>(per_cl, p.nch);
  } else {
    p.P = (int)std::max(1LL, std::min<long long>((long long)(per_cl / (p.npairs + (lone ? 0.8 : 0.0))), p.nch));
    p.Q = lone ? std::max(1, (int)(0.8 * p.P + 0.5)) : 0;
  }
  p.NS = std::max(p.P, p.Q);
  if (cl * (p.npairs * p.P + p.Q) > 0x7fffffffLL ||
      (long long)p.OW * p.C * p.OH * p.lblocks * kFbLB * p.NS > 0x7fffffffLL)
    return false;
  // more than 160 KB keeps one CTA per SM: its 512 tensor-memory columns are free
  p.smem = std::max(p.smem, (size_t)160 * 1024);
  *out = p;
  return true;
}

size_t bank_workspace_bytes(const FaBankParams &p) {
  return (size_t)p.NS * p.OW * p.C * p.OH * p.lblocks * kFbLB * sizeof(float);
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
  size_t bytes = (size_t)p.splits * p.Lpad * p.Mpad * sizeof(float);
  FaBankParams bp;
  if (make_bank_params(g, sms, &bp)) bytes = std::max(bytes, bank_workspace_bytes(bp));
  return bytes;
}

namespace {

int launch_fa_bank(FaBankParams p, bool conv, const float *x, const float *f, float *y, cudaStream_t st) {
  CUtensorMap gmap, xmap;
  int rc = encode_tensor_map_3d_box(&gmap, f, (uint64_t)p.Wg, (uint64_t)p.Hg, (uint64_t)p.B * p.L, kFbGCols,
                                    kFbGRows, kFbLB);
  if (rc) return rc;
  rc = encode_tensor_map_3d_box(&xmap, x, (uint64_t)p.W, (uint64_t)p.H, (uint64_t)p.B * p.C, kFbXCols,
                                (uint32_t)p.xrows, (uint32_t)p.CB);
  if (rc) return rc;
  // partial sums [OW][C*OH][NS][Lpad]: a CTA stores [1][CB*OH][1][64] boxes
  CUtensorMap omap;
  const uint64_t Lpad = (uint64_t)p.lblocks * kFbLB;
  const uint64_t odims[4] = {Lpad, (uint64_t)p.NS, (uint64_t)p.C * p.OH, (uint64_t)p.OW};
  const uint64_t ostr[3] = {Lpad * 4, Lpad * p.NS * 4, Lpad * p.NS * p.C * p.OH * 4};
  const uint32_t obox[4] = {(uint32_t)kFbLB, 1, (uint32_t)(p.CB * p.OH), 1};
  rc = encode_tensor_map_f32(&omap, p.part, 4, odims, ostr, obox);
  if (rc) return rc;
  auto kern = conv ? fa_bank_kernel<true> : fa_bank_kernel<false>;
  rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem),
                  "cudaFuncSetAttribute(fa_bank)");
  if (rc) return rc;
  const long long grid = (long long)p.cblocks * p.lblocks * (p.npairs * p.P + p.Q);
  rc = launch_pdl(kern, dim3((unsigned)grid), dim3(kFbThreads), p.smem, st, "fa_bank_kernel launch", p, gmap, xmap,
                  omap);
  if (rc) return rc;
  const long long nblk = (long long)p.OW * p.C * p.OH * p.lblocks;  // < 2^31: the plan checks it
  const int blocks = (int)std::min<long long>(nblk, 148LL * 16);
  rc = launch_pdl(fa_bank_reduce, dim3(blocks), dim3(128), 0, st, "fa_bank_reduce launch", p, y);
  if (rc) return rc;
  count_launches(2);
  return CCT_OK;
}

}  // namespace

int launch_fa_tc(const ConvGeom &g, const float *x, const float *f, float *y, float *work, unsigned *err,
                 cudaStream_t st) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (!work) return set_error(CCT_EINVAL, "tensor-core FilterAdjoint needs plan workspace");
  FaBankParams bp;
  // TMA reads both fields: 16-byte aligned bases (row pitches are checked by
  // the plan)
  if (make_bank_params(g, sms, &bp) && (reinterpret_cast<uintptr_t>(x) & 15) == 0 &&
      (reinterpret_cast<uintptr_t>(f) & 15) == 0) {
    bp.part = work;
    bp.err = err;
    return launch_fa_bank(bp, g.orient == CCT_CONVOLUTION, x, f, y, st);
  }
  FaTcParams p = make_params(g, sms);
  p.x = x;
  p.g = f;
  p.part = work;
  p.err = err;
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
