// Fused filter-bank convolution (ProjectFrame / BackProjectFrame with the
// BlockReduceSum fused, ConvolveHyperKernel.scala:153-199, 319-340, 574-645)
// as an implicit GEMM on the tcgen05 tensor cores, in split-BF16 precision:
//   x = xh + xl, f = fh + fl (bf16 hi + bf16 residual), and
//   y = sum xh*fh + xh*fl + xl*fh   accumulated in FP32 in tensor memory.
//
// GEMM view per image b: D[pixel m][filter n] = sum over (plane c, tap r,s)
//   A[m][c,r,s] * B[n][c,r,s],  A = im2col of the input planes, B = filters.
// The reduction walks "chunks": one filter tap x CB input planes.
//
// Warp roles (persistent CTAs, one per SM):
//   warps 0-15 producers, 4 groups of 4 warps (one warp per tensor-memory
//              lane quarter, one output pixel per lane).  Together they
//              split each landed halo block once into bf16 hi/lo; then group
//              j copies, for every chunk q = j (mod 4), the pixel's split
//              words of that tap into the chunk's tensor-memory stage
//              (tcgen05.st, row m = lane m): four chunks are in flight.
//   warp 16    MMA issuer: for filters of kBatchTaps or more taps the warp
//              probes the next 8 chunks at once and issues every ready one in
//              a batch (else one chunk per wait); one elected lane issues,
//              per 16-deep k-step of a chunk, with A from tensor memory and
//              B from shared memory,
//                A_hi x [B_hi; B_lo] (N = 2*NT) into [hh | small], then
//                A_lo x B_hi (N = NT) into the second half, so the two
//                small products never meet the large hi*hi sum (the tensor
//                core's FP32 accumulation would round them against it);
//                the epilogue adds the halves.  The concatenated first MMA
//                reads A_hi once for both products and halves the
//                instruction count (the tensor time is N/2 cycles per MMA
//                either way).  The double-buffered [hh | small]
//                accumulator is 4*NT columns, so NT <= 64.
//   warp 17    loader: 3-D TMA loads of the halo tile (zero fill at the
//              border) and bulk copies of the pre-packed filter chunks; the
//              warp probes the next 8 stages at once and each lane issues the
//              copy of one free stage, so a batch of copies goes out together
//              (one thread looping over them issued one per ~480 cycles);
//              for filters of fewer than kBatchTaps taps one thread issues one
//              copy per loop trip.
//   warps 18-25 epilogue, two per tensor-memory lane quarter taking
//              alternate 16-column blocks: tcgen05.ld of the accumulator,
//              optional ReLU, coalesced stores to the output planes.
// Every mbarrier wait is bounded; on a timeout the CTA raises the device
// error word, lets in-flight copies land, frees its tensor memory and exits.
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>
#include <unordered_map>

#include "cct_internal.h"
#include "frame_tc.h"
#include "sm100_util.cuh"

namespace cct {
namespace {

constexpr int kMT = 128;        // output pixels per tile (MMA M)
constexpr int kStages = 8;      // A/B chunk pipeline depth
constexpr int kGroups = 4;      // producer groups: group j builds chunks q = j (mod kGroups)
constexpr int kProdWarps = 4 * kGroups;
constexpr int kProdThreads = 32 * kProdWarps;
constexpr int kMmaWarp = kProdWarps, kLoadWarp = kProdWarps + 1;  // then the epilogue warps
// Filters of at least this many taps use the batched MMA issuer and the
// warp-wide loader; smaller ones (3x3: 9-chunk blocks) keep one chunk per
// loop trip, which measured faster for them (an eight-layer 3x3 stack: 5.3
// against 6.3 ms per step; 5x5 filter banks: 0.097 against 0.091 ms).
constexpr int kBatchTaps = 16;
constexpr int kEpiWarps = 8;  // two per lane quarter: the last tile's epilogue is the launch's tail
constexpr int kThreads = 32 * (kProdWarps + 2 + kEpiWarps);
static_assert(kStages % kGroups == 0, "a stage must always belong to the same producer group");

// Byte offset of element (n, k) inside one packed K-major operand image of
// rows x CB bf16 (no swizzle): core matrix (8 rows x 8 elements, 128 bytes)
// at (n/8)*SBO + (k/8)*LBO, LBO = 128, SBO = CB*16.
__host__ __device__ inline uint32_t packed_offset(int n, int k, int CB) {
  return (uint32_t)((n >> 3) * (CB * 16) + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2);
}

struct Barriers {
  uint64_t full[kStages], empty[kStages];
  uint64_t hfull[2], hempty[2];
  uint64_t dfull[2], dempty[2];
  uint64_t drain;  // MMA warp: all issued MMAs retired
  uint32_t tmem_slot;
  int abort_flag;
};

template <int CB>
__global__ void __launch_bounds__(kThreads, 1)
    frame_tc_kernel(const __grid_constant__ CUtensorMap xmap, const __grid_constant__ TcParams p) {
  // Shared memory: [landing: fp32 halo block, planes x TR x TC as TMA writes it]
  //                [split:   the same block as packed bf16 hi/lo per position]
  //                [kStages filter-chunk stages]
  // The split layout holds, per halo position, NCH = CB/4 16-byte chunks:
  // chunks 0..CB/8-1 = hi words (bf16x2 of planes 2j, 2j+1), then the lo
  // words.  Chunk k of position pos is stored at chunk slot k ^ (pos % NCH)
  // so that 8 lanes reading 8 consecutive positions hit distinct banks.
  constexpr int NCH = CB / 4;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ Barriers bars;
  const ConvGeom &g = p.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  uint8_t *landing = smem;
  uint8_t *split = smem + p.halo_bytes;
  uint8_t *bstage = smem + 2 * p.halo_bytes;
  const uint32_t bstage_bytes = 2u * p.NT * CB * 2;  // hi + lo images

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&bars.full[s], 5);    // the 4 warps of the chunk's group + loader expect_tx
      mbar_init(&bars.empty[s], 1);   // MMA commit
    }
    mbar_init(&bars.hfull[0], 1);     // halo block landed (TMA)
    mbar_init(&bars.hempty[0], kProdWarps);  // halo block converted (one arrival per producer warp)
    for (int h = 0; h < 2; ++h) {
      mbar_init(&bars.dfull[h], 1);
      mbar_init(&bars.dempty[h], kEpiWarps);  // one arrival per epilogue warp
    }
    mbar_init(&bars.drain, 1);
    bars.abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == kMmaWarp) tmem_alloc(&bars.tmem_slot, 512);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = bars.tmem_slot;
  // The set-up above touches no global memory, so it may overlap the previous
  // kernel in the stream (launched with programmatic serialisation): the
  // image, the packed filters and the output are only touched after this.
  grid_dependency_wait();
  allow_dependent_launch();

  const int RS = g.R * g.S;
  const int npix = g.OH * g.OW;
  const uint32_t dw = 2u * p.NT;  // accumulator width: [hh | small]
  auto d_col = [&](int d) { return d ? dw : 0u; };
  const uint32_t a_col0 = 2u * dw;  // stage s: hi at a_col0 + s*CB, lo at + CB/2
  volatile int *abort_flag = &bars.abort_flag;

  auto tile_decode = [&](int i, int &b, int &mt, int &nb) {
    nb = i % p.nblocks;
    const int rest = i / p.nblocks;
    mt = rest % p.tiles_m;
    b = rest / p.tiles_m;
  };

  if (warp < kProdWarps) {
    // ------------------------------------------------------------ producers
    const int quarter = warp & 3, group = warp >> 2;
    const int m = quarter * 32 + lane;  // pixel within the tile == TMEM lane
    const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
    const int npos = p.TR * p.TC;
    const float *land = reinterpret_cast<const float *>(landing);
    uint4 *spl = reinterpret_cast<uint4 *>(split);
    // The exit decision is taken jointly at the group's named barriers
    // (bar.red.or), so no producer can leave while the others wait there.
    uint32_t q = 0, hb = 0;
    bool failed = false;
    for (int i = blockIdx.x; i < p.total_tiles; i += gridDim.x) {
      int b, mt, nb;
      tile_decode(i, b, mt, nb);
      const int m0 = mt * kMT;
      const int pix = m0 + m;
      const bool valid = pix < npix;
      const int oy = valid ? pix / g.OW : 0, ox = valid ? pix % g.OW : 0;
      const int row0 = (m0 / g.OW) * g.down - g.low_r;
      const int pos0 = (oy * g.down - g.low_r - row0) * p.TC + (ox * g.down - g.low_c - p.start_c);
      for (int cb = 0; cb < p.NCB; ++cb, ++hb) {
        // 1. all producers convert the landed fp32 block into split bf16 hi/lo
        failed = named_sync_or(1, kProdThreads, failed || *abort_flag);  // previous block fully read
        if (failed) break;
        if (!mbar_wait(&bars.hfull[0], hb & 1, p.err)) failed = true;
        const int cvalid = min(CB, g.n - cb * CB);
        for (int pos = threadIdx.x; !failed && pos < npos; pos += kProdThreads) {
          uint4 *dst = spl + (size_t)pos * NCH;
          const int sw = pos % NCH;
#pragma unroll
          for (int k = 0; k < CB / 8; ++k) {  // 8 planes -> one hi and one lo chunk
            uint32_t hi[4], lo[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int c0 = 8 * k + 2 * j;
              const float v0 = (c0 < cvalid) ? land[c0 * npos + pos] : 0.0f;
              const float v1 = (c0 + 1 < cvalid) ? land[(c0 + 1) * npos + pos] : 0.0f;
              split_bf16x2(v0, v1, hi[j], lo[j]);
            }
            dst[k ^ sw] = make_uint4(hi[0], hi[1], hi[2], hi[3]);
            dst[(k + CB / 8) ^ sw] = make_uint4(lo[0], lo[1], lo[2], lo[3]);
          }
        }
        failed = named_sync_or(1, kProdThreads, failed);  // the split block is complete
        if (failed) break;
        if (lane == 0) mbar_arrive(&bars.hempty[0]);  // the landing buffer may be refilled
        // 2. this group's chunks: copy the pixel's split words of the tap to TMEM
        int r = 0, c = 0;
        for (int tap = 0; tap < RS; ++tap, ++q) {
          if ((int)(q % kGroups) == group) {
            const int s = q % kStages;
            bool bad = failed || *abort_flag;
            if (!bad) bad = !mbar_wait(&bars.empty[s], ((q / kStages) & 1) ^ 1, p.err);
            if (__any_sync(0xffffffffu, bad)) {  // warp-uniform: tcgen05.st is warp-collective
              failed = true;
            } else {
              tc_fence_after();
              const int pos = pos0 + r * p.TC + c;
              const uint4 *src = spl + (size_t)pos * NCH;
              const int sw = pos % NCH;
              const uint32_t acol = tmem + lane_base + a_col0 + (uint32_t)s * CB;
#pragma unroll
              for (int k = 0; k < NCH; k += 2) {
                const uint4 w0 = valid ? src[k ^ sw] : make_uint4(0, 0, 0, 0);
                const uint4 w1 = valid ? src[(k + 1) ^ sw] : make_uint4(0, 0, 0, 0);
                const uint32_t v8[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
                tmem_st8(acol + 4 * k, v8);  // hi words fill columns [0, CB/2), lo words [CB/2, CB)
              }
              tc_wait_st();
              tc_fence_before();
              __syncwarp();
              if (lane == 0) mbar_arrive(&bars.full[s]);
            }
          }
          if (++c == g.S) {
            c = 0;
            ++r;
          }
        }
      }
      if (failed) break;
    }
    if (failed) *abort_flag = 1;
  } else if (warp == kMmaWarp) {
    // ------------------------------------------------------------ MMA issuer
    // The whole warp walks the loop (its values stay warp-uniform); one
    // elected lane issues the tcgen05 instructions.
    const uint32_t idesc_n = idesc_bf16_f32(kMT, p.NT);
    const uint32_t idesc_2n = idesc_bf16_f32(kMT, 2 * p.NT);
    const uint32_t lbo = 128, sbo = CB * 16;
    const uint32_t bstage0 = smem_u32(bstage);
    uint32_t q = 0, tc = 0;
    bool failed = false;
    for (int i = blockIdx.x; i < p.total_tiles; i += gridDim.x, ++tc) {
      const int d = tc & 1;
      failed = __any_sync(0xffffffffu, failed || *abort_flag ||
                                           !mbar_wait(&bars.dempty[d], ((tc >> 1) & 1) ^ 1, p.err));
      if (failed) break;
      tc_fence_after();
      const uint32_t dt = tmem + d_col(d);
      const int nchunks = p.NCB * RS;
      if (RS >= kBatchTaps) {
        for (int k = 0; k < nchunks;) {
          // Lane i probes chunk q + i; every chunk ready in order from q is
          // issued in one batch, so the barrier probe, the vote and the fence
          // are paid once per batch instead of once per chunk.  A stage is at
          // most one phase ahead of this warp (its producers need the MMAs of
          // the chunk kStages earlier), so the parity test is exact.
          const bool ready = lane < kStages && k + lane < nchunks &&
                             mbar_test(&bars.full[(q + lane) % kStages], ((q + lane) / kStages) & 1);
          int nready = __ffs(~__ballot_sync(0xffffffffu, ready)) - 1;
          if (nready == 0) {
            failed = __any_sync(0xffffffffu, !mbar_wait(&bars.full[q % kStages], (q / kStages) & 1, p.err));
            if (failed) break;
            nready = 1;
          }
          tc_fence_after();
          if (elect_one()) {
            for (int i = 0; i < nready; ++i) {
              const uint32_t s = (q + i) % kStages;
              const uint32_t a_hi = tmem + a_col0 + s * CB;
              const uint32_t a_lo = a_hi + CB / 2;
              const uint32_t b_hi = bstage0 + s * bstage_bytes;
#pragma unroll
              for (int j = 0; j < CB / 16; ++j) {
                const uint32_t acc = (k + i > 0 || j > 0) ? 1u : 0u;
                const uint64_t dh = smem_desc_kmajor(b_hi + 256u * j, lbo, sbo);
                mma_bf16_ts(dt, a_hi + 8u * j, dh, idesc_2n, acc);       // [hi*hi | hi*lo]
                mma_bf16_ts(dt + p.NT, a_lo + 8u * j, dh, idesc_n, 1u);  // small half += lo*hi
              }
              tc_commit(&bars.empty[s]);
            }
          }
          __syncwarp();
          k += nready;
          q += nready;
        }
      } else {
        // one chunk per probe (filters of fewer taps: short blocks)
        for (int k = 0; k < nchunks; ++k, ++q) {
          const int s = q % kStages;
          failed = __any_sync(0xffffffffu, !mbar_wait(&bars.full[s], (q / kStages) & 1, p.err));
          if (failed) break;
          tc_fence_after();
          const uint32_t a_hi = tmem + a_col0 + (uint32_t)s * CB;
          const uint32_t a_lo = a_hi + CB / 2;
          const uint32_t b_hi = bstage0 + (uint32_t)s * bstage_bytes;
          if (elect_one()) {
#pragma unroll
            for (int j = 0; j < CB / 16; ++j) {
              const uint32_t acc = (k > 0 || j > 0) ? 1u : 0u;
              const uint64_t dh = smem_desc_kmajor(b_hi + 256u * j, lbo, sbo);
              mma_bf16_ts(dt, a_hi + 8u * j, dh, idesc_2n, acc);       // [hi*hi | hi*lo]
              mma_bf16_ts(dt + p.NT, a_lo + 8u * j, dh, idesc_n, 1u);  // small half += lo*hi
            }
            tc_commit(&bars.empty[s]);
          }
          __syncwarp();
        }
      }
      if (failed) break;
      if (elect_one()) tc_commit(&bars.dfull[d]);
      __syncwarp();
    }
    if (failed) *abort_flag = 1;
    // Every MMA issued has retired before tensor memory can be released.
    if (elect_one()) tc_commit(&bars.drain);
    __syncwarp();
    mbar_wait(&bars.drain, 0, p.err);
  } else if (warp == kLoadWarp) {
    // ------------------------------------------------------------ loader
    if (RS >= kBatchTaps) {
      // The whole warp walks the chunks (its values stay warp-uniform).  Lane i
      // probes the stage of chunk q + i; every chunk whose stage is free, in
      // order from q, has its filter copy issued at once by its own lane, so the
      // copies of a batch go out together instead of one loop trip each.  A
      // stage is at most one phase ahead of this warp (its next MMA needs this
      // warp's copy), so the parity test is exact.  Lane 0 alone issues the
      // halo blocks; every lane keeps the same bookkeeping.
      const uint32_t halo_tx = (uint32_t)(p.TC * p.TR * CB * 4);
      // Halo blocks in the producers' order: (tile, cb) for this CTA's tiles.
      int h_tile = blockIdx.x, h_cb = 0;  // next halo block to issue
      uint32_t h_issued = 0;
      auto halo_try = [&](bool block) -> int {
        // 1 issued, 0 not yet possible, -1 timed out (warp-uniform)
        if (h_tile >= p.total_tiles) return 0;
        const uint32_t parity = (h_issued & 1) ^ 1;
        int st = 0;
        if (lane == 0) st = block ? (mbar_wait(&bars.hempty[0], parity, p.err) ? 1 : -1)
                                  : (mbar_test(&bars.hempty[0], parity) ? 1 : 0);
        st = __shfl_sync(0xffffffffu, st, 0);
        if (st <= 0) return st;
        if (lane == 0) {
          int b, mt, nb;
          tile_decode(h_tile, b, mt, nb);
          const int row0 = ((mt * kMT) / g.OW) * g.down - g.low_r;
          mbar_arrive_expect_tx(&bars.hfull[0], halo_tx);
          tma_load_3d(landing, &xmap, &bars.hfull[0], p.start_c, row0, b * g.n + h_cb * CB);
        }
        ++h_issued;
        if (++h_cb == p.NCB) {
          h_cb = 0;
          h_tile += gridDim.x;
        }
        return 1;
      };
      bool ok = halo_try(true) >= 0;
      uint32_t q = 0, hb = 0;
      for (int i = blockIdx.x; ok && i < p.total_tiles && !__any_sync(0xffffffffu, *abort_flag != 0);
           i += gridDim.x) {
        int b, mt, nb;
        tile_decode(i, b, mt, nb);
        for (int cb = 0; ok && cb < p.NCB; ++cb, ++hb) {
          const uint8_t *bsrc = p.bpack + (((size_t)nb * p.NCB + cb) * RS) * bstage_bytes;
          for (int tap = 0; tap < RS;) {
            const bool free_stage = lane < kStages && tap + lane < RS &&
                                    mbar_test(&bars.empty[(q + lane) % kStages], (((q + lane) / kStages) & 1) ^ 1);
            int n = __ffs(~__ballot_sync(0xffffffffu, free_stage)) - 1;
            if (n == 0) {
              ok = !__any_sync(0xffffffffu,
                               lane == 0 && !mbar_wait(&bars.empty[q % kStages], ((q / kStages) & 1) ^ 1, p.err));
              if (!ok) break;
              n = 1;
            }
            if (lane < n) {
              const uint32_t s = (q + lane) % kStages;
              mbar_arrive_expect_tx(&bars.full[s], bstage_bytes);
              bulk_load(bstage + (size_t)s * bstage_bytes, bsrc + (size_t)(tap + lane) * bstage_bytes, bstage_bytes,
                        &bars.full[s]);
            }
            q += n;
            tap += n;
            // prefetch the next halo block as soon as the landing buffer is free
            if (h_issued == hb + 1 && halo_try(false) < 0) ok = false;
          }
          // the producers need the next block before they can go on
          if (ok && h_issued == hb + 1 && halo_try(true) < 0) ok = false;
        }
      }
      if (!ok) *abort_flag = 1;
      if (__any_sync(0xffffffffu, *abort_flag != 0) && lane == 0) {
        // Let copies that may still be in flight land before this CTA's
        // shared memory is released: the last kStages filter chunks and the
        // last halo block issued.
        for (uint32_t qq = q > kStages ? q - kStages : 0; qq < q; ++qq)
          mbar_wait(&bars.full[qq % kStages], (qq / kStages) & 1, p.err);
        if (h_issued > 0) mbar_wait(&bars.hfull[0], (h_issued - 1) & 1, p.err);
      }
    } else if (lane == 0) {
      // one thread, one chunk per loop trip (filters of fewer taps)
      const uint32_t halo_tx = (uint32_t)(p.TC * p.TR * CB * 4);
      // Halo blocks in the producers' order: (tile, cb) for this CTA's tiles.
      int h_tile = blockIdx.x, h_cb = 0;  // next halo block to issue
      uint32_t h_issued = 0;
      auto halo_ready_to_issue = [&](bool block) -> int {
        // 1 issued, 0 not yet possible, -1 timed out
        if (h_tile >= p.total_tiles) return 0;
        const uint32_t parity = (h_issued & 1) ^ 1;
        if (block) {
          if (!mbar_wait(&bars.hempty[0], parity, p.err)) return -1;
        } else if (!mbar_test(&bars.hempty[0], parity)) {
          return 0;
        }
        int b, mt, nb;
        tile_decode(h_tile, b, mt, nb);
        const int row0 = ((mt * kMT) / g.OW) * g.down - g.low_r;
        mbar_arrive_expect_tx(&bars.hfull[0], halo_tx);
        tma_load_3d(landing, &xmap, &bars.hfull[0], p.start_c, row0, b * g.n + h_cb * CB);
        ++h_issued;
        if (++h_cb == p.NCB) {
          h_cb = 0;
          h_tile += gridDim.x;
        }
        return 1;
      };
      bool ok = halo_ready_to_issue(true) >= 0;
      uint32_t q = 0, hb = 0;
      for (int i = blockIdx.x; ok && i < p.total_tiles && !*abort_flag; i += gridDim.x) {
        int b, mt, nb;
        tile_decode(i, b, mt, nb);
        for (int cb = 0; ok && cb < p.NCB; ++cb, ++hb) {
          const uint8_t *bsrc = p.bpack + (((size_t)nb * p.NCB + cb) * RS) * bstage_bytes;
          for (int tap = 0; tap < RS; ++tap, ++q) {
            const int s = q % kStages;
            if (!mbar_wait(&bars.empty[s], ((q / kStages) & 1) ^ 1, p.err)) { ok = false; break; }
            mbar_arrive_expect_tx(&bars.full[s], bstage_bytes);
            bulk_load(bstage + (size_t)s * bstage_bytes, bsrc + (size_t)tap * bstage_bytes, bstage_bytes,
                      &bars.full[s]);
            // prefetch the next halo block as soon as the landing buffer is free
            if (h_issued == hb + 1 && halo_ready_to_issue(false) < 0) ok = false;
          }
          // the producers need the next block before they can go on
          if (ok && h_issued == hb + 1 && halo_ready_to_issue(true) < 0) ok = false;
        }
      }
      if (!ok) *abort_flag = 1;
      if (*abort_flag) {
        // Let copies that may still be in flight land before this CTA's
        // shared memory is released: the last kStages filter chunks and the
        // last halo block issued.
        for (uint32_t qq = q > kStages ? q - kStages : 0; qq < q; ++qq)
          mbar_wait(&bars.full[qq % kStages], (qq / kStages) & 1, p.err);
        if (h_issued > 0) mbar_wait(&bars.hfull[0], (h_issued - 1) & 1, p.err);
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    const int sub = warp & 3;  // TMEM lane quarter this warp may access
    const int half = (warp - (kProdWarps + 2)) >> 2;  // which alternate 16-column blocks
    const int m = sub * 32 + lane;
    const uint32_t lane_base = (uint32_t)(sub * 32) << 16;
    const bool relu = (g.flags & CCT_FLAG_RELU) != 0;
    uint32_t tc = 0;
    for (int i = blockIdx.x; i < p.total_tiles; i += gridDim.x, ++tc) {
      if (__any_sync(0xffffffffu, *abort_flag != 0)) break;
      const int d = tc & 1;
      const bool bad = !mbar_wait(&bars.dfull[d], (tc >> 1) & 1, p.err);
      if (__any_sync(0xffffffffu, bad)) {  // warp-uniform: tcgen05.ld is warp-collective
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      int b, mt, nb;
      tile_decode(i, b, mt, nb);
      const int pix = mt * kMT + m;
      const bool valid = pix < npix;
      const int n0 = nb * p.NT;
      float *ybase = p.y + ((size_t)b * g.groups + n0) * npix + pix;
      for (int c = 16 * half; c < p.NT; c += 32) {
        uint32_t v[16], v2[16];
        tmem_ld16(tmem + lane_base + d_col(d) + c, v);
        tmem_ld16(tmem + lane_base + d_col(d) + p.NT + c, v2);
        tc_wait_ld();
        if (valid) {
#pragma unroll
          for (int t = 0; t < 16; ++t) {
            if (n0 + c + t < g.groups) {
              float val = __uint_as_float(v[t]);
              val += __uint_as_float(v2[t]);
              if (relu) val = fmaxf(val, 0.0f);
              ybase[(size_t)(c + t) * npix] = val;
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars.dempty[d]);
    }
  }

  // ---------------------------------------------------------------- teardown
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kMmaWarp) tmem_dealloc(tmem, 512);
}

// Pack filters into per-chunk bf16 hi/lo operand images:
// chunk (nb, cb, tap) = [hi NT x CB][lo NT x CB], row n = output plane
// nb*NT + n, column ci = input plane cb*CB + ci, value f[plane(n, c)][tap']
// with tap' flipped for convolution.  Rows/columns past the real counts are 0.
__global__ void pack_filters_kernel(ConvGeom g, const float *__restrict__ f, uint8_t *__restrict__ out,
                                    int NT, int CB, int NCB, int nblocks) {
  // the packed operand is at most a few hundred MB, so 32-bit indices suffice
  // (launch_pack_filters checks); 64-bit division would dominate this kernel
  const int RS = g.R * g.S;
  const int total = nblocks * NCB * RS * NT * CB;
  // the previous kernel (the last launch that read the packed operand) must
  // be done before it is rewritten; the consuming kernel may be scheduled now
  grid_dependency_wait();
  allow_dependent_launch();
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int ci = idx % CB;
    int rest = idx / CB;
    const int n = rest % NT;
    rest /= NT;
    const int tap = rest % RS;
    rest /= RS;
    const int cb = rest % NCB;
    const int nb = rest / NCB;
    const int k = nb * NT + n, c = cb * CB + ci;
    float v = 0.0f;
    if (k < g.groups && c < g.n) {
      // output plane o = k of image 0, term c -> filter plane
      int ip, fp;
      plane_pair(g, k, c, &ip, &fp);
      const int r = tap / g.S, s = tap - r * g.S;
      const int src = g.orient == CCT_CONVOLUTION ? (g.R - 1 - r) * g.S + (g.S - 1 - s) : tap;
      v = f[(size_t)fp * RS + src];
    }
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
    const size_t chunk = ((size_t)nb * NCB + cb) * RS + tap;
    uint8_t *img = out + chunk * (2u * NT * CB * 2);
    const uint32_t off = packed_offset(n, ci, CB);
    *reinterpret_cast<__nv_bfloat16 *>(img + off) = h;
    *reinterpret_cast<__nv_bfloat16 *>(img + NT * CB * 2 + off) = l;
  }
}

std::mutex g_tc_mu;
std::unordered_map<uint64_t, size_t> g_tc_attr;

template <int CB>
int launch_cb(const TcParams &p0, const float *x, cudaStream_t st) {
  TcParams p = p0;
  CUtensorMap map;
  int rc = encode_tensor_map_3d_box(&map, x, p.g.W, p.g.H, p.g.pin, p.TC, p.TR, CB);
  if (rc) return rc;
  const size_t smem = 2 * (size_t)p.halo_bytes + (size_t)kStages * 2u * p.NT * CB * 2;
  auto kern = frame_tc_kernel<CB>;
  {
    // Dynamic shared memory above 48 KB needs the opt-in attribute; keep the
    // largest size set so far per (device, instance).
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t key = ((uint64_t)dev << 32) | (uint64_t)CB;
    std::lock_guard<std::mutex> lk(g_tc_mu);
    size_t &have = g_tc_attr[key];
    if (have < smem) {
      rc = check_cuda(cudaFuncSetAttribute((const void *)kern,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                      "cudaFuncSetAttribute(frame_tc)");
      if (rc) return rc;
      have = smem;
    }
  }
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.gridDim = dim3(p.grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  rc = check_cuda(cudaLaunchKernelEx(&cfg, kern, map, p), "frame_tc_kernel launch");
  if (rc) return rc;
  count_launches(1);
  return check_cuda(cudaGetLastError(), "frame_tc_kernel launch");
}

}  // namespace

// Tile plan for the tensor-core kernel; returns false when the shape is
// outside what it handles (the FP32 frame kernel takes those).
bool frame_tc_plan(const ConvGeom &g, int sms, TcParams *out) {
  if (g.mode != CCT_PROJECT_FRAME_BLOCK_REDUCE_SUM && g.mode != CCT_BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM)
    return false;
  if (g.up != 1 || (g.down != 1 && g.down != 2)) return false;
  if (g.border != CCT_BORDER_ZERO && g.border != CCT_BORDER_FULL && g.border != CCT_BORDER_VALID)
    return false;
  if ((g.W & 3) != 0) return false;
  TcParams p{};
  p.g = g;
  const int npix = g.OH * g.OW;
  p.tiles_m = (npix + kMT - 1) / kMT;
  p.NT = std::min(64, ((g.groups + 15) / 16) * 16);
  p.nblocks = (g.groups + p.NT - 1) / p.NT;
  p.total_tiles = g.batch * p.tiles_m * p.nblocks;
  // rows of output spanned by any tile
  int max_rows = 0;
  for (int mt = 0; mt < p.tiles_m; ++mt) {
    const int first = (mt * kMT) / g.OW, last = (std::min(npix, (mt + 1) * kMT) - 1) / g.OW;
    max_rows = std::max(max_rows, last - first + 1);
  }
  p.TR = (max_rows - 1) * g.down + g.R;
  // x origin of the box: -low_c rounded down to a multiple of 4 (TMA rule)
  const int lc = -g.low_c;
  p.start_c = lc >= 0 ? (lc / 4) * 4 : -(((-lc) + 3) / 4) * 4;
  const int off = lc - p.start_c;
  p.TC = ((off + (g.OW - 1) * g.down + g.S) + 3) & ~3;
  if (p.TC > 256 || p.TR > 256) return false;
  const int cmax = ((g.n + 15) / 16) * 16;
  const size_t budget = 220 * 1024;
  p.CB = 0;
  for (int cb : {64, 32, 16}) {
    if (cb > cmax && cb != 16) continue;
    const size_t halo = (((size_t)p.TC * p.TR * cb * 4) + 1023) & ~(size_t)1023;
    const size_t bst = (size_t)kStages * 2u * p.NT * cb * 2;
    const int dw = 2 * p.NT;
    const int tcols = 2 * dw + kStages * cb;
    if (2 * halo + bst <= budget && tcols <= 512) {
      p.CB = cb;
      p.halo_bytes = (uint32_t)halo;
      break;
    }
  }
  if (!p.CB) return false;
  p.NCB = (g.n + p.CB - 1) / p.CB;
  p.grid = std::min(p.total_tiles, sms);
  p.pack_bytes = (size_t)p.nblocks * p.NCB * g.R * g.S * 2u * p.NT * p.CB * 2;
  *out = p;
  return true;
}

int launch_pack_filters(const TcParams &p, const float *f, uint8_t *packed, cudaStream_t st) {
  const long long total = (long long)p.nblocks * p.NCB * p.g.R * p.g.S * p.NT * p.CB;
  if (total > 0x7fffffffLL) return set_error(CCT_ENOTSUP, "packed filter operand too large");
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 16);
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(256);
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int rc = check_cuda(cudaLaunchKernelEx(&cfg, pack_filters_kernel, p.g, f, packed, p.NT, p.CB, p.NCB, p.nblocks),
                      "pack_filters_kernel launch");
  if (rc) return rc;
  count_launches(1);
  return check_cuda(cudaGetLastError(), "pack_filters_kernel launch");
}

int launch_frame_tc(const TcParams &p, const float *x, float *y, const uint8_t *packed,
                    unsigned *err, cudaStream_t st) {
  TcParams q = p;
  q.y = y;
  q.bpack = packed;
  q.err = err;
  switch (p.CB) {
    case 16: return launch_cb<16>(q, x, st);
    case 32: return launch_cb<32>(q, x, st);
    case 64: return launch_cb<64>(q, x, st);
    default: return set_error(CCT_ENOTSUP, "frame_tc: bad channel block %d", p.CB);
  }
}

}  // namespace cct
