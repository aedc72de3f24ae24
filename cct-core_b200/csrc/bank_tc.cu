// Fused filter-bank convolution on the tcgen05 tensor cores, split BF16:
// ProjectFrameBlockReduceSum / BackProjectFrameBlockReduceSum
// (ConvolveHyperKernel.scala:153-199, 319-340, 574-645), every border policy
// (:235-317), DownsampleOutput(1, 2) (:205-223), UpsampleInput(2-4)
// (:206-212, 405-459, as one sub-filter per output phase), any field width.
// Banks of at most 32 filters put two taps of a filter row into each MMA
// (paired taps: tap b's sums are read one grid position to the right).
//
// GEMM view, per image b and block of 64 filters:
//   D[filter k][position p] = sum over (plane c, tap t) F[k][c, t] * X[c][p + off(t)]
// M = the filter block, N = a tile of output positions, reduction = planes x
// taps.  Positions live on a padded output grid of pitch P = BW + (S-1)/step
// columns (a band of BW output columns plus the tap reach): the input value a
// position reads at tap t then sits at a fixed offset off(t) from the
// position on the same grid, so the B operand of tap t is a contiguous run of
// the halo in shared memory and the tensor core reads it through a shifted
// descriptor -- no per-tap copies.  Grid columns past the band's outputs are
// computed and discarded ((S-1)/P of the work).  DownsampleOutput(2) holds
// the input as its four polyphase components, each a stride-1 grid.
//
// Split precision.  x = xh + xl (+ xm) and f likewise, each term bf16.  The
// filter operand of one MMA is 128 rows: rows 0-63 ("big") multiply into the
// hi*hi sum only, rows 64-127 ("small") into the correction products:
//   2 terms (BF16X3): [Fh; Fl] x Xh  and  [0; Fh] x Xl
//                     -> big hh, small lh + hl
//   3 terms (BF16X6): [Fh; Fm] x Xh, [0; Fh] x Xm, [0; Fh] x Xl, [0; Fl] x Xh,
//                     [0; Fm] x Xm
//                     -> big hh, small mh + hm + hl + lh + mm
// The big rows never receive a small addend: the tensor core's FP32
// accumulation drops the bits of an addend below the accumulator's last
// place, and measured that way its error grows with the number of MMAs
// accumulated, so only hh goes into the big sum and zero rows (which add
// exactly 0) fill the big half of the other MMAs.  For long reductions the
// accumulator is also promoted: every seg_stages stages the epilogue adds it
// into an FP32 running sum (RN, CUDA cores) and the next MMA starts it
// afresh, which bounds the accumulation error by the segment length.  The
// epilogue adds each filter's big and small rows.
//
// Warp roles (one persistent CTA per SM, 640 threads):
//   warps 0-9   converters: for each (tile, plane block) fill a halo buffer:
//               plain loads of the input with the border policy applied
//               (zero, clamp, cyclic), split into bf16 terms, stored in the
//               K-major core-matrix layout [plane group][position][8 planes];
//               two buffers, so the next block is converted while the
//               current one is multiplied.  Then warps 0-7 store half of
//               the CTA's last tile with the epilogue warps.
//   warp 10     MMA issuer (one elected lane): per (tile, plane block, tap):
//               KS k-steps x nmma MMAs, A = filter chunk stage, B = halo.
//   warp 11     loader (one lane): bulk copies of the pre-packed filter
//               chunks (nb, plane block, tap) into a ring of stages, one copy
//               per stage of several taps.
//   warps 12-19 epilogue, two per tensor-memory lane quarter (alternate
//               column halves): promotion adds, then per 16-column chunk the
//               warps holding one filter block's parts write them to shared
//               memory, and each adds the parts of a share of the filters,
//               applies ReLU and stores.
// Every wait is bounded: on a timeout the CTA records it in the device error
// word, lets its copies and MMAs land, frees tensor memory and exits.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <unordered_map>

#include "bank_tc.h"
#include "sm100_util.cuh"

namespace cct {
namespace {

constexpr int kConvWarps = 10;  // ten: a 536-position halo takes two rounds of loads, not three
constexpr int kConvThreads = 32 * kConvWarps;
constexpr int kMmaWarp = kConvWarps;
constexpr int kLoadWarp = kConvWarps + 1;
constexpr int kEpiWarp0 = kConvWarps + 2;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 32 * (kEpiWarp0 + kEpiWarps);
constexpr int kMaxStages = 8;
constexpr int kPackThreads = 128;
constexpr uint32_t kAccCols = 256;  // one accumulator (N <= 256 fp32 columns)
// Epilogue exchange: eight part tiles of 32 filters x 16 positions (row
// pitch 17 floats: conflict-free by filter and by position).
constexpr int kXchPitch = 17;
constexpr int kXchFloats = 32 * kXchPitch;
constexpr size_t kXchBytes = 8 * kXchFloats * sizeof(float);

// Filter chunk row blocks (64 rows each) and the MMAs over them.
// Block contents: -1 zero, else the split term (0 hi, 1 mid / lo for 2 terms, 2 lo).
__host__ __device__ constexpr int block_term(int terms, int blk) {
  return terms == 2 ? (blk == 0 ? -1 : blk - 1)                          // Z Fh Fl
                    : (blk == 0 || blk == 3 || blk == 5 ? -1             // Z Fh Fm Z Fl Z Fm
                                                        : (blk == 1 ? 0 : blk == 2 ? 1 : blk == 4 ? 2 : 1));
}
// Paired taps (banks of at most 32 filters): a chunk of 32-row blocks
// [0 0 Fh_a Fh_b Fl_a Fl_b] for taps a and b = a + 1 of one filter row, the
// same 192 rows and MMAs as an unpaired two-term chunk: [Fh_a; Fh_b; Fl_a;
// Fl_b] x Xh and [0; 0; Fh_a; Fh_b] x Xl.  -1 zero, else (term, which tap).
__host__ __device__ constexpr int pair_block_term(int blk) { return blk < 2 ? -1 : blk < 4 ? 0 : 1; }
__host__ __device__ constexpr int pair_block_tap(int blk) { return blk & 1; }
template <int TERMS, bool PAIR>
struct MmaList;
template <>
struct MmaList<2, false> {
  static constexpr int n = 2;
  __device__ static int arow(int m) { return m == 0 ? 64 : 0; }  // [Fh; Fl], [0; Fh]
  __device__ static int bterm(int m) { return m; }               // Xh, Xl
};
template <>
struct MmaList<2, true> : MmaList<2, false> {};  // at tap a's offset
template <>
struct MmaList<3, false> {
  static constexpr int n = 5;
  // [Fh; Fm] x Xh, [0; Fh] x Xm, [0; Fh] x Xl, [0; Fl] x Xh, [0; Fm] x Xm
  __device__ static int arow(int m) { return m == 0 ? 64 : m == 3 ? 192 : m == 4 ? 320 : 0; }
  __device__ static int bterm(int m) { return m == 0 || m == 3 ? 0 : m == 2 ? 2 : 1; }
};

struct Bars {
  uint64_t full[kMaxStages], empty[kMaxStages];  // filter chunk stages
  uint64_t hfull[2], hempty[2];                  // halo buffers
  uint64_t dfull[2], dempty[2];                  // accumulators (one per segment in flight)
  uint64_t drain;                                // MMA warp: every MMA retired
  uint32_t tmem_slot;
  int abort_flag;
};

// Border policy of the input (ConvolveHyperKernel.scala:235-317): maps
// (iy, ix) into the field, or returns false for a zero.
__device__ __forceinline__ bool border_map(const ConvGeom &g, int iy, int ix, int &ry, int &rx) {
  if (g.border == CCT_BORDER_CLAMP) {
    ry = min(max(iy, 0), g.H - 1);
    rx = min(max(ix, 0), g.W - 1);
    return true;
  }
  if (g.border == CCT_BORDER_CYCLIC) {
    ry = ((iy % g.H) + g.H) % g.H;
    rx = ((ix % g.W) + g.W) % g.W;
    return true;
  }
  ry = iy;
  rx = ix;
  return iy >= 0 && iy < g.H && ix >= 0 && ix < g.W;
}

struct Item {
  int b, ph, band, tile, nb;
};
__device__ __forceinline__ Item decode(const BankParams &p, int i) {
  Item it;
  it.nb = i % p.nblocks;
  int rest = i / p.nblocks;
  it.tile = rest % p.tiles_band;
  rest /= p.tiles_band;
  it.band = rest % p.nbands;
  rest /= p.nbands;
  it.ph = rest % p.nph_out;
  it.b = rest / p.nph_out;
  return it;
}

// Reduction units of a work item: ts taps per filter row of its (sub-)filter,
// nu units, nst stages per plane block, and the first packed chunk of its
// filter block.  Every role derives its loop bounds from here.
struct ItemUnits {
  int ts, nu, nst;
  size_t chunk0;
};
template <bool PAIR>
__device__ __forceinline__ ItemUnits item_units(const BankParams &p, const Item &it) {
  ItemUnits r;
  int rows;
  if (p.up > 1) {
    const int rho = it.ph / p.up;
    rows = p.up_rq[rho];
    r.ts = p.up_sq[it.ph - rho * p.up];
  } else {
    rows = p.g.R;
    r.ts = p.g.S;
  }
  r.nu = rows * (PAIR ? (r.ts + 1) / 2 : r.ts);
  r.nst = (r.nu + p.T - 1) / p.T;
  r.chunk0 = (size_t)p.up_choff[it.ph] + (size_t)it.nb * p.NCB * r.nu;
  return r;
}

// Split 8*KG planes of one halo position into bf16 terms and store them as
// KG core-matrix rows (16 bytes per term).  src points at the position in
// the first plane; `cvalid` planes exist (the rest are zero).  All 8*KG loads
// are issued before the first store, so a converter thread keeps that many
// reads in flight.
template <int KG>
__device__ __forceinline__ void load_kgroups(const float *src, size_t plane, bool in, int cvalid, float (&v)[8 * KG]) {
#pragma unroll
  for (int j = 0; j < 8 * KG; ++j) v[j] = (in && j < cvalid) ? __ldg(src + j * plane) : 0.0f;
}

template <int TERMS, int KG>
__device__ __forceinline__ void store_kgroups(const float (&v)[8 * KG], uint8_t *dst, uint32_t kg_stride,
                                              uint32_t part_bytes) {
#pragma unroll
  for (int k = 0; k < KG; ++k) {
    uint8_t *d = dst + k * kg_stride;
    const float *w = v + 8 * k;
    if (TERMS == 2) {
      uint32_t hi[4], lo[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) split_bf16x2(w[2 * j], w[2 * j + 1], hi[j], lo[j]);
      *reinterpret_cast<uint4 *>(d) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<uint4 *>(d + part_bytes) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    } else {
      uint32_t hi[4], mi[4], lo[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) split3_bf16x2(w[2 * j], w[2 * j + 1], hi[j], mi[j], lo[j]);
      *reinterpret_cast<uint4 *>(d) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<uint4 *>(d + part_bytes) = make_uint4(mi[0], mi[1], mi[2], mi[3]);
      *reinterpret_cast<uint4 *>(d + 2 * (size_t)part_bytes) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
  }
}

template <int TERMS, int KG>
__device__ __forceinline__ void convert_kgroups(const float *src, size_t plane, bool in, int cvalid,
                                                uint8_t *dst, uint32_t kg_stride, uint32_t part_bytes) {
  float v[8 * KG];
  load_kgroups<KG>(src, plane, in, cvalid, v);
  store_kgroups<TERMS, KG>(v, dst, kg_stride, part_bytes);
}

// Final accumulator of work item `it` (S in tensor-memory columns at `sc`,
// plus the running sum at `rc` unless `first`), columns [cbeg, cbeg + ncol):
// the group of G warps holding one block of 32 filters' parts (this warp's
// lane quarter `quarter`, part `part`) writes each 16-column chunk into its
// own [filter][position] tile, and after a barrier each adds the parts of its
// share of the filters (a half, or a quarter) and stores them, so no warp
// waits on another's stores.  `release` (or null): arrived on once this
// warp's last accumulator load is done.
template <int TERMS, bool PAIR>
__device__ __forceinline__ void store_tile_columns(const BankParams &p, const Item &it, uint32_t sc, uint32_t rc,
                                                   bool first, int cbeg, int ncol, float *tiles, int bar_id,
                                                   int quarter, int part, int lane, uint64_t *release) {
  const ConvGeom &g = p.g;
  constexpr int G = PAIR ? 4 : 2;  // parts (warps) per group
  const int bar_count = 32 * G;
  const bool relu = (g.flags & CCT_FLAG_RELU) != 0;
  const size_t opl = (size_t)g.OH * g.OW;
  const int limit = PAIR ? p.tile_adv : p.N;  // columns of the tile with complete sums
  const int p0 = it.tile * p.tile_adv;
  // grid position (Y, X) of band `band` -> output (up*Y + rho, up*(band*BW + X) + kap)
  const int rho = it.ph / p.up, kap = it.ph - rho * p.up;
  const int ohv = (g.OH - rho + p.up - 1) / p.up;                                 // valid grid rows
  const int bw = min(p.BW, (g.OW - kap + p.up - 1) / p.up - it.band * p.BW);     // valid columns of the band
  const size_t ors = (size_t)p.up * g.OW;                                          // output row stride of a grid row
  // the group's 32 filters
  const int fb = it.nb * p.fblock + (PAIR ? 0 : (quarter & 1) * 32);
  float *ybase0 = p.y + (size_t)it.b * g.groups * opl + (size_t)rho * g.OW + (size_t)it.band * p.BW * p.up + kap +
                  (size_t)fb * opl;
  // The next chunk's accumulator load is in flight while a chunk is combined
  // and stored (18 warps: 96 registers a thread at most; three-term and
  // paired kernels have none to spare and load each chunk when they reach it).
  uint32_t n16[16], ne = 0;
  auto issue = [&](int c) {
    tmem_ld16(sc + c, n16);
    // paired taps: tap b's rows (quarters 1, 3) also need column c + 16
    if (PAIR && (quarter & 1) && c + 16 < p.N) tmem_ld1(sc + c + 16, ne);
  };
  constexpr bool kAhead = TERMS == 2 && !PAIR;
  if (kAhead) issue(cbeg);
  for (int c = cbeg; c < cbeg + ncol; c += 16) {
    if (!kAhead) issue(c);
    tc_wait_ld();
    const bool ext = PAIR && (quarter & 1) && c + 16 < p.N;
    uint32_t s16[16], r16[16], e1 = ne, e2 = 0;
#pragma unroll
    for (int t = 0; t < 16; ++t) s16[t] = n16[t];
    if (!first) {
      tmem_ld16(rc + c, r16);
      if (ext) tmem_ld1(rc + c + 16, e2);
      tc_wait_ld();
    }
    float v[17];
#pragma unroll
    for (int t = 0; t < 16; ++t) v[t] = __uint_as_float(s16[t]) + (first ? 0.0f : __uint_as_float(r16[t]));
    v[16] = ext ? __uint_as_float(e1) + (first ? 0.0f : __uint_as_float(e2)) : 0.0f;
    if (release && c + 16 >= cbeg + ncol) {  // the accumulator is read: release it
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(release);
    }
    {
      float *mine = tiles + part * kXchFloats + lane * kXchPitch;
      const bool sh = PAIR && (quarter & 1);  // tap b's sums sit one position to the right
#pragma unroll
      for (int t = 0; t < 16; ++t) mine[t] = sh ? v[t + 1] : v[t];
    }
    if (kAhead && c + 16 < cbeg + ncol) issue(c + 16);
    named_sync(bar_id, bar_count);  // every part of the chunk is in place
    // this warp's share: the parts of its filters, all loaded before the
    // barrier that lets the group overwrite the tiles
    float w[16];
    int t0, fl;
    if (p.vec4) {
      // lane -> (filter 8*i + lane/4, positions 4*(lane%4) .. +3), i in the share
      t0 = 4 * (lane & 3);
      fl = lane >> 2;
#pragma unroll
      for (int k = 0; k < 4 / G; ++k)
#pragma unroll
        for (int q = 0; q < G; ++q)
#pragma unroll
          for (int e = 0; e < 4; ++e)
            w[(k * G + q) * 4 + e] = tiles[q * kXchFloats + (8 * (part * (4 / G) + k) + fl) * kXchPitch + t0 + e];
    } else {
      // lane -> (filter 2*i + lane/16, position lane%16), i in the share
      t0 = lane & 15;
      fl = lane >> 4;
#pragma unroll
      for (int k = 0; k < 16 / G; ++k)
#pragma unroll
        for (int q = 0; q < G; ++q)
          w[k * G + q] = tiles[q * kXchFloats + (2 * (part * (16 / G) + k) + fl) * kXchPitch + t0];
    }
    named_sync(bar_id, bar_count);  // the tiles may be rewritten
    const int Gp = p0 + c + t0;
    const int Y = Gp / p.P, X = Gp - Y * p.P;
    const bool ok = Y < ohv && X < bw && c + t0 < limit;
    if (p.vec4) {
      float *yo = ybase0 + (size_t)Y * ors + X;  // up == 1 here
#pragma unroll
      for (int k = 0; k < 4 / G; ++k) {
        const int f = 8 * (part * (4 / G) + k) + fl;
        float o[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          float acc = w[(k * G) * 4 + e];
#pragma unroll
          for (int q = 1; q < G; ++q) acc = acc + w[(k * G + q) * 4 + e];  // parts in order
          o[e] = relu ? fmaxf(acc, 0.0f) : acc;
        }
        if (ok && fb + f < g.groups)
          *reinterpret_cast<float4 *>(yo + (size_t)f * opl) = make_float4(o[0], o[1], o[2], o[3]);
      }
    } else {
      float *yo = ybase0 + (size_t)Y * ors + (size_t)X * p.up;
#pragma unroll
      for (int k = 0; k < 16 / G; ++k) {
        const int f = 2 * (part * (16 / G) + k) + fl;
        float acc = w[k * G];
#pragma unroll
        for (int q = 1; q < G; ++q) acc = acc + w[k * G + q];  // parts in order
        if (relu) acc = fmaxf(acc, 0.0f);
        if (ok && fb + f < g.groups) yo[(size_t)f * opl] = acc;
      }
    }
  }
}

// The last tile of a CTA is stored by the converter warps as well as the
// epilogue warps (each taking a quarter of the columns): by then the
// converters have nothing left to fill.  Only when every item is one
// accumulation segment (the converters then wait on the last item's
// accumulator phase in order) and a quarter of a tile is whole chunks.
__device__ __forceinline__ bool helpers_store_last(const BankParams &p) { return !p.promote && p.N % 64 == 0; }

// CB16: 16-plane blocks (the converters pair their (phase, position) items);
// a separate instance, so the other plane blocks' code is unchanged.
template <int TERMS, bool PAIR, bool CB16>
__global__ void __launch_bounds__(kThreads, 1) bank_tc_kernel(const __grid_constant__ BankParams p) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ Bars bars;
  // epilogue exchange: 4 groups of 2 part tiles, or (paired taps) 2 groups of 4
  __shared__ float xch[8 * kXchFloats];
  __shared__ uint32_t unit_boff[kBankMaxTaps];  // MMA warp: B operand offset of each unit
  const ConvGeom &g = p.g;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint8_t *halo = smem;                                 // 2 x halo_bytes
  uint8_t *stage = smem + 2 * (size_t)p.halo_bytes;     // stages x stage_bytes

  if (threadIdx.x == 0) {
    for (int s = 0; s < p.stages; ++s) {
      mbar_init(&bars.full[s], 1);   // loader expect_tx
      mbar_init(&bars.empty[s], 1);  // MMA commit
    }
    for (int h = 0; h < 2; ++h) {
      mbar_init(&bars.hfull[h], kConvWarps);  // one arrival per converter warp
      mbar_init(&bars.hempty[h], 1);          // MMA commit
      mbar_init(&bars.dfull[h], 1);           // MMA commit
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
  // Nothing above touches global memory, so it may overlap the previous
  // kernel in the stream (programmatic serialisation).  When that kernel is
  // this launch's own filter pack, only the packed operand is still being
  // written: the pack waited for every earlier grid before it let this one
  // start, so the input is complete and the output no longer read, and only
  // the loader (which reads the packed operand) waits here.
  if (!p.after_pack) grid_dependency_wait();
  allow_dependent_launch();

  volatile int *abort_flag = &bars.abort_flag;

  if (warp < kConvWarps) {
    // ------------------------------------------------------------ converters
    const int nkg = p.CB / 8;                   // 2, 4 or 8 core-matrix columns
    const uint32_t kgs = (uint32_t)p.L * 16;     // bytes between them
    const size_t plane = (size_t)g.H * g.W;
    uint32_t hb = 0;
    bool failed = false;
    for (int i = blockIdx.x; i < p.total && !failed; i += gridDim.x) {
      const Item it = decode(p, i);
      const int p0 = it.tile * p.tile_adv;
      // strided input row / column of halo position 0
      const int rho = it.ph / p.up, kap = it.ph - rho * p.up;
      const int row0 = p.up > 1 ? p.up_sr[rho] : p.sr_min;
      const int col0 = it.band * p.BW + (p.up > 1 ? p.up_sc[kap] : p.sc_min);
      const float *xb = p.x + (size_t)it.b * g.n * plane;
      for (int cb = 0; cb < p.NCB; ++cb, ++hb) {
        const int buf = hb & 1;
        if (*abort_flag || !mbar_wait(&bars.hempty[buf], ((hb >> 1) & 1) ^ 1, p.err)) {
          failed = true;
          break;
        }
        uint8_t *hbase = halo + (size_t)buf * p.halo_bytes;
        const int cv = g.n - cb * p.CB;  // planes of this block that exist
        const float *xc = xb + (size_t)cb * p.CB * plane;
        if constexpr (CB16) {
          // 16-plane blocks: the (phase, position) items two at a time, both
          // items' loads issued before either is converted, so a thread has
          // as many loads in flight as with a 32-plane position
          const int total = p.nphase * p.L;
          for (int it = threadIdx.x; it < total; it += 2 * kConvThreads) {
            const float *src[2];
            bool in[2];
            uint8_t *dst[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int item = min(it + e * kConvThreads, total - 1);
              const int ph = item / p.L, q = item - ph * p.L;
              const int G = p0 + q;
              const int Y = G / p.P, X = G - Y * p.P;
              const int iy = g.down * (Y + row0) + p.phase_r[ph];
              const int ix = g.down * (col0 + X) + p.phase_c[ph];
              int ry, rx;
              in[e] = border_map(g, iy, ix, ry, rx);
              src[e] = in[e] ? xc + (size_t)ry * g.W + rx : xc;
              dst[e] = hbase + (size_t)ph * TERMS * p.part_bytes + (size_t)q * 16;
            }
            float va[16], vb[16];
            load_kgroups<2>(src[0], plane, in[0], cv, va);
            load_kgroups<2>(src[1], plane, in[1], cv, vb);
            store_kgroups<TERMS, 2>(va, dst[0], kgs, p.part_bytes);
            if (it + kConvThreads < total) store_kgroups<TERMS, 2>(vb, dst[1], kgs, p.part_bytes);
          }
        } else {
          for (int ph = 0; ph < p.nphase; ++ph) {
            uint8_t *hph = hbase + (size_t)ph * TERMS * p.part_bytes;
            for (int q = threadIdx.x; q < p.L; q += kConvThreads) {
              const int G = p0 + q;
              const int Y = G / p.P, X = G - Y * p.P;
              const int iy = g.down * (Y + row0) + p.phase_r[ph];
              const int ix = g.down * (col0 + X) + p.phase_c[ph];
              int ry, rx;
              const bool in = border_map(g, iy, ix, ry, rx);
              const float *src = in ? xc + (size_t)ry * g.W + rx : xc;
              uint8_t *dst = hph + (size_t)q * 16;
              int kg = 0;
              for (; kg + 4 <= nkg; kg += 4)
                convert_kgroups<TERMS, 4>(src + (size_t)kg * 8 * plane, plane, in, cv - kg * 8, dst + (size_t)kg * kgs,
                                          kgs, p.part_bytes);
              for (; kg < nkg; kg += 2)
                convert_kgroups<TERMS, 2>(src + (size_t)kg * 8 * plane, plane, in, cv - kg * 8, dst + (size_t)kg * kgs,
                                          kgs, p.part_bytes);
            }
          }
        }
        // the tensor core reads the halo through the async proxy
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(&bars.hfull[buf]);
      }
    }
    if (failed) *abort_flag = 1;
    if (helpers_store_last(p) && blockIdx.x < p.total && warp < 8) {
      // The CTA's last tile, upper half of the columns: wait for its
      // accumulator (one segment per item, so the phases of each buffer are
      // waited in order), then store through tiles in the halo, which no MMA
      // reads any more.
      constexpr int G = PAIR ? 4 : 2;
      int i_last = blockIdx.x, nitems = 0;
      for (int i = blockIdx.x; i < p.total; i += gridDim.x, ++nitems) i_last = i;
      const uint32_t u = (uint32_t)nitems - 1;  // the last item's segment (one per item)
      const int bi = (int)(u & 1);
      const uint32_t use = u >> 1;
      const int quarter = warp & 3, chalf = warp >> 2;  // converter warps 0-7: lane quarter, column quarter
      const int grp = PAIR ? chalf : (quarter & 1) * 2 + chalf;
      const int part = PAIR ? quarter : (quarter < 2 ? 0 : 1);
      const int bar_id = 6 + grp;  // epilogue groups use 2-5
      // every converter warp comes here, failed or not, so both (or all
      // four) warps of a group reach the barrier; they agree to skip if any
      // of them failed or the wait gives up
      bool bad = failed || *abort_flag != 0;
      if (!bad) bad = !mbar_wait(&bars.dfull[bi], use & 1, p.err);
      bad = named_sync_or(bar_id, 32 * G, bad);
      if (!bad) {
        tc_fence_after();
        const uint32_t sc = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)bi * kAccCols;
        float *tiles = reinterpret_cast<float *>(halo) + grp * G * kXchFloats;
        const int ncol = p.N / 4;
        store_tile_columns<TERMS, PAIR>(p, decode(p, i_last), sc, sc, true, p.N / 2 + chalf * ncol, ncol, tiles,
                                        bar_id, quarter, part, lane, nullptr);
      } else {
        *abort_flag = 1;
      }
    }
  } else if (warp == kMmaWarp) {
    // ------------------------------------------------------------ MMA issuer
    using ML = MmaList<TERMS, PAIR>;
    const uint32_t idesc = idesc_bf16_f32(128, p.N);
    // Operand descriptors are a template (layout, strides) plus the address
    // in 16-byte units; shared-memory addresses stay below 256 KB, so the
    // address field never carries into the stride fields.
    const uint64_t a_tmpl = smem_desc_kmajor(0, 128, (uint32_t)p.CB * 16);
    const uint64_t b_tmpl = smem_desc_kmajor(0, (uint32_t)p.L * 16, 128);
    const uint32_t stage0 = smem_u32(stage) >> 4, halo0 = smem_u32(halo) >> 4;
    const uint32_t chunk16 = p.chunk_bytes >> 4, part16 = p.part_bytes >> 4, stage16 = p.stage_bytes >> 4;
    const uint32_t kstep_b16 = 2u * p.L;              // B: two plane groups of L positions
    const uint32_t row16 = (uint32_t)p.CB / 8;        // A: one filter row (CB bf16) in 16-byte units
    // The issuing thread's own latency bounds the stage rate, so the loop
    // keeps to 32-bit descriptor words (the address field never carries into
    // the stride fields), per-MMA operand offsets in registers, the B offset
    // of each unit in a shared table, and stage / phase counters without
    // divisions.
    const uint32_t a_hi = (uint32_t)(a_tmpl >> 32), b_hi = (uint32_t)(b_tmpl >> 32);
    const uint32_t a_lo0 = (uint32_t)a_tmpl + stage0, b_lo0 = (uint32_t)b_tmpl + halo0;
    uint32_t aoff[ML::n], boff[ML::n];
#pragma unroll
    for (int m = 0; m < ML::n; ++m) {
      aoff[m] = (uint32_t)ML::arow(m) * row16;
      boff[m] = (uint32_t)ML::bterm(m) * part16;
    }
    int s = 0;             // stage slot
    uint32_t sph = 0;      // parity of the slot's current fill
    uint32_t hb = 0, u = 0;
    int table_key = -1;    // (sub-filter width, units) the unit table holds
    bool failed = false;
    for (int i = blockIdx.x; i < p.total && !failed; i += gridDim.x) {
      const ItemUnits iu = item_units<PAIR>(p, decode(p, i));
      if (iu.ts * 1024 + iu.nu != table_key) {
        // (re)written whenever the sub-filter width or the unit count changes
        // (output phases of UpsampleInput), so every unit k < nu has its entry
        // B offset of each unit (paired: of its first tap), in 16-byte units
        const int hs = PAIR ? (iu.ts + 1) / 2 : iu.ts;  // units per filter row
        for (int k = lane; k < iu.nu; k += 32) {
          const int tap = (k / hs) * p.tstride + (PAIR ? 2 : 1) * (k % hs);
          unit_boff[k] = (uint32_t)p.tap_phase[tap] * TERMS * part16 + (uint32_t)p.tap_off[tap];
        }
        __syncwarp();
        table_key = iu.ts * 1024 + iu.nu;
      }
      const int tstages = p.NCB * iu.nst;
      int seg_left = 0, done = 0, bi = 0;
      bool first = false;
      for (int cb = 0; cb < p.NCB && !failed; ++cb, ++hb) {
        const int buf = hb & 1;
        failed = __any_sync(0xffffffffu, *abort_flag || !mbar_wait(&bars.hfull[buf], (hb >> 1) & 1, p.err));
        if (failed) break;
        tc_fence_after();
        const uint32_t hlo = b_lo0 + (uint32_t)buf * (p.halo_bytes >> 4);
        for (int st = 0; st < iu.nst; ++st) {
          if (seg_left == 0) {
            // a new accumulation segment: wait until its accumulator is free
            bi = p.promote ? 0 : (int)(u & 1);
            const uint32_t use = p.promote ? u : (u >> 1);
            failed = __any_sync(0xffffffffu, !mbar_wait(&bars.dempty[bi], (use & 1) ^ 1, p.err));
            if (failed) break;
            tc_fence_after();
            seg_left = min(p.seg_stages, tstages - done);
            first = true;
          }
          failed = __any_sync(0xffffffffu, !mbar_wait(&bars.full[s], sph, p.err));
          if (failed) break;
          tc_fence_after();
          if (elect_one()) {
            const uint32_t dt = tmem + (uint32_t)bi * kAccCols;
            const int u0 = st * p.T, u1 = min(iu.nu, u0 + p.T);
            uint32_t alo = a_lo0 + (uint32_t)s * stage16;
            for (int k = u0; k < u1; ++k, alo += chunk16) {
              const uint32_t blo = hlo + unit_boff[k];
              for (int j = 0; j < p.KS; ++j) {
#pragma unroll
                for (int m = 0; m < ML::n; ++m) {
                  mma_bf16_ss(dt, desc_word(a_hi, alo + aoff[m] + 16u * j),
                              desc_word(b_hi, blo + boff[m] + (uint32_t)j * kstep_b16), idesc,
                              (first && m == 0) ? 0u : 1u);
                  first = false;
                }
              }
            }
            tc_commit(&bars.empty[s]);  // the stage may be refilled once these MMAs are done
          }
          __syncwarp();
          if (++s == p.stages) {
            s = 0;
            sph ^= 1u;
          }
          first = false;
          ++done;
          if (--seg_left == 0) {
            if (elect_one()) tc_commit(&bars.dfull[bi]);
            __syncwarp();
            ++u;
          }
        }
        if (failed) break;
        if (elect_one()) tc_commit(&bars.hempty[buf]);  // the halo buffer may be refilled
        __syncwarp();
      }
    }
    if (failed) *abort_flag = 1;
    // Every MMA issued retires before tensor and shared memory are released.
    if (elect_one()) tc_commit(&bars.drain);
    __syncwarp();
    mbar_wait(&bars.drain, 0, p.err);
  } else if (warp == kLoadWarp) {
    // ------------------------------------------------------------ loader
    // A bulk copy costs its issuing thread a few hundred cycles whatever its
    // size, so each stage (T consecutive taps of one plane block, contiguous
    // in the packed operand) is one copy.
    if (lane == 0) {
      if (p.after_pack) grid_dependency_wait();
      uint32_t q = 0;     // stages issued
      int s = 0;          // stage slot
      uint32_t sph = 0;   // parity of the slot's current fill
      bool ok = true;
      for (int i = blockIdx.x; ok && i < p.total && !*abort_flag; i += gridDim.x) {
        const ItemUnits iu = item_units<PAIR>(p, decode(p, i));
        const int NU = iu.nu;
        const uint8_t *src = p.bpack + iu.chunk0 * p.chunk_bytes;
        for (int cb = 0; ok && cb < p.NCB; ++cb)
          for (int st = 0; st < iu.nst; ++st, ++q) {
            if (!mbar_wait(&bars.empty[s], sph ^ 1u, p.err)) {
              ok = false;
              break;
            }
            const int t0 = st * p.T;
            const uint32_t bytes = (uint32_t)min(p.T, NU - t0) * p.chunk_bytes;
            mbar_arrive_expect_tx(&bars.full[s], bytes);
            bulk_load(stage + (size_t)s * p.stage_bytes, src + ((size_t)cb * NU + t0) * p.chunk_bytes, bytes,
                      &bars.full[s]);
            if (++s == p.stages) {
              s = 0;
              sph ^= 1u;
            }
          }
      }
      if (!ok) *abort_flag = 1;
      if (*abort_flag) {
        // copies still in flight land before shared memory is released
        for (uint32_t qq = q > (uint32_t)p.stages ? q - p.stages : 0; qq < q; ++qq)
          mbar_wait(&bars.full[qq % p.stages], (qq / p.stages) & 1, p.err);
      }
    }
  } else {
    // ------------------------------------------------------------ epilogue
    // Lane quarters: rows 0-63 hold hi*hi sums, rows 64-127 corrections; with
    // paired taps the quarters are tap a's hi*hi, tap b's hi*hi, a's and b's
    // corrections, tap b's one grid position to the right.  The warps holding
    // the parts of one block of 32 filters for the same columns form a group
    // (two warps, or with paired taps four): store_tile_columns.
    constexpr int G = PAIR ? 4 : 2;  // parts (warps) per group
    const int ew = warp - kEpiWarp0;
    const int quarter = warp & 3;         // tensor-memory lanes this warp may access
    const int half = ew >> 2;             // column half
    const int grp = PAIR ? half : (quarter & 1) * 2 + half;
    const int part = PAIR ? quarter : (quarter < 2 ? 0 : 1);  // this warp's part, and its share of filters
    const int bar_id = 2 + grp, bar_count = 32 * G;
    const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
    float *tiles = xch + grp * G * kXchFloats;  // the group's part tiles, [part][filter][pitch 17]
    const bool helped = helpers_store_last(p);
    uint32_t u = 0;
    bool failed = false;
    for (int i = blockIdx.x; i < p.total && !failed; i += gridDim.x) {
      const Item it = decode(p, i);
      const ItemUnits iu = item_units<PAIR>(p, it);
      const int nseg = (p.NCB * iu.nst + p.seg_stages - 1) / p.seg_stages;  // accumulation segments
      // the CTA's last tile: the converters store the upper half of the columns
      const bool last_item = i + (int)gridDim.x >= p.total;
      const int ncol = (helped && last_item) ? p.N / 4 : p.N / 2;
      const int cbeg = half * ncol;
      for (int seg = 0; seg < nseg; ++seg, ++u) {
        const int bi = p.promote ? 0 : (int)(u & 1);
        const uint32_t use = p.promote ? u : (u >> 1);
        bool bad = *abort_flag != 0 || !mbar_wait(&bars.dfull[bi], use & 1, p.err);
        bad = named_sync_or(bar_id, bar_count, bad);  // the group agrees
        if (bad) {
          failed = true;
          break;
        }
        tc_fence_after();
        const uint32_t sc = tmem + lane_base + (uint32_t)bi * kAccCols;
        const uint32_t rc = tmem + lane_base + kAccCols;  // running sum (promotion)
        const bool first = seg == 0, last = seg == nseg - 1;
        if (!last) {
          // promotion: R (+)= S, FP32 round to nearest, over the warp's column half
          for (int c = half * (p.N / 2); c < (half + 1) * (p.N / 2); c += 16) {
            uint32_t s16[16], r16[16];
            tmem_ld16(sc + c, s16);
            if (!first) tmem_ld16(rc + c, r16);
            tc_wait_ld();
            if (!first) {
#pragma unroll
              for (int t = 0; t < 16; ++t) s16[t] = __float_as_uint(__uint_as_float(s16[t]) + __uint_as_float(r16[t]));
            }
            tmem_st16(rc + c, s16);
          }
          tc_wait_st();
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&bars.dempty[bi]);
          continue;
        }
        // last segment: out = S (+ R) for every part of each filter
        store_tile_columns<TERMS, PAIR>(p, it, sc, rc, first, cbeg, ncol, tiles, bar_id, quarter, part, lane,
                                        &bars.dempty[bi]);
      }
    }
    if (failed) *abort_flag = 1;
  }

  // ---------------------------------------------------------------- teardown
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kMmaWarp) tmem_dealloc(tmem, 512);
}

// Pack the filter bank into per-chunk operand images: chunk (output phase,
// nb, cb, unit) = arows x CB bf16, column ci = plane cb*CB + ci, the filter
// value of the tap (flipped for convolution).  A unit is one tap, with row
// blocks of 64 as block_term() lists and row n of a block = filter nb*64 + n;
// or, paired, two taps a, a + 1 of a filter row, with row blocks of 32 as
// pair_block_term() and pair_block_tap() list and row n of a block = filter
// nb*32 + n (tap a + 1 past the row's end is 0).  With UpsampleInput the
// taps of a unit are those of its phase's sub-filter.  Layout: core matrices
// of 8 rows x 8 columns (128 bytes), row groups SBO = CB*16 bytes apart,
// column groups LBO = 128 bytes apart.  Rows or columns past the real counts
// are 0.
//
// One thread per core-matrix row (8 planes of one filter row: 8 loads in
// flight, one 16-byte store).  The launch is one CTA of 128 threads per SM:
// at 32 registers a thread its four warps fit in the registers a
// filter-bank CTA leaves free on each SM sub-partition, so with programmatic
// serialisation it is resident before the previous launch ends and runs the
// moment that launch is done (measured: 1.6 / 2.3 us less per forward /
// backward launch than one thread per value in 256-thread CTAs).
template <bool PAIR>
__global__ void __launch_bounds__(kPackThreads, 16) bank_pack_kernel(const __grid_constant__ BankParams p,
                                                                     const float *__restrict__ f,
                                                                     uint8_t *__restrict__ out) {
  const ConvGeom &g = p.g;
  const int CB8 = p.CB / 8, arows = p.arows;
  // every (phase, block, plane block, unit) slot of the largest phase; the
  // units a phase lacks are skipped.  Below 2^31 (checked at launch).
  const int total = p.nph_out * p.nblocks * p.NCB * p.nunits * arows * CB8;
  // the previous kernel (the last launch that read the packed operand) must
  // be done before it is rewritten; the consuming kernel may be scheduled now
  grid_dependency_wait();
  allow_dependent_launch();
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
    const int c8 = idx % CB8;
    int rest = idx / CB8;
    const int row = rest % arows;
    rest /= arows;
    const int unit = rest % p.nunits;
    rest /= p.nunits;
    const int cb = rest % p.NCB;
    rest /= p.NCB;
    const int nb = rest % p.nblocks;
    Item it{};
    it.ph = rest / p.nblocks;
    it.nb = nb;
    const ItemUnits iu = item_units<PAIR>(p, it);
    if (unit >= iu.nu) continue;
    const int hs = PAIR ? (iu.ts + 1) / 2 : iu.ts;
    int part, k, ss;
    if (PAIR) {
      const int blk = row >> 5;
      part = pair_block_term(blk);
      k = nb * 32 + (row & 31);
      ss = 2 * (unit % hs) + pair_block_tap(blk);
    } else {
      part = block_term(p.terms, row >> 6);
      k = nb * 64 + (row & 63);
      ss = unit % hs;
    }
    const int rr = unit / hs;
    int r = rr, s = ss;
    if (p.up > 1) {
      const int rho = it.ph / p.up;
      r = p.up_r0[rho] + p.up * rr;
      s = p.up_s0[it.ph - rho * p.up] + p.up * ss;
    }
    const bool live = part >= 0 && ss < iu.ts && r < g.R && s < g.S && k < g.groups;
    const int src = g.orient == CCT_CONVOLUTION ? (g.R - 1 - r) * g.S + (g.S - 1 - s) : r * g.S + s;
    // filter plane of (filter k, plane c), as plane_pair gives it: k*n + c
    // for projectFrame, c*groups + k for backProjectFrame
    const bool fwd = g.mode == CCT_PROJECT_FRAME_BLOCK_REDUCE_SUM;
    const int c0 = cb * p.CB + c8 * 8;
    const size_t taps = (size_t)g.R * g.S;
    const size_t fstride = fwd ? taps : (size_t)g.groups * taps;
    const float *fp = f + (fwd ? (size_t)k * g.n + c0 : (size_t)c0 * g.groups + k) * taps + src;
    float a[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) a[e] = (live && c0 + e < g.n) ? __ldg(fp + (size_t)e * fstride) : 0.0f;
    uint32_t w[4];
#pragma unroll
    for (int e = 0; e < 8; e += 2) {
      float v[2];
#pragma unroll
      for (int d = 0; d < 2; ++d) {
        const float x = a[e + d];
        const float h = __bfloat162float(__float2bfloat16_rn(x));
        if (part <= 0) {
          v[d] = h;  // a zero block holds x = 0
        } else if (p.terms == 2) {
          v[d] = x - h;  // rounded to bf16 below
        } else {
          const float m = __bfloat162float(__float2bfloat16_rn(x - h));
          v[d] = part == 1 ? m : (x - h) - m;
        }
      }
      const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[0], v[1]);  // v[0] in the low half
      w[e / 2] = *reinterpret_cast<const uint32_t *>(&b2);
    }
    const size_t chunk = iu.chunk0 + (size_t)cb * iu.nu + unit;
    const uint32_t off = (uint32_t)((row >> 3) * (p.CB * 16) + c8 * 128 + (row & 7) * 16);
    *reinterpret_cast<uint4 *>(out + chunk * ((size_t)arows * p.CB * 2) + off) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

std::mutex g_bank_mu;
std::unordered_map<uint64_t, size_t> g_bank_attr;

template <int TERMS, bool PAIR, bool CB16>
int launch_terms(const BankParams &p, cudaStream_t st) {
  auto kern = bank_tc_kernel<TERMS, PAIR, CB16>;
  {
    // Dynamic shared memory above 48 KB needs the opt-in attribute; keep the
    // largest size set so far per (device, instance).
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t key = ((uint64_t)dev << 32) | (uint64_t)(TERMS * 4 + (PAIR ? 2 : 0) + (CB16 ? 1 : 0));
    std::lock_guard<std::mutex> lk(g_bank_mu);
    size_t &have = g_bank_attr[key];
    if (have < p.smem_bytes) {
      const int rc = check_cuda(cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)p.smem_bytes),
                                "cudaFuncSetAttribute(bank_tc)");
      if (rc) return rc;
      have = p.smem_bytes;
    }
  }
  const int rc = launch_pdl(kern, dim3(p.grid), dim3(kThreads), p.smem_bytes, st, "bank_tc_kernel launch", p);
  if (rc) return rc;
  count_launches(1);
  return check_cuda(cudaGetLastError(), "bank_tc_kernel launch");
}

int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }
int pos_mod(int a, int b) { return ((a % b) + b) % b; }

}  // namespace

bool bank_tc_plan(const ConvGeom &g, int terms, int sms, BankParams *out) {
  if (g.mode != CCT_PROJECT_FRAME_BLOCK_REDUCE_SUM && g.mode != CCT_BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM)
    return false;
  if (terms != 2 && terms != 3) return false;
  if (g.fup != 1 || g.down < 1 || g.down > 2 || g.up < 1 || g.up > kBankMaxUp) return false;
  if (g.up > 1 && (g.down != 1 || g.border == CCT_BORDER_CLAMP)) return false;
  const int RS = g.R * g.S;
  if (RS > kBankMaxTaps || g.n < 1 || g.groups < 1) return false;
  BankParams p{};
  p.g = g;
  p.terms = terms;
  const int d = g.down, u = g.up;
  p.up = u;
  p.nph_out = u * u;
  int dr, dc;  // reach of the (sub-)filter on the grid, rows and columns
  int rq_max = 1, sq_max = 1;
  if (u > 1) {
    // UpsampleInput (ConvolveHyperKernel.scala:206-212, 405-459): output row
    // i = u*I + rho takes filter rows r with (rho - low_r + r) % u == 0, that
    // is r = r0 + u*rr, reading input row I + (rho - low_r + r0)/u + rr.
    // Phases without such rows keep one zero sub-filter row, so every phase
    // writes its outputs.
    for (int ph = 0; ph < u; ++ph) {
      const int r0 = pos_mod(g.low_r - ph, u), s0 = pos_mod(g.low_c - ph, u);
      p.up_r0[ph] = r0;
      p.up_s0[ph] = s0;
      p.up_rq[ph] = std::max(1, r0 < g.R ? (g.R - 1 - r0) / u + 1 : 0);
      p.up_sq[ph] = std::max(1, s0 < g.S ? (g.S - 1 - s0) / u + 1 : 0);
      p.up_sr[ph] = floor_div(ph - g.low_r + r0, u);
      p.up_sc[ph] = floor_div(ph - g.low_c + s0, u);
      rq_max = std::max(rq_max, p.up_rq[ph]);
      sq_max = std::max(sq_max, p.up_sq[ph]);
    }
    dr = rq_max - 1;
    dc = sq_max - 1;
    p.OHq = (g.OH + u - 1) / u;
    p.OWq = (g.OW + u - 1) / u;
    p.nphase = 1;
    p.tstride = sq_max;
  } else {
    // row / column shifts in strided units and the input phases the taps read
    p.sr_min = floor_div(-g.low_r, d);
    p.sc_min = floor_div(-g.low_c, d);
    dr = floor_div(g.R - 1 - g.low_r, d) - p.sr_min;
    dc = floor_div(g.S - 1 - g.low_c, d) - p.sc_min;
    p.OHq = g.OH;
    p.OWq = g.OW;
    p.tstride = g.S;
    rq_max = g.R;
    sq_max = g.S;
  }
  if (rq_max * p.tstride > kBankMaxTaps) return false;
  // Banks of at most 32 filters would leave half of each 128-row MMA empty:
  // two taps of a filter row share it instead (stride-1 grids only, where
  // tap a + 1 reads one grid position past tap a).
  p.pair = (terms == 2 && g.groups <= 32 && d == 1 && sq_max >= 2) ? 1 : 0;
  p.fblock = p.pair ? 32 : 64;
  p.nblocks = (g.groups + p.fblock - 1) / p.fblock;
  // units per phase: sub-filter rows x (columns, or column pairs)
  auto units_of = [&](int rows, int cols) { return rows * (p.pair ? (cols + 1) / 2 : cols); };
  p.nunits = 0;
  for (int ph = 0; ph < p.nph_out; ++ph) {
    const int nu = u > 1 ? units_of(p.up_rq[ph / u], p.up_sq[ph % u]) : units_of(g.R, g.S);
    p.nunits = std::max(p.nunits, nu);
  }
  p.nmma = terms == 2 ? 2 : 5;
  p.arows = terms == 2 ? 192 : 448;
  const size_t xch_bytes = kXchBytes;
  const int NU = p.nunits;
  int phase_of[2][2] = {{-1, -1}, {-1, -1}};
  if (u > 1) {
    phase_of[0][0] = 0;
  } else {
    for (int r = 0; r < g.R; ++r)
      for (int s = 0; s < g.S; ++s) {
        const int pr = pos_mod(r - g.low_r, d), pc = pos_mod(s - g.low_c, d);
        if (phase_of[pr][pc] < 0) {
          phase_of[pr][pc] = p.nphase;
          p.phase_r[p.nphase] = pr;
          p.phase_c[p.nphase] = pc;
          ++p.nphase;
        }
      }
  }
  // Band width BW, tile size N (positions) and plane block CB, by a cost
  // model: an M=128, 16-deep MMA over N positions takes N/2 tensor cycles and
  // reads 4 KB of filter plus 32*N bytes of halo from shared memory at about
  // 128 B per cycle, so its time is max(N/2, 32 + N/4) cycles; each tile also
  // pays a fixed hand-off (about 8 cycles per k-step).  Grid columns past a
  // band's outputs are paid for too, and the work items (image, band, tile,
  // filter block) run in waves of one per SM.  The
  // plan needs two halo buffers, at least three filter stages and the
  // epilogue's exchange buffers in shared memory; among equal costs the
  // larger plane block wins (fewer halo hand-offs).
  // dynamic shared memory: 227 KB per CTA less the static barriers and exchange buffers
  const size_t budget = 225 * 1024;
  const int cmax = ((g.n + 15) / 16) * 16;
  bool found = false;
  double best_cost = 0.0;
  int best_cb = 0;
  for (int bw : {p.OWq, 512, 256, 192, 128, 96, 64, 48, 32}) {
    if (bw > p.OWq || (bw == p.OWq && bw > 1024)) continue;
    const int nbands = (p.OWq + bw - 1) / bw;
    const int BW = (p.OWq + nbands - 1) / nbands;  // balanced bands
    const int P = BW + dc;
    const long long npos = (long long)p.OHq * P;
    for (int N : {256, 224, 192, 160, 128, 96, 64}) {
      const int adv = p.pair ? N - 4 : N;  // paired: the last 4 positions of a tile lack tap b's sums
      const long long tiles = (npos + adv - 1) / adv;
      const int L = ((N + dr * P + dc) + 7) & ~7;
      for (int CB : {64, 32, 16}) {
        if (CB > cmax && CB != 16) continue;
        const size_t part = (size_t)L * CB * 2;
        const size_t halo = (((size_t)p.nphase * terms * part) + 127) & ~(size_t)127;
        const size_t chunk = (size_t)p.arows * CB * 2;
        // Units per stage: each stage hand-off (the MMA thread's wait and
        // commit, the loader's refill) costs ~400 cycles of the issuing
        // thread's latency whatever the stage holds, so a stage takes as many
        // units as fit, up to ~2000 cycles of MMAs, in three stages; two
        // stages do when a stage holds at least ~1500 cycles of MMAs, enough
        // to cover the refill of the other (measured: 12 MMAs of N = 256 in
        // two stages beat 8 in three).
        const double tap_cycles = (CB / 16) * p.nmma * std::max(0.5 * N, 32.0 + 0.25 * N);
        auto fits = [&](int t, int st) { return 2 * halo + (size_t)st * t * chunk + xch_bytes <= budget; };
        auto ok_stages = [&](int t) { return fits(t, 3) || (fits(t, 2) && t * tap_cycles >= 1500.0); };
        int T = std::min(NU, std::max(1, (int)(2000.0 / tap_cycles)));
        while (T > 1 && !ok_stages(T)) --T;
        if (!ok_stages(T) || L * 16 >= (1 << 18)) continue;
        if (T * tap_cycles < 500.0 && T < NU && CB > 16) continue;  // a smaller plane block keeps stages long
        // work items run in waves over the SMs: a small problem takes smaller
        // tiles to occupy more of them
        const long long items = (long long)g.batch * p.nph_out * nbands * tiles * p.nblocks;
        const double waves = (double)((items + sms - 1) / sms);
        const double cost = waves * (std::max(0.5 * N, 32.0 + 0.25 * N) + 8.0);
        if (!found || cost < best_cost * 0.999 || (cost <= best_cost * 1.001 && CB > best_cb)) {
          p.nbands = nbands;
          p.BW = BW;
          p.P = P;
          p.N = N;
          p.CB = CB;
          p.L = L;
          p.part_bytes = (uint32_t)part;
          p.halo_bytes = (uint32_t)halo;
          p.chunk_bytes = (uint32_t)chunk;
          p.T = T;
          p.stage_bytes = (uint32_t)(T * chunk);
          p.stages = (int)std::min<size_t>(6, (budget - 2 * halo - xch_bytes) / p.stage_bytes);
          p.tile_adv = adv;
          p.tiles_band = (int)tiles;
          best_cost = cost;
          best_cb = CB;
          found = true;
        }
        break;  // the largest plane block that fits
      }
    }
  }
  if (!found) return false;
  if (u > 1) {
    // sub-filter tap (rr, ss) of any phase: grid offset rr*P + ss
    for (int rr = 0; rr < rq_max; ++rr)
      for (int ss = 0; ss < sq_max; ++ss) {
        p.tap_phase[rr * p.tstride + ss] = 0;
        p.tap_off[rr * p.tstride + ss] = rr * p.P + ss;
      }
  } else {
    for (int tap = 0; tap < RS; ++tap) {
      const int r = tap / g.S, s = tap % g.S;
      const int ar = r - g.low_r, ac = s - g.low_c;
      p.tap_phase[tap] = phase_of[pos_mod(ar, d)][pos_mod(ac, d)];
      p.tap_off[tap] = (floor_div(ar, d) - p.sr_min) * p.P + (floor_div(ac, d) - p.sc_min);
    }
  }
  p.NCB = (g.n + p.CB - 1) / p.CB;
  p.KS = p.CB / 16;
  p.nst = (NU + p.T - 1) / p.T;
  const int tstages = p.NCB * p.nst;
  // Promotion: the hi*hi accumulator takes at most 64 k-steps (1024 terms of
  // the reduction) before it is added into the FP32 running sum.
  const int kmax = 64;
  p.promote = p.NCB * NU * p.KS > kmax ? 1 : 0;
  p.seg_stages = p.promote ? std::max(1, kmax / (p.T * p.KS)) : tstages;
  // float4 stores: groups of 4 grid positions (p0, N and tile_adv are multiples of 4)
  // never straddle a grid row or the band's last output column, and land on
  // 16-byte aligned outputs
  // (up-sampled outputs are strided: scalar stores)
  p.vec4 = (u == 1 && p.P % 4 == 0 && p.BW % 4 == 0 && g.OW % 4 == 0 && p.N % 4 == 0) ? 1 : 0;
  const long long total = (long long)g.batch * p.nph_out * p.nbands * p.tiles_band * p.nblocks;
  if (total < 1 || total > 0x7fffffffLL) return false;
  p.total = (int)total;
  p.grid = std::min(p.total, sms);
  p.sms = sms;
  p.smem_bytes = 2 * (size_t)p.halo_bytes + (size_t)p.stages * p.stage_bytes;
  // packed chunks: each output phase's filter blocks, plane blocks and units
  size_t chunks = 0;
  for (int ph = 0; ph < p.nph_out; ++ph) {
    p.up_choff[ph] = (int)chunks;
    const int nu = u > 1 ? units_of(p.up_rq[ph / u], p.up_sq[ph % u]) : NU;
    chunks += (size_t)p.nblocks * p.NCB * nu;
  }
  p.pack_bytes = chunks * p.chunk_bytes;
  *out = p;
  return true;
}

int launch_bank_pack(const BankParams &p, const float *f, uint8_t *packed, cudaStream_t st) {
  const long long total = (long long)p.nph_out * p.nblocks * p.NCB * p.nunits * p.arows * (p.CB / 8);
  if (total > 0x7fffffffLL) return set_error(CCT_ENOTSUP, "packed filter operand too large");
  // one CTA per SM (more would wait for the filter-bank CTAs to leave)
  const int blocks = (int)std::min<long long>((total + kPackThreads - 1) / kPackThreads, p.sms);
  const int rc = p.pair ? launch_pdl(bank_pack_kernel<true>, dim3(blocks), dim3(kPackThreads), 0, st,
                                     "bank_pack_kernel launch", p, f, packed)
                        : launch_pdl(bank_pack_kernel<false>, dim3(blocks), dim3(kPackThreads), 0, st,
                                     "bank_pack_kernel launch", p, f, packed);
  if (rc) return rc;
  count_launches(1);
  return check_cuda(cudaGetLastError(), "bank_pack_kernel launch");
}

int launch_bank_tc(const BankParams &p, const float *x, float *y, const uint8_t *packed, unsigned *err,
                   cudaStream_t st, bool after_pack) {
  BankParams q = p;
  q.after_pack = after_pack ? 1 : 0;
  q.x = x;
  q.y = y;
  if ((reinterpret_cast<uintptr_t>(y) & 15) != 0) q.vec4 = 0;  // float4 stores need a 16-byte aligned output
  q.bpack = packed;
  q.err = err;
  const bool cb16 = p.CB == 16;
  if (p.pair) return cb16 ? launch_terms<2, true, true>(q, st) : launch_terms<2, true, false>(q, st);
  if (p.terms == 2) return cb16 ? launch_terms<2, false, true>(q, st) : launch_terms<2, false, false>(q, st);
  return cb16 ? launch_terms<3, false, true>(q, st) : launch_terms<3, false, false>(q, st);
}

}  // namespace cct

namespace cct {

bool frame_tc_choose(const ConvGeom &g, int precision, int sms, FrameTcChoice *out) {
  FrameTcChoice c{};
  BankParams bp{};
  const bool bank_ok = bank_tc_plan(g, precision == CCT_PREC_BF16X6 ? 3 : 2, sms, &bp);
  if (bank_ok && (bp.pair || g.groups > 32 || precision != CCT_PREC_BF16X3)) {
    c.bank = true;
    c.bp = bp;
    c.pack_bytes = bp.pack_bytes;
  } else if (precision == CCT_PREC_BF16X3 && frame_tc_plan(g, sms, &c.tp)) {
    c.bank = false;
    c.pack_bytes = c.tp.pack_bytes;
  } else if (bank_ok) {
    c.bank = true;
    c.bp = bp;
    c.pack_bytes = bp.pack_bytes;
  } else {
    return false;
  }
  *out = c;
  return true;
}

int frame_tc_pack(const FrameTcChoice &c, const float *f, uint8_t *packed, cudaStream_t st) {
  return c.bank ? launch_bank_pack(c.bp, f, packed, st) : launch_pack_filters(c.tp, f, packed, st);
}

int frame_tc_run(const FrameTcChoice &c, const float *x, float *y, const uint8_t *packed, unsigned *err,
                 cudaStream_t st, bool after_pack) {
  if (c.bank) return launch_bank_tc(c.bp, x, y, packed, err, st, after_pack);
  if ((reinterpret_cast<uintptr_t>(x) & 15) != 0)
    return set_error(CCT_EINVAL, "image pointer must be 16-byte aligned for the tensor-core path");
  return launch_frame_tc(c.tp, x, y, packed, err, st);
}

}  // namespace cct
