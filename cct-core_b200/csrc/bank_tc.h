// Tile plan and launchers of the filter-bank tensor-core kernel (bank_tc.cu):
// fused projectFrame / backProjectFrame (BlockReduceSum) as an implicit GEMM
// with the filter bank as the MMA's M operand and output positions as N.
#pragma once

#include "cct_internal.h"

namespace cct {

constexpr int kBankMaxTaps = 128;   // R * S per tile plan
constexpr int kBankMaxPhases = 4;   // input phases (DownsampleOutput(2): 2 x 2)
constexpr int kBankMaxUp = 4;       // UpsampleInput steps the kernel takes

struct BankParams {
  ConvGeom g;
  int terms;        // bf16 terms per split value: 2 (BF16X3) or 3 (BF16X6)
  int pair;         // 1: banks of at most 32 filters, two taps of a filter row per MMA
  int fblock;       // filters per block: 64, or 32 when paired
  int nunits;       // reduction units per plane block: taps, or tap pairs (R * ceil(S/2));
                    // with UpsampleInput the largest over the output phases
  int tile_adv;     // positions a tile advances: N, or N - 4 when paired
  int nmma;         // MMAs per 16-deep k-step: 2 or 5
  int arows;        // rows of one packed filter chunk (64 per block: 192 or 448)
  int CB;           // input planes per halo block (multiple of 16)
  int NCB;          // ceil(n / CB)
  int KS;           // 16-deep k-steps per chunk: CB / 16
  int N;            // positions per tile (MMA N, multiple of 32, <= 256)
  int P;            // pitch of the padded output grid (positions per grid row)
  int BW;           // output columns per band
  int nbands;       // ceil(OWq / BW)
  int tiles_band;   // tiles per band grid: ceil(OHq * P / tile_adv)
  int nblocks;      // filter blocks: ceil(groups / fblock)
  int total;        // work items: batch * nph_out * nbands * tiles_band * nblocks
  int L;            // halo positions per phase per tile (multiple of 8)
  int nphase;       // input phases held in the halo
  int phase_r[kBankMaxPhases], phase_c[kBankMaxPhases];  // row / column phase of each
  int sr_min, sc_min;  // smallest row / column shift (in strided units)
  int tap_phase[kBankMaxTaps];  // halo phase a tap reads
  int tap_off[kBankMaxTaps];    // position offset of a tap inside its phase
  int tstride;                  // tap index of filter row r, column s: r * tstride + s
  // UpsampleInput(up): each output phase (rho, kappa) = (i mod up, j mod up)
  // is a stride-1 convolution of the field with the sub-filter of taps
  // r = up_r0[rho] + up * rr, s = up_s0[kappa] + up * ss, on an output grid
  // of ceil(OH / up) x ceil(OW / up) positions.  up = 1 otherwise (one phase).
  int up, nph_out;              // step, output phases (up * up)
  int OHq, OWq;                 // output grid of one phase
  int up_r0[kBankMaxUp], up_s0[kBankMaxUp];  // first filter row / column of a phase
  int up_rq[kBankMaxUp], up_sq[kBankMaxUp];  // sub-filter rows / columns of a phase (>= 1)
  int up_sr[kBankMaxUp], up_sc[kBankMaxUp];  // input row / column of sub-tap 0 at grid position 0
  int up_choff[kBankMaxUp * kBankMaxUp];     // first packed chunk of each output phase
  uint32_t part_bytes;   // one split term of one phase: L * CB * 2
  uint32_t halo_bytes;   // one halo buffer: nphase * terms * part_bytes
  uint32_t chunk_bytes;  // one packed filter chunk (one unit, one plane block): arows * CB * 2
  int T;                 // units per stage (one bulk copy of T consecutive chunks)
  int nst;               // stages per (tile, plane block): ceil(nunits / T), the most of any phase
  uint32_t stage_bytes;  // T * chunk_bytes
  int stages;            // stage pipeline depth
  int seg_stages;        // stages per accumulation segment
  int promote;           // 1: segments are promoted into an FP32 running sum
  int vec4;              // 1: groups of 4 positions map to 4 aligned consecutive outputs (float4 stores)
  int grid;              // persistent CTAs
  int sms;               // SMs of the device
  size_t smem_bytes;     // dynamic shared memory
  size_t pack_bytes;     // bytes of the packed filter operand
  int after_pack;        // 1: the preceding grid in the stream is this launch's filter pack
  const float *x;
  const uint8_t *bpack;
  float *y;
  unsigned *err;
};

// terms: 2 or 3.  False when the shape is outside what the kernel handles.
bool bank_tc_plan(const ConvGeom &g, int terms, int sms, BankParams *out);
int launch_bank_pack(const BankParams &p, const float *f, uint8_t *packed, cudaStream_t st);
// after_pack: the launch directly follows its own filter pack on `st`.
int launch_bank_tc(const BankParams &p, const float *x, float *y, const uint8_t *packed,
                   unsigned *err, cudaStream_t st, bool after_pack = false);

}  // namespace cct

#include "frame_tc.h"

namespace cct {

// The tensor-core frame kernel a shape runs on: the filter-bank kernel
// (bank_tc.cu), with paired taps for banks of at most 32 output planes; where
// pairing does not apply to such a bank (DownsampleOutput(2), one-column
// filters) and the filter-bank kernel's 128-row MMA would be half empty, the
// positions-major kernel (frame_tc.cu) when it takes the shape.  Plans and
// the allocation-free entry point make the same choice.
struct FrameTcChoice {
  bool bank;        // true: bank_tc, false: frame_tc
  BankParams bp;
  TcParams tp;
  size_t pack_bytes;
};
// precision: CCT_PREC_BF16X3 or CCT_PREC_BF16X6 (bank_tc only).
bool frame_tc_choose(const ConvGeom &g, int precision, int sms, FrameTcChoice *out);
int frame_tc_pack(const FrameTcChoice &c, const float *f, uint8_t *packed, cudaStream_t st);
// after_pack: frame_tc_pack was the last launch on `st`.
int frame_tc_run(const FrameTcChoice &c, const float *x, float *y, const uint8_t *packed, unsigned *err,
                 cudaStream_t st, bool after_pack = false);

}  // namespace cct
