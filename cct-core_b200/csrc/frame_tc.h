// Tile plan and launchers of the tensor-core (split-BF16) frame kernel.
#pragma once

#include <cuda.h>

#include "cct_internal.h"

namespace cct {

struct TcParams {
  ConvGeom g;
  int tiles_m;      // 128-pixel tiles per image
  int NT;           // output planes per tile (MMA N, multiple of 16, <= 128)
  int nblocks;      // ceil(groups / NT)
  int total_tiles;  // batch * tiles_m * nblocks
  int TR, TC;       // halo box rows / cols (TC multiple of 4)
  int start_c;      // box x origin, a multiple of 4
  int CB;           // input planes per reduction chunk (16, 32 or 64)
  int NCB;          // ceil(n / CB)
  int grid;         // persistent CTAs
  uint32_t halo_bytes;
  size_t pack_bytes;  // bytes of the packed filter operand
  const uint8_t *bpack;
  float *y;
  unsigned *err;
};

bool frame_tc_plan(const ConvGeom &g, int sms, TcParams *out);
int launch_pack_filters(const TcParams &p, const float *f, uint8_t *packed, cudaStream_t st);
int launch_frame_tc(const TcParams &p, const float *x, float *y, const uint8_t *packed,
                    unsigned *err, cudaStream_t st);

}  // namespace cct
