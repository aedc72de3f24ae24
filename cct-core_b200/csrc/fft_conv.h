// FFT convolution plan and launchers.
#pragma once

#include <vector>

#include "cct_internal.h"

namespace cct {

struct FftParams {
  ConvGeom g;
  int Fr, Fc;         // expanded (power-of-two) grid
  int logN, logR;     // log2(Fc/2), log2(Fr)
  int ld;             // spectrum row length: Fc/2 + 1
  float scale;        // 1 / (Fr * Fc/2), folded into the filter spectrum
  size_t spec_elems;  // complex elements of the working spectrum (all output planes)
  size_t filter_elems;  // complex elements of the filter spectra (all filter planes)
  size_t tw_elems;    // complex twiddles: Fc/2 + Fr + (Fc/2 + 1)
  const float2 *tw_n, *tw_r, *tw_2n;
};

bool fft_plan(const ConvGeom &g, FftParams *out);
void fft_twiddles(const FftParams &p, std::vector<float> *host);
void fft_set_tables(FftParams *p, float2 *tw);
// FP64 host spectrum of a static filter (scaled), as float2 pairs.
void fft_static_spectrum(const FftParams &p, const float *host_filter, std::vector<float> *out);
int launch_fft_filter_spectrum(const FftParams &p, const float *f, float2 *G, cudaStream_t st);
int launch_fft_conv(const FftParams &p, const float *x, const float2 *G, float2 *spec, float *y,
                    cudaStream_t st);

}  // namespace cct
