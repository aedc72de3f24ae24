// FFT convolution (the reference's large-filter path,
// generator/DynamicConvolutionGenerator.scala:322-480 with the expanded shape
// of generator/FFTConvolutionUtils.scala:38-97), hand-written in FP32:
//
//   y = trim( IFFT2( FFT2(expand(x)) * G ) ),   G = FFT2(g) / (Fr * Fc/2)
//
// where expand(x) is the Fr x Fc power-of-two grid holding x with its border
// extension (Zero / Clamp / Cyclic) below/right of the field and, wrapped,
// above/left of it, and g holds the (flipped for convolution) filter centred
// at the origin with cyclic wrap-around.  This equals the direct convolution
// with the same border policy at every output point.
//
// Three kernels per run, each a shared-memory radix-4 Stockham FFT:
//   fft_rows_r2c   one expanded row per CTA: Fc reals packed as Fc/2 complex,
//                  N = Fc/2 point FFT, then the even/odd split to the
//                  Fc/2 + 1 non-negative frequencies;
//   fft_cols       a block of spectrum columns per CTA: Fr-point FFT down
//                  each column, times G, inverse FFT (or, for a dynamic
//                  filter's spectrum, forward FFT and scaling only);
//   fft_rows_c2r   one output row per CTA: inverse of the split, N-point
//                  inverse FFT, unpacked and trimmed to the field.
// Twiddles are computed in FP64 on the host and stored as float2.
#include <cmath>
#include <complex>
#include <vector>

#include "cct_internal.h"
#include "fft_conv.h"
#include "tile_common.cuh"

namespace cct {
namespace {

constexpr int kFftThreads = 256;

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }

// `cols` independent N-point DFTs (N = 2^logN) of the sequences a[c*N .. c*N+N)
// in shared memory, Stockham autosort with radix-4 stages (and one radix-2
// stage when logN is odd), ping-ponging with b.  tw[k] = exp(-2 pi i k / N).
// inverse: exp(+...) and no scaling.  Returns the buffer holding the result.
__device__ float2 *stockham(float2 *a, float2 *b, int N, int logN, int cols,
                            const float2 *__restrict__ tw, bool inverse) {
  int Ns = 1;
  for (int st = 0; st < logN / 2; ++st) {
    const int q = N / 4, tstep = N / (4 * Ns);
    for (int t = threadIdx.x; t < q * cols; t += blockDim.x) {
      const int c = t / q, j = t - c * q;
      const float2 *src = a + c * N;
      float2 *dst = b + c * N;
      const int k = j & (Ns - 1);
      float2 w1 = __ldg(tw + k * tstep), w2 = __ldg(tw + 2 * k * tstep), w3 = __ldg(tw + 3 * k * tstep);
      if (inverse) {
        w1 = conjf2(w1);
        w2 = conjf2(w2);
        w3 = conjf2(w3);
      }
      const float2 v0 = src[j];
      const float2 v1 = cmul(src[j + q], w1);
      const float2 v2 = cmul(src[j + 2 * q], w2);
      const float2 v3 = cmul(src[j + 3 * q], w3);
      const float2 t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), d = csub(v1, v3);
      // forward: t3 = -i*d ; inverse: t3 = +i*d
      const float2 t3 = inverse ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
      const int base = (j - k) * 4 + k;
      dst[base] = cadd(t0, t2);
      dst[base + Ns] = cadd(t1, t3);
      dst[base + 2 * Ns] = csub(t0, t2);
      dst[base + 3 * Ns] = csub(t1, t3);
    }
    __syncthreads();
    float2 *tmp = a;
    a = b;
    b = tmp;
    Ns *= 4;
  }
  if (logN & 1) {
    const int h = N / 2, tstep = N / (2 * Ns);
    for (int t = threadIdx.x; t < h * cols; t += blockDim.x) {
      const int c = t / h, j = t - c * h;
      const float2 *src = a + c * N;
      float2 *dst = b + c * N;
      const int k = j & (Ns - 1);
      float2 w = __ldg(tw + k * tstep);
      if (inverse) w = conjf2(w);
      const float2 v0 = src[j], v1 = cmul(src[j + h], w);
      const int base = (j - k) * 2 + k;
      dst[base] = cadd(v0, v1);
      dst[base + Ns] = csub(v0, v1);
    }
    __syncthreads();
    float2 *tmp = a;
    a = b;
    b = tmp;
  }
  return a;
}

// Expanded-grid coordinate -> field coordinate (or -1 = zero): positions past
// the field belong to the extension below the field when they are closer to
// it, else to the wrapped extension above it.
__device__ __forceinline__ int expand_index(int p, int n, int F, int border) {
  int v = p;
  if (p >= n) v = (p - n) < (F - p) ? p : p - F;
  return border_index(border, v, n);
}

// Row pass: one expanded row (image) or one filter row per CTA -> half spectrum.
// SRC 0: image plane `plane` of x expanded with the border; 1: filter plane
// `plane` centred at the origin (flipped for convolution).
template <int SRC>
__global__ void __launch_bounds__(kFftThreads)
    fft_rows_r2c(FftParams p, const float *__restrict__ src, float2 *__restrict__ spec, int planes) {
  extern __shared__ __align__(16) float2 fsm[];
  const int N = p.Fc / 2;
  float2 *a = fsm, *b = fsm + N;
  const int row = blockIdx.x % p.Fr, pl = blockIdx.x / p.Fr;
  if (pl >= planes) return;
  const ConvGeom &g = p.g;
  if (SRC == 0) {
    int ip, fp;
    plane_pair(g, pl, 0, &ip, &fp);
    const float *xp = src + (size_t)ip * g.H * g.W;
    const int sr = expand_index(row, g.H, p.Fr, g.border);
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
      float v[2];
      for (int e = 0; e < 2; ++e) {
        const int sc = expand_index(2 * n + e, g.W, p.Fc, g.border);
        v[e] = (sr >= 0 && sc >= 0) ? __ldg(xp + (size_t)sr * g.W + sc) : 0.0f;
      }
      a[n] = make_float2(v[0], v[1]);
    }
  } else {
    // g[(r - h) mod Fr][(s - h) mod Fc] = f[r][s] for convolution,
    // g[(h - r) mod Fr][(h - s) mod Fc] = f[r][s] for cross-correlation.
    const float *fp = src + (size_t)pl * g.R * g.S;
    const int hr = (g.R - 1) / 2, hc = (g.S - 1) / 2;
    const bool conv = g.orient == CCT_CONVOLUTION;
    // filter row r landing on this expanded row
    int r = conv ? row + hr : hr - row;
    if (conv) { if (r >= p.Fr) r -= p.Fr; } else { if (r < 0) r += p.Fr; }
    // rows far from the origin are empty; so are filter rows that do not exist
    const bool has = r >= 0 && r < g.R && ((conv ? (r - hr) : (hr - r)) % p.Fr + p.Fr) % p.Fr == row;
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
      float v[2] = {0.0f, 0.0f};
      if (has) {
        for (int e = 0; e < 2; ++e) {
          const int col = 2 * n + e;
          int s = conv ? col + hc : hc - col;
          if (conv) { if (s >= p.Fc) s -= p.Fc; } else { if (s < 0) s += p.Fc; }
          if (s >= 0 && s < g.S && ((conv ? (s - hc) : (hc - s)) % p.Fc + p.Fc) % p.Fc == col)
            v[e] = __ldg(fp + (size_t)r * g.S + s);
        }
      }
      a[n] = make_float2(v[0], v[1]);
    }
  }
  __syncthreads();
  float2 *z = stockham(a, b, N, p.logN, 1, p.tw_n, false);
  // X[k] = E[k] + W^k O[k], E = (Z[k] + conj Z[N-k]) / 2, O = (Z[k] - conj Z[N-k]) / 2i,
  // W = exp(-2 pi i / Fc), k = 0..N
  float2 *out = spec + ((size_t)pl * p.Fr + row) * p.ld;
  for (int k = threadIdx.x; k <= N; k += blockDim.x) {
    const float2 zk = z[k == N ? 0 : k], zn = conjf2(z[k == 0 ? 0 : N - k]);
    const float2 e = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y + zn.y));
    const float2 dd = make_float2(0.5f * (zk.x - zn.x), 0.5f * (zk.y - zn.y));
    const float2 o = make_float2(dd.y, -dd.x);  // dd / i
    out[k] = cadd(e, cmul(__ldg(p.tw_2n + k), o));
  }
}

// Column pass over CW spectrum columns per CTA.
// MODE 0: forward FFT, times G[fplane], inverse FFT (in place in spec).
// MODE 1: forward FFT and scaling by p.scale (a filter's spectrum).
template <int MODE, int CW>
__global__ void __launch_bounds__(kFftThreads)
    fft_cols(FftParams p, float2 *__restrict__ spec, const float2 *__restrict__ G, int planes) {
  extern __shared__ __align__(16) float2 fsm[];
  const int Fr = p.Fr, ncol = p.Fc / 2 + 1;
  const int cblocks = (ncol + CW - 1) / CW;
  const int pl = blockIdx.x / cblocks, c0 = (blockIdx.x - pl * cblocks) * CW;
  if (pl >= planes) return;
  float2 *a = fsm, *b = fsm + CW * Fr;
  float2 *sp = spec + (size_t)pl * Fr * p.ld;
  for (int t = threadIdx.x; t < CW * Fr; t += blockDim.x) {
    const int r = t / CW, c = t - r * CW;
    a[c * Fr + r] = (c0 + c < ncol) ? sp[(size_t)r * p.ld + c0 + c] : make_float2(0.0f, 0.0f);
  }
  __syncthreads();
  float2 *z = stockham(a, b, Fr, p.logR, CW, p.tw_r, false);
  if (MODE == 0) {
    int ip, fp;
    plane_pair(p.g, pl, 0, &ip, &fp);
    const float2 *gp = G + (size_t)fp * Fr * p.ld;
    for (int t = threadIdx.x; t < CW * Fr; t += blockDim.x) {
      const int c = t / Fr, r = t - c * Fr;
      if (c0 + c < ncol) z[t] = cmul(z[t], __ldg(gp + (size_t)r * p.ld + c0 + c));
    }
    __syncthreads();
    float2 *other = (z == a) ? b : a;
    z = stockham(z, other, Fr, p.logR, CW, p.tw_r, true);
  } else {
    for (int t = threadIdx.x; t < CW * Fr; t += blockDim.x) z[t] = make_float2(z[t].x * p.scale, z[t].y * p.scale);
    __syncthreads();
  }
  for (int t = threadIdx.x; t < CW * Fr; t += blockDim.x) {
    const int r = t / CW, c = t - r * CW;
    if (c0 + c < ncol) sp[(size_t)r * p.ld + c0 + c] = z[c * Fr + r];
  }
}

// Inverse row pass: half spectrum row -> real row, trimmed to the output.
__global__ void __launch_bounds__(kFftThreads)
    fft_rows_c2r(FftParams p, const float2 *__restrict__ spec, float *__restrict__ y, int planes) {
  extern __shared__ __align__(16) float2 fsm[];
  const int N = p.Fc / 2;
  float2 *a = fsm, *b = fsm + N;
  const ConvGeom &g = p.g;
  const int row = blockIdx.x % g.OH, pl = blockIdx.x / g.OH;
  if (pl >= planes) return;
  const float2 *in = spec + ((size_t)pl * p.Fr + row) * p.ld;
  // Z[k] = E[k] + i O[k], E = (X[k] + conj X[N-k]) / 2, O = (X[k] - conj X[N-k]) / 2 * conj(W^k)
  for (int k = threadIdx.x; k < N; k += blockDim.x) {
    const float2 xk = __ldg(in + k), xn = conjf2(__ldg(in + N - k));
    const float2 e = make_float2(0.5f * (xk.x + xn.x), 0.5f * (xk.y + xn.y));
    const float2 dd = make_float2(0.5f * (xk.x - xn.x), 0.5f * (xk.y - xn.y));
    const float2 o = cmul(dd, conjf2(__ldg(p.tw_2n + k)));
    a[k] = make_float2(e.x - o.y, e.y + o.x);  // e + i*o
  }
  __syncthreads();
  const float2 *z = stockham(a, b, N, p.logN, 1, p.tw_n, true);
  float *yr = y + ((size_t)pl * g.OH + row) * g.OW;
  const bool relu = (g.flags & CCT_FLAG_RELU) != 0;
  for (int j = threadIdx.x; j < g.OW; j += blockDim.x) {
    const float2 v = z[j >> 1];
    const float o = (j & 1) ? v.y : v.x;
    yr[j] = relu ? fmaxf(o, 0.0f) : o;
  }
}

int ilog2(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}
int pow2_at_least(int v) { return 1 << ilog2(v); }

template <typename K>
int set_smem(K kern, size_t bytes) {
  if (bytes <= 48 * 1024) return CCT_OK;
  return check_cuda(cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)bytes),
                    "cudaFuncSetAttribute(fft)");
}

// Spectrum columns per CTA in the column pass: 4, or 2 for 4096-point columns
// (the ping-pong buffers hold 2 x cols x Fr complex values).
int col_width(int Fr) { return Fr > 2048 ? 2 : 4; }

// One-dimensional forward FFT of length n in FP64 (iterative radix-2, natural
// order) of v[0], v[stride], ...; w[k] = exp(-2 pi i k / n), k < n/2.
void fft64(std::complex<double> *v, int n, int stride, const std::vector<std::complex<double>> &w,
           std::vector<std::complex<double>> *scratch) {
  std::vector<std::complex<double>> &t = *scratch;
  t.resize(n);
  for (int i = 0; i < n; ++i) t[i] = v[(size_t)i * stride];
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(t[i], t[j]);
  }
  for (int len = 2; len <= n; len <<= 1) {
    const int step = n / len;
    for (int i = 0; i < n; i += len)
      for (int k = 0; k < len / 2; ++k) {
        const std::complex<double> u = t[i + k], x = t[i + k + len / 2] * w[(size_t)k * step];
        t[i + k] = u + x;
        t[i + k + len / 2] = u - x;
      }
  }
  for (int i = 0; i < n; ++i) v[(size_t)i * stride] = t[i];
}

std::vector<std::complex<double>> twiddles64(int n) {
  std::vector<std::complex<double>> w(n / 2);
  for (int k = 0; k < n / 2; ++k) w[k] = std::polar(1.0, -2.0 * M_PI * k / n);
  return w;
}

}  // namespace

bool fft_plan(const ConvGeom &g, FftParams *out) {
  if (g.mode != CCT_PLANE_BY_PLANE || g.down != 1 || g.up != 1) return false;
  if (g.border != CCT_BORDER_ZERO && g.border != CCT_BORDER_CLAMP && g.border != CCT_BORDER_CYCLIC)
    return false;
  if (g.H < 2 || g.W < 2) return false;
  FftParams p{};
  p.g = g;
  const int hr = g.R / 2, hc = g.S / 2;  // apron (FFTConvolutionUtils.scala:63-64)
  auto size = [&](int n, int h) {
    switch (g.border) {
      case CCT_BORDER_CLAMP: return pow2_at_least(n + 2 * h);
      case CCT_BORDER_ZERO: return pow2_at_least(n + h);
      default: return (n & (n - 1)) == 0 ? n : pow2_at_least(n + 2 * h);
    }
  };
  p.Fr = size(g.H, hr);
  p.Fc = size(g.W, hc);
  if (p.Fc < 8) p.Fc = 8;
  if (p.Fr < 4) p.Fr = 4;
  if (p.Fr > 4096 || p.Fc > 8192) return false;
  if (g.R > p.Fr || g.S > p.Fc) return false;  // no tap may wrap onto another
  // the border extension must fit between the field and its wrapped copy
  if (g.border != CCT_BORDER_ZERO && ((p.Fr > g.H && p.Fr < g.H + 2 * hr) || (p.Fc > g.W && p.Fc < g.W + 2 * hc)))
    return false;
  p.logN = ilog2(p.Fc / 2);
  p.logR = ilog2(p.Fr);
  p.ld = p.Fc / 2 + 1;
  p.scale = 1.0f / ((float)p.Fr * (float)(p.Fc / 2));
  p.spec_elems = (size_t)g.pout * p.Fr * p.ld;
  p.filter_elems = (size_t)g.pf * p.Fr * p.ld;
  p.tw_elems = (size_t)(p.Fc / 2) + p.Fr + (p.Fc / 2 + 1);
  *out = p;
  return true;
}

void fft_twiddles(const FftParams &p, std::vector<float> *host) {
  host->resize(2 * p.tw_elems);
  float *h = host->data();
  const int N = p.Fc / 2;
  size_t o = 0;
  for (int k = 0; k < N; ++k, ++o) {
    h[2 * o] = (float)std::cos(-2.0 * M_PI * k / N);
    h[2 * o + 1] = (float)std::sin(-2.0 * M_PI * k / N);
  }
  for (int k = 0; k < p.Fr; ++k, ++o) {
    h[2 * o] = (float)std::cos(-2.0 * M_PI * k / p.Fr);
    h[2 * o + 1] = (float)std::sin(-2.0 * M_PI * k / p.Fr);
  }
  for (int k = 0; k <= N; ++k, ++o) {
    h[2 * o] = (float)std::cos(-2.0 * M_PI * k / p.Fc);
    h[2 * o + 1] = (float)std::sin(-2.0 * M_PI * k / p.Fc);
  }
}

void fft_set_tables(FftParams *p, float2 *tw) {
  p->tw_n = tw;
  p->tw_r = tw + p->Fc / 2;
  p->tw_2n = tw + p->Fc / 2 + p->Fr;
}

void fft_static_spectrum(const FftParams &p, const float *host_filter, std::vector<float> *out) {
  const ConvGeom &g = p.g;
  const int Fr = p.Fr, Fc = p.Fc, ld = p.ld;
  const int hr = (g.R - 1) / 2, hc = (g.S - 1) / 2;
  out->assign(2 * p.filter_elems, 0.0f);
  std::vector<std::complex<double>> grid((size_t)Fr * Fc);
  const double scale = 1.0 / ((double)Fr * (double)(Fc / 2));
  const std::vector<std::complex<double>> wc = twiddles64(Fc), wr = twiddles64(Fr);
  std::vector<std::complex<double>> scratch;
  for (int pl = 0; pl < g.pf; ++pl) {
    std::fill(grid.begin(), grid.end(), std::complex<double>(0.0, 0.0));
    const float *f = host_filter + (size_t)pl * g.R * g.S;
    for (int r = 0; r < g.R; ++r)
      for (int s = 0; s < g.S; ++s) {
        int gr, gc;
        if (g.orient == CCT_CONVOLUTION) {
          gr = ((r - hr) % Fr + Fr) % Fr;
          gc = ((s - hc) % Fc + Fc) % Fc;
        } else {
          gr = ((hr - r) % Fr + Fr) % Fr;
          gc = ((hc - s) % Fc + Fc) % Fc;
        }
        grid[(size_t)gr * Fc + gc] += f[(size_t)r * g.S + s];
      }
    for (int r = 0; r < Fr; ++r) fft64(grid.data() + (size_t)r * Fc, Fc, 1, wc, &scratch);
    for (int c = 0; c <= Fc / 2; ++c) fft64(grid.data() + c, Fr, Fc, wr, &scratch);
    float *o = out->data() + 2 * (size_t)pl * Fr * ld;
    for (int r = 0; r < Fr; ++r)
      for (int c = 0; c <= Fc / 2; ++c) {
        const std::complex<double> v = grid[(size_t)r * Fc + c] * scale;
        o[2 * ((size_t)r * ld + c)] = (float)v.real();
        o[2 * ((size_t)r * ld + c) + 1] = (float)v.imag();
      }
  }
}

template <int MODE, int CW>
int launch_cols(const FftParams &p, float2 *spec, const float2 *G, int planes, cudaStream_t st) {
  const size_t col_smem = sizeof(float2) * 2 * CW * p.Fr;
  int rc = set_smem(fft_cols<MODE, CW>, col_smem);
  if (rc) return rc;
  const int cblocks = (p.Fc / 2 + 1 + CW - 1) / CW;
  fft_cols<MODE, CW><<<cblocks * planes, kFftThreads, col_smem, st>>>(p, spec, G, planes);
  return CCT_OK;
}

int launch_fft_filter_spectrum(const FftParams &p, const float *f, float2 *G, cudaStream_t st) {
  const size_t row_smem = sizeof(float2) * p.Fc;  // a + b of Fc/2 each
  int rc = set_smem(fft_rows_r2c<1>, row_smem);
  if (rc) return rc;
  const int planes = p.g.pf;
  fft_rows_r2c<1><<<p.Fr * planes, kFftThreads, row_smem, st>>>(p, f, G, planes);
  rc = col_width(p.Fr) == 4 ? launch_cols<1, 4>(p, G, nullptr, planes, st)
                            : launch_cols<1, 2>(p, G, nullptr, planes, st);
  if (rc) return rc;
  count_launches(2);
  return check_cuda(cudaGetLastError(), "fft filter spectrum launch");
}

int launch_fft_conv(const FftParams &p, const float *x, const float2 *G, float2 *spec, float *y,
                    cudaStream_t st) {
  const size_t row_smem = sizeof(float2) * p.Fc;
  int rc = set_smem(fft_rows_r2c<0>, row_smem);
  if (!rc) rc = set_smem(fft_rows_c2r, row_smem);
  if (rc) return rc;
  const int planes = p.g.pout;
  fft_rows_r2c<0><<<p.Fr * planes, kFftThreads, row_smem, st>>>(p, x, spec, planes);
  rc = col_width(p.Fr) == 4 ? launch_cols<0, 4>(p, spec, G, planes, st)
                            : launch_cols<0, 2>(p, spec, G, planes, st);
  if (rc) return rc;
  fft_rows_c2r<<<p.g.OH * planes, kFftThreads, row_smem, st>>>(p, spec, y, planes);
  count_launches(3);
  return check_cuda(cudaGetLastError(), "fft convolution launch");
}

}  // namespace cct
