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
// Three kernels per run:
//   fft_rows_r2c   expanded rows (Fc reals packed as N = Fc/2 complex): N-point
//                  FFT, then the even/odd split to the Fc/2 + 1 non-negative
//                  frequencies;
//   fft_cols       blocks of spectrum columns: Fr-point FFT down each
//                  column, times G, inverse FFT (or, for a dynamic filter's
//                  spectrum, forward FFT and scaling only);
//   fft_rows_c2r   output rows: inverse of the split, N-point inverse FFT,
//                  unpacked and trimmed to the field.
// Each FFT is a Stockham autosort in radix-16 passes (radix 2/4/8 for the
// last): every thread keeps 16 complex values in registers and does one
// 16-point (or 16/R R-point) DFT per pass, so an N-point FFT takes
// ceil(log2 N / 4) shared-memory exchanges.  Shared-memory sequences are
// padded by one element every 16 so the strided exchanges stay free of bank
// conflicts.  Twiddles are computed in FP64 on the host and stored as float2.
#include <cmath>
#include <complex>
#include <vector>

#include "cct_internal.h"
#include "fft_conv.h"
#include "sm100_util.cuh"
#include "tile_common.cuh"

namespace cct {
namespace {

constexpr int kRowThreads = 256;
constexpr int kColThreads = 512;
__host__ __device__ constexpr int col_stride(int Fr) { return Fr + Fr / 16 + 8; }

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }

// Spectrum layout of one plane (Fr rows x ld columns, ld a multiple of 4):
// blocks of 4 columns, each block all Fr rows of its 4 columns (32 bytes per
// row).  A row pass reads and writes 32-byte row segments; a column pass
// reads its columns as one contiguous stretch per block.
__host__ __device__ __forceinline__ size_t spec_index(int r, int c, int Fr) {
  return ((size_t)(c >> 2) * Fr + r) * 4 + (c & 3);
}

// multiply by -i (forward transform) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 rot(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
// multiply by exp(-+ 2 pi i j / 16): forward uses the minus sign
template <bool INV>
__device__ __forceinline__ float2 w16(float2 a, float c, float s) {
  return cmul(a, make_float2(c, INV ? s : -s));
}

template <bool INV>
__device__ __forceinline__ void dft2(float2 *v) {
  const float2 a = v[0];
  v[0] = cadd(a, v[1]);
  v[1] = csub(a, v[1]);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2 &a0, float2 &a1, float2 &a2, float2 &a3) {
  const float2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = rot<INV>(csub(a1, a3));
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, t3);
  a3 = csub(t1, t3);
}

template <bool INV>
__device__ __forceinline__ void dft8(float2 *v) {
  constexpr float h = 0.70710678118654752f;  // cos(pi/4)
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<INV>(e0, e1, e2, e3);
  dft4<INV>(o0, o1, o2, o3);
  o1 = w16<INV>(o1, h, h);   // W8^1
  o2 = rot<INV>(o2);         // W8^2
  o3 = w16<INV>(o3, -h, h);  // W8^3
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}

template <bool INV>
__device__ __forceinline__ void dft16(float2 *v) {
  constexpr float c1 = 0.92387953251128674f, s1 = 0.38268343236508978f;  // cos, sin(pi/8)
  constexpr float h = 0.70710678118654752f;
  // n = 4p + q: 4-point DFTs over p, twiddles W16^(q k1), 4-point DFTs over q
#pragma unroll
  for (int q = 0; q < 4; ++q) dft4<INV>(v[q], v[q + 4], v[q + 8], v[q + 12]);
  v[5] = w16<INV>(v[5], c1, s1);     // q=1 k1=1
  v[9] = w16<INV>(v[9], h, h);       // q=1 k1=2
  v[13] = w16<INV>(v[13], s1, c1);   // q=1 k1=3
  v[6] = w16<INV>(v[6], h, h);       // q=2 k1=1
  v[10] = rot<INV>(v[10]);           // q=2 k1=2
  v[14] = w16<INV>(v[14], -h, h);    // q=2 k1=3
  v[7] = w16<INV>(v[7], s1, c1);     // q=3 k1=1
  v[11] = w16<INV>(v[11], -h, h);    // q=3 k1=2
  v[15] = w16<INV>(v[15], -c1, -s1); // q=3 k1=3 (W16^9)
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) dft4<INV>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
  // X[k1 + 4 k2] sits in v[4 k1 + k2]: transpose to natural order
  float2 t[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) t[m] = v[4 * (m & 3) + (m >> 2)];
#pragma unroll
  for (int m = 0; m < 16; ++m) v[m] = t[m];
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2 *v) {
  if (R == 2) dft2<INV>(v);
  if (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
  if (R == 8) dft8<INV>(v);
  if (R == 16) dft16<INV>(v);
}

// One Stockham pass of radix R over an N-point sequence (T = N/16 threads,
// thread tt owns butterflies j = tt + q*T, q < 16/R): twiddles
// w_(Ns R)^(m k) on input m (k = j mod Ns), then the R-point DFT.
template <int R, bool INV>
__device__ __forceinline__ void pass_compute(float2 (&v)[16], int N, int Ns, int T, int tt,
                                             const float2 *__restrict__ tw) {
#pragma unroll
  for (int q = 0; q < 16 / R; ++q) {
    const int j = tt + q * T, k = j & (Ns - 1);
    if (k) {
      // w^m for m < R from two table reads (w and w^4) and at most two
      // products (w^m = (w^4)^a w^b, m = 4a + b), instead of R-1 scattered
      // reads per butterfly
      const int step = N / (Ns * R);
      float2 p[4], p4[4];
      p[0] = make_float2(1.0f, 0.0f);
      p[1] = __ldg(tw + k * step);
      if (R > 2) {
        p[2] = cmul(p[1], p[1]);
        p[3] = cmul(p[2], p[1]);
      }
      if (R > 4) {
        p4[0] = make_float2(1.0f, 0.0f);
        p4[1] = __ldg(tw + 4 * k * step);
        p4[2] = cmul(p4[1], p4[1]);
        p4[3] = cmul(p4[2], p4[1]);
      }
#pragma unroll
      for (int m = 1; m < R; ++m) {
        const float2 w = (m < 4) ? p[m] : ((m & 3) ? cmul(p4[m >> 2], p[m & 3]) : p4[m >> 2]);
        v[q * R + m] = cmul(v[q * R + m], INV ? conjf2(w) : w);
      }
    }
    dft<R, INV>(v + q * R);
  }
}

template <int R>
__device__ __forceinline__ void pass_load(const float2 *s, float2 (&v)[16], int N, int T, int tt) {
#pragma unroll
  for (int q = 0; q < 16 / R; ++q)
#pragma unroll
    for (int m = 0; m < R; ++m) v[q * R + m] = s[pad16(tt + q * T + m * (N / R))];
}

template <int R>
__device__ __forceinline__ void pass_store(float2 *s, const float2 (&v)[16], int Ns, int T, int tt) {
#pragma unroll
  for (int q = 0; q < 16 / R; ++q) {
    const int j = tt + q * T, k = j & (Ns - 1), base = (j - k) * R + k;
#pragma unroll
    for (int m = 0; m < R; ++m) s[pad16(base + m * Ns)] = v[q * R + m];
  }
}

// N-point FFT (N = 2^LOGN >= 16) of the sequence whose first-pass inputs
// v[m] = x[tt + m*T] the caller loaded; the result lands in natural order in
// s (padded).  The passes (radix 16, the last 2..16) are fixed at compile
// time.  Every thread of the CTA takes part (the passes synchronise the CTA).
template <int LOGN, bool INV, int NS_LOG = 0, bool FIRST = true>
__device__ __forceinline__ void fft_passes(float2 *s, float2 (&v)[16], int tt, const float2 *__restrict__ tw) {
  if constexpr (NS_LOG < LOGN) {
    constexpr int B = (LOGN - NS_LOG) >= 4 ? 4 : (LOGN - NS_LOG);
    constexpr int R = 1 << B, N = 1 << LOGN, T = N / 16;
    if (!FIRST) pass_load<R>(s, v, N, T, tt);
    pass_compute<R, INV>(v, N, 1 << NS_LOG, T, tt, tw);
    __syncthreads();
    pass_store<R>(s, v, 1 << NS_LOG, T, tt);
    __syncthreads();
    fft_passes<LOGN, INV, NS_LOG + B, false>(s, v, tt, tw);
  }
}

// Expanded-grid coordinate -> field coordinate (or -1 = zero): positions past
// the field belong to the extension below the field when they are closer to
// it, else to the wrapped extension above it.
__device__ __forceinline__ int expand_index(int p, int n, int F, int border) {
  int v = p;
  if (p >= n) v = (p - n) < (F - p) ? p : p - F;
  return border_index(border, v, n);
}

// Filter tap landing on expanded coordinate `pos` (or -1): g[(r - h) mod F]
// = f[r] for convolution, g[(h - r) mod F] = f[r] for cross-correlation.
__device__ __forceinline__ int filter_index(int pos, int h, int R, int F, bool conv) {
  int r = conv ? pos + h : h - pos;
  if (conv) {
    if (r >= F) r -= F;
  } else {
    if (r < 0) r += F;
  }
  return (r >= 0 && r < R) ? r : -1;
}

// Row pass: rows_per_cta sequences of N = Fc/2 complex points per CTA.
// SRC 0: image plane rows expanded with the border; 1: filter plane rows
// centred at the origin (flipped for convolution).
template <int SRC, int LOGN>
__global__ void __launch_bounds__(kRowThreads, 4)
    fft_rows_r2c(FftParams p, const float *__restrict__ src, float2 *__restrict__ spec, int planes) {
  extern __shared__ __align__(16) float2 fsm[];
  grid_dependency_wait();  // launched with programmatic serialisation
  allow_dependent_launch();
  constexpr int N = 1 << LOGN, T = N / 16, per = kRowThreads / T;
  const int sub = threadIdx.x / T, tt = threadIdx.x - sub * T;
  const int gr = blockIdx.x * per + sub;
  const bool active = gr < planes * p.Fr;
  const int row = gr % p.Fr, pl = gr / p.Fr;
  float2 *s = fsm + sub * (N + N / 16);
  const ConvGeom &g = p.g;
  float2 v[16];
  if (SRC == 0) {
    int ip = 0, fp;
    if (active) plane_pair(g, pl, 0, &ip, &fp);
    const float *xp = src + (size_t)ip * g.H * g.W;
    const int sr = active ? expand_index(row, g.H, p.Fr, g.border) : -1;
    // positions inside the field map to themselves: one 8-byte load per pair
    // (an 8-byte aligned plane of even width keeps every row aligned); the
    // border positions take the expansion rule
    const bool pairs = sr >= 0 && (g.W & 1) == 0 && (reinterpret_cast<uintptr_t>(xp) & 7) == 0;
    const float2 *row2 = reinterpret_cast<const float2 *>(xp + (size_t)(sr < 0 ? 0 : sr) * g.W);
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int n = tt + m * T;
      if (pairs && 2 * n + 1 < g.W) {
        v[m] = __ldg(row2 + n);
      } else {
        float e[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int sc = expand_index(2 * n + k, g.W, p.Fc, g.border);
          e[k] = (sr >= 0 && sc >= 0) ? __ldg(xp + (size_t)sr * g.W + sc) : 0.0f;
        }
        v[m] = make_float2(e[0], e[1]);
      }
    }
  } else {
    const float *fp = src + (size_t)pl * g.R * g.S;
    const bool conv = g.orient == CCT_CONVOLUTION;
    const int r = active ? filter_index(row, (g.R - 1) / 2, g.R, p.Fr, conv) : -1;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int n = tt + m * T;
      float e[2] = {0.0f, 0.0f};
      if (r >= 0) {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const int c = filter_index(2 * n + k, (g.S - 1) / 2, g.S, p.Fc, conv);
          if (c >= 0) e[k] = __ldg(fp + (size_t)r * g.S + c);
        }
      }
      v[m] = make_float2(e[0], e[1]);
    }
  }
  fft_passes<LOGN, false>(s, v, tt, p.tw_n);
  if (!active) return;
  // X[k] = E[k] + W^k O[k], E = (Z[k] + conj Z[N-k]) / 2, O = (Z[k] - conj Z[N-k]) / 2i,
  // W = exp(-2 pi i / Fc), k = 0..N
  float2 *out = spec + (size_t)pl * p.Fr * p.ld;
  for (int k = tt; k <= N; k += T) {
    const float2 zk = s[pad16(k == N ? 0 : k)], zn = conjf2(s[pad16(k == 0 ? 0 : N - k)]);
    const float2 e = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y + zn.y));
    const float2 dd = make_float2(0.5f * (zk.x - zn.x), 0.5f * (zk.y - zn.y));
    const float2 o = make_float2(dd.y, -dd.x);  // dd / i
    out[spec_index(row, k, p.Fr)] = cadd(e, cmul(__ldg(p.tw_2n + k), o));
  }
}

// Column pass over blockDim/T spectrum columns per CTA (c fastest across
// threads, so each warp reads 32-byte row segments).
// MODE 0: forward FFT, times G[fplane], inverse FFT, in place in spec.
// MODE 1: forward FFT and scaling by p.scale (a filter's spectrum).
template <int MODE, int LOGR>
__global__ void __launch_bounds__(kColThreads, 2)
    fft_cols(FftParams p, float2 *__restrict__ spec, const float2 *__restrict__ G, int planes) {
  extern __shared__ __align__(16) float2 fsm[];
  grid_dependency_wait();  // launched with programmatic serialisation
  allow_dependent_launch();
  constexpr int Fr = 1 << LOGR, T = Fr / 16, CW = kColThreads / T;
  const int ncol = p.Fc / 2 + 1;
  const int cblocks = (ncol + CW - 1) / CW;
  const int pl = blockIdx.x / cblocks, c0 = (blockIdx.x - pl * cblocks) * CW;
  const int c = threadIdx.x % CW, tt = threadIdx.x / CW, col = c0 + c;
  const bool active = col < ncol;
  // column stride = 8 (mod 16) complex: the CW columns a warp touches fall
  // on alternate halves of the banks
  float2 *s = fsm + c * col_stride(Fr);
  float2 *sp = spec + (size_t)pl * Fr * p.ld + spec_index(0, col, Fr);  // row r at sp[4 r]
  float2 v[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) v[m] = active ? sp[(size_t)(tt + m * T) * 4] : make_float2(0.0f, 0.0f);
  fft_passes<LOGR, false>(s, v, tt, p.tw_r);
  if (MODE == 0) {
    int ip, fp;
    plane_pair(p.g, pl, 0, &ip, &fp);
    const float2 *gp = G + (size_t)fp * Fr * p.ld + spec_index(0, col, Fr);
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int r = tt + m * T;
      v[m] = active ? cmul(s[pad16(r)], __ldg(gp + (size_t)r * 4)) : make_float2(0.0f, 0.0f);
    }
    fft_passes<LOGR, true>(s, v, tt, p.tw_r);
    if (!active) return;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int r = tt + m * T;
      sp[(size_t)r * 4] = s[pad16(r)];
    }
  } else {
    if (!active) return;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int r = tt + m * T;
      sp[(size_t)r * 4] = cscale(s[pad16(r)], p.scale);
    }
  }
}

// Inverse row pass: half-spectrum rows -> real rows, trimmed to the output.
template <int LOGN>
__global__ void __launch_bounds__(kRowThreads, 4)
    fft_rows_c2r(FftParams p, const float2 *__restrict__ spec, float *__restrict__ y, int planes) {
  extern __shared__ __align__(16) float2 fsm[];
  grid_dependency_wait();  // launched with programmatic serialisation
  allow_dependent_launch();
  const ConvGeom &g = p.g;
  constexpr int N = 1 << LOGN, T = N / 16, per = kRowThreads / T;
  const int sub = threadIdx.x / T, tt = threadIdx.x - sub * T;
  const int gr = blockIdx.x * per + sub;
  const bool active = gr < planes * g.OH;
  const int row = gr % g.OH, pl = gr / g.OH;
  float2 *s = fsm + sub * (N + N / 16);
  const float2 *in = spec + (size_t)pl * p.Fr * p.ld;
  // Z[k] = E[k] + i O[k], E = (X[k] + conj X[N-k]) / 2, O = (X[k] - conj X[N-k]) / 2 * conj(W^k)
  float2 v[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    const int k = tt + m * T;
    float2 z = make_float2(0.0f, 0.0f);
    if (active) {
      const float2 xk = __ldg(in + spec_index(row, k, p.Fr)), xn = conjf2(__ldg(in + spec_index(row, N - k, p.Fr)));
      const float2 e = make_float2(0.5f * (xk.x + xn.x), 0.5f * (xk.y + xn.y));
      const float2 dd = make_float2(0.5f * (xk.x - xn.x), 0.5f * (xk.y - xn.y));
      const float2 o = cmul(dd, conjf2(__ldg(p.tw_2n + k)));
      z = make_float2(e.x - o.y, e.y + o.x);  // e + i*o
    }
    v[m] = z;
  }
  fft_passes<LOGN, true>(s, v, tt, p.tw_n);
  if (!active) return;
  float *yr = y + ((size_t)pl * g.OH + row) * g.OW;
  const bool relu = (g.flags & CCT_FLAG_RELU) != 0;
  if ((g.OW & 1) == 0 && (reinterpret_cast<uintptr_t>(y) & 7) == 0) {
    // an aligned field of even width keeps every output row 8-byte aligned:
    // one pair per store
    float2 *yr2 = reinterpret_cast<float2 *>(yr);
    for (int j = tt; j < g.OW / 2; j += T) {
      float2 z = s[pad16(j)];
      if (relu) z = make_float2(fmaxf(z.x, 0.0f), fmaxf(z.y, 0.0f));
      yr2[j] = z;
    }
  } else {
    for (int j = tt; j < g.OW; j += T) {
      const float2 z = s[pad16(j >> 1)];
      const float o = (j & 1) ? z.y : z.x;
      yr[j] = relu ? fmaxf(o, 0.0f) : o;
    }
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
  // the register FFTs want at least 16 points per sequence
  if (p.Fc < 32) p.Fc = 32;
  if (p.Fr < 16) p.Fr = 16;
  if (p.Fr > 4096 || p.Fc > 8192) return false;
  if (g.R > p.Fr || g.S > p.Fc) return false;  // no tap may wrap onto another
  // the border extension must fit between the field and its wrapped copy
  if (g.border != CCT_BORDER_ZERO && ((p.Fr > g.H && p.Fr < g.H + 2 * hr) || (p.Fc > g.W && p.Fc < g.W + 2 * hc)))
    return false;
  p.logN = ilog2(p.Fc / 2);
  p.logR = ilog2(p.Fr);
  p.ld = ((p.Fc / 2 + 1) + 3) & ~3;  // whole 4-column blocks (spec_index)
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
        o[2 * spec_index(r, c, Fr)] = (float)v.real();
        o[2 * spec_index(r, c, Fr) + 1] = (float)v.imag();
      }
  }
}

// Kernel instantiation for the transform length (2^4 .. 2^12 points).
#define CCT_FFT_LOG_SWITCH(LOGV, CALL)                     \
  switch (LOGV) {                                          \
    case 4: { constexpr int L = 4; CALL; } break;          \
    case 5: { constexpr int L = 5; CALL; } break;          \
    case 6: { constexpr int L = 6; CALL; } break;          \
    case 7: { constexpr int L = 7; CALL; } break;          \
    case 8: { constexpr int L = 8; CALL; } break;          \
    case 9: { constexpr int L = 9; CALL; } break;          \
    case 10: { constexpr int L = 10; CALL; } break;        \
    case 11: { constexpr int L = 11; CALL; } break;        \
    case 12: { constexpr int L = 12; CALL; } break;        \
    default: return set_error(CCT_ENOTSUP, "FFT length 2^%d", (int)(LOGV)); \
  }

template <int MODE, int L>
int launch_cols_t(const FftParams &p, float2 *spec, const float2 *G, int planes, cudaStream_t st) {
  constexpr int Fr = 1 << L, cw = kColThreads / (Fr / 16);
  const size_t smem = sizeof(float2) * (size_t)cw * col_stride(Fr);
  int rc = set_smem(fft_cols<MODE, L>, smem);
  if (rc) return rc;
  const int cblocks = (p.Fc / 2 + 1 + cw - 1) / cw;
  return launch_pdl(fft_cols<MODE, L>, dim3(cblocks * planes), dim3(kColThreads), smem, st, "fft_cols launch", p,
                    spec, G, planes);
}

template <int MODE>
int launch_cols(const FftParams &p, float2 *spec, const float2 *G, int planes, cudaStream_t st) {
  CCT_FFT_LOG_SWITCH(p.logR, return (launch_cols_t<MODE, L>(p, spec, G, planes, st)))
  return CCT_OK;
}

// Rows per CTA and shared memory of the row passes.
void row_shape(const FftParams &p, int rows, int *per, int *blocks, size_t *smem) {
  const int N = p.Fc / 2, T = N / 16;
  *per = kRowThreads / T;
  *blocks = (rows + *per - 1) / *per;
  *smem = sizeof(float2) * (size_t)(*per) * (N + N / 16);
}

template <int SRC, int L>
int launch_r2c_t(const FftParams &p, const float *src, float2 *spec, int planes, cudaStream_t st) {
  int per, blocks;
  size_t smem;
  row_shape(p, p.Fr * planes, &per, &blocks, &smem);
  int rc = set_smem(fft_rows_r2c<SRC, L>, smem);
  if (rc) return rc;
  return launch_pdl(fft_rows_r2c<SRC, L>, dim3(blocks), dim3(kRowThreads), smem, st, "fft_rows_r2c launch", p,
                    src, spec, planes);
}

template <int L>
int launch_c2r_t(const FftParams &p, const float2 *spec, float *y, int planes, cudaStream_t st) {
  int per, blocks;
  size_t smem;
  row_shape(p, p.g.OH * planes, &per, &blocks, &smem);
  int rc = set_smem(fft_rows_c2r<L>, smem);
  if (rc) return rc;
  return launch_pdl(fft_rows_c2r<L>, dim3(blocks), dim3(kRowThreads), smem, st, "fft_rows_c2r launch", p, spec,
                    y, planes);
}

int launch_fft_filter_spectrum(const FftParams &p, const float *f, float2 *G, cudaStream_t st) {
  const int planes = p.g.pf;
  int rc = CCT_OK;
  CCT_FFT_LOG_SWITCH(p.logN, rc = (launch_r2c_t<1, L>(p, f, G, planes, st)))
  if (!rc) rc = launch_cols<1>(p, G, nullptr, planes, st);
  if (rc) return rc;
  count_launches(2);
  return check_cuda(cudaGetLastError(), "fft filter spectrum launch");
}

int launch_fft_conv(const FftParams &p, const float *x, const float2 *G, float2 *spec, float *y,
                    cudaStream_t st) {
  const int planes = p.g.pout;
  int rc = CCT_OK;
  CCT_FFT_LOG_SWITCH(p.logN, rc = (launch_r2c_t<0, L>(p, x, spec, planes, st)))
  if (!rc) rc = launch_cols<0>(p, spec, G, planes, st);
  if (rc) return rc;
  CCT_FFT_LOG_SWITCH(p.logN, rc = (launch_c2r_t<L>(p, spec, y, planes, st)))
  if (rc) return rc;
  count_launches(3);
  return check_cuda(cudaGetLastError(), "fft convolution launch");
}

}  // namespace cct
