/*
 * CPU oracle for the field-convolution hot path.  TEST INFRASTRUCTURE ONLY
 * (see conv_oracle.h): the checker for tests/, smoke() and the CPU baseline.
 *
 * Build: oracle/Makefile (gcc -O3 -ffp-contract=off so that the only fused
 * multiply-adds are the explicit fmaf() calls, as in the reference kernel
 * where `columnSum += tile * filter` contracts under -cl-mad-enable while
 * `rowSum += columnSum` and `reductionAccumulator += rowSum` are plain adds).
 */
#include "conv_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define ERR(...)                                      \
  do {                                                \
    if (err && errlen > 0) snprintf(err, errlen, __VA_ARGS__); \
    return 1;                                         \
  } while (0)

/* ConvolveHyperKernel.scala:824-830 (lowHalo). */
static int low_halo(int border, int fsize) {
  if (border == OR_FULL) return fsize - 1;
  if (border == OR_VALID) return 0;
  return (fsize - 1) / 2;
}

static int eff_sampling(const oracle_desc *d) {
  /* CogFunctionAPI.scala:1139-1143: step-1 sampling is NoSampling. */
  if (d->sampling != OR_NOSAMPLE && d->step == 1) return OR_NOSAMPLE;
  return d->sampling;
}

static int plane_count(int p) { return p <= 0 ? 1 : p; }

int oracle_output_shape(const oracle_desc *d, int *out_rows, int *out_cols,
                        int *out_planes, char *err, int errlen) {
  int sampling = eff_sampling(d);
  if (d->rows < 1 || d->cols < 1 || d->f_rows < 1 || d->f_cols < 1)
    ERR("field and filter sizes must be positive");
  if (d->border < OR_ZERO || d->border > OR_FULL) ERR("bad border policy");
  if (d->orient != OR_XCORR && d->orient != OR_CONV) ERR("bad orientation");
  if (sampling < OR_NOSAMPLE || sampling > OR_UP) ERR("bad sampling policy");
  if (sampling != OR_NOSAMPLE && d->step < 1) ERR("sampling step must be >= 1");
  if (d->mode < OR_PLANE || d->mode > OR_FILTER_ADJOINT_REDUCE) ERR("bad vector mode");
  int step = sampling == OR_NOSAMPLE ? 1 : d->step;
  /* DynamicConvolutionGenerator.scala:497-505: odd filters for centred borders. */
  if (d->border != OR_VALID && d->border != OR_FULL &&
      (d->f_rows % 2 == 0 || d->f_cols % 2 == 0))
    ERR("filter must be of odd shape for this border policy");
  /* :509-526: down-sampled input must divide after border contraction. */
  if (sampling == OR_DOWN) {
    int cr = 0, cc = 0;
    if (d->border == OR_VALID) { cr = d->f_rows - 1; cc = d->f_cols - 1; }
    if (d->border == OR_FULL) { cr = 1 - d->f_rows; cc = 1 - d->f_cols; }
    if ((d->rows - cr) % step != 0 || (d->cols - cc) % step != 0)
      ERR("input size must be divisible by the downsampling step after border contraction");
  }
  /* :530-535 */
  if (sampling == OR_UP && d->border == OR_CLAMP)
    ERR("integrated upsampling with BorderClamp convolution not supported");

  /* ConvolveHyperKernel.outputFieldType :1306-1347; FilterAdjoint upsamples
   * the second operand instead of the input (:1313-1326). */
  int fa = d->mode == OR_FILTER_ADJOINT || d->mode == OR_FILTER_ADJOINT_REDUCE;
  int fup = (fa && sampling == OR_UP) ? step : 1;
  int ur = d->rows, uc = d->cols;
  if (sampling == OR_UP && !fa) { ur *= step; uc *= step; }
  int br = ur, bc = uc;
  if (d->border == OR_VALID) { br = ur - d->f_rows * fup + 1; bc = uc - d->f_cols * fup + 1; }
  if (d->border == OR_FULL) { br = ur + d->f_rows * fup - 1; bc = uc + d->f_cols * fup - 1; }
  if (br < 1 || bc < 1) ERR("BorderValid filter larger than the input");
  if (sampling == OR_DOWN) { br = (br + step - 1) / step; bc = (bc + step - 1) / step; }

  int pin = plane_count(d->planes), pf = plane_count(d->f_planes);
  int batch = d->batch < 1 ? 1 : d->batch;
  int oplanes;
  if (d->mode == OR_PLANE) {
    /* :1368-1375 */
    if (!(d->planes <= 0 || d->f_planes <= 0 || d->planes == d->f_planes))
      ERR("plane-by-plane convolution needs a scalar operand or equal tensor shapes");
    oplanes = d->planes <= 0 ? pf : pin;
  } else if (fa) {
    /* :1366-1377 checks, :1414-1429 output planes */
    if (pf % batch != 0) ERR("filter planes must be a multiple of the batch size");
    if (pin % batch != 0) ERR("input planes must be a multiple of the batch size");
    oplanes = (pin / batch) * (pf / batch) * (d->mode == OR_FILTER_ADJOINT ? batch : 1);
  } else {
    /* frameInputChecks :1349-1356 */
    if (pin % batch != 0) ERR("input planes must be a multiple of the batch size");
    int n = pin / batch;
    if (pf % n != 0) ERR("filter planes must be a multiple of the per-image planes");
    if (d->mode == OR_PROJECT || d->mode == OR_BACKPROJECT)
      oplanes = pf * batch;
    else
      oplanes = batch * (pf / n);
  }
  if (out_rows) *out_rows = br;
  if (out_cols) *out_cols = bc;
  if (out_planes) *out_planes = oplanes;
  return 0;
}

/* Plane mixing: which (input plane, filter plane) pairs feed output plane o,
 * in the order the reference accumulates them (ConvolveHyperKernel.scala
 * :124-199 tensorElement setup, :319-340 filter tensorElement, :593-603 loop). */
typedef struct {
  int mode, pin, pf, batch, n, groups;
} plane_map;

static plane_map make_map(const oracle_desc *d) {
  plane_map m;
  m.mode = d->mode;
  m.pin = plane_count(d->planes);
  m.pf = plane_count(d->f_planes);
  m.batch = d->batch < 1 ? 1 : d->batch;
  m.n = m.pin / m.batch;
  if (m.mode == OR_FILTER_ADJOINT || m.mode == OR_FILTER_ADJOINT_REDUCE)
    m.groups = m.pf / m.batch;  /* gradient planes per image */
  else
    m.groups = m.pf / (m.n > 0 ? m.n : 1);
  return m;
}

static int map_terms(const plane_map *m, int o) {
  (void)o;
  if (m->mode == OR_PROJECT_REDUCE || m->mode == OR_BACKPROJECT_REDUCE) return m->n;
  if (m->mode == OR_FILTER_ADJOINT_REDUCE) return m->batch;
  return 1;
}

static void map_pair(const plane_map *m, int o, int t, int *ip, int *fp) {
  switch (m->mode) {
    case OR_PLANE:
      *ip = m->pin == 1 ? 0 : o;
      *fp = m->pf == 1 ? 0 : o;
      break;
    case OR_PROJECT: {               /* out b*F+p = x[b*N + p%N] (*) f[p] */
      int b = o / m->pf, p = o % m->pf;
      *ip = b * m->n + p % m->n;
      *fp = p;
      break;
    }
    case OR_PROJECT_REDUCE: {        /* out b*K+k = sum_c x[b*N+c] (*) f[k*N+c] */
      int b = o / m->groups, k = o % m->groups;
      *ip = b * m->n + t;
      *fp = k * m->n + t;
      break;
    }
    case OR_BACKPROJECT: {           /* out b*F+w = x[b*N + w%N] (*) f[L*(w%N) + w/N] */
      int b = o / m->pf, w = o % m->pf;
      *ip = b * m->n + w % m->n;
      *fp = m->groups * (w % m->n) + w / m->n;
      break;
    }
    case OR_BACKPROJECT_REDUCE: {    /* out b*L+l = sum_n x[b*N+n] (*) f[n*L+l] */
      int b = o / m->groups, l = o % m->groups;
      *ip = b * m->n + t;
      *fp = t * m->groups + l;
      break;
    }
    case OR_FILTER_ADJOINT: {        /* out B*w+b = x[b*C + w%C] (*) g[b*L + w/C] (:187, 333, 575-590) */
      int b = o % m->batch, w = o / m->batch;
      *ip = b * m->n + w % m->n;
      *fp = b * m->groups + w / m->n;
      break;
    }
    default: {                       /* out w = sum_b x[b*C + w%C] (*) g[b*L + w/C] */
      *ip = t * m->n + o % m->n;
      *fp = t * m->groups + o / m->n;
      break;
    }
  }
}

/* Border extension of one input coordinate, in input (pre-sampling) space.
 * Returns -1 for "reads zero". ConvolveHyperKernel.scala:235-317. */
static inline int border_index(int border, int v, int n) {
  switch (border) {
    case OR_CLAMP:
      return v < 0 ? 0 : (v >= n ? n - 1 : v);
    case OR_CYCLIC: {
      int r = v % n;
      return r < 0 ? r + n : r;
    }
    case OR_VALID:                   /* high-side protection only */
      return v >= n ? n - 1 : (v < 0 ? -1 : v);
    default:                         /* ZERO, FULL */
      return (v >= 0 && v < n) ? v : -1;
  }
}

/* Floor division for the up-sampled coordinate (exact when divisible). */
static inline int div_floor(int a, int b) {
  int q = a / b;
  return (a % b != 0 && ((a < 0) != (b < 0))) ? q - 1 : q;
}

#define DEFINE_CONV(NAME, T, FMA)                                              \
  typedef struct {                                                             \
    const oracle_desc *d;                                                      \
    const T *x, *f;                                                            \
    T *y;                                                                      \
    int orows, ocols, oplanes;                                                 \
    int next; /* work counter */                                               \
    pthread_mutex_t lock;                                                      \
  } NAME##_job;                                                                \
                                                                               \
  static void NAME##_rows(NAME##_job *j, int o, int i0, int i1) {              \
    const oracle_desc *d = j->d;                                               \
    plane_map m = make_map(d);                                                 \
    int sampling = eff_sampling(d);                                            \
    int step = sampling == OR_NOSAMPLE ? 1 : d->step;                          \
    int down = sampling == OR_DOWN ? step : 1;                                 \
    /* FilterAdjoint upsamples the gradient (taps at multiples of fup), the \
     * other modes the input (:1313-1326) */                                  \
    int fa = d->mode == OR_FILTER_ADJOINT || d->mode == OR_FILTER_ADJOINT_REDUCE; \
    int up = (sampling == OR_UP && !fa) ? step : 1;                            \
    int fup = (sampling == OR_UP && fa) ? step : 1;                            \
    int FR = d->f_rows, FS = d->f_cols;                                        \
    int R = FR * fup, S = FS * fup, H = d->rows, W = d->cols;                  \
    int hr = low_halo(d->border, R), hc = low_halo(d->border, S);              \
    int terms = map_terms(&m, o);                                              \
    size_t page = (size_t)H * W, fpage = (size_t)FR * FS;                      \
    for (int i = i0; i < i1; i++) {                                            \
      for (int jj = 0; jj < j->ocols; jj++) {                                  \
        T acc = 0;                                                             \
        for (int t = 0; t < terms; t++) {                                      \
          int ip, fp;                                                          \
          map_pair(&m, o, t, &ip, &fp);                                        \
          const T *xp = j->x + (size_t)ip * page;                              \
          const T *fpp = j->f + (size_t)fp * fpage;                            \
          T rowSum = 0;                                                        \
          /* post-sampling origin of this output's window */                   \
          int pr0 = i * down - hr, pc0 = jj * down - hc;                       \
          for (int r = 0; r < R; r++) {                                        \
            int pr = pr0 + r;                                                  \
            if (up > 1 && ((pr % up) + up) % up != 0) continue; /* :429 */     \
            int sr = border_index(d->border, up > 1 ? div_floor(pr, up) : pr, H); \
            T colSum = 0;                                                      \
            int er = d->orient == OR_CONV ? R - 1 - r : r;                     \
            for (int s = 0; s < S; s++) {                                      \
              int pc = pc0 + s;                                                \
              if (up > 1 && ((pc % up) + up) % up != 0) continue;              \
              int sc = border_index(d->border, up > 1 ? div_floor(pc, up) : pc, W); \
              T v = (sr < 0 || sc < 0) ? (T)0 : xp[(size_t)sr * W + sc];       \
              int es = d->orient == OR_CONV ? S - 1 - s : s;                   \
              T w = (er % fup == 0 && es % fup == 0)                           \
                        ? fpp[(size_t)(er / fup) * FS + es / fup] : (T)0;      \
              colSum = FMA(v, w, colSum);                                      \
            }                                                                  \
            rowSum = rowSum + colSum;                                          \
          }                                                                    \
          acc = (terms == 1) ? rowSum : acc + rowSum;                          \
        }                                                                      \
        j->y[(size_t)o * j->orows * j->ocols + (size_t)i * j->ocols + jj] = acc; \
      }                                                                        \
    }                                                                          \
  }                                                                            \
                                                                               \
  enum { NAME##_ROWS_PER_ITEM = 4 };                                           \
  static void *NAME##_worker(void *arg) {                                      \
    NAME##_job *j = (NAME##_job *)arg;                                         \
    int blocks = (j->orows + NAME##_ROWS_PER_ITEM - 1) / NAME##_ROWS_PER_ITEM; \
    int total = blocks * j->oplanes;                                           \
    for (;;) {                                                                 \
      pthread_mutex_lock(&j->lock);                                            \
      int item = j->next++;                                                    \
      pthread_mutex_unlock(&j->lock);                                          \
      if (item >= total) break;                                                \
      int o = item / blocks, blk = item % blocks;                              \
      int i0 = blk * NAME##_ROWS_PER_ITEM;                                     \
      int i1 = i0 + NAME##_ROWS_PER_ITEM;                                      \
      if (i1 > j->orows) i1 = j->orows;                                        \
      NAME##_rows(j, o, i0, i1);                                               \
    }                                                                          \
    return NULL;                                                               \
  }                                                                            \
                                                                               \
  int NAME(const oracle_desc *d, const T *x, const T *f, T *y, int threads) {  \
    NAME##_job j;                                                              \
    if (oracle_output_shape(d, &j.orows, &j.ocols, &j.oplanes, NULL, 0)) return 1; \
    j.d = d; j.x = x; j.f = f; j.y = y; j.next = 0;                            \
    pthread_mutex_init(&j.lock, NULL);                                         \
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);            \
    if (threads < 1) threads = 1;                                              \
    if (threads > 256) threads = 256;                                          \
    pthread_t tid[256];                                                        \
    int started = 0;                                                           \
    for (int t = 1; t < threads; t++)                                          \
      if (pthread_create(&tid[started], NULL, NAME##_worker, &j) == 0) started++; \
    NAME##_worker(&j);                                                         \
    for (int t = 0; t < started; t++) pthread_join(tid[t], NULL);              \
    pthread_mutex_destroy(&j.lock);                                            \
    return 0;                                                                  \
  }

static inline float fma32(float a, float b, float c) { return fmaf(a, b, c); }
static inline double fma64(double a, double b, double c) { return fma(a, b, c); }

DEFINE_CONV(oracle_conv_f32, float, fma32)
DEFINE_CONV(oracle_conv_f64, double, fma64)

/* One 1-D pass of the separable convolution (ConvolveRows2DHyperKernel.scala
 * :66-160): out[i] = sum_k in[i - halo + k] * f'[k], f' flipped for CONV,
 * accumulated as one fused multiply-add chain from 0. */
static void sep_pass(const float *in, float *out, int n_lines, int len,
                     size_t line_stride, size_t elem_stride, const float *f,
                     int flen, int border, int orient) {
  int halo = (flen - 1) / 2;
  for (int l = 0; l < n_lines; l++) {
    const float *ip = in + (size_t)l * line_stride;
    float *op = out + (size_t)l * line_stride;
    for (int i = 0; i < len; i++) {
      float sum = 0.0f;
      for (int k = 0; k < flen; k++) {
        int idx = border_index(border, i - halo + k, len);
        float v = idx < 0 ? 0.0f : ip[(size_t)idx * elem_stride];
        float w = orient == OR_CONV ? f[flen - 1 - k] : f[k];
        sum = fmaf(v, w, sum);
      }
      op[(size_t)i * elem_stride] = sum;
    }
  }
}

int oracle_separable_f32(int rows, int cols, int planes, const float *x,
                         const float *row_f, int row_len, const float *col_f,
                         int col_len, int border, int orient, float *y) {
  if (border != OR_ZERO && border != OR_CLAMP && border != OR_CYCLIC) return 1;
  if (row_len % 2 == 0 || col_len % 2 == 0) return 1;
  size_t page = (size_t)rows * cols;
  float *tmp = (float *)malloc(page * sizeof(float));
  if (!tmp) return 1;
  for (int p = 0; p < planes; p++) {
    sep_pass(x + p * page, tmp, rows, cols, cols, 1, row_f, row_len, border, orient);
    sep_pass(tmp, y + p * page, cols, rows, 1, cols, col_f, col_len, border, orient);
  }
  free(tmp);
  return 0;
}

/* Scalar field (*) matrix field (ScalarMatrixConvolve2DHyperKernel.scala:
 * 59-85; reached from CogFunctionAPI.scala:1209-1216 when a scalar field is
 * convolved with a matrix field).  Output plane p = row * mcols + col is the
 * cross-correlation of x with the size x size matrix at (row, col), summed as
 * ONE fused multiply-add chain from 0 over the taps in row-major order (the
 * kernel's `sum += inputPixel * filterElement`, contracted under
 * -cl-mad-enable), with halo size / 2 and the border's index rule.  The
 * matrix field is stored tensor-element-major: element (r, c) of matrix p at
 * mats[(r * size + c) * (mrows * mcols) + p]. */
int oracle_scalar_matrix_f32(int rows, int cols, const float *x, const float *mats,
                             int mrows, int mcols, int size, int border, float *y) {
  if (border != OR_ZERO && border != OR_CLAMP && border != OR_CYCLIC) return 1;
  if (size < 1 || size % 2 == 0 || mrows < 1 || mcols < 1) return 1;
  const int L = mrows * mcols, h = size / 2;
  const size_t page = (size_t)rows * cols;
  for (int p = 0; p < L; p++)
    for (int i = 0; i < rows; i++)
      for (int j = 0; j < cols; j++) {
        float sum = 0.0f;
        for (int r = 0; r < size; r++) {
          const int si = border_index(border, i - h + r, rows);
          for (int c = 0; c < size; c++) {
            const int sj = border_index(border, j - h + c, cols);
            const float v = (si < 0 || sj < 0) ? 0.0f : x[(size_t)si * cols + sj];
            sum = fmaf(v, mats[(size_t)(r * size + c) * L + p], sum);
          }
        }
        y[(size_t)p * page + (size_t)i * cols + j] = sum;
      }
  return 0;
}

/* ColorField planes (ColorPlaneHyperKernel.scala:38-44 reads a pixel of the
 * RGBA UNORM_INT8 image, OpenCLBuffer.scala:135-136): channel byte c reads
 * as c / 255 (the OpenCL conversion for UNORM_INT8, rounded to nearest).
 * planes[k * n + i] = channel k (red, green, blue) of pixel i. */
void oracle_color_unpack(int n, const unsigned char *rgba, float *planes) {
  for (int i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) planes[(size_t)k * n + i] = (float)rgba[4 * (size_t)i + k] / 255.0f;
}

/* MergeColorPlanes (CreateColorFieldHyperKernel.scala:35-40) writes
 * (red, green, blue, 1) to the UNORM_INT8 image: per channel
 * convert_uchar_sat_rte(v * 255.0f) (NaN -> 0, saturate to [0, 255], round
 * half to even). */
void oracle_color_pack(int n, const float *planes, unsigned char *rgba) {
  for (int i = 0; i < n; i++) {
    for (int k = 0; k < 3; k++) {
      const float v = planes[(size_t)k * n + i] * 255.0f;
      float q = v > 0.0f ? v : 0.0f; /* NaN -> 0 */
      if (q > 255.0f) q = 255.0f;
      rgba[4 * (size_t)i + k] = (unsigned char)nearbyintf(q);
    }
    rgba[4 * (size_t)i + 3] = 255;
  }
}
