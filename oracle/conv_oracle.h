/*
 * CPU oracle for the field-convolution hot path.  TEST INFRASTRUCTURE ONLY:
 * used by tests/, the smoke check and the CPU baseline leg of bench.py as the
 * checker.  The product path never links or calls this code.
 *
 * Restates, per output element and in the reference's summation order, the
 * direct convolution that cct-core generates as OpenCL C in
 *   src/main/scala/cogx/compiler/codegenerator/opencl/hyperkernels/ConvolveHyperKernel.scala
 * (border handling :235-317, sampling :205-223 and :404-459, orientation
 * :345-384, plane mixing :124-199 and :319-340, output :574-645) and the
 * output-shape / legality rules of ConvolveHyperKernel.outputFieldType
 * (:1297-1450) and DynamicConvolutionGenerator.convolveDirectly
 * (generator/DynamicConvolutionGenerator.scala:484-539).
 *
 * Parity is pinned by the reference's own golden vectors
 * (src/test/resources/platform/opencl/hyperkernels/convolutionDynamic/) and
 * the known-answer tests of src/test/scala/cogx/StaticConvolutionSpec.scala.
 */
#ifndef CCT_CONV_ORACLE_H
#define CCT_CONV_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Same numeric codes as the product C-ABI (include/cct_conv.h). */
enum { OR_ZERO = 0, OR_CLAMP = 1, OR_CYCLIC = 2, OR_VALID = 3, OR_FULL = 4 };
enum { OR_XCORR = 0, OR_CONV = 1 };
enum { OR_NOSAMPLE = 0, OR_DOWN = 1, OR_UP = 2 };
enum { OR_PLANE = 0, OR_PROJECT = 1, OR_PROJECT_REDUCE = 2,
       OR_BACKPROJECT = 3, OR_BACKPROJECT_REDUCE = 4,
       OR_FILTER_ADJOINT = 5, OR_FILTER_ADJOINT_REDUCE = 6 };

typedef struct {
  int rows, cols;          /* input field shape (rows = 1 for a 1-D field)   */
  int planes;              /* input tensor points (1 for a ScalarField)       */
  int f_rows, f_cols;      /* filter field shape                              */
  int f_planes;            /* filter tensor points                            */
  int batch;               /* logical images in the input (frame modes)       */
  int border, orient, sampling, step, mode;
} oracle_desc;

/* Output shape + legality.  Returns 0 and fills the outputs, or a non-zero
 * code with a message in err (err may be NULL). */
int oracle_output_shape(const oracle_desc *d, int *out_rows, int *out_cols,
                        int *out_planes, char *err, int errlen);

/* Direct convolution in the reference's order, FP32 with fused multiply-add
 * per tap (the reference builds with -cl-mad-enable) and separate adds for
 * the row and plane sums.  threads <= 0 means all online cores. */
int oracle_conv_f32(const oracle_desc *d, const float *x, const float *f,
                    float *y, int threads);
/* The same loops in double precision. */
int oracle_conv_f64(const oracle_desc *d, const double *x, const double *f,
                    double *y, int threads);

/* Separable convolution: rows pass then columns pass
 * (ConvolveRows2DHyperKernel.scala / ConvolveColumns2DHyperKernel.scala).
 * border in {ZERO, CLAMP, CYCLIC}; planes processed independently. */
int oracle_separable_f32(int rows, int cols, int planes, const float *x,
                         const float *row_f, int row_len, const float *col_f,
                         int col_len, int border, int orient, float *y);

/* Scalar field cross-correlated with every matrix of a matrix field
 * (ScalarMatrixConvolve2DHyperKernel.scala): one output plane per matrix,
 * one fma chain per output over the taps in row-major order.  border in
 * {ZERO, CLAMP, CYCLIC}; size odd.  mats is tensor-element-major. */
int oracle_scalar_matrix_f32(int rows, int cols, const float *x, const float *mats,
                             int mrows, int mcols, int size, int border, float *y);

/* ColorField <-> planes: RGBA8 pixels (alpha ignored on read, 255 on write)
 * to three float planes (byte / 255) and back (saturate, x 255, round half to
 * even), as the OpenCL UNORM_INT8 image conversions. */
void oracle_color_unpack(int n, const unsigned char *rgba, float *planes);
void oracle_color_pack(int n, const float *planes, unsigned char *rgba);

#ifdef __cplusplus
}
#endif
#endif
