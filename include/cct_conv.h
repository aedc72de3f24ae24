/*
 * cct_conv.h -- C-ABI of the B200 field-convolution backend (libcctconv.so).
 *
 * Drop-in replacement for the device half of cct-core's convolution path:
 * the Scala ComputeGraph keeps building `ConvolveOp` nodes, and the code
 * generator's `case op: ConvolveOp =>` arm hands them to this library instead
 * of emitting OpenCL ConvolveHyperKernel/FFT2DHyperKernel text.  Plain C types
 * only (ints, float pointers, an opaque plan handle, a CUDA stream passed as
 * void*), so JNI, Panama, ctypes or C++ can bind it unchanged.
 *
 * Memory layout (identical to cct-core's FieldMemoryLayoutImpl, so no repack):
 * a field with P tensor planes of rows x cols is P consecutive pages, each
 * page row-major with rowStride = cols and no padding
 * (src/main/scala/cogx/platform/types/FieldMemoryLayoutImpl.scala:250-311).
 * Frame modes index image plane b*N + c, filter plane k*N + c, fused output
 * plane b*K + k.
 *
 * Errors: every entry point returns CCT_OK (0) or a negative status and never
 * throws; cct_last_error_string() describes the last failure on the calling
 * thread.  This replaces the reference's RuntimeException from event status
 * (src/main/scala/cogx/platform/opencl/OpenCLDeviceKernel.scala:106-147).
 */
#ifndef CCT_CONV_H
#define CCT_CONV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CCT_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------- */
enum {
  CCT_OK = 0,
  CCT_EINVAL = -1,    /* descriptor rejected (same rules as the reference)   */
  CCT_ENOTSUP = -2,   /* legal in the reference, not offered by this library */
  CCT_ENOMEM = -3,    /* device or host allocation failed                    */
  CCT_ECUDA = -4,     /* CUDA runtime / launch error                         */
  CCT_ETIMEOUT = -5,  /* a bounded device wait gave up                       */
  CCT_ENODEV = -6     /* no sm_100 device visible                            */
};

/* ---- policies: numeric values are part of the ABI ----------------------- */
/* BorderPolicy (src/main/scala/cogx/platform/types/BorderPolicy.scala:30-134) */
enum { CCT_BORDER_ZERO = 0, CCT_BORDER_CLAMP = 1, CCT_BORDER_CYCLIC = 2,
       CCT_BORDER_VALID = 3, CCT_BORDER_FULL = 4 };
/* FilterOrientation (src/main/scala/cogx/platform/types/FilterOrientation.scala:28-30) */
enum { CCT_CROSS_CORRELATION = 0, CCT_CONVOLUTION = 1 };
/* ConvolutionSamplingPolicy (src/main/scala/cogx/platform/types/ConvolutionSamplingPolicy.scala:27-31) */
enum { CCT_SAMPLE_NONE = 0, CCT_SAMPLE_DOWN = 1, CCT_SAMPLE_UP = 2 };
/* VectorMode (src/main/scala/cogx/compiler/parser/op/BinaryOpcode.scala:36-46).
 * FILTER_ADJOINT (crossCorrelateFilterAdjoint / convolveFilterAdjoint,
 * CogFunctionAPI.scala:1480-1511): the "filter" operand is the gradient field
 * of batch*L planes; output plane B*w + b (w = l*C + c) is image plane
 * b*C + c correlated with gradient plane b*L + l (ConvolveHyperKernel.scala
 * :187, 333, 575-590), and UpsampleInput upsamples the gradient, not the
 * image (:1313-1326).  FILTER_ADJOINT_BLOCK_REDUCE_SUM sums the B images of
 * each w in order (the fused blockReduceSum(filterAdjoint(..), B)). */
enum { CCT_PLANE_BY_PLANE = 0, CCT_PROJECT_FRAME = 1,
       CCT_PROJECT_FRAME_BLOCK_REDUCE_SUM = 2, CCT_BACK_PROJECT_FRAME = 3,
       CCT_BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM = 4, CCT_FILTER_ADJOINT = 5,
       CCT_FILTER_ADJOINT_BLOCK_REDUCE_SUM = 6 };
/* Arithmetic of the multi-plane kernels.  FP32 is the reference's
 * arithmetic; BF16X3 splits each FP32 operand into bf16 hi+lo and sums the
 * hi*hi + hi*lo + lo*hi products on tcgen05 tensor cores in FP32.  BF16X3
 * applies to the BlockReduceSum modes: the frame modes (PROJECT_FRAME_ and
 * BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM) and FILTER_ADJOINT_BLOCK_REDUCE_SUM
 * (the weight gradient, with BorderValid and no sampling).  BF16X6 (frame
 * modes only) splits each operand into three bf16 terms hi+mid+lo and sums
 * the six products down to 2^-16 of hi*hi (hh, hm, mh, hl, lh, mm): FP32-level
 * accuracy for compositions such as a stack of layers, at about twice the
 * tensor work of BF16X3.  Shapes the tensor-core kernels do not take run on
 * the FP32 kernels. */
enum { CCT_PREC_FP32 = 0, CCT_PREC_BF16X3 = 1, CCT_PREC_BF16X6 = 2 };
/* Direct vs FFT (ConvolutionFFTUsePolicy.scala:24-28 UseFFTNever/Always/WhenBest) */
enum { CCT_ALGO_AUTO = 0, CCT_ALGO_DIRECT = 1, CCT_ALGO_FFT = 2 };
/* flags */
#define CCT_FLAG_RELU 0x1u   /* fuse max(y, 0) into the store (CogFunctionAPI.scala:109) */

/* ---- descriptor: one ConvolveOp applied to (image, filter) field types ---- */
typedef struct cct_conv_desc {
  int32_t struct_size;   /* sizeof(cct_conv_desc), for ABI evolution           */
  int32_t image_rows;    /* image field shape; 1-D fields use rows = 1         */
  int32_t image_cols;
  int32_t image_planes;  /* tensor points; 0 = ScalarField (tensor order 0)    */
  int32_t filter_rows;
  int32_t filter_cols;
  int32_t filter_planes; /* 0 = ScalarField                                    */
  int32_t batch_size;    /* logical images in the image field (frame modes)    */
  int32_t border;        /* CCT_BORDER_*                                       */
  int32_t orientation;   /* CCT_CROSS_CORRELATION / CCT_CONVOLUTION            */
  int32_t sampling;      /* CCT_SAMPLE_*                                       */
  int32_t step;          /* sampling step (ignored for CCT_SAMPLE_NONE)        */
  int32_t vector_mode;   /* CCT_PLANE_BY_PLANE ... BLOCK_REDUCE_SUM            */
  int32_t precision;     /* CCT_PREC_*                                         */
  int32_t algo;          /* CCT_ALGO_*                                         */
  uint32_t flags;        /* CCT_FLAG_*                                         */
} cct_conv_desc;

typedef struct cct_conv_plan cct_conv_plan;

/* Fill a descriptor with defaults (scalar fields, BorderZero, convolution,
 * no sampling, plane-by-plane, FP32, AUTO). */
void cct_conv_desc_init(cct_conv_desc *desc);

/* Output field shape + legality of a descriptor, without touching the GPU.
 * Replaces ConvolveHyperKernel.outputFieldType
 * (src/main/scala/cogx/compiler/codegenerator/opencl/hyperkernels/ConvolveHyperKernel.scala:1297-1450)
 * and the checks of DynamicConvolutionGenerator.convolveDirectly
 * (src/main/scala/cogx/compiler/codegenerator/opencl/generator/DynamicConvolutionGenerator.scala:484-539). */
int cct_conv_output_shape(const cct_conv_desc *desc, int32_t *out_rows,
                          int32_t *out_cols, int32_t *out_planes);

/* Compile-time half of the reference's DynamicConvolutionGenerator.apply
 * (generator/DynamicConvolutionGenerator.scala:76-150, direct/FFT triage) and
 * ConvolveHyperKernel.apply (hyperkernels/ConvolveHyperKernel.scala:1003-1148,
 * parameter choice): validates, picks the kernel family and tile shape for
 * the current device, and allocates every device buffer the plan needs so
 * that cct_conv_run allocates nothing. */
int cct_conv_plan_create(const cct_conv_desc *desc, cct_conv_plan **plan);
int cct_conv_plan_destroy(cct_conv_plan *plan);

/* Kernel family the plan chose: 0 direct stencil, 1 frame FP32, 2 frame
 * BF16X3 tensor core, 3 FFT, 4 FilterAdjoint FP32, 5 FilterAdjoint BF16X3
 * tensor core. */
int cct_conv_plan_algo(const cct_conv_plan *plan, int32_t *algo_out);

/* Static filter (the reference's ConstantFieldKernel filter): its FFT
 * spectrum, or its packed tensor-core operand, is computed once here in
 * FP64 / on the device, as the reference does on the host at compile time
 * (generator/DynamicConvolutionGenerator.scala:342-350, 376-405).  After this
 * call cct_conv_run accepts filter == NULL.  host_filter holds
 * filter_planes x filter_rows x filter_cols floats. */
int cct_conv_plan_set_static_filter(cct_conv_plan *plan, const float *host_filter);

/* One step of the op: device pointers in the planar layout above, enqueued on
 * `stream` (a cudaStream_t; NULL = legacy default stream).  Replaces the
 * per-step launch OpenCLDeviceKernel.phase1Clock -> put{2,3}DRangeKernel
 * (src/main/scala/cogx/platform/opencl/OpenCLDeviceKernel.scala:67-104,
 * 189-215).  Asynchronous; allocates nothing.  filter may be NULL after
 * cct_conv_plan_set_static_filter. */
int cct_conv_run(const cct_conv_plan *plan, const float *image,
                 const float *filter, float *out, void *stream);

/* The same step with HOST buffers: pinned staging + device copies owned by
 * the plan, H2D of image (and filter unless static), the kernel, D2H of the
 * result, then a stream synchronise.  What a JNI caller holding Java direct
 * buffers uses in place of OpenCLBuffer.write/read
 * (src/main/scala/cogx/platform/opencl/OpenCLBuffer.scala:207-230). */
int cct_conv_run_host(cct_conv_plan *plan, const float *host_image,
                      const float *host_filter, float *host_out, void *stream);

/* Separable convolution: rows pass then columns pass, BorderZero / Clamp /
 * Cyclic, odd 1-D filters, every plane of the image.  Replaces
 * ConvolveRows2DHyperKernel + ConvolveColumns2DHyperKernel
 * (hyperkernels/ConvolveRows2DHyperKernel.scala:37-160,
 * hyperkernels/ConvolveColumns2DHyperKernel.scala:37-160) behind
 * convolveSeparable / crossCorrelateSeparable (api/CogFunctionAPI.scala:1277-1366).
 * tmp is a device buffer of planes*rows*cols floats. */
int cct_conv_separable(int32_t rows, int32_t cols, int32_t planes,
                       const float *image, const float *row_filter,
                       int32_t row_len, const float *col_filter,
                       int32_t col_len, int32_t border, int32_t orientation,
                       float *tmp, float *out, void *stream);

/* A ScalarField cross-correlated with every matrix of a MatrixField: the form
 * api/CogFunctionAPI.scala:1209-1216 selects for convolve/crossCorrelate of a
 * scalar field with a matrix field; replaces
 * hyperkernels/ScalarMatrixConvolve2DHyperKernel.scala:43-160.
 *   image     rows x cols
 *   matrices  a matrix field of matrix_rows x matrix_cols points, each a
 *             size x size matrix, stored tensor-element-major: element
 *             (r, c) of matrix p = row * matrix_cols + col is at
 *             matrices[(r * size + c) * matrix_rows * matrix_cols + p]
 *   out       matrix_rows * matrix_cols planes of rows x cols (a vector field)
 * Each output is one fused multiply-add chain from 0 over the taps in
 * row-major order, as the reference kernel sums.  The reference's
 * restrictions and messages hold: BorderZero / Clamp / Cyclic, no sampling
 * (step 1 counts as none), cross-correlation only, odd size. */
int cct_conv_scalar_matrix(int32_t rows, int32_t cols, const float *image,
                           const float *matrices, int32_t matrix_rows,
                           int32_t matrix_cols, int32_t size, int32_t border,
                           int32_t orientation, int32_t sampling, int32_t step,
                           float *out, void *stream);

/* Colour-field convolution (generator/DynamicConvolutionGenerator.scala:
 * 89-106).  A ColorField is an RGBA8 image, 4 bytes per pixel, as the
 * reference's UNORM_INT8 image buffer (platform/opencl/OpenCLBuffer.scala:
 * 135-136); alpha is ignored on input.  Each of red, green, blue (byte / 255)
 * is convolved with the one scalar filter as `desc` describes: the image
 * shape, filter shape, border, orientation, sampling and algorithm of a
 * plane-by-plane convolution (image_planes 0 or 1, filter_planes 0 or 1,
 * FP32).  The result is an RGBA8 colour field of the output shape
 * (cct_conv_output_shape of desc) with each channel saturate(v * 255)
 * rounded half to even and alpha 255, as CreateColorFieldHyperKernel writes
 * (hyperkernels/CreateColorFieldHyperKernel.scala:35-40).  Image and output
 * must be 4-byte aligned device pointers; the plan owns six planes of
 * workspace. */
typedef struct cct_color_plan cct_color_plan;
int cct_color_plan_create(const cct_conv_desc *desc, cct_color_plan **plan);
int cct_color_plan_set_static_filter(cct_color_plan *plan, const float *host_filter);
int cct_color_run(const cct_color_plan *plan, const uint8_t *image,
                  const float *filter, uint8_t *out, void *stream);
int cct_color_plan_destroy(cct_color_plan *plan);

/* Allocation-free variant of the BF16X3 BlockReduceSum frame convolution (no
 * counterpart in the reference, which always lets its runtime own device
 * buffers).  For callers that cannot call cudaMalloc when they convolve:
 * hosts that reserve all device memory up front in their own arena, and
 * latency-sensitive callers for whom cudaMalloc/cudaFree (which may
 * synchronise the device) are off limits.  It creates no plan and allocates
 * nothing: image, filter and out are the caller's device pointers; the
 * kernel's only scratch, the packed bf16 hi/lo filter operand, lives in a
 * fixed device array of 4 MiB (held by every GPU that loads the library
 * until exit).  Descriptors whose packed operand exceeds 4 MiB are rejected
 * with CCT_EINVAL; shapes the tensor-core kernel does not take return
 * CCT_ENOTSUP.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and caches it for the life of the CUDA
 * context; make that first call before any stream capture.  All calls on a
 * device share the array: calls that overlap on the GPU race and must be
 * ordered by the caller.  A bounded wait that gives up inside this kernel is
 * recorded in the same statically allocated device error word as every
 * plan's kernels, and reported (then cleared) by cct_device_status(). */
int cct_conv_run_noalloc(const cct_conv_desc *desc, const float *image,
                         const float *filter, float *out, void *stream);

/* ---- checkpoint records ---------------------------------------------------
 * What ComputeGraph.write / readFromFile
 * (src/main/scala/cogx/runtime/ComputeGraph.scala:523-727) save for a kernel
 * of this backend, in place of the OpenCL kernel's source code and
 * work-group parameters (platform/opencl/OpenCLDeviceKernel.scala:219-229,
 * OpenCLRestoredDeviceKernel.scala:53-64).  A plan or graph is determined by
 * its descriptors and constant filters, so a record holds those (and a
 * graph's step count); restoring creates new plans on the current device.
 *
 * A record is an array of 32-bit words (store it with the saver's
 * writeIntArray): magic 0x4B544343, format version 1, kind (1 plan,
 * 2 graph), layer count, step count (low, high word); per layer the number
 * of descriptor fields (15), the fields image_rows .. flags in declaration
 * order, the constant filter's element count (low, high; 0 = none) and its
 * values as IEEE-754 bits; last an FNV-1a 32-bit hash of the preceding
 * words' bytes (each word little-endian).
 *
 * *_save: with words == NULL, only *n_words is set (the size to allocate);
 * else the record is written if capacity (in words) suffices, CCT_EINVAL
 * otherwise.  A saved plan's constant filter is read back from the device.
 * *_restore: CCT_EINVAL on a bad magic, version, kind, length or checksum.
 * cct_record_describe: the kind, layer count, step count and up to
 * max_descs layer descriptors of a record, without touching a device. */
int cct_conv_plan_save(const cct_conv_plan *plan, uint32_t *words,
                       size_t capacity, size_t *n_words);
int cct_conv_plan_restore(const uint32_t *words, size_t n_words,
                          cct_conv_plan **plan);
int cct_record_describe(const uint32_t *words, size_t n_words, int32_t *kind,
                        int32_t *n_layers, int64_t *time,
                        cct_conv_desc *descs, int32_t max_descs);

/* ---- stacked convolution graphs (ComputeGraph step) --------------------- */
/* A ComputeGraph whose fields form a chain of convolutions: layer i reads
 * layer i-1's output field.  Replaces the reference's ComputeGraph
 * construction and its evaluator's per-kernel dispatch for such graphs
 * (src/main/scala/cogx/runtime/ComputeGraph.scala:56, step :228-279,
 * reset :288): the layers' launches are captured once into a CUDA graph and
 * every step replays it.  The graph owns every field: the input field
 * (index 0) and each layer's output (index i); filters are static (the
 * reference's constant filter fields), set once per layer.
 *
 * cct_graph_create   layer descriptors; each layer's image shape must equal
 *                    the previous layer's output shape.  CCT_EINVAL with a
 *                    message naming the layer otherwise.
 * cct_graph_set_filter  host filter of one layer (as cct_conv_plan_set_static_filter).
 * cct_graph_field    device pointer and element count of field `index`.
 * cct_graph_step     `count` steps on `stream` (asynchronous; the first step
 *                    captures the launch sequence, and fails with CCT_EINVAL
 *                    while a layer has no filter).  Kernel-side timeouts are
 *                    reported by cct_device_status.
 * cct_graph_step_host  one step from a host input to the host copy of the
 *                    last layer's output (synchronous).
 * cct_graph_time     steps taken since creation or the last reset.
 * cct_graph_reset    sets the step count to 0 (the fields keep their values). */
typedef struct cct_graph cct_graph;
int cct_graph_create(const cct_conv_desc *layers, int32_t n_layers, cct_graph **out);
int cct_graph_destroy(cct_graph *graph);
int cct_graph_set_filter(cct_graph *graph, int32_t layer, const float *host_filter);
int cct_graph_field(const cct_graph *graph, int32_t index, float **device_ptr, size_t *elems);
int cct_graph_step(cct_graph *graph, int64_t count, void *stream);
int cct_graph_step_host(cct_graph *graph, const float *host_in, float *host_out, void *stream);
int64_t cct_graph_time(const cct_graph *graph);
int cct_graph_reset(cct_graph *graph);
/* Checkpoint records of a graph (format above): every layer's descriptor and
 * constant filter, and the step count.  Restoring recreates the graph on the
 * current device with zeroed fields and the saved step count. */
int cct_graph_save(const cct_graph *graph, uint32_t *words, size_t capacity,
                   size_t *n_words);
int cct_graph_restore(const uint32_t *words, size_t n_words, cct_graph **graph);

/* ---- kernel circuits (ComputeGraph step over a DAG) --------------------- */
/* A ComputeGraph as a directed acyclic graph of operations over fields: the
 * reference's KernelCircuit, enqueued in one fixed order every step
 * (src/main/scala/cogx/runtime/execution/GPUSupervisor.scala:128-215), its
 * fields packed into shared device buffers once nothing reads them any more
 * (runtime/allocation/InOrderSharedLatchAllocator.scala:34: in-order
 * execution, buffers binned by field size), inputs fed by sensors and
 * results read by actuators (runtime/Sensor.scala:73).  The launches are
 * captured once into a CUDA graph and every step replays it.
 *
 * Fields 0 .. n_inputs-1 are the inputs (sensors); field n_inputs + i is the
 * output of node i.  Nodes are listed in execution order: a node reads only
 * fields defined before it.  Inputs and the listed outputs keep buffers of
 * their own; every other field shares a buffer of its size with fields whose
 * last reader has run.
 *
 * cct_circuit_node   op CCT_NODE_CONV: `conv` describes the convolution, in0
 *                    is its image field (shape as conv.image_*), in1 its
 *                    filter field or -1 for a static filter set with
 *                    cct_circuit_set_filter.  ADD / SUB / MUL: in0 op in1
 *                    (equal element counts).  RELU: max(in0, 0).  SCALE:
 *                    in0 * scalar.  Elementwise outputs take in0's shape.
 * cct_circuit_assign the buffer assignment alone (host only, no device):
 *                    field_buffer[n_inputs + n_nodes] and the buffer count.
 * cct_circuit_create validates and plans every node, allocates the buffers
 *                    (zeroed); CCT_EINVAL with a message naming the node.
 * cct_circuit_step   `count` steps on `stream` (the first captures; fails
 *                    with CCT_EINVAL while a static-filter node has none).
 * cct_circuit_step_host  copies each host input in, steps once, copies each
 *                    listed output to the host (synchronous).
 * cct_circuit_buffers  device buffers in use and their bytes. */
enum {
  CCT_NODE_CONV = 0,
  CCT_NODE_ADD = 1,
  CCT_NODE_SUB = 2,
  CCT_NODE_MUL = 3,
  CCT_NODE_RELU = 4,
  CCT_NODE_SCALE = 5
};
typedef struct {
  int32_t rows, cols, planes; /* planes < 1: a scalar field (1 plane) */
} cct_field_shape;
typedef struct {
  int32_t op;          /* CCT_NODE_*                                       */
  int32_t in0, in1;    /* input fields; -1 where unused                    */
  float scalar;        /* CCT_NODE_SCALE factor                            */
  cct_conv_desc conv;  /* CCT_NODE_CONV                                    */
} cct_circuit_node;
typedef struct cct_circuit cct_circuit;
int cct_circuit_assign(const cct_field_shape *inputs, int32_t n_inputs,
                       const cct_circuit_node *nodes, int32_t n_nodes,
                       const int32_t *outputs, int32_t n_outputs,
                       int32_t *field_buffer, int32_t *n_buffers);
int cct_circuit_create(const cct_field_shape *inputs, int32_t n_inputs,
                       const cct_circuit_node *nodes, int32_t n_nodes,
                       const int32_t *outputs, int32_t n_outputs,
                       cct_circuit **out);
int cct_circuit_destroy(cct_circuit *circuit);
int cct_circuit_set_filter(cct_circuit *circuit, int32_t node, const float *host_filter);
int cct_circuit_field(const cct_circuit *circuit, int32_t field, float **device_ptr,
                      size_t *elems);
int cct_circuit_buffers(const cct_circuit *circuit, int32_t *n_buffers, size_t *bytes);
int cct_circuit_step(cct_circuit *circuit, int64_t count, void *stream);
int cct_circuit_step_host(cct_circuit *circuit, const float *const *host_inputs,
                          float *const *host_outputs, void *stream);
int64_t cct_circuit_time(const cct_circuit *circuit);
int cct_circuit_reset(cct_circuit *circuit);

/* ---- request serving (continuous batching) ------------------------------ */
/* No counterpart in the reference, whose ComputeGraphs are stepped by one
 * caller at a time.  A server serves one GPU with a scheduler thread.
 * Requests (a convolution, or a step of a resident cct_graph) arrive from
 * any thread; each is admitted when device memory for its fields can be
 * had: from the server's chunks of device memory, or from the device's free
 * HBM (cudaMemGetInfo) less `hbm_reserve_bytes`, claimed as a new chunk;
 * `arena_bytes`, if nonzero, caps what the server holds.  Its inputs are
 * copied in, and admitted
 * requests are batched into one persistent kernel launch (a captured CUDA
 * graph per launch slot) whose CTAs pull tiles of every request in the
 * batch.  Up to `slots` launches are in flight on their own streams, so
 * requests that arrive while others run are admitted and overlap with them.
 * Requests too large to gain from batching run on their own plan on the
 * same streams.  Every route computes each output with the reference's
 * per-output FP32 order, so a result is bit-identical alone and in a mix.
 *
 * Convolution requests: FP32, BorderZero, no sampling, odd square filters up
 * to 9x9 in the batch kernel (other descriptors run on their own plan);
 * PLANE_BY_PLANE or PROJECT_FRAME_BLOCK_REDUCE_SUM with batch_size 1.
 * Host pointers must stay valid until the request completes; pinned host
 * memory (cct_host_alloc) gives full copy bandwidth.
 * flags CCT_SERVE_PER_CALL: no batching; each request alone, in arrival
 * order, through its plan with a synchronise per request (the plain
 * per-call dispatch that serving is compared with). */
enum { CCT_SERVE_CONV = 0, CCT_SERVE_GRAPH_STEP = 1 };
enum { CCT_SERVE_PER_CALL = 0x1 };
typedef struct cct_server_config {
  int32_t struct_size;  /* sizeof(cct_server_config) */
  int32_t slots;        /* launches in flight (1..8; 0 = 3) */
  int32_t max_batch;    /* requests per launch (1..256; 0 = 64) */
  int32_t flags;
  uint64_t arena_bytes; /* cap on the HBM the server holds (0 = none: admission by free HBM) */
  uint64_t hbm_reserve_bytes; /* free HBM the server leaves to other work (0 = 2 GiB) */
} cct_server_config;
typedef struct cct_serve_request {
  int32_t struct_size;  /* sizeof(cct_serve_request) */
  int32_t kind;         /* CCT_SERVE_CONV or CCT_SERVE_GRAPH_STEP */
  cct_conv_desc desc;   /* CCT_SERVE_CONV */
  const float *image;   /* host input (the graph's input field for a step) */
  const float *filter;  /* host filter, or NULL for resident filter filter_id */
  int32_t filter_id;
  int32_t reserved;
  float *out;           /* host output (the graph's last field for a step) */
  cct_graph *graph;     /* CCT_SERVE_GRAPH_STEP */
} cct_serve_request;
typedef struct cct_server cct_server;
void cct_server_config_init(cct_server_config *cfg);
void cct_serve_request_init(cct_serve_request *req);
int cct_server_create(const cct_server_config *cfg, cct_server **out);
/* Waits for every submitted request, then stops the scheduler. */
int cct_server_destroy(cct_server *server);
/* A filter bank kept resident on the device; requests name it by id. */
int cct_server_add_filter(cct_server *server, const float *host_filter, size_t elems, int32_t *id);
/* Queues a request (CCT_EINVAL if it can never fit: larger than the cap, or
 * than the device's memory less the reserve; or malformed). */
int cct_server_submit(cct_server *server, const cct_serve_request *req, uint64_t *ticket);
/* CCT_OK once the request's output is in host memory; CCT_ETIMEOUT after
 * timeout_ms (< 0: no limit); the request's own error status otherwise.
 * latency_us (may be NULL): submit to completion, as seen by the scheduler. */
int cct_server_wait(cct_server *server, uint64_t ticket, int32_t timeout_ms, double *latency_us);
/* Open-loop replay: submits req[i] at arrival_s[i] seconds after the call
 * (a client thread), waits for all, and writes each latency in µs.
 * Returns the first error status, or CCT_OK. */
int cct_server_replay(cct_server *server, const cct_serve_request *reqs, const double *arrival_s,
                      int32_t n, double *latency_us);
/* Counters since creation: requests completed, persistent launches, requests
 * that ran on their own plan, peak arena bytes in use. */
int cct_server_stats(const cct_server *server, uint64_t *completed, uint64_t *batches,
                     uint64_t *solo, uint64_t *peak_arena_bytes);
/* Page-locked host memory for request buffers. */
int cct_host_alloc(void **ptr, size_t bytes);
int cct_host_free(void *ptr);

/* ---- device memory helpers (the JNI side has no CUDA runtime) ----------- */
int cct_malloc(void **ptr, size_t bytes);
int cct_free(void *ptr);
int cct_memcpy_h2d(void *dst, const void *src, size_t bytes, void *stream);
int cct_memcpy_d2h(void *dst, const void *src, size_t bytes, void *stream);
int cct_stream_create(void **stream);
int cct_stream_destroy(void *stream);
int cct_stream_synchronize(void *stream);

/* ---- diagnostics --------------------------------------------------------- */
/* Device-side status of this library's kernels on the current device since
 * the last call: CCT_OK, or CCT_ETIMEOUT when a bounded wait inside a kernel
 * gave up (that kernel returned early and its output is undefined).  The
 * reference surfaces device failures as a CLEvent error status
 * (src/main/scala/cogx/platform/opencl/OpenCLDeviceKernel.scala:106-147).
 * Reading clears the status; the call synchronises with the device.  It
 * covers plans, graphs, servers and cct_conv_run_noalloc alike: all of them
 * record into one statically allocated word per device. */
int cct_device_status(void);
/* Failure-detection self-test (no counterpart in the reference): launches a
 * kernel whose mbarrier wait never completes, so the library's bounded wait
 * gives up after about one second, records the timeout and returns.  Returns
 * CCT_OK when the kernel came back on its own (elapsed_ms, may be NULL, is the
 * host-side duration); the following cct_device_status() then reports
 * CCT_ETIMEOUT, and the context stays usable. */
int cct_selftest_wait_timeout(double *elapsed_ms);
const char *cct_last_error_string(void);
int cct_abi_version(void);
/* Kernel launches issued by this process so far (all plans, all threads). */
uint64_t cct_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* CCT_CONV_H */
