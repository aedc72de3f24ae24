"""Host-side mirror of cct-core's convolution operators over libcctconv.

Names, argument meaning and error behaviour follow the reference's
``CogFunctionAPI`` (src/main/scala/cogx/api/CogFunctionAPI.scala):

  crossCorrelate(field, filter, borderPolicy, samplingPolicy)          :1245
  convolve(field, filter, borderPolicy, samplingPolicy)                :1264
  convolveSeparable / crossCorrelateSeparable(field, row, col, border) :1277-1366
  projectFrame(field, filter, borderPolicy, samplingPolicy, batchSize) :1370
  projectFrameBlockReduceSum(...)                                      :1395
  backProjectFrame(...)                                                :1425
  backProjectFrameBlockReduceSum(...)                                  :1450

Fields are CUDA float32 tensors in cct-core's planar layout: ``(cols,)`` is a
1-D ScalarField, ``(rows, cols)`` a 2-D ScalarField, ``(planes, rows,
cols)`` a 2-D VectorField (tensor planes first, each plane row-major) and
``(size, size, rows, cols)`` a 2-D MatrixField of size x size matrices (tensor
elements first).  A ColorField is a CUDA uint8 tensor ``(rows, cols, 4)``:
RGBA bytes per pixel, the reference's UNORM_INT8 image.

convolve / crossCorrelate also take the two special operand pairs of
CogFunctionAPI.convolveInternal (:1128-1238): a ScalarField with a MatrixField
filter (ScalarMatrixConvolve2D, :1209-1216) and a ColorField image
(DynamicConvolutionGenerator.scala:89-106).
torch only supplies device memory and the current stream; every convolution
runs in libcctconv's CUDA kernels.  Illegal arguments raise ``ValueError``
with the reference's message (the reference throws from ``require``).
"""
import ctypes
import threading

import torch

from . import _lib
from ._lib import CctError, Plan, launch_count  # noqa: F401

__all__ = [
    "BorderZero", "BorderClamp", "BorderCyclic", "BorderValid", "BorderFull",
    "NoSamplingConvolution", "UpsampleInputConvolution", "DownsampleOutputConvolution",
    "UseFFTNever", "UseFFTAlways", "UseFFTWhenBest",
    "convolve", "crossCorrelate", "convolveSeparable", "crossCorrelateSeparable",
    "projectFrame", "projectFrameBlockReduceSum", "backProjectFrame",
    "backProjectFrameBlockReduceSum", "crossCorrelateFilterAdjoint", "convolveFilterAdjoint",
    "filterAdjointBlockReduceSum", "make_desc", "plan_for", "CctError", "Plan",
]


class _Policy:
    def __init__(self, name, code):
        self.name, self.code = name, code

    def __repr__(self):
        return self.name


BorderZero = _Policy("BorderZero", _lib.BORDER_ZERO)
BorderClamp = _Policy("BorderClamp", _lib.BORDER_CLAMP)
BorderCyclic = _Policy("BorderCyclic", _lib.BORDER_CYCLIC)
BorderValid = _Policy("BorderValid", _lib.BORDER_VALID)
BorderFull = _Policy("BorderFull", _lib.BORDER_FULL)
UseFFTNever = _Policy("UseFFTNever", _lib.ALGO_DIRECT)
UseFFTAlways = _Policy("UseFFTAlways", _lib.ALGO_FFT)
UseFFTWhenBest = _Policy("UseFFTWhenBest", _lib.ALGO_AUTO)


class _Sampling:
    def __init__(self, name, code, step):
        self.name, self.code, self.step = name, code, step

    def __repr__(self):
        return f"{self.name}({self.step})" if self.code else self.name


NoSamplingConvolution = _Sampling("NoSamplingConvolution", _lib.SAMPLE_NONE, 1)


def UpsampleInputConvolution(step):
    return _Sampling("UpsampleInputConvolution", _lib.SAMPLE_UP, int(step))


def DownsampleOutputConvolution(step):
    return _Sampling("DownsampleOutputConvolution", _lib.SAMPLE_DOWN, int(step))


_PLANS = {}
_PLANS_LOCK = threading.Lock()


def _shape_of(t, what):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{what} must be a torch.Tensor")
    if t.dtype != torch.float32:
        raise TypeError(f"{what} must be float32")
    if t.dim() == 1:
        return 1, t.shape[0], 0
    if t.dim() == 2:
        return t.shape[0], t.shape[1], 0
    if t.dim() == 3:
        return t.shape[1], t.shape[2], t.shape[0]
    raise ValueError(f"{what}: only 1-D and 2-D scalar or vector fields are supported")


def make_desc(field_shape, filter_shape, border, orientation, sampling, mode, batch=1,
              precision=_lib.PREC_FP32, algo=_lib.ALGO_AUTO, flags=0):
    """field_shape / filter_shape: (rows, cols, planes) with planes 0 = ScalarField."""
    rows, cols, planes = field_shape
    frows, fcols, fplanes = filter_shape
    return _lib.new_desc(image_rows=rows, image_cols=cols, image_planes=planes,
                         filter_rows=frows, filter_cols=fcols, filter_planes=fplanes,
                         batch_size=batch, border=border.code, orientation=orientation,
                         sampling=sampling.code, step=sampling.step, vector_mode=mode,
                         precision=precision, algo=algo, flags=flags)


def plan_for(desc, device=None):
    """Cached plan for a descriptor on the current CUDA device."""
    dev = torch.cuda.current_device() if device is None else device
    key = (dev, desc.key())
    with _PLANS_LOCK:
        p = _PLANS.get(key)
        if p is None:
            with torch.cuda.device(dev):
                p = Plan(desc)
            _PLANS[key] = p
    return p


def _out_tensor(shape, planes, like, squeeze_scalar, one_d):
    orows, ocols, _ = shape
    if one_d:
        return torch.empty((ocols,) if planes == 1 and squeeze_scalar else (planes, ocols),
                           device=like.device, dtype=torch.float32)
    if planes == 1 and squeeze_scalar:
        return torch.empty((orows, ocols), device=like.device, dtype=torch.float32)
    return torch.empty((planes, orows, ocols), device=like.device, dtype=torch.float32)


def _run(field, filt, border, orientation, sampling, mode, batch, precision=_lib.PREC_FP32,
         algo=_lib.ALGO_AUTO, relu=False):
    if not field.is_cuda or not filt.is_cuda:
        raise ValueError("fields must live on a CUDA device")
    fs, ks = _shape_of(field, "field"), _shape_of(filt, "filter")
    if (field.dim() == 1) != (filt.dim() == 1):
        raise ValueError("field and filter must have the same dimensionality")
    desc = make_desc(fs, ks, border, orientation, sampling, mode, batch, precision, algo,
                     _lib.FLAG_RELU if relu else 0)
    try:
        shape = _lib.output_shape(desc)
    except CctError as e:
        raise ValueError(str(e)) from None
    plan = plan_for(desc, field.device.index)
    x = field.contiguous()
    f = filt.contiguous()
    planes = shape[2]
    # ScalarField result when both inputs are scalar (plane-by-plane), and the
    # length-1 BlockReduceSum result is sliced to a ScalarField
    # (CogFunctionAPI.scala:1406-1409, 1461-1464).
    # ...and a FilterAdjoint result of one plane is a ScalarField
    # (ConvolveHyperKernel.scala:1414-1429).
    squeeze = (fs[2] == 0 and ks[2] == 0) or (
        mode in (_lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, _lib.BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM,
                 _lib.FILTER_ADJOINT, _lib.FILTER_ADJOINT_BLOCK_REDUCE_SUM)
        and planes == 1)
    y = _out_tensor(shape, planes, field, squeeze, field.dim() == 1)
    stream = torch.cuda.current_stream(field.device).cuda_stream
    plan.run(x.data_ptr(), f.data_ptr(), y.data_ptr(), stream)
    return y


def _is_color_field(t):
    return isinstance(t, torch.Tensor) and t.dtype == torch.uint8 and t.dim() == 3 and t.shape[2] == 4


def _is_matrix_field(t):
    return isinstance(t, torch.Tensor) and t.dim() == 4


def _scalar_matrix(field, matrices, border, orientation, sampling):
    """ScalarField (*) MatrixField -> VectorField of one plane per matrix,
    plane index row * matrix_cols + col (ScalarMatrixConvolve2DHyperKernel)."""
    if not field.is_cuda or not matrices.is_cuda:
        raise ValueError("fields must live on a CUDA device")
    if matrices.dtype != torch.float32:
        raise TypeError("filter must be float32")
    if field.dim() != 2:
        raise ValueError("a MatrixField filter needs a 2-D ScalarField input")
    rows, cols, _ = _shape_of(field, "field")
    size, size2, mrows, mcols = matrices.shape
    if size != size2:
        raise ValueError("matrix in field must be square")
    x, m = field.contiguous(), matrices.contiguous()
    y = torch.empty((mrows * mcols, rows, cols), device=field.device, dtype=torch.float32)
    st = _lib.LIB.cct_conv_scalar_matrix(rows, cols, x.data_ptr(), m.data_ptr(), mrows, mcols, size,
                                         border.code, orientation, sampling.code, sampling.step,
                                         y.data_ptr(),
                                         ctypes.c_void_p(torch.cuda.current_stream(field.device).cuda_stream))
    if st == _lib.EINVAL:
        raise ValueError(_lib.LIB.cct_last_error_string().decode())
    _lib.check(st)
    return y


_COLOR_PLANS = {}


def _color(field, filt, border, orientation, sampling, algo):
    """ColorField convolution: red, green, blue each convolved with the
    scalar filter, merged back into a ColorField of the output shape."""
    if not field.is_cuda or not filt.is_cuda:
        raise ValueError("fields must live on a CUDA device")
    rows, cols = field.shape[0], field.shape[1]
    frows, fcols, fplanes = _shape_of(filt, "filter")
    if fplanes != 0 or filt.dim() != 2:
        raise ValueError("a ColorField is convolved with a 2-D ScalarField filter")
    desc = make_desc((rows, cols, 0), (frows, fcols, 0), border, orientation, sampling,
                     _lib.PLANE_BY_PLANE, algo=algo)
    try:
        orows, ocols, _ = _lib.output_shape(desc)
    except CctError as e:
        raise ValueError(str(e)) from None
    dev = field.device.index
    key = (dev, desc.key())
    with _PLANS_LOCK:
        plan = _COLOR_PLANS.get(key)
        if plan is None:
            with torch.cuda.device(dev):
                plan = _lib.ColorPlan(desc)
            _COLOR_PLANS[key] = plan
    x, f = field.contiguous(), filt.contiguous()
    y = torch.empty((orows, ocols, 4), device=field.device, dtype=torch.uint8)
    plan.run(x.data_ptr(), f.data_ptr(), y.data_ptr(), torch.cuda.current_stream(field.device).cuda_stream)
    return y


def crossCorrelate(field, filter, borderPolicy, samplingPolicy=NoSamplingConvolution,
                   fftUse=UseFFTWhenBest):
    if _is_color_field(field):
        return _color(field, filter, borderPolicy, _lib.CROSS_CORRELATION, samplingPolicy, fftUse.code)
    if _is_matrix_field(filter):
        return _scalar_matrix(field, filter, borderPolicy, _lib.CROSS_CORRELATION, samplingPolicy)
    return _run(field, filter, borderPolicy, _lib.CROSS_CORRELATION, samplingPolicy,
                _lib.PLANE_BY_PLANE, 1, algo=fftUse.code)


def convolve(field, filter, borderPolicy, samplingPolicy=NoSamplingConvolution,
             fftUse=UseFFTWhenBest):
    if _is_color_field(field):
        return _color(field, filter, borderPolicy, _lib.CONVOLUTION, samplingPolicy, fftUse.code)
    if _is_matrix_field(filter):
        return _scalar_matrix(field, filter, borderPolicy, _lib.CONVOLUTION, samplingPolicy)
    return _run(field, filter, borderPolicy, _lib.CONVOLUTION, samplingPolicy,
                _lib.PLANE_BY_PLANE, 1, algo=fftUse.code)


def projectFrame(field, filter, borderPolicy, samplingPolicy=NoSamplingConvolution, batchSize=1):
    return _run(field, filter, borderPolicy, _lib.CROSS_CORRELATION, samplingPolicy,
                _lib.PROJECT_FRAME, batchSize)


def projectFrameBlockReduceSum(field, filter, borderPolicy, samplingPolicy=NoSamplingConvolution,
                               batchSize=1, precision=_lib.PREC_FP32, relu=False):
    return _run(field, filter, borderPolicy, _lib.CROSS_CORRELATION, samplingPolicy,
                _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, batchSize, precision, relu=relu)


def backProjectFrame(field, filter, borderPolicy, samplingPolicy=NoSamplingConvolution, batchSize=1):
    return _run(field, filter, borderPolicy, _lib.CONVOLUTION, samplingPolicy,
                _lib.BACK_PROJECT_FRAME, batchSize)


def backProjectFrameBlockReduceSum(field, filter, borderPolicy,
                                   samplingPolicy=NoSamplingConvolution, batchSize=1,
                                   precision=_lib.PREC_FP32, relu=False):
    return _run(field, filter, borderPolicy, _lib.CONVOLUTION, samplingPolicy,
                _lib.BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM, batchSize, precision, relu=relu)


def crossCorrelateFilterAdjoint(field, filter, borderPolicy, samplingPolicy=NoSamplingConvolution,
                                batchSize=1):
    """Weight-gradient plane mixing (CogFunctionAPI.scala:1480-1487): `filter`
    is the gradient field of batchSize*L planes; output plane B*w + b,
    w = l*C + c, correlates image plane b*C + c with gradient plane b*L + l.
    UpsampleInput upsamples the gradient."""
    return _run(field, filter, borderPolicy, _lib.CROSS_CORRELATION, samplingPolicy,
                _lib.FILTER_ADJOINT, batchSize)


def convolveFilterAdjoint(field, filter, borderPolicy, samplingPolicy=NoSamplingConvolution,
                          batchSize=1):
    """As crossCorrelateFilterAdjoint with the (upsampled) gradient flipped
    (CogFunctionAPI.scala:1503-1510)."""
    return _run(field, filter, borderPolicy, _lib.CONVOLUTION, samplingPolicy,
                _lib.FILTER_ADJOINT, batchSize)


def filterAdjointBlockReduceSum(field, filter, borderPolicy, samplingPolicy=NoSamplingConvolution,
                                batchSize=1, orientation=_lib.CROSS_CORRELATION, precision=_lib.PREC_FP32):
    """blockReduceSum(crossCorrelateFilterAdjoint(...), batchSize) fused, the
    form the reference's optimizer emits (FilterAdjointBlockReduceSum): plane
    w sums the batchSize images' planes in order.  precision PREC_BF16X3 runs
    it on the tensor cores (split BF16, within 1e-5 of FP64)."""
    return _run(field, filter, borderPolicy, orientation, samplingPolicy,
                _lib.FILTER_ADJOINT_BLOCK_REDUCE_SUM, batchSize, precision)


def _separable(field, rowFilter, columnFilter, borderPolicy, orientation):
    if field.dim() not in (2, 3):
        raise ValueError("field must be 2D")
    if rowFilter.dim() != 1 or columnFilter.dim() != 1:
        raise ValueError("row and column filters must be 1D")
    rows, cols, planes = _shape_of(field, "field")
    x = field.contiguous()
    y = torch.empty_like(x)
    tmp = torch.empty_like(x)
    rf, cf = rowFilter.contiguous(), columnFilter.contiguous()
    stream = torch.cuda.current_stream(field.device).cuda_stream
    st = _lib.LIB.cct_conv_separable(rows, cols, max(planes, 1), x.data_ptr(), rf.data_ptr(),
                                     rf.numel(), cf.data_ptr(), cf.numel(), borderPolicy.code,
                                     orientation, tmp.data_ptr(), y.data_ptr(),
                                     ctypes.c_void_p(stream))
    if st == _lib.EINVAL:
        raise ValueError(_lib.LIB.cct_last_error_string().decode())
    _lib.check(st)
    return y


def convolveSeparable(field, rowFilter, columnFilter, borderPolicy):
    return _separable(field, rowFilter, columnFilter, borderPolicy, _lib.CONVOLUTION)


def crossCorrelateSeparable(field, rowFilter, columnFilter, borderPolicy):
    return _separable(field, rowFilter, columnFilter, borderPolicy, _lib.CROSS_CORRELATION)
