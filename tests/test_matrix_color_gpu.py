"""ScalarField (*) MatrixField and ColorField convolution on the GPU, through
the C-ABI (via the cctconv mirror), against the oracle.

ScalarMatrixConvolve2D is FP32 fma chains in the reference's order, so it
must match the oracle bit for bit.  Colour convolution is byte in, byte out:
bit-exact on every direct path; through the FFT path (1e-5 normwise in the
planes) a channel may differ by one step where a value sits on a rounding
boundary.
"""
import numpy as np
import pytest
import torch

import oracle as O
from helpers import bitwise_equal

pytestmark = pytest.mark.gpu

C = None


def setup_module():
    global C
    import cctconv
    C = cctconv


def _pol(border):
    return {O.ZERO: C.BorderZero, O.CLAMP: C.BorderClamp, O.CYCLIC: C.BorderCyclic,
            O.VALID: C.BorderValid, O.FULL: C.BorderFull}[border]


@pytest.mark.parametrize("size", [1, 3, 5, 7, 9, 11, 13, 21])
@pytest.mark.parametrize("shape,mgrid", [((4, 5), (2, 3)), ((45, 70), (1, 1)), ((97, 130), (3, 4)),
                                         ((256, 256), (8, 4))])
def test_scalar_matrix_bitwise(size, shape, mgrid):
    rng = np.random.default_rng(size * 1000 + shape[0])
    x = rng.uniform(-1, 1, shape).astype(np.float32)
    mats = rng.uniform(-1, 1, (size, size) + mgrid).astype(np.float32)
    xd, md = torch.from_numpy(x).cuda(), torch.from_numpy(mats).cuda()
    for border in (O.ZERO, O.CLAMP, O.CYCLIC):
        y = C.crossCorrelate(xd, md, _pol(border))
        torch.cuda.synchronize()
        assert y.shape == (mgrid[0] * mgrid[1],) + shape
        assert bitwise_equal(y.cpu().numpy(), O.scalar_matrix(x, mats, border)), (size, shape, border)


def test_scalar_matrix_reference_test_case():
    """StaticConvolutionSpec.scala:2361-2393 on the GPU: 4x5 field, 2x3 matrix
    field of 3x3 matrices, BorderClamp, against convolve of the flipped
    matrices (the reference's ~==)."""
    from helpers import ref_field_approx_equal
    rng = np.random.default_rng(5)
    x = rng.random((4, 5)).astype(np.float32)
    mats = rng.random((3, 3, 2, 3)).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    y = C.crossCorrelate(xd, torch.from_numpy(mats).cuda(), C.BorderClamp).cpu().numpy()
    expected = np.stack([C.convolve(xd, torch.from_numpy(np.ascontiguousarray(mats[::-1, ::-1, r, c])).cuda(),
                                    C.BorderClamp).cpu().numpy() for r in range(2) for c in range(3)])
    assert ref_field_approx_equal(y, expected)


def test_scalar_matrix_errors_through_the_api():
    x = torch.zeros((8, 8), device="cuda")
    m = torch.zeros((3, 3, 2, 2), device="cuda")
    with pytest.raises(ValueError, match="convolution not supported yet"):
        C.convolve(x, m, C.BorderZero)
    with pytest.raises(ValueError, match="unsupported: BorderValid"):
        C.crossCorrelate(x, m, C.BorderValid)
    with pytest.raises(ValueError, match="sampling not supported yet"):
        C.crossCorrelate(x, m, C.BorderZero, C.DownsampleOutputConvolution(2))
    # step-1 sampling is NoSampling (CogFunctionAPI.scala:1139-1143)
    C.crossCorrelate(x, m, C.BorderZero, C.DownsampleOutputConvolution(1))
    with pytest.raises(ValueError, match="square"):
        C.crossCorrelate(x, torch.zeros((3, 5, 2, 2), device="cuda"), C.BorderZero)


def _color_case(rows, cols, fr, fc, border, orient, sampling=O.NOSAMPLE, step=1, seed=0):
    rng = np.random.default_rng(seed)
    rgba = rng.integers(0, 256, (rows, cols, 4), dtype=np.uint8)
    f = rng.uniform(-1, 1, (fr, fc)).astype(np.float32)
    f /= np.abs(f).sum() * 0.9  # keep most results inside [0, 1] so the rounding is exercised
    return rgba, f, O.make_desc(rows, cols, fr, fc, border=border, orient=orient, sampling=sampling, step=step)


def _samp(sampling, step):
    if sampling == O.DOWN:
        return C.DownsampleOutputConvolution(step)
    if sampling == O.UP:
        return C.UpsampleInputConvolution(step)
    return C.NoSamplingConvolution


@pytest.mark.parametrize("border", [O.ZERO, O.CLAMP, O.CYCLIC, O.VALID, O.FULL])
@pytest.mark.parametrize("orient", [O.CONV, O.XCORR])
@pytest.mark.parametrize("sampling,step", [(O.NOSAMPLE, 1), (O.DOWN, 2), (O.UP, 2)])
def test_color_direct_bitwise(border, orient, sampling, step):
    rows, cols = (48, 64)
    if sampling == O.DOWN and border == O.VALID:
        rows, cols = 50, 66  # (size - 2) divisible by 2 for a 3x3 filter
    if sampling == O.DOWN and border == O.FULL:
        rows, cols = 46, 62
    rgba, f, d = _color_case(rows, cols, 3, 5 if border in (O.VALID, O.FULL) else 3, border, orient,
                             sampling, step, seed=border * 10 + orient)
    fn = C.convolve if orient == O.CONV else C.crossCorrelate
    if sampling == O.UP and border == O.CLAMP:
        with pytest.raises(ValueError, match="BorderClamp"):
            fn(torch.from_numpy(rgba).cuda(), torch.from_numpy(f).cuda(), _pol(border), _samp(sampling, step),
               C.UseFFTNever)
        return
    y = fn(torch.from_numpy(rgba).cuda(), torch.from_numpy(f).cuda(), _pol(border), _samp(sampling, step),
           C.UseFFTNever)
    torch.cuda.synchronize()
    want = O.color_conv(d, rgba, f)
    assert y.dtype == torch.uint8 and tuple(y.shape) == want.shape
    assert np.array_equal(y.cpu().numpy(), want)


@pytest.mark.parametrize("border", [O.ZERO, O.CLAMP, O.CYCLIC])
def test_color_fft_path(border):
    rgba, f, d = _color_case(128, 96, 31, 31, border, O.CONV, seed=7)
    y = C.convolve(torch.from_numpy(rgba).cuda(), torch.from_numpy(f).cuda(), _pol(border),
                   C.NoSamplingConvolution, C.UseFFTAlways).cpu().numpy()
    want = O.color_conv(d, rgba, f)
    diff = np.abs(y.astype(int) - want.astype(int))
    assert diff.max() <= 1
    assert (diff > 0).mean() < 1e-3
    assert np.all(y[..., 3] == 255)


def test_color_errors():
    img = torch.zeros((8, 8, 4), dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError, match="2-D ScalarField filter"):
        C.convolve(img, torch.zeros((2, 3, 3), device="cuda"), C.BorderZero)
