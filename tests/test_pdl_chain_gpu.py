"""Kernels of every family queued back to back on one stream, each reading
the previous one's output, with no synchronisation between them.  Every
kernel is launched with programmatic stream serialisation and waits for its
predecessor before touching global memory, so the chained results must equal
the same launches run one at a time with a device synchronisation after each
(bit for bit: every kernel is deterministic)."""
import ctypes

import numpy as np
import pytest
import torch

import cctconv as C
from cctconv import _lib

pytestmark = pytest.mark.gpu


def _chain(sync):
    torch.manual_seed(0)
    P, H, W = 8, 128, 128
    s = torch.cuda.current_stream().cuda_stream
    x = torch.rand((P, H, W), device="cuda")
    f5 = torch.rand((5, 5), device="cuda") - 0.5
    f31 = torch.rand((31, 31), device="cuda") / 961.0
    fk = torch.randn((16 * P, 3, 3), device="cuda") * 0.1  # 16 filters of P planes
    fb = torch.randn((16 * P, 3, 3), device="cuda") * 0.1
    ga = torch.randn((16, H - 4, W - 4), device="cuda")   # FilterAdjoint gradient
    rf = torch.rand(7, device="cuda") - 0.5
    cf = torch.rand(5, device="cuda") - 0.5
    direct = _lib.Plan(C.make_desc((H, W, P), (5, 5, 0), C.BorderZero, _lib.CONVOLUTION,
                                   C.NoSamplingConvolution, _lib.PLANE_BY_PLANE, algo=_lib.ALGO_DIRECT))
    fft = _lib.Plan(C.make_desc((H, W, P), (31, 31, 0), C.BorderCyclic, _lib.CONVOLUTION,
                                C.NoSamplingConvolution, _lib.PLANE_BY_PLANE, algo=_lib.ALGO_FFT))
    fwd = _lib.Plan(C.make_desc((H, W, P), (3, 3, 16 * P), C.BorderZero, _lib.CROSS_CORRELATION,
                                C.NoSamplingConvolution, _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, 1,
                                _lib.PREC_BF16X3))
    bwd = _lib.Plan(C.make_desc((H, W, 16), (3, 3, 16 * P), C.BorderZero, _lib.CONVOLUTION,
                                C.NoSamplingConvolution, _lib.BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM, 1,
                                _lib.PREC_FP32))
    fa = _lib.Plan(C.make_desc((H, W, P), (H - 4, W - 4, 16), C.BorderValid, _lib.CROSS_CORRELATION,
                               C.NoSamplingConvolution, _lib.FILTER_ADJOINT_BLOCK_REDUCE_SUM, 1,
                               _lib.PREC_BF16X3))
    assert fft.algo == _lib.PLAN_FFT and fwd.algo == _lib.PLAN_FRAME_BF16X3
    assert fa.algo == _lib.PLAN_FILTER_ADJOINT_BF16X3
    y1 = torch.empty_like(x)
    y2 = torch.empty_like(x)
    y3 = torch.empty_like(x)
    tmp = torch.empty_like(x)
    y4 = torch.empty((16, H, W), device="cuda")
    y5 = torch.empty_like(x)
    y6 = torch.empty((16 * P, 5, 5), device="cuda")

    def step(fn):
        fn()
        if sync:
            torch.cuda.synchronize()

    for _ in range(3):  # three rounds, so each kernel also follows its own previous launch
        step(lambda: direct.run(x.data_ptr(), f5.data_ptr(), y1.data_ptr(), s))
        step(lambda: fft.run(y1.data_ptr(), f31.data_ptr(), y2.data_ptr(), s))
        step(lambda: _lib.check(_lib.LIB.cct_conv_separable(H, W, P, y2.data_ptr(), rf.data_ptr(), 7,
                                                            cf.data_ptr(), 5, _lib.BORDER_ZERO,
                                                            _lib.CONVOLUTION, tmp.data_ptr(), y3.data_ptr(),
                                                            ctypes.c_void_p(s))))
        step(lambda: fwd.run(y3.data_ptr(), fk.data_ptr(), y4.data_ptr(), s))
        step(lambda: bwd.run(y4.data_ptr(), fb.data_ptr(), y5.data_ptr(), s))
        step(lambda: fa.run(y5.data_ptr(), ga.data_ptr(), y6.data_ptr(), s))
        step(lambda: x.copy_(y5 * 0.5))
    torch.cuda.synchronize()
    assert _lib.LIB.cct_device_status() == _lib.OK
    return [t.cpu().numpy() for t in (y1, y2, y3, y4, y5, y6)]


def test_back_to_back_chain_equals_synchronised_runs():
    chained = _chain(sync=False)
    stepped = _chain(sync=True)
    for i, (a, b) in enumerate(zip(chained, stepped)):
        assert np.isfinite(a).all(), i
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), i
