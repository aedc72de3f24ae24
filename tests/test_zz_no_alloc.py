"""The allocation-free entry point, cct_conv_run_noalloc, against the plan
entry point on the same inputs.

Callers that cannot call cudaMalloc when they convolve (hosts that reserve
all device memory up front in their own arena, or latency-sensitive callers
that avoid cudaMalloc/cudaFree because they may synchronise the device) use
this entry point: it takes device pointers, creates no plan and keeps its only
scratch, the packed filter operand, in a fixed 4 MiB device array.

This file is collected last so that a failure here, in a run that stops at the
first failure, comes after every other test has run.  It must also pass alone
in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
from cctconv import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-5  # normwise, as for the other split-BF16 tensor-core tests


def _desc(H, W, R, planes, fplanes, batch, orient, mode, border=_lib.BORDER_ZERO, down=1):
    return _lib.new_desc(image_rows=H, image_cols=W, image_planes=planes, filter_rows=R,
                         filter_cols=R, filter_planes=fplanes, batch_size=batch, border=border,
                         orientation=orient, sampling=_lib.SAMPLE_DOWN if down > 1 else _lib.SAMPLE_NONE,
                         step=down, vector_mode=mode, precision=_lib.PREC_BF16X3)


def _run_noalloc(desc, x, f, y):
    st = _lib.LIB.cct_conv_run_noalloc(ctypes.byref(desc), ctypes.c_void_p(x.data_ptr()),
                                       ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return st


CASES = [
    # the filter-bank configuration: B=16 C=32 K=64, 64x64, 5x5 (forward and backward)
    (64, 64, 5, 16 * 32, 64 * 32, 16, _lib.CROSS_CORRELATION, _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, 1),
    (64, 64, 5, 16 * 64, 64 * 32, 16, _lib.CONVOLUTION, _lib.BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM, 1),
    # a down-sampled layer with a partial filter block
    (32, 32, 3, 2 * 40, 130 * 40, 2, _lib.CROSS_CORRELATION, _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, 2),
]


@pytest.mark.parametrize("H,W,R,planes,fplanes,batch,orient,mode,down", CASES)
def test_noalloc_matches_plan_entry_point(H, W, R, planes, fplanes, batch, orient, mode, down):
    desc = _desc(H, W, R, planes, fplanes, batch, orient, mode, down=down)
    gen = torch.Generator(device="cuda").manual_seed(H * 7 + planes)
    x = torch.randn((planes, H, W), device="cuda", generator=gen)
    f = torch.randn((fplanes, R, R), device="cuda", generator=gen)

    plan = _lib.Plan(desc)
    assert plan.algo == _lib.PLAN_FRAME_BF16X3
    orows, ocols, oplanes = plan.shape
    ref = torch.empty((oplanes, orows, ocols), device="cuda")
    plan.run(x.data_ptr(), f.data_ptr(), ref.data_ptr(), torch.cuda.current_stream().cuda_stream)
    plan.close()

    outs = []
    for _ in range(2):  # two calls in a row share the scratch array
        y = torch.full((oplanes, orows, ocols), float("nan"), device="cuda")
        assert _run_noalloc(desc, x, f, y) == _lib.OK, _lib.LIB.cct_last_error_string()
        outs.append(y)
    torch.cuda.synchronize()
    r = ref.double()
    for y in outs:
        assert not torch.isnan(y).any()
        err = (y.double() - r).abs().max().item() / r.abs().max().item()
        assert err <= TOL, err
        assert torch.equal(y, ref)  # the same kernel and tile plan as the plan entry point


def test_noalloc_rejects_filter_banks_beyond_the_limit():
    # 512 filters x 512 planes x 3x3: the packed operand is far above 4 MiB
    desc = _desc(28, 28, 3, 512, 512 * 512, 1, _lib.CROSS_CORRELATION,
                 _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM)
    x = torch.zeros((512, 28, 28), device="cuda")
    f = torch.zeros((512 * 512, 3, 3), device="cuda")
    y = torch.zeros((512, 28, 28), device="cuda")
    assert _run_noalloc(desc, x, f, y) == _lib.EINVAL
    assert b"at most" in _lib.LIB.cct_last_error_string()


def test_noalloc_only_takes_the_tensor_core_frame_kernel():
    # DownsampleOutput(3) is outside the tensor-core frame kernels
    desc = _desc(18, 18, 3, 4, 8, 1, _lib.CROSS_CORRELATION, _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM,
                 down=3)
    x = torch.zeros((4, 18, 18), device="cuda")
    f = torch.zeros((8, 3, 3), device="cuda")
    y = torch.zeros((2, 6, 6), device="cuda")
    assert _run_noalloc(desc, x, f, y) == _lib.ENOTSUP


def test_noalloc_result_matches_fp64_oracle():
    """Independent of the plan path: the filter-bank forward against FP64."""
    rng = np.random.default_rng(3)
    B, C, K, H, W, R = 2, 16, 32, 24, 24, 3
    x = rng.standard_normal((B * C, H, W)).astype(np.float32)
    f = rng.standard_normal((K * C, R, R)).astype(np.float32)
    desc = _desc(H, W, R, B * C, K * C, B, _lib.CROSS_CORRELATION, _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM)
    xd, fd = torch.from_numpy(x).cuda(), torch.from_numpy(f).cuda()
    y = torch.empty((B * K, H, W), device="cuda")
    assert _run_noalloc(desc, xd, fd, y) == _lib.OK
    torch.cuda.synchronize()
    od = O.make_desc(H, W, R, R, planes=B * C, f_planes=K * C, batch=B, border=O.ZERO,
                     orient=O.XCORR, mode=O.PROJECT_REDUCE)
    assert O.rel_errors(y.cpu().numpy(), O.conv(od, x, f, np.float64))[0] <= TOL


def _filter_bank_case():
    B, C, K, H, W, R = 2, 16, 32, 24, 24, 3
    desc = _desc(H, W, R, B * C, K * C, B, _lib.CROSS_CORRELATION, _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM)
    gen = torch.Generator(device="cuda").manual_seed(11)
    x = torch.randn((B * C, H, W), device="cuda", generator=gen)
    f = torch.randn((K * C, R, R), device="cuda", generator=gen)
    return desc, x, f, (B * K, H, W)


def test_noalloc_timeouts_are_reported_by_device_status():
    """A bounded wait that gives up is recorded in the library's one device
    error word, which this entry point's kernel shares with every plan; a
    call does not clear it, and cct_device_status() reports and clears it."""
    desc, x, f, oshape = _filter_bank_case()
    y = torch.empty(oshape, device="cuda")
    assert _run_noalloc(desc, x, f, y) == _lib.OK
    torch.cuda.synchronize()
    assert _lib.LIB.cct_device_status() == _lib.OK  # a clean run records nothing
    # record a timeout in the word (a wait on a barrier nobody arrives on,
    # which gives up after about a second and returns: no fault)
    assert _lib.LIB.cct_selftest_wait_timeout(None) == _lib.OK
    y2 = torch.empty(oshape, device="cuda")
    assert _run_noalloc(desc, x, f, y2) == _lib.OK
    torch.cuda.synchronize()
    assert _lib.LIB.cct_device_status() == _lib.ETIMEOUT  # still recorded after the call
    assert _lib.LIB.cct_device_status() == _lib.OK  # reading cleared it
    assert torch.equal(y, y2)  # and the context still computes the same result


def test_noalloc_allocates_no_device_memory():
    """Free device memory is the same before and after 100 calls (after the
    first, which loads the kernels and looks up the scratch address)."""
    desc, x, f, oshape = _filter_bank_case()
    y = torch.empty(oshape, device="cuda")
    assert _run_noalloc(desc, x, f, y) == _lib.OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(100):
        assert _run_noalloc(desc, x, f, y) == _lib.OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert _lib.LIB.cct_device_status() == _lib.OK
