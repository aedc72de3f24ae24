"""Maximum sizes: fields of more than 2^31 elements (over 8 GiB per operand),
so that every 32-bit element index would overflow.  The planes repeat a few
seeded base planes, so the first, middle and last planes (and images) can be
checked bit for bit against the oracle on one plane or image each."""
import gc

import numpy as np
import pytest
import torch

import oracle as O
from cctconv import _lib
from helpers import bitwise_equal

pytestmark = pytest.mark.gpu

BIG = 2 ** 31


def _free():
    gc.collect()
    torch.cuda.empty_cache()


def _repeat_planes(base, planes):
    """(planes, H, W) CUDA tensor whose plane p is base[p % len(base)]."""
    n = base.shape[0]
    x = torch.empty((planes,) + base.shape[1:], device="cuda")
    bd = torch.from_numpy(base).cuda()
    for i in range(n):
        x[i::n] = bd[i]
    return x


def _desc(od, precision=_lib.PREC_FP32):
    return _lib.new_desc(image_rows=od.rows, image_cols=od.cols, image_planes=od.planes,
                         filter_rows=od.f_rows, filter_cols=od.f_cols, filter_planes=od.f_planes,
                         batch_size=od.batch, border=od.border, orientation=od.orient,
                         sampling=od.sampling, step=od.step, vector_mode=od.mode, precision=precision)


def test_plain_convolve_over_2g_elements():
    H = W = 256
    P = BIG // (H * W) + 3  # 32771 planes: 8.6 GB in, 8.6 GB out
    rng = np.random.default_rng(41)
    base = rng.uniform(-1, 1, (5, H, W)).astype(np.float32)
    f = rng.uniform(-1, 1, (5, 5)).astype(np.float32)
    x = _repeat_planes(base, P)
    y = torch.empty_like(x)
    od = O.make_desc(H, W, 5, 5, planes=P, border=O.ZERO, orient=O.CONV)
    plan = _lib.Plan(_desc(od))
    fd = torch.from_numpy(f).cuda()
    plan.run(x.data_ptr(), fd.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert _lib.LIB.cct_device_status() == _lib.OK
    one = O.make_desc(H, W, 5, 5, border=O.ZERO, orient=O.CONV)
    for p in (0, 1, P // 2, P - 2, P - 1):
        assert bitwise_equal(y[p].cpu().numpy(), O.conv(one, base[p % 5], f)[0]), p
    plan.close()
    del x, y
    _free()


def test_separable_over_2g_elements():
    import cctconv as C
    H = W = 256
    P = BIG // (H * W) + 3
    rng = np.random.default_rng(42)
    base = rng.uniform(-1, 1, (3, H, W)).astype(np.float32)
    row = rng.uniform(-1, 1, 5).astype(np.float32)
    col = rng.uniform(-1, 1, 7).astype(np.float32)
    x = _repeat_planes(base, P)
    y = C.convolveSeparable(x, torch.from_numpy(row).cuda(), torch.from_numpy(col).cuda(), C.BorderZero)
    torch.cuda.synchronize()
    for p in (0, P // 2, P - 1):
        assert bitwise_equal(y[p].cpu().numpy(), O.separable(base[p % 3], row, col, O.ZERO, O.CONV)), p
    del x, y
    _free()


@pytest.mark.parametrize("precision", [_lib.PREC_FP32, _lib.PREC_BF16X3])
def test_frame_block_reduce_over_2g_elements(precision):
    """projectFrameBlockReduceSum with 16400 images of 32 planes of 64x64
    (2.15e9 input elements, 4.3e9 output elements): images repeat 3 base
    images, the first and last checked against the oracle."""
    Cin, K, H, W, R = 32, 64, 64, 64, 5
    Bn = BIG // (Cin * H * W) + 16  # 16400 images
    rng = np.random.default_rng(43)
    base = rng.standard_normal((3 * Cin, H, W)).astype(np.float32)
    f = (rng.standard_normal((K * Cin, R, R)) * 0.1).astype(np.float32)
    x = torch.empty((Bn * Cin, H, W), device="cuda")
    bd = torch.from_numpy(base).cuda()
    xv = x.view(Bn, Cin, H, W)
    for i in range(3):
        xv[i::3] = bd[i * Cin:(i + 1) * Cin]
    y = torch.empty((Bn * K, H, W), device="cuda")
    od = O.make_desc(H, W, R, R, planes=Bn * Cin, f_planes=K * Cin, batch=Bn, border=O.ZERO,
                     orient=O.XCORR, mode=O.PROJECT_REDUCE)
    plan = _lib.Plan(_desc(od, precision))
    assert plan.algo == (_lib.PLAN_FRAME_BF16X3 if precision == _lib.PREC_BF16X3 else _lib.PLAN_FRAME_F32)
    fd = torch.from_numpy(f).cuda()
    plan.run(x.data_ptr(), fd.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert _lib.LIB.cct_device_status() == _lib.OK
    one = O.make_desc(H, W, R, R, planes=Cin, f_planes=K * Cin, batch=1, border=O.ZERO,
                      orient=O.XCORR, mode=O.PROJECT_REDUCE)
    for b in (0, Bn - 1):
        got = y[b * K:(b + 1) * K].cpu().numpy()
        img = base[(b % 3) * Cin:(b % 3 + 1) * Cin]
        if precision == _lib.PREC_FP32:
            assert bitwise_equal(got, O.conv(one, img, f)), b
        else:
            err = O.rel_errors(got, O.conv(one, img, f, np.float64))[0]
            assert err <= 1e-5, (b, err)
    plan.close()
    del x, y, xv
    _free()
