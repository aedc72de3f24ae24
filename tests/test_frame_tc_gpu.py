"""Tensor-core (split-BF16, FP32 accumulate) frame kernels against the FP64
oracle.  Tolerance: normwise relative error max|y - ref| / max|ref| <= 1e-5,
the rel-err bound the path is specified to; RMS error is reported too."""
import numpy as np
import pytest
import torch

import oracle as O
from cctconv import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _desc(od, precision=_lib.PREC_BF16X3, flags=0):
    return _lib.new_desc(image_rows=od.rows, image_cols=od.cols, image_planes=od.planes,
                         filter_rows=od.f_rows, filter_cols=od.f_cols, filter_planes=od.f_planes,
                         batch_size=od.batch, border=od.border, orientation=od.orient,
                         sampling=od.sampling, step=od.step, vector_mode=od.mode,
                         precision=precision, flags=flags)


def run_tc(od, x, f, flags=0, expect_tc=True, precision=_lib.PREC_BF16X3):
    plan = _lib.Plan(_desc(od, precision=precision, flags=flags))
    if expect_tc:
        assert plan.algo == _lib.PLAN_FRAME_BF16X3
    orows, ocols, oplanes = plan.shape
    xd = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    fd = torch.from_numpy(np.ascontiguousarray(f, np.float32)).cuda()
    yd = torch.full((oplanes, orows, ocols), float("nan"), device="cuda")
    plan.run(xd.data_ptr(), fd.data_ptr(), yd.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert _lib.LIB.cct_device_status() == _lib.OK
    plan.close()
    return yd.cpu().numpy()


def check(y, od, x, f, relu=False, tol=TOL):
    ref = O.conv(od, x, f, np.float64)
    if relu:
        ref = np.maximum(ref, 0)
    assert not np.isnan(y).any()
    mx, rms = O.rel_errors(y, ref)
    assert mx <= tol, (mx, rms)
    return mx, rms


def _cfg2():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((16 * 32, 64, 64)).astype(np.float32)
    f = (rng.standard_normal((64 * 32, 5, 5)) * np.sqrt(2.0 / 800)).astype(np.float32)
    g = rng.standard_normal((16 * 64, 64, 64)).astype(np.float32)
    return x, f, g


def test_config2_project_frame_bf16x3():
    x, f, _ = _cfg2()
    od = O.make_desc(64, 64, 5, 5, planes=512, f_planes=2048, batch=16, border=O.ZERO,
                     orient=O.XCORR, mode=O.PROJECT_REDUCE)
    mx, rms = check(run_tc(od, x, f), od, x, f)
    print(f"projectFrame bf16x3: normwise max {mx:.3e} rms {rms:.3e}")


def test_config2_back_project_frame_bf16x3():
    _, f, g = _cfg2()
    od = O.make_desc(64, 64, 5, 5, planes=1024, f_planes=2048, batch=16, border=O.ZERO,
                     orient=O.CONV, mode=O.BACKPROJECT_REDUCE)
    mx, rms = check(run_tc(od, g, f), od, g, f)
    print(f"backProjectFrame bf16x3: normwise max {mx:.3e} rms {rms:.3e}")


TC_CASES = [
    # (H, W, C, K, B, R, border, sampling, step, mode)
    (16, 16, 16, 16, 1, 3, O.ZERO, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (20, 36, 3, 24, 2, 3, O.ZERO, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (28, 28, 64, 48, 2, 3, O.ZERO, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (32, 32, 40, 130, 1, 3, O.ZERO, O.DOWN, 2, O.PROJECT_REDUCE),
    (24, 40, 8, 16, 3, 5, O.VALID, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (12, 20, 8, 16, 2, 5, O.FULL, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (36, 12, 17, 9, 2, 7, O.ZERO, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (56, 56, 32, 32, 1, 1, O.ZERO, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (16, 16, 32, 16, 2, 3, O.ZERO, O.NOSAMPLE, 1, O.BACKPROJECT_REDUCE),
    (44, 48, 24, 72, 2, 5, O.ZERO, O.DOWN, 2, O.BACKPROJECT_REDUCE),
    # a 208-wide halo: 16-plane blocks (two 32-plane halo buffers do not fit)
    (24, 200, 32, 64, 1, 5, O.ZERO, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    # border policies the halo loads map per element (ConvolveHyperKernel.scala:235-317)
    (30, 31, 20, 70, 2, 7, O.CLAMP, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (30, 30, 20, 70, 2, 7, O.CLAMP, O.DOWN, 2, O.PROJECT_REDUCE),
    (30, 30, 20, 70, 2, 3, O.CYCLIC, O.DOWN, 2, O.PROJECT_REDUCE),
    (40, 44, 17, 130, 2, 5, O.CYCLIC, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (33, 37, 5, 7, 3, 3, O.VALID, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (33, 37, 5, 7, 3, 3, O.FULL, O.NOSAMPLE, 1, O.BACKPROJECT_REDUCE),
    (21, 23, 12, 20, 2, 5, O.CLAMP, O.NOSAMPLE, 1, O.BACKPROJECT_REDUCE),
    # odd widths (no 16-byte rule on the halo loads) and 1-wide fields
    (9, 9, 1, 1, 1, 9, O.ZERO, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (1, 300, 8, 8, 1, 1, O.ZERO, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (300, 1, 8, 8, 1, 1, O.CYCLIC, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    # fields wider than one band of output columns
    (64, 520, 16, 16, 1, 5, O.CLAMP, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (40, 1027, 4, 16, 1, 9, O.CYCLIC, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (64, 64, 32, 64, 2, 11, O.ZERO, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    # banks of at most 32 filters: two taps per MMA (even, odd and 2-wide filters)
    (40, 50, 3, 32, 2, 2, O.VALID, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (61, 67, 30, 40, 2, 6, O.FULL, O.NOSAMPLE, 1, O.BACKPROJECT_REDUCE),
    (100, 1000, 24, 20, 1, 7, O.CYCLIC, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (37, 29, 70, 31, 3, 9, O.ZERO, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    # UpsampleInput: one sub-filter per output phase (ConvolveHyperKernel.scala:206-212, 405-459)
    (32, 32, 32, 64, 2, 3, O.ZERO, O.UP, 2, O.BACKPROJECT_REDUCE),
    (32, 32, 64, 32, 2, 3, O.ZERO, O.UP, 2, O.BACKPROJECT_REDUCE),
    (32, 32, 32, 64, 2, 4, O.VALID, O.UP, 2, O.BACKPROJECT_REDUCE),
    (17, 23, 70, 20, 2, 5, O.CYCLIC, O.UP, 2, O.PROJECT_REDUCE),
    (20, 20, 8, 100, 2, 3, O.FULL, O.UP, 3, O.BACKPROJECT_REDUCE),
    (16, 16, 8, 8, 1, 1, O.ZERO, O.UP, 2, O.PROJECT_REDUCE),
    (30, 40, 16, 16, 2, 5, O.ZERO, O.UP, 4, O.BACKPROJECT_REDUCE),
    (33, 31, 12, 40, 2, 6, O.FULL, O.UP, 2, O.PROJECT_REDUCE),
]


@pytest.mark.parametrize("H,W,C,K,B,R,border,samp,step,mode", TC_CASES)
def test_tc_shapes(H, W, C, K, B, R, border, samp, step, mode):
    rng = np.random.default_rng(H * 100 + C * 7 + K)
    if mode == O.PROJECT_REDUCE:
        planes, orient = B * C, O.XCORR
    else:
        planes, orient = B * K, O.CONV
    od = O.make_desc(H, W, R, R, planes=planes, f_planes=K * C, batch=B, border=border,
                     orient=orient, sampling=samp, step=step, mode=mode)
    x = rng.standard_normal((planes, H, W)).astype(np.float32)
    f = rng.standard_normal((K * C, R, R)).astype(np.float32)
    check(run_tc(od, x, f), od, x, f)


def test_tc_relu_and_static_filter():
    rng = np.random.default_rng(77)
    H, W, C, K, B, R = 32, 32, 16, 32, 2, 3
    od = O.make_desc(H, W, R, R, planes=B * C, f_planes=K * C, batch=B, border=O.ZERO,
                     orient=O.XCORR, sampling=O.DOWN, step=2, mode=O.PROJECT_REDUCE)
    x = rng.standard_normal((B * C, H, W)).astype(np.float32)
    f = rng.standard_normal((K * C, R, R)).astype(np.float32)
    check(run_tc(od, x, f, flags=_lib.FLAG_RELU), od, x, f, relu=True)
    plan = _lib.Plan(_desc(od))
    plan.set_static_filter(f.ctypes.data)
    y = np.zeros((B * K, H // 2, W // 2), np.float32)
    plan.run_host(x.ctypes.data, 0, y.ctypes.data, 0)
    plan.close()
    check(y, od, x, f)


def test_tc_unsupported_shapes_use_fp32_kernel():
    # DownsampleOutput(3) is outside the tensor-core kernels: the plan takes an
    # FP32 kernel, bit-exact with the FP32 oracle.
    rng = np.random.default_rng(3)
    od = O.make_desc(18, 18, 3, 3, planes=8, f_planes=16, batch=1, border=O.CLAMP,
                     orient=O.XCORR, sampling=O.DOWN, step=3, mode=O.PROJECT_REDUCE)
    x = rng.standard_normal((8, 18, 18)).astype(np.float32)
    f = rng.standard_normal((16, 3, 3)).astype(np.float32)
    y = run_tc(od, x, f, expect_tc=False)
    plan = _lib.Plan(_desc(od))
    assert plan.algo in (_lib.PLAN_FRAME_F32, _lib.PLAN_DIRECT)
    plan.close()
    assert np.array_equal(y, O.conv(od, x, f))


# Three-term split (BF16X6): the six products down to 2^-16 of hi*hi, with the
# hi*hi accumulator promoted into an FP32 running sum every 64 k-steps, so the
# error stays near FP32 level whatever the reduction length.
X6_TOL = 3e-6
X6_CASES = [
    # (H, W, C, K, B, R, border, sampling, step, mode)
    (28, 28, 512, 512, 1, 3, O.ZERO, O.NOSAMPLE, 1, O.PROJECT_REDUCE),   # a 4608-long reduction
    (56, 56, 256, 256, 1, 3, O.ZERO, O.DOWN, 2, O.PROJECT_REDUCE),
    (64, 64, 32, 64, 2, 5, O.ZERO, O.NOSAMPLE, 1, O.BACKPROJECT_REDUCE),
    (40, 44, 17, 70, 2, 5, O.CYCLIC, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (48, 48, 3, 64, 2, 3, O.ZERO, O.NOSAMPLE, 1, O.PROJECT_REDUCE),
    (40, 40, 64, 128, 2, 5, O.ZERO, O.UP, 2, O.BACKPROJECT_REDUCE),
]


@pytest.mark.parametrize("H,W,C,K,B,R,border,samp,step,mode", X6_CASES)
def test_tc_three_term_split(H, W, C, K, B, R, border, samp, step, mode):
    rng = np.random.default_rng(H + 3 * C + K)
    if mode == O.PROJECT_REDUCE:
        planes, orient = B * C, O.XCORR
    else:
        planes, orient = B * K, O.CONV
    od = O.make_desc(H, W, R, R, planes=planes, f_planes=K * C, batch=B, border=border,
                     orient=orient, sampling=samp, step=step, mode=mode)
    x = rng.standard_normal((planes, H, W)).astype(np.float32)
    f = (rng.standard_normal((K * C, R, R)) * np.sqrt(2.0 / (C * R * R))).astype(np.float32)
    mx, rms = check(run_tc(od, x, f, precision=_lib.PREC_BF16X6), od, x, f, tol=X6_TOL)
    print(f"BF16X6 {H}x{W} C{C} K{K}: normwise max {mx:.3e} rms {rms:.3e}")


def test_tc_repeatable():
    """Same inputs, same plan, two runs: identical bits (no races)."""
    rng = np.random.default_rng(5)
    od = O.make_desc(64, 64, 5, 5, planes=4 * 32, f_planes=64 * 32, batch=4, border=O.ZERO,
                     orient=O.XCORR, mode=O.PROJECT_REDUCE)
    x = rng.standard_normal((128, 64, 64)).astype(np.float32)
    f = rng.standard_normal((2048, 5, 5)).astype(np.float32)
    a = run_tc(od, x, f)
    b = run_tc(od, x, f)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("mode,relu", [(O.PROJECT_REDUCE, False), (O.PROJECT_REDUCE, True),
                                       (O.BACKPROJECT_REDUCE, False)])
def test_tc_partial_last_wave_two_plane_blocks(mode, relu):
    """176 tiles on 148 SMs (a partial second wave), 64 input planes as two
    32-plane halo blocks of 9 taps each: within tolerance of FP64, ReLU
    applied once, and bit-identical run to run."""
    rng = np.random.default_rng(91 + mode)
    H, W, C, K, B, R = 32, 64, 64, 48, 11, 3
    if mode == O.PROJECT_REDUCE:
        planes, orient = B * C, O.XCORR
    else:
        planes, orient = B * K, O.CONV
    od = O.make_desc(H, W, R, R, planes=planes, f_planes=K * C, batch=B, border=O.ZERO,
                     orient=orient, mode=mode)
    x = rng.standard_normal((planes, H, W)).astype(np.float32)
    f = rng.standard_normal((K * C, R, R)).astype(np.float32)
    flags = _lib.FLAG_RELU if relu else 0
    a = run_tc(od, x, f, flags=flags)
    check(a, od, x, f, relu=relu)
    b = run_tc(od, x, f, flags=flags)
    assert np.array_equal(a, b)


def _random_cases(n, seed):
    """Seeded random shapes over every border, both directions, down 2 and
    up 2/3, both precisions, with and without ReLU."""
    import random
    rng = random.Random(seed)
    out = []
    for _ in range(n):
        border = rng.choice([O.ZERO, O.CLAMP, O.CYCLIC, O.VALID, O.FULL])
        odd = border in (O.ZERO, O.CLAMP, O.CYCLIC)
        R = rng.choice([1, 3, 5] if odd else [1, 2, 3, 4, 5])
        samp = rng.choice(["none", "none", "down", "up"])
        if samp == "up" and border == O.CLAMP:
            border = O.ZERO  # integrated upsampling with BorderClamp is refused
        H, W = rng.randint(max(R, 2), 40), rng.randint(max(R, 2), 44)
        if samp == "down":
            cr = R - 1 if border == O.VALID else (1 - R if border == O.FULL else 0)
            H += (H - cr) % 2
            W += (W - cr) % 2
        out.append((H, W, rng.randint(1, 2), rng.randint(1, 40), rng.randint(1, 80), R, border,
                    {"none": (O.NOSAMPLE, 1), "down": (O.DOWN, 2), "up": (O.UP, rng.choice([2, 3]))}[samp],
                    rng.random() < 0.5, rng.random() < 0.25, rng.random() < 0.3))
    return out


@pytest.mark.parametrize("H,W,B,C,K,R,border,samp,back,x6,relu", _random_cases(40, 11))
def test_tc_random_shapes(H, W, B, C, K, R, border, samp, back, x6, relu):
    rng = np.random.default_rng(H * 7919 + W * 31 + C * 3 + K)
    sampling, step = samp
    if back:
        planes, orient, mode = B * K, O.CONV, O.BACKPROJECT_REDUCE
    else:
        planes, orient, mode = B * C, O.XCORR, O.PROJECT_REDUCE
    od = O.make_desc(H, W, R, R, planes=planes, f_planes=K * C, batch=B, border=border,
                     orient=orient, sampling=sampling, step=step, mode=mode)
    x = rng.standard_normal((planes, H, W)).astype(np.float32)
    f = (rng.standard_normal((K * C, R, R)) * np.sqrt(2.0 / (C * R * R))).astype(np.float32)
    prec = _lib.PREC_BF16X6 if x6 else _lib.PREC_BF16X3
    y = run_tc(od, x, f, flags=_lib.FLAG_RELU if relu else 0, precision=prec)
    check(y, od, x, f, relu=relu, tol=X6_TOL if x6 else TOL)
