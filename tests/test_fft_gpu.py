"""FFT convolution plans against the FP64 oracle.

The reference sends plane-by-plane convolutions under BorderZero, BorderClamp
and BorderCyclic without integrated sampling to its FFT generator when the
policy allows it (generator/DynamicConvolutionGenerator.scala:108-158) and
sizes the transform by generator/FFTConvolutionUtils.scala:38-97.  The FFT
path computes in FP32, so it is checked against the FP64 direct oracle within
a normwise 1e-5 (max |error| / max |reference|), and the large-kernel case
reports its max and RMS error beside the bound.
"""
import numpy as np
import pytest
import torch

import cctconv
import oracle as O
from cctconv import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-5

BORDERS = {"zero": (_lib.BORDER_ZERO, O.ZERO), "clamp": (_lib.BORDER_CLAMP, O.CLAMP),
           "cyclic": (_lib.BORDER_CYCLIC, O.CYCLIC)}
ORIENTS = {"conv": (_lib.CONVOLUTION, O.CONV), "xcorr": (_lib.CROSS_CORRELATION, O.XCORR)}


def _desc(H, W, R, S, pin, pf, border, orient, algo=_lib.ALGO_FFT, flags=0,
          sampling=_lib.SAMPLE_NONE, step=1):
    return _lib.new_desc(image_rows=H, image_cols=W, image_planes=pin, filter_rows=R,
                         filter_cols=S, filter_planes=pf, batch_size=1, border=border,
                         orientation=orient, sampling=sampling, step=step,
                         vector_mode=_lib.PLANE_BY_PLANE, precision=_lib.PREC_FP32, algo=algo,
                         flags=flags)


def _run(plan, x, f):
    orows, ocols, oplanes = plan.shape
    y = torch.full((max(oplanes, 1), orows, ocols), float("nan"), device="cuda")
    # a null filter pointer selects the plan's static filter
    plan.run(x.data_ptr(), 0 if f is None else f.data_ptr(), y.data_ptr(),
             torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return y.cpu().numpy()


def _oracle(H, W, R, S, pin, pf, ob, oo, x, f):
    od = O.make_desc(H, W, R, S, planes=pin, f_planes=pf, border=ob, orient=oo,
                     mode=O.PLANE)
    return O.conv(od, x, f, np.float64)


SHAPES = [
    # H, W, R, S, image planes, filter planes (0 = ScalarField)
    (37, 50, 9, 9, 0, 0),
    (64, 64, 15, 15, 3, 3),
    (20, 130, 7, 3, 0, 3),
    (33, 31, 5, 11, 2, 0),
    (128, 96, 31, 31, 0, 0),
    (2, 9, 3, 3, 0, 0),
]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s)))
@pytest.mark.parametrize("border", list(BORDERS))
@pytest.mark.parametrize("orient", list(ORIENTS))
def test_fft_matches_fp64_direct(shape, border, orient):
    H, W, R, S, pin, pf = shape
    (cb, ob), (co, oo) = BORDERS[border], ORIENTS[orient]
    rng = np.random.default_rng(H * 1000 + W + R)
    x = rng.uniform(-1, 1, (max(pin, 1), H, W)).astype(np.float32)
    f = rng.uniform(-1, 1, (max(pf, 1), R, S)).astype(np.float32)
    plan = _lib.Plan(_desc(H, W, R, S, pin, pf, cb, co))
    if plan.algo != _lib.PLAN_FFT:
        # the transform grid cannot hold this border extension: direct, as
        # the reference falls back when the FFT cannot take the case
        pytest.skip("FFT grid does not hold the extension")
    y = _run(plan, torch.from_numpy(x).cuda(), torch.from_numpy(f).cuda())
    plan.close()
    ref = _oracle(H, W, R, S, pin, pf, ob, oo, x, f)
    emax, erms = O.rel_errors(y.reshape(ref.shape), ref)
    assert emax <= TOL, (emax, erms)


def test_fft_plans_are_taken_for_the_standard_shapes():
    for H, W, R, S, pin, pf in SHAPES[:5]:
        for cb, _ in BORDERS.values():
            plan = _lib.Plan(_desc(H, W, R, S, pin, pf, cb, _lib.CONVOLUTION))
            assert plan.algo == _lib.PLAN_FFT, (H, W, R, S, cb)
            plan.close()


@pytest.mark.parametrize("border", list(BORDERS))
def test_fft_static_filter_matches_dynamic(border):
    """A static filter's spectrum is made once on the host in FP64
    (DynamicConvolutionGenerator.scala:342-350); the result agrees with the
    dynamic filter's device spectrum and with the oracle."""
    cb, ob = BORDERS[border]
    H, W, R = 100, 120, 21
    rng = np.random.default_rng(11)
    x = rng.uniform(-1, 1, (4, H, W)).astype(np.float32)
    f = rng.uniform(-1, 1, (4, R, R)).astype(np.float32)
    xd, fd = torch.from_numpy(x).cuda(), torch.from_numpy(f).cuda()
    dyn = _lib.Plan(_desc(H, W, R, R, 4, 4, cb, _lib.CROSS_CORRELATION))
    sta = _lib.Plan(_desc(H, W, R, R, 4, 4, cb, _lib.CROSS_CORRELATION))
    assert dyn.algo == sta.algo == _lib.PLAN_FFT
    sta.set_static_filter(f.ctypes.data)
    yd, ys = _run(dyn, xd, fd), _run(sta, xd, None)
    ref = _oracle(H, W, R, R, 4, 4, ob, O.XCORR, x, f)
    assert O.rel_errors(yd, ref)[0] <= TOL
    assert O.rel_errors(ys, ref)[0] <= TOL
    # the static spectrum is FP64-rounded once, the dynamic one in FP32
    assert O.rel_errors(ys, ref)[0] <= O.rel_errors(yd, ref)[0] * 1.5 + 1e-7
    dyn.close()
    sta.close()


def test_fft_large_kernel_2048_cyclic_gaussian():
    """2048x2048 uniform[0,1] field, 63x63 normalised Gaussian (sigma 10),
    BorderCyclic, against the FP64 cyclic convolution and the direct kernel."""
    n, k, sigma = 2048, 63, 10.0
    rng = np.random.default_rng(2048)
    x = rng.uniform(0, 1, (n, n)).astype(np.float32)
    r = np.arange(k) - k // 2
    g = np.exp(-(r[:, None] ** 2 + r[None, :] ** 2) / (2 * sigma * sigma))
    f = (g / g.sum()).astype(np.float32)
    xd, fd = torch.from_numpy(x).cuda(), torch.from_numpy(f).cuda()
    ref = O.cyclic_conv_fft64(x, f, O.CONV)
    y = cctconv.convolve(xd, fd, cctconv.BorderCyclic, fftUse=cctconv.UseFFTAlways)
    torch.cuda.synchronize()
    emax, erms = O.rel_errors(y.cpu().numpy(), ref)
    print(f"fft 2048^2 (*) 63^2 cyclic: max rel {emax:.3e} rms rel {erms:.3e}")
    assert emax <= TOL and erms <= TOL
    yd = cctconv.convolve(xd, fd, cctconv.BorderCyclic, fftUse=cctconv.UseFFTNever)
    torch.cuda.synchronize()
    dmax, _ = O.rel_errors(yd.cpu().numpy(), ref)
    assert dmax <= TOL


def test_fft_when_best_takes_fft_for_large_filters_only():
    big = _lib.Plan(_desc(2048, 2048, 63, 63, 0, 0, _lib.BORDER_CYCLIC, _lib.CONVOLUTION,
                          algo=_lib.ALGO_AUTO))
    small = _lib.Plan(_desc(256, 256, 5, 5, 0, 0, _lib.BORDER_ZERO, _lib.CONVOLUTION,
                            algo=_lib.ALGO_AUTO))
    never = _lib.Plan(_desc(2048, 2048, 63, 63, 0, 0, _lib.BORDER_CYCLIC, _lib.CONVOLUTION,
                            algo=_lib.ALGO_DIRECT))
    assert big.algo == _lib.PLAN_FFT
    assert small.algo != _lib.PLAN_FFT
    assert never.algo != _lib.PLAN_FFT
    for p in (big, small, never):
        p.close()


def _launch_us(plan, x, f, y, reps=10):
    st = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        plan.run(x.data_ptr(), f.data_ptr(), y.data_ptr(), st)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        plan.run(x.data_ptr(), f.data_ptr(), y.data_ptr(), st)
    b.record()
    b.synchronize()
    return a.elapsed_time(b) * 1e3 / reps


@pytest.mark.parametrize("R", [15, 31])
def test_fft_when_best_takes_the_measured_faster_path(R):
    """UseFFTWhenBest on a 1024x1024 field with a 15x15 or 31x31 filter (where
    the modelled costs are close, so the plan times both paths on the
    device): the plan takes the path that is faster here, or one within 20%
    of it (the FFT must win by 1.2x to be taken over the exact direct path)."""
    n = 1024
    auto = _lib.Plan(_desc(n, n, R, R, 0, 0, _lib.BORDER_ZERO, _lib.CONVOLUTION, algo=_lib.ALGO_AUTO))
    direct = _lib.Plan(_desc(n, n, R, R, 0, 0, _lib.BORDER_ZERO, _lib.CONVOLUTION, algo=_lib.ALGO_DIRECT))
    fft = _lib.Plan(_desc(n, n, R, R, 0, 0, _lib.BORDER_ZERO, _lib.CONVOLUTION, algo=_lib.ALGO_FFT))
    assert fft.algo == _lib.PLAN_FFT and direct.algo != _lib.PLAN_FFT
    x = torch.rand((n, n), device="cuda")
    f = torch.rand((R, R), device="cuda")
    y = torch.empty((n, n), device="cuda")
    fh = f.cpu().numpy()
    fft.set_static_filter(fh.ctypes.data)  # the triage times the FFT with a static filter
    t_direct = _launch_us(direct, x, f, y)
    t_fft = min(_launch_us(fft, x, f, y), _launch_us(fft, x, f, y))
    faster = _lib.PLAN_FFT if t_fft < t_direct else direct.algo
    slower_ok = max(t_direct, t_fft) <= 1.2 * min(t_direct, t_fft)
    print(f"{R}x{R} on {n}^2: direct {t_direct:.1f} us, fft {t_fft:.1f} us, auto took algo {auto.algo}")
    assert auto.algo == faster or slower_ok, (t_direct, t_fft, auto.algo)
    for p in (auto, direct, fft):
        p.close()


@pytest.mark.parametrize("case", ["valid", "full", "downsample", "upsample", "frame"])
def test_fft_always_falls_back_where_the_fft_cannot_go(case):
    """UseFFTAlways on a form the FFT generator does not take runs the direct
    kernels, bit-exact with the FP32 oracle."""
    H, W, R = 24, 28, 5
    rng = np.random.default_rng(5)
    kw = dict(border=_lib.BORDER_ZERO, ob=O.ZERO, sampling=_lib.SAMPLE_NONE, step=1, osamp=O.NOSAMPLE)
    if case == "valid":
        kw.update(border=_lib.BORDER_VALID, ob=O.VALID)
    elif case == "full":
        kw.update(border=_lib.BORDER_FULL, ob=O.FULL)
    elif case == "downsample":
        kw.update(sampling=_lib.SAMPLE_DOWN, step=2, osamp=O.DOWN)
    elif case == "upsample":
        kw.update(sampling=_lib.SAMPLE_UP, step=2, osamp=O.UP)
    x = rng.uniform(-1, 1, (2, H, W)).astype(np.float32)
    f = rng.uniform(-1, 1, (4 if case == "frame" else 2, R, R)).astype(np.float32)
    mode = _lib.PROJECT_FRAME if case == "frame" else _lib.PLANE_BY_PLANE
    desc = _lib.new_desc(image_rows=H, image_cols=W, image_planes=2, filter_rows=R,
                         filter_cols=R, filter_planes=f.shape[0], batch_size=1,
                         border=kw["border"], orientation=_lib.CONVOLUTION,
                         sampling=kw["sampling"], step=kw["step"], vector_mode=mode,
                         precision=_lib.PREC_FP32, algo=_lib.ALGO_FFT)
    plan = _lib.Plan(desc)
    assert plan.algo != _lib.PLAN_FFT
    y = _run(plan, torch.from_numpy(x).cuda(), torch.from_numpy(f).cuda())
    od = O.make_desc(H, W, R, R, planes=2, f_planes=f.shape[0], border=kw["ob"], orient=O.CONV,
                     sampling=kw["osamp"], step=kw["step"],
                     mode=O.PROJECT if case == "frame" else O.PLANE)
    ref = O.conv(od, x, f, np.float32)
    assert np.array_equal(y.reshape(ref.shape).view(np.uint32), ref.view(np.uint32))
    plan.close()


@pytest.mark.parametrize("border", list(BORDERS))
def test_fft_known_answers(border):
    """An impulse filter returns the field; a normalised filter on a constant
    field returns the constant (Clamp and Cyclic extend the constant)."""
    cb, _ = BORDERS[border]
    H, W, R = 50, 70, 11
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, (H, W)).astype(np.float32)
    imp = np.zeros((R, R), np.float32)
    imp[R // 2, R // 2] = 1
    plan = _lib.Plan(_desc(H, W, R, R, 0, 0, cb, _lib.CONVOLUTION))
    assert plan.algo == _lib.PLAN_FFT
    y = _run(plan, torch.from_numpy(x).cuda(), torch.from_numpy(imp).cuda())
    assert np.abs(y[0] - x).max() <= 1e-6
    if border != "zero":
        c = np.full((H, W), 0.75, np.float32)
        box = np.full((R, R), 1.0 / (R * R), np.float32)
        y = _run(plan, torch.from_numpy(c).cuda(), torch.from_numpy(box).cuda())
        assert np.abs(y[0] - 0.75).max() <= 1e-6
    plan.close()


def test_fft_relu_flag():
    H, W, R = 40, 40, 13
    rng = np.random.default_rng(9)
    x = rng.uniform(-1, 1, (H, W)).astype(np.float32)
    f = rng.uniform(-1, 1, (R, R)).astype(np.float32)
    plan = _lib.Plan(_desc(H, W, R, R, 0, 0, _lib.BORDER_ZERO, _lib.CROSS_CORRELATION,
                           flags=_lib.FLAG_RELU))
    assert plan.algo == _lib.PLAN_FFT
    y = _run(plan, torch.from_numpy(x).cuda(), torch.from_numpy(f).cuda())
    ref = np.maximum(_oracle(H, W, R, R, 0, 0, O.ZERO, O.XCORR, x, f), 0)
    assert (y >= 0).all()
    assert O.rel_errors(y.reshape(ref.shape), ref)[0] <= TOL


def test_fft_repeated_runs_are_identical():
    H, W, R = 96, 96, 17
    rng = np.random.default_rng(4)
    x = torch.from_numpy(rng.uniform(-1, 1, (3, H, W)).astype(np.float32)).cuda()
    f = torch.from_numpy(rng.uniform(-1, 1, (3, R, R)).astype(np.float32)).cuda()
    plan = _lib.Plan(_desc(H, W, R, R, 3, 3, _lib.BORDER_CLAMP, _lib.CONVOLUTION))
    a, b = _run(plan, x, f), _run(plan, x, f)
    assert np.array_equal(a, b)
    plan.close()
