"""GPU parity: libcctconv's CUDA kernels, called through the C-ABI, against
the oracle on the same seeded inputs.

The FP32 direct, separable and frame kernels keep the reference's summation
order, so they must match the FP32 oracle bit for bit; the golden vectors
are checked with the reference's own ~== (RefFieldMemory.scala:433-485).
"""
import itertools

import numpy as np
import pytest
import torch

import oracle as O
from cctconv import _lib
from helpers import (ADJOINT_BORDER, ADJOINT_SAMPLING, bitwise_equal, golden_case,
                     legal_in_reference, ref_field_approx_equal)

pytestmark = pytest.mark.gpu


def _desc_from_oracle(od, precision=_lib.PREC_FP32, algo=_lib.ALGO_AUTO, flags=0):
    return _lib.new_desc(image_rows=od.rows, image_cols=od.cols, image_planes=od.planes,
                         filter_rows=od.f_rows, filter_cols=od.f_cols, filter_planes=od.f_planes,
                         batch_size=od.batch, border=od.border, orientation=od.orient,
                         sampling=od.sampling, step=od.step, vector_mode=od.mode,
                         precision=precision, algo=algo, flags=flags)


def gpu_conv(od, x, f, precision=_lib.PREC_FP32, algo=_lib.ALGO_AUTO, flags=0, want_algo=None):
    """Run one descriptor on the GPU through the C-ABI; returns (y, plan algo)."""
    desc = _desc_from_oracle(od, precision, algo, flags)
    plan = _lib.Plan(desc)
    if want_algo is not None:
        assert plan.algo == want_algo
    orows, ocols, oplanes = plan.shape
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).cuda()
    fd = torch.from_numpy(np.ascontiguousarray(f, dtype=np.float32)).cuda()
    yd = torch.full((oplanes, orows, ocols), float("nan"), device="cuda")
    plan.run(xd.data_ptr(), fd.data_ptr(), yd.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    out = yd.cpu().numpy()
    plan.close()
    return out, plan.algo


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    major, _ = torch.cuda.get_device_capability()
    assert major == 10, "needs an sm_100 GPU"


@pytest.mark.parametrize("i", range(25))
def test_golden_convolve(golden, i):
    sampling, step, border, a = golden_case(golden, i)
    if not legal_in_reference(sampling, step, border):
        pytest.skip("Upsample + BorderClamp is rejected by the reference")
    x, k, wx = a["x"], a["k"], a["wx"]
    od = O.make_desc(x.shape[0], x.shape[1], k.shape[0], k.shape[1], border=border,
                     orient=O.CONV, sampling=sampling, step=step)
    y, _ = gpu_conv(od, x, k)
    assert ref_field_approx_equal(y[0], wx)
    assert bitwise_equal(y[0], O.conv(od, x, k)[0])


@pytest.mark.parametrize("i", range(25))
def test_golden_adjoint(golden, i):
    sampling, step, border, a = golden_case(golden, i)
    if border not in ADJOINT_BORDER:
        pytest.skip("BorderClamp has no convolution-form adjoint")
    y, k, wty = a["y"], a["k"], a["wty"]
    od = O.make_desc(y.shape[0], y.shape[1], k.shape[0], k.shape[1],
                     border=ADJOINT_BORDER[border], orient=O.XCORR,
                     sampling=ADJOINT_SAMPLING[sampling], step=step)
    got, _ = gpu_conv(od, y, k)
    assert ref_field_approx_equal(got[0], wty)
    assert bitwise_equal(got[0], O.conv(od, y, k)[0])


SIZES = [(37, 45), (64, 64), (1, 50), (5, 3), (97, 31)]
FILTERS = [(1, 1), (3, 3), (5, 5), (7, 7), (9, 9), (13, 11), (3, 5)]
SAMPLINGS = [(O.NOSAMPLE, 1), (O.DOWN, 2), (O.DOWN, 3), (O.UP, 2), (O.UP, 3)]


def _cases():
    rng = np.random.default_rng(2024)
    out = []
    for (h, w), (fr, fc), border, (samp, step), orient in itertools.product(
            SIZES, FILTERS, range(5), SAMPLINGS, (O.XCORR, O.CONV)):
        if h == 1 and fr != 1:
            continue
        od = O.make_desc(h, w, fr, fc, border=border, orient=orient, sampling=samp, step=step)
        try:
            O.output_shape(od)
        except ValueError:
            continue
        out.append(od)
    idx = rng.choice(len(out), size=min(160, len(out)), replace=False)
    return [out[i] for i in sorted(idx)]


@pytest.mark.parametrize("od", _cases(), ids=lambda d: (
    f"{d.rows}x{d.cols}_f{d.f_rows}x{d.f_cols}_b{d.border}_o{d.orient}_s{d.sampling}x{d.step}"))
def test_plane_sweep_bitwise(od):
    rng = np.random.default_rng(od.rows * 1000 + od.f_rows * 10 + od.border)
    x = rng.uniform(-1, 1, (od.rows, od.cols)).astype(np.float32)
    f = rng.uniform(-1, 1, (od.f_rows, od.f_cols)).astype(np.float32)
    y, _ = gpu_conv(od, x, f)
    assert bitwise_equal(y, O.conv(od, x, f))


MODE_CASES = [
    # (mode, planes, f_planes, batch, filter, border, sampling, step)
    (O.PLANE, 4, 0, 1, 5, O.CLAMP, O.NOSAMPLE, 1),
    (O.PLANE, 0, 6, 1, 3, O.CYCLIC, O.DOWN, 2),
    (O.PLANE, 5, 5, 1, 7, O.ZERO, O.UP, 2),
    (O.PROJECT, 6, 12, 2, 3, O.ZERO, O.NOSAMPLE, 1),
    (O.PROJECT, 4, 8, 1, 5, O.VALID, O.DOWN, 2),
    (O.BACKPROJECT, 6, 12, 2, 3, O.FULL, O.NOSAMPLE, 1),
    (O.BACKPROJECT, 8, 8, 2, 5, O.ZERO, O.UP, 2),
    (O.PROJECT_REDUCE, 6, 24, 2, 3, O.ZERO, O.NOSAMPLE, 1),
    (O.PROJECT_REDUCE, 8, 40, 2, 5, O.CLAMP, O.DOWN, 2),
    (O.PROJECT_REDUCE, 3, 3, 1, 1, O.CYCLIC, O.NOSAMPLE, 1),
    (O.PROJECT_REDUCE, 4, 36, 1, 7, O.ZERO, O.UP, 2),
    (O.PROJECT_REDUCE, 6, 30, 3, 9, O.ZERO, O.NOSAMPLE, 1),
    (O.BACKPROJECT_REDUCE, 10, 20, 2, 3, O.ZERO, O.NOSAMPLE, 1),
    (O.BACKPROJECT_REDUCE, 8, 32, 2, 5, O.CYCLIC, O.DOWN, 2),
    (O.BACKPROJECT_REDUCE, 34, 17 * 3, 2, 3, O.ZERO, O.NOSAMPLE, 1),
    (O.BACKPROJECT_REDUCE, 4, 12, 1, 5, O.FULL, O.UP, 3),
    # unfused frame modes with several 16-filter blocks (the FP32 frame kernel
    # without its reduce: every input plane's result to its own output plane)
    (O.PROJECT, 2 * 5, 37 * 5, 2, 7, O.CLAMP, O.NOSAMPLE, 1),
    (O.BACKPROJECT, 2 * 6, 6 * 20, 2, 3, O.CYCLIC, O.DOWN, 2),
]


@pytest.mark.parametrize("mode", [O.PROJECT, O.BACKPROJECT])
def test_unfused_frame_modes_take_the_frame_kernel(mode):
    od = O.make_desc(32, 40, 5, 5, planes=2 * 8, f_planes=40 * 8, batch=2, border=O.ZERO, orient=O.XCORR,
                     mode=mode)
    x = np.random.default_rng(4).normal(size=(16, 32, 40)).astype(np.float32)
    f = np.random.default_rng(5).normal(size=(320, 5, 5)).astype(np.float32)
    y, algo = gpu_conv(od, x, f)
    assert algo == _lib.PLAN_FRAME_F32
    assert bitwise_equal(y, O.conv(od, x, f))


@pytest.mark.parametrize("mode,planes,fplanes,batch,fs,border,samp,step", MODE_CASES)
@pytest.mark.parametrize("orient", [O.XCORR, O.CONV])
def test_vector_modes_bitwise(mode, planes, fplanes, batch, fs, border, samp, step, orient):
    rng = np.random.default_rng(planes * 131 + fplanes)
    h, w = (24, 36) if samp != O.DOWN else (24, 36)
    od = O.make_desc(h, w, fs, fs, planes=planes, f_planes=fplanes, batch=batch, border=border,
                     orient=orient, sampling=samp, step=step, mode=mode)
    x = rng.normal(size=(max(planes, 1), h, w)).astype(np.float32)
    f = rng.normal(size=(max(fplanes, 1), fs, fs)).astype(np.float32)
    y, _ = gpu_conv(od, x, f)
    assert bitwise_equal(y, O.conv(od, x, f))


def test_config1_plain_convolve_bitwise():
    """256x256 field (*) 5x5 filter, BorderZero, U[-1,1] seed 1."""
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, (256, 256)).astype(np.float32)
    f = rng.uniform(-1, 1, (5, 5)).astype(np.float32)
    od = O.make_desc(256, 256, 5, 5, border=O.ZERO, orient=O.CONV)
    y, algo = gpu_conv(od, x, f, want_algo=_lib.PLAN_DIRECT)
    assert bitwise_equal(y, O.conv(od, x, f))
    assert O.rel_errors(y, O.conv(od, x, f, np.float64))[0] < 1e-6


def _cfg2_inputs():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((16 * 32, 64, 64)).astype(np.float32)
    f = (rng.standard_normal((64 * 32, 5, 5)) * np.sqrt(2.0 / 800)).astype(np.float32)
    g = rng.standard_normal((16 * 64, 64, 64)).astype(np.float32)
    return x, f, g


def test_config2_project_frame_fp32_bitwise():
    x, f, _ = _cfg2_inputs()
    od = O.make_desc(64, 64, 5, 5, planes=512, f_planes=2048, batch=16, border=O.ZERO,
                     orient=O.XCORR, mode=O.PROJECT_REDUCE)
    y, _ = gpu_conv(od, x, f, want_algo=_lib.PLAN_FRAME_F32)
    assert bitwise_equal(y, O.conv(od, x, f))
    assert O.rel_errors(y, O.conv(od, x, f, np.float64))[0] < 1e-5


def test_config2_back_project_frame_fp32_bitwise():
    _, f, g = _cfg2_inputs()
    od = O.make_desc(64, 64, 5, 5, planes=1024, f_planes=2048, batch=16, border=O.ZERO,
                     orient=O.CONV, mode=O.BACKPROJECT_REDUCE)
    y, _ = gpu_conv(od, g, f, want_algo=_lib.PLAN_FRAME_F32)
    assert bitwise_equal(y, O.conv(od, g, f))
    assert O.rel_errors(y, O.conv(od, g, f, np.float64))[0] < 1e-5


def test_batched_planes_share_one_filter():
    """4096 planes of 256x256 against one 5x5 filter (the HBM-bound form of
    the plain convolve): every plane equals the single-plane result."""
    rng = np.random.default_rng(9)
    P = 4096
    x = torch.empty((P, 256, 256), device="cuda").uniform_(-1, 1, generator=torch.Generator(
        device="cuda").manual_seed(9))
    f = rng.uniform(-1, 1, (5, 5)).astype(np.float32)
    od = O.make_desc(256, 256, 5, 5, planes=P, f_planes=0, border=O.ZERO, orient=O.CONV)
    plan = _lib.Plan(_desc_from_oracle(od))
    fd = torch.from_numpy(f).cuda()
    y = torch.empty_like(x)
    plan.run(x.data_ptr(), fd.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    od1 = O.make_desc(256, 256, 5, 5, border=O.ZERO, orient=O.CONV)
    for p in (0, 1, 1234, P - 1):
        xp = x[p].cpu().numpy()
        assert bitwise_equal(y[p].cpu().numpy(), O.conv(od1, xp, f)[0])
    plan.close()


def test_relu_flag():
    rng = np.random.default_rng(4)
    x = rng.normal(size=(6, 20, 20)).astype(np.float32)
    f = rng.normal(size=(12, 3, 3)).astype(np.float32)
    od = O.make_desc(20, 20, 3, 3, planes=6, f_planes=12, batch=2, orient=O.XCORR,
                     sampling=O.DOWN, step=2, mode=O.PROJECT_REDUCE)
    y, _ = gpu_conv(od, x, f, flags=_lib.FLAG_RELU)
    assert bitwise_equal(y, np.maximum(O.conv(od, x, f), 0))


@pytest.mark.parametrize("border", [O.ZERO, O.CLAMP, O.CYCLIC])
@pytest.mark.parametrize("orient", [O.XCORR, O.CONV])
def test_separable_bitwise(border, orient):
    rng = np.random.default_rng(17)
    x = rng.uniform(-1, 1, (3, 45, 70)).astype(np.float32)
    row = rng.uniform(-1, 1, 7).astype(np.float32)
    col = rng.uniform(-1, 1, 5).astype(np.float32)
    import cctconv as C
    pol = {O.ZERO: C.BorderZero, O.CLAMP: C.BorderClamp, O.CYCLIC: C.BorderCyclic}[border]
    fn = C.convolveSeparable if orient == O.CONV else C.crossCorrelateSeparable
    y = fn(torch.from_numpy(x).cuda(), torch.from_numpy(row).cuda(), torch.from_numpy(col).cuda(), pol)
    torch.cuda.synchronize()
    assert bitwise_equal(y.cpu().numpy(), O.separable(x, row, col, border, orient))


# filter lengths with compiled kernels (<= 9: TMA-staged under BorderZero when
# the width is a multiple of 4, register-window otherwise), the generic fused
# tile (longer) and the two-pass form (> 96 KB tile); fields smaller than,
# equal to and a few tiles larger than one tile, ragged in rows and columns
@pytest.mark.parametrize("rlen,clen", [(1, 1), (3, 9), (9, 3), (5, 5), (7, 1), (11, 13), (33, 17),
                                       (301, 3), (3, 301)])
@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 1, 4), (2, 32, 64), (2, 97, 150), (2, 97, 152),
                                   (1, 257, 196)])
def test_separable_lengths(rlen, clen, shape):
    import cctconv as C
    rng = np.random.default_rng(rlen * 100 + clen)
    x = rng.uniform(-1, 1, shape).astype(np.float32)
    row = rng.uniform(-1, 1, rlen).astype(np.float32)
    col = rng.uniform(-1, 1, clen).astype(np.float32)
    xd, rd, cd = (torch.from_numpy(a).cuda() for a in (x, row, col))
    for border, pol in [(O.ZERO, C.BorderZero), (O.CLAMP, C.BorderClamp), (O.CYCLIC, C.BorderCyclic)]:
        for orient, fn in [(O.XCORR, C.crossCorrelateSeparable), (O.CONV, C.convolveSeparable)]:
            y = fn(xd, rd, cd, pol)
            torch.cuda.synchronize()
            assert bitwise_equal(y.cpu().numpy(), O.separable(x, row, col, border, orient)), \
                (rlen, clen, shape, border, orient)


def test_separable_even_length_rejected():
    """Filters must be of odd size (ConvolveRows2DHyperKernel.scala:218-219)."""
    import cctconv as C
    x = torch.zeros((8, 8), device="cuda")
    with pytest.raises(ValueError, match="odd"):
        C.convolveSeparable(x, torch.ones(4, device="cuda"), torch.ones(3, device="cuda"), C.BorderZero)


def test_edge_cases():
    rng = np.random.default_rng(8)
    # 1x1 field, filter larger than the field (centred borders), prime sizes
    for (h, w, r, border) in [(1, 1, 3, O.ZERO), (1, 1, 5, O.CYCLIC), (1, 1, 3, O.CLAMP),
                              (2, 3, 7, O.CYCLIC), (3, 2, 9, O.ZERO), (13, 17, 15, O.CLAMP),
                              (7, 7, 7, O.VALID), (1, 1, 1, O.FULL)]:
        od = O.make_desc(h, w, r, r, border=border, orient=O.CONV)
        x = rng.uniform(-1, 1, (h, w)).astype(np.float32)
        f = rng.uniform(-1, 1, (r, r)).astype(np.float32)
        y, _ = gpu_conv(od, x, f)
        assert bitwise_equal(y, O.conv(od, x, f)), (h, w, r, border)


def test_python_api_matches_abi():
    import cctconv as C
    rng = np.random.default_rng(12)
    x = torch.from_numpy(rng.normal(size=(2 * 3, 16, 16)).astype(np.float32)).cuda()
    f = torch.from_numpy(rng.normal(size=(4 * 3, 3, 3)).astype(np.float32)).cuda()
    y = C.projectFrameBlockReduceSum(x, f, C.BorderZero, batchSize=2)
    od = O.make_desc(16, 16, 3, 3, planes=6, f_planes=12, batch=2, orient=O.XCORR,
                     mode=O.PROJECT_REDUCE)
    torch.cuda.synchronize()
    assert bitwise_equal(y.cpu().numpy(), O.conv(od, x.cpu().numpy(), f.cpu().numpy()))
    with pytest.raises(ValueError, match="BorderClamp"):
        C.convolve(x[0], f[0], C.BorderClamp, C.UpsampleInputConvolution(2))
    s = C.convolve(x[0], f[0], C.BorderZero)
    assert s.shape == (16, 16)


def test_run_host_equals_device_run():
    rng = np.random.default_rng(21)
    x = rng.normal(size=(4, 32, 32)).astype(np.float32)
    f = rng.normal(size=(8, 5, 5)).astype(np.float32)
    od = O.make_desc(32, 32, 5, 5, planes=4, f_planes=8, batch=1, orient=O.XCORR,
                     mode=O.PROJECT_REDUCE)
    plan = _lib.Plan(_desc_from_oracle(od))
    y = np.zeros((2, 32, 32), np.float32)
    plan.run_host(x.ctypes.data, f.ctypes.data, y.ctypes.data, 0)
    assert bitwise_equal(y, O.conv(od, x, f))
    # static filter: filter pointer NULL afterwards
    plan.set_static_filter(f.ctypes.data)
    y2 = np.zeros_like(y)
    plan.run_host(x.ctypes.data, 0, y2.ctypes.data, 0)
    assert bitwise_equal(y2, y)
    plan.close()


def test_null_pointers_rejected():
    od = O.make_desc(16, 16, 3, 3)
    plan = _lib.Plan(_desc_from_oracle(od))
    with pytest.raises(_lib.CctError) as e:
        plan.run(0, 0, 0, 0)
    assert e.value.status == _lib.EINVAL
    plan.close()


def test_native_launches_counted():
    before = _lib.launch_count()
    od = O.make_desc(16, 16, 3, 3)
    gpu_conv(od, np.ones((16, 16), np.float32), np.ones((3, 3), np.float32))
    assert _lib.launch_count() == before + 1
