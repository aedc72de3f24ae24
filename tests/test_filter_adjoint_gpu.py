"""FilterAdjoint (weight-gradient plane mixing) on the GPU against the FP32
oracle, bit for bit, and through the reference-named API."""
import numpy as np
import pytest
import torch

import cctconv as C
import oracle as O
from cctconv import _lib

pytestmark = pytest.mark.gpu

CASES = [
    # planes per image C, gradient planes per image L, image rows, cols, gradient rows, cols, batch,
    # border, sampling, step
    (3, 4, 71, 23, 65, 17, 1, O.VALID, O.NOSAMPLE, 1),
    (2, 3, 63, 67, 47, 51, 2, O.VALID, O.NOSAMPLE, 1),
    (3, 4, 15, 27, 11, 23, 3, O.VALID, O.NOSAMPLE, 1),
    (1, 4, 15, 27, 11, 23, 7, O.VALID, O.NOSAMPLE, 1),
    (4, 2, 36, 36, 16, 16, 2, O.VALID, O.UP, 2),
    (2, 2, 35, 35, 10, 10, 1, O.VALID, O.UP, 3),
    (2, 3, 27, 27, 16, 16, 2, O.VALID, O.DOWN, 2),
    (2, 2, 20, 24, 5, 7, 2, O.ZERO, O.NOSAMPLE, 1),
    (2, 2, 20, 24, 5, 5, 2, O.FULL, O.NOSAMPLE, 1),
    (32, 64, 68, 68, 64, 64, 2, O.VALID, O.NOSAMPLE, 1),  # a 5x5 filter gradient of a 64x64 layer
]


def _run(desc, x, g):
    plan = _lib.Plan(desc)
    orows, ocols, oplanes = plan.shape
    y = torch.full((max(oplanes, 1), orows, ocols), float("nan"), device="cuda")
    xd, gd = torch.from_numpy(x).cuda(), torch.from_numpy(g).cuda()  # kept alive across the run
    plan.run(xd.data_ptr(), gd.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    plan.close()
    return y.cpu().numpy()


@pytest.mark.parametrize("mode", [O.FILTER_ADJOINT, O.FILTER_ADJOINT_REDUCE], ids=["fa", "fa_reduce"])
@pytest.mark.parametrize("orient", [O.XCORR, O.CONV], ids=["xcorr", "conv"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(map(str, c)))
def test_filter_adjoint_matches_oracle_bitwise(case, orient, mode):
    Cn, L, rows, cols, gr, gc, batch, border, sampling, step = case
    rng = np.random.default_rng(rows * 31 + gr)
    x = rng.uniform(-1, 1, (batch * Cn, rows, cols)).astype(np.float32)
    g = rng.uniform(-1, 1, (batch * L, gr, gc)).astype(np.float32)
    desc = _lib.new_desc(image_rows=rows, image_cols=cols, image_planes=batch * Cn, filter_rows=gr,
                         filter_cols=gc, filter_planes=batch * L, batch_size=batch, border=border,
                         orientation=orient, sampling=sampling, step=step,
                         vector_mode=_lib.FILTER_ADJOINT if mode == O.FILTER_ADJOINT
                         else _lib.FILTER_ADJOINT_BLOCK_REDUCE_SUM)
    y = _run(desc, x, g)
    od = O.make_desc(rows, cols, gr, gc, planes=batch * Cn, f_planes=batch * L, batch=batch,
                     border=border, orient=orient, sampling=sampling, step=step, mode=mode)
    ref = O.conv(od, x, g, np.float32)
    assert y.size == ref.size
    assert np.array_equal(y.reshape(ref.shape).view(np.uint32), ref.view(np.uint32))


def test_filter_adjoint_api_and_scalar_result():
    """crossCorrelateFilterAdjoint of two ScalarFields is a ScalarField; the
    vector form follows the reference's plane order."""
    rng = np.random.default_rng(1)
    x = torch.from_numpy(rng.uniform(-1, 1, (40, 40)).astype(np.float32)).cuda()
    g = torch.from_numpy(rng.uniform(-1, 1, (36, 36)).astype(np.float32)).cuda()
    y = C.crossCorrelateFilterAdjoint(x, g, C.BorderValid)
    assert y.shape == (5, 5)
    yc = C.convolveFilterAdjoint(x, g, C.BorderValid, C.UpsampleInputConvolution(1))
    assert yc.shape == (5, 5)
    xv = torch.from_numpy(rng.uniform(-1, 1, (2 * 3, 20, 20)).astype(np.float32)).cuda()
    gv = torch.from_numpy(rng.uniform(-1, 1, (2 * 4, 16, 16)).astype(np.float32)).cuda()
    fa = C.crossCorrelateFilterAdjoint(xv, gv, C.BorderValid, batchSize=2)
    red = C.filterAdjointBlockReduceSum(xv, gv, C.BorderValid, batchSize=2)
    assert fa.shape == (3 * 4 * 2, 5, 5) and red.shape == (12, 5, 5)
    torch.cuda.synchronize()
    # plane B*w + b of the unreduced form, summed over b in order, is the reduced form
    acc = fa[0::2] + fa[1::2]
    assert torch.equal(acc, red)
    with pytest.raises(ValueError, match="multiple of the batchSize"):
        C.crossCorrelateFilterAdjoint(xv, gv[:7], C.BorderValid, batchSize=2)


def test_small_results_take_the_filter_adjoint_kernel():
    """BorderValid, unsampled, results up to 8 wide run on the dedicated
    FilterAdjoint kernel; up-sampled gradients stay on the generic kernel."""
    def algo(sampling, step, out):
        d = _lib.new_desc(image_rows=64 + out - 1, image_cols=64 + out - 1, image_planes=2 * 32,
                          filter_rows=64, filter_cols=64, filter_planes=2 * 64, batch_size=2,
                          border=_lib.BORDER_VALID, orientation=_lib.CROSS_CORRELATION,
                          sampling=sampling, step=step, vector_mode=_lib.FILTER_ADJOINT_BLOCK_REDUCE_SUM)
        p = _lib.Plan(d)
        a = p.algo
        p.close()
        return a
    assert algo(_lib.SAMPLE_NONE, 1, 5) == _lib.PLAN_FILTER_ADJOINT
    assert algo(_lib.SAMPLE_NONE, 1, 9) == _lib.PLAN_DIRECT


def test_filter_adjoint_weight_gradient_timing():
    """The weight gradient of the B=16, C=32, K=64, 64x64, 5x5 layer: image
    padded to 68x68, gradient 64x64, 2048 result planes of 5x5."""
    B, Cn, K = 16, 32, 64
    rng = np.random.default_rng(7)
    x = torch.from_numpy(rng.standard_normal((B * Cn, 68, 68)).astype(np.float32)).cuda()
    g = torch.from_numpy(rng.standard_normal((B * K, 64, 64)).astype(np.float32)).cuda()
    d = _lib.new_desc(image_rows=68, image_cols=68, image_planes=B * Cn, filter_rows=64, filter_cols=64,
                      filter_planes=B * K, batch_size=B, border=_lib.BORDER_VALID,
                      orientation=_lib.CROSS_CORRELATION, vector_mode=_lib.FILTER_ADJOINT_BLOCK_REDUCE_SUM)
    plan = _lib.Plan(d)
    assert plan.algo == _lib.PLAN_FILTER_ADJOINT
    y = torch.empty((Cn * K, 5, 5), device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    for _ in range(3):
        plan.run(x.data_ptr(), g.data_ptr(), y.data_ptr(), st)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(10):
        plan.run(x.data_ptr(), g.data_ptr(), y.data_ptr(), st)
    b.record()
    b.synchronize()
    ms = a.elapsed_time(b) / 10
    print(f"weight gradient B=16 C=32 K=64 64x64 5x5: {ms:.3f} ms, "
          f"{2 * B * Cn * K * 64 * 64 * 25 / ms / 1e9:.1f} GFLOP/s")
    # spot-check planes against the oracle
    od = O.make_desc(68, 68, 64, 64, planes=B * Cn, f_planes=B * K, batch=B, border=O.VALID,
                     orient=O.XCORR, mode=O.FILTER_ADJOINT_REDUCE)
    ref = O.conv(od, x.cpu().numpy(), g.cpu().numpy(), np.float32).reshape(Cn * K, 5, 5)
    got = y.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    plan.close()


TC_CASES = [
    # C, L, image rows, cols, gradient rows, cols, batch (BorderValid, no sampling)
    (32, 64, 68, 68, 64, 64, 4),    # the 5x5 weight gradient of a 64x64 layer (M = 800: 7 row tiles)
    (3, 4, 71, 23, 65, 17, 2),      # gradient width not a multiple of 16, L below 16
    (5, 72, 20, 21, 16, 17, 3),     # L = 72: two column blocks; 4x5 results
    (1, 16, 9, 9, 1, 1, 5),         # 1x1 gradient: one pixel per chunk
    (7, 24, 40, 33, 33, 31, 1),     # one image, 8x3 results
    # gradient-planes form (image and gradient widths multiples of 4)
    (16, 40, 36, 40, 32, 36, 3),    # 5x5 results, a ragged 16-column gradient block
    (70, 20, 13, 16, 9, 12, 2),     # three 32-plane blocks of the image
    (8, 100, 20, 24, 16, 20, 2),    # two 64-plane gradient blocks
    (12, 6, 6, 16, 6, 16, 2),       # a 1x1 result
    (9, 4, 7, 20, 5, 16, 1),        # 3x5 results, fewer chunks than splits
]


@pytest.mark.parametrize("orient", [O.XCORR, O.CONV], ids=["xcorr", "conv"])
@pytest.mark.parametrize("case", TC_CASES, ids=lambda c: "-".join(map(str, c)))
def test_filter_adjoint_reduce_tensor_cores(case, orient):
    """FilterAdjointBlockReduceSum in split BF16 on the tensor cores: normwise
    max error <= 1e-5 against the FP64 oracle (RMS reported), and the same
    bits on a second run (the split partial sums are added in split order)."""
    Cn, L, rows, cols, gr, gc, batch = case
    rng = np.random.default_rng(rows * 7 + gc)
    x = rng.standard_normal((batch * Cn, rows, cols)).astype(np.float32)
    g = rng.standard_normal((batch * L, gr, gc)).astype(np.float32)
    desc = _lib.new_desc(image_rows=rows, image_cols=cols, image_planes=batch * Cn, filter_rows=gr,
                         filter_cols=gc, filter_planes=batch * L, batch_size=batch, border=_lib.BORDER_VALID,
                         orientation=orient, vector_mode=_lib.FILTER_ADJOINT_BLOCK_REDUCE_SUM,
                         precision=_lib.PREC_BF16X3)
    plan = _lib.Plan(desc)
    assert plan.algo == _lib.PLAN_FILTER_ADJOINT_BF16X3
    plan.close()
    y1 = _run(desc, x, g)
    assert _lib.LIB.cct_device_status() == _lib.OK
    y2 = _run(desc, x, g)
    od = O.make_desc(rows, cols, gr, gc, planes=batch * Cn, f_planes=batch * L, batch=batch,
                     border=O.VALID, orient=orient, mode=O.FILTER_ADJOINT_REDUCE)
    ref = O.conv(od, x, g, np.float64)
    mx, rms = O.rel_errors(y1.reshape(ref.shape), ref)
    assert mx <= 1e-5, (mx, rms)
    assert np.array_equal(y1, y2)


def test_filter_adjoint_tensor_cores_through_the_api():
    rng = np.random.default_rng(3)
    x = torch.from_numpy(rng.standard_normal((2 * 4, 12, 12)).astype(np.float32)).cuda()
    g = torch.from_numpy(rng.standard_normal((2 * 8, 10, 10)).astype(np.float32)).cuda()
    y = C.filterAdjointBlockReduceSum(x, g, C.BorderValid, batchSize=2, precision=_lib.PREC_BF16X3)
    ref = C.filterAdjointBlockReduceSum(x, g, C.BorderValid, batchSize=2)
    torch.cuda.synchronize()
    assert y.shape == ref.shape == (32, 3, 3)
    assert O.rel_errors(y.cpu().numpy(), ref.cpu().numpy().astype(np.float64))[0] <= 1e-5
