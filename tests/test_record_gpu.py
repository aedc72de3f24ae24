"""Checkpoint records on the GPU: a plan or graph saved to a record and
restored computes the same bits as the original, keeps its constant filters
and (for a graph) its step count, and saves back to the same record."""
import numpy as np
import pytest
import torch

import cctconv as C
from cctconv import _lib

pytestmark = pytest.mark.gpu


def _run(plan, x, f=None):
    orows, ocols, oplanes = plan.shape
    y = torch.full((max(oplanes, 1), orows, ocols), float("nan"), device="cuda")
    plan.run(x.data_ptr(), 0 if f is None else f.data_ptr(), y.data_ptr(),
             torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert _lib.LIB.cct_device_status() == _lib.OK
    return y.cpu().numpy()


CASES = [
    # (field shape, filter shape, border, orientation, sampling, mode, batch, precision, algo)
    ((64, 64, 0), (5, 5, 0), C.BorderZero, _lib.CONVOLUTION, C.NoSamplingConvolution, _lib.PLANE_BY_PLANE, 1,
     _lib.PREC_FP32, _lib.ALGO_DIRECT),
    ((256, 256, 0), (31, 31, 0), C.BorderCyclic, _lib.CONVOLUTION, C.NoSamplingConvolution,
     _lib.PLANE_BY_PLANE, 1, _lib.PREC_FP32, _lib.ALGO_FFT),
    ((32, 32, 2 * 16), (3, 3, 24 * 16), C.BorderZero, _lib.CROSS_CORRELATION, C.DownsampleOutputConvolution(2),
     _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, 2, _lib.PREC_BF16X3, _lib.ALGO_AUTO),
    ((20, 20, 2 * 8), (3, 3, 8 * 4), C.BorderClamp, _lib.CONVOLUTION, C.NoSamplingConvolution,
     _lib.BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM, 2, _lib.PREC_FP32, _lib.ALGO_AUTO),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_plan_record_round_trip(case):
    fs, ks, border, orient, samp, mode, batch, prec, algo = CASES[case]
    desc = C.make_desc(fs, ks, border, orient, samp, mode, batch, prec, algo)
    rng = np.random.default_rng(case)
    x = torch.from_numpy(rng.standard_normal((max(fs[2], 1), fs[0], fs[1])).astype(np.float32)).cuda()
    f = rng.standard_normal((max(ks[2], 1), ks[0], ks[1])).astype(np.float32)
    plan = _lib.Plan(desc)
    plan.set_static_filter(f.ctypes.data)
    want = _run(plan, x)
    rec = plan.save()
    kind, descs, t = _lib.describe_record(rec)
    assert kind == 1 and t == 0 and descs[0].key() == desc.key()
    plan.close()
    back = _lib.Plan.restore(rec)
    assert back.algo == _lib.Plan(desc).algo
    assert np.array_equal(_run(back, x), want)  # the constant filter came back too
    assert np.array_equal(back.save(), rec)
    back.close()


def test_plan_record_without_constant_filter():
    desc = C.make_desc((40, 40, 0), (3, 3, 0), C.BorderCyclic, _lib.CROSS_CORRELATION,
                       C.NoSamplingConvolution, _lib.PLANE_BY_PLANE)
    plan = _lib.Plan(desc)
    rec = plan.save()
    assert rec.size == 6 + 1 + 15 + 2 + 1  # header, one layer without filter values, checksum
    back = _lib.Plan.restore(rec)
    x = torch.randn((1, 40, 40), device="cuda")
    f = torch.randn((1, 3, 3), device="cuda")
    assert np.array_equal(_run(back, x, f), _run(plan, x, f))


def test_graph_record_round_trip():
    """A three-layer stack (BF16X3 frame layers with ReLU and a downsample)
    stepped twice, saved, restored: same step count, same output for the
    same input."""
    B, H = 2, 32
    layers = [(3, 16, 1), (16, 16, 2), (16, 32, 1)]  # (C, K, down)
    descs, rng = [], np.random.default_rng(3)
    h = H
    for c, k, down in layers:
        samp = C.DownsampleOutputConvolution(down) if down > 1 else C.NoSamplingConvolution
        descs.append(C.make_desc((h, h, B * c), (3, 3, k * c), C.BorderZero, _lib.CROSS_CORRELATION, samp,
                                 _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, B, _lib.PREC_BF16X3,
                                 flags=_lib.FLAG_RELU))
        h //= down
    g = _lib.Graph(descs)
    filters = [(rng.standard_normal((k * c, 3, 3)) * 0.2).astype(np.float32) for c, k, _ in layers]
    for i, f in enumerate(filters):
        g.set_filter(i + 1, f.ctypes.data)
    x = rng.standard_normal((B * 3, H, H)).astype(np.float32)
    out_elems = B * 32 * (H // 2) ** 2
    y1 = np.zeros(out_elems, np.float32)
    g.step_host(x.ctypes.data, y1.ctypes.data)
    g.step_host(x.ctypes.data, y1.ctypes.data)
    assert g.time == 2
    rec = g.save()
    kind, rdescs, t = _lib.describe_record(rec)
    assert kind == 2 and t == 2 and [d.key() for d in rdescs] == [d.key() for d in descs]
    g.close()
    back = _lib.Graph.restore(rec)
    assert back.time == 2
    y2 = np.zeros(out_elems, np.float32)
    back.step_host(x.ctypes.data, y2.ctypes.data)
    assert back.time == 3
    assert np.array_equal(y1, y2)
    back.reset()
    assert back.time == 0
    back.close()


def test_restore_rejects_a_plan_record_as_graph():
    plan = _lib.Plan(C.make_desc((16, 16, 0), (3, 3, 0), C.BorderZero, _lib.CONVOLUTION,
                                 C.NoSamplingConvolution, _lib.PLANE_BY_PLANE))
    rec = plan.save()
    with pytest.raises(_lib.CctError, match="plan, not a graph"):
        _lib.Graph.restore(rec)
