"""Kernel circuits on the device against the FP32 oracle.

A circuit step runs its nodes in order over shared buffers, so every listed
output must equal the oracle's convolutions and numpy's elementwise
operations chained the same way, bit for bit on the FP32 kernels (the direct
and frame kernels follow the reference's summation order; the elementwise
operations are single IEEE operations).  Steps repeat with the same results,
the host step moves inputs and outputs, and a filter can come from a field.
"""
import numpy as np
import pytest
import torch

import oracle as O
from cctconv import _lib
from cctconv import circuit as K

pytestmark = pytest.mark.gpu


def _frame(rows, cols, cin, cout, batch, r=3, relu=False):
    d = _lib.new_desc(image_rows=rows, image_cols=cols, image_planes=batch * cin, filter_rows=r, filter_cols=r,
                      filter_planes=cout * cin, batch_size=batch, vector_mode=_lib.PROJECT_FRAME_BLOCK_REDUCE_SUM,
                      flags=_lib.FLAG_RELU if relu else 0)
    od = O.make_desc(rows, cols, r, r, planes=batch * cin, f_planes=cout * cin, batch=batch, border=O.ZERO,
                     orient=O.CONV, mode=O.PROJECT_REDUCE)
    return d, od


def test_residual_blocks_match_the_oracle():
    rows, cols, c, batch = 32, 32, 8, 2
    d, od = _frame(rows, cols, c, c, batch)
    nodes = [K.conv(0, d), K.relu(1), K.conv(2, d), K.add(3, 0), K.relu(4),
             K.conv(5, d), K.relu(6), K.conv(7, d), K.add(8, 5), K.relu(9)]
    circ = K.Circuit([(rows, cols, batch * c)], nodes, outputs=[5, 10])
    rng = np.random.default_rng(11)
    fs = {i: (rng.standard_normal((c * c, 3, 3)) * 0.2).astype(np.float32) for i in (0, 2, 5, 7)}
    for i, f in fs.items():
        circ.set_filter(i, f)
    n, nbytes = circ.buffers()
    assert n == 5 and nbytes == 5 * rows * cols * batch * c * 4
    x = rng.standard_normal((batch * c, rows, cols)).astype(np.float32)
    y1 = np.zeros_like(x)
    y2 = np.zeros_like(x)
    circ.step_host([x], [y1, y2])

    relu = lambda a: np.maximum(a, np.float32(0))  # noqa: E731
    a = relu(O.conv(od, x, fs[0]))
    b = relu(O.conv(od, a, fs[2]) + x)
    e = relu(O.conv(od, b, fs[5]))
    want = relu(O.conv(od, e, fs[7]) + b)
    assert np.array_equal(y1, b)
    assert np.array_equal(y2, want)

    # the captured step replays with the same results, field views read the outputs
    xd = circ.field(0)
    xd.copy_(torch.from_numpy(x.ravel()).cuda())
    assert circ.step(3) == 4
    torch.cuda.synchronize()
    assert _lib.LIB.cct_device_status() == _lib.OK
    assert np.array_equal(circ.field(10).cpu().numpy().reshape(want.shape), want)
    circ.close()


def test_elementwise_nodes_and_a_filter_from_a_field():
    rows, cols, c, batch = 24, 40, 4, 3
    d, od = _frame(rows, cols, c, 6, batch)
    inputs = [(rows, cols, batch * c), (3, 3, 6 * c), (rows, cols, batch * 6)]
    # a convolution whose filter is input field 1, then elementwise arithmetic
    nodes = [K.conv(0, d, filter_field=1), K.sub(3, 2), K.mul(4, 2), K.scale(5, -0.75), K.relu(6)]
    circ = K.Circuit(inputs, nodes, outputs=[4, 7])
    rng = np.random.default_rng(5)
    x = rng.standard_normal((batch * c, rows, cols)).astype(np.float32)
    f = rng.standard_normal((6 * c, 3, 3)).astype(np.float32)
    z = rng.standard_normal((batch * 6, rows, cols)).astype(np.float32)
    o1 = np.zeros((batch * 6, rows, cols), np.float32)
    o2 = np.zeros_like(o1)
    circ.step_host([x, f, z], [o1, o2])
    conv = O.conv(od, x, f)
    s = conv - z
    m = s * z
    want = np.maximum(m * np.float32(-0.75), np.float32(0))
    assert np.array_equal(o1, s)
    assert np.array_equal(o2, want)
    # a new filter in the input field changes the next step
    f2 = (f * np.float32(0.5)).astype(np.float32)
    circ.step_host([x, f2, z], [o1, o2])
    assert np.array_equal(o1, O.conv(od, x, f2) - z)
    circ.close()


def test_split_precision_nodes_in_a_circuit():
    rows, cols, c, k, batch = 32, 32, 16, 64, 4
    d = _lib.new_desc(image_rows=rows, image_cols=cols, image_planes=batch * c, filter_rows=5, filter_cols=5,
                      filter_planes=k * c, batch_size=batch, orientation=_lib.CROSS_CORRELATION,
                      vector_mode=_lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, precision=_lib.PREC_BF16X3)
    od = O.make_desc(rows, cols, 5, 5, planes=batch * c, f_planes=k * c, batch=batch, border=O.ZERO,
                     orient=O.XCORR, mode=O.PROJECT_REDUCE)
    circ = K.Circuit([(rows, cols, batch * c)], [K.conv(0, d), K.relu(1)], outputs=[2])
    rng = np.random.default_rng(9)
    f = (rng.standard_normal((k * c, 5, 5)) * np.sqrt(2.0 / (c * 25))).astype(np.float32)
    circ.set_filter(0, f)
    x = rng.standard_normal((batch * c, rows, cols)).astype(np.float32)
    y = np.zeros((batch * k, rows, cols), np.float32)
    circ.step_host([x], [y])
    ref = np.maximum(O.conv(od, x, f, np.float64), 0)
    mx, _ = O.rel_errors(y, ref)
    assert mx <= 1e-5
    circ.close()


def test_a_static_filter_node_without_its_filter_is_refused():
    d, _ = _frame(16, 16, 4, 4, 1)
    circ = K.Circuit([(16, 16, 4)], [K.conv(0, d)], outputs=[1])
    with pytest.raises(_lib.CctError) as e:
        circ.step()
    assert "has no filter" in str(e.value)
    circ.close()
