"""The CPU oracle pinned against the reference's own golden vectors and
known-answer tests (no GPU).

Golden vectors: src/test/resources/platform/opencl/hyperkernels/convolutionDynamic/
(25 cases, read by src/test/scala/cogx/DynamicConvolutionSpec.scala:131-203).
Known answers: src/test/scala/cogx/StaticConvolutionSpec.scala:36-236.
"""
import numpy as np
import pytest

import oracle as O
from helpers import (ADJOINT_BORDER, ADJOINT_SAMPLING, golden_case, legal_in_reference,
                     ref_field_approx_equal)


@pytest.mark.parametrize("i", range(25))
def test_golden_forward(golden, i):
    """convolve(x, k, border, sampling) ~== wx, as DynamicConvolutionSpec checks."""
    sampling, step, border, a = golden_case(golden, i)
    x, k, wx = a["x"], a["k"], a["wx"]
    desc = O.make_desc(x.shape[0], x.shape[1], k.shape[0], k.shape[1], border=border,
                       orient=O.CONV, sampling=sampling, step=step)
    if not legal_in_reference(sampling, step, border):
        with pytest.raises(ValueError, match="upsampling with BorderClamp"):
            O.output_shape(desc)
        return
    assert O.output_shape(desc) == (wx.shape[0], wx.shape[1], 1)
    y32 = O.conv(desc, x, k)[0]
    y64 = O.conv(desc, x, k, np.float64)[0]
    assert ref_field_approx_equal(y32, wx)
    # the golden values are float32 roundings of the exact result
    assert np.max(np.abs(y64 - wx)) < 5e-7
    assert O.rel_errors(y32, y64)[0] < 2e-7


@pytest.mark.parametrize("i", range(25))
def test_golden_adjoint(golden, i):
    """wty is the adjoint applied to y: crossCorrelate with the adjoint border
    and the reverse sampling (these files ship with the reference but no test
    of it reads them)."""
    sampling, step, border, a = golden_case(golden, i)
    if border not in ADJOINT_BORDER:
        pytest.skip("BorderClamp has no convolution-form adjoint")
    y, k, wty = a["y"], a["k"], a["wty"]
    desc = O.make_desc(y.shape[0], y.shape[1], k.shape[0], k.shape[1],
                       border=ADJOINT_BORDER[border], orient=O.XCORR,
                       sampling=ADJOINT_SAMPLING[sampling], step=step)
    assert O.output_shape(desc)[:2] == wty.shape
    got = O.conv(desc, y, k, np.float64)[0]
    assert np.max(np.abs(got - wty)) < 5e-7


def _run2d(img, ker, border, orient):
    desc = O.make_desc(img.shape[0], img.shape[1], ker.shape[0], ker.shape[1], border=border,
                       orient=orient)
    return O.conv(desc, img, ker)[0]


KERNEL = np.array([[0.25, 0.50, 0.25], [0.50, 1.00, 0.50], [0.25, 0.50, 0.25]], np.float32)
IMAGE = np.array([[0, 1, 2, 3], [2, 3, 4, 5], [8, 7, 6, 4], [5, 4, 9, 8]], np.float32)


def test_known_answer_1d():
    """StaticConvolutionSpec.scala:62-87 ("scalar convolve scalar, 1D")."""
    img = np.array([[1, 2, 3, 4]], np.float32)
    ker = np.array([[0.25, 0.5, 0.25]], np.float32)
    assert np.allclose(_run2d(img, ker, O.CLAMP, O.CONV), [[1.25, 2.0, 3.0, 3.75]])
    assert np.allclose(_run2d(img, ker, O.CYCLIC, O.CONV), [[2.0, 2.0, 3.0, 3.0]])
    assert np.allclose(_run2d(img, ker, O.ZERO, O.CONV), [[1.0, 2.0, 3.0, 2.75]])


def test_known_answer_2d():
    """StaticConvolutionSpec.scala:89-127 and :182-204."""
    clamp = [[3.0, 6.0, 10.0, 13.0], [12.5, 14.0, 15.75, 16.75],
             [22.5, 22.5, 23.0, 22.0], [22.0, 23.5, 28.25, 29.25]]
    cyclic = [[10.5, 10.5, 15.5, 15.5], [13.75, 14.0, 15.75, 15.50],
              [22.0, 22.5, 23.0, 22.5], [18.75, 19.0, 22.75, 22.5]]
    zero = [[2.25, 5.0, 8.0, 7.5], [9.5, 14.0, 15.75, 12.5],
            [16.75, 22.5, 23.0, 16.75], [12.75, 18.0, 20.75, 16.0]]
    assert np.array_equal(_run2d(IMAGE, KERNEL, O.CLAMP, O.CONV), np.float32(clamp))
    assert np.array_equal(_run2d(IMAGE, KERNEL, O.CYCLIC, O.CONV), np.float32(cyclic))
    assert np.array_equal(_run2d(IMAGE, KERNEL, O.ZERO, O.CONV), np.float32(zero))


def test_known_answer_xcorr():
    """StaticConvolutionSpec.scala:206-236 ("scalar cross-correlate scalar, 2D")."""
    ker = np.float32([[1, 2, 0], [0, 3, 0], [0, 0, 0]])
    want = np.float32([[0, 5, 11, 17], [6, 11, 17, 23], [30, 29, 29, 26], [39, 34, 46, 38]])
    assert np.array_equal(_run2d(IMAGE, ker, O.CLAMP, O.XCORR), want)


@pytest.mark.parametrize("border", [O.ZERO, O.CLAMP, O.CYCLIC])
def test_separable_equals_full(border):
    """DynamicConvolutionSpec.scala:75-109: separable == full 2-D filter."""
    rng = np.random.default_rng(7)
    x = rng.uniform(-1, 1, (10, 10)).astype(np.float32)
    row = np.float32([0.1, 0.3, 0.4, 0.2, 0.0])
    col = np.float32([0.0, 0.5, -0.4, -0.2, -0.1])
    full = np.outer(col, row).astype(np.float32)
    for orient in (O.CONV, O.XCORR):
        sep = O.separable(x, row, col, border, orient)
        ref = _run2d(x, full, border, orient)
        assert np.max(np.abs(sep - ref)) < 1e-5


def test_fft64_matches_direct64():
    rng = np.random.default_rng(3)
    x = rng.uniform(0, 1, (64, 32))
    f = rng.uniform(-1, 1, (7, 5))
    desc = O.make_desc(64, 32, 7, 5, border=O.CYCLIC, orient=O.CONV)
    direct = O.conv(desc, x, f, np.float64)[0]
    assert np.max(np.abs(O.cyclic_conv_fft64(x, f, O.CONV) - direct)) < 1e-12


SHAPE_CASES = [
    # (rows, cols, fr, fc, border, sampling, step) -> (orows, ocols) or error text
    ((64, 64, 5, 5, O.ZERO, O.NOSAMPLE, 1), (64, 64)),
    ((64, 64, 5, 5, O.VALID, O.NOSAMPLE, 1), (60, 60)),
    ((64, 64, 5, 5, O.FULL, O.NOSAMPLE, 1), (68, 68)),
    ((64, 64, 3, 3, O.ZERO, O.DOWN, 2), (32, 32)),
    ((65, 64, 3, 3, O.ZERO, O.DOWN, 2), "divisible by the downsampling step"),
    ((61, 61, 6, 6, O.VALID, O.DOWN, 4), (14, 14)),
    ((10, 12, 3, 3, O.ZERO, O.UP, 3), (30, 36)),
    ((10, 12, 3, 3, O.CLAMP, O.UP, 3), "upsampling with BorderClamp"),
    ((10, 12, 3, 3, O.CLAMP, O.UP, 1), (10, 12)),
    ((10, 12, 4, 3, O.ZERO, O.NOSAMPLE, 1), "odd shape"),
    ((10, 12, 4, 3, O.FULL, O.NOSAMPLE, 1), (13, 14)),
    ((4, 4, 5, 5, O.VALID, O.NOSAMPLE, 1), "larger than the input"),
]


@pytest.mark.parametrize("args,want", SHAPE_CASES)
def test_output_shape_rules(args, want):
    rows, cols, fr, fc, border, sampling, step = args
    desc = O.make_desc(rows, cols, fr, fc, border=border, sampling=sampling, step=step)
    if isinstance(want, str):
        with pytest.raises(ValueError, match=want):
            O.output_shape(desc)
    else:
        assert O.output_shape(desc)[:2] == want


def test_frame_plane_counts():
    # projectFrame: B*F planes; fused: B*K; backProjectFrame: B*F; fused: B*L
    d = O.make_desc(8, 8, 3, 3, planes=16 * 32, f_planes=64 * 32, batch=16, mode=O.PROJECT)
    assert O.output_shape(d)[2] == 16 * 64 * 32
    d.mode = O.PROJECT_REDUCE
    assert O.output_shape(d)[2] == 16 * 64
    d = O.make_desc(8, 8, 3, 3, planes=16 * 64, f_planes=64 * 32, batch=16, mode=O.BACKPROJECT_REDUCE)
    assert O.output_shape(d)[2] == 16 * 32
    d = O.make_desc(8, 8, 3, 3, planes=30, f_planes=64, batch=16, mode=O.PROJECT)
    with pytest.raises(ValueError, match="multiple of the batch"):
        O.output_shape(d)
    d = O.make_desc(8, 8, 3, 3, planes=3, f_planes=4, mode=O.PLANE)
    with pytest.raises(ValueError, match="plane-by-plane"):
        O.output_shape(d)


def _plane_xcorr64(x, f, border=O.ZERO, orient=O.XCORR):
    return O.conv(O.make_desc(x.shape[0], x.shape[1], f.shape[0], f.shape[1], border=border,
                              orient=orient), x, f, np.float64)[0]


def test_frame_semantics_by_composition():
    """projectFrame / backProjectFrame index semantics pinned by plane-wise
    compositions, as StaticConvolutionSpec.scala:536-584 and :1653-1905 do."""
    rng = np.random.default_rng(11)
    B, N, K, H, W, R = 2, 3, 4, 9, 7, 3
    x = rng.normal(size=(B * N, H, W))
    f = rng.normal(size=(K * N, R, R))
    # projectFrame
    d = O.make_desc(H, W, R, R, planes=B * N, f_planes=K * N, batch=B, orient=O.XCORR, mode=O.PROJECT)
    y = O.conv(d, x, f, np.float64)
    for b in range(B):
        for p in range(K * N):
            assert np.allclose(y[b * K * N + p], _plane_xcorr64(x[b * N + p % N], f[p]))
    # fused projectFrame
    d.mode = O.PROJECT_REDUCE
    y = O.conv(d, x, f, np.float64)
    for b in range(B):
        for k in range(K):
            ref = sum(_plane_xcorr64(x[b * N + c], f[k * N + c]) for c in range(N))
            assert np.allclose(y[b * K + k], ref)
    # backProjectFrame: image planes N per image, L = F / N logical filters
    d = O.make_desc(H, W, R, R, planes=B * N, f_planes=K * N, batch=B, orient=O.CONV, mode=O.BACKPROJECT)
    y = O.conv(d, x, f, np.float64)
    L = K
    for b in range(B):
        for w in range(K * N):
            ref = _plane_xcorr64(x[b * N + w % N], f[L * (w % N) + w // N], orient=O.CONV)
            assert np.allclose(y[b * K * N + w], ref)
    d.mode = O.BACKPROJECT_REDUCE
    y = O.conv(d, x, f, np.float64)
    for b in range(B):
        for l in range(L):
            ref = sum(_plane_xcorr64(x[b * N + n], f[n * L + l], orient=O.CONV) for n in range(N))
            assert np.allclose(y[b * L + l], ref)


def test_fused_backproject_is_adjoint_of_projectframe():
    """<projectFrame(x), g> == <x, backProjectFrame(g)> for BorderZero."""
    rng = np.random.default_rng(5)
    B, C, K, H, W, R = 2, 3, 5, 8, 6, 5
    x = rng.normal(size=(B * C, H, W))
    g = rng.normal(size=(B * K, H, W))
    f = rng.normal(size=(K * C, R, R))
    fwd = O.conv(O.make_desc(H, W, R, R, planes=B * C, f_planes=K * C, batch=B, orient=O.XCORR,
                             mode=O.PROJECT_REDUCE), x, f, np.float64)
    bwd = O.conv(O.make_desc(H, W, R, R, planes=B * K, f_planes=K * C, batch=B, orient=O.CONV,
                             mode=O.BACKPROJECT_REDUCE), g, f, np.float64)
    assert abs(np.sum(fwd * g) - np.sum(x * bwd)) < 1e-9 * np.sum(np.abs(fwd * g))


def test_poor_float_semantics():
    assert O.poor_float_equal([1.0, 0.0], [1.0 + 1e-4, 1e-3])
    assert not O.poor_float_equal([1.0], [1.01])


# ---------------------------------------------------------------- FilterAdjoint
def _fa(x, g, border=O.VALID, orient=O.CONV, sampling=O.NOSAMPLE, step=1, batch=1,
        mode=O.FILTER_ADJOINT, dtype=np.float32, planes=None, g_planes=None):
    x = np.asarray(x, dtype)
    g = np.asarray(g, dtype)
    rows, cols = x.shape[-2:]
    d = O.make_desc(rows, cols, g.shape[-2], g.shape[-1],
                    planes=x.shape[0] if planes is None else planes,
                    f_planes=g.shape[0] if g_planes is None else g_planes,
                    batch=batch, border=border, orient=orient, sampling=sampling, step=step, mode=mode)
    return O.conv(d, x, g, dtype)


@pytest.mark.parametrize("n_in,f_size,down", [(1 + 15, 16, 1), (5 + 15, 16, 1), (9 + 15, 16, 1),
                                              (137, 128, 1), (27, 16, 2), (32, 24, 3)])
def test_filter_adjoint_constant_known_answers(n_in, f_size, down):
    """StaticConvolutionSpec.scala:992-1037: a constant 0.5 field and an all-ones
    gradient give f_size^2 * 0.5 at every output."""
    x = np.full((n_in, n_in), 0.5, np.float32)
    g = np.ones((f_size, f_size), np.float32)
    y = _fa(x[None], g[None], sampling=O.DOWN if down > 1 else O.NOSAMPLE, step=down,
            planes=0, g_planes=0)
    out = (n_in - f_size + 1) // down
    assert y.shape[-2:] == (out, out)
    assert np.all(y == f_size * f_size * 0.5)


@pytest.mark.parametrize("orient", [O.CONV, O.XCORR])
@pytest.mark.parametrize("n_in,f_size,up", [(137, 64, 2), (35, 10, 3), (210, 50, 4)])
def test_filter_adjoint_upsampled_gradient_known_answers(orient, n_in, f_size, up):
    """StaticConvolutionSpec.scala:1039-1147: UpsampleInput upsamples the
    gradient; output side n - f*up + 1."""
    x = np.full((n_in, n_in), 0.5, np.float32)
    g = np.ones((f_size, f_size), np.float32)
    y = _fa(x[None], g[None], orient=orient, sampling=O.UP, step=up, planes=0, g_planes=0)
    out = n_in - f_size * up + 1
    assert y.shape[-2:] == (out, out)
    assert np.all(y == f_size * f_size * 0.5)


@pytest.mark.parametrize("orient", [O.CONV, O.XCORR])
def test_filter_adjoint_upsampled_sparse_input(orient):
    """StaticConvolutionSpec.scala:1075-1097 / 1124-1146 (360, 50, 7)."""
    n_in, f_size, up = 360, 50, 7
    x = np.zeros((n_in, n_in), np.float32)
    x[:up, :up] = 0.5
    g = np.ones((f_size, f_size), np.float32)
    y = _fa(x[None], g[None], orient=orient, sampling=O.UP, step=up, planes=0, g_planes=0).reshape(
        n_in - f_size * up + 1, -1)
    want = np.zeros_like(y)
    if orient == O.CONV:
        want[0, 0] = 0.5
    else:
        want[:up, :up] = 0.5
    assert np.array_equal(y, want)


@pytest.mark.parametrize("n", [2, 3, 5])
def test_filter_adjoint_upsample_flip_order(n):
    """StaticConvolutionSpec.scala:1152-1189: a 1x1 gradient upsampled by the
    field size reads the first element (cross-correlation) or the last
    (convolution)."""
    x = (n * np.arange(n)[:, None] + np.arange(n)[None, :] + 1).astype(np.float32)
    g = np.ones((1, 1), np.float32)
    yc = _fa(x[None], g[None], orient=O.CONV, sampling=O.UP, step=n, planes=0, g_planes=0)
    yx = _fa(x[None], g[None], orient=O.XCORR, sampling=O.UP, step=n, planes=0, g_planes=0)
    assert yc.ravel().tolist() == [n * n] and yx.ravel().tolist() == [1.0]


@pytest.mark.parametrize("C,L,rows,cols,out,batch", [(3, 4, 71, 23, 7, 1), (2, 2, 19, 17, 7, 1),
                                                     (1, 4, 31, 23, 12, 1), (6, 1, 23, 29, 7, 1),
                                                     (2, 3, 63, 67, 17, 2), (3, 4, 15, 27, 5, 3),
                                                     (1, 4, 15, 27, 5, 7), (6, 1, 15, 27, 5, 8)])
def test_filter_adjoint_plane_mixing_by_composition(C, L, rows, cols, out, batch):
    """StaticConvolutionSpec.scala:1950-2050: output plane i (b = i % B,
    w = i / B) is crossCorrelate(image[b*C + w%C], grad[b*L + w/C], BorderValid);
    the block-reduced form sums the B images of w in order."""
    rng = np.random.default_rng(C * 100 + L)
    kr, kc = rows - out + 1, cols - out + 1
    x = rng.uniform(-1, 1, (batch * C, rows, cols)).astype(np.float32)
    g = rng.uniform(-1, 1, (batch * L, kr, kc)).astype(np.float32)
    y = _fa(x, g, orient=O.XCORR, batch=batch).reshape(C * L * batch, out, -1)
    for i in range(C * L * batch):
        b, w = i % batch, i // batch
        want = _fa(x[b * C + w % C][None], g[b * L + w // C][None], orient=O.XCORR, planes=0,
                   g_planes=0, mode=O.PLANE)
        assert np.array_equal(y[i], want.reshape(y[i].shape)), i
    y64 = _fa(x, g, orient=O.XCORR, batch=batch, dtype=np.float64).reshape(C * L * batch, out, -1)
    r64 = _fa(x, g, orient=O.XCORR, batch=batch, dtype=np.float64,
              mode=O.FILTER_ADJOINT_REDUCE).reshape(C * L, out, -1)
    for w in range(C * L):
        acc = np.zeros_like(r64[w])
        for b in range(batch):
            acc = acc + y64[w * batch + b]
        assert np.array_equal(acc, r64[w])


def test_filter_adjoint_shape_rules():
    def shape(mode, planes, f_planes, batch, sampling=O.NOSAMPLE, step=1):
        return O.output_shape(O.make_desc(40, 40, 8, 8, planes=planes, f_planes=f_planes, batch=batch,
                                          border=O.VALID, orient=O.XCORR, sampling=sampling,
                                          step=step, mode=mode))
    assert shape(O.FILTER_ADJOINT, 6, 8, 2) == (33, 33, 3 * 4 * 2)
    assert shape(O.FILTER_ADJOINT_REDUCE, 6, 8, 2) == (33, 33, 12)
    assert shape(O.FILTER_ADJOINT, 6, 8, 2, O.UP, 2) == (40 - 16 + 1, 25, 24)
    with pytest.raises(ValueError):
        shape(O.FILTER_ADJOINT, 6, 7, 2)


# ---- ScalarMatrixConvolve2D and colour fields -----------------------------

def _np_border(border, v, n):
    if border == O.CLAMP:
        return min(max(v, 0), n - 1)
    if border == O.CYCLIC:
        return v % n
    return v if 0 <= v < n else -1


@pytest.mark.parametrize("border", [O.ZERO, O.CLAMP, O.CYCLIC])
def test_scalar_matrix_oracle_restates_the_kernel_loop(border):
    """One fma chain per output over the taps in row-major order
    (ScalarMatrixConvolve2DHyperKernel.scala:59-85), output plane
    row * matrix_cols + col; checked against a float32 loop written here."""
    rng = np.random.default_rng(31)
    rows, cols, size, mr, mc = 6, 7, 3, 2, 3
    x = rng.uniform(-1, 1, (rows, cols)).astype(np.float32)
    mats = rng.uniform(-1, 1, (size, size, mr, mc)).astype(np.float32)
    y = O.scalar_matrix(x, mats, border)
    h = size // 2
    for p in range(mr * mc):
        for i in range(rows):
            for j in range(cols):
                s = np.float32(0)
                for r in range(size):
                    for c in range(size):
                        si, sj = _np_border(border, i - h + r, rows), _np_border(border, j - h + c, cols)
                        v = np.float32(0) if si < 0 or sj < 0 else x[si, sj]
                        # fma in float64 is exact for a float32 product, then one rounding
                        s = np.float32(np.float64(v) * np.float64(mats[r, c, p // mc, p % mc]) + np.float64(s))
                assert y[p, i, j] == s, (p, i, j)


def test_scalar_matrix_matches_reference_test_by_convolve_of_flipped_matrices():
    """StaticConvolutionSpec.scala:2361-2393: crossCorrelate(scalar, matrixField,
    BorderClamp) ~== the vector field of convolve(scalar, matrix.flip,
    BorderClamp), row-major over the matrix field (4x5 field, 2x3 matrices of
    3x3)."""
    rng = np.random.default_rng(32)
    x = rng.random((4, 5)).astype(np.float32)
    mats = rng.random((3, 3, 2, 3)).astype(np.float32)
    y = O.scalar_matrix(x, mats, O.CLAMP)
    expected = np.stack([O.conv(O.make_desc(4, 5, 3, 3, border=O.CLAMP, orient=O.CONV), x,
                                np.ascontiguousarray(mats[::-1, ::-1, r, c]))[0]
                         for r in range(2) for c in range(3)])
    assert ref_field_approx_equal(y, expected)


def test_color_conversions_known_answers():
    """UNORM_INT8 read: byte / 255; MergeColorPlanes write:
    convert_uchar_sat_rte(v * 255) with alpha 255."""
    rgba = np.array([[[0, 1, 128, 7], [254, 255, 51, 0]]], dtype=np.uint8)
    planes = O.color_unpack(rgba)
    assert planes.shape == (3, 1, 2)
    for k in range(3):
        for j in range(2):
            assert planes[k, 0, j] == np.float32(rgba[0, j, k]) / np.float32(255)
    back = O.color_pack(planes)
    assert np.array_equal(back[..., :3], rgba[..., :3]) and np.all(back[..., 3] == 255)
    v = np.array([np.nan, -0.5, 0.0, 2.5 / 255, 3.5 / 255, 0.999, 1.0, 7.0], dtype=np.float32)
    got = O.color_pack(np.stack([v[None, :]] * 3))[0, :, 0]
    want = []
    for f in v:
        s = np.float32(f) * np.float32(255)
        s = 0.0 if not s > 0 else min(float(s), 255.0)
        want.append(int(np.rint(s)))  # numpy rounds half to even
    assert list(got) == want
    assert list(got[:3]) == [0, 0, 0] and got[-1] == 255


def test_color_conv_is_three_plane_convs():
    rng = np.random.default_rng(33)
    rgba = rng.integers(0, 256, (9, 11, 4), dtype=np.uint8)
    f = rng.uniform(-0.3, 0.3, (3, 3)).astype(np.float32)
    d = O.make_desc(9, 11, 3, 3, border=O.CYCLIC, orient=O.CONV)
    out = O.color_conv(d, rgba, f)
    planes = O.color_unpack(rgba)
    for k in range(3):
        yk = O.conv(d, planes[k], f)[0]
        assert np.array_equal(out[..., k], O.color_pack(np.stack([yk] * 3))[..., 0])
    assert np.all(out[..., 3] == 255)
