"""ctypes front end of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, as the checker.  The product path
(``cctconv`` and ``libcctconv.so``) never touches it.

The C restatement lives in ``conv_oracle.c``; the FP64 FFT helper below is
the float64 stand-in for the reference's host FFT of static filters
(commons-math3 3.6.1 ``FastFourierTransformer``, used from
``generator/DynamicConvolutionGenerator.scala:342-350``), restated with
numpy's FFT: a cyclic convolution computed in float64 is exact to ~1e-15, so
any float64 FFT is an adequate reference for it.
"""
import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = None

ZERO, CLAMP, CYCLIC, VALID, FULL = range(5)
XCORR, CONV = 0, 1
NOSAMPLE, DOWN, UP = 0, 1, 2
PLANE, PROJECT, PROJECT_REDUCE, BACKPROJECT, BACKPROJECT_REDUCE, FILTER_ADJOINT, FILTER_ADJOINT_REDUCE = range(7)


class OracleDesc(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "rows", "cols", "planes", "f_rows", "f_cols", "f_planes", "batch",
        "border", "orient", "sampling", "step", "mode")]


def build():
    """Compile liboracle.so (gcc only)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = _HERE / "liboracle.so"
        if not path.exists():
            build()
        L = ctypes.CDLL(str(path))
        P = ctypes.POINTER
        L.oracle_output_shape.argtypes = [P(OracleDesc), P(ctypes.c_int), P(ctypes.c_int),
                                          P(ctypes.c_int), ctypes.c_char_p, ctypes.c_int]
        for name, ct in (("oracle_conv_f32", ctypes.c_float), ("oracle_conv_f64", ctypes.c_double)):
            fn = getattr(L, name)
            fn.argtypes = [P(OracleDesc), P(ct), P(ct), P(ct), ctypes.c_int]
        L.oracle_separable_f32.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           P(ctypes.c_float), P(ctypes.c_float), ctypes.c_int,
                                           P(ctypes.c_float), ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, P(ctypes.c_float)]
        L.oracle_scalar_matrix_f32.argtypes = [ctypes.c_int, ctypes.c_int, P(ctypes.c_float),
                                               P(ctypes.c_float), ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_int, P(ctypes.c_float)]
        L.oracle_color_unpack.argtypes = [ctypes.c_int, P(ctypes.c_ubyte), P(ctypes.c_float)]
        L.oracle_color_pack.argtypes = [ctypes.c_int, P(ctypes.c_float), P(ctypes.c_ubyte)]
        _LIB = L
    return _LIB


def make_desc(rows, cols, f_rows, f_cols, planes=0, f_planes=0, batch=1,
              border=ZERO, orient=CONV, sampling=NOSAMPLE, step=1, mode=PLANE):
    return OracleDesc(rows, cols, planes, f_rows, f_cols, f_planes, batch,
                      border, orient, sampling, step, mode)


def output_shape(desc):
    r, c, p = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    err = ctypes.create_string_buffer(256)
    rc = lib().oracle_output_shape(ctypes.byref(desc), ctypes.byref(r), ctypes.byref(c),
                                   ctypes.byref(p), err, 256)
    if rc:
        raise ValueError(err.value.decode())
    return r.value, c.value, p.value


def conv(desc, x, f, dtype=np.float32, threads=0):
    """Run the oracle; x and f are arrays of planes (any shape, C order)."""
    orows, ocols, oplanes = output_shape(desc)
    ct = ctypes.c_float if dtype == np.float32 else ctypes.c_double
    x = np.ascontiguousarray(x, dtype=dtype)
    f = np.ascontiguousarray(f, dtype=dtype)
    y = np.zeros((oplanes, orows, ocols), dtype=dtype)
    fn = lib().oracle_conv_f32 if dtype == np.float32 else lib().oracle_conv_f64
    P = ctypes.POINTER(ct)
    rc = fn(ctypes.byref(desc), x.ctypes.data_as(P), f.ctypes.data_as(P), y.ctypes.data_as(P),
            int(threads))
    if rc:
        raise ValueError("oracle rejected descriptor")
    return y


def separable(x, row_f, col_f, border, orient):
    x = np.ascontiguousarray(x, dtype=np.float32)
    planes = 1 if x.ndim == 2 else x.shape[0]
    rows, cols = x.shape[-2:]
    y = np.zeros_like(x)
    rf = np.ascontiguousarray(row_f, dtype=np.float32)
    cf = np.ascontiguousarray(col_f, dtype=np.float32)
    P = ctypes.POINTER(ctypes.c_float)
    rc = lib().oracle_separable_f32(rows, cols, planes, x.ctypes.data_as(P), rf.ctypes.data_as(P),
                                    rf.size, cf.ctypes.data_as(P), cf.size, border, orient,
                                    y.ctypes.data_as(P))
    if rc:
        raise ValueError("oracle rejected separable arguments")
    return y


def cyclic_conv_fft64(x, f, orient=CONV):
    """Float64 cyclic convolution (BorderCyclic, no sampling) of one plane by
    FFT, centred like the direct form: y[i,j] = sum x[(i-h+r)%H, (j-h+s)%W] f'[r,s]."""
    x = np.asarray(x, dtype=np.float64)
    f = np.asarray(f, dtype=np.float64)
    H, W = x.shape
    R, S = f.shape
    fp = f if orient == XCORR else f[::-1, ::-1]
    # y = sum_{r,s} fp[r,s] x[i + r - hr, j + s - hs]  ==  x (*) g with g[-(r-hr), -(s-hs)] = fp[r,s]
    g = np.zeros((H, W))
    hr, hs = (R - 1) // 2, (S - 1) // 2
    for r in range(R):
        for s in range(S):
            g[(-(r - hr)) % H, (-(s - hs)) % W] += fp[r, s]
    return np.real(np.fft.ifft2(np.fft.fft2(x) * np.fft.fft2(g)))


def rel_errors(y, ref):
    """Normwise errors: max|d|/max|ref| and rms(d)/rms(ref)."""
    y = np.asarray(y, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    d = y - ref
    mx = float(np.max(np.abs(ref))) if ref.size else 0.0
    rms = float(np.sqrt(np.mean(ref ** 2))) if ref.size else 0.0
    return (float(np.max(np.abs(d))) / mx if mx > 0 else float(np.max(np.abs(d), initial=0.0)),
            float(np.sqrt(np.mean(d ** 2))) / rms if rms > 0 else 0.0)


def poor_float_equal(a, b):
    """cct-core's ``~==`` (cogmath/algebra/real/PoorFloat.scala:43-51):
    |a-b| < 10*2^-12 * max(|a|,|b|), or absolute 10*2^-12 when one side is 0."""
    eps = 10.0 * 2.0 ** -12
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    diff = np.abs(a - b)
    mag = np.maximum(np.abs(a), np.abs(b))
    zero = (a == 0) | (b == 0)
    ok = np.where(zero, diff < eps, diff < eps * mag)
    return bool(np.all(ok))


if __name__ == "__main__":
    build()
    print(os.path.join(_HERE, "liboracle.so"))


def scalar_matrix(x, mats, border):
    """Scalar field (rows, cols) cross-correlated with a matrix field given as
    (size, size, mrows, mcols) (tensor-element-major, as stored); returns
    (mrows * mcols, rows, cols)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    mats = np.ascontiguousarray(mats, dtype=np.float32)
    size, size2, mr, mc = mats.shape
    assert size == size2
    rows, cols = x.shape
    y = np.zeros((mr * mc, rows, cols), dtype=np.float32)
    P = ctypes.POINTER(ctypes.c_float)
    rc = lib().oracle_scalar_matrix_f32(rows, cols, x.ctypes.data_as(P), mats.ctypes.data_as(P), mr, mc,
                                        size, border, y.ctypes.data_as(P))
    if rc:
        raise ValueError("oracle rejected scalar-matrix arguments")
    return y


def color_unpack(rgba):
    """(rows, cols, 4) uint8 -> (3, rows, cols) float32 planes (byte / 255)."""
    rgba = np.ascontiguousarray(rgba, dtype=np.uint8)
    rows, cols, _ = rgba.shape
    out = np.zeros((3, rows, cols), dtype=np.float32)
    lib().oracle_color_unpack(rows * cols, rgba.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                              out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    return out


def color_pack(planes):
    """(3, rows, cols) float32 -> (rows, cols, 4) uint8, alpha 255."""
    planes = np.ascontiguousarray(planes, dtype=np.float32)
    _, rows, cols = planes.shape
    out = np.zeros((rows, cols, 4), dtype=np.uint8)
    lib().oracle_color_pack(rows * cols, planes.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)))
    return out


def color_conv(desc, rgba, f):
    """ColorField convolution (DynamicConvolutionGenerator.scala:89-106): the
    red, green and blue planes each convolved with the scalar filter as
    `desc` describes (its plane counts are ignored), then merged."""
    d = OracleDesc(*[getattr(desc, n) for n, _ in OracleDesc._fields_])
    d.planes, d.f_planes = 3, 0
    return color_pack(conv(d, color_unpack(rgba), f))
