"""Generate the golden-vector fixture for the field-convolution parity tests.

Reads the 25 dynamic-convolution cases that the reference ships under
``src/test/resources/platform/opencl/hyperkernels/convolutionDynamic/`` and
writes them to ``convolution_dynamic.npz`` next to this script.

Each case ``i`` in the reference consists of
  * ``x{i}.fld``   input ScalarField
  * ``k{i}.fld``   filter ScalarField
  * ``wx{i}.fld``  convolve(x, k, border, sampling)       (ConvolutionOrientation)
  * ``y{i}.fld``   a field shaped like ``wx``
  * ``wty{i}.fld`` crossCorrelate(y, k) mapped back to x's shape: the adjoint
  * ``{i}.hdr``    sampling policy name + step, border policy name

File formats (reference ``src/test/scala/cogx/helper/fieldio/FieldIO.scala``
and ``src/test/scala/cogx/DynamicConvolutionSpec.scala:40-72``): Java
``DataOutputStream`` big-endian ints, UTF-16 chars, a long tick, then
big-endian float32 values with columns in the inner loop.

Run (only where the reference tree is present):
    python tests/golden/make_golden.py <reference_root>
"""
import struct
import sys
from pathlib import Path

import numpy as np

SUBDIR = "src/test/resources/platform/opencl/hyperkernels/convolutionDynamic"

BORDERS = {"BorderZero": 0, "BorderClamp": 1, "BorderCyclic": 2,
           "BorderValid": 3, "BorderFull": 4}
SAMPLINGS = {"NoSamplingConvolution": 0, "DownsampleOutputConvolution": 1,
             "UpsampleInputConvolution": 2}


def _read_int(buf, pos):
    return struct.unpack_from(">i", buf, pos)[0], pos + 4


def _read_chars(buf, pos, n):
    s = buf[pos:pos + 2 * n].decode("utf-16-be")
    return s, pos + 2 * n


def read_fld(path):
    buf = Path(path).read_bytes()
    pos = 0
    n, pos = _read_int(buf, pos)
    kind, pos = _read_chars(buf, pos, n)
    if kind != "ScalarLattice":
        raise ValueError(f"{path}: unsupported tensor kind {kind}")
    ndims, pos = _read_int(buf, pos)
    dims = []
    for _ in range(ndims):
        d, pos = _read_int(buf, pos)
        dims.append(d)
    tdims, pos = _read_int(buf, pos)
    for _ in range(tdims):
        _, pos = _read_int(buf, pos)
    pos += 8  # tick
    count = int(np.prod(dims))
    data = np.frombuffer(buf, dtype=">f4", count=count, offset=pos)
    if pos + 4 * count != len(buf):
        raise ValueError(f"{path}: trailing bytes")
    return data.astype(np.float32).reshape(dims)


def read_hdr(path):
    buf = Path(path).read_bytes()
    pos = 0
    n, pos = _read_int(buf, pos)
    sampling, pos = _read_chars(buf, pos, n)
    step, pos = _read_int(buf, pos)
    n, pos = _read_int(buf, pos)
    border, pos = _read_chars(buf, pos, n)
    return SAMPLINGS[sampling], step, BORDERS[border]


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference_root>  (the cct-core source tree)")
    root = Path(sys.argv[1])
    src = root / SUBDIR
    out = {}
    for i in range(25):
        sampling, step, border = read_hdr(src / f"{i}.hdr")
        out[f"hdr{i}"] = np.array([sampling, step, border], dtype=np.int32)
        for name in ("x", "k", "wx", "y", "wty"):
            out[f"{name}{i}"] = read_fld(src / f"{name}{i}.fld")
    dst = Path(__file__).with_name("convolution_dynamic.npz")
    np.savez_compressed(dst, **out)
    print(f"wrote {dst} ({dst.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
