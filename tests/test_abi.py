"""libcctconv.so loads, exports every declared symbol, and its host-side
descriptor logic agrees with the oracle's restatement (no GPU needed)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from cctconv import _lib

HEADERS = sorted((Path(__file__).resolve().parent.parent / "include").glob("*.h"))


def declared_functions():
    names = []
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^[A-Za-z_][\w \*]*?\b(cct_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(_lib.LIB, n), n
        assert n in _lib.SIGNATURES, f"{n} not bound in cctconv._lib"


def test_abi_version_and_desc_size():
    assert _lib.LIB.cct_abi_version() == 1
    d = _lib.new_desc()
    assert d.struct_size == ctypes.sizeof(_lib.ConvDesc) == 64
    assert d.batch_size == 1 and d.orientation == _lib.CONVOLUTION


def _oracle_desc(d):
    return O.make_desc(d.image_rows, d.image_cols, d.filter_rows, d.filter_cols,
                       planes=d.image_planes, f_planes=d.filter_planes, batch=d.batch_size,
                       border=d.border, orient=d.orientation, sampling=d.sampling, step=d.step,
                       mode=d.vector_mode)


def test_output_shape_agrees_with_oracle_on_random_descriptors():
    rng = np.random.default_rng(1234)
    n_ok = n_err = 0
    for _ in range(4000):
        d = _lib.new_desc(
            image_rows=int(rng.integers(1, 40)), image_cols=int(rng.integers(1, 40)),
            image_planes=int(rng.choice([0, 1, 2, 3, 4, 6, 8, 12])),
            filter_rows=int(rng.integers(1, 10)), filter_cols=int(rng.integers(1, 10)),
            filter_planes=int(rng.choice([0, 1, 2, 3, 4, 6, 8, 12, 24])),
            batch_size=int(rng.choice([1, 2, 3, 4])), border=int(rng.integers(0, 5)),
            orientation=int(rng.integers(0, 2)), sampling=int(rng.integers(0, 3)),
            step=int(rng.integers(1, 5)), vector_mode=int(rng.integers(0, 5)))
        try:
            want = O.output_shape(_oracle_desc(d))
        except ValueError:
            want = None
        try:
            got = _lib.output_shape(d)
        except _lib.CctError as e:
            assert e.status == _lib.EINVAL
            got = None
        assert got == want, (d.key(), got, want)
        n_ok += got is not None
        n_err += got is None
    assert n_ok > 500 and n_err > 500


@pytest.mark.parametrize("field,expect", [
    (dict(struct_size=12), "struct_size"),
    (dict(border=9), "bad border"),
    (dict(precision=7), "bad precision"),
    (dict(flags=0x10), "unknown flags"),
    (dict(filter_rows=4, filter_cols=3), "odd shape"),
])
def test_invalid_descriptors_report_einval(field, expect):
    d = _lib.new_desc(image_rows=16, image_cols=16, filter_rows=3, filter_cols=3)
    for k, v in field.items():
        setattr(d, k, v)
    with pytest.raises(_lib.CctError, match=expect) as e:
        _lib.output_shape(d)
    assert e.value.status == _lib.EINVAL


def test_reference_error_messages():
    d = _lib.new_desc(image_rows=10, image_cols=10, filter_rows=3, filter_cols=3,
                      border=_lib.BORDER_CLAMP, sampling=_lib.SAMPLE_UP, step=2)
    with pytest.raises(_lib.CctError, match="Integrated upsampling with BorderClamp"):
        _lib.output_shape(d)
    d = _lib.new_desc(image_rows=11, image_cols=10, filter_rows=3, filter_cols=3,
                      sampling=_lib.SAMPLE_DOWN, step=2)
    with pytest.raises(_lib.CctError, match="divisible by the downsampling step"):
        _lib.output_shape(d)


def test_plan_without_gpu_is_enodev():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    d = _lib.new_desc(image_rows=16, image_cols=16, filter_rows=3, filter_cols=3)
    with pytest.raises(_lib.CctError) as e:
        _lib.Plan(d)
    assert e.value.status == _lib.ENODEV


def test_struct_layouts_match_the_header(tmp_path):
    """ctypes mirrors of the ABI structs have the C compiler's sizes and offsets."""
    import subprocess
    src = tmp_path / "layout.c"
    inc = Path(__file__).resolve().parent.parent / "include"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "cct_conv.h"\n'
        "int main(void) {\n"
        '  printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(cct_conv_desc), sizeof(cct_server_config),\n'
        "         sizeof(cct_serve_request), offsetof(cct_serve_request, image),\n"
        "         offsetof(cct_serve_request, filter_id), offsetof(cct_serve_request, out),\n"
        "         offsetof(cct_serve_request, graph));\n  return 0;\n}\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(inc), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    R = _lib.ServeRequest
    assert got == [ctypes.sizeof(_lib.ConvDesc), ctypes.sizeof(_lib.ServerConfig), ctypes.sizeof(R),
                   R.image.offset, R.filter_id.offset, R.out.offset, R.graph.offset]


def test_server_and_graph_need_a_device():
    cfg = _lib.ServerConfig()
    _lib.LIB.cct_server_config_init(ctypes.byref(cfg))
    assert cfg.struct_size == ctypes.sizeof(_lib.ServerConfig)
    assert cfg.slots == 3 and cfg.max_batch == 64 and cfg.arena_bytes == 0  # admission by free HBM
    assert cfg.hbm_reserve_bytes == 2 << 30
    h = ctypes.c_void_p()
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert _lib.LIB.cct_server_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.ENODEV
    bad = _lib.ServerConfig()
    _lib.LIB.cct_server_config_init(ctypes.byref(bad))
    bad.slots = 9
    rc = _lib.LIB.cct_server_create(ctypes.byref(bad), ctypes.byref(h))
    assert rc in (_lib.EINVAL, _lib.ENODEV)


@pytest.mark.parametrize("border,orient,sampling,step,size,msg", [
    (_lib.BORDER_FULL, _lib.CROSS_CORRELATION, _lib.SAMPLE_NONE, 1, 3, "unsupported: BorderFull"),
    (_lib.BORDER_VALID, _lib.CROSS_CORRELATION, _lib.SAMPLE_NONE, 1, 3, "unsupported: BorderValid"),
    (_lib.BORDER_ZERO, _lib.CONVOLUTION, _lib.SAMPLE_NONE, 1, 3, "convolution not supported yet"),
    (_lib.BORDER_CLAMP, _lib.CROSS_CORRELATION, _lib.SAMPLE_DOWN, 2, 3, "sampling not supported yet"),
    (_lib.BORDER_CYCLIC, _lib.CROSS_CORRELATION, _lib.SAMPLE_UP, 3, 3, "sampling not supported yet"),
    (_lib.BORDER_ZERO, _lib.CROSS_CORRELATION, _lib.SAMPLE_NONE, 1, 4, "odd size"),
])
def test_scalar_matrix_reference_restrictions(border, orient, sampling, step, size, msg):
    """ScalarMatrixConvolve2DHyperKernel.scala:118-152 rejects these before
    any device work."""
    rc = _lib.LIB.cct_conv_scalar_matrix(8, 8, 16, 16, 2, 2, size, border, orient, sampling, step, 16, None)
    assert rc == _lib.EINVAL
    assert msg in _lib.LIB.cct_last_error_string().decode()


def test_color_plan_descriptor_checks():
    h = ctypes.c_void_p()
    for kw, msg in [(dict(image_planes=3), "one colour field"), (dict(filter_planes=2), "scalar filter"),
                    (dict(vector_mode=_lib.PROJECT_FRAME), "plane by plane"),
                    (dict(precision=_lib.PREC_BF16X3), "FP32")]:
        d = _lib.new_desc(image_rows=8, image_cols=8, filter_rows=3, filter_cols=3, **kw)
        assert _lib.LIB.cct_color_plan_create(ctypes.byref(d), ctypes.byref(h)) == _lib.EINVAL
        assert msg in _lib.LIB.cct_last_error_string().decode()
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    d = _lib.new_desc(image_rows=8, image_cols=8, filter_rows=3, filter_cols=3)
    assert _lib.LIB.cct_color_plan_create(ctypes.byref(d), ctypes.byref(h)) == _lib.ENODEV


def _fnv1a(words):
    h = 2166136261
    for w in words:
        for b in range(4):
            h ^= (int(w) >> (8 * b)) & 0xFF
            h = (h * 16777619) & 0xFFFFFFFF
    return h


def _record(kind, layers, time=0):
    """A checkpoint record built here from the documented word layout."""
    w = [0x4B544343, 1, kind, len(layers), time & 0xFFFFFFFF, time >> 32]
    for fields, filt in layers:
        w += [15] + [int(v) & 0xFFFFFFFF for v in fields]
        n = len(filt)
        w += [n & 0xFFFFFFFF, n >> 32]
        w += list(np.asarray(filt, dtype=np.float32).view(np.uint32))
    w.append(_fnv1a(w))
    return np.array(w, dtype=np.uint32)


def test_checkpoint_record_format_and_checks():
    """cct_record_describe parses the documented layout (no device) and
    rejects bad magic, versions, checksums and lengths."""
    fields = [64, 64, 512, 5, 5, 2048, 16, _lib.BORDER_ZERO, _lib.CROSS_CORRELATION, _lib.SAMPLE_NONE, 1,
              _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, _lib.PREC_BF16X3, 0, 1]
    filt = np.linspace(-1, 1, 2048 * 25, dtype=np.float32)
    rec = _record(1, [(fields, filt)])
    kind, descs, t = _lib.describe_record(rec)
    assert kind == 1 and t == 0 and len(descs) == 1
    d = descs[0]
    assert (d.image_rows, d.image_cols, d.image_planes, d.filter_planes, d.batch_size) == (64, 64, 512, 2048, 16)
    assert (d.vector_mode, d.precision, d.flags) == (_lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, _lib.PREC_BF16X3, 1)
    assert d.struct_size == ctypes.sizeof(_lib.ConvDesc)
    g = _record(2, [(fields, []), (fields, filt[:10])], time=(5 << 32) + 7)
    kind, descs, t = _lib.describe_record(g)
    assert kind == 2 and len(descs) == 2 and t == (5 << 32) + 7
    for bad, msg in [(np.concatenate([[0x12345678], rec[1:]]), "magic"),
                     (rec[:-2], "checksum"),
                     (np.concatenate([rec[:-1], [rec[-1] ^ 1]]), "checksum"),
                     (rec[:5], "too short")]:
        with pytest.raises(_lib.CctError, match=msg):
            _lib.describe_record(bad)
    v2 = rec.copy()
    v2[1] = 2
    v2[-1] = _fnv1a(v2[:-1])
    with pytest.raises(_lib.CctError, match="version 2"):
        _lib.describe_record(v2)
    short = _record(1, [(fields, filt)])[:-1]
    short = np.concatenate([short[:-100], [_fnv1a(short[:-100])]]).astype(np.uint32)
    with pytest.raises(_lib.CctError, match="truncated"):
        _lib.describe_record(short)


def test_checkpoint_restore_needs_a_device_and_save_a_plan():
    import torch
    h = ctypes.c_void_p()
    n = ctypes.c_size_t()
    assert _lib.LIB.cct_conv_plan_save(None, None, 0, ctypes.byref(n)) == _lib.EINVAL
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    fields = [16, 16, 0, 3, 3, 0, 1, 0, 1, 0, 1, 0, 0, 0, 0]
    rec = _record(1, [(fields, np.ones(9, np.float32))])
    assert _lib.LIB.cct_conv_plan_restore(ctypes.c_void_p(rec.ctypes.data), rec.size, ctypes.byref(h)) == _lib.ENODEV
    grec = _record(2, [(fields, [])])
    assert _lib.LIB.cct_conv_plan_restore(ctypes.c_void_p(grec.ctypes.data), grec.size,
                                          ctypes.byref(h)) == _lib.EINVAL
    assert "graph, not a plan" in _lib.LIB.cct_last_error_string().decode()
