"""ctypes binding of libcctconv.so (the C-ABI declared in include/cct_conv.h).

The library is built in-tree (``cct-core_b200/csrc/libcctconv.so``).  There is
no fallback: if the shared library is missing or fails to load, importing
this module raises.
"""
import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("CCT_CONV_LIB", _PKG.parent / "csrc" / "libcctconv.so"))

# status codes
OK, EINVAL, ENOTSUP, ENOMEM, ECUDA, ETIMEOUT, ENODEV = 0, -1, -2, -3, -4, -5, -6
# policies (numeric values are the ABI's)
BORDER_ZERO, BORDER_CLAMP, BORDER_CYCLIC, BORDER_VALID, BORDER_FULL = range(5)
CROSS_CORRELATION, CONVOLUTION = 0, 1
SAMPLE_NONE, SAMPLE_DOWN, SAMPLE_UP = 0, 1, 2
(PLANE_BY_PLANE, PROJECT_FRAME, PROJECT_FRAME_BLOCK_REDUCE_SUM, BACK_PROJECT_FRAME,
 BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM, FILTER_ADJOINT, FILTER_ADJOINT_BLOCK_REDUCE_SUM) = range(7)
PREC_FP32, PREC_BF16X3, PREC_BF16X6 = 0, 1, 2
ALGO_AUTO, ALGO_DIRECT, ALGO_FFT = 0, 1, 2
FLAG_RELU = 0x1
PLAN_DIRECT, PLAN_FRAME_F32, PLAN_FRAME_BF16X3, PLAN_FFT, PLAN_FILTER_ADJOINT, PLAN_FILTER_ADJOINT_BF16X3 = range(6)


class ConvDesc(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_int32),
        ("image_rows", ctypes.c_int32),
        ("image_cols", ctypes.c_int32),
        ("image_planes", ctypes.c_int32),
        ("filter_rows", ctypes.c_int32),
        ("filter_cols", ctypes.c_int32),
        ("filter_planes", ctypes.c_int32),
        ("batch_size", ctypes.c_int32),
        ("border", ctypes.c_int32),
        ("orientation", ctypes.c_int32),
        ("sampling", ctypes.c_int32),
        ("step", ctypes.c_int32),
        ("vector_mode", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("algo", ctypes.c_int32),
        ("flags", ctypes.c_uint32),
    ]

    def key(self):
        return tuple(getattr(self, n) for n, _ in self._fields_)


class CctError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"[{status}] {message}")
        self.status = status


class ServerConfig(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_int32), ("slots", ctypes.c_int32),
                ("max_batch", ctypes.c_int32), ("flags", ctypes.c_int32),
                ("arena_bytes", ctypes.c_uint64), ("hbm_reserve_bytes", ctypes.c_uint64)]


class ServeRequest(ctypes.Structure):
    _fields_ = [("struct_size", ctypes.c_int32), ("kind", ctypes.c_int32), ("desc", ConvDesc),
                ("image", ctypes.c_void_p), ("filter", ctypes.c_void_p),
                ("filter_id", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("out", ctypes.c_void_p), ("graph", ctypes.c_void_p)]


SERVE_CONV, SERVE_GRAPH_STEP = 0, 1
SERVE_PER_CALL = 0x1

NODE_CONV, NODE_ADD, NODE_SUB, NODE_MUL, NODE_RELU, NODE_SCALE = range(6)


class FieldShape(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_int32), ("cols", ctypes.c_int32), ("planes", ctypes.c_int32)]


class CircuitNode(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int32), ("in0", ctypes.c_int32), ("in1", ctypes.c_int32),
                ("scalar", ctypes.c_float), ("conv", ConvDesc)]

# Every symbol include/cct_conv.h declares, with (restype, argtypes).
_P = ctypes.c_void_p
_I = ctypes.c_int
_I32 = ctypes.c_int32
_PI32 = ctypes.POINTER(ctypes.c_int32)
SIGNATURES = {
    "cct_conv_desc_init": (None, [ctypes.POINTER(ConvDesc)]),
    "cct_conv_output_shape": (_I, [ctypes.POINTER(ConvDesc), _PI32, _PI32, _PI32]),
    "cct_conv_plan_create": (_I, [ctypes.POINTER(ConvDesc), ctypes.POINTER(_P)]),
    "cct_conv_plan_destroy": (_I, [_P]),
    "cct_conv_plan_algo": (_I, [_P, _PI32]),
    "cct_conv_plan_set_static_filter": (_I, [_P, _P]),
    "cct_conv_run": (_I, [_P, _P, _P, _P, _P]),
    "cct_conv_run_host": (_I, [_P, _P, _P, _P, _P]),
    "cct_conv_separable": (_I, [_I32, _I32, _I32, _P, _P, _I32, _P, _I32, _I32, _I32, _P, _P, _P]),
    "cct_conv_run_noalloc": (_I, [ctypes.POINTER(ConvDesc), _P, _P, _P, _P]),
    "cct_conv_scalar_matrix": (_I, [_I32, _I32, _P, _P, _I32, _I32, _I32, _I32, _I32, _I32, _I32, _P, _P]),
    "cct_color_plan_create": (_I, [ctypes.POINTER(ConvDesc), ctypes.POINTER(_P)]),
    "cct_color_plan_set_static_filter": (_I, [_P, _P]),
    "cct_color_run": (_I, [_P, _P, _P, _P, _P]),
    "cct_color_plan_destroy": (_I, [_P]),
    "cct_graph_create": (_I, [ctypes.POINTER(ConvDesc), _I32, ctypes.POINTER(_P)]),
    "cct_graph_destroy": (_I, [_P]),
    "cct_graph_set_filter": (_I, [_P, _I32, _P]),
    "cct_graph_field": (_I, [_P, _I32, ctypes.POINTER(_P), ctypes.POINTER(ctypes.c_size_t)]),
    "cct_graph_step": (_I, [_P, ctypes.c_int64, _P]),
    "cct_graph_step_host": (_I, [_P, _P, _P, _P]),
    "cct_graph_time": (ctypes.c_int64, [_P]),
    "cct_graph_reset": (_I, [_P]),
    "cct_graph_save": (_I, [_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "cct_graph_restore": (_I, [_P, ctypes.c_size_t, ctypes.POINTER(_P)]),
    "cct_circuit_assign": (_I, [ctypes.POINTER(FieldShape), _I32, ctypes.POINTER(CircuitNode), _I32, _PI32, _I32,
                                _PI32, _PI32]),
    "cct_circuit_create": (_I, [ctypes.POINTER(FieldShape), _I32, ctypes.POINTER(CircuitNode), _I32, _PI32, _I32,
                                ctypes.POINTER(_P)]),
    "cct_circuit_destroy": (_I, [_P]),
    "cct_circuit_set_filter": (_I, [_P, _I32, _P]),
    "cct_circuit_field": (_I, [_P, _I32, ctypes.POINTER(_P), ctypes.POINTER(ctypes.c_size_t)]),
    "cct_circuit_buffers": (_I, [_P, _PI32, ctypes.POINTER(ctypes.c_size_t)]),
    "cct_circuit_step": (_I, [_P, ctypes.c_int64, _P]),
    "cct_circuit_step_host": (_I, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P), _P]),
    "cct_circuit_time": (ctypes.c_int64, [_P]),
    "cct_circuit_reset": (_I, [_P]),
    "cct_conv_plan_save": (_I, [_P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
    "cct_conv_plan_restore": (_I, [_P, ctypes.c_size_t, ctypes.POINTER(_P)]),
    "cct_record_describe": (_I, [_P, ctypes.c_size_t, _PI32, _PI32, ctypes.POINTER(ctypes.c_int64),
                                 ctypes.POINTER(ConvDesc), _I32]),
    "cct_server_config_init": (None, [ctypes.POINTER(ServerConfig)]),
    "cct_serve_request_init": (None, [ctypes.POINTER(ServeRequest)]),
    "cct_server_create": (_I, [ctypes.POINTER(ServerConfig), ctypes.POINTER(_P)]),
    "cct_server_destroy": (_I, [_P]),
    "cct_server_add_filter": (_I, [_P, _P, ctypes.c_size_t, _PI32]),
    "cct_server_submit": (_I, [_P, ctypes.POINTER(ServeRequest), ctypes.POINTER(ctypes.c_uint64)]),
    "cct_server_wait": (_I, [_P, ctypes.c_uint64, _I32, ctypes.POINTER(ctypes.c_double)]),
    "cct_server_replay": (_I, [_P, ctypes.POINTER(ServeRequest), ctypes.POINTER(ctypes.c_double), _I32,
                               ctypes.POINTER(ctypes.c_double)]),
    "cct_server_stats": (_I, [_P] + [ctypes.POINTER(ctypes.c_uint64)] * 4),
    "cct_host_alloc": (_I, [ctypes.POINTER(_P), ctypes.c_size_t]),
    "cct_host_free": (_I, [_P]),
    "cct_malloc": (_I, [ctypes.POINTER(_P), ctypes.c_size_t]),
    "cct_free": (_I, [_P]),
    "cct_memcpy_h2d": (_I, [_P, _P, ctypes.c_size_t, _P]),
    "cct_memcpy_d2h": (_I, [_P, _P, ctypes.c_size_t, _P]),
    "cct_stream_create": (_I, [ctypes.POINTER(_P)]),
    "cct_stream_destroy": (_I, [_P]),
    "cct_stream_synchronize": (_I, [_P]),
    "cct_device_status": (_I, []),
    "cct_selftest_wait_timeout": (_I, [ctypes.POINTER(ctypes.c_double)]),
    "cct_last_error_string": (ctypes.c_char_p, []),
    "cct_abi_version": (_I, []),
    "cct_launch_count": (ctypes.c_uint64, []),
}


def _load():
    if not LIB_PATH.exists():
        raise ImportError(f"libcctconv.so not built: {LIB_PATH} (run `make -C cct-core_b200/csrc`)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


LIB = _load()


def check(status):
    if status != OK:
        raise CctError(status, LIB.cct_last_error_string().decode(errors="replace"))
    return status


def new_desc(**fields):
    d = ConvDesc()
    LIB.cct_conv_desc_init(ctypes.byref(d))
    for k, v in fields.items():
        setattr(d, k, int(v))
    return d


def output_shape(desc):
    r, c, p = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    check(LIB.cct_conv_output_shape(ctypes.byref(desc), ctypes.byref(r), ctypes.byref(c),
                                    ctypes.byref(p)))
    return r.value, c.value, p.value


def _save_record(fn, handle):
    """Checkpoint record of a plan or graph as a numpy uint32 array."""
    import numpy as np
    n = ctypes.c_size_t()
    check(fn(handle, None, 0, ctypes.byref(n)))
    words = np.zeros(n.value, dtype=np.uint32)
    check(fn(handle, ctypes.c_void_p(words.ctypes.data), n.value, ctypes.byref(n)))
    return words


def describe_record(words):
    """(kind, layer descriptors, step count) of a checkpoint record; kind 1
    is a plan, 2 a graph.  Needs no device."""
    import numpy as np
    w = np.ascontiguousarray(words, dtype=np.uint32)
    kind, n, t = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
    check(LIB.cct_record_describe(ctypes.c_void_p(w.ctypes.data), w.size, ctypes.byref(kind),
                                  ctypes.byref(n), ctypes.byref(t), None, 0))
    descs = (ConvDesc * n.value)()
    check(LIB.cct_record_describe(ctypes.c_void_p(w.ctypes.data), w.size, None, None, None, descs, n.value))
    return kind.value, list(descs), t.value


class Plan:
    """Owning wrapper of a cct_conv_plan."""

    def __init__(self, desc, _handle=None):
        self.desc = desc
        self.shape = output_shape(desc)
        h = ctypes.c_void_p()
        if _handle is None:
            check(LIB.cct_conv_plan_create(ctypes.byref(desc), ctypes.byref(h)))
        else:
            h = _handle
        self.handle = h
        a = ctypes.c_int32()
        check(LIB.cct_conv_plan_algo(h, ctypes.byref(a)))
        self.algo = a.value

    def save(self):
        """Checkpoint record (numpy uint32 words): descriptor + constant filter."""
        return _save_record(LIB.cct_conv_plan_save, self.handle)

    @classmethod
    def restore(cls, words):
        import numpy as np
        w = np.ascontiguousarray(words, dtype=np.uint32)
        h = ctypes.c_void_p()
        check(LIB.cct_conv_plan_restore(ctypes.c_void_p(w.ctypes.data), w.size, ctypes.byref(h)))
        _, descs, _ = describe_record(w)
        return cls(descs[0], _handle=h)

    def set_static_filter(self, host_ptr):
        check(LIB.cct_conv_plan_set_static_filter(self.handle, ctypes.c_void_p(host_ptr)))

    def run(self, x_ptr, f_ptr, y_ptr, stream=0):
        check(LIB.cct_conv_run(self.handle, ctypes.c_void_p(x_ptr), ctypes.c_void_p(f_ptr),
                               ctypes.c_void_p(y_ptr), ctypes.c_void_p(stream)))

    def run_host(self, x_ptr, f_ptr, y_ptr, stream=0):
        check(LIB.cct_conv_run_host(self.handle, ctypes.c_void_p(x_ptr), ctypes.c_void_p(f_ptr),
                                    ctypes.c_void_p(y_ptr), ctypes.c_void_p(stream)))

    def close(self):
        if self.handle:
            LIB.cct_conv_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ColorPlan:
    """Owning wrapper of a cct_color_plan (colour-field convolution: RGBA8 in
    and out, the three colour planes convolved with one scalar filter)."""

    def __init__(self, desc):
        self.desc = desc
        self.shape = output_shape(desc)
        h = ctypes.c_void_p()
        check(LIB.cct_color_plan_create(ctypes.byref(desc), ctypes.byref(h)))
        self.handle = h

    def set_static_filter(self, host_ptr):
        check(LIB.cct_color_plan_set_static_filter(self.handle, ctypes.c_void_p(host_ptr)))

    def run(self, x_ptr, f_ptr, y_ptr, stream=0):
        check(LIB.cct_color_run(self.handle, ctypes.c_void_p(x_ptr), ctypes.c_void_p(f_ptr),
                                ctypes.c_void_p(y_ptr), ctypes.c_void_p(stream)))

    def close(self):
        if self.handle:
            LIB.cct_color_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    """Owning wrapper of a cct_graph: a chain of convolution layers stepped
    as one captured launch sequence."""

    def __init__(self, descs, _handle=None):
        if _handle is None:
            arr = (ConvDesc * len(descs))(*descs)
            h = ctypes.c_void_p()
            check(LIB.cct_graph_create(arr, len(descs), ctypes.byref(h)))
        else:
            h = _handle
        self.handle = h
        self.descs = list(descs)
        self.shapes = [output_shape(d) for d in descs]

    def set_filter(self, layer, host_ptr):
        check(LIB.cct_graph_set_filter(self.handle, layer, ctypes.c_void_p(host_ptr)))

    def field(self, index):
        """(device pointer, element count) of field `index` (0 = input)."""
        p, n = ctypes.c_void_p(), ctypes.c_size_t()
        check(LIB.cct_graph_field(self.handle, index, ctypes.byref(p), ctypes.byref(n)))
        return p.value, n.value

    def step(self, count=1, stream=0):
        check(LIB.cct_graph_step(self.handle, count, ctypes.c_void_p(stream)))
        return self.time

    def step_host(self, in_ptr, out_ptr, stream=0):
        check(LIB.cct_graph_step_host(self.handle, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr),
                                      ctypes.c_void_p(stream)))

    @property
    def time(self):
        return int(LIB.cct_graph_time(self.handle))

    def reset(self):
        check(LIB.cct_graph_reset(self.handle))
        return 0

    def save(self):
        """Checkpoint record (numpy uint32 words): layer descriptors, constant
        filters and the step count."""
        return _save_record(LIB.cct_graph_save, self.handle)

    @classmethod
    def restore(cls, words):
        import numpy as np
        w = np.ascontiguousarray(words, dtype=np.uint32)
        h = ctypes.c_void_p()
        check(LIB.cct_graph_restore(ctypes.c_void_p(w.ctypes.data), w.size, ctypes.byref(h)))
        _, descs, _ = describe_record(w)
        return cls(descs, _handle=h)

    def close(self):
        if self.handle:
            LIB.cct_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def launch_count():
    return int(LIB.cct_launch_count())
