"""Kernel circuits: a ComputeGraph step over a DAG of fields.

The reference compiles a ``ComputeGraph`` into a KernelCircuit and steps it by
enqueueing every kernel in one fixed order (src/main/scala/cogx/runtime/
execution/GPUSupervisor.scala:128-215), with fields sharing device buffers
once all their readers have run (runtime/allocation/
InOrderSharedLatchAllocator.scala:34).  ``Circuit`` is that step on
libcctconv: nodes are convolutions (any ``cct_conv_desc``) and elementwise
operations, listed in execution order; field ``i < len(inputs)`` is an input
(sensor) and field ``len(inputs) + k`` is node ``k``'s output; the listed
outputs (actuators) and the inputs keep buffers of their own.

    c = Circuit([(64, 64, 16)], [conv(0, d1), relu(1), conv(2, d2), add(3, 0), relu(4)], outputs=[5])
"""
import ctypes

import numpy as np
import torch

from . import _lib


def conv(image, desc, filter_field=-1):
    """Convolution node: `desc` describes it, `image` is its image field;
    `filter_field` a field holding its filter, or -1 for a static filter set
    with Circuit.set_filter."""
    return _lib.CircuitNode(op=_lib.NODE_CONV, in0=image, in1=filter_field, scalar=0.0, conv=desc)


def add(a, b):
    return _lib.CircuitNode(op=_lib.NODE_ADD, in0=a, in1=b, scalar=0.0)


def sub(a, b):
    return _lib.CircuitNode(op=_lib.NODE_SUB, in0=a, in1=b, scalar=0.0)


def mul(a, b):
    return _lib.CircuitNode(op=_lib.NODE_MUL, in0=a, in1=b, scalar=0.0)


def relu(a):
    return _lib.CircuitNode(op=_lib.NODE_RELU, in0=a, in1=-1, scalar=0.0)


def scale(a, s):
    return _lib.CircuitNode(op=_lib.NODE_SCALE, in0=a, in1=-1, scalar=float(s))


def _arrays(inputs, nodes, outputs):
    shp = (_lib.FieldShape * max(len(inputs), 1))(*[_lib.FieldShape(*s) for s in inputs])
    nds = (_lib.CircuitNode * len(nodes))(*nodes)
    outs = (ctypes.c_int32 * max(len(outputs), 1))(*outputs)
    return shp, nds, outs


def assign(inputs, nodes, outputs):
    """Buffer of every field under the in-order sharing rule, and the buffer
    count (host only: no device is touched)."""
    shp, nds, outs = _arrays(inputs, nodes, outputs)
    fb = (ctypes.c_int32 * (len(inputs) + len(nodes)))()
    nb = ctypes.c_int32()
    _lib.check(_lib.LIB.cct_circuit_assign(shp, len(inputs), nds, len(nodes), outs, len(outputs), fb,
                                           ctypes.byref(nb)))
    return list(fb), nb.value


class _DeviceArray:
    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False),
                                         "version": 3, "strides": None}


class Circuit:
    """Owning wrapper of a cct_circuit."""

    def __init__(self, inputs, nodes, outputs):
        self.inputs = [tuple(s) for s in inputs]
        self.nodes = list(nodes)
        self.outputs = list(outputs)
        shp, nds, outs = _arrays(self.inputs, self.nodes, self.outputs)
        h = ctypes.c_void_p()
        _lib.check(_lib.LIB.cct_circuit_create(shp, len(self.inputs), nds, len(self.nodes), outs,
                                               len(self.outputs), ctypes.byref(h)))
        self.handle = h

    def set_filter(self, node, host_filter):
        f = np.ascontiguousarray(host_filter, dtype=np.float32)
        _lib.check(_lib.LIB.cct_circuit_set_filter(self.handle, node, ctypes.c_void_p(f.ctypes.data)))

    def field_ptr(self, index):
        p, n = ctypes.c_void_p(), ctypes.c_size_t()
        _lib.check(_lib.LIB.cct_circuit_field(self.handle, index, ctypes.byref(p), ctypes.byref(n)))
        return p.value, n.value

    def field(self, index):
        """torch view (flat) of field `index`; shared buffers hold a field's
        value only until a later node reuses them within the step."""
        ptr, n = self.field_ptr(index)
        return torch.as_tensor(_DeviceArray(ptr, n), device="cuda")

    def buffers(self):
        n, b = ctypes.c_int32(), ctypes.c_size_t()
        _lib.check(_lib.LIB.cct_circuit_buffers(self.handle, ctypes.byref(n), ctypes.byref(b)))
        return n.value, b.value

    def step(self, count=1, stream=None):
        s = torch.cuda.current_stream().cuda_stream if stream is None else stream
        _lib.check(_lib.LIB.cct_circuit_step(self.handle, count, ctypes.c_void_p(s)))
        return self.time

    def step_host(self, host_inputs, host_outputs, stream=None):
        """One step from host float32 arrays (one per input) into host arrays
        (one per listed output)."""
        s = torch.cuda.current_stream().cuda_stream if stream is None else stream
        ins = (ctypes.c_void_p * max(len(host_inputs), 1))(*[a.ctypes.data for a in host_inputs])
        outs = (ctypes.c_void_p * max(len(host_outputs), 1))(*[a.ctypes.data for a in host_outputs])
        _lib.check(_lib.LIB.cct_circuit_step_host(self.handle, ins, outs, ctypes.c_void_p(s)))

    @property
    def time(self):
        return int(_lib.LIB.cct_circuit_time(self.handle))

    def reset(self):
        _lib.check(_lib.LIB.cct_circuit_reset(self.handle))

    def close(self):
        if self.handle:
            _lib.check(_lib.LIB.cct_circuit_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
