"""Stacked convolution graphs: the ComputeGraph step of a CNN layer stack.

In the reference a user builds a ``ComputeGraph`` whose fields are a chain of
``projectFrameBlockReduceSum`` (+ ``rectify``) layers over constant filter
banks and calls ``step`` (src/main/scala/cogx/runtime/ComputeGraph.scala:56,
228-279).  ``LayerStack`` is that graph on libcctconv: one descriptor per
layer, all fields resident on the device, and each step one replay of the
captured launch sequence (``cct_graph_step``).  ReLU is fused into the
producing layer's epilogue.
"""
import numpy as np
import torch

from . import _lib


class _DeviceArray:
    """Zero-copy view of a graph-owned device buffer for torch.as_tensor."""

    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4",
                                         "data": (ptr, False), "version": 3, "strides": None}


class LayerStack:
    """A chain of filter-bank layers on a batch of multi-plane fields.

    input_shape: (rows, cols, planes) of one sample; batch: samples per step;
    layers: sequence of (filters, filter_size, downsample_step, relu).
    precision: _lib.PREC_FP32 or _lib.PREC_BF16X3.
    """

    def __init__(self, input_shape, batch, layers, precision=_lib.PREC_FP32,
                 border=_lib.BORDER_ZERO):
        rows, cols, planes = input_shape
        self.batch = batch
        self.descs, self.filter_shapes, self.field_shapes = [], [], [(batch * planes, rows, cols)]
        for k, size, down, relu in layers:
            d = _lib.new_desc(image_rows=rows, image_cols=cols, image_planes=batch * planes,
                              filter_rows=size, filter_cols=size, filter_planes=k * planes,
                              batch_size=batch, border=border, orientation=_lib.CROSS_CORRELATION,
                              sampling=_lib.SAMPLE_DOWN if down > 1 else _lib.SAMPLE_NONE,
                              step=down, vector_mode=_lib.PROJECT_FRAME_BLOCK_REDUCE_SUM,
                              precision=precision, flags=_lib.FLAG_RELU if relu else 0)
            orows, ocols, oplanes = _lib.output_shape(d)
            self.descs.append(d)
            self.filter_shapes.append((k * planes, size, size))
            self.field_shapes.append((oplanes, orows, ocols))
            rows, cols, planes = orows, ocols, k
        self.graph = _lib.Graph(self.descs)
        # 2 * batch * K * out_rows * out_cols * C * R * R per layer
        self.flops_per_step = 0.0
        for (oplanes, orows, ocols), (kc, r, s), (k, _, _, _) in zip(
                self.field_shapes[1:], self.filter_shapes, layers):
            self.flops_per_step += 2.0 * oplanes * orows * ocols * (kc // k) * r * s

    def set_filters(self, filters):
        """Host float32 filter banks, one per layer, shaped (K*C, R, R)."""
        for i, f in enumerate(filters):
            f = np.ascontiguousarray(f, dtype=np.float32)
            if f.shape != self.filter_shapes[i]:
                raise ValueError(f"layer {i + 1} filter shape {f.shape} != {self.filter_shapes[i]}")
            self.graph.set_filter(i + 1, f.ctypes.data)

    def field(self, index):
        """torch view of field `index` (0 = input, i = layer i's output)."""
        ptr, _ = self.graph.field(index)
        return torch.as_tensor(_DeviceArray(ptr, self.field_shapes[index]), device="cuda")

    @property
    def input(self):
        return self.field(0)

    @property
    def output(self):
        return self.field(len(self.descs))

    def step(self, count=1, stream=None):
        s = torch.cuda.current_stream().cuda_stream if stream is None else stream
        return self.graph.step(count, s)

    def step_host(self, host_in, host_out, stream=None):
        s = torch.cuda.current_stream().cuda_stream if stream is None else stream
        self.graph.step_host(host_in.data_ptr(), host_out.data_ptr(), s)

    def reset(self):
        return self.graph.reset()

    def close(self):
        self.graph.close()


def eight_layer_stack(batch, precision=_lib.PREC_FP32, rows=224, cols=224, planes=3):
    """The eight-layer 3x3 stack: widths 64, 64, 128, 128, 256, 256, 512, 512,
    DownsampleOutput(2) on layers 2, 4 and 6, ReLU between layers."""
    widths = [64, 64, 128, 128, 256, 256, 512, 512]
    layers = [(k, 3, 2 if i in (1, 3, 5) else 1, i < 7) for i, k in enumerate(widths)]
    return LayerStack((rows, cols, planes), batch, layers, precision)
