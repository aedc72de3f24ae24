"""Stacked convolution graphs (the ComputeGraph step of a CNN layer stack)
against per-layer plans and the FP64 oracle.

A graph step replays the captured launches of every layer, so its fields must
equal what the layers' plans produce one call at a time (bit for bit: the same
kernels on the same inputs), the FP32 stack must equal the FP32 oracle chained
layer by layer (bit for bit), and the split-BF16 stack must stay within the
normwise 1e-5 of FP64 at every layer.
"""
import numpy as np
import pytest
import torch

import oracle as O
from cctconv import _lib
from cctconv.graph import LayerStack, eight_layer_stack

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _filters(stack, seed):
    rng = np.random.default_rng(seed)
    out = []
    for kc, r, s in stack.filter_shapes:
        c = kc // (stack.field_shapes[len(out) + 1][0] // stack.batch)
        out.append((rng.standard_normal((kc, r, s)) * np.sqrt(2.0 / (c * r * s))).astype(np.float32))
    return out


def _oracle_layer(desc, x, f, dtype):
    od = O.make_desc(desc.image_rows, desc.image_cols, desc.filter_rows, desc.filter_cols,
                     planes=desc.image_planes, f_planes=desc.filter_planes, batch=desc.batch_size,
                     border=O.ZERO, orient=O.XCORR,
                     sampling=O.DOWN if desc.sampling == _lib.SAMPLE_DOWN else O.NOSAMPLE,
                     step=desc.step, mode=O.PROJECT_REDUCE)
    y = O.conv(od, x, f, dtype)
    if desc.flags & _lib.FLAG_RELU:
        y = np.maximum(y, 0)
    return y


SMALL = [(64, 3, 1, True), (64, 3, 2, True), (128, 3, 1, True), (128, 3, 2, False)]


@pytest.mark.parametrize("precision", [_lib.PREC_FP32, _lib.PREC_BF16X3], ids=["fp32", "bf16x3"])
def test_graph_step_matches_per_layer_plans(precision):
    stack = LayerStack((32, 32, 3), 2, SMALL, precision)
    filters = _filters(stack, 1)
    stack.set_filters(filters)
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, stack.field_shapes[0]).astype(np.float32)
    stack.input.copy_(torch.from_numpy(x))
    assert stack.step() == 1
    torch.cuda.synchronize()
    assert _lib.LIB.cct_device_status() == _lib.OK
    cur = torch.from_numpy(x).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for i, d in enumerate(stack.descs):
        plan = _lib.Plan(d)
        fd = torch.from_numpy(filters[i]).cuda()
        y = torch.empty(stack.field_shapes[i + 1], device="cuda")
        plan.run(cur.data_ptr(), fd.data_ptr(), y.data_ptr(), stream)
        torch.cuda.synchronize()
        got = stack.field(i + 1)
        assert torch.equal(got, y), f"layer {i + 1}"
        plan.close()
        cur = y
    stack.close()


def test_graph_fp32_stack_is_the_chained_fp32_oracle():
    stack = LayerStack((24, 28, 3), 2, SMALL, _lib.PREC_FP32)
    filters = _filters(stack, 3)
    stack.set_filters(filters)
    x = np.random.default_rng(4).uniform(-1, 1, stack.field_shapes[0]).astype(np.float32)
    stack.input.copy_(torch.from_numpy(x))
    stack.step()
    torch.cuda.synchronize()
    cur = x
    for i, d in enumerate(stack.descs):
        cur = _oracle_layer(d, cur, filters[i], np.float32)
        got = stack.field(i + 1).cpu().numpy()
        assert np.array_equal(got.reshape(cur.shape).view(np.uint32), cur.view(np.uint32)), i + 1
    stack.close()


def test_graph_bf16x3_layers_within_tolerance_of_fp64():
    stack = LayerStack((32, 32, 3), 2, SMALL, _lib.PREC_BF16X3)
    filters = _filters(stack, 5)
    stack.set_filters(filters)
    x = np.random.default_rng(6).uniform(-1, 1, stack.field_shapes[0]).astype(np.float32)
    stack.input.copy_(torch.from_numpy(x))
    stack.step()
    torch.cuda.synchronize()
    prev, chain = x, x.astype(np.float64)
    for i, d in enumerate(stack.descs):
        got = stack.field(i + 1).cpu().numpy()
        ref = _oracle_layer(d, prev, filters[i], np.float64)  # this layer alone, on the GPU's input
        assert O.rel_errors(got.reshape(ref.shape), ref)[0] <= TOL, i + 1
        chain = _oracle_layer(d, chain, filters[i].astype(np.float64), np.float64)
        prev = got
    # end to end the per-layer errors add up across the stack
    emax, erms = O.rel_errors(prev.reshape(chain.shape), chain)
    assert emax <= 4 * len(stack.descs) * TOL and erms <= len(stack.descs) * TOL
    stack.close()


def test_graph_replays_are_identical_and_count_steps():
    stack = LayerStack((32, 32, 3), 2, SMALL, _lib.PREC_BF16X3)
    stack.set_filters(_filters(stack, 7))
    stack.input.uniform_(-1, 1)
    n0 = _lib.launch_count()
    stack.step()
    torch.cuda.synchronize()
    first = stack.output.clone()
    n1 = _lib.launch_count()
    assert stack.step(3) == 4
    torch.cuda.synchronize()
    assert torch.equal(stack.output, first)
    # each replay counts the graph's kernel nodes: one per layer here (static filters)
    assert _lib.launch_count() - n1 == 3 * len(stack.descs)
    assert n1 - n0 >= len(stack.descs)
    assert stack.reset() == 0 and stack.graph.time == 0
    stack.close()


def test_graph_new_filter_is_seen_by_the_captured_graph():
    stack = LayerStack((16, 16, 3), 1, SMALL[:2], _lib.PREC_FP32)
    filters = _filters(stack, 8)
    stack.set_filters(filters)
    stack.input.uniform_(-1, 1)
    stack.step()
    torch.cuda.synchronize()
    a = stack.output.clone()
    filters[1] = filters[1] * 2
    stack.set_filters(filters)
    stack.step()
    torch.cuda.synchronize()
    # ReLU(2 z) = 2 ReLU(z), exactly in floating point
    assert torch.equal(stack.output, 2 * a)
    stack.close()


def test_graph_host_step():
    stack = LayerStack((16, 20, 3), 2, SMALL[:3], _lib.PREC_FP32)
    filters = _filters(stack, 9)
    stack.set_filters(filters)
    x = np.random.default_rng(10).uniform(-1, 1, stack.field_shapes[0]).astype(np.float32)
    hx = torch.from_numpy(x).pin_memory()
    hy = torch.empty(stack.field_shapes[-1]).pin_memory()
    stack.step_host(hx, hy)
    cur = x
    for i, d in enumerate(stack.descs):
        cur = _oracle_layer(d, cur, filters[i], np.float32)
    assert np.array_equal(hy.numpy().reshape(cur.shape), cur)
    stack.close()


def test_graph_rejects_mismatched_layers_and_missing_filters():
    a = _lib.new_desc(image_rows=16, image_cols=16, image_planes=3, filter_rows=3, filter_cols=3,
                      filter_planes=8 * 3, batch_size=1, vector_mode=_lib.PROJECT_FRAME_BLOCK_REDUCE_SUM)
    b = _lib.new_desc(image_rows=16, image_cols=16, image_planes=4, filter_rows=3, filter_cols=3,
                      filter_planes=8 * 4, batch_size=1, vector_mode=_lib.PROJECT_FRAME_BLOCK_REDUCE_SUM)
    with pytest.raises(_lib.CctError, match="layer 2 reads"):
        _lib.Graph([a, b])
    g = _lib.Graph([a])
    with pytest.raises(_lib.CctError, match="no filter"):
        g.step()
    with pytest.raises(_lib.CctError, match="Negative step count"):
        g.step(-1)
    g.close()


def test_eight_layer_stack_224_batch1():
    """The 224x224x3 eight-layer stack at batch 1 in split BF16: one step,
    every layer within 1e-5 of FP64 applied to the GPU's own layer input."""
    stack = eight_layer_stack(1, _lib.PREC_BF16X3)
    filters = _filters(stack, 11)
    stack.set_filters(filters)
    x = np.random.default_rng(12).uniform(-1, 1, stack.field_shapes[0]).astype(np.float32)
    stack.input.copy_(torch.from_numpy(x))
    stack.step()
    torch.cuda.synchronize()
    assert _lib.LIB.cct_device_status() == _lib.OK
    prev = x
    for i, d in enumerate(stack.descs):
        got = stack.field(i + 1).cpu().numpy()
        ref = _oracle_layer(d, prev, filters[i], np.float64)
        assert O.rel_errors(got.reshape(ref.shape), ref)[0] <= TOL, i + 1
        prev = got
    stack.close()


def test_eight_layer_stack_batch8_three_term_split_end_to_end():
    """The 224x224x3 eight-layer stack at batch 8 in the three-term split
    (BF16X6): the last layer's output, after all eight layers from the input,
    within 1e-5 (normwise) of the same stack in FP64 (zero-border 3x3
    cross-correlations, DownsampleOutput(2) on layers 2, 4 and 6, ReLU
    between layers).  The two-term split (BF16X3) keeps each layer under
    1e-5 but compounds to about 1.4e-5 over eight layers."""
    import torch.nn.functional as F
    B = 8
    stack = eight_layer_stack(B, _lib.PREC_BF16X6)
    filters = _filters(stack, 21)
    stack.set_filters(filters)
    x = np.random.default_rng(22).uniform(-1, 1, stack.field_shapes[0]).astype(np.float32)
    stack.input.copy_(torch.from_numpy(x))
    stack.step()
    torch.cuda.synchronize()
    assert _lib.LIB.cct_device_status() == _lib.OK
    got = stack.output.double().reshape(B, 512, 28, 28)
    a = torch.from_numpy(x).cuda().double().reshape(B, 3, 224, 224)
    for i, d in enumerate(stack.descs):
        k = d.filter_planes // (d.image_planes // B)
        w = torch.from_numpy(filters[i]).cuda().double().reshape(k, d.image_planes // B, 3, 3)
        a = F.conv2d(a, w, padding=1, stride=d.step if d.sampling == _lib.SAMPLE_DOWN else 1)
        if d.flags & _lib.FLAG_RELU:
            a = a.clamp_min(0)
    err = ((got - a).abs().max() / a.abs().max()).item()
    rms = ((got - a).pow(2).mean() / a.pow(2).mean()).sqrt().item()
    print(f"eight-layer stack, batch 8, BF16X6: normwise max {err:.3e} rms {rms:.3e}")
    assert err <= TOL, err
    stack.close()
