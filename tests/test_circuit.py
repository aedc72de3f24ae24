"""Kernel-circuit buffer assignment (host only, no device).

The rule follows the reference's in-order shared-latch allocator
(runtime/allocation/InOrderSharedLatchAllocator.scala:34): kernels run in the
listed order, a field's buffer may be given to a later field of the same size
once every reader of the field has run, and inputs and outputs keep buffers
of their own.  The checks restate that rule independently and compare.
"""
import pytest

from cctconv import _lib
from cctconv import circuit as K


def _desc(rows, cols, cin, cout, r=3, batch=2, down=1):
    return _lib.new_desc(image_rows=rows, image_cols=cols, image_planes=batch * cin, filter_rows=r, filter_cols=r,
                         filter_planes=cout * cin, batch_size=batch,
                         sampling=_lib.SAMPLE_DOWN if down > 1 else _lib.SAMPLE_NONE, step=down,
                         vector_mode=_lib.PROJECT_FRAME_BLOCK_REDUCE_SUM)


def _elems(inputs, nodes):
    out = [r * c * max(p, 1) for r, c, p in inputs]
    for n in nodes:
        if n.op == _lib.NODE_CONV:
            r, c, p = _lib.output_shape(n.conv)
            out.append(r * c * p)
        else:
            out.append(out[n.in0])
    return out


def _check_rule(inputs, nodes, outputs, fb, nb):
    """Every field's buffer is its own while the field is live (from its
    definition until its last reader has run), fields sharing a buffer have
    the same size, and inputs and outputs never share."""
    nin = len(inputs)
    nf = nin + len(nodes)
    elems = _elems(inputs, nodes)
    last = [-1] * nf
    for i, n in enumerate(nodes):
        last[n.in0] = i
        if n.op in (_lib.NODE_CONV, _lib.NODE_ADD, _lib.NODE_SUB, _lib.NODE_MUL) and n.in1 >= 0:
            last[n.in1] = i
    sealed = set(range(nin)) | set(outputs)
    assert sorted(set(fb)) == list(range(nb))
    for f in range(nf):
        for g in range(nf):
            if f == g or fb[f] != fb[g]:
                continue
            assert elems[f] == elems[g], (f, g)
            assert f not in sealed and g not in sealed, (f, g)
            a, b = (f, g) if f < g else (g, f)
            # a is defined first: its last reader must run before b is written
            a_end = last[a] if last[a] >= 0 else a - nin
            assert a_end < b - nin, f"field {b} reuses field {a}'s buffer while {a} is still read"


def _residual(rows=32, cols=32, c=8):
    d = _desc(rows, cols, c, c)
    nodes = [K.conv(0, d), K.relu(1), K.conv(2, d), K.add(3, 0), K.relu(4),
             K.conv(5, d), K.relu(6), K.conv(7, d), K.add(8, 5), K.relu(9)]
    return [(rows, cols, 2 * c)], nodes, [10]


def test_residual_blocks_share_buffers():
    inputs, nodes, outputs = _residual()
    fb, nb = K.assign(inputs, nodes, outputs)
    _check_rule(inputs, nodes, outputs, fb, nb)
    # input, output, and three buffers cycling through the nine inner fields
    assert nb == 5
    assert fb == [0, 1, 2, 1, 2, 1, 2, 3, 2, 3, 4]


def test_chain_of_convolutions_uses_two_inner_buffers():
    d = _desc(16, 16, 4, 4)
    nodes = [K.conv(0, d)] + [K.conv(i, d) for i in range(1, 8)]
    fb, nb = K.assign([(16, 16, 8)], nodes, [8])
    _check_rule([(16, 16, 8)], nodes, [8], fb, nb)
    assert nb == 4


def test_fields_of_different_sizes_never_share():
    d1 = _desc(32, 32, 4, 8)
    d2 = _desc(32, 32, 8, 8, down=2)
    d3 = _desc(16, 16, 8, 8)
    nodes = [K.conv(0, d1), K.relu(1), K.conv(2, d2), K.relu(3), K.conv(4, d3), K.relu(5)]
    fb, nb = K.assign([(32, 32, 8)], nodes, [6])
    _check_rule([(32, 32, 8)], nodes, [6], fb, nb)
    assert fb[2] != fb[4]


def test_outputs_and_unread_fields():
    d = _desc(16, 16, 4, 4)
    # field 1 is an output read later too; field 3 is read by nobody
    nodes = [K.conv(0, d), K.relu(1), K.scale(2, 0.5), K.add(2, 1)]
    fb, nb = K.assign([(16, 16, 8)], nodes, [1, 4])
    _check_rule([(16, 16, 8)], nodes, [1, 4], fb, nb)
    assert len({fb[0], fb[1], fb[4]}) == 3


def test_dynamic_filter_field_counts_as_read():
    d = _desc(16, 16, 4, 4)
    nodes = [K.relu(1), K.conv(0, d, filter_field=2), K.conv(3, d, filter_field=2)]
    inputs = [(16, 16, 8), (3, 3, 16)]
    fb, nb = K.assign(inputs, nodes, [4])
    _check_rule(inputs, nodes, [4], fb, nb)


@pytest.mark.parametrize("case,message", [
    ("later", "not defined before it"),
    ("shape", "convolves a"),
    ("sizes", "combines fields"),
    ("output", "names field"),
    ("filter", "needs a filter of"),
    ("op", "unknown op"),
])
def test_invalid_circuits_are_rejected(case, message):
    d = _desc(16, 16, 4, 4)
    inputs, outputs = [(16, 16, 8)], [1]
    nodes = [K.conv(0, d)]
    if case == "later":
        nodes = [K.relu(1)]
    elif case == "shape":
        nodes = [K.conv(0, _desc(20, 16, 4, 4))]
    elif case == "sizes":
        inputs = [(16, 16, 8), (16, 16, 4)]
        nodes = [K.add(0, 1)]
        outputs = [2]
    elif case == "output":
        outputs = [7]
    elif case == "filter":
        inputs = [(16, 16, 8), (3, 3, 8)]
        nodes = [K.conv(0, d, filter_field=1)]
        outputs = [2]
    elif case == "op":
        nodes = [_lib.CircuitNode(op=99, in0=0, in1=-1)]
    with pytest.raises(_lib.CctError) as e:
        K.assign(inputs, nodes, outputs)
    assert message in str(e.value)
