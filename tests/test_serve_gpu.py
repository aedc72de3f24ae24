"""Request serving: continuous batching gives every request the result it gets
alone, bit for bit, and the FP32 oracle's result.

Requests of uneven sizes (fields 32-1024 on a side, 3x3 to 9x9 filters, 1-64
input planes, 1-64 filters) arrive as a burst; the server admits them as
device memory frees up and batches them into persistent launches.  Each
result is compared with the same request served alone (per-call dispatch,
one request at a time) and with the FP32 oracle.
"""
import numpy as np
import pytest
import torch

import oracle as O
from cctconv import _lib
from cctconv.graph import LayerStack
from cctconv.serve import Server, conv_request, graph_request

pytestmark = pytest.mark.gpu


def _desc(side, R, C, K):
    if K == 1:  # convolve: each of the C planes with one filter
        return _lib.new_desc(image_rows=side, image_cols=side, image_planes=C if C > 1 else 0,
                             filter_rows=R, filter_cols=R, filter_planes=0, batch_size=1,
                             orientation=_lib.CONVOLUTION, vector_mode=_lib.PLANE_BY_PLANE)
    return _lib.new_desc(image_rows=side, image_cols=side, image_planes=C, filter_rows=R,
                         filter_cols=R, filter_planes=K * C, batch_size=1,
                         orientation=_lib.CROSS_CORRELATION,
                         vector_mode=_lib.PROJECT_FRAME_BLOCK_REDUCE_SUM)


def _oracle(side, R, C, K, x, f):
    if K == 1:
        od = O.make_desc(side, side, R, R, planes=C if C > 1 else 0, f_planes=0, orient=O.CONV,
                         mode=O.PLANE)
    else:
        od = O.make_desc(side, side, R, R, planes=C, f_planes=K * C, batch=1, orient=O.XCORR,
                         mode=O.PROJECT_REDUCE)
    return O.conv(od, x, f, np.float32)


class Mix:
    """Seeded requests with pinned host buffers."""

    def __init__(self, n, seed, max_side=200):
        rng = np.random.default_rng(seed)
        self.specs, self.x, self.f, self.outs = [], [], [], []
        for _ in range(n):
            side = int(np.exp(rng.uniform(np.log(32), np.log(max_side))))
            R = int(rng.choice([3, 5, 7, 9]))
            C = int(rng.choice([1, 4, 16]))
            K = int(rng.choice([1, 16]))
            x = torch.from_numpy(rng.uniform(-1, 1, (C, side, side)).astype(np.float32)).pin_memory()
            fp = 1 if K == 1 else K * C
            f = torch.from_numpy(rng.uniform(-1, 1, (fp, R, R)).astype(np.float32)).pin_memory()
            self.specs.append((side, R, C, K))
            self.x.append(x)
            self.f.append(f)

    def requests(self):
        reqs, outs = [], []
        for (side, R, C, K), x, f in zip(self.specs, self.x, self.f):
            planes = C if K == 1 else K
            y = torch.full((planes, side, side), float("nan")).pin_memory()
            outs.append(y)
            reqs.append(conv_request(_desc(side, R, C, K), x.data_ptr(), y.data_ptr(), f.data_ptr()))
        return reqs, outs


def _serve_all(server, reqs):
    tickets = [server.submit(r) for r in reqs]
    return [server.wait(t, 60000) for t in tickets]


def test_results_alone_and_in_the_mix_are_identical_and_exact():
    mix = Mix(48, seed=1)
    alone = Server(per_call=True)
    reqs_a, outs_a = mix.requests()
    _serve_all(alone, reqs_a)
    alone.close()

    server = Server(slots=3, max_batch=16)
    reqs_m, outs_m = mix.requests()
    _serve_all(server, reqs_m)
    st = server.stats()
    server.close()
    assert st["completed"] == len(reqs_m)
    assert st["batches"] < len(reqs_m)  # requests shared launches
    for i, ((side, R, C, K), x, f) in enumerate(zip(mix.specs, mix.x, mix.f)):
        a, m = outs_a[i].numpy(), outs_m[i].numpy()
        assert np.array_equal(a.view(np.uint32), m.view(np.uint32)), (i, mix.specs[i])
        ref = _oracle(side, R, C, K, x.numpy(), f.numpy())
        assert np.array_equal(m.reshape(ref.shape).view(np.uint32), ref.view(np.uint32)), i


# Requests spanning the serving stream's ranges (side 32-1024, 3x3-9x9, 1-64
# planes, 1-64 filters): the largest run alone on their own plan, the small
# ones share batch launches.  (side, R, planes, filters)
WIDE = [(1024, 9, 1, 1), (1024, 3, 64, 1), (1024, 5, 4, 16), (724, 7, 16, 1), (512, 3, 64, 64),
        (362, 9, 16, 16), (256, 5, 64, 16), (181, 3, 4, 64), (128, 9, 64, 1), (90, 7, 16, 64),
        (64, 5, 1, 16), (45, 3, 64, 64), (32, 9, 4, 1), (32, 3, 1, 64), (600, 5, 1, 64),
        (100, 3, 16, 16)]


class SpecMix(Mix):
    def __init__(self, specs, seed):
        rng = np.random.default_rng(seed)
        self.specs, self.x, self.f = [], [], []
        for side, R, C, K in specs:
            self.specs.append((side, R, C, K))
            self.x.append(torch.from_numpy(rng.uniform(-1, 1, (C, side, side)).astype(np.float32)).pin_memory())
            fp = 1 if K == 1 else K * C
            self.f.append(torch.from_numpy(rng.uniform(-1, 1, (fp, R, R)).astype(np.float32)).pin_memory())


def test_serving_ranges_alone_and_in_the_mix_match_the_oracle():
    """Every request of a mix spanning the stream's full size ranges: served
    alone, served in the mix (batched and solo routes both taken), and the
    FP32 oracle agree bit for bit."""
    mix = SpecMix(WIDE, seed=9)
    alone = Server(per_call=True)
    reqs_a, outs_a = mix.requests()
    _serve_all(alone, reqs_a)
    alone.close()
    server = Server(slots=3, max_batch=16)
    reqs_m, outs_m = mix.requests()
    _serve_all(server, reqs_m)
    st = server.stats()
    server.close()
    assert st["completed"] == len(reqs_m)
    assert st["solo"] > 0 and st["batches"] > 0, st  # both routes taken
    for i, ((side, R, C, K), x, f) in enumerate(zip(mix.specs, mix.x, mix.f)):
        a, m = outs_a[i].numpy(), outs_m[i].numpy()
        assert np.array_equal(a.view(np.uint32), m.view(np.uint32)), (i, mix.specs[i])
        ref = _oracle(side, R, C, K, x.numpy(), f.numpy())
        assert np.array_equal(m.reshape(ref.shape).view(np.uint32), ref.view(np.uint32)), (i, mix.specs[i])


def test_admission_waits_for_arena_room():
    """An arena that holds only a few requests at once still serves them all."""
    mix = Mix(24, seed=2, max_side=96)
    reqs, outs = mix.requests()
    server = Server(slots=3, max_batch=8, arena_bytes=8 << 20)
    _serve_all(server, reqs)
    st = server.stats()
    server.close()
    assert st["completed"] == len(reqs)
    assert st["peak_arena_bytes"] <= 8 << 20
    for i, ((side, R, C, K), x, f) in enumerate(zip(mix.specs, mix.x, mix.f)):
        ref = _oracle(side, R, C, K, x.numpy(), f.numpy())
        assert np.array_equal(outs[i].numpy().reshape(ref.shape).view(np.uint32), ref.view(np.uint32)), i


def test_admission_by_free_hbm():
    """With no cap, a server claims device memory from the device's free HBM
    less its reserve: leaving all but 128 MiB of the free memory to other
    work, it still serves every request (within those 128 MiB); a request
    larger than the device's memory less the reserve is rejected at once."""
    free, total = torch.cuda.mem_get_info()
    server = Server(slots=2, max_batch=8, hbm_reserve_bytes=free - (128 << 20))
    mix = Mix(12, seed=3, max_side=128)
    reqs, outs = mix.requests()
    _serve_all(server, reqs)
    st = server.stats()
    server.close()
    assert st["completed"] == len(reqs)
    assert st["peak_arena_bytes"] <= 128 << 20
    for i, ((side, R, C, K), x, f) in enumerate(zip(mix.specs, mix.x, mix.f)):
        ref = _oracle(side, R, C, K, x.numpy(), f.numpy())
        assert np.array_equal(outs[i].numpy().reshape(ref.shape).view(np.uint32), ref.view(np.uint32)), i
    server = Server(hbm_reserve_bytes=total - (64 << 20))
    x = torch.zeros((16, 1024, 1024)).pin_memory()
    y = torch.zeros((16, 1024, 1024)).pin_memory()
    f = torch.zeros((1, 3, 3)).pin_memory()
    with pytest.raises(_lib.CctError, match="arena holds"):  # 128 MiB of fields
        server.submit(conv_request(_desc(1024, 3, 16, 1), x.data_ptr(), y.data_ptr(), f.data_ptr()))
    server.close()


def test_resident_filters_and_rejections():
    server = Server(arena_bytes=4 << 20)
    rng = np.random.default_rng(3)
    f = rng.uniform(-1, 1, (16 * 4, 5, 5)).astype(np.float32)
    fid = server.add_filter(f)
    x = torch.from_numpy(rng.uniform(-1, 1, (4, 64, 64)).astype(np.float32)).pin_memory()
    y = torch.empty((16, 64, 64)).pin_memory()
    d = _desc(64, 5, 4, 16)
    server.wait(server.submit(conv_request(d, x.data_ptr(), y.data_ptr(), None, fid)))
    ref = _oracle(64, 5, 4, 16, x.numpy(), f)
    assert np.array_equal(y.numpy().view(np.uint32), ref.view(np.uint32))
    with pytest.raises(_lib.CctError, match="no resident filter"):
        server.submit(conv_request(d, x.data_ptr(), y.data_ptr(), None, fid + 7))
    big = _desc(1024, 3, 16, 1)  # 64 MiB of fields: never fits a 4 MiB arena
    with pytest.raises(_lib.CctError, match="arena holds"):
        server.submit(conv_request(big, x.data_ptr(), y.data_ptr(), x.data_ptr()))
    with pytest.raises(_lib.CctError, match="FP32"):
        dd = _desc(64, 5, 4, 16)
        dd.precision = _lib.PREC_BF16X3
        server.submit(conv_request(dd, x.data_ptr(), y.data_ptr(), None, fid))
    server.close()


def test_graph_step_requests_match_stepping_the_graph():
    layers = [(16, 3, 1, True), (16, 3, 2, False)]
    stack = LayerStack((32, 32, 3), 1, layers, _lib.PREC_FP32)
    rng = np.random.default_rng(4)
    stack.set_filters([rng.standard_normal(s).astype(np.float32) * 0.2 for s in stack.filter_shapes])
    inputs = [torch.from_numpy(rng.uniform(-1, 1, stack.field_shapes[0]).astype(np.float32)).pin_memory()
              for _ in range(4)]
    # direct stepping
    want = []
    for x in inputs:
        stack.input.copy_(x.cuda())
        stack.step()
        torch.cuda.synchronize()
        want.append(stack.output.cpu().numpy().copy())
    server = Server(slots=2)
    outs = [torch.empty(stack.field_shapes[-1]).pin_memory() for _ in inputs]
    reqs = [graph_request(stack.graph, x.data_ptr(), y.data_ptr()) for x, y in zip(inputs, outs)]
    # interleave convolution requests so graph steps and batches mix
    mix = Mix(6, seed=5, max_side=64)
    creqs, couts = mix.requests()
    tickets = []
    for i, r in enumerate(reqs):
        tickets.append(server.submit(r))
        tickets.append(server.submit(creqs[i]))
    for t in tickets:
        server.wait(t, 60000)
    server.close()
    for w, y in zip(want, outs):
        assert np.array_equal(w, y.numpy())
    stack.close()


def test_replay_reports_latencies():
    mix = Mix(40, seed=6, max_side=128)
    reqs, outs = mix.requests()
    server = Server(slots=3, max_batch=16)
    arrivals = np.cumsum(np.random.default_rng(7).exponential(1 / 2000.0, len(reqs)))
    lat = server.replay(reqs, arrivals)
    server.close()
    assert (lat > 0).all() and np.isfinite(lat).all()
    for i, ((side, R, C, K), x, f) in enumerate(zip(mix.specs, mix.x, mix.f)):
        if i % 5 == 0:
            ref = _oracle(side, R, C, K, x.numpy(), f.numpy())
            assert np.array_equal(outs[i].numpy().reshape(ref.shape).view(np.uint32), ref.view(np.uint32))
