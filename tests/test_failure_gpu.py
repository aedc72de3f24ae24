"""Failure detection on the device, without a GPU fault: a kernel whose
mbarrier wait never completes gives up after its time limit, records the
timeout, and returns; the host reads CCT_ETIMEOUT and the context keeps
working."""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O
from cctconv import _lib

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives():
    assert _lib.LIB.cct_device_status() == _lib.OK  # nothing pending
    ms = ctypes.c_double()
    assert _lib.LIB.cct_selftest_wait_timeout(ctypes.byref(ms)) == _lib.OK
    assert 500.0 <= ms.value <= 10000.0, ms.value  # about one second
    assert _lib.LIB.cct_device_status() == _lib.ETIMEOUT
    assert b"bounded wait" in _lib.LIB.cct_last_error_string()
    assert _lib.LIB.cct_device_status() == _lib.OK  # reading clears it
    # the context still runs kernels correctly
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, (64, 64)).astype(np.float32)
    f = rng.uniform(-1, 1, (5, 5)).astype(np.float32)
    desc = _lib.new_desc(image_rows=64, image_cols=64, filter_rows=5, filter_cols=5)
    plan = _lib.Plan(desc)
    xd, fd = torch.from_numpy(x).cuda(), torch.from_numpy(f).cuda()
    y = torch.empty((64, 64), device="cuda")
    plan.run(xd.data_ptr(), fd.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    plan.close()
    ref = O.conv(O.make_desc(64, 64, 5, 5), x, f, np.float32)
    assert np.array_equal(y.cpu().numpy().reshape(ref.shape), ref)
