"""Request serving over libcctconv (cct_server_*).

A ``Server`` owns a scheduler thread and device memory claimed from free HBM:
requests (a convolution with host buffers, or one step of a resident
``LayerStack`` graph) are admitted as device memory frees up and batched into
persistent launches, with several launches in flight.  ``per_call=True``
gives the plain per-call dispatch serving is compared with: one request at a
time, synchronised.
"""
import ctypes

import numpy as np

from . import _lib


def conv_request(desc, image_ptr, out_ptr, filter_ptr=None, filter_id=-1):
    r = _lib.ServeRequest()
    _lib.LIB.cct_serve_request_init(ctypes.byref(r))
    r.kind = _lib.SERVE_CONV
    r.desc = desc
    r.image, r.out = image_ptr, out_ptr
    r.filter = filter_ptr
    r.filter_id = filter_id
    return r


def graph_request(graph, image_ptr, out_ptr):
    r = _lib.ServeRequest()
    _lib.LIB.cct_serve_request_init(ctypes.byref(r))
    r.kind = _lib.SERVE_GRAPH_STEP
    r.graph = graph.handle.value if hasattr(graph, "handle") else graph
    r.image, r.out = image_ptr, out_ptr
    return r


class Server:
    def __init__(self, slots=3, max_batch=64, arena_bytes=0, per_call=False, hbm_reserve_bytes=0):
        """arena_bytes: cap on the device memory the server holds (0: none,
        requests are admitted by the device's free HBM less
        hbm_reserve_bytes, 0 meaning the library's 2 GiB)."""
        cfg = _lib.ServerConfig()
        _lib.LIB.cct_server_config_init(ctypes.byref(cfg))
        cfg.slots, cfg.max_batch, cfg.arena_bytes = slots, max_batch, arena_bytes
        if hbm_reserve_bytes:
            cfg.hbm_reserve_bytes = hbm_reserve_bytes
        cfg.flags = _lib.SERVE_PER_CALL if per_call else 0
        h = ctypes.c_void_p()
        _lib.check(_lib.LIB.cct_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.handle = h
        self._keep = []

    def add_filter(self, host_filter):
        """Keeps a float32 filter bank resident; returns its id."""
        f = np.ascontiguousarray(host_filter, dtype=np.float32)
        i = ctypes.c_int32()
        _lib.check(_lib.LIB.cct_server_add_filter(self.handle, f.ctypes.data, f.size, ctypes.byref(i)))
        return i.value

    def submit(self, request):
        t = ctypes.c_uint64()
        _lib.check(_lib.LIB.cct_server_submit(self.handle, ctypes.byref(request), ctypes.byref(t)))
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        """Latency in µs once the request is done (raises on its error)."""
        lat = ctypes.c_double()
        _lib.check(_lib.LIB.cct_server_wait(self.handle, ticket, timeout_ms, ctypes.byref(lat)))
        return lat.value

    def replay(self, requests, arrival_s):
        """Open-loop replay: request i submitted at arrival_s[i]; returns latencies (µs)."""
        n = len(requests)
        arr = (_lib.ServeRequest * n)(*requests)
        t = np.ascontiguousarray(arrival_s, dtype=np.float64)
        lat = np.empty(n, dtype=np.float64)
        P = ctypes.POINTER(ctypes.c_double)
        _lib.check(_lib.LIB.cct_server_replay(self.handle, arr, t.ctypes.data_as(P), n,
                                              lat.ctypes.data_as(P)))
        return lat

    def stats(self):
        v = [ctypes.c_uint64() for _ in range(4)]
        _lib.check(_lib.LIB.cct_server_stats(self.handle, *[ctypes.byref(x) for x in v]))
        return dict(zip(("completed", "batches", "solo", "peak_arena_bytes"), (x.value for x in v)))

    def close(self):
        if self.handle:
            _lib.LIB.cct_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
