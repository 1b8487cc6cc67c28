"""Python binding of the served form (include/visar_serve.h).

    srv = Server(pool_bytes=8 << 30)              # or mode=PLAIN for the per-call baseline
    rid = srv.submit(x, [batch.gaussian((5, 5)), batch.resize(0.5, 0.5)])
    y = srv.wait(rid)                              # torch view of the result (device)
    srv.release(rid)                               # after y is no longer used

Inputs are CUDA tensors that stay valid until their request completes.
"""
import ctypes

import numpy as np

from . import Image, _check, desc, lib
from .batch import Stage, _as_tensor

BATCHED, PLAIN = 0, 1


class ServerConfig(ctypes.Structure):
    _fields_ = [("pool_bytes", ctypes.c_size_t), ("mode", ctypes.c_int), ("max_inflight", ctypes.c_int),
                ("streams", ctypes.c_int)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("released", ctypes.c_uint64),
                ("rounds", ctypes.c_uint64), ("launches", ctypes.c_uint64), ("fallback_calls", ctypes.c_uint64),
                ("pool_bytes", ctypes.c_size_t), ("pool_used", ctypes.c_size_t), ("pool_reserved", ctypes.c_size_t),
                ("mean_batch", ctypes.c_double), ("deferred", ctypes.c_uint64), ("solo", ctypes.c_uint64),
                ("schedule_s", ctypes.c_double), ("build_s", ctypes.c_double), ("upload_s", ctypes.c_double),
                ("launch_s", ctypes.c_double)]


class TraceRequest(ctypes.Structure):
    _fields_ = [("arrival_s", ctypes.c_double), ("input", Image), ("stages", ctypes.POINTER(Stage)),
                ("nstages", ctypes.c_size_t)]


lib.visar_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(ctypes.c_void_p)]
lib.visar_server_submit.argtypes = [ctypes.c_void_p, ctypes.POINTER(Image), ctypes.POINTER(Stage), ctypes.c_size_t,
                                    ctypes.POINTER(ctypes.c_uint64)]
lib.visar_server_poll.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(Image)]
lib.visar_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Image)]
lib.visar_server_release.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
lib.visar_server_get_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ServerStats)]
lib.visar_server_destroy.argtypes = [ctypes.c_void_p]
lib.visar_server_destroy.restype = None
lib.visar_server_fake_round_error.argtypes = [ctypes.c_void_p, ctypes.c_int]
lib.visar_server_run_trace.argtypes = [ctypes.c_void_p, ctypes.POINTER(TraceRequest), ctypes.c_size_t,
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]


def _stage_array(stages):
    """ctypes array of visar_stage from the batch module's stage builders; warp
    stages carry their (single) matrix in d[]."""
    arr = (Stage * len(stages))()
    keep = []
    for k, (st, kp) in enumerate(stages):
        arr[k] = st
        if kp is not None:  # a per-image matrix given for one request: move it into d[]
            m = np.asarray(kp, np.float64).ravel()
            for j in range(len(m)):
                arr[k].d[j] = float(m[j])
            arr[k].per_image = None
        keep.append(kp)
    return arr, keep


class Server:
    def __init__(self, pool_bytes=0, mode=BATCHED, max_inflight=0, streams=0):
        cfg = ServerConfig(pool_bytes, mode, max_inflight, streams)
        h = ctypes.c_void_p()
        _check(lib.visar_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._keep = {}

    def close(self):
        if getattr(self, "_h", None) and lib is not None:  # (module globals are gone at interpreter exit)
            lib.visar_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def submit(self, x, stages):
        arr, keep = _stage_array(stages)
        rid = ctypes.c_uint64()
        _check(lib.visar_server_submit(self._h, ctypes.byref(desc(x)), arr, len(stages), ctypes.byref(rid)))
        self._keep[rid.value] = (x, arr, keep)
        return rid.value

    def poll(self, rid):
        done = ctypes.c_int()
        img = Image()
        _check(lib.visar_server_poll(self._h, rid, ctypes.byref(done), ctypes.byref(img)))
        return _as_tensor(img, self) if done.value else None

    def wait(self, rid):
        img = Image()
        _check(lib.visar_server_wait(self._h, rid, ctypes.byref(img)))
        return _as_tensor(img, self)

    def release(self, rid):
        _check(lib.visar_server_release(self._h, rid))
        self._keep.pop(rid, None)

    def stats(self):
        st = ServerStats()
        _check(lib.visar_server_get_stats(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def fake_round_error(self, cuda_error):
        """The next completed scheduling round reports `cuda_error` (a
        cudaError_t value) as if the device had raised it (failure-path tests)."""
        _check(lib.visar_server_fake_round_error(self._h, int(cuda_error)))

    def run_trace(self, trace):
        """trace: list of (arrival_s, tensor, stages). Returns (latency_ms array, elapsed_s)."""
        n = len(trace)
        reqs = (TraceRequest * max(1, n))()
        keep = []
        for i, (t, x, stages) in enumerate(trace):
            arr, kp = _stage_array(stages)
            keep.append((x, arr, kp))
            reqs[i].arrival_s = float(t)
            reqs[i].input = desc(x)
            reqs[i].stages = ctypes.cast(arr, ctypes.POINTER(Stage))
            reqs[i].nstages = len(stages)
        lat = (ctypes.c_double * max(1, n))()
        el = ctypes.c_double()
        _check(lib.visar_server_run_trace(self._h, reqs, n, lat, ctypes.byref(el)))
        return np.array(lat[:n]), el.value
