"""Serving time-lapse PIV (include/mqp.h, mqp_server_*): each stream keeps its
last frames and their integral images on the device; every submitted frame
t+1 becomes a request PIV(frame t, frame t+1) that a worker thread admits as
execution slots and device memory free up, overlapping on the device with
the other requests.  Results equal PIV() on the same pair.

    srv = Server(slots=4)
    sid = srv.open_stream(frame0, setPIVParameters(interSize=32, searchMargin=16, step=8))
    rid = srv.submit(sid, frame1)
    VF, SN, latency_ms = srv.result(rid)
    srv.stats()   # p50 / p99 latency, IA/s, requests admitted while others ran
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from .piv import PIVParameters, get_vectorfield_size


class Server:
    def __init__(self, device: int = 0, slots: int = 4, hbm_budget_bytes: int = 0, chunk3d_budget: int = 0):
        self.lib = _lib.load()
        o = _lib.MqpServerOptions()
        o.slots = slots
        o.hbm_budget_bytes = hbm_budget_bytes
        o.chunk3d_budget = chunk3d_budget
        h = C.c_void_p()
        rc = self.lib.mqp_server_create(int(device), C.byref(o), C.byref(h))
        if rc != _lib.MQP_OK:
            raise _lib.MQPError(rc, "mqp_server_create failed")
        self.handle = h
        self._streams = {}

    def _check(self, rc):
        if rc != _lib.MQP_OK:
            msg = self.lib.mqp_server_last_error(self.handle)
            raise _lib.MQPError(rc, msg.decode() if msg else "server error")

    def open_stream(self, first_frame, params: PIVParameters) -> int:
        """A time-lapse stream: its first frame and the parameters of every request."""
        a = np.asarray(first_frame)
        nd = a.ndim
        params.ndims = nd
        dt = np.float64 if a.dtype == np.float64 else np.float32
        f = np.asfortranarray(a, dtype=dt)
        dims = (C.c_int64 * 3)(*(list(a.shape) + [1] * (3 - nd)))
        sid = C.c_int32()
        cp = params.to_c()
        self._check(self.lib.mqp_server_open_stream(self.handle, f.ctypes.data_as(C.c_void_p),
                                                    _lib.MQP_F64 if dt == np.float64 else _lib.MQP_F32, nd, dims,
                                                    C.byref(cp), C.byref(sid)))
        vf = tuple(get_vectorfield_size(a.shape, params))
        self._streams[sid.value] = (a.shape, dt, vf, bool(params.computeSN))
        return sid.value

    def submit(self, stream_id: int, frame) -> int:
        shape, dt, _, _ = self._streams[stream_id]
        f = np.asfortranarray(np.asarray(frame), dtype=dt)
        if f.shape != shape:
            raise AssertionError("PIV inputs need to have the same size.")
        rid = C.c_uint64()
        self._check(self.lib.mqp_server_submit(self.handle, int(stream_id), f.ctypes.data_as(C.c_void_p),
                                               C.byref(rid)))
        self._req_stream = getattr(self, "_req_stream", {})
        self._req_stream[rid.value] = stream_id
        return rid.value

    def result(self, request_id: int, wait_ms: int = -1):
        """(VF, SN or None, latency_ms) of a request; waits (wait_ms < 0), polls
        (0) or waits at most wait_ms."""
        sid = self._req_stream[request_id]
        shape, _, vf, sn = self._streams[sid]
        nd = len(shape)
        VF = np.zeros((nd,) + vf, dtype=np.float64, order="F")
        SN = np.zeros(vf, dtype=np.float64, order="F") if sn else None
        lat = C.c_double()
        self._check(self.lib.mqp_server_result(self.handle, C.c_uint64(request_id), int(wait_ms),
                                               VF.ctypes.data_as(C.c_void_p),
                                               SN.ctypes.data_as(C.c_void_p) if SN is not None else None,
                                               C.byref(lat)))
        del self._req_stream[request_id]
        return VF, SN, lat.value

    def stats(self) -> dict:
        st = _lib.MqpServerStats()
        self._check(self.lib.mqp_server_get_stats(self.handle, C.byref(st)))
        return {f: getattr(st, f) for f, _ in _lib.MqpServerStats._fields_}

    def reset_stats(self):
        self._check(self.lib.mqp_server_reset_stats(self.handle))

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mqp_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
