"""Time-lapse ingest (include/mqp.h, mqp_tiff_* and mqp_frame_source_*):
multi-page TIFF stacks read natively into Julia-ordered arrays (dimension 1 =
image rows), and a frame source that reads frames ahead into pinned host
buffers and feeds a serving stream.  The reference reads such stacks with
LIBTIFF before calling PIV on consecutive frames (README.md:55-68).

    img = read_tiff("stack.tif", 0)                     # page 0: (H, W)
    vol = read_tiff("stack.tif", 0, 64)                 # pages 0..63: (H, W, 64)
    for k, frame in FrameSource("stack.tif"):           # 2D+t frames, read ahead
        ...
    for rid in serve_tiff(srv, "stack.tif", params):    # request per frame t+1
        VF, SN, ms = srv.result(rid)
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib


def _code(dtype):
    return _lib.MQP_F64 if np.dtype(dtype) == np.float64 else _lib.MQP_F32


class TiffFile:
    """An open (memory-mapped) TIFF file: info() and read()."""

    def __init__(self, path):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.mqp_tiff_open(os.fsencode(path), C.byref(h))
        self.handle = h
        if rc != _lib.MQP_OK:
            msg = self.lib.mqp_tiff_last_error(h).decode() if h else "cannot open"
            self.close()
            raise _lib.MQPError(rc, f"{path}: {msg}")

    def info(self) -> dict:
        i = _lib.MqpTiffInfo()
        _lib.check(self.lib.mqp_tiff_get_info(self.handle, C.byref(i)), None)
        return {f: getattr(i, f) for f, _ in _lib.MqpTiffInfo._fields_}

    def read(self, first_page=0, npages=None, dtype=np.float32) -> np.ndarray:
        """Pages [first_page, first_page + npages) as an (H, W) array for one
        page or (H, W, npages) otherwise, column-major, of dtype."""
        info = self.info()
        one = npages is None
        n = 1 if one else int(npages)
        out = np.zeros((info["height"], info["width"], n), dtype=np.dtype(dtype), order="F")
        rc = self.lib.mqp_tiff_read(self.handle, int(first_page), n, _code(dtype), out.ctypes.data_as(C.c_void_p))
        if rc != _lib.MQP_OK:
            raise _lib.MQPError(rc, self.lib.mqp_tiff_last_error(self.handle).decode())
        return out[:, :, 0] if one else out

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mqp_tiff_close(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tiff_info(path) -> dict:
    with TiffFile(path) as t:
        return t.info()


def read_tiff(path, first_page=0, npages=None, dtype=np.float32) -> np.ndarray:
    with TiffFile(path) as t:
        return t.read(first_page, npages, dtype)


class FrameSource:
    """Frames of pages_per_frame consecutive pages (1: 2D+t; the depth: 3D+t),
    read ahead by a native thread into a ring of pinned host buffers.
    Iterating yields (index, frame); a frame is a view of a ring buffer, valid
    until the next one is taken (copy it to keep it)."""

    def __init__(self, path, pages_per_frame=1, dtype=np.float32, ring=3):
        self.lib = _lib.load()
        self.dtype = np.dtype(dtype)
        h = C.c_void_p()
        rc = self.lib.mqp_frame_source_create(os.fsencode(path), int(pages_per_frame), _code(dtype), int(ring),
                                              C.byref(h))
        self.handle = h
        if rc != _lib.MQP_OK:
            msg = self.lib.mqp_frame_source_last_error(h).decode() if h else "cannot create"
            self.close()
            raise _lib.MQPError(rc, f"{path}: {msg}")
        frames, dims, pinned = C.c_int64(), (C.c_int64 * 3)(), C.c_int32()
        _lib.check(self.lib.mqp_frame_source_info(self.handle, C.byref(frames), dims, C.byref(pinned)), None)
        self.frames = frames.value
        self.shape = (dims[0], dims[1]) if pages_per_frame == 1 else (dims[0], dims[1], dims[2])
        self.pinned = bool(pinned.value)

    def next(self):
        """(index, frame) of the next frame, or None after the last."""
        ptr, idx = C.c_void_p(), C.c_int64()
        rc = self.lib.mqp_frame_source_next(self.handle, C.byref(ptr), C.byref(idx))
        if rc == _lib.MQP_ERR_NOT_FOUND:
            return None
        if rc != _lib.MQP_OK:
            raise _lib.MQPError(rc, self.lib.mqp_frame_source_last_error(self.handle).decode())
        n = int(np.prod(self.shape))
        buf = (C.c_char * (n * self.dtype.itemsize)).from_address(ptr.value)
        flat = np.frombuffer(buf, dtype=self.dtype, count=n)
        return idx.value, flat.reshape(self.shape, order="F")

    def __iter__(self):
        while True:
            r = self.next()
            if r is None:
                return
            yield r

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mqp_frame_source_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve_tiff(server, path, params, pages_per_frame=1, dtype=np.float32, ring=3):
    """A served time-lapse stream straight from a TIFF stack: opens a stream
    on the first frame, then submits PIV(frame t, frame t+1) for every
    following frame as it is read ahead; yields each request id (collect the
    results with server.result)."""
    with FrameSource(path, pages_per_frame, dtype, ring) as src:
        first = src.next()
        if first is None:
            return
        sid = server.open_stream(first[1], params)
        for _, frame in src:
            yield server.submit(sid, frame)
