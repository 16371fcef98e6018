"""ctypes binding of the C ABI in include/mqp.h (libmqp_b200.so).

The library is built in-tree by ``python -m multi_quickpiv_b200.build``.
There is no fallback: when the library is missing, loading fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libmqp_b200.so")

MQP_OK = 0
MQP_ERR_INVALID = -1
MQP_ERR_UNSUPPORTED = -2
MQP_ERR_CUDA = -3
MQP_ERR_OOM = -4
MQP_ERR_TIMEOUT = -5
MQP_ERR_BUSY = -6
MQP_ERR_NOT_FOUND = -7

MQP_FFTCC, MQP_ZNCC, MQP_NSQECC, MQP_MASK_NSQECC = 0, 1, 2, 3
MQP_TUNE_CHUNK3D, MQP_TUNE_CHUNK3D_BUDGET, MQP_TUNE_HOST_PIECES = 1, 2, 3
MQP_F32, MQP_F64 = 0, 1

# every symbol declared in include/mqp.h, with its ctypes signature
I64x3 = C.c_int64 * 3


class MqpParams(C.Structure):
    _fields_ = [
        ("corr_alg", C.c_int32),
        ("interSize", C.c_int32 * 3),
        ("searchMargin", C.c_int32 * 3),
        ("overlap", C.c_int32 * 3),
        ("step", C.c_int32 * 3),
        ("has_step", C.c_int32),
        ("multipass", C.c_int32),
        ("computeSN", C.c_int32),
        ("unpadded", C.c_int32),
        ("good_pad", C.c_int32),
        ("odd_pad", C.c_int32),
        ("threshold", C.c_double),
        ("mask_threshold", C.c_double),
        ("ovp_th", C.c_double),
        ("refine", C.c_int32),
        ("reserved", C.c_int32 * 7),
    ]


class MqpProfile(C.Structure):
    _fields_ = [
        ("launches_integral", C.c_int64),
        ("launches_piv", C.c_int64),
        ("launches_other", C.c_int64),
        ("ms_integral", C.c_double),
        ("ms_piv", C.c_double),
        ("ms_other", C.c_double),
        ("ia_count", C.c_int64),
    ]


class MqpBatchItem(C.Structure):
    _fields_ = [
        ("img1", C.c_void_p), ("img2", C.c_void_p), ("mask", C.c_void_p), ("mask_skip", C.c_void_p),
        ("dtype", C.c_int32), ("ndims", C.c_int32), ("dims", C.c_int64 * 3),
        ("params", MqpParams),
        ("VF", C.c_void_p), ("SN", C.c_void_p),
    ]


class MqpBatchOptions(C.Structure):
    _fields_ = [("use_graph", C.c_int32), ("grab", C.c_int32), ("chunk3d", C.c_int64),
                ("chunk3d_budget", C.c_int64), ("reserved", C.c_int32 * 8)]


class MqpServerOptions(C.Structure):
    _fields_ = [("slots", C.c_int32), ("reserved0", C.c_int32), ("hbm_budget_bytes", C.c_int64),
                ("hbm_reserve_bytes", C.c_int64), ("chunk3d_budget", C.c_int64), ("reserved", C.c_int32 * 8)]


class MqpServerStats(C.Structure):
    _fields_ = [("completed", C.c_int64), ("failed", C.c_int64), ("queued", C.c_int64), ("running", C.c_int64),
                ("admitted_while_busy", C.c_int64), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("max_ms", C.c_double), ("ia_done", C.c_int64), ("ia_per_s", C.c_double),
                ("budget_bytes", C.c_int64), ("in_use_bytes", C.c_int64), ("wait_p50_ms", C.c_double),
                ("wait_p99_ms", C.c_double), ("run_p50_ms", C.c_double), ("run_p99_ms", C.c_double)]


class MqpField(C.Structure):
    _fields_ = [("ncomp", C.c_int32), ("ndims", C.c_int32), ("dims", C.c_int64 * 4)]


class MqpPostParams(C.Structure):
    _fields_ = [
        ("op", C.c_int32),
        ("radius", C.c_int32 * 4),
        ("max_angle", C.c_double),
        ("normalize", C.c_int32),
        ("scale_by_similarity", C.c_int32),
        ("similarity_exponent", C.c_double),
        ("threshold", C.c_double),
        ("cmp", C.c_int32),
        ("replace", C.c_int32),
        ("min_speed", C.c_double),
        ("divide_by", C.c_int32),
        ("circle", C.c_int32),
        ("reserved", C.c_int32 * 8),
    ]


class MqpTiffInfo(C.Structure):
    _fields_ = [("width", C.c_int64), ("height", C.c_int64), ("pages", C.c_int64), ("bits", C.c_int32),
                ("sample_format", C.c_int32), ("compression", C.c_int32), ("tiled", C.c_int32),
                ("uniform", C.c_int32)]


class MqpTrajParams(C.Structure):
    _fields_ = [
        ("ndims", C.c_int32),
        ("dims", C.c_int64 * 3),
        ("frames", C.c_int64),
        ("T0", C.c_int32),
        ("T1", C.c_int32),
        ("sub_lo", C.c_int64 * 3),
        ("sub_hi", C.c_int64 * 3),
        ("step", C.c_int64 * 3),
        ("scale", C.c_double * 3),
        ("grid", C.c_int32),
        ("numpoints", C.c_int64),
        ("seed", C.c_uint64),
        ("reserved", C.c_int32 * 8),
    ]


(MQP_POST_MAGNITUDES, MQP_POST_AVERAGE, MQP_POST_SIMILARITY_AVG, MQP_POST_COLLECTIVENESS, MQP_POST_TH_MASK,
 MQP_POST_STD_MASK, MQP_POST_REPLACE, MQP_POST_LOCAL_MAGNITUDE, MQP_POST_MATLAB_DIVERGENCE,
 MQP_POST_DIVERGENCE) = range(10)
MQP_REPLACE_ZERO, MQP_REPLACE_MEDIAN, MQP_REPLACE_MEAN = 0, 1, 2
MQP_DIVIDE_NONE, MQP_DIVIDE_N, MQP_DIVIDE_MAGS = 0, 1, 2

SIGNATURES = {
    "mqp_abi_version": (C.c_int, []),
    "mqp_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    "mqp_destroy": (C.c_int, [C.c_void_p]),
    "mqp_last_error": (C.c_char_p, [C.c_void_p]),
    "mqp_vf_dims": (C.c_int, [C.POINTER(MqpParams), C.c_int, I64x3, I64x3]),
    "mqp_piv": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                          I64x3, C.POINTER(MqpParams), C.c_void_p, C.c_void_p, I64x3]),
    "mqp_piv_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                 I64x3, C.POINTER(MqpParams), C.c_void_p, C.c_void_p, C.c_void_p]),
    "mqp_correlation_planes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                         I64x3, C.POINTER(MqpParams), C.c_int64, C.c_int64, C.c_void_p]),
    "mqp_piv2d_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int64 * 2, C.POINTER(MqpParams),
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p, C.c_int]),
    "mqp_profile_enable": (C.c_int, [C.c_void_p, C.c_int]),
    "mqp_profile_read": (C.c_int, [C.c_void_p, C.POINTER(MqpProfile)]),
    "mqp_set_tuning": (C.c_int, [C.c_void_p, C.c_int, C.c_int64]),
    "mqp_batch_plan_create": (C.c_int, [C.c_void_p, C.POINTER(MqpBatchItem), C.c_int32, C.POINTER(MqpBatchOptions),
                                        C.POINTER(C.c_void_p)]),
    "mqp_batch_plan_run": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mqp_batch_plan_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "mqp_batch_plan_destroy": (C.c_int, [C.c_void_p]),
    "mqp_server_create": (C.c_int, [C.c_int, C.POINTER(MqpServerOptions), C.POINTER(C.c_void_p)]),
    "mqp_server_open_stream": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, I64x3, C.POINTER(MqpParams),
                                         C.POINTER(C.c_int32)]),
    "mqp_server_submit": (C.c_int, [C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_uint64)]),
    "mqp_server_result": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p, C.c_void_p,
                                    C.POINTER(C.c_double)]),
    "mqp_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(MqpServerStats)]),
    "mqp_server_reset_stats": (C.c_int, [C.c_void_p]),
    "mqp_server_last_error": (C.c_char_p, [C.c_void_p]),
    "mqp_server_destroy": (C.c_int, [C.c_void_p]),
    "mqp_postprocess_device": (C.c_int, [C.c_void_p, C.POINTER(MqpPostParams), C.POINTER(MqpField), C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mqp_postprocess": (C.c_int, [C.c_void_p, C.POINTER(MqpPostParams), C.POINTER(MqpField), C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mqp_tiff_open": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "mqp_tiff_get_info": (C.c_int, [C.c_void_p, C.POINTER(MqpTiffInfo)]),
    "mqp_tiff_read": (C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_int, C.c_void_p]),
    "mqp_tiff_last_error": (C.c_char_p, [C.c_void_p]),
    "mqp_tiff_close": (C.c_int, [C.c_void_p]),
    "mqp_frame_source_create": (C.c_int, [C.c_char_p, C.c_int64, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "mqp_frame_source_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), I64x3, C.POINTER(C.c_int32)]),
    "mqp_frame_source_next": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_int64)]),
    "mqp_frame_source_last_error": (C.c_char_p, [C.c_void_p]),
    "mqp_frame_source_destroy": (C.c_int, [C.c_void_p]),
    "mqp_traj_count": (C.c_int, [C.POINTER(MqpTrajParams), C.POINTER(C.c_int64)]),
    "mqp_trajectories_device": (C.c_int, [C.c_void_p, C.POINTER(MqpTrajParams), C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "mqp_trajectories": (C.c_int, [C.c_void_p, C.POINTER(MqpTrajParams), C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
}

_lib = None
_lock = threading.Lock()


class MQPError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[mqp {code}] {msg}")
        self.code = code


def load(path: str = LIB_PATH):
    """Load libmqp_b200.so (cached).  Raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise ImportError(f"native library {path} is missing: build it with "
                              "`python -m multi_quickpiv_b200.build` (there is no CPU fallback)")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(rc: int, ctx=None):
    if rc != MQP_OK:
        lib = load()
        msg = lib.mqp_last_error(ctx)
        raise MQPError(rc, msg.decode() if msg else "unknown error")


class Context:
    """An mqp_ctx bound to one CUDA device (owns device buffers + a stream)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.mqp_create(C.byref(h), int(device)), None)
        self.handle = h
        self.device = device

    def profile_enable(self, on: bool = True):
        check(self.lib.mqp_profile_enable(self.handle, int(on)), self.handle)

    def profile_read(self) -> dict:
        out = MqpProfile()
        check(self.lib.mqp_profile_read(self.handle, C.byref(out)), self.handle)
        return {f: getattr(out, f) for f, _ in MqpProfile._fields_}

    def set_chunk3d(self, ias: int = 0, budget_bytes: int = 0):
        """IAs per 3D chunk (0: as many as budget_bytes of scratch hold)."""
        check(self.lib.mqp_set_tuning(self.handle, MQP_TUNE_CHUNK3D, int(ias)), self.handle)
        check(self.lib.mqp_set_tuning(self.handle, MQP_TUNE_CHUNK3D_BUDGET, int(budget_bytes)), self.handle)

    def set_host_pieces(self, pieces: int = 3):
        """Column pieces of the pipelined host-array 2D path (1: copy first)."""
        check(self.lib.mqp_set_tuning(self.handle, MQP_TUNE_HOST_PIECES, int(pieces)), self.handle)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.mqp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_ctx_cache = {}


def default_context(device: int = 0) -> Context:
    with _lock:
        c = _ctx_cache.get(device)
    if c is None:
        c = Context(device)
        with _lock:
            _ctx_cache[device] = c
    return c
