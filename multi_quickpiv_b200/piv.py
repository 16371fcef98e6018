"""Host-side mirror of multi_quickPIV's PIV API, driving the sm_100a kernels.

Same names, argument meanings and error behaviour as the Julia package:

    pivparams = setPIVParameters(interSize=(32, 32), searchMargin=(16, 16),
                                 step=(16, 16), threshold=1000)
    VF, SN = PIV(img1, img2, pivparams)            # src/multi_quickPIV.jl:17-19
    VF, SN = PIV(img1, img2, mask, pivparams)      # masked NSQECC (:22-24)

Arrays keep Julia's logical axes: axis 0 of a NumPy array is Julia's
dimension 1.  ``VF`` has shape (N, vf_1, ..., vf_N) (``VF[0]`` = U along
dimension 1), ``SN`` has shape (vf_1, ..., vf_N) or is None.  CUDA tensors
(torch) are processed in place on their device and the results are CUDA
tensors.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, replace
from typing import Callable, Optional, Tuple

import numpy as np

from . import _lib


def maxval(a) -> float:
    """maxval (src/utils/common_ops.jl:29-47): the skip filter function.  It is
    the only filter the native path evaluates."""
    return float(np.max(a))


def toDims3(x):
    """toDims3 (src/piv_parameters.jl:8-11)."""
    if x is None:
        return None
    if isinstance(x, (int, np.integer)):
        return (int(x),) * 3
    x = tuple(int(v) for v in x)
    if len(x) == 2:
        return (x[0], x[1], 0)
    if len(x) == 3:
        return x
    raise TypeError("expected an Integer, a 2-tuple or a 3-tuple")


_ALG_NAMES = {"fftcc": _lib.MQP_FFTCC, "zncc": _lib.MQP_ZNCC, "nsqecc": _lib.MQP_NSQECC}


def parseCorr(corr: str) -> str:
    """parseCorr (src/piv_parameters.jl:13-22).  The reference maps "znc",
    "fftc" and "nsqec" to types it never defines (UndefVarError); those raise
    here.  Any other unknown string selects NSQECC, as in the reference."""
    c = corr.lower()
    if c == "zncc":
        return "zncc"
    if c == "fft":
        return "fftcc"
    if c == "nsqecc":
        return "nsqecc"
    if c in ("znc", "fftc", "nsqec"):
        raise NameError(f"UndefVarError: the correlation type for {corr!r} is not defined")
    return "nsqecc"


@dataclass
class PIVParameters:
    """PIVParameters (src/piv_parameters.jl:28-45).  Field values are the
    stored ones (see setPIVParameters for the unpadded/good_pad swap)."""
    corr_alg: str = "nsqecc"
    unpadded: bool = True
    good_pad: bool = True
    odd_pad: bool = False
    interSize: Tuple[int, int, int] = (32, 32, 32)
    searchMargin: Tuple[int, int, int] = (10, 10, 10)
    overlap: Tuple[int, int, int] = (0, 0, 0)
    step: Optional[Tuple[int, int, int]] = None
    multipass: int = 1
    computeSN: bool = False
    filtFun: Callable = maxval
    threshold: float = -1.0
    mask_filtFun: Callable = maxval
    mask_threshold: float = -1.0
    ndims: int = 3
    ovp_th: float = 0.5
    # beyond the reference: multi-pass refinement.  False / 0: the reference's
    # loop (every pass repeats scale 1); True / 1 / "shift": whole-pixel
    # predictor shifts; 2 / "deform": window deformation around the
    # interpolated predictor (no masks)
    refine: object = False

    def to_c(self) -> _lib.MqpParams:
        if self.filtFun is not maxval or self.mask_filtFun is not maxval:
            raise NotImplementedError("only filtFun = maxval crosses the native boundary")
        p = _lib.MqpParams()
        p.corr_alg = _ALG_NAMES[self.corr_alg]
        for d in range(3):
            p.interSize[d] = int(self.interSize[d])
            p.searchMargin[d] = int(self.searchMargin[d])
            p.overlap[d] = int(self.overlap[d])
            p.step[d] = int(self.step[d]) if self.step is not None else 0
        p.has_step = 0 if self.step is None else 1
        p.multipass = int(self.multipass)
        p.computeSN = int(bool(self.computeSN))
        p.unpadded = int(bool(self.unpadded))
        p.good_pad = int(bool(self.good_pad))
        p.odd_pad = int(bool(self.odd_pad))
        p.threshold = float(self.threshold)
        p.mask_threshold = float(self.mask_threshold)
        p.ovp_th = float(self.ovp_th)
        p.refine = refine_code(self.refine)
        return p


def refine_code(refine) -> int:
    """mqp_params.refine for PIVParameters.refine: 0 (False), 1 (True or
    "shift": whole-pixel predictors) or 2 ("deform": window deformation)."""
    if isinstance(refine, str):
        codes = {"none": 0, "shift": 1, "deform": 2}
        if refine not in codes:
            raise ValueError(f"refine must be one of {sorted(codes)} or 0, 1, 2")
        return codes[refine]
    if isinstance(refine, (bool, np.bool_)):
        return int(refine)
    r = int(refine)
    if r not in (0, 1, 2):
        raise ValueError("refine must be 0, 1 or 2")
    return r


def setPIVParameters(corr_alg="nsqecc", unpadded=True, good_pad=True, odd_pad=False,
                     interSize=32, searchMargin=10, overlap=0, step=None,
                     multipass=1, computeSN=False, filtFun=maxval, threshold=-1.0,
                     mask_filtFun=maxval, mask_threshold=-1.0, ndims=3, ovp_th=0.5,
                     refine=False) -> PIVParameters:
    """setPIVParameters (src/piv_parameters.jl:67-81).  Like the reference's
    positional constructor (:48-64) it stores ``good_pad`` in ``unpadded``
    and ``unpadded`` in ``good_pad``."""
    return PIVParameters(parseCorr(corr_alg), bool(good_pad), bool(unpadded), bool(odd_pad),
                         toDims3(interSize), toDims3(searchMargin), toDims3(overlap), toDims3(step),
                         int(multipass), bool(computeSN), filtFun, float(threshold), mask_filtFun,
                         float(mask_threshold), int(ndims), float(ovp_th), refine)


def _ovp(p: PIVParameters, scale=1):
    """_ovp (src/piv_parameters.jl:83)."""
    return tuple(v * scale for v in p.overlap[:p.ndims])


def _isize(p: PIVParameters, scale=1):
    """_isize (src/piv_parameters.jl:84)."""
    return tuple(v * scale for v in p.interSize[:p.ndims])


def _smarg(p: PIVParameters, scale=1):
    """_smarg (src/piv_parameters.jl:85)."""
    return tuple(v * scale for v in p.searchMargin[:p.ndims])


def _ssize(p: PIVParameters, scale=1):
    """_ssize (src/piv_parameters.jl:86)."""
    return tuple(i + 2 * m for i, m in zip(_isize(p, scale), _smarg(p, scale)))


def _step(p: PIVParameters, scale=1):
    """_step (src/piv_parameters.jl:87)."""
    if p.step is None:
        return tuple(i - o for i, o in zip(_isize(p, scale), _ovp(p, scale)))
    return tuple(v * scale for v in p.step[:p.ndims])


def get_vectorfield_size(input_size, pivparams: PIVParameters, scale=1):
    """get_vectorfield_size (src/utils/piv_ops.jl:6-14)."""
    out = []
    for n, i, s in zip(input_size, _isize(pivparams), _step(pivparams)):
        stop = int(n) - int(i) + 1
        out.append(0 if stop < 1 else (stop - 1) // int(s) + 1)
    return tuple(out)


# ---------------------------------------------------------------------------
def _is_torch_cuda(x) -> bool:
    t = type(x)
    return t.__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _dtype_code(dt) -> int:
    if dt == np.float32:
        return _lib.MQP_F32
    if dt == np.float64:
        return _lib.MQP_F64
    raise TypeError(f"PIV inputs must be Float32 or Float64 arrays, got {dt}")


def _host_array(a, dtype):
    a = np.asarray(a)
    if a.dtype not in (np.float32, np.float64):
        a = a.astype(np.float64)
    return np.asfortranarray(a, dtype=dtype)


def _dims3(shape):
    d = (C.c_int64 * 3)(1, 1, 1)
    for i, s in enumerate(shape):
        d[i] = int(s)
    return d


def _split_args(args):
    """The three PIV methods of src/multi_quickPIV.jl:17-29."""
    params = None
    arrays = []
    for a in args:
        if isinstance(a, PIVParameters):
            params = a
        else:
            arrays.append(a)
    if len(arrays) > 2:
        raise TypeError("PIV(img1, img2[, mask[, mask_IA]][, pivparams])")
    return arrays, (params if params is not None else setPIVParameters())


def PIV(input1, input2, *args, precision=np.float64, context: Optional[_lib.Context] = None):
    """PIV (src/multi_quickPIV.jl:17-29) on the B200 path.

    PIV(img1, img2[, pivparams])                 standard PIV
    PIV(img1, img2, mask[, pivparams])           masked NSQECC
    PIV(img1, img2, mask_VF, mask_IA[, pivparams])  skip mask + IA mask

    Returns (VF, SN) with VF of shape (N, vf...) and SN None unless
    ``pivparams.computeSN``.
    """
    masks, pivparams = _split_args(args)
    if _is_torch_cuda(input1):
        return _piv_torch(input1, input2, masks, pivparams, precision, context)
    a1, a2 = np.asarray(input1), np.asarray(input2)
    if a1.shape != a2.shape or any(np.asarray(m).shape != a1.shape for m in masks):
        raise AssertionError("PIV inputs need to have the same size.")
    N = a1.ndim
    if N not in (2, 3):
        raise ValueError("PIV inputs must be 2D or 3D arrays")
    pivparams.ndims = N
    work = np.float64 if (a1.dtype == np.float64 or a2.dtype == np.float64) else np.float32
    h1, h2 = _host_array(a1, work), _host_array(a2, work)
    mask = mask_skip = None
    if len(masks) == 1:
        mask = _host_array(masks[0], work)
    elif len(masks) == 2:
        mask_skip = _host_array(masks[0], work)
        mask = _host_array(masks[1], work)
    ctx = context or _lib.default_context(0)
    cp = pivparams.to_c()
    dims = _dims3(a1.shape)
    vfd = (C.c_int64 * 3)()
    _lib.check(ctx.lib.mqp_vf_dims(C.byref(cp), N, dims, vfd), None)
    vf = tuple(int(vfd[d]) for d in range(N))
    VF = np.zeros((N,) + vf, dtype=np.float64, order="F")
    SN = np.zeros(vf, dtype=np.float64, order="F") if pivparams.computeSN else None
    ptr = lambda x: None if x is None else x.ctypes.data_as(C.c_void_p)
    rc = ctx.lib.mqp_piv(ctx.handle, ptr(h1), ptr(h2), ptr(mask), ptr(mask_skip), _dtype_code(work), N,
                         dims, C.byref(cp), ptr(VF), ptr(SN), vfd)
    _lib.check(rc, ctx.handle)
    if precision != np.float64:
        VF = VF.astype(precision)
        SN = SN.astype(precision) if SN is not None else None
    return VF, SN


def _colmajor_torch(t):
    """A column-major (Julia-order) contiguous copy/view of a CUDA tensor."""
    nd = t.dim()
    perm = tuple(range(nd - 1, -1, -1))
    return t.permute(perm).contiguous().permute(perm)


def _piv_torch(input1, input2, masks, pivparams, precision, context):
    import torch
    if input1.shape != input2.shape or any(m.shape != input1.shape for m in masks):
        raise AssertionError("PIV inputs need to have the same size.")
    N = input1.dim()
    pivparams.ndims = N
    dev = input1.device.index or 0
    work = torch.float64 if torch.float64 in (input1.dtype, input2.dtype) else torch.float32
    t1 = _colmajor_torch(input1.to(work))
    t2 = _colmajor_torch(input2.to(work))
    tm = ts = None
    if len(masks) == 1:
        tm = _colmajor_torch(masks[0].to(work))
    elif len(masks) == 2:
        ts = _colmajor_torch(masks[0].to(work))
        tm = _colmajor_torch(masks[1].to(work))
    ctx = context or _lib.default_context(dev)
    cp = pivparams.to_c()
    dims = _dims3(input1.shape)
    vfd = (C.c_int64 * 3)()
    _lib.check(ctx.lib.mqp_vf_dims(C.byref(cp), N, dims, vfd), None)
    vf = tuple(int(vfd[d]) for d in range(N))
    # (N, vf...) column-major == reversed-shape C-contiguous, viewed back
    VFt = torch.zeros(tuple(reversed((N,) + vf)), dtype=torch.float64, device=input1.device)
    SNt = torch.zeros(tuple(reversed(vf)), dtype=torch.float64, device=input1.device) if pivparams.computeSN else None
    stream = torch.cuda.current_stream(input1.device).cuda_stream
    vp = lambda x: None if x is None else C.c_void_p(x.data_ptr())
    rc = ctx.lib.mqp_piv_device(ctx.handle, vp(t1), vp(t2), vp(tm), vp(ts),
                                _lib.MQP_F64 if work == torch.float64 else _lib.MQP_F32, N, dims,
                                C.byref(cp), vp(VFt), vp(SNt), C.c_void_p(stream))
    _lib.check(rc, ctx.handle)
    VF = VFt.permute(tuple(range(N, -1, -1)))
    SN = SNt.permute(tuple(range(N - 1, -1, -1))) if SNt is not None else None
    if precision != np.float64:
        tdt = torch.float32 if precision == np.float32 else torch.float64
        VF = VF.to(tdt)
        SN = SN.to(tdt) if SN is not None else None
    return VF, SN


def correlation_planes(input1, input2, pivparams: PIVParameters, ia_begin=0, ia_end=None,
                       mask=None, context: Optional[_lib.Context] = None) -> np.ndarray:
    """The fully-overlapping similarity planes of IAs [ia_begin, ia_end)
    (column-major IA order), shape (2SM1+1, ..., n_ia).  A debugging view of
    tmp_data[1] after crosscorrelation! (src/multi_quickPIV.jl:77)."""
    a1, a2 = np.asarray(input1), np.asarray(input2)
    if a1.shape != a2.shape:
        raise AssertionError("PIV inputs need to have the same size.")
    N = a1.ndim
    pivparams.ndims = N
    work = np.float64 if (a1.dtype == np.float64 or a2.dtype == np.float64) else np.float32
    h1, h2 = _host_array(a1, work), _host_array(a2, work)
    hm = _host_array(mask, work) if mask is not None else None
    n_ia = int(np.prod(get_vectorfield_size(a1.shape, pivparams)))
    ia_end = n_ia if ia_end is None else ia_end
    P = tuple(2 * m + 1 for m in _smarg(pivparams))
    out = np.zeros(P + (max(ia_end - ia_begin, 0),), dtype=np.float64, order="F")
    ctx = context or _lib.default_context(0)
    cp = pivparams.to_c()
    ptr = lambda x: None if x is None else x.ctypes.data_as(C.c_void_p)
    rc = ctx.lib.mqp_correlation_planes(ctx.handle, ptr(h1), ptr(h2), ptr(hm), _dtype_code(work), N,
                                        _dims3(a1.shape), C.byref(cp), int(ia_begin), int(ia_end), ptr(out))
    _lib.check(rc, ctx.handle)
    return out
