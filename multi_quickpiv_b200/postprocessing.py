"""Vector-field post-processing on the GPU, mirroring
src/postprocessing/postprocessing.jl of multi_quickPIV (same names, argument
meaning and defaults).  Fields are (ncomp, d1, ..., dN) arrays as PIV returns
them: NumPy arrays (computed on the device through the context's buffers,
returned as NumPy) or torch CUDA tensors (computed in place on the device,
returned as tensors).  The kernels are in csrc/mqp_post.cuh.

Functions that cannot run in the reference are provided with the behaviour
they were written to have (TH_filtering, remove_low_SN, divergence,
multiscale_divergence, average_NDT, meanReplace, the arrays form of
collectiveness); local_magnitude_mask and normalize_vectorfield also accept
3D fields.  A custom `fun` (masking) or replacement callable runs on the host,
as closures cannot cross the C ABI.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional

import numpy as np

from . import _lib


# ---------------------------------------------------------------------------
# plumbing
# ---------------------------------------------------------------------------
def _is_torch(x) -> bool:
    try:
        import torch
        return isinstance(x, torch.Tensor) and x.is_cuda
    except Exception:
        return False


def _as_field(arrays):
    """VF, or separate component arrays (U, V[, W]) stacked into one VF."""
    if len(arrays) == 1:
        return arrays[0]
    if _is_torch(arrays[0]):
        import torch
        return torch.stack(list(arrays), 0)
    return np.stack([np.asarray(a) for a in arrays], 0)


def _radius4(radius, nd):
    """toDims3(radius)[1:N] (src/piv_parameters.jl:8-11, as localOp takes it,
    postprocessing.jl:65,74,85): an Integer repeats on every axis, a shorter
    tuple is padded with radius 0 (a 2-tuple on a 3D field averages in-plane
    only)."""
    if np.isscalar(radius):
        r = [int(radius)] * nd
    else:
        r = [int(x) for x in radius][:nd]
        r += [0] * (nd - len(r))
    return (C.c_int32 * 4)(*(r + [0] * (4 - nd)))


def _field(shape, ncomp):
    f = _lib.MqpField()
    f.ncomp = ncomp
    f.ndims = len(shape)
    for d in range(4):
        f.dims[d] = int(shape[d]) if d < len(shape) else 1
    return f


def _params(op, radius=0, nd=1, **kw):
    p = _lib.MqpPostParams()
    p.op = op
    p.radius = _radius4(radius, nd)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _colmajor_torch(t):
    nd = t.dim()
    perm = tuple(range(nd - 1, -1, -1))
    return t.permute(perm).contiguous().permute(perm)


def _torch_empty_colmajor(shape, dtype, device):
    import torch
    t = torch.empty(tuple(reversed(shape)), dtype=dtype, device=device)
    return t.permute(tuple(range(len(shape) - 1, -1, -1)))


def _run(op, inp, ncomp, grid, p, mask=None, out_vec=False, out_scalar=False, outf=False, mask_out=False,
         context: Optional[_lib.Context] = None):
    """One post-processing op; returns (out, outf, mask_out) (None where unused)."""
    f = _field(grid, ncomp)
    if _is_torch(inp):
        import torch
        dev = inp.device
        ctx = context or _lib.default_context(dev.index or 0)
        x = _colmajor_torch(inp.to(torch.float64))
        m = _colmajor_torch(mask.to(torch.uint8)) if mask is not None else None
        o = _torch_empty_colmajor(((ncomp,) if out_vec else ()) + tuple(grid), torch.float64, dev) \
            if (out_vec or out_scalar) else None
        of = _torch_empty_colmajor(tuple(grid), torch.float32, dev) if outf else None
        mo = _torch_empty_colmajor(tuple(grid), torch.uint8, dev) if mask_out else None
        vp = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = ctx.lib.mqp_postprocess_device(ctx.handle, C.byref(p), C.byref(f), vp(x), vp(m), vp(o), vp(of), vp(mo),
                                            C.c_void_p(stream))
        _lib.check(rc, ctx.handle)
        return o, of, (mo.bool() if mo is not None else None)
    ctx = context or _lib.default_context(0)
    x = np.asfortranarray(np.asarray(inp, dtype=np.float64))
    m = np.asfortranarray(np.asarray(mask, dtype=np.uint8)) if mask is not None else None
    o = np.zeros(((ncomp,) if out_vec else ()) + tuple(grid), dtype=np.float64, order="F") \
        if (out_vec or out_scalar) else None
    of = np.zeros(tuple(grid), dtype=np.float32, order="F") if outf else None
    mo = np.zeros(tuple(grid), dtype=np.uint8, order="F") if mask_out else None
    ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    rc = ctx.lib.mqp_postprocess(ctx.handle, C.byref(p), C.byref(f), ptr(x), ptr(m), ptr(o), ptr(of), ptr(mo))
    _lib.check(rc, ctx.handle)
    return o, of, (mo.astype(bool) if mo is not None else None)


def _grid(VF):
    return tuple(VF.shape[1:])


# ---------------------------------------------------------------------------
# magnitudes, averaging, collectiveness (postprocessing.jl:134-523)
# ---------------------------------------------------------------------------
def magnitudes(*arrays, context=None):
    """magnitudes(VF) / magnitudes(U, V[, W]) (postprocessing.jl:134-192)."""
    VF = _as_field(arrays)
    g = _grid(VF)
    out, _, _ = _run(_lib.MQP_POST_MAGNITUDES, VF, VF.shape[0], g, _params(_lib.MQP_POST_MAGNITUDES, 0, len(g)),
                     out_scalar=True, context=context)
    return out


speeds = magnitudes
velocities = magnitudes


def average(radius, *arrays, context=None):
    """average(radius, VF) (postprocessing.jl:339-381): window mean per component."""
    VF = _as_field(arrays)
    g = _grid(VF)
    out, _, _ = _run(_lib.MQP_POST_AVERAGE, VF, VF.shape[0], g, _params(_lib.MQP_POST_AVERAGE, radius, len(g)),
                     out_vec=True, context=context)
    return out


def average_NDT(radius1, radius2, *arrays, context=None):
    """Space-time average: the last grid axis is time (+-radius2), the others
    are space (+-radius1).  The reference's average_NDT (postprocessing.jl:386-414)
    computes two local means and discards them."""
    VF = _as_field(arrays)
    g = _grid(VF)
    r1 = [int(radius1)] * (len(g) - 1) if np.isscalar(radius1) else [int(x) for x in radius1]
    r1 = (r1 + [0] * len(g))[:len(g) - 1]  # toDims3 padding of the spatial radii
    return average(tuple(r1) + (int(radius2),), VF, context=context)


def collectiveness(radius, *arrays, max_angle=40, context=None):
    """collectiveness(radius, VF; max_angle=40) (postprocessing.jl:240-331), Float32."""
    VF = _as_field(arrays)
    g = _grid(VF)
    _, outf, _ = _run(_lib.MQP_POST_COLLECTIVENESS, VF, VF.shape[0], g,
                      _params(_lib.MQP_POST_COLLECTIVENESS, radius, len(g), max_angle=float(max_angle)), outf=True,
                      context=context)
    return outf


def similarityAveraging(radius, *arrays, max_angle=20, normalize=True, scale_by_similarity=True,
                        similarity_exponent=2, context=None):
    """similarityAveraging(radius, VF; ...) (postprocessing.jl:475-523, the VF method)."""
    VF = _as_field(arrays)
    g = _grid(VF)
    p = _params(_lib.MQP_POST_SIMILARITY_AVG, radius, len(g), max_angle=float(max_angle),
                normalize=int(bool(normalize)), scale_by_similarity=int(bool(scale_by_similarity)),
                similarity_exponent=float(similarity_exponent))
    out, _, _ = _run(_lib.MQP_POST_SIMILARITY_AVG, VF, VF.shape[0], g, p, out_vec=True, context=context)
    return out


# ---------------------------------------------------------------------------
# masking and filtering (postprocessing.jl:527-741)
# ---------------------------------------------------------------------------
def zeroReplace(coords, radius, VF):
    """zeroReplace (postprocessing.jl:539-545)."""
    return np.zeros(VF.shape[0])


def medianReplace(coords, radius, VF):
    """medianReplace (postprocessing.jl:547-553): window median per component."""
    sl = tuple(slice(max(0, c - r), c + r + 1) for c, r in zip(coords, _radius4(radius, len(coords))[:len(coords)]))
    return np.array([np.median(np.asarray(VF)[(k,) + sl]) for k in range(VF.shape[0])])


def meanReplace(coords, radius, VF):
    """meanReplace (postprocessing.jl:555-561): the window mean its docstring
    describes (the reference's body computes the median and its VF method
    cannot be called)."""
    sl = tuple(slice(max(0, c - r), c + r + 1) for c, r in zip(coords, _radius4(radius, len(coords))[:len(coords)]))
    return np.array([np.mean(np.asarray(VF)[(k,) + sl]) for k in range(VF.shape[0])])


zeroReplace.kind = _lib.MQP_REPLACE_ZERO
medianReplace.kind = _lib.MQP_REPLACE_MEDIAN
meanReplace.kind = _lib.MQP_REPLACE_MEAN


def _map_of(VF, fun):
    return magnitudes(VF) if fun is magnitudes or fun is None else fun(VF)


def STD_masking(n, *arrays, fun=None, context=None):
    """STD_masking(n, VF; fun=magnitudes) (postprocessing.jl:586-609):
    |map - mean| > n * std (n-1 normalised)."""
    VF = _as_field(arrays)
    m = _map_of(VF, fun)
    g = tuple(m.shape)
    _, _, mask = _run(_lib.MQP_POST_STD_MASK, m, 1, g, _params(_lib.MQP_POST_STD_MASK, 0, len(g), threshold=float(n)),
                      mask_out=True, context=context)
    return mask


def TH_masking(th, *arrays, fun=None, cmp=">", context=None):
    """TH_masking(th, VF; fun=magnitudes, cmp=(x,th)->x>th) (postprocessing.jl:652-670);
    cmp is ">" or "<" (or a callable, applied on the host)."""
    VF = _as_field(arrays)
    m = _map_of(VF, fun)
    if callable(cmp):
        return cmp(m, th)
    g = tuple(m.shape)
    p = _params(_lib.MQP_POST_TH_MASK, 0, len(g), threshold=float(th), cmp=0 if cmp == ">" else 1)
    _, _, mask = _run(_lib.MQP_POST_TH_MASK, m, 1, g, p, mask_out=True, context=context)
    return mask


def _replace(VF, mask, replaceFun, radius, context):
    g = _grid(VF)
    kind = getattr(replaceFun, "kind", None)
    if kind is None:  # a user callable: replacements computed on the host, as the reference does
        VFh = np.asarray(VF.cpu() if _is_torch(VF) else VF, dtype=np.float64)
        out = VFh.copy()
        mh = np.asarray(mask.cpu() if _is_torch(mask) else mask)
        for idx in zip(*np.nonzero(mh)):
            out[(slice(None),) + tuple(int(i) for i in idx)] = replaceFun(tuple(int(i) for i in idx), radius, VFh)
        return out
    p = _params(_lib.MQP_POST_REPLACE, radius, len(g), replace=int(kind))
    out, _, _ = _run(_lib.MQP_POST_REPLACE, VF, VF.shape[0], g, p, mask=mask, out_vec=True, context=context)
    return out


def STD_filtering(n, *arrays, fun=None, replaceFun=meanReplace, radius=2, context=None):
    """STD_filtering(n, VF; fun, replaceFun=meanReplace, radius=2) (postprocessing.jl:615-643):
    masked vectors replaced from the original field."""
    VF = _as_field(arrays)
    return _replace(VF, STD_masking(n, VF, fun=fun, context=context), replaceFun, radius, context)


def TH_filtering(th, *arrays, fun=None, cmp=">", replaceFun=meanReplace, radius=2, context=None):
    """TH_filtering(th, VF; ...) (postprocessing.jl:676-706, which calls the
    undefined `replacefun`): TH_masking then the replacement."""
    VF = _as_field(arrays)
    return _replace(VF, TH_masking(th, VF, fun=fun, cmp=cmp, context=context), replaceFun, radius, context)


def remove_low_SN(SN, threshold, *arrays, replace=zeroReplace, radius=1, context=None):
    """remove_low_SN(SN, threshold, VF; replace=zeroReplace, radius=1)
    (postprocessing.jl:712-732, which passes an unknown keyword): vectors with
    SN < threshold replaced."""
    VF = _as_field(arrays)
    return TH_filtering(threshold, VF, fun=lambda x: SN, cmp="<", replaceFun=replace, radius=radius, context=context)


def local_magnitude_mask(ratio, VF, radius=4, context=None):
    """local_magnitude_mask(ratio, VF; radius=4) (postprocessing.jl:202-218):
    returns (VF with the removed vectors zeroed, removed mask)."""
    g = _grid(VF)
    p = _params(_lib.MQP_POST_LOCAL_MAGNITUDE, radius, len(g), threshold=float(ratio))
    out, _, removed = _run(_lib.MQP_POST_LOCAL_MAGNITUDE, VF, VF.shape[0], g, p, out_vec=True, mask_out=True,
                           context=context)
    return out, removed


def apply_mask(mask, VF):
    """apply_mask!(mask, VF) (postprocessing.jl:110-115), out of place."""
    return VF * mask[None]


# ---------------------------------------------------------------------------
# divergence (postprocessing.jl:745-980)
# ---------------------------------------------------------------------------
def matlab_divergence(VF, context=None):
    """matlab_divergence(VF) (postprocessing.jl:918-941), Float32."""
    g = _grid(VF)
    _, outf, _ = _run(_lib.MQP_POST_MATLAB_DIVERGENCE, VF, VF.shape[0], g,
                      _params(_lib.MQP_POST_MATLAB_DIVERGENCE, 0, len(g)), outf=True, context=context)
    return outf


def normalize_sink(radii, typ=np.float32, scales=None, circle=False):
    """normalize_sink(radii; typ, scales, circle) (postprocessing.jl:757-773)."""
    radii = tuple(int(r) for r in radii)
    size = tuple(2 * r + 1 for r in radii)
    center = np.array([(s + 1) // 2 for s in size], dtype=np.float64)
    sc = np.ones(len(radii)) if scales is None else np.asarray(scales, dtype=np.float64)
    grids = np.meshgrid(*[np.arange(1, s + 1, dtype=np.float64) for s in size], indexing="ij")
    m = np.sqrt(sum((center[d] * sc[d] - grids[d] * sc[d]) ** 2 for d in range(len(size))))
    if circle:
        m = m * (m <= max(radii))
    m[tuple(int(c) - 1 for c in center)] = 1
    return m.astype(typ)


def sink(radii, dim=1):
    """sink(radii, dim=1) (postprocessing.jl:813-818), dim 1-based."""
    sm = normalize_sink(radii)
    center = [(s + 1) // 2 for s in sm.shape]
    grids = np.meshgrid(*[np.arange(1, s + 1) for s in sm.shape], indexing="ij")
    with np.errstate(invalid="ignore", divide="ignore"):
        out = np.where(sm == 0, 0, (center[dim - 1] - grids[dim - 1]) / sm).astype(sm.dtype)
    out[np.isnan(out)] = 0
    return out


def normalize_vectorfield(VF, normalize=True, min_speed=0):
    """normalize_vectorfield(VF; normalize=true, min_speed=0) (postprocessing.jl:826-845)."""
    M = magnitudes(VF)
    out = VF * 1.0
    if min_speed > 0:
        out = out * (M > min_speed)[None]
    if normalize:
        M = M + (M == 0) * 1.0
        out = out / M[None]
    return out


def divergence(radii, VF, normalize=False, min_speed=0, divide_by="N", circle=False, context=None):
    """divergence(radii, VF; normalize=false, min_speed=0, divide_by="N",
    circle=false) (postprocessing.jl:853-903, which cannot run): the sink
    pattern of half-size `radii` correlated with the (normalised) field,
    summed over components, / count ("N") or / local |VF| sum ("mags")."""
    g = _grid(VF)
    dv = {"N": _lib.MQP_DIVIDE_N, "mags": _lib.MQP_DIVIDE_MAGS}.get(divide_by, _lib.MQP_DIVIDE_NONE)
    # divergence uses its radii as given (normalize_sink, postprocessing.jl:757-781):
    # a shorter tuple repeats its last entry
    if not np.isscalar(radii):
        r = [int(x) for x in radii][:len(g)]
        radii = tuple(r + [r[-1]] * (len(g) - len(r)))
    p = _params(_lib.MQP_POST_DIVERGENCE, radii, len(g), normalize=int(bool(normalize)),
                min_speed=float(min_speed), divide_by=dv, circle=int(bool(circle)))
    out, _, _ = _run(_lib.MQP_POST_DIVERGENCE, VF, VF.shape[0], g, p, out_scalar=True, context=context)
    return out


def multiscale_divergence(radii, VF, min_value=0.2, normalize=True, min_speed=0, divide_by="N", context=None):
    """multiscale_divergence(radii, VF; ...) (postprocessing.jl:948-980):
    (max_divergence_scale, max_divergence, max_convergence_scale, max_convergence)."""
    mod = None
    if _is_torch(VF):
        import torch as mod
    xp = mod if mod is not None else np
    g = _grid(VF)
    zeros = (lambda dt: mod.zeros(g, dtype=dt, device=VF.device)) if mod is not None else (lambda dt: np.zeros(g, dt))
    mxd, mxc = zeros(xp.float64), zeros(xp.float64)
    sd, sc = zeros(xp.int64), zeros(xp.int64)
    for rad in radii:
        r0 = int(rad) if np.isscalar(rad) else int(rad[0])
        d = -1 * divergence(rad, VF, normalize=normalize, min_speed=min_speed, divide_by=divide_by, context=context)
        c = -1 * d
        up = (d > min_value) & (d > mxd)
        sd = xp.where(up, r0, sd)
        mxd = xp.where(up, d, mxd)
        uc = (c > min_value) & (c > mxc)
        sc = xp.where(uc, r0, sc)
        mxc = xp.where(uc, c, mxc)
    return sd, mxd, sc, mxc


# ---------------------------------------------------------------------------
# pseudo-trajectories (postprocessing.jl:988-1120)
# ---------------------------------------------------------------------------
def _traj_range(r):
    """A sampling range as (lo, hi), 1-based inclusive like Julia's lo:hi:
    None (or an empty range) selects the reference's default 2:dims-1; a
    (lo, hi) pair is taken as is; a Python range(a, b) means a:b-1."""
    if r is None:
        return 1, 0
    if isinstance(r, range):
        return (r.start, r.stop - 1) if len(r) else (1, 0)
    lo, hi = r
    return int(lo), int(hi)


def _trajectories(comps, T0, T1, numpoints, subregion, scale, grid, step, seed, context):
    nd = len(comps)
    shape = tuple(comps[0].shape)
    if any(tuple(c.shape) != shape for c in comps) or len(shape) != nd + 1:
        raise AssertionError("U, V(, W) must be (d1, d2[, d3], frames) arrays of the same size")
    p = _lib.MqpTrajParams()
    p.ndims = nd
    for d in range(nd):
        p.dims[d] = int(shape[d])
    p.frames = int(shape[nd])
    p.T0, p.T1 = int(T0), int(T1)
    sub = subregion if subregion is not None else (None,) * nd
    sc = (scale,) * 3 if np.isscalar(scale) else tuple(scale) + (1,) * (3 - len(scale))
    st = (step,) * 3 if np.isscalar(step) else tuple(step) + (1,) * (3 - len(step))
    for d in range(nd):
        p.sub_lo[d], p.sub_hi[d] = _traj_range(sub[d])
        p.step[d] = int(st[d])
        p.scale[d] = float(sc[d])
    p.grid = int(bool(grid))
    p.numpoints = int(numpoints)
    p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    lib = _lib.load()
    npts = C.c_int64()
    _lib.check(lib.mqp_traj_count(C.byref(p), C.byref(npts)), None)
    n, numT = int(npts.value), int(T1) - int(T0)
    if _is_torch(comps[0]):
        import torch
        dev = comps[0].device
        ctx = context or _lib.default_context(dev.index or 0)
        dt = torch.float64 if any(c.dtype == torch.float64 for c in comps) else torch.float32
        xs = [_colmajor_torch(c.to(dt)) for c in comps]
        outs = [_torch_empty_colmajor((numT, n), torch.float32, dev) for _ in range(nd)]
        vp = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = ctx.lib.mqp_trajectories_device(ctx.handle, C.byref(p), _lib.MQP_F64 if dt == torch.float64 else _lib.MQP_F32,
                                             vp(xs[0]), vp(xs[1]), vp(xs[2] if nd == 3 else None), vp(outs[0]),
                                             vp(outs[1]), vp(outs[2] if nd == 3 else None), C.c_void_p(stream))
        _lib.check(rc, ctx.handle)
    else:
        ctx = context or _lib.default_context(0)
        dt = np.float64 if any(np.asarray(c).dtype == np.float64 for c in comps) else np.float32
        xs = [np.asfortranarray(np.asarray(c, dtype=dt)) for c in comps]
        outs = [np.zeros((numT, n), dtype=np.float32, order="F") for _ in range(nd)]
        ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
        rc = ctx.lib.mqp_trajectories(ctx.handle, C.byref(p), _lib.MQP_F64 if dt == np.float64 else _lib.MQP_F32,
                                      ptr(xs[0]), ptr(xs[1]), ptr(xs[2] if nd == 3 else None), ptr(outs[0]),
                                      ptr(outs[1]), ptr(outs[2] if nd == 3 else None))
        _lib.check(rc, ctx.handle)
    return tuple(outs) + ((None,) if nd == 2 else ())


def PIVtrajectories(U, V, W, T0, T1, numpoints, subregion=None, scale=(1, 1, 1), seed=0, context=None):
    """PIVtrajectories(U, V, W, T0, T1, numpoints; subregion, scale)
    (postprocessing.jl:988-1050) on the GPU: numpoints particles from random
    integer positions of the sampling region, followed through frames T0 (1-based)
    onwards; returns (TrajectoriesY, TrajectoriesX, TrajectoriesZ), Float32
    arrays of shape (T1 - T0, numpoints) with 1-based positions.  U, V, W are
    (d1, d2, d3, frames) arrays (NumPy or torch CUDA); W = None follows a 2D
    field over time (then TrajectoriesZ is None).  The starting positions come
    from a counter-based generator seeded by `seed` (Julia's rand stream cannot
    be reproduced outside Julia)."""
    comps = [U, V] + ([W] if W is not None else [])
    return _trajectories(comps, T0, T1, numpoints, subregion, scale, False, 1, seed, context)


def PIVtrajectories_grid(U, V, W, T0, T1, numpoints=0, subregion=None, step=(1, 1, 1), scale=(1, 1, 1),
                         context=None):
    """PIVtrajectories_grid(U, V, W, T0, T1, numpoints; subregion, step, scale)
    (postprocessing.jl:1055-1120) on the GPU: one particle per point of the
    sampling grid (step apart, y fastest); numpoints is unused, as in the
    reference."""
    comps = [U, V] + ([W] if W is not None else [])
    return _trajectories(comps, T0, T1, numpoints, subregion, scale, True, step, 0, context)
