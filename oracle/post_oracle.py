"""CPU restatement of multi_quickPIV's vector-field post-processing
(src/postprocessing/postprocessing.jl), the checker of the device kernels.

TEST INFRASTRUCTURE: only tests/ may import this module.  Plain NumPy loops
over Float64 fields of shape (ncomp, d1, ..., dN) (the VF array PIV returns,
axis 0 = components); windows are clamped at the field border as localOp
does (postprocessing.jl:62-72).

Functions the reference cannot run (kwargs to positional methods, undefined
names) are restated with the behaviour they were written to have; each one
says what is broken and what is computed instead.
"""
from __future__ import annotations

import math

import numpy as np


def _cosd(deg):
    return math.cos(math.radians(deg))


def _window(idx, radius, size):
    """localOp's ROI (postprocessing.jl:66-70): max(1, c-r):min(size, c+r)."""
    return tuple(slice(max(0, i - r), min(s - 1, i + r) + 1) for i, r, s in zip(idx, radius, size))


def _radii(radius, nd):
    """toDims3(radius)[1:N] as localOp and the window operations take it
    (postprocessing.jl:65,74,85; toDims3, src/piv_parameters.jl:8-11): an
    Integer repeats on every axis, a 2-tuple gets radius 0 on axis 3.  Grids
    of 4 axes (space-time fields) take a 4-tuple as given and pad shorter
    tuples with 0 the same way."""
    if np.isscalar(radius):
        return (int(radius),) * nd
    r = tuple(int(x) for x in radius)
    return (r + (0,) * nd)[:nd]


def _sink_radii(radii, nd):
    """divergence's radii, which it uses as given (normalize_sink,
    postprocessing.jl:757-781): an Integer repeats, a shorter tuple repeats
    its last entry."""
    if np.isscalar(radii):
        return (int(radii),) * nd
    r = tuple(int(x) for x in radii)
    return (r + (r[-1],) * nd)[:nd] if len(r) < nd else r[:nd]


def magnitudes(VF):
    """magnitudes(VF) (postprocessing.jl:178-192)."""
    VF = np.asarray(VF, dtype=np.float64)
    s = np.zeros(VF.shape[1:])
    for c in range(VF.shape[0]):
        s = s + VF[c] ** 2
    return np.sqrt(s)


def average(radius, VF):
    """average(radius, VF) (postprocessing.jl:364-381): window means."""
    VF = np.asarray(VF, dtype=np.float64)
    size = VF.shape[1:]
    r = _radii(radius, len(size))
    out = VF.copy()
    for idx in np.ndindex(*size):
        w = _window(idx, r, size)
        for c in range(VF.shape[0]):
            out[(c,) + idx] = np.mean(VF[(c,) + w])
    return out


def collectiveness(radius, VF, max_angle=40):
    """collectiveness(radius, VF; max_angle) (postprocessing.jl:291-331):
    the fraction of window vectors within max_angle of the centre's (Float32)."""
    VF = np.asarray(VF, dtype=np.float64)
    size = VF.shape[1:]
    r = _radii(radius, len(size))
    min_dot = _cosd(max_angle)
    M = magnitudes(VF)
    out = np.zeros(size, dtype=np.float32)
    with np.errstate(invalid="ignore", divide="ignore"):
        for idx in np.ndindex(*size):
            nvec = VF[(slice(None),) + idx] / M[idx]
            w = _window(idx, r, size)
            sub = VF[(slice(None),) + w] / M[w]
            dot = np.tensordot(nvec, sub, axes=(0, 0))
            out[idx] = np.float32(np.count_nonzero(dot > min_dot) / dot.size)
    return out


def similarityAveraging(radius, VF, max_angle=20, normalize=True, scale_by_similarity=True, similarity_exponent=2):
    """similarityAveraging(radius, VF; ...) (postprocessing.jl:475-523), the
    VF method: sum of the similar window vectors, / its norm if normalize,
    * (similar/count)^exponent if scale_by_similarity; zero vectors stay."""
    VF = np.asarray(VF, dtype=np.float64)
    size = VF.shape[1:]
    r = _radii(radius, len(size))
    min_dot = _cosd(max_angle)
    M = magnitudes(VF)
    out = VF.copy()
    with np.errstate(invalid="ignore", divide="ignore"):
        for idx in np.ndindex(*size):
            if M[idx] == 0:
                continue
            nvec = VF[(slice(None),) + idx] / M[idx]
            w = _window(idx, r, size)
            avg = np.zeros(VF.shape[0])
            nsim = 0
            for lidx in np.ndindex(*[s.stop - s.start for s in w]):
                l = tuple(s.start + j for s, j in zip(w, lidx))
                nv = VF[(slice(None),) + l] / M[l]
                if float(np.sum(nvec * nv)) > min_dot:
                    avg += nv * M[l]
                    nsim += 1
            n = int(np.prod([s.stop - s.start for s in w]))
            fac = 1.0
            if normalize:
                fac /= math.sqrt(float(np.sum(avg ** 2)))
            if scale_by_similarity:
                fac *= (nsim / n) ** similarity_exponent
            out[(slice(None),) + idx] = avg * fac
    return out


def STD_masking(n, VF, fun=magnitudes):
    """STD_masking(n, VF; fun) (postprocessing.jl:598-609): |map - mean| > n*std
    (std with n-1 normalisation)."""
    m = np.asarray(fun(VF), dtype=np.float64)
    mean = float(np.mean(m))
    std = float(np.std(m, ddof=1))
    return np.abs(m - mean) > n * std


def TH_masking(th, VF, fun=magnitudes, cmp=lambda x, th: x > th):
    """TH_masking(th, VF; fun, cmp) (postprocessing.jl:660-670)."""
    return cmp(np.asarray(fun(VF), dtype=np.float64), th)


def zeroReplace(coords, radius, VF):
    """zeroReplace (postprocessing.jl:539-545)."""
    return np.zeros(np.asarray(VF).shape[0])


def medianReplace(coords, radius, VF):
    """medianReplace (postprocessing.jl:547-553): window median per component
    (Statistics.median: mean of the two middle values for even counts)."""
    VF = np.asarray(VF, dtype=np.float64)
    w = _window(coords, _radii(radius, VF.ndim - 1), VF.shape[1:])
    return np.array([np.median(VF[(c,) + w]) for c in range(VF.shape[0])])


def meanReplace(coords, radius, VF):
    """meanReplace (postprocessing.jl:555-561).  Its VF method has the wrong
    arity (VF::Array... passes a tuple to localOp) and both methods call
    median; restated as the window mean the docstring (:529-535) describes."""
    VF = np.asarray(VF, dtype=np.float64)
    w = _window(coords, _radii(radius, VF.ndim - 1), VF.shape[1:])
    return np.array([np.mean(VF[(c,) + w]) for c in range(VF.shape[0])])


def _filter(mask, VF, replaceFun, radius):
    VF = np.asarray(VF, dtype=np.float64)
    out = VF.copy()
    for idx in zip(*np.nonzero(mask)):
        out[(slice(None),) + tuple(int(i) for i in idx)] = replaceFun(tuple(int(i) for i in idx), radius, VF)
    return out


def STD_filtering(n, VF, fun=magnitudes, replaceFun=meanReplace, radius=2):
    """STD_filtering(n, VF; fun, replaceFun, radius) (postprocessing.jl:630-643):
    masked vectors replaced from the ORIGINAL field."""
    return _filter(STD_masking(n, VF, fun), VF, replaceFun, radius)


def TH_filtering(th, VF, fun=magnitudes, cmp=lambda x, th: x > th, replaceFun=meanReplace, radius=2):
    """TH_filtering (postprocessing.jl:692-706).  The reference calls the
    undefined `replacefun` (:702); restated with replaceFun."""
    return _filter(TH_masking(th, VF, fun, cmp), VF, replaceFun, radius)


def remove_low_SN(SN, threshold, VF, replace=zeroReplace, radius=1):
    """remove_low_SN (postprocessing.jl:723-732).  The reference passes
    `replace=` to TH_filtering, which has no such keyword; restated as
    TH_filtering with fun = SN, cmp = (x < th) and replaceFun = replace."""
    return TH_filtering(threshold, VF, fun=lambda x: SN, cmp=lambda x, th: x < th, replaceFun=replace, radius=radius)


def local_magnitude_mask(ratio, VF, radius=4):
    """local_magnitude_mask(ratio, VF; radius) (postprocessing.jl:202-218):
    keep v when |v| / mean(|w|, window without v) < ratio; returns (VF .* keep,
    removed).  The reference's VF_c[c,:,:] makes it 2D-only (:215); the same
    rule is applied on any grid dimension here."""
    VF = np.asarray(VF, dtype=np.float64)
    size = VF.shape[1:]
    r = _radii(radius, len(size))
    mags = magnitudes(VF)
    keep = np.zeros(size, dtype=bool)
    with np.errstate(invalid="ignore", divide="ignore"):
        for idx in np.ndindex(*size):
            w = _window(idx, r, size)
            s = float(np.sum(mags[w])) - mags[idx]
            cnt = mags[w].size - 1
            keep[idx] = mags[idx] / (s / cnt) < ratio
    out = VF.copy()
    for c in range(VF.shape[0]):
        out[c] = np.where(keep, VF[c], np.copysign(0.0, VF[c]))
    return out, ~keep


def matlab_divergence(VF):
    """matlab_divergence(VF) (postprocessing.jl:918-941): per-component central
    differences, one-sided at the border, accumulated in Float32."""
    VF = np.asarray(VF, dtype=np.float64)
    size = VF.shape[1:]
    nd = VF.shape[0]
    out = np.zeros(size, dtype=np.float32)
    with np.errstate(invalid="ignore", divide="ignore"):
        for idx in np.ndindex(*size):
            acc = np.float32(0)
            for i in range(nd):
                cm = list(idx)
                cp = list(idx)
                cm[i] = max(0, min(size[i] - 1, idx[i] - 1))
                cp[i] = max(0, min(size[i] - 1, idx[i] + 1))
                d = (VF[(i,) + tuple(cp)] - VF[(i,) + tuple(cm)]) / abs(cm[i] - cp[i])
                acc = np.float32(acc + np.float32(d))
            out[idx] = acc
    return out


def normalize_sink(radii, typ=np.float32, scales=None, circle=False):
    """normalize_sink (postprocessing.jl:757-773)."""
    radii = tuple(int(r) for r in radii)
    size = tuple(2 * r + 1 for r in radii)
    center = np.array([(s + 1) // 2 for s in size])
    scales = np.ones(len(radii)) if scales is None else np.asarray(scales, dtype=np.float64)
    out = np.zeros(size, dtype=typ)
    rmax = max(radii)
    for idx in np.ndindex(*size):
        ci = np.array(idx) + 1
        m = math.sqrt(float(np.sum((center * scales - ci * scales) ** 2)))
        if circle:
            m *= float(m <= rmax)
        out[idx] = m
    out[tuple(c - 1 for c in center)] = 1
    return out


def sink(radii, dim=1, magnitudes_=None):
    """sink(radii, dim) / sink! (postprocessing.jl:787-818), dim 1-based."""
    sm = normalize_sink(radii) if magnitudes_ is None else magnitudes_
    center = np.array([(s + 1) // 2 for s in sm.shape])
    out = np.zeros(sm.shape, dtype=sm.dtype)
    for idx in np.ndindex(*sm.shape):
        if sm[idx] != 0:
            out[idx] = (center[dim - 1] - (idx[dim - 1] + 1)) / sm[idx]
    out[np.isnan(out)] = 0
    return out


def normalize_vectorfield(VF, normalize=True, min_speed=0):
    """normalize_vectorfield (postprocessing.jl:826-845); the reference indexes
    VF[c, 1:d1, 1:d2] (2D only), restated for any grid dimension."""
    VF = np.asarray(VF, dtype=np.float64)
    out = VF.copy()
    M = magnitudes(VF)
    if min_speed > 0:
        out = out * (M > min_speed)[None]
    if normalize:
        M = np.where(M == 0, 1.0, M)
        out = out / M[None]
    return out


def fftcc_crop(F, G):
    """FFTCC_crop(F, G) (src/crosscorrelation_algorithms/fftcc.jl:175-197): the
    zero-padded correlation sum_x F(x) G(i + x - div(size(F), 2)), cropped to
    size(G), through an FFT of size(F) + size(G) - 1."""
    F = np.asarray(F, dtype=np.float64)
    G = np.asarray(G, dtype=np.float64)
    cs = tuple(f + g - 1 for f, g in zip(F.shape, G.shape))
    ax = tuple(range(F.ndim))
    cc = np.fft.irfftn(np.conj(np.fft.rfftn(F, cs, axes=ax)) * np.fft.rfftn(G, cs, axes=ax), cs, axes=ax)
    cc = np.roll(cc, tuple(f // 2 for f in F.shape), axis=tuple(range(F.ndim)))
    return cc[tuple(slice(0, g) for g in G.shape)]


def divergence(radii, VF, normalize=False, min_speed=0, divide_by="N", circle=False):
    """divergence(radii, VF; ...) (postprocessing.jl:853-903).  The reference
    passes keywords to the positional allocate_tmp_data (:872) and FFTCC_crop
    does the same, so it cannot run; restated as written: the sum over
    components of FFTCC_crop(sink_c, VFn_c), divided by the count of non-zero
    sink magnitudes ("N") or the window sum of |VFn| ("mags")."""
    VF = np.asarray(VF, dtype=np.float64)
    radii = _sink_radii(radii, VF.ndim - 1)
    VFn = normalize_vectorfield(VF, normalize=normalize, min_speed=min_speed)
    sm = normalize_sink(radii, typ=np.float64, circle=circle)
    out = np.zeros(VF.shape[1:])
    for c in range(VF.shape[0]):
        out += fftcc_crop(sink(radii, c + 1, sm), VFn[c])
    if divide_by == "N":
        out /= float(np.sum(sm > 0))
    elif divide_by == "mags":
        out /= fftcc_crop(np.ones(sm.shape), magnitudes(VFn))
    return out


def multiscale_divergence(radii_list, VF, min_value=0.2, normalize=True, min_speed=0, divide_by="N"):
    """multiscale_divergence (postprocessing.jl:948-980): per vector the
    largest divergence and convergence over the scales, and the scale (the
    first radius) that gave it."""
    VF = np.asarray(VF, dtype=np.float64)
    size = VF.shape[1:]
    mxd = np.zeros(size)
    mxc = np.zeros(size)
    sd = np.zeros(size, dtype=np.int64)
    sc = np.zeros(size, dtype=np.int64)
    for rad in radii_list:
        d = -1 * divergence(rad, VF, normalize=normalize, min_speed=min_speed, divide_by=divide_by)
        rr = _sink_radii(rad, len(size))[0]
        for i in np.ndindex(*size):
            divg = d[i]
            conv = -1 * divg
            if divg > min_value and divg > mxd[i]:
                sd[i] = rr
                mxd[i] = divg
            if conv > min_value and conv > mxc[i]:
                sc[i] = rr
                mxc[i] = conv
    return sd, mxd, sc, mxc


def average_NDT(radius1, radius2, VF):
    """average_NDT (postprocessing.jl:386-414): its loop computes two local
    means and discards them (and the VF method iterates an undefined
    `arrays`); restated as the space-time window mean its name describes:
    the last grid axis is time, averaged over +-radius2, the others over
    +-radius1."""
    VF = np.asarray(VF, dtype=np.float64)
    nd = VF.ndim - 1
    r = _radii(radius1, nd - 1) + (int(radius2),)
    return average(r, VF)


# --------------------------------------------------------------------------
# pseudo-trajectories (postprocessing.jl:988-1120)
# --------------------------------------------------------------------------
_M64 = (1 << 64) - 1


def traj_hash(seed, p, d):
    """The random variant's starting-position generator (a build-defined
    replacement for Julia's rand): splitmix64's finaliser of
    seed + (3p + d + 1) * 0x9E3779B97F4A7C15, in 64-bit unsigned arithmetic."""
    z = (seed + (3 * p + d + 1) * 0x9E3779B97F4A7C15) & _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def pivtrajectories(comps, T0, T1, numpoints=0, subregion=None, scale=(1, 1, 1), grid=False, step=(1, 1, 1),
                    seed=0):
    """PIVtrajectories / PIVtrajectories_grid (postprocessing.jl:988-1120),
    one particle at a time as the reference's loop: comps = [U, V(, W)],
    (d1, d2[, d3], frames) arrays; subregion per axis as (lo, hi) 1-based
    inclusive, (1, 0) = the default 2:dims-1.  Positions are Float32 and
    1-based; the displacement is sampled at round(Int64, pos) (ties to even,
    :1037/:1104) and the trajectory freezes once that leaves the field
    (:1040-1045).  Starting positions: the grid in the reference's loop order
    (y fastest, :1070), or traj_hash for the random variant (the reference
    calls rand, :1009)."""
    nd = len(comps)
    dims = comps[0].shape[:nd]
    numT = T1 - T0
    sub = subregion if subregion is not None else [(1, 0)] * nd
    sc = (scale,) * 3 if np.isscalar(scale) else tuple(scale)
    st = (step,) * 3 if np.isscalar(step) else tuple(step)
    lo, ln, stp = [], [], []
    for d in range(nd):
        a, b = sub[d]
        if a > b:
            a, b = 2, dims[d] - 1
        s_ = st[d] if grid else 1
        lo.append(a)
        stp.append(s_)
        ln.append((b - a) // s_ + 1)
    n = int(np.prod(ln)) if grid else int(numpoints)
    out = [np.zeros((numT, n), dtype=np.float32, order="F") for _ in range(nd)]

    def sample(q, frame1):
        return [np.float32(float(sc[d]) * float(comps[d][tuple(x - 1 for x in q) + (frame1 - 1,)]))
                for d in range(nd)]

    for p in range(n):
        if grid:
            rem, s = p, []
            for d in range(nd):
                s.append(lo[d] + stp[d] * (rem % ln[d]))
                rem //= ln[d]
        else:
            s = [lo[d] + stp[d] * (traj_hash(seed, p, d) % ln[d]) for d in range(nd)]
        pos = [np.float32(x) for x in s]
        for d in range(nd):
            out[d][0, p] = pos[d]
        dv = sample(s, T0)
        for t in range(1, numT):
            pos = [np.float32(pos[d] + dv[d]) for d in range(nd)]
            for d in range(nd):
                out[d][t, p] = pos[d]
            r = [np.rint(x) for x in pos]
            if any(not (1 <= x <= dims[d]) for d, x in enumerate(r)):
                for d in range(nd):
                    out[d][t:, p] = out[d][t - 1, p]
                break
            dv = sample([int(x) for x in r], T0 + t)
    return tuple(out)
