"""NumPy Float64 restatement of multi_quickPIV's PIV hot path (TEST ORACLE).

Test infrastructure only: the CUDA product never imports this module.  Every
function cites the Julia source it restates (paths relative to the
multi_quickPIV repository).  Julia is 1-based and column-major; here arrays
keep the SAME logical axes (axis 0 = Julia dimension 1 = rows/"y"), and all
coordinates named ``*_TLF``/``*_BRB``/``*_off`` keep the reference's 1-based
values so the formulas read like the Julia code.  Slicing converts to 0-based
at the last moment.

FFTW (FFTW_jll 3.3.10+0, FFTW.jl 1.6.0, not vendored in the reference) is
replaced by NumPy's pocketfft in Float64: both compute the same unnormalised
real DFT, and they differ only by rounding (~1e-16 relative).  The transform
size is the reference's own ``good_size_real`` choice so even the rounding
structure follows the reference.

Quirks reproduced on purpose (they change VF/SN):
  Q1  search-window border offset short by 2 (src/utils/piv_ops.jl:72)
  Q2  constructor swaps ``unpadded``/``good_pad`` (src/piv_parameters.jl:57-59)
  Q3  column-major strict-``>`` argmax starting from 0 (src/utils/common_ops.jl:98-124)
  Q5  SN region one short of the peak region (src/utils/piv_ops.jl:336-367)
  Q7  ZNCC subtracts the mean of the whole clipped search region (src/utils/zncc_ops.jl:17-25)
  Q8  skipped interrogation areas leave zeros (src/multi_quickPIV.jl:69)
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional, Sequence, Tuple

import numpy as np

ALGS = ("fftcc", "zncc", "nsqecc", "mask_nsqecc")


# --------------------------------------------------------------------------
# parameters: src/piv_parameters.jl
# --------------------------------------------------------------------------
def to_dims3(x):
    """toDims3 (src/piv_parameters.jl:8-11)."""
    if x is None:
        return None
    if isinstance(x, (int, np.integer)):
        return (int(x), int(x), int(x))
    x = tuple(int(v) for v in x)
    if len(x) == 2:
        return (x[0], x[1], 0)
    if len(x) == 3:
        return x
    raise ValueError("dims must be an Integer, a 2-tuple or a 3-tuple")


def parse_corr(corr: str) -> str:
    """parseCorr (src/piv_parameters.jl:13-22).  "znc"/"fftc"/"nsqec" name
    undefined Julia types there (UndefVarError); unknown strings fall back to
    NSQECC."""
    c = corr.lower()
    if c == "zncc":
        return "zncc"
    if c == "fft":
        return "fftcc"
    if c == "nsqecc":
        return "nsqecc"
    if c in ("znc", "fftc", "nsqec"):
        raise ValueError(f"corr_alg {corr!r} names an undefined algorithm type in the reference")
    return "nsqecc"


@dataclass
class OracleParams:
    """PIVParameters (src/piv_parameters.jl:28-45)."""
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
    threshold: float = -1.0
    mask_threshold: float = -1.0
    ndims: int = 3
    ovp_th: float = 0.5


def set_piv_parameters(corr_alg="nsqecc", unpadded=True, good_pad=True, odd_pad=False,
                       interSize=32, searchMargin=10, overlap=0, step=None,
                       multipass=1, computeSN=False, threshold=-1.0,
                       mask_threshold=-1.0, ndims=3, ovp_th=0.5) -> OracleParams:
    """setPIVParameters (src/piv_parameters.jl:67-81) through the positional
    constructor (:48-64), which stores ``good_pad`` in ``unpadded`` and vice
    versa (Q2)."""
    return OracleParams(parse_corr(corr_alg), bool(good_pad), bool(unpadded), bool(odd_pad),
                        to_dims3(interSize), to_dims3(searchMargin), to_dims3(overlap),
                        to_dims3(step), int(multipass), bool(computeSN), float(threshold),
                        float(mask_threshold), int(ndims), float(ovp_th))


def _ovp(p, scale=1):
    """_ovp (src/piv_parameters.jl:83)."""
    return np.array(p.overlap[:p.ndims], dtype=np.int64) * scale


def _isize(p, scale=1):
    """_isize (src/piv_parameters.jl:84)."""
    return np.array(p.interSize[:p.ndims], dtype=np.int64) * scale


def _smarg(p, scale=1):
    """_smarg (src/piv_parameters.jl:85)."""
    return np.array(p.searchMargin[:p.ndims], dtype=np.int64) * scale


def _ssize(p, scale=1):
    """_ssize (src/piv_parameters.jl:86)."""
    return _isize(p, scale) + 2 * _smarg(p, scale)


def _step(p, scale=1):
    """_step (src/piv_parameters.jl:87)."""
    if p.step is None:
        return _isize(p, scale) - _ovp(p, scale)
    return np.array(p.step[:p.ndims], dtype=np.int64) * scale


# --------------------------------------------------------------------------
# geometry: src/utils/piv_ops.jl, src/utils/common_ops.jl
# --------------------------------------------------------------------------
def get_vectorfield_size(input_size, isize, step):
    """get_vectorfield_size (src/utils/piv_ops.jl:11-14):
    ``length.(StepRange.(1, step, size .- isize .+ 1))``."""
    out = []
    for n, i, s in zip(input_size, isize, step):
        stop = int(n) - int(i) + 1
        out.append(0 if stop < 1 else (stop - 1) // int(s) + 1)
    return tuple(out)


def linear2cartesian(lidx: int, size) -> Tuple[int, ...]:
    """linear2cartesian (src/utils/common_ops.jl:54-67), 1-based, column-major."""
    if len(size) == 2:
        h = size[0]
        x = -(-lidx // h)
        y = lidx - (x - 1) * h
        return (y, x)
    h, w = size[0], size[1]
    z = -(-lidx // (h * w))
    x = -(-(lidx - (z - 1) * h * w) // h)
    y = lidx - (x - 1) * h - (z - 1) * h * w
    return (y, x, z)


def get_interrogation_coordinates(vf_idx, vf_size, isize, step):
    """get_interrogation_coordinates (src/utils/piv_ops.jl:38-50)."""
    vfc = np.array(linear2cartesian(vf_idx, vf_size), dtype=np.int64)
    IR_TLF = 1 + (vfc - 1) * step
    IR_BRB = IR_TLF + isize - 1
    return IR_TLF, IR_BRB


def get_search_coordinates(IR_TLF, IR_BRB, input_size, SM, displacement=None):
    """get_search_coordinates (src/utils/piv_ops.jl:59-76), including the
    off-by-2 top/left/front offset of :72 (Q1)."""
    size = np.asarray(input_size, dtype=np.int64)
    d = np.zeros_like(SM) if displacement is None else np.asarray(displacement, dtype=np.int64)
    SR_TLF = np.maximum(1, IR_TLF - SM + d)
    SR_BRB = np.minimum(size, IR_BRB + SM + d)
    SR_TLF_off = np.abs(np.minimum(0, IR_TLF - (SM + d - 1)))
    SR_BRB_off = np.abs(np.minimum(0, size - (IR_BRB + SM + d)))
    return SR_TLF, SR_BRB, SR_TLF_off, SR_BRB_off


def coords_for(vf_idx, vf_size, input_size, isize, SM, step):
    """get_interrogation_and_search_coordinates (src/utils/piv_ops.jl:82-85)."""
    IR_TLF, IR_BRB = get_interrogation_coordinates(vf_idx, vf_size, isize, step)
    return (IR_TLF, IR_BRB) + get_search_coordinates(IR_TLF, IR_BRB, input_size, SM)


def _sl(lo1, hi1):
    """1-based inclusive [lo1, hi1] -> 0-based slice."""
    return slice(int(lo1) - 1, int(hi1))


def maxval(a) -> float:
    """maxval (src/utils/common_ops.jl:29-47): the maximum for finite input."""
    return float(np.max(a))


def skip_inter_region(img1, IR_TLF, IR_BRB, threshold) -> bool:
    """skip_inter_region (src/utils/piv_ops.jl:134-146)."""
    if threshold < 0:
        return False
    view = img1[tuple(_sl(a, b) for a, b in zip(IR_TLF, IR_BRB))]
    return maxval(view) < threshold


def skip_inter_region_masked(img1, mask, IR_TLF, IR_BRB, threshold, mask_threshold) -> bool:
    """Masked skip_inter_region (src/utils/piv_ops.jl:148-157): both tests use
    ``> 0`` thresholds."""
    sl = tuple(_sl(a, b) for a, b in zip(IR_TLF, IR_BRB))
    skip = False
    if threshold > 0:
        skip = maxval(img1[sl]) < threshold
    if mask_threshold > 0:
        skip = skip or (maxval(mask[sl]) < mask_threshold)
    return skip


# --------------------------------------------------------------------------
# FFT sizes: src/utils/fft_ops.jl:145-198
# --------------------------------------------------------------------------
def _root(base, goal, mul=1):
    """root (src/utils/fft_ops.jl:165-171)."""
    n = 0
    while mul * base ** (n + 1) < goal:
        n += 1
    return n


def good_size_real(n: int) -> int:
    """good_size_real (src/utils/fft_ops.jl:175-198)."""
    if n <= 6:
        return n
    bestfac = 2 * n
    for n5 in range(0, _root(11, bestfac, 5) + 1):
        x = 5 ** n5
        while x < n:
            x *= 2
        while True:
            if x < n:
                x *= 3
            elif x > n:
                if x < bestfac:
                    bestfac = x
                if x & 1 == 1:
                    break
                x >>= 1
            else:
                return n
    return bestfac


def compute_csize_and_paddings(size_F, size_G, unpadded=False, good_pad=False, odd_pad=False):
    """compute_csize_and_paddings (src/utils/fft_ops.jl:145-158)."""
    size_F = np.asarray(size_F)
    size_G = np.asarray(size_G)
    csize0 = np.maximum(size_F, size_G) if unpadded else size_F + size_G - 1
    if good_pad:
        csize1 = np.array([good_size_real(int(c)) for c in csize0])
    else:
        csize1 = csize0 + (csize0 % 2 == 1) * int(odd_pad)
    r2c_pad = np.zeros_like(csize1)
    r2c_pad[0] = 1 + (csize1[0] % 2 == 0)
    return csize1, r2c_pad, csize1 - csize0


# --------------------------------------------------------------------------
# copies: src/utils/piv_ops.jl:95-127, zncc_ops.jl:3-25, masked_nsqecc_ops.jl:19-42
# --------------------------------------------------------------------------
def copy_inter_region(img, IR_TLF, IR_BRB, cs):
    """copy_inter_region! (src/utils/piv_ops.jl:99-109)."""
    pad = np.zeros(tuple(cs), dtype=np.float64)
    src = img[tuple(_sl(a, b) for a, b in zip(IR_TLF, IR_BRB))]
    pad[tuple(slice(0, s) for s in src.shape)] = src
    return pad


def copy_search_region(img, SR_TLF, SR_BRB, SR_TLF_off, cs):
    """copy_search_region! (src/utils/piv_ops.jl:115-127): the clipped search
    region lands at 1+SR_TLF_off (1-based) in the zeroed pad."""
    pad = np.zeros(tuple(cs), dtype=np.float64)
    src = img[tuple(_sl(a, b) for a, b in zip(SR_TLF, SR_BRB))]
    pad[tuple(slice(int(o), int(o) + s) for o, s in zip(SR_TLF_off, src.shape))] = src
    return pad


def copy_inter_region_minus_mean(img, IR_TLF, IR_BRB, cs):
    """copy_inter_region_minus_mean! (src/utils/zncc_ops.jl:7-12)."""
    pad = np.zeros(tuple(cs), dtype=np.float64)
    src = np.asarray(img[tuple(_sl(a, b) for a, b in zip(IR_TLF, IR_BRB))], dtype=np.float64)
    pad[tuple(slice(0, s) for s in src.shape)] = src - src.sum() / src.size
    return pad


def copy_search_region_minus_mean(img, SR_TLF, SR_BRB, SR_TLF_off, cs):
    """copy_search_region_minus_mean! (src/utils/zncc_ops.jl:18-25): the mean
    of the whole clipped search region (Q7); the pad outside it stays 0."""
    pad = np.zeros(tuple(cs), dtype=np.float64)
    src = np.asarray(img[tuple(_sl(a, b) for a, b in zip(SR_TLF, SR_BRB))], dtype=np.float64)
    pad[tuple(slice(int(o), int(o) + s) for o, s in zip(SR_TLF_off, src.shape))] = src - src.sum() / src.size
    return pad


# --------------------------------------------------------------------------
# correlation kernels
# --------------------------------------------------------------------------
def fftcc(padF, padG, nd=None):
    """_FFTCC! (src/crosscorrelation_algorithms/fftcc.jl:101-126) with corr_dot!
    (src/utils/fft_ops.jl:95-105): c2r(conj(r2c(F)) .* r2c(G)) / prod(csize),
    i.e. cc[s] = sum_x F(x) G(x+s) (circular).  The transform runs over the
    last ``nd`` axes (all of them by default), so stacked pads batch."""
    nd = padF.ndim if nd is None else nd
    axes = tuple(range(-nd, 0))
    shape = padF.shape[-nd:]
    Fh = np.fft.rfftn(padF, axes=axes)
    Gh = np.fft.rfftn(padG, axes=axes)
    return np.fft.irfftn(np.conj(Fh) * Gh, s=shape, axes=axes)


def integral_array_sq(padG, SS):
    """integralArraySQ! (src/utils/common_ops.jl:142-180) over pad_G[1:SS]:
    int[r,c(,z)] = sum of squares over the box below (r,c(,z)), with a zero
    first row/column/plane."""
    sub = np.asarray(padG[tuple(slice(0, int(s)) for s in SS)], dtype=np.float64) ** 2
    out = np.zeros(tuple(int(s) + 1 for s in SS), dtype=np.float64)
    acc = sub
    for ax in range(sub.ndim):
        acc = np.cumsum(acc, axis=ax)
    out[tuple(slice(1, None) for _ in SS)] = acc
    return out


def window_sums(int_arr, isize, SM):
    """add_numerator_nsqecc (src/utils/common_ops.jl:203-245): the sum over the
    interrogation-sized window of pad_G for every fully-overlapping
    translation k = 1:2SM+1 (same sign order as the reference)."""
    P = [2 * int(m) + 1 for m in SM]
    nd = len(P)
    if nd == 2:
        ih, iw = int(isize[0]), int(isize[1])
        T = slice(0, P[0]); L = slice(0, P[1])
        D = slice(ih, ih + P[0]); R = slice(iw, iw + P[1])
        out = np.zeros(P)
        out += int_arr[D, R]
        out += int_arr[T, L]
        out -= int_arr[T, R]
        out -= int_arr[D, L]
        return out
    ih, iw, id_ = (int(v) for v in isize)
    T = slice(0, P[0]); L = slice(0, P[1]); F = slice(0, P[2])
    D = slice(ih, ih + P[0]); R = slice(iw, iw + P[1]); B = slice(id_, id_ + P[2])
    out = np.zeros(P)
    out += int_arr[D, R, B]
    out -= int_arr[T, L, F]
    out -= int_arr[T, R, B]
    out -= int_arr[D, L, B]
    out -= int_arr[D, R, F]
    out += int_arr[D, L, F]
    out += int_arr[T, R, F]
    out += int_arr[T, L, B]
    return out


def zncc_from_cc(cc, sumF2, S2win, SM):
    """fftcc2zncc! (src/utils/zncc_ops.jl:29-50) on the fully-overlapping block."""
    fov = tuple(slice(0, 2 * int(m) + 1) for m in SM)
    out = cc.copy()
    den = np.sqrt(S2win) * math.sqrt(sumF2)
    with np.errstate(divide="ignore", invalid="ignore"):
        out[fov] = cc[fov] / den
    return out


def nsqecc_from_cc(cc, sumF2, S2win, SM):
    """fftcc2nsqecc! (src/utils/nsqecc_ops.jl:1-25): den/(den+num) with
    num = sumF2 + sum_win(G^2) - 2cc and den = sqrt(sum_win(G^2))*sqrt(sumF2)."""
    fov = tuple(slice(0, 2 * int(m) + 1) for m in SM)
    out = cc.copy()
    num = cc[fov] * -2.0
    num = num + sumF2
    num = num + S2win
    den = np.sqrt(S2win) * math.sqrt(sumF2)
    with np.errstate(divide="ignore", invalid="ignore"):
        out[fov] = den / (num + den)
    return out


def masknsqecc_from_cc(cc1, cc2, sumF2, SM):
    """fftcc2masknsqecc! (src/utils/masked_nsqecc_ops.jl:123-142)."""
    fov = tuple(slice(0, 2 * int(m) + 1) for m in SM)
    out = cc1.copy()
    num = cc1[fov] * -2.0
    num = num + sumF2
    num = num + cc2[fov]
    den = np.sqrt(np.abs(cc2[fov])) * math.sqrt(sumF2)
    with np.errstate(divide="ignore", invalid="ignore"):
        out[fov] = den / (num + den)
    return out


def mask_sumF2(maskF_win, mask_win):
    """The sumF2 loop of _mask_NSQECC! (src/crosscorrelation_algorithms/mask_nsqecc.jl:141-149):
    sum(maskF^2 / wi), wi = mask where mask > 0 else 1."""
    wi = np.where(mask_win > 0, mask_win, 1.0)
    return float(np.sum(maskF_win * maskF_win / wi))


# --------------------------------------------------------------------------
# peak, sub-pixel, SN: src/utils/common_ops.jl:98-124, src/utils/piv_ops.jl:249-367
# --------------------------------------------------------------------------
def first_fullovp_peak(cmat, SM, TLF_off, BRB_off):
    """first_fullovp_peak (src/utils/common_ops.jl:98-124): strict ``>`` scan in
    column-major order over [1+TLF_off, 1+2SM-BRB_off] starting from
    max_value = 0 (Q3).  Returns the 1-based peak and its value; (0,..) and 0
    when no value is > 0."""
    lo = [1 + int(o) for o in TLF_off]
    hi = [1 + 2 * int(m) - int(o) for m, o in zip(SM, BRB_off)]
    nd = len(lo)
    if any(h < l for l, h in zip(lo, hi)):
        return tuple([0] * nd), 0.0
    sub = cmat[tuple(slice(l - 1, h) for l, h in zip(lo, hi))]
    flat = sub.ravel(order="F")
    with np.errstate(invalid="ignore"):
        ok = flat > 0
    if not ok.any():
        return tuple([0] * nd), 0.0
    m = np.max(flat[ok])
    idx = int(np.flatnonzero(ok & (flat == m))[0])
    loc = np.unravel_index(idx, sub.shape, order="F")
    return tuple(int(l + i) for l, i in zip(lo, loc)), float(m)


def gaussian_refinement(cmat, peak, maxv, SM, TLF_off, BRB_off):
    """gaussian_refinement (src/utils/piv_ops.jl:282-291) with gaussian /
    gaussian_2D / gaussian_3D (:294-326).  Returns the refined 1-based peak."""
    nd = len(peak)
    inside = all(p > 1 + int(o) for p, o in zip(peak, TLF_off)) and \
        all(p < 1 + 2 * int(m) - int(o) for p, m, o in zip(peak, SM, BRB_off))
    if not inside:
        return np.array(peak, dtype=np.float64)
    nb = cmat[tuple(slice(p - 2, p + 1) for p in peak)]
    minv = float(np.min(nb))
    c0 = tuple(p - 1 for p in peak)
    out = np.array(peak, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        mx = math.log(1 + maxv - minv)
        for d in range(nd):
            lo = list(c0); lo[d] -= 1
            hi = list(c0); hi[d] += 1
            a = math.log(1 + float(cmat[tuple(lo)]) - minv)
            b = math.log(1 + float(cmat[tuple(hi)]) - minv)
            num = a - b
            den = 2 * a - 4 * mx + 2 * b
            out[d] += np.float64(num) / np.float64(den)
    return out


def gaussian_displacement(cmat, SM, TLF_off, BRB_off):
    """gaussian_displacement (src/utils/piv_ops.jl:249-273), unpadded branch."""
    center = np.asarray(SM, dtype=np.float64) + 1
    peak, mv = first_fullovp_peak(cmat, SM, TLF_off, BRB_off)
    return gaussian_refinement(cmat, peak, mv, SM, TLF_off, BRB_off) - center


def compute_SN(cmat, SM, TLF_off, BRB_off):
    """compute_SN (src/utils/piv_ops.jl:336-367): max/((sum-max)/(len-1)) over
    [1+TLF_off, 2SM-BRB_off] (Q5).  The reference throws a BoundsError for 3D
    (:357-360); this build defines 3D SN as the same formula over 3 axes."""
    lo = [1 + int(o) for o in TLF_off]
    hi = [2 * int(m) - int(o) for m, o in zip(SM, BRB_off)]
    sub = cmat[tuple(slice(l - 1, h) for l, h in zip(lo, hi))]
    n = sub.size
    mx = float(np.max(sub))
    with np.errstate(divide="ignore", invalid="ignore"):
        avg = (float(np.sum(sub)) - mx) / (n - 1)
        return np.float64(mx) / np.float64(avg)


def sn_kappa(cmat, SM, TLF_off, BRB_off):
    """Condition number of compute_SN for one IA (test infrastructure, not a
    reference function): SN = top / den over the region compute_SN reads, so
    an absolute error e on every similarity value moves SN by at most
    e / |top| + e / |den| relative, to first order; kappa = scale / |top| +
    scale / |den| with scale the largest magnitude on the lags
    first_fullovp_peak searches ([1+TLF_off, 1+2SM-BRB_off])."""
    lo = [1 + int(o) for o in TLF_off]
    hi = [2 * int(m) - int(o) for m, o in zip(SM, BRB_off)]
    sub = cmat[tuple(slice(l - 1, h) for l, h in zip(lo, hi))]
    reg = cmat[tuple(slice(l - 1, h + 1) for l, h in zip(lo, hi))]
    if sub.size < 2 or not np.isfinite(sub).all():
        return np.inf
    top = float(np.max(sub))
    den = (float(np.sum(sub)) - top) / (sub.size - 1)
    scale = float(np.max(np.abs(reg)))
    with np.errstate(divide="ignore", invalid="ignore"):
        k = scale / abs(top) + scale / abs(den)
    return k if np.isfinite(k) else np.inf


# --------------------------------------------------------------------------
# one interrogation area, end to end
# --------------------------------------------------------------------------
@dataclass
class IAResult:
    displacement: np.ndarray
    sn: float
    skipped: bool
    corr: Optional[np.ndarray] = field(default=None, repr=False)


def correlate_ia(alg, img1, img2, mask, coords, isize, SM, cs):
    """prepare_inputs! + crosscorrelation! for one interrogation area
    (fftcc.jl:58-71/97-126, zncc.jl:62-76/113-144, nsqecc.jl:65-80/111-138,
    mask_nsqecc.jl:66-82/126-160).  Returns the correlation matrix of size cs
    whose fully-overlapping block [0:2SM+1] holds the similarity values."""
    IR_TLF, IR_BRB, SR_TLF, SR_BRB, TLF_off, BRB_off = coords
    SS = isize + 2 * SM
    fov_is = tuple(slice(0, int(i)) for i in isize)
    if alg == "fftcc":
        pF = copy_inter_region(img1, IR_TLF, IR_BRB, cs)
        pG = copy_search_region(img2, SR_TLF, SR_BRB, TLF_off, cs)
        return fftcc(pF, pG)
    if alg in ("zncc", "nsqecc"):
        if alg == "zncc":
            pF = copy_inter_region_minus_mean(img1, IR_TLF, IR_BRB, cs)
            pG = copy_search_region_minus_mean(img2, SR_TLF, SR_BRB, TLF_off, cs)
        else:
            pF = copy_inter_region(img1, IR_TLF, IR_BRB, cs)
            pG = copy_search_region(img2, SR_TLF, SR_BRB, TLF_off, cs)
        int2 = integral_array_sq(pG, SS)
        sumF2 = float(np.sum(pF[fov_is] ** 2))
        cc = fftcc(pF, pG)
        S2 = window_sums(int2, isize, SM)
        if alg == "zncc":
            return zncc_from_cc(cc, sumF2, S2, SM)
        return nsqecc_from_cc(cc, sumF2, S2, SM)
    if alg == "mask_nsqecc":
        pF = copy_inter_region(img1, IR_TLF, IR_BRB, cs)
        pM = copy_inter_region(mask, IR_TLF, IR_BRB, cs)
        pF = pF * pM
        pG = copy_search_region(img2, SR_TLF, SR_BRB, TLF_off, cs)
        pG2 = pG * pG
        sumF2 = mask_sumF2(pF[fov_is], pM[fov_is])
        cc1 = fftcc(pF, pG)
        cc2 = fftcc(pM, pG2)
        return masknsqecc_from_cc(cc1, cc2, sumF2, SM)
    raise ValueError(alg)


def fft_size(p, isize, SS):
    """The transform size the reference plans (allocate_tmp_data, e.g.
    src/crosscorrelation_algorithms/fftcc.jl:42), honouring the stored
    (swapped, Q2) flags.  Only unpadded=good_pad=true is a supported path
    (src/utils/piv_ops.jl:261-266 prints ERROR otherwise)."""
    cs, _, _ = compute_csize_and_paddings(isize, SS, unpadded=p.unpadded,
                                          good_pad=p.good_pad, odd_pad=p.odd_pad)
    return cs


def piv_single_pass(img1, img2, p: OracleParams, mask=None, mask_skip=None,
                    predictor=None, scale=1, keep_corr=False, kappa_out=None):
    """One pass of PIV_CPU (src/multi_quickPIV.jl:40-96) at ``scale``.

    ``predictor`` (integer array (N, *vf_size), optional) shifts each search
    window by a whole-pixel displacement; this multi-pass predictor is
    build-defined (the reference never passes one, src/utils/piv_ops.jl:64,84):
    the search window is the one of a virtual interrogation area moved by the
    predictor (clamped inside the image), and the reported displacement is
    predictor + measured.

    ``kappa_out`` (array of the vector-field shape, optional) receives each
    IA's SN condition number (sn_kappa); test infrastructure.
    """
    img1 = np.asarray(img1)
    img2 = np.asarray(img2)
    N = img1.ndim
    if img1.shape != img2.shape:
        raise AssertionError("PIV inputs need to have the same size.")
    if not (p.unpadded and p.good_pad):
        raise ValueError("only unpadded=good_pad=true is supported by the reference's peak search")
    alg = "mask_nsqecc" if mask is not None else p.corr_alg
    isize, SM, step = _isize(p, scale), _smarg(p, scale), _step(p, scale)
    SS = isize + 2 * SM
    cs = fft_size(p, isize, SS)
    size = img1.shape
    vf_size = get_vectorfield_size(size, isize, step)
    VF = np.zeros((N,) + vf_size, dtype=np.float64)
    SN = np.zeros(vf_size, dtype=np.float64) if p.computeSN else None
    corrs = {} if keep_corr else None
    nvf = int(np.prod(vf_size)) if len(vf_size) else 0
    for vf_idx in range(1, nvf + 1):
        IR_TLF, IR_BRB = get_interrogation_coordinates(vf_idx, vf_size, isize, step)
        vfc = tuple(c - 1 for c in linear2cartesian(vf_idx, vf_size))
        d = None
        if predictor is not None:
            d = np.array([int(predictor[(n,) + vfc]) for n in range(N)], dtype=np.int64)
            d = np.clip(d, 1 - IR_TLF, np.asarray(size) - IR_BRB)
            vIR_TLF, vIR_BRB = IR_TLF + d, IR_BRB + d
        else:
            vIR_TLF, vIR_BRB = IR_TLF, IR_BRB
        SR = get_search_coordinates(vIR_TLF, vIR_BRB, size, SM)
        coords = (IR_TLF, IR_BRB) + SR
        if mask is not None:
            mskip = mask if mask_skip is None else mask_skip
            if skip_inter_region_masked(img1, mskip, IR_TLF, IR_BRB, p.threshold, p.mask_threshold):
                continue
        elif skip_inter_region(img1, IR_TLF, IR_BRB, p.threshold):
            continue
        cm = correlate_ia(alg, img1, img2, mask, coords, isize, SM, cs)
        disp = gaussian_displacement(cm, SM, SR[2], SR[3])
        if d is not None:
            disp = disp + d
        VF[(slice(None),) + vfc] = disp
        if SN is not None and scale == 1:
            SN[vfc] = compute_SN(cm, SM, SR[2], SR[3])
        if kappa_out is not None:
            kappa_out[vfc] = sn_kappa(cm, SM, SR[2], SR[3])
        if keep_corr:
            corrs[vfc] = cm[tuple(slice(0, 2 * int(m) + 1) for m in SM)].copy()
    if keep_corr:
        return VF, SN, corrs
    return VF, SN


def PIV(img1, img2, p: OracleParams, mask=None, mask_skip=None, refine=False, keep_corr=False, kappa_out=None):
    """PIV (src/multi_quickPIV.jl:17-29).

    With ``refine=False`` (the reference's behaviour) every pass of the
    multipass loop re-runs the scale-1 geometry (Q6), so the result equals a
    single pass.  With ``refine=True`` (or 1) the build-defined multi-pass
    runs scales 2^(m-1), ..., 2, 1 with integer predictors taken from the
    nearest coarser vector (see predictor_from_coarse); with ``refine=2`` (or
    "deform") each finer pass runs on the pair deformed around the previous
    pass's interpolated field (deform_images) and adds that field back at
    its IA centres."""
    N = np.asarray(img1).ndim
    p.ndims = N
    if not refine or p.multipass <= 1:
        return piv_single_pass(img1, img2, p, mask=mask, mask_skip=mask_skip, keep_corr=keep_corr,
                               kappa_out=kappa_out)
    size = np.asarray(img1).shape
    pred = None
    prev = None
    deform = refine in (2, "deform")
    if deform and mask is not None:
        raise ValueError("window deformation does not take masks")
    for level in range(p.multipass - 1, -1, -1):
        scale = 2 ** level
        a1, a2 = np.asarray(img1), np.asarray(img2)
        if prev is not None and deform and prev[0].size:
            # the deforming refinement: the pair resampled around the dense
            # predictor of the previous pass; this pass measures the residual
            isz_c, st_c = _isize(p, prev[1]), _step(p, prev[1])
            a1, a2 = deform_images(a1, a2, prev[0], isz_c, st_c)
        elif prev is not None and not deform:
            pred = predictor_from_coarse(prev[0], prev[1], size, p, scale)
        VF, SN = piv_single_pass(a1, a2, p, mask=mask, mask_skip=mask_skip,
                                 predictor=pred, scale=scale, kappa_out=kappa_out if level == 0 else None)
        if prev is not None and deform and prev[0].size and VF.size:
            isz_f, st_f = _isize(p, scale), _step(p, scale)
            vf = VF.shape[1:]
            cen = np.stack(np.meshgrid(*[np.arange(n) * st_f[d] + 0.5 * (isz_f[d] - 1)
                                         for d, n in enumerate(vf)], indexing="ij"), -1)
            D = deform_predictor(prev[0], _isize(p, prev[1]), _step(p, prev[1]), cen)
            live = np.ones(vf, dtype=bool)
            if p.threshold >= 0:
                for k in np.ndindex(*vf):
                    sl = tuple(slice(k[d] * st_f[d], k[d] * st_f[d] + isz_f[d]) for d in range(N))
                    live[k] = not (np.max(a1[sl]) < p.threshold)
            for d in range(N):
                VF[d] = np.where(live, VF[d] + D[..., d], VF[d])
        prev = (VF, scale)
    return VF, SN


def _deform_weights(f, n):
    """Clamped multilinear index/weight along one axis: f in fractional index
    units, n points; returns (j0, j1, t)."""
    f = np.clip(f, 0.0, float(n - 1))
    j0 = np.minimum(np.floor(f).astype(np.int64), n - 1)
    j1 = np.minimum(j0 + 1, n - 1)
    return j0, j1, f - j0


def deform_predictor(VFc, isz_c, st_c, pos):
    """Build-defined dense predictor (the deforming refinement): the coarse
    vectors at their IA centres j * step + (interSize - 1) / 2 (0-based),
    interpolated multilinearly at positions pos (array (..., N)), clamped to
    the outermost centres; non-finite vectors count as 0.  Weights multiply
    and terms accumulate in corner order k = 0 .. 2^N - 1 (axis d set when bit
    d of k is), each product and sum rounded on its own."""
    N = VFc.shape[0]
    vf_c = VFc.shape[1:]
    V = np.where(np.isfinite(VFc), VFc, 0.0)
    js = [_deform_weights((pos[..., d] - 0.5 * (isz_c[d] - 1)) / st_c[d], vf_c[d]) for d in range(N)]
    D = np.zeros(pos.shape[:-1] + (N,))
    for k in range(1 << N):
        w = np.ones(pos.shape[:-1])
        idx = []
        for d in range(N):
            up = (k >> d) & 1
            j0, j1, t = js[d]
            w = w * (t if up else 1.0 - t)
            idx.append(j1 if up else j0)
        for c in range(N):
            D[..., c] = D[..., c] + w * V[(c,) + tuple(idx)]
    return D


def _deform_sample(img, pos):
    N = img.ndim
    js = [_deform_weights(pos[..., d], img.shape[d]) for d in range(N)]
    s = np.zeros(pos.shape[:-1])
    x = img.astype(np.float64)
    for k in range(1 << N):
        w = np.ones(pos.shape[:-1])
        idx = []
        for d in range(N):
            up = (k >> d) & 1
            j0, j1, t = js[d]
            w = w * (t if up else 1.0 - t)
            idx.append(j1 if up else j0)
        s = s + w * x[tuple(idx)]
    return s


def deform_images(img1, img2, VFc, isz_c, st_c):
    """The deforming refinement's resampled pair: img1(p - D(p)/2) and
    img2(p + D(p)/2), multilinear, clamped at the border, in FP64 and then
    the images' precision."""
    shape = img1.shape
    grids = np.meshgrid(*[np.arange(n, dtype=np.float64) for n in shape], indexing="ij")
    pos = np.stack(grids, -1)
    D = deform_predictor(VFc, isz_c, st_c, pos)
    o1 = _deform_sample(img1, pos + (-0.5 * D))
    o2 = _deform_sample(img2, pos + 0.5 * D)
    return o1.astype(img1.dtype), o2.astype(img2.dtype)


def predictor_from_coarse(VFc, scale_c, size, p, scale_f):
    """Build-defined multi-pass predictor: every fine interrogation area takes
    the rounded (half away from zero) displacement of the coarse
    interrogation area whose centre is nearest to its own centre (ties to the
    higher index), per axis."""
    N = VFc.shape[0]
    isz_c, st_c = _isize(p, scale_c), _step(p, scale_c)
    isz_f, st_f = _isize(p, scale_f), _step(p, scale_f)
    vf_f = get_vectorfield_size(size, isz_f, st_f)
    vf_c = VFc.shape[1:]
    if any(v == 0 for v in vf_c):  # the coarse pass had no IA: no shift
        return np.zeros((N,) + vf_f, dtype=np.int64)
    idx = []
    for d in range(N):
        jf = np.arange(vf_f[d])
        # centres in doubled coordinates to stay in integers: 2*(TLF-1) + isize - 1
        cf = 2 * jf * st_f[d] + isz_f[d] - 1
        # nearest coarse centre: argmin |2*jc*st_c + isz_c - 1 - cf|
        jc = np.floor((cf - (isz_c[d] - 1) + st_c[d]) / (2 * st_c[d])).astype(np.int64)
        idx.append(np.clip(jc, 0, vf_c[d] - 1))
    grids = np.meshgrid(*idx, indexing="ij")
    pred = np.zeros((N,) + vf_f, dtype=np.int64)
    for n in range(N):
        v = VFc[n][tuple(grids)]
        pred[n] = np.where(np.isfinite(v), np.sign(v) * np.floor(np.abs(v) + 0.5), 0).astype(np.int64)
    return pred


def get_vf_size_for(size, p, scale=1):
    return get_vectorfield_size(size, _isize(p, scale), _step(p, scale))


# --------------------------------------------------------------------------
# brute force (independent check of the FFT restatement)
# --------------------------------------------------------------------------
def brute_force_cc(padF, padG, isize, SM):
    """Direct spatial cc[s] = sum_x F(x) G(x+s) on the fully-overlapping block."""
    P = [2 * int(m) + 1 for m in SM]
    F = padF[tuple(slice(0, int(i)) for i in isize)]
    out = np.zeros(P)
    for s in np.ndindex(*P):
        G = padG[tuple(slice(si, si + int(i)) for si, i in zip(s, isize))]
        out[s] = float(np.sum(F * G))
    return out
