"""Shared comparison helpers for the parity tests."""
import numpy as np

import oracle.piv_oracle as O

# FP32 FFTs and planes with FP64 normalisation, against the Float64 oracle:
PLANE_RTOL = 2e-6      # |plane - oracle| <= PLANE_RTOL * max|oracle plane| on the searched lags
MASK_PLANE_RTOL = 5e-5 # masked NSQECC, IAs whose mask covers >= 25 %: the FP32 FFT error scales with
                       # the whole window while the masked sums scale with the covered part
VF_ATOL = 1e-3         # px, whenever the integer peak agrees
SN_RTOL = 1e-4         # plus the conditioning term |SN|^2/|max| * 1e-6


def searched_region(shape, IS, SM, st, k):
    """Lag box [TLF_off, 2SM - BRB_off] the reference searches for IA k
    (0-based vector-field coordinates), as slices."""
    vf = O.get_vectorfield_size(shape, IS, st)
    lin = int(np.ravel_multi_index(k, vf, order="F")) + 1
    c = O.coords_for(lin, vf, shape, np.asarray(IS), np.asarray(SM), np.asarray(st))
    return tuple(slice(int(t), 2 * int(m) - int(b) + 1) for t, m, b in zip(c[4], SM, c[5]))


def mask_coverage(mask, shape, IS, st):
    """Fraction of each IA covered by a positive mask, per vector-field cell."""
    vf = O.get_vectorfield_size(shape, IS, st)
    cov = np.zeros(vf)
    for k in np.ndindex(*vf):
        sl = tuple(slice(c * s, c * s + i) for c, s, i in zip(k, st, IS))
        cov[k] = float(np.mean(mask[sl] > 0))
    return cov


def compare_planes(planes, oracle_corr, shape, IS, SM, st, skip=None):
    """Max relative plane error on the searched lags, and a per-IA near-tie
    flag (top two oracle candidates closer than the FP32 error bound).
    IAs flagged in `skip` are left out of the plane comparison."""
    vf = O.get_vectorfield_size(shape, IS, st)
    worst = 0.0
    near_tie = np.zeros(vf, dtype=bool)
    for k, cm in oracle_corr.items():
        if skip is not None and skip[k]:
            continue
        ia = int(np.ravel_multi_index(k, vf, order="F"))
        reg = searched_region(shape, IS, SM, st, k)
        a = planes[..., ia][reg]
        b = cm[reg]
        if b.size == 0:
            continue
        fin = np.isfinite(b)
        assert np.array_equal(fin, np.isfinite(a)), f"non-finite lags differ at IA {k}"
        if not fin.any():  # e.g. an all-zero mask: 0/0 everywhere, as in the reference
            continue
        scale = np.max(np.abs(b[fin]))
        worst = max(worst, float(np.max(np.abs(a[fin] - b[fin]))) / scale)
        v = np.sort(b[fin].ravel())[::-1]
        near_tie[k] = v.size > 1 and (v[0] - v[1]) <= 4 * PLANE_RTOL * scale
    return worst, near_tie


def sn_ok(SN, SNo):
    tol = SN_RTOL * np.abs(SNo) + SNo ** 2 * 1e-6
    return (np.abs(SN - SNo) <= tol) | ~np.isfinite(SNo)
