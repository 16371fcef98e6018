"""Shared comparison helpers for the parity tests."""
import numpy as np

import oracle.piv_oracle as O

# FP32 FFTs and planes with FP64 normalisation, against the Float64 oracle:
PLANE_RTOL = 2e-6      # |plane - oracle| <= PLANE_RTOL * max|oracle plane| on the searched lags
MASK_PLANE_RTOL = 5e-5 # masked NSQECC, IAs whose mask covers >= 25 %: the FP32 FFT error scales with
                       # the whole window while the masked sums scale with the covered part
VF_ATOL = 1e-3         # px, whenever the integer peak agrees
SN_RTOL = 1e-4         # relative; widened only per IA by its computed condition number (sn_ok)


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


def sn_condition_from(scale, top, den):
    """Condition number of compute_SN (src/utils/piv_ops.jl:336-367),
    SN = top / den with den the mean of the SN region without its maximum,
    under an absolute error of at most e on every plane value: to first order
    |dSN| / |SN| <= e / |top| + e / |den|, so with e = PLANE_RTOL * scale the
    relative SN error is at most PLANE_RTOL * kappa,
    kappa = scale / |top| + scale / |den|."""
    scale = np.asarray(scale, dtype=np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        k = scale / np.abs(top) + scale / np.abs(den)
    return np.where(np.isfinite(k), k, np.inf)


def sn_condition(oracle_corr, shape, IS, SM, st):
    """Per-IA kappa (sn_condition_from) from the oracle's similarity blocks
    (keep_corr=True), on the region compute_SN reads: [TLF_off,
    2SM - 1 - BRB_off] per axis."""
    vf = O.get_vectorfield_size(shape, IS, st)
    kappa = np.full(vf, np.inf)
    for k, cm in oracle_corr.items():
        reg = searched_region(shape, IS, SM, st, k)
        sreg = tuple(slice(r.start, r.stop - 1) for r in reg)
        b = cm[sreg]
        if b.size < 2 or not np.isfinite(b).all():
            continue
        top = float(np.max(b))
        den = (float(np.sum(b)) - top) / (b.size - 1)
        kappa[k] = sn_condition_from(float(np.max(np.abs(cm[reg]))), top, den)
    return kappa


def sn_ok(SN, SNo, kappa=None):
    """|SN - SNo| <= max(SN_RTOL, PLANE_RTOL * kappa) * |SNo|: 1e-4 relative,
    except where the IA's own condition number (sn_condition) times the plane
    tolerance is larger.  Without kappa the plain 1e-4 applies."""
    rel = SN_RTOL if kappa is None else np.maximum(SN_RTOL, PLANE_RTOL * np.asarray(kappa))
    diff = np.abs(SN - SNo)
    with np.errstate(invalid="ignore"):  # an infinite kappa times SN = 0 (a skipped IA)
        within = diff <= rel * np.abs(SNo)
    return (diff == 0) | within | ~np.isfinite(SNo)
