"""Parity at the full sizes of the benchmarked workloads: every interrogation
area of the 256^2 Float64 FFTCC pair, of the 2048^2 Float32 Lamb-Oseen vortex
pair (NSQECC and ZNCC, 64,009 IAs each) and of the 512x512x256 Float32 shear
volumes (FFTCC, 14,415 IAs), through the C ABI (PIV -> mqp_piv), against the
C++/OpenMP Float64 restatement of the reference (oracle/cpu, itself checked
against the NumPy oracle in test_cpu_port.py).

Per workload the test states and bounds:
  - the largest sub-pixel error over the IAs whose integer peak agrees
    (<= 1e-3 px);
  - the number of near-tie IAs (the oracle's two largest similarity values on
    the searched lags closer than 4 x PLANE_RTOL x the largest magnitude),
    the only IAs allowed a different integer peak;
  - the largest SN relative error over the IAs within the plain 1e-4 budget,
    and the number of IAs that need their computed SN condition number
    (PLANE_RTOL x kappa > 1e-4, kappa = scale/|top| + scale/|den|, see
    tests.helpers.sn_condition_from) together with the largest error relative
    to that bound.
The figures are printed (pytest -s) as one PARITY line per workload.
"""
import json

import numpy as np
import pytest

import oracle.cpu_ref as CR
from multi_quickpiv_b200 import PIV, setPIVParameters, synth
from tests.helpers import PLANE_RTOL, SN_RTOL, VF_ATOL, sn_condition_from

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def port():
    CR.build()
    if not CR.available():
        pytest.fail("the C++ oracle port (oracle/cpu) is not built")


def _params(alg, IS, SM, st, thr=-1.0):
    pp = setPIVParameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True, threshold=thr)
    pp.ndims = len(IS)
    return pp


def _parity(name, i1, i2, pp, max_near_tie_frac, max_cond_frac):
    VF, SN = PIV(i1, i2, pp)
    VFc, SNc, D = CR.piv(i1, i2, pp.to_c(), diag=True)
    assert VF.shape == VFc.shape and SN.shape == SNc.shape
    n_ia = int(np.prod(SN.shape))
    live = D["skipped"] == 0
    # skipped IAs: zeros on both sides, bit for bit
    assert np.array_equal(VF[:, ~live], VFc[:, ~live]) and np.array_equal(SN[~live], SNc[~live])
    near_tie = live & ((D["top1"] - D["top2"]) <= 4 * PLANE_RTOL * D["scale"])
    err = np.abs(VF - VFc).max(axis=0)
    agree = live & (err <= VF_ATOL)
    bad = live & ~agree & ~near_tie
    assert not bad.any(), (name, np.argwhere(bad)[:5], float(err[bad].max()))
    max_subpx = float(err[agree].max()) if agree.any() else 0.0
    # SN: plain 1e-4 relative, or the IA's own condition-number bound
    kappa = sn_condition_from(D["scale"], D["top1"], D["sn_den"])
    fin = live & np.isfinite(SNc) & ~near_tie
    rel = np.zeros_like(SNc)
    rel[fin] = np.abs(SN[fin] - SNc[fin]) / np.abs(SNc[fin])
    plain = fin & (rel <= SN_RTOL)
    needs = fin & ~plain
    bound = np.maximum(SN_RTOL, PLANE_RTOL * kappa)
    assert (rel[needs] <= bound[needs]).all(), (name, np.argwhere(needs & (rel > bound))[:5])
    assert np.array_equal(np.isfinite(SN[live]), np.isfinite(SNc[live]))
    stats = {
        "workload": name, "ias": n_ia, "skipped": int((~live).sum()),
        "max_subpixel_err_px": max_subpx,
        "near_ties": int(near_tie.sum()),
        "near_tie_peak_moved": int((near_tie & (err > VF_ATOL)).sum()),
        "sn_max_rel_err_plain": float(rel[plain].max()) if plain.any() else 0.0,
        "sn_needing_condition": int(needs.sum()),
        "sn_cond_max_err_over_bound": float((rel[needs] / bound[needs]).max()) if needs.any() else 0.0,
        "sn_cond_max_kappa_used": float(kappa[needs].max()) if needs.any() else 0.0,
    }
    print("PARITY " + json.dumps(stats), flush=True)
    assert max_subpx <= VF_ATOL
    assert stats["near_ties"] <= max_near_tie_frac * n_ia, stats
    assert stats["sn_needing_condition"] <= max_cond_frac * n_ia, stats
    return VF, stats


def test_fullsize_shift256_fftcc():
    """256x256 Float64 FFTCC, IS 32, SM 16, step 16, threshold 0: all 225 IAs."""
    i1, i2, shift = synth.pair_2d_shift()
    VF, st = _parity("shift256_fftcc", i1, i2, _params("fft", (32, 32), (16, 16), (16, 16), thr=0.0), 0.01, 0.0)
    assert st["near_ties"] == 0


@pytest.mark.parametrize("alg", ["nsqecc", "zncc"])
def test_fullsize_vortex2048(alg):
    """2048x2048 Float32 Lamb-Oseen vortex pair with ramp and gain, IS 32,
    SM 16, step 8: all 64,009 IAs, built exactly as the benchmark builds it."""
    i1, i2, _ = synth.pair_2d_vortex()
    assert i1.shape == (2048, 2048) and i1.dtype == np.float32
    VF, st = _parity(f"vortex2048_{alg}", i1, i2, _params(alg, (32, 32), (16, 16), (8, 8)), 0.001,
                     0.0 if alg == "nsqecc" else 0.01)
    assert st["ias"] == 64009


def test_fullsize_shear512x512x256_fftcc():
    """512x512x256 Float32 FFTCC, IS 32^3, SM 16^3, step 16^3: all 14,415 IAs;
    the interior recovers the imposed shift plus shear."""
    i1, i2, (shift, shear) = synth.pair_3d_shear()
    VF, st = _parity("shear512x512x256_fftcc", i1, i2, _params("fft", (32, 32, 32), (16, 16, 16), (16, 16, 16)),
                     0.001, 0.0)
    assert st["ias"] == 14415
    vf = VF.shape[1:]
    inner = VF[:, 2:-2, 2:-2, 2:-2]
    zc = (np.arange(vf[2]) * 16 + 15.5)[2:-2]
    assert np.abs(np.median(inner[1]) - shift[1]) < 0.05
    assert np.abs(np.median(inner[2]) - shift[2]) < 0.05
    u1 = np.median(inner[0], axis=(0, 1))
    assert np.max(np.abs(u1 - (shift[0] + shear * zc))) < 0.1
