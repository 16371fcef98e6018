"""The C++/OpenMP restatement (oracle/cpu, the timed CPU baseline) agrees with
the NumPy oracle and with the committed golden fixtures."""
import glob
import os

import numpy as np
import pytest

import oracle.cpu_ref as CR
import oracle.piv_oracle as O
from multi_quickpiv_b200 import setPIVParameters, synth

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.fixture(scope="module", autouse=True)
def built():
    CR.build()


def _params(alg, IS, SM, st, thr=-1.0):
    pp = setPIVParameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True, threshold=thr)
    pp.ndims = len(IS)
    return pp.to_c()


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", [((32, 32), (16, 16), (16, 16)), ((16, 16), (8, 8), (8, 8)),
                                 ((32, 32), (10, 10), (16, 16)), ((24, 32), (12, 8), (12, 10))])
def test_port_matches_numpy_oracle_2d(alg, cfg):
    IS, SM, st = cfg
    i1, i2, _ = synth.pair_2d_shift(shape=(112, 100), seed_stream=31)
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 2
    VF, SN = O.piv_single_pass(i1, i2, po)
    VFc, SNc = CR.piv(i1, i2, _params(alg, IS, SM, st))
    assert np.allclose(VFc, VF, rtol=0, atol=1e-9)
    assert np.allclose(SNc, SN, rtol=1e-9, atol=0)


def test_port_masked_and_3d_match_numpy_oracle():
    i1, i2, _ = synth.pair_2d_shift(shape=(96, 96), seed_stream=32)
    m = synth.ellipse_mask(np.random.default_rng(5), i1.shape, cover=0.6).astype(np.float64)
    po = O.set_piv_parameters(interSize=(32, 32), searchMargin=(16, 16), step=(16, 16), computeSN=True)
    po.ndims = 2
    VF, SN = O.piv_single_pass(i1, i2, po, mask=m)
    VFc, SNc = CR.piv(i1, i2, _params("nsqecc", (32, 32), (16, 16), (16, 16)), mask=m)
    assert np.allclose(VFc, VF, rtol=0, atol=1e-7)
    a, b, _ = synth.pair_3d_shear(shape=(48, 40, 40), seed_stream=33)
    po = O.set_piv_parameters(corr_alg="fft", interSize=(16, 16, 16), searchMargin=(8, 8, 8), step=(16, 16, 16),
                              computeSN=True)
    po.ndims = 3
    VF, SN = O.piv_single_pass(a, b, po)
    VFc, SNc = CR.piv(a, b, _params("fft", (16, 16, 16), (8, 8, 8), (16, 16, 16)))
    assert np.allclose(VFc, VF, rtol=0, atol=1e-9)
    assert np.allclose(SNc, SN, rtol=1e-9, atol=0)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_port_reproduces_golden(path):
    z = np.load(path)
    mask = z["mask"] if "mask" in z.files else None
    cp = _params(str(z["alg"]), tuple(z["interSize"]), tuple(z["searchMargin"]), tuple(z["step"]),
                 float(z["threshold"]))
    VF, SN = CR.piv(z["img1"], z["img2"], cp, mask=mask)
    tol = 1e-7 if mask is not None else 1e-9
    assert np.allclose(VF, z["VF"], rtol=0, atol=tol, equal_nan=True)


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
def test_port_diagnostics_match_numpy_planes(alg):
    """The port's per-IA diagnostics (largest and second-largest similarity on
    the searched lags, largest magnitude, SN denominator) agree with the NumPy
    oracle's similarity blocks; they feed the near-tie and SN-conditioning
    counts of the full-size parity tests."""
    from tests.helpers import searched_region
    IS, SM, st = (32, 32), (16, 16), (16, 16)
    i1, i2, _ = synth.pair_2d_shift(shape=(112, 100), seed_stream=34)
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 2
    _, _, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    _, _, D = CR.piv(i1, i2, _params(alg, IS, SM, st), diag=True)
    for k, cm in Co.items():
        reg = searched_region(i1.shape, IS, SM, st, k)
        v = np.sort(cm[reg].ravel())[::-1]
        assert abs(D["top1"][k] - v[0]) <= 1e-9 * abs(v[0])
        assert abs(D["top2"][k] - v[1]) <= 1e-9 * abs(v[0])
        assert abs(D["scale"][k] - np.max(np.abs(v))) <= 1e-9 * abs(v[0])
        sreg = tuple(slice(r.start, r.stop - 1) for r in reg)
        b = cm[sreg]
        den = (b.sum() - b.max()) / (b.size - 1)
        assert abs(D["sn_den"][k] - den) <= 1e-9 * np.max(np.abs(b))
    assert (D["skipped"] == 0).all()
