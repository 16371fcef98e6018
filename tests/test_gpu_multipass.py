"""GPU multi-pass refinement (mqp_params.refine) against the oracle's
refined multipass, 2D and 3D, through the C ABI."""
import numpy as np
import pytest

import oracle.piv_oracle as O
from multi_quickpiv_b200 import PIV, setPIVParameters, synth
from tests.helpers import VF_ATOL, sn_ok

pytestmark = pytest.mark.gpu


def _run(i1, i2, alg, IS, SM, st, passes, mask=None):
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, multipass=passes,
                              computeSN=True)
    po.ndims = i1.ndim
    vf = O.get_vf_size_for(i1.shape, po)
    kappa = np.full(vf, np.inf)
    VFo, SNo = O.PIV(i1, i2, po, mask=mask, refine=True, kappa_out=kappa)
    pp = setPIVParameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, multipass=passes, computeSN=True,
                          refine=True)
    VF, SN = PIV(i1, i2, *([mask] if mask is not None else []), pp)
    assert VF.shape == VFo.shape
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0)
    # a coarse-pass near-tie can move one fine predictor; none occur on these inputs
    assert bad.sum() == 0, (np.argwhere(bad)[:5], np.abs(VF - VFo).max())
    assert sn_ok(SN, SNo, kappa).all()
    return VF


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
def test_two_pass_2d_large_shift(alg, gpu):
    i1, i2, _ = synth.pair_2d_shift(shape=(160, 176), shift=(9.4, -6.2), seed_stream=40, dtype=np.float32)
    VF = _run(i1, i2, alg, (16, 16), (4, 4), (16, 16), 2)
    inner = VF[:, 1:-1, 1:-1]
    assert abs(np.median(inner[0]) - 9.4) < 0.1 and abs(np.median(inner[1]) + 6.2) < 0.1


def test_three_pass_2d(gpu):
    i1, i2, _ = synth.pair_2d_vortex(shape=(192, 160), core=40.0, peak=7.0)
    _run(i1, i2, "nsqecc", (8, 8), (4, 4), (8, 8), 3)


def test_two_pass_2d_masked(gpu):
    i1, i2, _ = synth.pair_2d_shift(shape=(128, 128), shift=(6.3, 5.1), seed_stream=41)
    mask = synth.ellipse_mask(np.random.default_rng(8), i1.shape, cover=0.8)
    _run(i1, i2, "nsqecc", (16, 16), (4, 4), (16, 16), 2, mask=mask)


@pytest.mark.parametrize("alg", ["fft", "nsqecc"])
def test_two_pass_3d(alg, gpu):
    i1, i2, _ = synth.pair_3d_shear(shape=(96, 80, 80), seed_stream=42, shift=(5.6, -4.3, 2.2), shear=0.0)
    VF = _run(i1, i2, alg, (16, 16, 16), (8, 8, 8), (16, 16, 16), 2)
    inner = VF[:, 1:-1, 1:-1, 1:-1]
    assert abs(np.median(inner[0]) - 5.6) < 0.1


def _run_deform(i1, i2, alg, IS, SM, st, passes, max_bad_frac=0.0):
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, multipass=passes,
                              computeSN=True)
    po.ndims = i1.ndim
    vf = O.get_vf_size_for(i1.shape, po)
    kappa = np.full(vf, np.inf)
    VFo, SNo = O.PIV(i1, i2, po, refine=2, kappa_out=kappa)
    pp = setPIVParameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, multipass=passes, computeSN=True,
                          refine="deform")
    VF, SN = PIV(i1, i2, pp)
    assert VF.shape == VFo.shape
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0)
    assert bad.mean() <= max_bad_frac, (np.argwhere(bad)[:5], np.abs(VF - VFo).max())
    assert (sn_ok(SN, SNo, kappa) | bad).all()
    return VF


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
def test_deforming_refinement_2d(alg, gpu):
    """refine = 2: each finer pass runs on the pair deformed around the
    interpolated coarser field (mqp_deform.cuh), against the oracle's
    restatement (O.PIV(refine=2))."""
    i1, i2, _ = synth.pair_2d_vortex(shape=(176, 160), core=40.0, peak=6.0)
    _run_deform(i1, i2, alg, (16, 16), (4, 4), (8, 8), 2)


def test_deforming_refinement_three_passes_float64(gpu):
    i1, i2, _ = synth.pair_2d_shift(shape=(160, 144), shift=(5.4, -3.3), seed_stream=43)
    VF = _run_deform(i1, i2, "nsqecc", (8, 8), (4, 4), (8, 8), 3)
    inner = VF[:, 2:-2, 2:-2]
    assert abs(np.median(inner[0]) - 5.4) < 0.1 and abs(np.median(inner[1]) + 3.3) < 0.1


def test_deforming_refinement_3d(gpu):
    i1, i2, _ = synth.pair_3d_shear(shape=(64, 64, 64), seed_stream=44, shift=(3.4, -2.1, 1.2), shear=0.02)
    _run_deform(i1, i2, "fft", (16, 16, 16), (4, 4, 4), (16, 16, 16), 2)


def test_deforming_refinement_rejects_masks(gpu):
    from multi_quickpiv_b200 import _lib
    i1, i2, _ = synth.pair_2d_shift(shape=(96, 96), seed_stream=45)
    mask = np.ones_like(i1)
    pp = setPIVParameters(interSize=(16, 16), searchMargin=(4, 4), step=(16, 16), multipass=2, refine="deform")
    with pytest.raises(_lib.MQPError) as e:
        PIV(i1, i2, mask, pp)
    assert e.value.code == _lib.MQP_ERR_UNSUPPORTED


@pytest.mark.parametrize("alg", ["fft", "zncc"])
def test_three_pass_2d_from_window256(alg, gpu):
    """interSize 32 / margin 16 in three passes: the coarsest (interSize 128,
    margin 64) runs on the search-window-256 kernel."""
    i1, i2, _ = synth.pair_2d_shift(shape=(416, 384), shift=(27.3, -33.6), seed_stream=42, dtype=np.float32)
    VF = _run(i1, i2, alg, (32, 32), (16, 16), (32, 32), 3)
    inner = VF[:, 2:-2, 2:-2]
    assert abs(np.median(inner[0]) - 27.3) < 0.2 and abs(np.median(inner[1]) + 33.6) < 0.2
