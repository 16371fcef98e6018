"""GPU parity of the 3D kernels against the Float64 oracle and the committed
3D golden fixtures, through the C ABI (multi_quickpiv_b200.PIV -> mqp_piv),
and the 512x512x256 FFTCC workload against the C++ restatement on sampled
interrogation areas."""
import glob
import os

import numpy as np
import pytest

import oracle.piv_oracle as O
from multi_quickpiv_b200 import PIV, correlation_planes, setPIVParameters, synth
from tests.helpers import MASK_PLANE_RTOL, PLANE_RTOL, VF_ATOL, compare_planes, mask_coverage, sn_condition, sn_ok

pytestmark = pytest.mark.gpu

GOLDEN3D = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*3d*.npz")))


def _params(alg, IS, SM, st, thr=-1.0):
    return setPIVParameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True, threshold=thr)


def _check(VF, SN, planes, VFo, SNo, corr, shape, IS, SM, st, rtol=PLANE_RTOL, skip=None):
    assert VF.shape == VFo.shape
    worst, near_tie = compare_planes(planes, corr, shape, IS, SM, st, skip=skip)
    assert worst <= rtol, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any(), (np.argwhere(bad)[:5], np.abs(VF - VFo).max())
    if SN is not None:
        assert (sn_ok(SN, SNo, sn_condition(corr, shape, IS, SM, st)) | near_tie).all()


@pytest.mark.parametrize("path", GOLDEN3D, ids=lambda p: os.path.basename(p)[:-4])
def test_piv3d_reproduces_golden(path, gpu):
    z = np.load(path)
    IS, SM, st = (tuple(int(v) for v in z[k]) for k in ("interSize", "searchMargin", "step"))
    pp = _params(str(z["alg"]), IS, SM, st, float(z["threshold"]))
    VF, SN = PIV(z["img1"], z["img2"], pp)
    planes = correlation_planes(z["img1"], z["img2"], pp)
    vf = VF.shape[1:]
    corr = {k: z["planes"][..., int(np.ravel_multi_index(k, vf, order="F"))] for k in np.ndindex(*vf)}
    _check(VF, SN, planes, z["VF"], z["SN"], corr, z["img1"].shape, IS, SM, st)


CASES = [
    ((40, 36, 40), (16, 16, 16), (8, 8, 8), (12, 10, 12)),
    ((72, 64, 64), (32, 32, 32), (16, 16, 16), (16, 16, 16)),
    ((36, 36, 30), (24, 20, 18), (4, 6, 4), (6, 8, 6)),
    ((48, 40, 44), (16, 12, 20), (8, 10, 6), (16, 14, 12)),
]


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", CASES, ids=["n32", "n64", "n32full", "aniso"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_piv3d_matches_oracle(alg, cfg, dtype, gpu):
    shape, IS, SM, st = cfg
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=31, dtype=dtype)
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 3
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    pp = _params(alg, IS, SM, st)
    VF, SN = PIV(i1, i2, pp)
    planes = correlation_planes(i1, i2, pp)
    _check(VF, SN, planes, VFo, SNo, Co, shape, IS, SM, st)


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
def test_piv3d_length128_matches_oracle(alg, gpu):
    """Search windows 65..128 (here 96): the 3D kernels at FFT length 128."""
    shape, IS, SM, st = (104, 96, 96), (32, 32, 32), (32, 32, 32), (48, 48, 48)
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=36, shift=(9.4, -7.3, 5.2))
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 3
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    pp = _params(alg, IS, SM, st)
    VF, SN = PIV(i1, i2, pp)
    planes = correlation_planes(i1, i2, pp)
    _check(VF, SN, planes, VFo, SNo, Co, shape, IS, SM, st)


def test_piv3d_masked(gpu):
    shape, IS, SM, st = (48, 44, 40), (16, 16, 16), (8, 8, 8), (8, 8, 8)
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=32, dtype=np.float64)
    mask = synth.ellipse_mask(np.random.default_rng(5), shape, cover=0.7)
    po = O.set_piv_parameters(interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 3
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, mask=mask, keep_corr=True)
    pp = _params("nsqecc", IS, SM, st)
    VF, SN = PIV(i1, i2, mask, pp)
    planes = correlation_planes(i1, i2, pp, mask=mask)
    sparse = mask_coverage(mask, shape, IS, st) < 0.25
    worst, near_tie = compare_planes(planes, Co, shape, IS, SM, st, skip=sparse)
    assert worst <= MASK_PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any(), np.abs(VF - VFo).max()


def test_piv3d_threshold_skip(gpu):
    shape, IS, SM, st = (40, 40, 40), (16, 16, 16), (8, 8, 8), (12, 12, 12)
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=33, dtype=np.float64)
    i1 = i1.copy()
    i1[:16, :16, :16] = -50.0
    VF, SN = PIV(i1, i2, _params("fft", IS, SM, st, thr=0.0))
    assert np.all(VF[:, 0, 0, 0] == 0) and SN[0, 0, 0] == 0
    po = O.set_piv_parameters(corr_alg="fft", interSize=IS, searchMargin=SM, step=st, computeSN=True, threshold=0.0)
    po.ndims = 3
    VFo, _ = O.piv_single_pass(i1, i2, po)
    assert np.max(np.abs(VF - VFo)) < VF_ATOL


def test_piv3d_chunking_is_invisible(gpu):
    """Chunk boundaries of the 3D launch do not change any vector."""
    import multi_quickpiv_b200._lib as L
    shape, IS, SM, st = (72, 64, 64), (32, 32, 32), (16, 16, 16), (16, 16, 16)
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=34)
    pp = _params("nsqecc", IS, SM, st)
    ref, sref = PIV(i1, i2, pp)
    ctx = L.Context(0)
    try:
        ctx.set_chunk3d(5)
        VF, SN = PIV(i1, i2, pp, context=ctx)
    finally:
        ctx.close()
    assert np.array_equal(VF, ref) and np.array_equal(SN, sref)


def test_piv3d_torch_device_path(gpu):
    import torch
    shape, IS, SM, st = (40, 36, 40), (16, 16, 16), (8, 8, 8), (12, 10, 12)
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=35)
    pp = _params("zncc", IS, SM, st)
    VF, SN = PIV(i1, i2, pp)
    VFd, SNd = PIV(torch.from_numpy(i1).cuda(), torch.from_numpy(i2).cuda(), pp)
    assert np.array_equal(VFd.cpu().numpy(), VF) and np.array_equal(SNd.cpu().numpy(), SN)


DIRECT_CASES = [((24, 20, 20), (4, 4, 4), (2, 2, 2), (4, 4, 4)),
                ((28, 24, 24), (8, 8, 8), (4, 4, 4), (8, 8, 8)),
                ((24, 24, 20), (6, 4, 8), (2, 3, 2), (6, 5, 6)),
                ((26, 22, 24), (6, 2, 4), (3, 1, 2), (4, 3, 4))]


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", DIRECT_CASES, ids=["is4", "is8", "aniso", "tiled_aniso"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_piv3d_direct_small_windows(alg, cfg, dtype, gpu):
    """Search windows up to 16 per axis: the direct (spatial) correlation,
    register-tiled for (interSize, lags) along dim 2 in the tiled list (4/5,
    8/9, 2/3) and one lag per lane otherwise (4/7)."""
    shape, IS, SM, st = cfg
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=37, shift=(1.3, -0.7, 0.9), shear=0.0, dtype=dtype)
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 3
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    pp = _params(alg, IS, SM, st)
    VF, SN = PIV(i1, i2, pp)
    planes = correlation_planes(i1, i2, pp)
    _check(VF, SN, planes, VFo, SNo, Co, shape, IS, SM, st)


def test_piv3d_direct_masked(gpu):
    shape, IS, SM, st = (24, 24, 24), (8, 8, 8), (4, 4, 4), (4, 4, 4)
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=38, shift=(1.2, 0.4, -0.8), shear=0.0,
                                    dtype=np.float64)
    mask = synth.ellipse_mask(np.random.default_rng(6), shape, cover=0.7)
    po = O.set_piv_parameters(interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 3
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, mask=mask, keep_corr=True)
    pp = _params("nsqecc", IS, SM, st)
    VF, SN = PIV(i1, i2, mask, pp)
    planes = correlation_planes(i1, i2, pp, mask=mask)
    sparse = mask_coverage(mask, shape, IS, st) < 0.25
    worst, near_tie = compare_planes(planes, Co, shape, IS, SM, st, skip=sparse)
    assert worst <= MASK_PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie & ~sparse
    assert not bad.any(), np.abs(VF - VFo).max()


@pytest.mark.parametrize("cfg", [((48, 40, 100), (16, 16, 16), (8, 8, 8), (8, 8, 12)),
                                 ((40, 36, 96), (32, 32, 32), (16, 16, 16), (16, 16, 16)),
                                 ((100, 104, 128), (32, 32, 32), (32, 32, 32), (48, 48, 32))],
                         ids=["n32", "n64", "n128"])
def test_host_pipeline_3d_matches_device(cfg, gpu):
    """3D FFTCC from host arrays with at least 64 z-planes takes the pipelined
    copy path (z-plane pieces, IA layers as their planes arrive); VF and SN
    equal the device-array path's bit for bit."""
    import torch
    shape, IS, SM, st = cfg
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=41, shift=(1.4, -0.6, 2.2))
    pp = _params("fft", IS, SM, st)
    VF, SN = PIV(i1, i2, pp)
    dev = torch.device("cuda", 0)
    VFd, SNd = PIV(torch.from_numpy(i1).to(dev), torch.from_numpy(i2).to(dev), pp)
    assert np.array_equal(VF, VFd.cpu().numpy(), equal_nan=True)
    assert np.array_equal(SN, SNd.cpu().numpy(), equal_nan=True)


def test_volume_smaller_than_window_gives_empty_field(gpu):
    pp = _params("fft", (16, 16, 16), (8, 8, 8), (8, 8, 8))
    i1 = np.random.default_rng(64).random((40, 10, 40)).astype(np.float32)
    po = O.set_piv_parameters(corr_alg="fft", interSize=(16, 16, 16), searchMargin=(8, 8, 8), step=(8, 8, 8),
                              computeSN=True)
    po.ndims = 3
    VFo, SNo = O.piv_single_pass(i1, i1, po)
    VF, SN = PIV(i1, i1, pp)
    assert VF.shape == VFo.shape and VF.size == 0


@pytest.mark.parametrize("IS,SM", [((8, 8, 8), (4, 4, 4)), ((16, 16, 16), (8, 8, 8))], ids=["direct", "fft"])
def test_constant_volumes_zncc_has_no_peak(IS, SM, gpu):
    i1 = np.full((40, 40, 40), 3.0, dtype=np.float32)
    st = IS
    po = O.set_piv_parameters(corr_alg="zncc", interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 3
    VFo, SNo = O.piv_single_pass(i1, i1, po)
    VF, SN = PIV(i1, i1, _params("zncc", IS, SM, st))
    assert np.array_equal(VF, VFo) and np.all(VF == -(SM[0] + 1))
    assert np.all(np.isnan(SN)) and np.all(np.isnan(SNo))
