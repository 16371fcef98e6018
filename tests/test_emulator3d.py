"""CPU check of the 3D kernels' logic: tests/native/mqp_emu3d.cu runs the
kernels' own per-thread phase functions (r2c along z, the k3-slab 2D
correlation, the c2r along k3, normalisation from integral volumes, peak,
3x3x3 Gaussian fit, SN) on the host, against the Float64 oracle and the
committed 3D golden fixtures."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

import oracle.piv_oracle as O
from multi_quickpiv_b200 import synth
from tests.helpers import MASK_PLANE_RTOL, PLANE_RTOL, VF_ATOL, compare_planes, mask_coverage, sn_condition, sn_ok
from tests.native import build_emu

ALG = {"fft": 0, "zncc": 1, "nsqecc": 2}
GOLDEN3D = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*3d*.npz")))


@pytest.fixture(scope="module")
def emu():
    return C.CDLL(build_emu.build())


def run_emu3(emu, i1, i2, alg, IS, SM, st, thr=-1.0, mask=None, mask_skip=None, mthr=-1.0):
    vf = O.get_vectorfield_size(i1.shape, IS, st)
    n = int(np.prod(vf))
    P = tuple(2 * m + 1 for m in SM)
    VF = np.zeros((3,) + vf, order="F")
    SN = np.zeros(vf, order="F")
    PL = np.zeros(P + (n,), order="F")
    dt = 1 if i1.dtype == np.float64 else 0
    f1, f2 = np.asfortranarray(i1), np.asfortranarray(i2)
    fm = np.asfortranarray(mask, dtype=i1.dtype) if mask is not None else None
    fs = np.asfortranarray(mask_skip, dtype=i1.dtype) if mask_skip is not None else None
    p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    iv = lambda t: (C.c_int * 3)(*[int(x) for x in t])
    code = 3 if mask is not None else ALG[alg]
    rc = emu.mqp_emu_piv3d(p(f1), p(f2), p(fm), p(fs), dt, iv(i1.shape), iv(IS), iv(SM), iv(st), code,
                           C.c_double(thr), C.c_double(mthr), 1, p(VF), p(SN), p(PL), C.c_longlong(0),
                           C.c_longlong(n))
    assert rc == 0
    return VF, SN, PL


def check_against(VF, SN, PL, VFo, SNo, corr, shape, IS, SM, st, rtol=PLANE_RTOL, skip=None):
    worst, near_tie = compare_planes(PL, corr, shape, IS, SM, st, skip=skip)
    assert worst <= rtol, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any(), np.abs(VF - VFo).max()
    assert (sn_ok(SN, SNo, sn_condition(corr, shape, IS, SM, st)) | near_tie).all()


@pytest.mark.parametrize("path", GOLDEN3D, ids=lambda p: os.path.basename(p)[:-4])
def test_emulated_3d_reproduces_golden(emu, path):
    z = np.load(path)
    IS, SM, st = (tuple(int(v) for v in z[k]) for k in ("interSize", "searchMargin", "step"))
    alg = str(z["alg"])
    VF, SN, PL = run_emu3(emu, z["img1"], z["img2"], alg, IS, SM, st, thr=float(z["threshold"]))
    vf = VF.shape[1:]
    corr = {k: z["planes"][..., int(np.ravel_multi_index(k, vf, order="F"))] for k in np.ndindex(*vf)}
    check_against(VF, SN, PL, z["VF"], z["SN"], corr, z["img1"].shape, IS, SM, st)


CASES = [
    # shape, IS, SM, step: N = 32 (pruned F), N = 64 (pruned F), N = 32 (full F), anisotropic
    ((40, 36, 40), (16, 16, 16), (8, 8, 8), (12, 10, 12)),
    ((72, 64, 64), (32, 32, 32), (16, 16, 16), (16, 16, 16)),
    ((36, 36, 30), (24, 20, 18), (4, 6, 4), (6, 8, 6)),
    ((48, 40, 44), (16, 12, 20), (8, 10, 6), (16, 14, 12)),
]


@pytest.mark.parametrize("alg", ["fft", "nsqecc"])
def test_emulated_3d_length128_matches_oracle(emu, alg):
    """Search windows 65..128 (here 96): the 3D kernels at FFT length 128."""
    shape, IS, SM, st = (104, 96, 96), (32, 32, 32), (32, 32, 32), (48, 48, 48)
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=36, shift=(9.4, -7.3, 5.2))
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 3
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    VF, SN, PL = run_emu3(emu, i1, i2, alg, IS, SM, st)
    check_against(VF, SN, PL, VFo, SNo, Co, shape, IS, SM, st)


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", CASES, ids=["n32", "n64", "n32full", "aniso"])
def test_emulated_3d_matches_oracle(emu, alg, cfg):
    shape, IS, SM, st = cfg
    dtype = np.float32 if alg != "zncc" else np.float64
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=31, dtype=dtype)
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 3
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    VF, SN, PL = run_emu3(emu, i1, i2, alg, IS, SM, st)
    check_against(VF, SN, PL, VFo, SNo, Co, shape, IS, SM, st)


def test_emulated_3d_masked(emu):
    shape, IS, SM, st = (48, 44, 40), (16, 16, 16), (8, 8, 8), (8, 8, 8)
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=32, dtype=np.float64)
    mask = synth.ellipse_mask(np.random.default_rng(5), shape, cover=0.7)
    po = O.set_piv_parameters(interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 3
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, mask=mask, keep_corr=True)
    VF, SN, PL = run_emu3(emu, i1, i2, "nsqecc", IS, SM, st, mask=mask)
    sparse = mask_coverage(mask, shape, IS, st) < 0.25
    worst, near_tie = compare_planes(PL, Co, shape, IS, SM, st, skip=sparse)
    assert worst <= MASK_PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any(), np.abs(VF - VFo).max()


def test_emulated_3d_threshold_skip(emu):
    shape, IS, SM, st = (40, 40, 40), (16, 16, 16), (8, 8, 8), (12, 12, 12)
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=33, dtype=np.float64)
    i1 = i1.copy()
    i1[:16, :16, :16] = -50.0
    po = O.set_piv_parameters(corr_alg="fft", interSize=IS, searchMargin=SM, step=st, computeSN=True,
                              threshold=0.0)
    po.ndims = 3
    VFo, SNo = O.piv_single_pass(i1, i2, po)
    VF, SN, _ = run_emu3(emu, i1, i2, "fft", IS, SM, st, thr=0.0)
    assert np.all(VF[:, 0, 0, 0] == 0) and SN[0, 0, 0] == 0 and np.all(VFo[:, 0, 0, 0] == 0)
    assert np.max(np.abs(VF - VFo)) < VF_ATOL


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", [((24, 20, 20), (4, 4, 4), (2, 2, 2), (4, 4, 4)),
                                 ((28, 24, 24), (8, 8, 8), (4, 4, 4), (8, 8, 8)),
                                 ((24, 24, 20), (6, 4, 8), (2, 3, 2), (6, 5, 6)),
                                 ((26, 22, 24), (6, 2, 4), (3, 1, 2), (4, 3, 4))],
                         ids=["is4", "is8", "aniso", "tiled_aniso"])
def test_emulated_3d_direct_small_windows(emu, alg, cfg):
    """Small 3D windows take the direct (spatial) correlation kernel."""
    shape, IS, SM, st = cfg
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=37, shift=(1.3, -0.7, 0.9), shear=0.0)
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 3
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    VF, SN, PL = run_emu3(emu, i1, i2, alg, IS, SM, st)
    worst, near_tie = compare_planes(PL, Co, shape, IS, SM, st)
    assert worst <= PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any(), np.abs(VF - VFo).max()
    assert (sn_ok(SN, SNo, sn_condition(Co, shape, IS, SM, st)) | near_tie | ~np.isfinite(SNo)).all()


def test_emulated_3d_direct_masked(emu):
    shape, IS, SM, st = (24, 24, 24), (8, 8, 8), (4, 4, 4), (4, 4, 4)
    i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=38, shift=(1.2, 0.4, -0.8), shear=0.0,
                                    dtype=np.float64)
    mask = synth.ellipse_mask(np.random.default_rng(6), shape, cover=0.7)
    po = O.set_piv_parameters(interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 3
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, mask=mask, keep_corr=True)
    VF, SN, PL = run_emu3(emu, i1, i2, "nsqecc", IS, SM, st, mask=mask)
    sparse = mask_coverage(mask, shape, IS, st) < 0.25
    worst, near_tie = compare_planes(PL, Co, shape, IS, SM, st, skip=sparse)
    assert worst <= MASK_PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie & ~sparse
    assert not bad.any(), np.abs(VF - VFo).max()
