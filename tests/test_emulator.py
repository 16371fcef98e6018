"""CPU check of the fused 2D kernel's logic: tests/native/mqp_emu.cu runs the
kernel's own per-lane phase functions (register FFTs, staging, r2c/c2r
splits, window geometry, normalisation, peak, Gaussian fit, SN) on the host."""
import ctypes as C

import numpy as np
import pytest

import oracle.piv_oracle as O
from multi_quickpiv_b200 import synth
from tests.helpers import MASK_PLANE_RTOL, PLANE_RTOL, VF_ATOL, compare_planes, mask_coverage, sn_condition, sn_ok
from tests.native import build_emu

ALG = {"fft": 0, "zncc": 1, "nsqecc": 2}


@pytest.fixture(scope="module")
def emu():
    return C.CDLL(build_emu.build())


@pytest.mark.parametrize("n", [4, 8, 16, 32, 64, 128])
def test_register_fft(emu, n):
    g = np.random.default_rng(n)
    x = (g.normal(size=n) + 1j * g.normal(size=n)).astype(np.complex64)
    for inv in (0, 1):
        io = np.stack([x.real, x.imag], -1).astype(np.float32).ravel().copy()
        assert emu.mqp_emu_fft(n, inv, io.ctypes.data_as(C.c_void_p)) == 0
        y = io[0::2] + 1j * io[1::2]
        ref = np.fft.ifft(x.astype(np.complex128)) * n if inv else np.fft.fft(x.astype(np.complex128))
        assert np.max(np.abs(y - ref)) / np.max(np.abs(ref)) < 3e-7


def run_emu(emu, i1, i2, alg, IS, SM, st, thr=-1.0, mask=None, mask_skip=None, mthr=-1.0):
    vf = O.get_vectorfield_size(i1.shape, IS, st)
    n = vf[0] * vf[1]
    P1, P2 = 2 * SM[0] + 1, 2 * SM[1] + 1
    VF = np.zeros((2,) + vf, order="F")
    SN = np.zeros(vf, order="F")
    PL = np.zeros((P1, P2, n), order="F")
    dt = 1 if i1.dtype == np.float64 else 0
    f1, f2 = np.asfortranarray(i1), np.asfortranarray(i2)
    fm = np.asfortranarray(mask, dtype=i1.dtype) if mask is not None else None
    fs = np.asfortranarray(mask_skip, dtype=i1.dtype) if mask_skip is not None else None
    p = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    code = 3 if mask is not None else ALG[alg]
    rc = emu.mqp_emu_piv2d(p(f1), p(f2), p(fm), p(fs), dt, i1.shape[0], i1.shape[1], IS[0], IS[1], SM[0], SM[1],
                           st[0], st[1], code, C.c_double(thr), C.c_double(mthr), 1, p(VF), p(SN), p(PL),
                           C.c_longlong(0), C.c_longlong(n))
    assert rc == 0
    return VF, SN, PL


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", [((32, 32), (16, 16), (16, 16)), ((16, 16), (8, 8), (8, 8)),
                                 ((32, 32), (10, 10), (16, 16)), ((24, 32), (12, 8), (12, 10)),
                                 ((8, 12), (20, 18), (12, 12)), ((40, 36), (12, 14), (16, 16))])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_emulated_kernel_matches_oracle(emu, alg, cfg, dtype):
    IS, SM, st = cfg
    i1, i2, _ = synth.pair_2d_shift(shape=(112, 100), seed_stream=21)
    i1, i2 = i1.astype(dtype), i2.astype(dtype)
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 2
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    VF, SN, PL = run_emu(emu, i1, i2, alg, IS, SM, st)
    worst, near_tie = compare_planes(PL, Co, i1.shape, IS, SM, st)
    assert worst <= PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any()
    assert (sn_ok(SN, SNo, sn_condition(Co, i1.shape, IS, SM, st)) | near_tie).all()


def test_emulated_threshold_skip(emu):
    i1, i2, _ = synth.pair_2d_shift(shape=(96, 96))
    i1 = i1.copy()
    i1[:40, :40] = -10.0
    VF, SN, _ = run_emu(emu, i1, i2, "fft", (32, 32), (16, 16), (16, 16), thr=0.0)
    assert np.all(VF[:, 0, 0] == 0) and SN[0, 0] == 0


@pytest.mark.parametrize("cfg", [((32, 32), (16, 16), (16, 16)), ((16, 16), (8, 8), (8, 8)),
                                 ((24, 32), (12, 8), (12, 10))])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_emulated_masked_nsqecc(emu, cfg, dtype):
    IS, SM, st = cfg
    i1, i2, _ = synth.pair_2d_shift(shape=(112, 100), seed_stream=22)
    i1, i2 = i1.astype(dtype), i2.astype(dtype)
    mask = synth.ellipse_mask(np.random.default_rng(7), i1.shape, cover=0.7).astype(dtype)
    po = O.set_piv_parameters(interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 2
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, mask=mask, keep_corr=True)
    VF, SN, PL = run_emu(emu, i1, i2, "nsqecc", IS, SM, st, mask=mask)
    # masked sums of a nearly empty mask sit at the FP32 FFT noise floor (it
    # scales with the whole window); planes are compared where the mask covers
    # at least a quarter of the IA, displacements everywhere
    sparse = mask_coverage(mask, i1.shape, IS, st) < 0.25
    worst, near_tie = compare_planes(PL, Co, i1.shape, IS, SM, st, skip=sparse)
    assert worst <= MASK_PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any(), np.abs(VF - VFo).max()


def test_emulated_masked_skip(emu):
    i1, i2, _ = synth.pair_2d_shift(shape=(96, 96))
    mask = np.ones_like(i1)
    skipm = np.ones_like(i1)
    skipm[:40, :40] = 0.0
    po = O.set_piv_parameters(interSize=(32, 32), searchMargin=(16, 16), step=(16, 16), computeSN=True,
                              mask_threshold=0.5)
    po.ndims = 2
    VFo, SNo = O.piv_single_pass(i1, i2, po, mask=mask, mask_skip=skipm)
    VF, SN, _ = run_emu(emu, i1, i2, "nsqecc", (32, 32), (16, 16), (16, 16), mask=mask, mask_skip=skipm, mthr=0.5)
    assert np.all(VF[:, 0, 0] == 0) and np.all(VFo[:, 0, 0] == 0)
    assert np.max(np.abs(VF - VFo)) < 1e-3


BIG = [((64, 64), (32, 32), (32, 32)), ((40, 48), (30, 24), (20, 24)), ((72, 40), (20, 30), (24, 20)),
       ((64, 32), (32, 40), (32, 24)), ((16, 24), (48, 40), (16, 16))]


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", BIG, ids=["is64", "aniso", "unpruned", "wide_sm", "lags97"])
def test_emulated_big_window_matches_oracle(emu, alg, cfg):
    """Search windows 65..128: the 128-thread block kernel's phases."""
    IS, SM, st = cfg
    i1, i2, _ = synth.pair_2d_shift(shape=(232, 216), shift=(9.3, -12.6), seed_stream=23)
    i1, i2 = i1.astype(np.float32), i2.astype(np.float32)
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 2
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    VF, SN, PL = run_emu(emu, i1, i2, alg, IS, SM, st)
    worst, near_tie = compare_planes(PL, Co, i1.shape, IS, SM, st)
    assert worst <= PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any(), np.abs(VF - VFo).max()
    assert (sn_ok(SN, SNo, sn_condition(Co, i1.shape, IS, SM, st)) | near_tie).all()


def test_emulated_big_window_masked(emu):
    IS, SM, st = (64, 64), (32, 32), (32, 32)
    i1, i2, _ = synth.pair_2d_shift(shape=(224, 224), shift=(7.2, 5.4), seed_stream=24)
    mask = synth.ellipse_mask(np.random.default_rng(9), i1.shape, cover=0.7)
    po = O.set_piv_parameters(interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 2
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, mask=mask, keep_corr=True)
    VF, SN, PL = run_emu(emu, i1, i2, "nsqecc", IS, SM, st, mask=mask)
    sparse = mask_coverage(mask, i1.shape, IS, st) < 0.25
    worst, near_tie = compare_planes(PL, Co, i1.shape, IS, SM, st, skip=sparse)
    assert worst <= MASK_PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any(), np.abs(VF - VFo).max()


SMALL = [((8, 8), (4, 4), (8, 8)), ((4, 4), (2, 2), (4, 4)), ((6, 8), (3, 2), (5, 6)), ((12, 8), (2, 3), (6, 8))]


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", SMALL, ids=["is8", "is4", "aniso", "is12x8"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_emulated_direct_small_windows(emu, alg, cfg, dtype):
    """Small windows take the direct (spatial) correlation kernel."""
    IS, SM, st = cfg
    i1, i2, _ = synth.pair_2d_shift(shape=(72, 68), shift=(1.3, -0.6), seed_stream=26)
    i1, i2 = i1.astype(dtype), i2.astype(dtype)
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 2
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    VF, SN, PL = run_emu(emu, i1, i2, alg, IS, SM, st)
    worst, near_tie = compare_planes(PL, Co, i1.shape, IS, SM, st)
    assert worst <= PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any(), np.abs(VF - VFo).max()
    assert (sn_ok(SN, SNo, sn_condition(Co, i1.shape, IS, SM, st)) | near_tie | ~np.isfinite(SNo)).all()


def test_emulated_direct_masked(emu):
    IS, SM, st = (8, 8), (4, 4), (8, 8)
    i1, i2, _ = synth.pair_2d_shift(shape=(72, 72), shift=(1.2, 2.1), seed_stream=27)
    mask = synth.ellipse_mask(np.random.default_rng(4), i1.shape, cover=0.7)
    po = O.set_piv_parameters(interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 2
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, mask=mask, keep_corr=True)
    VF, SN, PL = run_emu(emu, i1, i2, "nsqecc", IS, SM, st, mask=mask)
    sparse = mask_coverage(mask, i1.shape, IS, st) < 0.25
    worst, near_tie = compare_planes(PL, Co, i1.shape, IS, SM, st, skip=sparse)
    assert worst <= MASK_PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie & ~sparse
    assert not bad.any(), np.abs(VF - VFo).max()


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", [((32, 32), (16, 16), (8, 8)), ((16, 16), (8, 8), (8, 8)), ((8, 12), (20, 18), (12, 12))])
def test_emulated_team_and_warp_kernels_agree(emu, alg, cfg, monkeypatch):
    """Pruned FFTCC/ZNCC/NSQECC run on the one-warp-per-IA kernel or (opt-in,
    MQP_TUNE_PIV2D_TEAM=1 on the GPU) on the team kernel (one IA per team of
    N threads).  Both emulations match the oracle and each other within the
    FP32 plane tolerance."""
    IS, SM, st = cfg
    i1, i2, _ = synth.pair_2d_vortex(shape=(120, 112), seed_stream=27, core=30.0)
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 2
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    out = {}
    for mode in ("team", "warp"):
        monkeypatch.setenv("MQP_EMU_PIV2D_TEAM", "1" if mode == "team" else "0")
        VF, SN, PL = run_emu(emu, i1, i2, alg, IS, SM, st)
        worst, near_tie = compare_planes(PL, Co, i1.shape, IS, SM, st)
        assert worst <= PLANE_RTOL, (mode, worst)
        bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
        assert not bad.any(), mode
        assert (sn_ok(SN, SNo, sn_condition(Co, i1.shape, IS, SM, st)) | near_tie).all(), mode
        out[mode] = PL
    fin = np.isfinite(out["warp"])
    assert np.array_equal(fin, np.isfinite(out["team"]))  # 0/0 lags (ZNCC in the padding) alike
    scale = np.max(np.abs(out["warp"][fin]))
    assert np.max(np.abs(out["team"][fin] - out["warp"][fin])) <= 2 * PLANE_RTOL * scale


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", [((64, 64), (64, 64), (64, 64)), ((128, 128), (32, 32), (96, 96)),
                                 ((100, 80), (70, 50), (90, 80)), ((128, 128), (64, 64), (128, 128)),
                                 ((40, 120), (100, 20), (70, 60))])
def test_emulated_window256_kernel_matches_oracle(emu, alg, cfg):
    """Search windows of 129..256: one 256-thread block per IA over a scratch slot."""
    IS, SM, st = cfg
    i1, i2, _ = synth.pair_2d_vortex(shape=(330, 300), seed_stream=23, core=60.0)
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 2
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    VF, SN, PL = run_emu(emu, i1, i2, alg, IS, SM, st)
    worst, near_tie = compare_planes(PL, Co, i1.shape, IS, SM, st)
    assert worst <= PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any()
    assert (sn_ok(SN, SNo, sn_condition(Co, i1.shape, IS, SM, st)) | near_tie).all()


@pytest.mark.parametrize("alg", ["zncc"])
@pytest.mark.parametrize("cfg", [((32, 32), (16, 16), (8, 8)), ((16, 16), (8, 8), (8, 8)), ((32, 32), (9, 13), (12, 16)),
                                 ((16, 16), (5, 3), (6, 10))])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_emulated_onchip_window_sums(emu, alg, cfg, dtype, monkeypatch):
    """ZNCC with an interrogation window of half the FFT length takes its
    window sums from an on-chip table built from the pixels (lw_rows /
    lw_cols) instead of integral images: both routes match the oracle and
    each other to FP64 rounding in the sums."""
    IS, SM, st = cfg
    i1, i2, _ = synth.pair_2d_vortex(shape=(130, 118), seed_stream=29, core=35.0)
    i1, i2 = i1.astype(dtype), i2.astype(dtype)
    po = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True)
    po.ndims = 2
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, keep_corr=True)
    out = {}
    for mode in ("lw", "integral"):
        monkeypatch.setenv("MQP_EMU_PIV2D_NO_LW", "1" if mode == "integral" else "0")
        VF, SN, PL = run_emu(emu, i1, i2, alg, IS, SM, st)
        worst, near_tie = compare_planes(PL, Co, i1.shape, IS, SM, st)
        assert worst <= PLANE_RTOL, (mode, worst)
        bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
        assert not bad.any(), mode
        assert (sn_ok(SN, SNo, sn_condition(Co, i1.shape, IS, SM, st)) | near_tie).all(), mode
        out[mode] = (VF, PL)
    fin = np.isfinite(out["lw"][1])
    assert np.array_equal(fin, np.isfinite(out["integral"][1]))
    scale = np.max(np.abs(out["lw"][1][fin]))
    assert np.max(np.abs(out["lw"][1][fin] - out["integral"][1][fin])) <= 3e-7 * scale  # FP32 quotient: an ulp or two
    assert np.max(np.abs(out["lw"][0] - out["integral"][0])) < 1e-5
