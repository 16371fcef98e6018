"""GPU parity of the fused 2D kernel against the Float64 oracle, through the
C ABI (multi_quickpiv_b200.PIV -> mqp_piv)."""
import numpy as np
import pytest

import oracle.piv_oracle as O
from multi_quickpiv_b200 import PIV, correlation_planes, setPIVParameters, synth
from tests.helpers import MASK_PLANE_RTOL, PLANE_RTOL, VF_ATOL, compare_planes, mask_coverage, sn_condition, sn_ok

pytestmark = pytest.mark.gpu

def _oracle_params(alg, IS, SM, st, thr=-1.0, sn=True):
    p = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=sn, threshold=thr)
    p.ndims = len(IS)
    return p


def _compare(img1, img2, alg, IS, SM, st, thr=-1.0):
    po = _oracle_params(alg, IS, SM, st, thr)
    VFo, SNo, Co = O.piv_single_pass(img1, img2, po, keep_corr=True)
    pp = setPIVParameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True, threshold=thr)
    VF, SN = PIV(img1, img2, pp)
    assert VF.shape == VFo.shape and SN.shape == SNo.shape
    planes = correlation_planes(img1, img2, pp)
    worst, near_tie = compare_planes(planes, Co, img1.shape, IS, SM, st)
    assert worst <= PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any(), (np.argwhere(bad)[:5], np.abs(VF - VFo).max())
    assert (sn_ok(SN, SNo, sn_condition(Co, img1.shape, IS, SM, st)) | near_tie).all()
    return VF, VFo


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", [((32, 32), (16, 16), (16, 16)), ((16, 16), (8, 8), (8, 8)),
                                 ((32, 32), (10, 10), (16, 16)), ((24, 32), (12, 8), (12, 10)),
                                 ((8, 12), (20, 18), (12, 12)), ((40, 36), (12, 14), (16, 16))])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_piv2d_matches_oracle(alg, cfg, dtype, gpu):
    i1, i2, _ = synth.pair_2d_shift(shape=(160, 144))
    _compare(i1.astype(dtype), i2.astype(dtype), alg, *cfg)


def test_shift_workload_256_fftcc(gpu):
    """The 256x256 Float64 FFTCC workload with threshold 0 and SN."""
    i1, i2, shift = synth.pair_2d_shift()
    VF, VFo = _compare(i1, i2, "fft", (32, 32), (16, 16), (16, 16), thr=0.0)
    # interior vectors recover the imposed shift
    inner = VF[:, 2:-2, 2:-2]
    assert np.abs(np.median(inner[0]) - shift[0]) < 0.1
    assert np.abs(np.median(inner[1]) - shift[1]) < 0.1


@pytest.mark.parametrize("alg", ["zncc", "nsqecc"])
def test_vortex_crop_float32(alg, gpu):
    i1, i2, _ = synth.pair_2d_vortex(shape=(256, 320), core=60.0)
    _compare(i1, i2, alg, (32, 32), (16, 16), (8, 8))


def test_threshold_skip_leaves_zeros(gpu):
    i1, i2, _ = synth.pair_2d_shift(shape=(128, 128))
    i1 = i1.copy()
    i1[:48, :48] = -100.0  # IAs fully inside stay below the threshold
    VF, VFo = _compare(i1, i2, "fft", (32, 32), (16, 16), (16, 16), thr=0.0)
    assert np.all(VF[:, 0, 0] == 0.0) and np.all(VFo[:, 0, 0] == 0.0)


def test_float32_precision_output(gpu):
    i1, i2, _ = synth.pair_2d_shift(shape=(96, 96))
    pp = setPIVParameters(corr_alg="fft", interSize=(32, 32), searchMargin=(16, 16), step=(16, 16))
    VF, SN = PIV(i1, i2, pp, precision=np.float32)
    assert VF.dtype == np.float32 and SN is None


@pytest.mark.parametrize("cfg", [((32, 32), (16, 16), (16, 16)), ((16, 16), (8, 8), (8, 8)),
                                 ((24, 32), (12, 8), (12, 10))])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_masked_nsqecc_matches_oracle(cfg, dtype, gpu):
    """PIV(img1, img2, mask, pivparams) (src/multi_quickPIV.jl:22-24): masked
    NSQECC with an ellipse mask, against the oracle's restatement of
    _mask_NSQECC! (src/crosscorrelation_algorithms/mask_nsqecc.jl:126-160)."""
    IS, SM, st = cfg
    i1, i2, _ = synth.pair_2d_shift(shape=(128, 112), seed_stream=23)
    i1, i2 = i1.astype(dtype), i2.astype(dtype)
    mask = synth.ellipse_mask(np.random.default_rng(8), i1.shape, cover=0.7).astype(dtype)
    po = _oracle_params("nsqecc", IS, SM, st)
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, mask=mask, keep_corr=True)
    pp = setPIVParameters(interSize=IS, searchMargin=SM, step=st, computeSN=True)
    VF, SN = PIV(i1, i2, mask, pp)
    planes = correlation_planes(i1, i2, pp, mask=mask)
    sparse = mask_coverage(mask, i1.shape, IS, st) < 0.25
    worst, near_tie = compare_planes(planes, Co, i1.shape, IS, SM, st, skip=sparse)
    assert worst <= MASK_PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any(), np.nanmax(np.abs(VF - VFo))


def test_double_masked_skip(gpu):
    """PIV(img1, img2, mask_VF, mask_IA, pivparams) (src/multi_quickPIV.jl:27-29):
    the first mask drives the skip test (mask_threshold > 0), the second the
    correlation."""
    i1, i2, _ = synth.pair_2d_shift(shape=(96, 96), seed_stream=24)
    mask_ia = np.ones_like(i1)
    mask_vf = np.ones_like(i1)
    mask_vf[:40, :40] = 0.0
    pp = setPIVParameters(interSize=(32, 32), searchMargin=(16, 16), step=(16, 16), computeSN=True,
                          mask_threshold=0.5)
    VF, SN = PIV(i1, i2, mask_vf, mask_ia, pp)
    po = O.set_piv_parameters(interSize=(32, 32), searchMargin=(16, 16), step=(16, 16), computeSN=True,
                              mask_threshold=0.5)
    po.ndims = 2
    VFo, SNo = O.piv_single_pass(i1, i2, po, mask=mask_ia, mask_skip=mask_vf)
    assert np.all(VF[:, 0, 0] == 0) and np.all(VFo[:, 0, 0] == 0)
    assert np.nanmax(np.abs(VF - VFo)) < VF_ATOL


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", [((64, 64), (32, 32), (32, 32)), ((40, 48), (30, 24), (20, 24)),
                                 ((72, 40), (20, 30), (24, 20)), ((16, 24), (48, 40), (16, 16))],
                         ids=["is64", "aniso", "unpruned", "lags97"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_piv2d_big_window_matches_oracle(alg, cfg, dtype, gpu):
    """Search windows 65..128 run on the 128-thread block kernel."""
    i1, i2, _ = synth.pair_2d_shift(shape=(264, 248), shift=(9.3, -12.6), seed_stream=25)
    _compare(i1.astype(dtype), i2.astype(dtype), alg, *cfg)


def test_piv2d_big_window_masked(gpu):
    IS, SM, st = (64, 64), (32, 32), (32, 32)
    i1, i2, _ = synth.pair_2d_shift(shape=(224, 224), shift=(7.2, 5.4), seed_stream=24)
    mask = synth.ellipse_mask(np.random.default_rng(9), i1.shape, cover=0.7)
    po = _oracle_params("nsqecc", IS, SM, st)
    VFo, SNo, Co = O.piv_single_pass(i1, i2, po, mask=mask, keep_corr=True)
    pp = setPIVParameters(interSize=IS, searchMargin=SM, step=st, computeSN=True)
    VF, SN = PIV(i1, i2, mask, pp)
    planes = correlation_planes(i1, i2, pp, mask=mask)
    sparse = mask_coverage(mask, i1.shape, IS, st) < 0.25
    worst, near_tie = compare_planes(planes, Co, i1.shape, IS, SM, st, skip=sparse)
    assert worst <= MASK_PLANE_RTOL, worst
    bad = (np.abs(VF - VFo) > VF_ATOL).any(axis=0) & ~near_tie
    assert not bad.any(), np.abs(VF - VFo).max()


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc", "masked"])
@pytest.mark.parametrize("cfg", [((32, 32), (16, 16), (16, 16)), ((64, 48), (32, 24), (24, 32)),
                                 ((8, 8), (4, 4), (8, 8))], ids=["n64", "n128", "direct"])
def test_host_pipeline_matches_device(alg, cfg, gpu):
    """Host arrays at least 1024 columns wide take the pipelined copy path
    (column pieces, per-piece integral columns and IA columns); its VF and SN
    equal the device-array path's bit for bit."""
    import torch
    IS, SM, st = cfg
    g = np.random.default_rng(61)
    shape = (300, 1300)  # 1300 columns: the last piece ends off a 64-column boundary
    i1 = (g.random(shape) * 100).astype(np.float32)
    i2 = np.roll(i1, (2, -3), axis=(0, 1)) + g.normal(0, 2, shape).astype(np.float32)
    masks = []
    if alg == "masked":
        masks = [synth.ellipse_mask(np.random.default_rng(7), shape, cover=0.6).astype(np.float32)]
    pp = setPIVParameters(corr_alg="nsqecc" if alg == "masked" else alg, interSize=IS, searchMargin=SM, step=st,
                          computeSN=True)
    VF, SN = PIV(i1, i2, *masks, pp)
    dev = torch.device("cuda", 0)
    tm = [torch.from_numpy(m).to(dev) for m in masks]
    VFd, SNd = PIV(torch.from_numpy(i1).to(dev), torch.from_numpy(i2).to(dev), *tm, pp)
    assert np.array_equal(VF, VFd.cpu().numpy(), equal_nan=True)
    assert np.array_equal(SN, SNd.cpu().numpy(), equal_nan=True)


def test_host_pieces_are_invisible(gpu):
    """MQP_TUNE_HOST_PIECES changes only how the host-array path overlaps its
    copies: 1 (copy first), 2, 3 and 16 pieces give the same VF and SN; out
    of range values are refused."""
    from multi_quickpiv_b200 import _lib
    g = np.random.default_rng(62)
    shape = (256, 1100)
    i1 = (g.random(shape) * 100).astype(np.float32)
    i2 = np.roll(i1, (1, 2), axis=(0, 1)) + g.normal(0, 2, shape).astype(np.float32)
    pp = setPIVParameters(corr_alg="zncc", interSize=32, searchMargin=16, step=8, computeSN=True)
    ctx = _lib.Context(0)
    ref = None
    for pieces in (1, 2, 3, 16):
        ctx.set_host_pieces(pieces)
        VF, SN = PIV(i1, i2, pp, context=ctx)
        if ref is None:
            ref = (VF, SN)
        assert np.array_equal(VF, ref[0]) and np.array_equal(SN, ref[1], equal_nan=True)
    for bad in (0, 17):
        with pytest.raises(Exception):
            ctx.set_host_pieces(bad)
    ctx.close()


@pytest.mark.parametrize("shape", [(20, 100), (100, 20), (31, 31)])
def test_image_smaller_than_window_gives_empty_field(shape, gpu):
    """An axis shorter than interSize has no interrogation area: the vector
    field is empty along it (get_vectorfield_size), from host and device
    arrays, without error."""
    import torch
    pp = setPIVParameters(corr_alg="nsqecc", interSize=32, searchMargin=8, step=16, computeSN=True)
    po = _oracle_params("nsqecc", (32, 32), (8, 8), (16, 16))
    i1 = np.random.default_rng(63).random(shape).astype(np.float32)
    VFo, SNo = O.piv_single_pass(i1, i1, po)
    VF, SN = PIV(i1, i1, pp)
    assert VF.shape == VFo.shape and SN.shape == SNo.shape and VF.size == 0
    VFd, SNd = PIV(torch.from_numpy(i1).cuda(), torch.from_numpy(i1).cuda(), pp)
    assert tuple(VFd.shape) == VFo.shape and VFd.numel() == 0


def test_constant_images_zncc_has_no_peak(gpu):
    """Constant windows make every ZNCC value 0/0: the reference's peak search
    finds no maximum above 0 (first_fullovp_peak) and reports -(SM+1) with a
    NaN SN; the GPU path gives exactly that, like the oracle."""
    i1 = np.full((96, 80), 5.0, dtype=np.float32)
    IS, SM, st = (16, 16), (4, 4), (16, 16)
    po = _oracle_params("zncc", IS, SM, st)
    VFo, SNo = O.piv_single_pass(i1, i1, po)
    pp = setPIVParameters(corr_alg="zncc", interSize=IS, searchMargin=SM, step=st, computeSN=True)
    VF, SN = PIV(i1, i1, pp)
    assert np.array_equal(VF, VFo) and np.all(VF == -(SM[0] + 1))
    assert np.all(np.isnan(SN)) and np.all(np.isnan(SNo))


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
def test_team_kernel_matches_oracle(alg, gpu):
    """The opt-in team kernel (one IA per 64-thread team) in a child process
    with MQP_TUNE_PIV2D_TEAM=1, against the oracle."""
    import json
    import os
    import subprocess
    import sys
    code = f"""
import sys, json, numpy as np
sys.path.insert(0, {os.path.dirname(os.path.dirname(os.path.abspath(__file__)))!r})
import oracle.piv_oracle as O
from multi_quickpiv_b200 import PIV, setPIVParameters, synth
i1, i2, _ = synth.pair_2d_vortex(shape=(192, 176), core=40.0)
pp = setPIVParameters(corr_alg={alg!r}, interSize=(32, 32), searchMargin=(16, 16), step=(8, 8), computeSN=True)
VF, SN = PIV(i1, i2, pp)
po = O.set_piv_parameters(corr_alg={alg!r}, interSize=(32, 32), searchMargin=(16, 16), step=(8, 8), computeSN=True)
VFo, SNo = O.PIV(i1, i2, po)
print(json.dumps({{"err": float(np.max(np.abs(VF - VFo)))}}))
"""
    env = dict(os.environ, MQP_TUNE_PIV2D_TEAM="1")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert json.loads(r.stdout.strip().splitlines()[-1])["err"] <= VF_ATOL


@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
@pytest.mark.parametrize("cfg", [((64, 64), (64, 64), (64, 64)), ((128, 128), (32, 32), (96, 96)),
                                 ((100, 80), (70, 50), (90, 80)), ((128, 128), (64, 64), (128, 128))],
                         ids=["is64sm64", "is128sm32", "aniso", "ss256"])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_piv2d_window256_matches_oracle(alg, cfg, dtype, gpu):
    """Search windows 129..256 run on the 256-thread block kernel."""
    i1, i2, _ = synth.pair_2d_vortex(shape=(460, 420), seed_stream=26, core=80.0, peak=20.0)
    _compare(i1.astype(dtype), i2.astype(dtype), alg, *cfg)


def test_piv2d_window256_threshold_skip(gpu):
    i1, i2, _ = synth.pair_2d_shift(shape=(384, 384), shift=(30.2, -41.7), seed_stream=27)
    i1 = i1.copy()
    i1[:140, :140] = -5.0
    VF, VFo = _compare(i1, i2, "fft", (128, 128), (64, 64), (128, 128), thr=0.0)
    assert np.all(VF[:, 0, 0] == 0)


def test_piv2d_window_limits(gpu):
    from multi_quickpiv_b200 import MQPError, _lib
    i1, i2, _ = synth.pair_2d_shift(shape=(320, 320))
    mask = np.ones_like(i1)
    with pytest.raises(MQPError) as e:  # a mask at a search window above 128
        PIV(i1, i2, mask, setPIVParameters(interSize=(64, 64), searchMargin=(40, 40), step=(64, 64)))
    assert e.value.code == _lib.MQP_ERR_UNSUPPORTED
    with pytest.raises(MQPError) as e:  # above 256
        PIV(i1, i2, setPIVParameters(interSize=(64, 64), searchMargin=(100, 100), step=(64, 64)))
    assert e.value.code == _lib.MQP_ERR_UNSUPPORTED


@pytest.mark.parametrize("alg", ["fft", "nsqecc", "zncc"])
@pytest.mark.parametrize("shape,IS,SM,st,thr", [((160, 144), 32, 16, 8, -1.0), ((258, 250), 32, 16, 8, -1.0),
                                                ((203, 177), 16, 8, 4, -1.0), ((96, 100), 32, 10, 16, 0.0),
                                                ((300, 260), 24, 12, 6, -1.0), ((68, 64), 32, 16, 4, -1.0)],
                         ids=["base", "h_not_mult4", "odd", "thr", "is24", "small"])
def test_staged_windows_equal_unstaged(alg, shape, IS, SM, st, thr, gpu, monkeypatch):
    """FP32 FFTCC / NSQECC / ZNCC stage each warp's next search window into shared
    memory by TMA (68 x 64 tile, row start rounded down to 4 pixels, zero
    fill outside the image); images whose row pitch is not a multiple of 16
    bytes take the unstaged kernel.  Both give the same vector field bit for
    bit, borders and skipped IAs included."""
    import torch
    i1, i2, _ = synth.pair_2d_shift(shape=shape, shift=(3.7, -2.2), seed_stream=31, dtype=np.float32)
    i1 = i1.copy()
    if thr >= 0:
        i1[:40, :40] = -1.0
    p = setPIVParameters(corr_alg=alg, interSize=(IS, IS), searchMargin=(SM, SM), step=(st, st), computeSN=True,
                         threshold=thr)
    d1, d2 = torch.from_numpy(i1).cuda(), torch.from_numpy(i2).cuda()
    out = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("MQP_TUNE_PIV2D_TMA", mode)
        VF, SN = PIV(d1, d2, p)
        out[mode] = (VF.cpu().numpy(), SN.cpu().numpy())
    assert np.array_equal(out["1"][0], out["0"][0], equal_nan=True)
    assert np.array_equal(out["1"][1], out["0"][1], equal_nan=True)
    assert np.isfinite(out["1"][0]).all()
