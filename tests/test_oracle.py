"""CPU tests of the oracle: brute-force correlation, known-answer shifts, the
reference quirks the hot path depends on, and the committed golden fixtures.
(The reference's own test suite is empty, so these pin the restatement.)"""
import glob
import os

import numpy as np
import pytest

import oracle.piv_oracle as O
from multi_quickpiv_b200 import synth

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


# ---- parameters (src/piv_parameters.jl) -------------------------------------
def test_defaults_and_constructor_swap():
    p = O.set_piv_parameters()
    assert p.corr_alg == "nsqecc" and p.interSize == (32, 32, 32) and p.searchMargin == (10, 10, 10)
    assert p.step is None and p.threshold == -1.0 and not p.computeSN
    # Q2: the positional constructor stores good_pad in unpadded and vice versa
    q = O.set_piv_parameters(unpadded=False, good_pad=True)
    assert q.unpadded is True and q.good_pad is False
    q = O.set_piv_parameters(unpadded=True, good_pad=False)
    assert q.unpadded is False and q.good_pad is True


def test_parse_corr():
    assert O.parse_corr("FFT") == "fftcc"
    assert O.parse_corr("zncc") == "zncc"
    assert O.parse_corr("whatever") == "nsqecc"
    with pytest.raises(ValueError):
        O.parse_corr("znc")


def test_to_dims3_and_accessors():
    p = O.set_piv_parameters(interSize=(32, 24), searchMargin=16, overlap=(8, 4), step=None)
    p.ndims = 2
    assert tuple(O._isize(p)) == (32, 24) and tuple(O._smarg(p)) == (16, 16)
    assert tuple(O._ssize(p)) == (64, 56)
    assert tuple(O._step(p)) == (24, 20)
    assert tuple(O._step(p, 2)) == (48, 40)


@pytest.mark.parametrize("n,expect", [(5, 5), (7, 8), (52, 54), (64, 64), (66, 72), (97, 108), (128, 128),
                                      (130, 135), (33, 36)])
def test_good_size_real(n, expect):
    """good_size_real (src/utils/fft_ops.jl:175-198).  Its power-of-5 loop is
    bounded by root(11, ...), so at most one factor 5 is tried: 97 -> 108
    (2^2 3^3), not 100 (2^2 5^2)."""
    assert O.good_size_real(n) == expect
    m = expect
    for f in (2, 3, 5):
        while m % f == 0:
            m //= f
    assert m == 1 or n <= 6


def test_vectorfield_sizes_of_the_workloads():
    assert O.get_vectorfield_size((256, 256), (32, 32), (16, 16)) == (15, 15)
    assert O.get_vectorfield_size((2048, 2048), (32, 32), (8, 8)) == (253, 253)
    assert O.get_vectorfield_size((512, 512, 256), (32, 32, 32), (16, 16, 16)) == (31, 31, 15)
    assert O.get_vectorfield_size((31, 40), (32, 32), (8, 8)) == (0, 2)


def test_linear2cartesian_column_major():
    assert O.linear2cartesian(1, (3, 4)) == (1, 1)
    assert O.linear2cartesian(4, (3, 4)) == (1, 2)
    assert O.linear2cartesian(3 * 4 + 2, (3, 4, 5)) == (2, 1, 2)


def test_search_offset_is_short_by_two():
    """Q1 (src/utils/piv_ops.jl:72): for an IA at the image edge the offset
    is SM-1-IR_TLF, two less than the true out-of-bounds count."""
    IR_TLF, IR_BRB = np.array([1]), np.array([32])
    SR_TLF, SR_BRB, toff, boff = O.get_search_coordinates(IR_TLF, IR_BRB, (256,), np.array([16]))
    assert SR_TLF[0] == 1 and SR_BRB[0] == 48 and toff[0] == 14 and boff[0] == 0
    IR_TLF, IR_BRB = np.array([225]), np.array([256])
    SR_TLF, SR_BRB, toff, boff = O.get_search_coordinates(IR_TLF, IR_BRB, (256,), np.array([16]))
    assert SR_BRB[0] == 256 and boff[0] == 16


# ---- correlation kernels vs brute force -------------------------------------
@pytest.mark.parametrize("shape,IS,SM", [((48, 48), (16, 16), (16, 16)), ((40, 56), (24, 32), (8, 12)),
                                         ((20, 22, 24), (8, 10, 12), (6, 6, 6))])
def test_fftcc_equals_direct_correlation(shape, IS, SM):
    g = np.random.default_rng(0)
    SS = tuple(i + 2 * m for i, m in zip(IS, SM))
    cs = tuple(O.good_size_real(s) for s in SS)
    F = np.zeros(cs)
    G = np.zeros(cs)
    F[tuple(slice(0, i) for i in IS)] = g.normal(size=IS)
    G[tuple(slice(0, s) for s in SS)] = g.normal(size=SS)
    cc = O.fftcc(F, G)
    ref = O.brute_force_cc(F, G, IS, SM)
    blk = cc[tuple(slice(0, 2 * m + 1) for m in SM)]
    assert np.allclose(blk, ref, rtol=1e-12, atol=1e-10)


def _direct_similarity(alg, F, G, IS, SM):
    """Spatial-domain definitions: ZNCC with the reference's search-region
    mean (Q7), NSQECC = den/(den+num)."""
    P = [2 * m + 1 for m in SM]
    out = np.zeros(P)
    for s in np.ndindex(*P):
        Gw = G[tuple(slice(si, si + i) for si, i in zip(s, IS))]
        if alg == "zncc":
            out[s] = np.sum(F * Gw) / (np.sqrt(np.sum(F * F)) * np.sqrt(np.sum(Gw * Gw)))
        else:
            num = np.sum((F - Gw) ** 2)
            den = np.sqrt(np.sum(F * F)) * np.sqrt(np.sum(Gw * Gw))
            out[s] = den / (den + num)
    return out


@pytest.mark.parametrize("alg", ["zncc", "nsqecc"])
def test_normalised_correlations_equal_spatial_definitions(alg):
    i1, i2, _ = synth.pair_2d_shift(shape=(96, 96), seed_stream=5)
    p = O.set_piv_parameters(corr_alg=alg, interSize=(16, 16), searchMargin=(8, 8), step=(16, 16), computeSN=True)
    p.ndims = 2
    _, _, corr = O.piv_single_pass(i1, i2, p, keep_corr=True)
    vf = O.get_vectorfield_size(i1.shape, (16, 16), (16, 16))
    isz, sm = np.array([16, 16]), np.array([8, 8])
    for k in [(2, 2), (0, 0), (vf[0] - 1, 1)]:
        coords = O.coords_for(int(np.ravel_multi_index(k, vf, order="F")) + 1, vf, i1.shape, isz, sm, np.array([16, 16]))
        cs = O.fft_size(p, isz, isz + 2 * sm)
        if alg == "zncc":
            F = O.copy_inter_region_minus_mean(i1, coords[0], coords[1], cs)
            G = O.copy_search_region_minus_mean(i2, coords[2], coords[3], coords[4], cs)
        else:
            F = O.copy_inter_region(i1, coords[0], coords[1], cs)
            G = O.copy_search_region(i2, coords[2], coords[3], coords[4], cs)
        ref = _direct_similarity(alg, F[:16, :16], G, (16, 16), (8, 8))
        assert np.allclose(corr[k], ref, rtol=1e-9, atol=1e-12)


# ---- peak search, refinement, SN ---------------------------------------------
def test_first_max_in_column_major_order_and_zero_floor():
    """Q3 (src/utils/common_ops.jl:98-124)."""
    c = np.zeros((5, 5))
    c[3, 1] = 2.0
    c[1, 3] = 2.0  # later in column-major order
    peak, mv = O.first_fullovp_peak(c, [2, 2], [0, 0], [0, 0])
    assert peak == (4, 2) and mv == 2.0
    neg = -np.ones((5, 5))
    peak, mv = O.first_fullovp_peak(neg, [2, 2], [0, 0], [0, 0])
    assert peak == (0, 0)
    d = O.gaussian_displacement(neg, np.array([2, 2]), [0, 0], [0, 0])
    assert np.all(d == -3.0)  # -(SM+1)


def test_gaussian_refinement_recovers_a_sampled_gaussian():
    x = np.arange(9)
    for x0, y0 in [(4.2, 3.7), (4.0, 4.0), (3.55, 4.45)]:
        # log(1 + c - min) is exactly quadratic for c = min + exp(q) - 1
        q = -((x[:, None] - x0) ** 2 + (x[None, :] - y0) ** 2) / 3.0
        c = np.exp(q) - 1 + 5.0
        d = O.gaussian_displacement(c, np.array([4, 4]), [0, 0], [0, 0])
        # the fit uses log(1 + c - min(3x3)), close to but not exactly q
        assert abs(d[0] - (x0 - 4)) < 0.15 and abs(d[1] - (y0 - 4)) < 0.15


def test_no_refinement_at_search_edge():
    c = np.zeros((9, 9))
    c[0, 4] = 1.0
    d = O.gaussian_displacement(c, np.array([4, 4]), [0, 0], [0, 0])
    assert d[0] == -4.0 and d[1] == 0.0


def test_sn_region_is_one_short():
    """Q5 (src/utils/piv_ops.jl:336-367): region [1+off, 2SM-off] excludes the
    last lag, so a peak there does not enter SN."""
    c = np.ones((5, 5))
    c[4, 4] = 100.0
    assert O.compute_SN(c, [2, 2], [0, 0], [0, 0]) == 1.0
    c[1, 1] = 10.0
    # region sum 25, max 10: mean of the other 15 values is 1
    assert O.compute_SN(c, [2, 2], [0, 0], [0, 0]) == pytest.approx(10.0)


# ---- known answers ------------------------------------------------------------
@pytest.mark.parametrize("alg", ["fft", "zncc", "nsqecc"])
def test_integer_shift_known_answer(alg):
    g = np.random.default_rng(3)
    base = g.normal(size=(160, 160))
    d = (3, -2)
    i1 = base[16:144, 16:144]
    i2 = base[16 - d[0]:144 - d[0], 16 - d[1]:144 - d[1]]
    p = O.set_piv_parameters(corr_alg=alg, interSize=(32, 32), searchMargin=(8, 8), step=(16, 16))
    VF, _ = O.PIV(i1, i2, p)
    inner = VF[:, 1:-1, 1:-1]
    # the integer peak is exact; the Gaussian fit on a white-noise peak may
    # move it by a fraction of a pixel
    assert np.all(np.round(inner[0]) == d[0]) and np.all(np.round(inner[1]) == d[1])
    assert np.median(np.abs(inner[0] - d[0])) < 0.05 and np.median(np.abs(inner[1] - d[1])) < 0.05


def test_subpixel_shift_known_answer():
    i1, i2, shift = synth.pair_2d_shift(shape=(256, 256), shift=(2.3, -1.7), seed_stream=7)
    p = O.set_piv_parameters(corr_alg="fft", interSize=(32, 32), searchMargin=(16, 16), step=(16, 16))
    VF, _ = O.PIV(i1, i2, p)
    inner = VF[:, 2:-2, 2:-2]
    assert abs(np.median(inner[0]) - 2.3) < 0.1 and abs(np.median(inner[1]) + 1.7) < 0.1


def test_skip_leaves_zero_vectors():
    """Q8 (src/multi_quickPIV.jl:69)."""
    i1, i2, _ = synth.pair_2d_shift(shape=(96, 96))
    i1 = i1.copy()
    i1[:32, :32] = -50.0
    p = O.set_piv_parameters(corr_alg="fft", interSize=(32, 32), searchMargin=(16, 16), step=(32, 32),
                             threshold=0.0, computeSN=True)
    VF, SN = O.PIV(i1, i2, p)
    assert np.all(VF[:, 0, 0] == 0) and SN[0, 0] == 0
    assert np.any(VF[:, 1, 1] != 0)


def test_multipass_without_refine_equals_single_pass():
    """Q6: the reference's pass loop re-runs the scale-1 geometry."""
    i1, i2, _ = synth.pair_2d_shift(shape=(96, 96))
    p1 = O.set_piv_parameters(corr_alg="fft", interSize=(32, 32), searchMargin=(16, 16), step=(16, 16))
    p3 = O.set_piv_parameters(corr_alg="fft", interSize=(32, 32), searchMargin=(16, 16), step=(16, 16), multipass=3)
    assert np.array_equal(O.PIV(i1, i2, p1)[0], O.PIV(i1, i2, p3)[0])


# ---- golden fixtures --------------------------------------------------------
@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_oracle_reproduces_golden(path):
    z = np.load(path)
    alg = str(z["alg"])
    p = O.set_piv_parameters(corr_alg=alg, interSize=tuple(z["interSize"]), searchMargin=tuple(z["searchMargin"]),
                             step=tuple(z["step"]), computeSN=True, threshold=float(z["threshold"]))
    p.ndims = z["img1"].ndim
    mask = z["mask"] if "mask" in z.files else None
    VF, SN = O.piv_single_pass(z["img1"], z["img2"], p, mask=mask)
    assert np.allclose(VF, z["VF"], rtol=0, atol=1e-9, equal_nan=True)
    assert np.allclose(SN, z["SN"], rtol=1e-9, atol=0, equal_nan=True)
