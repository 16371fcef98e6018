"""CPU check of the post-processing kernels' logic (csrc/mqp_post.cuh, run
through the host emulator) against the NumPy restatement of
src/postprocessing/postprocessing.jl (oracle/post_oracle.py)."""
import ctypes as C
import math

import numpy as np
import pytest

import oracle.post_oracle as PO
from tests.native import build_emu

OPS = dict(MAG=0, AVG=1, SIM=2, COLL=3, TH=4, STD=5, REPL=6, LOCMAG=7, MDIV=8, DIV=9)


@pytest.fixture(scope="module")
def emu():
    return C.CDLL(build_emu.build())


def run(emu, op, VF, radius=0, mask=None, p=(0.0, 0.0, 0.0), i=(0, 0, 0), scalar_in=False):
    VF = np.asfortranarray(VF, dtype=np.float64)
    grid = VF.shape if scalar_in else VF.shape[1:]
    nc = 1 if scalar_in else VF.shape[0]
    nd = len(grid)
    r = [radius] * nd if np.isscalar(radius) else list(radius)
    out = np.zeros((nc,) + grid if op in (OPS["AVG"], OPS["SIM"], OPS["REPL"], OPS["LOCMAG"]) else grid, order="F")
    outf = np.zeros(grid, dtype=np.float32, order="F")
    mo = np.zeros(grid, dtype=np.uint8, order="F")
    m = None if mask is None else np.asfortranarray(mask, dtype=np.uint8)
    ptr = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)
    rc = emu.mqp_emu_post(op, nc, nd, (C.c_int * 4)(*grid, *[1] * (4 - nd)), (C.c_int * 4)(*r, *[0] * (4 - nd)),
                          ptr(VF), ptr(m), ptr(out), ptr(outf), ptr(mo), C.c_double(p[0]), C.c_double(p[1]),
                          C.c_double(p[2]), i[0], i[1], i[2])
    assert rc == 0
    return out, outf, mo.astype(bool)


def field(shape, seed, zeros=True, nan=False):
    g = np.random.default_rng(seed)
    VF = g.normal(0, 2, shape)
    VF[0] += 1.5  # a mean flow, so directions cluster
    if zeros:
        VF[(slice(None),) + tuple(g.integers(0, s, 3) for s in shape[1:])] = 0.0
    if nan:
        VF[(0,) + tuple(g.integers(0, s, 2) for s in shape[1:])] = np.nan
    return VF


SHAPES = [(2, 13, 11), (3, 7, 6, 5)]


@pytest.mark.parametrize("shape", SHAPES)
def test_magnitudes_average(emu, shape):
    VF = field(shape, 1)
    out, _, _ = run(emu, OPS["MAG"], VF)
    assert np.array_equal(out, PO.magnitudes(VF))
    for r in (1, 2, (2, 1, 3)[:len(shape) - 1]):
        out, _, _ = run(emu, OPS["AVG"], VF, radius=r)
        assert np.allclose(out, PO.average(r, VF), rtol=1e-13, atol=1e-14)


def test_average_space_time(emu):
    VF = field((2, 9, 8, 6), 2, zeros=False)  # 2D + t
    out, _, _ = run(emu, OPS["AVG"], VF, radius=(2, 2, 1))
    assert np.allclose(out, PO.average_NDT(2, 1, VF), rtol=1e-13)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("angle", [40, 20])
def test_collectiveness(emu, shape, angle):
    VF = field(shape, 3)
    _, outf, _ = run(emu, OPS["COLL"], VF, radius=2, p=(math.cos(math.radians(angle)), 0, 0))
    assert np.array_equal(outf, PO.collectiveness(2, VF, max_angle=angle))


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("norm,scale,ex", [(True, True, 2), (False, True, 3), (True, False, 2), (False, False, 1)])
def test_similarity_averaging(emu, shape, norm, scale, ex):
    VF = field(shape, 4)
    out, _, _ = run(emu, OPS["SIM"], VF, radius=1, p=(math.cos(math.radians(20)), ex, 0), i=(int(norm), int(scale), 0))
    ref = PO.similarityAveraging(1, VF, max_angle=20, normalize=norm, scale_by_similarity=scale,
                                 similarity_exponent=ex)
    assert np.allclose(out, ref, rtol=1e-12, atol=1e-14, equal_nan=True)


@pytest.mark.parametrize("shape", SHAPES)
def test_masks_and_filters(emu, shape):
    VF = field(shape, 5)
    VF[(slice(None),) + tuple(s // 2 for s in shape[1:])] = 40.0  # an outlier
    M = PO.magnitudes(VF)
    _, _, m = run(emu, OPS["STD"], M, p=(1.8, 0, 0), scalar_in=True)
    assert np.array_equal(m, PO.STD_masking(1.8, VF))
    _, _, t = run(emu, OPS["TH"], M, p=(3.0, 0, 0), i=(0, 0, 0), scalar_in=True)
    assert np.array_equal(t, PO.TH_masking(3.0, VF))
    _, _, t2 = run(emu, OPS["TH"], M, p=(1.0, 0, 0), i=(1, 0, 0), scalar_in=True)
    assert np.array_equal(t2, PO.TH_masking(1.0, VF, cmp=lambda x, th: x < th))
    for kind, fn in ((0, PO.zeroReplace), (1, PO.medianReplace), (2, PO.meanReplace)):
        out, _, _ = run(emu, OPS["REPL"], VF, radius=2, mask=m, i=(kind, 0, 0))
        assert np.allclose(out, PO.STD_filtering(1.8, VF, replaceFun=fn, radius=2), rtol=1e-13)
    SN = np.abs(field((1,) + shape[1:], 6)[0]) * 3
    _, _, low = run(emu, OPS["TH"], SN, p=(2.0, 0, 0), i=(1, 0, 0), scalar_in=True)
    out, _, _ = run(emu, OPS["REPL"], VF, radius=1, mask=low, i=(0, 0, 0))
    assert np.array_equal(out, PO.remove_low_SN(SN, 2.0, VF))


def test_median_even_and_nan(emu):
    VF = np.arange(2 * 4 * 1, dtype=np.float64).reshape((2, 4, 1))
    VF[1, 2, 0] = np.nan
    mask = np.ones((4, 1), dtype=bool)
    out, _, _ = run(emu, OPS["REPL"], VF, radius=1, mask=mask, i=(1, 0, 0))
    ref = PO._filter(mask, VF, PO.medianReplace, 1)
    assert np.allclose(out, ref, equal_nan=True)


@pytest.mark.parametrize("shape", SHAPES)
def test_local_magnitude_mask(emu, shape):
    VF = field(shape, 7, nan=True)
    out, _, removed = run(emu, OPS["LOCMAG"], VF, radius=2, p=(1.6, 0, 0))
    ref, rem = PO.local_magnitude_mask(1.6, VF, radius=2)
    assert np.array_equal(removed, rem)
    assert np.array_equal(np.signbit(out), np.signbit(ref)) and np.allclose(out, ref, equal_nan=True)


@pytest.mark.parametrize("shape", SHAPES + [(2, 1, 5)])
def test_matlab_divergence(emu, shape):
    VF = field(shape, 8, zeros=False)
    _, outf, _ = run(emu, OPS["MDIV"], VF)
    assert np.array_equal(outf, PO.matlab_divergence(VF), equal_nan=True)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("kw", [dict(normalize=False, divide_by="N"), dict(normalize=True, divide_by="mags"),
                                dict(normalize=True, min_speed=1.0, divide_by="N", circle=True),
                                dict(normalize=False, divide_by="none")])
def test_divergence(emu, shape, kw):
    VF = field(shape, 9)
    radii = (2, 3, 1)[:len(shape) - 1]
    dv = {"N": 1, "mags": 2}.get(kw["divide_by"], 0)
    out, _, _ = run(emu, OPS["DIV"], VF, radius=radii, p=(0, kw.get("min_speed", 0), 0),
                    i=(int(kw["normalize"]), dv, int(kw.get("circle", False))))
    ref = PO.divergence(radii, VF, **kw)
    assert np.allclose(out, ref, rtol=1e-10, atol=1e-12)


def test_divergence_of_a_source_is_negative():
    """A radial source field gives the 'convergence' sign the reference's
    comment warns about (divergence computes convergence)."""
    y, x = np.mgrid[-6:7, -6:7].astype(float)
    VF = np.stack([y, x])
    d = PO.divergence((2, 2), VF, normalize=True)
    assert d[6, 6] < 0
