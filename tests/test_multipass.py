"""Multi-pass refinement on the CPU: the predictor the GPU builds between
passes (mqp_multipass.cuh, run here through the host emulator) equals the
oracle's, and the oracle's refined multipass recovers displacements larger
than one pass's search margin."""
import ctypes as C

import numpy as np
import pytest

import oracle.piv_oracle as O
from multi_quickpiv_b200 import synth
from tests.native import build_emu


@pytest.fixture(scope="module")
def emu():
    return C.CDLL(build_emu.build())


def emu_predictor(emu, VFc, vf_f, isz_f, st_f, isz_c, st_c):
    nd = VFc.shape[0]
    iv = lambda t: (C.c_int * 3)(*(list(int(x) for x in t) + [1] * (3 - len(t))))
    pred = np.zeros((nd,) + tuple(vf_f), dtype=np.int32, order="F")
    src = np.asfortranarray(VFc, dtype=np.float64)
    rc = emu.mqp_emu_predictor(nd, iv(vf_f), iv(VFc.shape[1:]), iv(isz_f), iv(st_f), iv(isz_c), iv(st_c),
                               src.ctypes.data_as(C.c_void_p), pred.ctypes.data_as(C.c_void_p))
    assert rc == 0
    return pred


@pytest.mark.parametrize("nd", [2, 3])
@pytest.mark.parametrize("geom", [((32, 16), (16, 8)), ((64, 32), (32, 16)), ((48, 24), (24, 12)),
                                  ((32, 32), (16, 16))])
def test_predictor_matches_oracle(emu, nd, geom):
    (isc, stc), (isf, stf) = geom
    size = (200, 176, 96)[:nd]
    p = O.set_piv_parameters(interSize=isf, searchMargin=4, step=stf)
    p.ndims = nd
    vf_c = O.get_vectorfield_size(size, (isc,) * nd, (stc,) * nd)
    vf_f = O.get_vectorfield_size(size, (isf,) * nd, (stf,) * nd)
    g = np.random.default_rng(nd * 100 + isc)
    VFc = g.normal(0, 6, (nd,) + vf_c)
    VFc.ravel()[::7] = np.round(VFc.ravel()[::7]) + 0.5   # exact halves round away from zero
    VFc.ravel()[::11] = np.nan                              # degenerate coarse windows
    # the oracle expresses scales through its accessors; pose the same geometry
    scale_c, scale_f = isc // isf, 1
    pred_o = O.predictor_from_coarse(VFc, scale_c, size, p, scale_f) if isc % isf == 0 and stc == stf * scale_c \
        else None
    pred = emu_predictor(emu, VFc, vf_f, (isf,) * nd, (stf,) * nd, (isc,) * nd, (stc,) * nd)
    if pred_o is not None:
        assert np.array_equal(pred, pred_o)
    # independent restatement: nearest coarse centre per axis, ties up
    for k in np.ndindex(*vf_f):
        jc = []
        for d in range(nd):
            cf = k[d] * stf + (isf - 1) / 2
            cc = np.arange(vf_c[d]) * stc + (isc - 1) / 2
            dist = np.abs(cc - cf)
            jc.append(int(np.flatnonzero(dist == dist.min())[-1]))
        v = VFc[(slice(None),) + tuple(jc)]
        exp = np.where(np.isfinite(v), np.sign(v) * np.floor(np.abs(v) + 0.5), 0)
        assert np.array_equal(pred[(slice(None),) + k], exp.astype(np.int32)), (k, jc)


def test_predictor_empty_coarse_field(emu):
    VFc = np.zeros((2, 0, 5))
    pred = emu_predictor(emu, VFc, (4, 5), (16, 16), (8, 8), (64, 64), (32, 32))
    assert not pred.any()


def test_refined_multipass_recovers_large_shift():
    """A 9.4 px shift is outside a single pass's +-4 px search; two passes
    (scale 2: IS 32, SM 8) find it and the fine pass refines it."""
    i1, i2, _ = synth.pair_2d_shift(shape=(160, 160), shift=(9.4, -6.2), seed_stream=40)
    p = O.set_piv_parameters(corr_alg="nsqecc", interSize=16, searchMargin=4, step=16, multipass=2)
    VF1, _ = O.PIV(i1, i2, p)
    p = O.set_piv_parameters(corr_alg="nsqecc", interSize=16, searchMargin=4, step=16, multipass=2)
    VF2, _ = O.PIV(i1, i2, p, refine=True)
    inner2 = VF2[:, 1:-1, 1:-1]
    assert abs(np.median(inner2[0]) - 9.4) < 0.1 and abs(np.median(inner2[1]) + 6.2) < 0.1
    inner1 = VF1[:, 1:-1, 1:-1]
    assert abs(np.median(inner1[0]) - 9.4) > 1.0
