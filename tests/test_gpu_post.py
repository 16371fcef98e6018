"""GPU post-processing (multi_quickpiv_b200.postprocessing -> the C ABI ->
csrc/mqp_post.cuh) against the NumPy restatement of
src/postprocessing/postprocessing.jl, on a PIV vector field of the vortex
workload and on random 3D fields, through both the host and the device
(torch) entry points."""
import numpy as np
import pytest

import oracle.post_oracle as PO
from multi_quickpiv_b200 import PIV, postprocessing as PP, setPIVParameters, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vf2d(gpu):
    i1, i2, _ = synth.pair_2d_vortex(shape=(384, 352), core=60.0)
    VF, SN = PIV(i1, i2, setPIVParameters(interSize=(32, 32), searchMargin=(16, 16), step=(16, 16), computeSN=True))
    VF = VF.copy()
    VF[:, 3, 4] = [25.0, -30.0]   # an outlier
    VF[:, 10, 2] = 0.0            # a zero vector
    return VF, SN


def vf3d():
    g = np.random.default_rng(11)
    VF = g.normal(0, 1, (3, 9, 8, 7))
    VF[0] += 1.0
    VF[:, 2, 3, 4] = 0.0
    return VF


def both(fn, VF, *a, **k):
    """fn on the host array and on a torch CUDA copy; returns both as NumPy."""
    import torch
    h = fn(*a, VF, **k) if a else fn(VF, **k)
    t = torch.from_numpy(np.ascontiguousarray(VF)).cuda()
    d = fn(*a, t, **k) if a else fn(t, **k)
    conv = lambda x: x.cpu().numpy() if hasattr(x, "cpu") else x
    if isinstance(h, tuple):
        return tuple(conv(x) for x in h), tuple(conv(x) for x in d)
    return conv(h), conv(d)


def test_two_tuple_radius_on_3d_field_is_in_plane(gpu):
    """localOp takes toDims3(radius)[1:N] (postprocessing.jl:65,85;
    src/piv_parameters.jl:11): a 2-tuple radius on a 3D field is radius 0 along
    axis 3, so the average never mixes z layers."""
    VF = vf3d()
    h, d = both(PP.average, VF, (2, 1))
    assert np.allclose(h, PO.average((2, 1), VF), rtol=1e-13) and np.array_equal(d, h)
    assert np.allclose(h, PO.average((2, 1, 0), VF), rtol=1e-13)
    for z in range(VF.shape[3]):
        assert np.allclose(h[..., z], PO.average((2, 1), VF[..., z]), rtol=1e-13)
    h, d = both(PP.collectiveness, VF, (2, 2))
    assert np.array_equal(h, PO.collectiveness((2, 2, 0), VF)) and np.array_equal(d, h)


@pytest.mark.parametrize("which", ["2d", "3d"])
def test_window_ops(which, vf2d):
    VF = vf2d[0] if which == "2d" else vf3d()
    h, d = both(PP.magnitudes, VF)
    assert np.array_equal(h, PO.magnitudes(VF)) and np.array_equal(d, h)
    h, d = both(PP.average, VF, 2)
    assert np.allclose(h, PO.average(2, VF), rtol=1e-13) and np.array_equal(d, h)
    h, d = both(PP.collectiveness, VF, 2)
    assert np.array_equal(h, PO.collectiveness(2, VF)) and np.array_equal(d, h)
    h, d = both(PP.similarityAveraging, VF, 1)
    assert np.allclose(h, PO.similarityAveraging(1, VF), rtol=1e-12, atol=1e-14) and np.array_equal(d, h)
    h, d = both(PP.matlab_divergence, VF)
    assert np.array_equal(h, PO.matlab_divergence(VF)) and np.array_equal(d, h)


@pytest.mark.parametrize("which", ["2d", "3d"])
def test_filters(which, vf2d):
    VF = vf2d[0] if which == "2d" else vf3d()
    h = PP.STD_masking(1.8, VF)
    assert np.array_equal(h, PO.STD_masking(1.8, VF))
    for rf, rfo in ((PP.medianReplace, PO.medianReplace), (PP.meanReplace, PO.meanReplace),
                    (PP.zeroReplace, PO.zeroReplace)):
        h, d = both(PP.STD_filtering, VF, 1.8, replaceFun=rf)
        assert np.allclose(h, PO.STD_filtering(1.8, VF, replaceFun=rfo), rtol=1e-13) and np.array_equal(d, h)
    h, d = both(PP.TH_filtering, VF, 5.0, replaceFun=PP.medianReplace)
    assert np.allclose(h, PO.TH_filtering(5.0, VF, replaceFun=PO.medianReplace), rtol=1e-13)
    (h, hm), (d, dm) = both(PP.local_magnitude_mask, VF, 1.8)
    r, rm = PO.local_magnitude_mask(1.8, VF)
    assert np.array_equal(hm, rm) and np.array_equal(h, r) and np.array_equal(d, h)


def test_remove_low_sn(vf2d):
    VF, SN = vf2d
    th = float(np.percentile(SN, 20))
    out = PP.remove_low_SN(SN, th, VF)
    assert np.array_equal(out, PO.remove_low_SN(SN, th, VF))


@pytest.mark.parametrize("kw", [dict(), dict(normalize=True, divide_by="mags"),
                                dict(normalize=True, min_speed=0.5, circle=True)])
def test_divergence(kw, vf2d):
    VF = vf2d[0]
    h, d = both(PP.divergence, VF, (2, 2), **kw)
    assert np.allclose(h, PO.divergence((2, 2), VF, **kw), rtol=1e-10, atol=1e-12) and np.array_equal(d, h)
    V3 = vf3d()
    h3 = PP.divergence((1, 2, 1), V3, **kw)
    assert np.allclose(h3, PO.divergence((1, 2, 1), V3, **kw), rtol=1e-10, atol=1e-12)
    outs = PP.multiscale_divergence([(1, 1), (2, 2), (3, 3)], VF)
    refs = PO.multiscale_divergence([(1, 1), (2, 2), (3, 3)], VF)
    for a, b in zip(outs, refs):
        assert np.allclose(a, b, rtol=1e-10, atol=1e-12)


def test_empty_field(gpu):
    """A vector field with no vectors (an image shorter than the window) passes
    through the post-processing ops as an empty result, from host and device
    arrays."""
    import torch
    VF = np.zeros((2, 0, 5))
    assert PP.magnitudes(VF).shape == (0, 5)
    assert PP.average(2, VF).shape == (2, 0, 5)
    assert PP.STD_filtering(1.8, VF, replaceFun=PP.medianReplace).shape == (2, 0, 5)
    out = PP.average(2, torch.zeros((2, 0, 5), dtype=torch.float64, device="cuda"))
    assert tuple(out.shape) == (2, 0, 5)
