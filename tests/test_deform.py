"""The deforming multi-pass refinement (mqp_params.refine = 2) on the CPU:
the kernels' resampling functions (host emulation of mqp_deform.cuh) equal
the oracle's restatement bit for bit, and on a linear shear the deforming
refinement is more accurate than whole-pixel shifting."""
import ctypes as C

import numpy as np
import pytest

import oracle.piv_oracle as O
from multi_quickpiv_b200 import synth
from tests.native import build_emu


@pytest.fixture(scope="module")
def emu():
    return C.CDLL(build_emu.build())


@pytest.mark.parametrize("nd,dtype", [(2, np.float32), (2, np.float64), (3, np.float32)])
def test_emulated_resampling_equals_oracle(emu, nd, dtype):
    g = np.random.default_rng(4 + nd)
    shape = (37, 30) if nd == 2 else (26, 24, 17)
    i1 = g.normal(100, 30, shape).astype(dtype)
    i2 = g.normal(100, 30, shape).astype(dtype)
    isz, st = (16,) * nd, (8,) * nd
    vf = tuple((n - 16) // 8 + 1 for n in shape)
    VFc = g.normal(0, 2.5, (nd,) + vf)
    VFc[(0,) + tuple(min(1, v - 1) for v in vf)] = np.nan  # non-finite coarse vectors count as 0
    o1, o2 = O.deform_images(i1, i2, VFc, isz, st)
    f1, f2 = np.asfortranarray(i1), np.asfortranarray(i2)
    e1 = np.zeros(shape, dtype=dtype, order="F")
    e2 = np.zeros(shape, dtype=dtype, order="F")
    V = np.asfortranarray(VFc)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    iv = lambda t: (C.c_int * 3)(*(list(t) + [1] * (3 - len(t))))
    rc = emu.mqp_emu_deform(p(f1), p(f2), 0 if dtype == np.float32 else 1, nd, (C.c_longlong * 3)(*(list(shape) + [1] * (3 - nd))),
                            p(V), iv(vf), iv(isz), iv(st), p(e1), p(e2))
    assert rc == 0
    assert np.array_equal(e1, o1) and np.array_equal(e2, o2)


def test_deformation_beats_shifting_on_a_shear():
    g = synth.rng(9)
    shape = (160, 160)
    pos, pk = synth._particles(g, shape, 0.02, 8.0)
    a = 0.08  # du1/dx2: 1.3 px across a 16 px window
    u = np.stack([a * (pos[:, 1] - 80.0), np.zeros(len(pos))], 1)
    i1 = synth.render(shape, pos, pk, 1.2) + g.normal(0, 10, shape)
    i2 = synth.render(shape, pos + u, pk, 1.2) + g.normal(0, 10, shape)
    err = {}
    for r in (1, 2):
        po = O.set_piv_parameters(corr_alg="nsqecc", interSize=(16, 16), searchMargin=(4, 4), step=(8, 8), multipass=2)
        VF, _ = O.PIV(i1, i2, po, refine=r)
        cx = np.arange(VF.shape[2]) * 8 + 7.5
        err[r] = np.median(np.abs(VF[0] - a * (cx - 80.0))[2:-2, 2:-2])
    assert err[2] < 0.75 * err[1], err
