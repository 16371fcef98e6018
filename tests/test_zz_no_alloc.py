"""mqp_piv2d_noalloc: the allocation-free 2D entry point for callers that
cannot allocate GPU memory (frameworks owning all device memory through their
own pools, real-time loops that must avoid cudaMalloc mid-run, hosts with a
pre-planned device budget).  It must give what the regular device entry point
(mqp_piv_device) gives, call after call, on the shared scratch array built
into the library.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from multi_quickpiv_b200 import _lib, setPIVParameters, synth
from multi_quickpiv_b200.piv import _colmajor_torch
from tests.helpers import VF_ATOL, sn_ok

pytestmark = pytest.mark.gpu


def _dev(a, torch):
    return _colmajor_torch(torch.from_numpy(np.ascontiguousarray(a)).cuda())


@pytest.mark.parametrize("alg", ["nsqecc", "zncc", "fft"])
def test_noalloc_matches_device_entry_twice(alg, gpu):
    import torch
    lib = _lib.load()
    ctx = gpu
    i1, i2, _ = synth.pair_2d_vortex(shape=(320, 288), seed_stream=41, core=50.0)
    d1, d2 = _dev(i1, torch), _dev(i2, torch)
    p = setPIVParameters(corr_alg=alg, interSize=(32, 32), searchMargin=(16, 16), step=(8, 8), computeSN=True)
    p.ndims = 2
    cp = p.to_c()
    vf = ((320 - 32) // 8 + 1, (288 - 32) // 8 + 1)
    dims3 = (C.c_int64 * 3)(320, 288, 1)
    dims2 = (C.c_int64 * 2)(320, 288)
    VFr = torch.zeros((vf[1], vf[0], 2), dtype=torch.float64, device="cuda")
    SNr = torch.zeros((vf[1], vf[0]), dtype=torch.float64, device="cuda")
    rc = lib.mqp_piv_device(ctx.handle, C.c_void_p(d1.data_ptr()), C.c_void_p(d2.data_ptr()), None, None,
                            _lib.MQP_F32, 2, dims3, C.byref(cp), C.c_void_p(VFr.data_ptr()),
                            C.c_void_p(SNr.data_ptr()), None)
    _lib.check(rc, ctx.handle)
    torch.cuda.synchronize()
    ref_vf, ref_sn = VFr.cpu().numpy(), SNr.cpu().numpy()
    err = C.create_string_buffer(512)
    for call in range(2):
        VF = torch.full((vf[1], vf[0], 2), float("nan"), dtype=torch.float64, device="cuda")
        SN = torch.full((vf[1], vf[0]), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.mqp_piv2d_noalloc(C.c_void_p(d1.data_ptr()), C.c_void_p(d2.data_ptr()), _lib.MQP_F32, dims2,
                                   C.byref(cp), C.c_void_p(VF.data_ptr()), C.c_void_p(SN.data_ptr()), None,
                                   err, len(err))
        assert rc == _lib.MQP_OK, err.value.decode()
        torch.cuda.synchronize()
        got_vf, got_sn = VF.cpu().numpy(), SN.cpu().numpy()
        assert np.all(np.isfinite(got_vf)), f"call {call}: vector field not fully written"
        assert np.max(np.abs(got_vf - ref_vf)) <= VF_ATOL, f"call {call}"
        assert sn_ok(got_sn, ref_sn).all(), f"call {call}"


def test_noalloc_rejects_images_beyond_its_scratch(gpu):
    import torch
    lib = _lib.load()
    p = setPIVParameters(corr_alg="nsqecc", interSize=(32, 32), searchMargin=(16, 16), step=(8, 8))
    p.ndims = 2
    cp = p.to_c()
    small = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(16, dtype=torch.float64, device="cuda")
    err = C.create_string_buffer(512)
    # 4096 x 4096 NSQECC needs one 134 MB integral image: above the built-in scratch
    rc = lib.mqp_piv2d_noalloc(C.c_void_p(small.data_ptr()), C.c_void_p(small.data_ptr()), _lib.MQP_F32,
                               (C.c_int64 * 2)(4096, 4096), C.byref(cp), C.c_void_p(out.data_ptr()), None, None,
                               err, len(err))
    assert rc == _lib.MQP_ERR_INVALID
    assert b"scratch" in err.value
