"""mqp_piv2d_noalloc: the allocation-free 2D entry point, for callers that
cannot allocate GPU memory while they compute a vector field (code under a
framework that owns all device memory through its own pool, real-time loops
that must not meet cudaMalloc's implicit synchronisation mid-run, hosts that
plan every device byte up front).  It runs the same kernels as the regular
device entry point (mqp_piv_device) on the same inputs, so its vector field
and SN must equal that entry point's bit for bit, call after call, on the
shared scratch array built into the library.  This file is collected last on
purpose."""
import ctypes as C

import numpy as np
import pytest

from multi_quickpiv_b200 import _lib, setPIVParameters, synth
from multi_quickpiv_b200.piv import _colmajor_torch

pytestmark = pytest.mark.gpu


def _dev(a, torch):
    return _colmajor_torch(torch.from_numpy(np.ascontiguousarray(a)).cuda())


def _vf(n, IS, st):
    return (n - IS) // st + 1


CASES = [
    # (alg, shape, IS, SM, step, dtype): the kernel launch_piv2d picks
    ("nsqecc", (320, 288), 32, 16, 8, np.float32),   # FFT length 64
    ("zncc", (320, 288), 32, 16, 8, np.float32),
    ("fft", (320, 288), 32, 16, 8, np.float32),
    ("nsqecc", (200, 176), 8, 4, 4, np.float32),     # search window 16: direct spatial kernel
    ("zncc", (320, 288), 64, 32, 16, np.float32),    # search window 128: block kernel, FFT length 128
    ("nsqecc", (256, 240), 32, 16, 16, np.float64),  # Float64 images
    ("zncc", (1400, 1400), 32, 16, 16, np.float32),  # three integral images, 47.6 of 48 MiB of scratch
]


@pytest.mark.parametrize("alg,shape,IS,SM,step,dtype", CASES,
                         ids=["nsqecc64", "zncc64", "fft64", "direct16", "zncc128", "f64", "zncc1400"])
def test_noalloc_equals_device_entry_twice(alg, shape, IS, SM, step, dtype, gpu):
    import torch
    lib = _lib.load()
    ctx = gpu
    H, W = shape
    i1, i2, _ = synth.pair_2d_vortex(shape=shape, seed_stream=41, core=min(H, W) / 6.0, dtype=dtype)
    d1, d2 = _dev(i1, torch), _dev(i2, torch)
    p = setPIVParameters(corr_alg=alg, interSize=(IS, IS), searchMargin=(SM, SM), step=(step, step),
                         computeSN=True)
    p.ndims = 2
    cp = p.to_c()
    code = _lib.MQP_F32 if dtype == np.float32 else _lib.MQP_F64
    vf = (_vf(H, IS, step), _vf(W, IS, step))
    VFr = torch.zeros((vf[1], vf[0], 2), dtype=torch.float64, device="cuda")
    SNr = torch.zeros((vf[1], vf[0]), dtype=torch.float64, device="cuda")
    rc = lib.mqp_piv_device(ctx.handle, C.c_void_p(d1.data_ptr()), C.c_void_p(d2.data_ptr()), None, None,
                            code, 2, (C.c_int64 * 3)(H, W, 1), C.byref(cp), C.c_void_p(VFr.data_ptr()),
                            C.c_void_p(SNr.data_ptr()), None)
    _lib.check(rc, ctx.handle)
    torch.cuda.synchronize()
    ref_vf, ref_sn = VFr.cpu().numpy(), SNr.cpu().numpy()
    assert np.isfinite(ref_vf).all()
    err = C.create_string_buffer(512)
    for call in range(2):
        VF = torch.full((vf[1], vf[0], 2), float("nan"), dtype=torch.float64, device="cuda")
        SN = torch.full((vf[1], vf[0]), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.mqp_piv2d_noalloc(C.c_void_p(d1.data_ptr()), C.c_void_p(d2.data_ptr()), code,
                                   (C.c_int64 * 2)(H, W), C.byref(cp), C.c_void_p(VF.data_ptr()),
                                   C.c_void_p(SN.data_ptr()), None, err, len(err))
        assert rc == _lib.MQP_OK, err.value.decode()
        torch.cuda.synchronize()
        got_vf, got_sn = VF.cpu().numpy(), SN.cpu().numpy()
        assert np.array_equal(got_vf, ref_vf), f"call {call}: max diff {np.nanmax(np.abs(got_vf - ref_vf))}"
        assert np.array_equal(got_sn, ref_sn), f"call {call}"


def _call(lib, cp, dims, vf_ptr=None):
    import torch
    small = torch.zeros(16, dtype=torch.float32, device="cuda")
    err = C.create_string_buffer(512)
    rc = lib.mqp_piv2d_noalloc(C.c_void_p(small.data_ptr()), C.c_void_p(small.data_ptr()), _lib.MQP_F32,
                               (C.c_int64 * 2)(*dims), C.byref(cp), vf_ptr, None, None, err, len(err))
    return rc, err.value


def test_noalloc_rejects_images_beyond_its_scratch(gpu):
    lib = _lib.load()
    p = setPIVParameters(corr_alg="nsqecc", interSize=(32, 32), searchMargin=(16, 16), step=(8, 8))
    p.ndims = 2
    # 4096 x 4096 NSQECC needs one 134 MB integral image: above the built-in scratch
    import torch
    vf = torch.zeros(16, dtype=torch.float64, device="cuda")  # never written: the call is rejected first
    rc, msg = _call(lib, p.to_c(), (4096, 4096), C.c_void_p(vf.data_ptr()))
    assert rc == _lib.MQP_ERR_INVALID and b"scratch" in msg


def test_noalloc_rejects_refinement_and_accepts_empty_fields(gpu):
    lib = _lib.load()
    p = setPIVParameters(corr_alg="nsqecc", interSize=(16, 16), searchMargin=(8, 8), step=(16, 16),
                         multipass=2, refine=True)
    p.ndims = 2
    rc, msg = _call(lib, p.to_c(), (64, 64))
    assert rc == _lib.MQP_ERR_UNSUPPORTED and b"refine" in msg
    q = setPIVParameters(corr_alg="nsqecc", interSize=(32, 32), searchMargin=(16, 16), step=(8, 8))
    q.ndims = 2
    cq = q.to_c()
    cq.multipass = 0
    rc, msg = _call(lib, cq, (64, 64))
    assert rc == _lib.MQP_ERR_INVALID and b"multipass" in msg
    # an image shorter than the window has an empty vector field: OK without a VF address
    rc, msg = _call(lib, q.to_c(), (16, 64))
    assert rc == _lib.MQP_OK, msg
