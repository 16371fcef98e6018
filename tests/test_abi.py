"""The C ABI library (no GPU needed): it loads, exports every symbol that
include/mqp.h declares, and its host-side parameter logic mirrors the
reference."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import multi_quickpiv_b200 as mq
from multi_quickpiv_b200 import _lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "mqp.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"MQP_API\s+[\w\s\*]+?\b(mqp_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = declared_symbols()
    assert len(syms) >= 8
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) <= set(_lib.SIGNATURES), "binding lacks a declared symbol"


@pytest.mark.parametrize("cname,py", [("mqp_params", "MqpParams"), ("mqp_profile", "MqpProfile"),
                                      ("mqp_field", "MqpField"), ("mqp_post_params", "MqpPostParams"),
                                      ("mqp_batch_item", "MqpBatchItem"), ("mqp_batch_options", "MqpBatchOptions"),
                                      ("mqp_server_options", "MqpServerOptions"),
                                      ("mqp_server_stats", "MqpServerStats"),
                                      ("mqp_traj_params", "MqpTrajParams"), ("mqp_tiff_info", "MqpTiffInfo")])
def test_abi_version_and_struct_layout(tmp_path, cname, py):
    """Each ctypes mirror matches the C layout (size and every field offset),
    checked by compiling a probe against include/mqp.h."""
    import subprocess
    lib = _lib.load()
    assert lib.mqp_abi_version() == 1
    st = getattr(_lib, py)
    fields = [f for f, _ in st._fields_]
    src = tmp_path / "probe.c"
    src.write_text(f'#include <stdio.h>\n#include <stddef.h>\n#include "mqp.h"\nint main(void){{printf("%zu", sizeof({cname}));' +
                   "".join(f'printf(" %zu", offsetof({cname}, {f}));' for f in fields) + "return 0;}\n")
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert got[0] == C.sizeof(st)
    assert got[1:] == [getattr(st, f).offset for f in fields]


def test_vf_dims_matches_reference_formula():
    lib = _lib.load()
    for shape, IS, st in [((2048, 2048), 32, 8), ((256, 200), 32, 16), ((31, 64), 32, 8)]:
        p = mq.setPIVParameters(interSize=(IS, IS), searchMargin=(16, 16), step=(st, st))
        p.ndims = 2
        out = (C.c_int64 * 3)()
        assert lib.mqp_vf_dims(C.byref(p.to_c()), 2, (C.c_int64 * 3)(shape[0], shape[1], 1), out) == 0
        assert tuple(out)[:2] == mq.get_vectorfield_size(shape, p)


def test_vf_dims_rejects_bad_parameters():
    lib = _lib.load()
    p = mq.setPIVParameters(interSize=(32, 32), searchMargin=(16, 16), step=(0, 8)).to_c()
    out = (C.c_int64 * 3)()
    assert lib.mqp_vf_dims(C.byref(p), 2, (C.c_int64 * 3)(64, 64, 1), out) == _lib.MQP_ERR_INVALID
    assert b"step" in lib.mqp_last_error(None)
    assert lib.mqp_vf_dims(C.byref(p), 4, (C.c_int64 * 3)(64, 64, 1), out) == _lib.MQP_ERR_INVALID


def test_set_piv_parameters_mirrors_reference():
    p = mq.setPIVParameters()
    assert p.corr_alg == "nsqecc" and p.interSize == (32, 32, 32) and p.searchMargin == (10, 10, 10)
    q = mq.setPIVParameters(unpadded=False)
    assert q.unpadded is True and q.good_pad is False  # src/piv_parameters.jl:57-59
    assert mq.setPIVParameters(corr_alg="fft").corr_alg == "fftcc"
    assert mq.setPIVParameters(corr_alg="anything").corr_alg == "nsqecc"
    with pytest.raises(NameError):
        mq.setPIVParameters(corr_alg="fftc")
    with pytest.raises(NotImplementedError):
        mq.setPIVParameters(filtFun=np.mean).to_c()


def test_piv_rejects_mismatched_sizes_before_any_device_work():
    with pytest.raises(AssertionError, match="same size"):
        mq.PIV(np.zeros((64, 64)), np.zeros((64, 32)))


def test_no_cpu_fallback_when_library_missing(tmp_path, monkeypatch):
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError, match="no CPU fallback"):
        _lib.load(str(tmp_path / "missing.so"))
