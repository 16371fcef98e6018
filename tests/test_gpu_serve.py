"""The serving runtime on the GPU: interleaved time-lapse streams (2D
NSQECC, 2D ZNCC, 3D FFTCC) submitted faster than they complete give, for
every request, exactly PIV(frame t, frame t+1) of that pair alone, while
requests are admitted as others run (continuous batching)."""
import numpy as np
import pytest

import multi_quickpiv_b200 as mq
from multi_quickpiv_b200 import synth
from multi_quickpiv_b200.serve import Server

pytestmark = pytest.mark.gpu


def test_interleaved_streams_equal_single_calls(gpu):
    specs = [((256, 256), mq.setPIVParameters(corr_alg="nsqecc", interSize=32, searchMargin=16, step=8,
                                               computeSN=True)),
             ((192, 224), mq.setPIVParameters(corr_alg="zncc", interSize=(24, 32), searchMargin=(12, 16),
                                               step=(12, 16), computeSN=True)),
             ((64, 56, 48), mq.setPIVParameters(corr_alg="fft", interSize=16, searchMargin=8, step=12,
                                                 computeSN=True))]
    srv = Server(slots=3)
    try:
        streams, frames = [], []
        for k, (shape, p) in enumerate(specs):
            tg = synth.TaylorGreenStream(shape, seed_stream=60 + k)
            fr = [tg.next() for _ in range(6)]
            frames.append(fr)
            streams.append(srv.open_stream(fr[0], p))
        reqs = []
        for t in range(1, 6):  # interleaved, submitted without waiting
            for k, sid in enumerate(streams):
                reqs.append((k, t, srv.submit(sid, frames[k][t])))
        for k, t, rid in reqs:
            VF, SN, lat = srv.result(rid)
            VFr, SNr = mq.PIV(frames[k][t - 1], frames[k][t], specs[k][1])
            assert np.array_equal(VF, VFr, equal_nan=True), (k, t)
            assert np.array_equal(SN, SNr, equal_nan=True), (k, t)
            assert lat > 0
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0
        assert st["admitted_while_busy"] > 0
        assert 0 < st["p50_ms"] <= st["p99_ms"]
    finally:
        srv.close()


def test_server_errors(gpu):
    srv = Server(slots=1)
    try:
        import ctypes as C
        with pytest.raises(mq.MQPError, match="unknown stream"):
            srv._check(srv.lib.mqp_server_submit(srv.handle, 99, C.c_void_p(1), C.byref(C.c_uint64())))
        p = mq.setPIVParameters(interSize=16, searchMargin=8, step=16, multipass=2, refine=True)
        with pytest.raises(mq.MQPError, match="single-pass"):
            srv.open_stream(np.zeros((64, 64), np.float32), p)
    finally:
        srv.close()
