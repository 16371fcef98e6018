"""Serving straight from a TIFF time-lapse stack (multi_quickpiv_b200.ingest:
the native reader and the read-ahead frame source feeding a server stream)
gives the same vectors as PIV on the arrays the stack was written from."""
import numpy as np
import pytest

from multi_quickpiv_b200 import PIV, setPIVParameters, synth
from multi_quickpiv_b200.ingest import FrameSource, serve_tiff
from multi_quickpiv_b200.serve import Server
from tests.tiff_writer import write_tiff

pytestmark = pytest.mark.gpu


def test_serving_a_tiff_stack_equals_piv_on_the_frames(tmp_path, gpu):
    tg = synth.TaylorGreenStream((256, 240), seed_stream=91)
    frames = [np.clip(tg.next(), 0, 65535).astype(np.uint16) for _ in range(5)]
    path = str(tmp_path / "tl.tif")
    write_tiff(path, frames, rows_per_strip=16)
    p = setPIVParameters(interSize=(32, 32), searchMargin=(16, 16), step=(16, 16), computeSN=True)
    with FrameSource(path) as src:
        assert src.pinned and src.frames == 5
    srv = Server(slots=2)
    try:
        rids = list(serve_tiff(srv, path, p))
        assert len(rids) == 4
        for t, rid in enumerate(rids):
            VF, SN, _ = srv.result(rid)
            VFr, SNr = PIV(frames[t].astype(np.float32), frames[t + 1].astype(np.float32), p)
            assert np.array_equal(VF, VFr) and np.array_equal(SN, SNr)
    finally:
        srv.close()
