"""Batched PIV plans on the GPU: every pair of a mixed batch (2D/3D, sizes,
FFTCC/ZNCC/NSQECC/masked, single- and multi-pass) gives exactly the vectors
and SN of a single-pair PIV call, on every run of the captured graph and
for every tuning option."""
import numpy as np
import pytest

import multi_quickpiv_b200 as mq
from multi_quickpiv_b200 import synth
from multi_quickpiv_b200.batch import BatchPlan

pytestmark = pytest.mark.gpu


def _pairs():
    g = np.random.default_rng(5)
    pairs = []
    for k, (shape, alg, IS, SM, st, mp, masked) in enumerate([
        ((256, 192), "nsqecc", 32, 16, 8, 1, False),
        ((160, 304), "zncc", 32, 16, 16, 1, False),
        ((200, 200), "fft", 16, 8, 8, 1, False),
        ((320, 256), "nsqecc", 8, 4, 8, 3, False),
        ((192, 160), "fft", 16, 4, 16, 2, False),
        ((176, 176), "nsqecc", 16, 8, 16, 1, True),
        ((128, 144), "zncc", 24, 12, 12, 1, False),
        ((64, 48, 56), "fft", 16, 8, 12, 1, False),
        ((72, 64, 64), "nsqecc", 32, 16, 16, 1, False),
        ((80, 72, 72), "fft", 16, 8, 16, 2, False),
        ((352, 320), "nsqecc", 16, 8, 16, 3, False),  # coarse pass IS 64 / SM 32: the 128-point block kernel
        ((288, 288), "zncc", 16, 8, 16, 3, True),
        ((24, 300), "nsqecc", 32, 16, 16, 1, False),  # shorter than the window: an empty vector field
    ]):
        if len(shape) == 2:
            i1, i2, _ = synth.pair_2d_shift(shape=shape, shift=(3.3, -2.6), seed_stream=50 + k, dtype=np.float32)
        else:
            i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=50 + k, shift=(3.1, -1.4, 2.2))
        nd = len(shape)
        p = mq.setPIVParameters(corr_alg=alg, interSize=(IS,) * nd, searchMargin=(SM,) * nd, step=(st,) * nd,
                                computeSN=True, multipass=mp, refine=mp > 1)
        mask = synth.ellipse_mask(g, shape, cover=0.7).astype(np.float32) if masked else None
        pairs.append((i1, i2, p) + ((mask,) if masked else ()))
    return pairs


@pytest.fixture(scope="module")
def reference(gpu):
    pairs = _pairs()
    ref = [mq.PIV(pr[0], pr[1], *pr[3:], pr[2]) for pr in pairs]
    return pairs, ref


@pytest.mark.parametrize("opt", [dict(), dict(use_graph=0, grab=1), dict(grab=4, chunk3d=7)])
def test_batch_equals_single_pair_calls(reference, opt):
    import torch
    pairs, ref = reference
    plan = BatchPlan(pairs, opt)
    for _ in range(2):  # graph replays give the same result
        plan.run()
        torch.cuda.synchronize()
        for (VF, SN), (VFr, SNr) in zip(plan.results(), ref):
            assert np.array_equal(VF.cpu().numpy(), VFr, equal_nan=True)
            assert np.array_equal(SN.cpu().numpy(), SNr, equal_nan=True)  # NaN SN where a mask leaves no data
    info = plan.info()
    assert info["total_ia"] > 0 and info["launches"] > 0
    plan.close()


def test_batch_rejects_unsupported_window(gpu):
    i1, i2, _ = synth.pair_2d_shift(shape=(400, 400))
    p = mq.setPIVParameters(interSize=(96, 96), searchMargin=(48, 48), step=(64, 64))
    with pytest.raises(mq.MQPError, match="batch item 0"):
        BatchPlan([(i1, i2, p)])
