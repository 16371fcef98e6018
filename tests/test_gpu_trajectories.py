"""GPU pseudo-trajectories (PIVtrajectories / PIVtrajectories_grid,
src/postprocessing/postprocessing.jl:988-1120) through the C ABI, bit for bit
against the oracle's per-particle restatement: Float32 positions, the same
rounding and freezing, the same seeded starts."""
import numpy as np
import pytest

import oracle.post_oracle as PO
from multi_quickpiv_b200 import postprocessing as PP

pytestmark = pytest.mark.gpu


def _field(shape, dtype, seed, amp=1.8):
    g = np.random.default_rng(seed)
    return [(g.normal(0, amp, shape)).astype(dtype) for _ in range(len(shape) - 1)]


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nd", [3, 2])
def test_random_starts_match_oracle(dtype, nd, gpu):
    shape = (14, 12, 10, 9) if nd == 3 else (20, 18, 9)
    comps = _field(shape, dtype, 5)
    sub = [(3, 10), (1, 0), (2, 8)][:nd]
    ref = PO.pivtrajectories(comps, 2, 9, numpoints=300, subregion=sub, scale=(1.0, 0.5, 2.0), seed=77)
    W = comps[2] if nd == 3 else None
    got = PP.PIVtrajectories(comps[0], comps[1], W, 2, 9, 300, subregion=sub, scale=(1.0, 0.5, 2.0), seed=77)
    for d in range(nd):
        assert got[d].shape == (7, 300) and got[d].dtype == np.float32
        assert np.array_equal(got[d], ref[d]), d
    # some particles left the field and froze, others kept moving
    moved = np.abs(got[0][-1] - got[0][0]) > 0
    assert moved.any()


@pytest.mark.parametrize("nd", [3, 2])
def test_grid_matches_oracle_host_and_device(nd, gpu):
    import torch
    shape = (16, 15, 11, 6) if nd == 3 else (24, 21, 6)
    comps = _field(shape, np.float32, 6, amp=1.3)
    step = (3, 2, 4)[:nd]
    ref = PO.pivtrajectories(comps, 1, 6, grid=True, step=step)
    W = comps[2] if nd == 3 else None
    host = PP.PIVtrajectories_grid(comps[0], comps[1], W, 1, 6, 0, step=step)
    tc = [torch.from_numpy(c).cuda() for c in comps]
    dev = PP.PIVtrajectories_grid(tc[0], tc[1], tc[2] if nd == 3 else None, 1, 6, 0, step=step)
    for d in range(nd):
        assert np.array_equal(host[d], ref[d])
        assert np.array_equal(dev[d].cpu().numpy(), ref[d])


def test_trajectories_of_a_piv_time_series(gpu):
    """Trajectories over the vector fields PIV returns for a Taylor-Green
    stream (the serving workload's frames, 2D + t)."""
    from multi_quickpiv_b200 import PIV, setPIVParameters, synth
    tg = synth.TaylorGreenStream((256, 256), seed_stream=90)
    frames = [tg.next() for _ in range(5)]
    p = setPIVParameters(interSize=(32, 32), searchMargin=(8, 8), step=(16, 16))
    VFs = [PIV(frames[k], frames[k + 1], p)[0] for k in range(4)]
    U = np.stack([v[0] for v in VFs], -1)
    V = np.stack([v[1] for v in VFs], -1)
    # displacements in pixels, positions in vector-field cells: scale 1/step
    ref = PO.pivtrajectories([U, V], 1, 4, grid=True, scale=(1 / 16, 1 / 16))
    got = PP.PIVtrajectories_grid(U, V, None, 1, 4, 0, scale=(1 / 16, 1 / 16))
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1]) and got[2] is None


def test_invalid_requests_raise(gpu):
    from multi_quickpiv_b200 import _lib
    comps = _field((8, 8, 8, 4), np.float32, 7)
    with pytest.raises(_lib.MQPError):
        PP.PIVtrajectories(comps[0], comps[1], comps[2], 3, 3, 10)      # T1 must exceed T0
    with pytest.raises(_lib.MQPError):
        PP.PIVtrajectories(comps[0], comps[1], comps[2], 1, 6, 10)      # frame 5 does not exist
    with pytest.raises(_lib.MQPError):
        PP.PIVtrajectories(comps[0], comps[1], comps[2], 1, 3, 10, subregion=[(0, 4), None, None])
