"""Generates the golden fixtures in this folder from the NumPy oracle
(oracle/piv_oracle.py).  The reference (Julia + FFTW) cannot run here and its
own test suite is empty, so these fixtures pin the oracle's outputs on small
seeded inputs; the CPU tests check that the oracle and its C++ port still
reproduce them and the GPU tests compare the CUDA path against them.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle.piv_oracle as O  # noqa: E402
from multi_quickpiv_b200 import synth  # noqa: E402

CASES = [
    # name, shape, alg, IS, SM, step, threshold, masked
    ("shift2d_fft_32_16_16", (128, 112), "fft", (32, 32), (16, 16), (16, 16), 0.0, False),
    ("shift2d_zncc_32_16_8", (80, 80), "zncc", (32, 32), (16, 16), (8, 8), -1.0, False),
    ("shift2d_nsqecc_32_10_16", (112, 96), "nsqecc", (32, 32), (10, 10), (16, 16), -1.0, False),
    ("shift2d_nsqecc_16_8_8", (64, 80), "nsqecc", (16, 16), (8, 8), (8, 8), -1.0, False),
    ("vortex2d_zncc_aniso", (96, 128), "zncc", (24, 32), (12, 8), (12, 10), -1.0, False),
    ("shift2d_mask_32_16_16", (96, 96), "nsqecc", (32, 32), (16, 16), (16, 16), -1.0, True),
    ("shear3d_fft_16_8_16", (40, 40, 40), "fft", (16, 16, 16), (8, 8, 8), (16, 16, 16), -1.0, False),
    ("shear3d_nsqecc_16_4_12", (44, 40, 36), "nsqecc", (16, 16, 16), (4, 4, 4), (12, 12, 12), -1.0, False),
]


def inputs(name, shape):
    if name.startswith("shift2d"):
        i1, i2, _ = synth.pair_2d_shift(shape=shape, seed_stream=11)
    elif name.startswith("vortex2d"):
        i1, i2, _ = synth.pair_2d_vortex(shape=shape, seed_stream=12, core=20.0, peak=4.0)
    else:
        i1, i2, _ = synth.pair_3d_shear(shape=shape, seed_stream=13)
    return i1, i2


def main():
    for name, shape, alg, IS, SM, st, thr, masked in CASES:
        i1, i2 = inputs(name, shape)
        mask = None
        if masked:
            mask = synth.ellipse_mask(np.random.default_rng(99), shape, cover=0.6)
        p = O.set_piv_parameters(corr_alg=alg, interSize=IS, searchMargin=SM, step=st, computeSN=True,
                                 threshold=thr)
        p.ndims = len(shape)
        VF, SN, corr = O.piv_single_pass(i1, i2, p, mask=mask, keep_corr=True)
        vf = VF.shape[1:]
        P = tuple(2 * m for m in SM)
        planes = np.zeros(tuple(x + 1 for x in P) + (int(np.prod(vf)),))
        for k, cm in corr.items():
            ia = int(np.ravel_multi_index(k, vf, order="F"))
            planes[..., ia] = cm
        out = dict(img1=i1, img2=i2, VF=VF, SN=SN, planes=planes, alg=alg, interSize=IS, searchMargin=SM,
                   step=st, threshold=thr)
        if mask is not None:
            out["mask"] = mask
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, VF.shape, os.path.getsize(os.path.join(HERE, name + ".npz")))


if __name__ == "__main__":
    main()
