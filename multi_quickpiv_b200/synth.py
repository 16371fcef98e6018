"""Seeded synthetic particle images for the PIV workloads.

The reference ships no dataset (its README uses a local TIFF); these
generators stand in for it with the shapes, sizes and value distributions of
the five benchmark workloads:

* ``pair_2d_shift``   256x256 Float64, Poisson particles (0.02/px, sigma 1.2 px,
  peak U[500,1000]), N(0,10^2) noise per image, uniform (2.3, -1.7) px shift.
* ``pair_2d_vortex``  2048x2048 Float32, the same particles plus a 0-300 ramp
  along dim 2 and a per-image gain U[0.8,1.2]; Lamb-Oseen vortex (core 200 px,
  peak 6 px) centred in the image.
* ``pair_3d_shear``   512x512x256 Float32, 0.005 particles/voxel, sigma 1.0,
  noise 10; uniform (1.5, -0.8, 0.6) shift plus du/dz = 0.01 shear on dim 1.
* ``batch_mixed``     64 uneven pairs (2D 512^2..4096x2048, 3D 128^3..256^3),
  window sizes {16,32,64}, 25 % with ellipse masks.
* ``taylor_green_stream``  time-lapse frames advected by a time-varying
  Taylor-Green field (4 px/frame).

Images are NumPy arrays whose axis 0 is the reference's dimension 1 (rows).
Stream ``k`` of a workload uses ``numpy.random.default_rng(20261203 + k)``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

SEED_BASE = 20261203


def rng(k: int = 0) -> np.random.Generator:
    return np.random.default_rng(SEED_BASE + k)


def render(shape: Sequence[int], centres: np.ndarray, peaks: np.ndarray, sigma: float,
           dtype=np.float64, chunk: int = 16384) -> np.ndarray:
    """Sum of isotropic Gaussian spots ``peak * exp(-|x-c|^2 / (2 sigma^2))``
    sampled at integer pixel positions (0-based), truncated at 4 sigma."""
    shape = tuple(int(s) for s in shape)
    nd = len(shape)
    R = int(math.ceil(4.0 * sigma))
    offs = np.arange(-R, R + 1)
    out = np.zeros(int(np.prod(shape)), dtype=np.float64)
    strides = np.cumprod((1,) + shape[:-1])  # column-major linear index
    for a in range(0, len(centres), chunk):
        c = centres[a:a + chunk]
        pk = peaks[a:a + chunk]
        base = np.floor(c).astype(np.int64)
        w = pk.copy()
        lin = np.zeros((len(c),), dtype=np.int64)
        ok = np.ones((len(c),), dtype=bool)
        # build the separable stamp one axis at a time
        wts = np.ones((len(c),) + (1,) * nd)
        idx = np.zeros((len(c),) + (1,) * nd, dtype=np.int64)
        valid = np.ones((len(c),) + (1,) * nd, dtype=bool)
        for d in range(nd):
            pos = base[:, d:d + 1] + offs[None, :]            # (n, 2R+1)
            g = np.exp(-((pos - c[:, d:d + 1]) ** 2) / (2.0 * sigma * sigma))
            shp = [len(c)] + [1] * nd
            shp[1 + d] = len(offs)
            wts = wts * g.reshape(shp)
            idx = idx + (pos * strides[d]).reshape(shp)
            valid = valid & ((pos >= 0) & (pos < shape[d])).reshape(shp)
        wts = wts * w.reshape((-1,) + (1,) * nd)
        wts = np.broadcast_to(wts, np.broadcast_shapes(wts.shape, idx.shape, valid.shape))
        idx = np.broadcast_to(idx, wts.shape)
        valid = np.broadcast_to(valid, wts.shape)
        out += np.bincount(idx[valid], weights=wts[valid], minlength=out.size)
        del lin, ok
    return out.reshape(shape, order="F").astype(dtype)


def _particles(g: np.random.Generator, shape, density, margin):
    lo = -np.asarray(margin, dtype=np.float64)
    hi = np.asarray(shape, dtype=np.float64) + margin
    vol = float(np.prod(hi - lo))
    n = g.poisson(density * vol)
    pos = lo + g.random((n, len(shape))) * (hi - lo)
    peaks = g.uniform(500.0, 1000.0, n)
    return pos, peaks


def pair_2d_shift(shape=(256, 256), shift=(2.3, -1.7), seed_stream=0, dtype=np.float64):
    """Uniformly shifted 2D particle pair (the 256x256 FFTCC workload)."""
    g = rng(seed_stream)
    pos, pk = _particles(g, shape, 0.02, 8.0)
    i1 = render(shape, pos, pk, 1.2) + g.normal(0.0, 10.0, shape)
    i2 = render(shape, pos + np.asarray(shift)[None, :], pk, 1.2) + g.normal(0.0, 10.0, shape)
    return i1.astype(dtype), i2.astype(dtype), np.asarray(shift, dtype=np.float64)


def lamb_oseen(pos, centre, core=200.0, peak=6.0):
    """Lamb-Oseen displacement (dim1, dim2) at ``pos``, scaled to max |u| = peak."""
    r_vec = pos - centre[None, :]
    r = np.sqrt(np.sum(r_vec ** 2, axis=1))
    prof = lambda rr: (1.0 - np.exp(-(rr ** 2) / core ** 2)) / np.maximum(rr, 1e-9)
    rs = np.linspace(1.0, 5 * core, 20001)
    scale = peak / np.max(prof(rs))
    ut = scale * prof(r)
    u1 = ut * (r_vec[:, 1] / np.maximum(r, 1e-9))
    u2 = -ut * (r_vec[:, 0] / np.maximum(r, 1e-9))
    return np.stack([u1, u2], axis=1)


def pair_2d_vortex(shape=(2048, 2048), seed_stream=1, dtype=np.float32, core=200.0, peak=6.0):
    """2D pair with ramp, per-image gain and a Lamb-Oseen vortex (the 2048^2
    ZNCC/NSQECC workload).  Returns (img1, img2, flow) where flow(pos) gives
    the true displacement."""
    g = rng(seed_stream)
    pos, pk = _particles(g, shape, 0.02, 8.0)
    centre = (np.asarray(shape, dtype=np.float64) - 1.0) / 2.0
    disp = lamb_oseen(pos, centre, core, peak)
    ramp = np.broadcast_to(np.linspace(0.0, 300.0, shape[1])[None, :], shape)
    g1, g2 = g.uniform(0.8, 1.2, 2)
    i1 = g1 * (render(shape, pos, pk, 1.2) + ramp) + g.normal(0.0, 10.0, shape)
    i2 = g2 * (render(shape, pos + disp, pk, 1.2) + ramp) + g.normal(0.0, 10.0, shape)
    flow = lambda p: lamb_oseen(np.atleast_2d(p), centre, core, peak)
    return i1.astype(dtype), i2.astype(dtype), flow


def pair_3d_shear(shape=(512, 512, 256), seed_stream=2, dtype=np.float32,
                  shift=(1.5, -0.8, 0.6), shear=0.01):
    """3D pair with uniform shift plus du1/dz shear (the 512x512x256 workload)."""
    g = rng(seed_stream)
    pos, pk = _particles(g, shape, 0.005, 6.0)
    disp = np.tile(np.asarray(shift, dtype=np.float64), (len(pos), 1))
    disp[:, 0] += shear * pos[:, 2]
    i1 = render(shape, pos, pk, 1.0, dtype=np.float32) + g.normal(0.0, 10.0, shape).astype(np.float32)
    i2 = render(shape, pos + disp, pk, 1.0, dtype=np.float32) + g.normal(0.0, 10.0, shape).astype(np.float32)
    return i1.astype(dtype), i2.astype(dtype), (np.asarray(shift), shear)


def ellipse_mask(g: np.random.Generator, shape, cover=0.3) -> np.ndarray:
    """Binary mask made of 5-20 random ellipses (ellipsoids in 3D) covering
    about ``cover`` of the area."""
    shape = tuple(shape)
    nd = len(shape)
    k = int(g.integers(5, 21))
    grids = np.meshgrid(*[np.arange(s, dtype=np.float32) for s in shape], indexing="ij")
    vol = float(np.prod(shape))
    per = cover * vol / k
    m = np.zeros(shape, dtype=bool)
    for _ in range(k):
        c = g.random(nd) * np.asarray(shape)
        ratios = g.uniform(0.5, 2.0, nd)
        unit = (math.gamma(nd / 2 + 1) / math.pi ** (nd / 2) * per / np.prod(ratios)) ** (1.0 / nd)
        ax = ratios * unit
        acc = np.zeros(shape, dtype=np.float32)
        for d in range(nd):
            acc += ((grids[d] - c[d]) / ax[d]) ** 2
        m |= acc <= 1.0
    return m.astype(np.float32)


@dataclass
class BatchItem:
    img1: np.ndarray
    img2: np.ndarray
    mask: Optional[np.ndarray]
    interSize: int
    searchMargin: int
    corr_alg: str


def batch_mixed(n_pairs=64, seed_stream=3, frac_3d=0.25, frac_masked=0.25,
                size_scale=1.0) -> List[BatchItem]:
    """The uneven batched workload: 64 pairs of mixed size and dimensionality.
    ``size_scale`` < 1 shrinks every image (for CPU tests)."""
    g = rng(seed_stream)
    items = []
    for i in range(n_pairs):
        is3d = g.random() < frac_3d
        IS = int(g.choice([16, 32, 64]))
        if is3d:
            side = int(round(math.exp(g.uniform(math.log(128), math.log(256))) * size_scale))
            shape = (max(side, 3 * IS),) * 3
            dens, sig = 0.005, 1.0
        else:
            h = int(round(math.exp(g.uniform(math.log(512), math.log(4096))) * size_scale))
            w = int(round(math.exp(g.uniform(math.log(512), math.log(2048))) * size_scale))
            shape = (max(h, 3 * IS), max(w, 3 * IS))
            dens, sig = 0.02, 1.2
        pos, pk = _particles(g, shape, dens, 6.0)
        shift = g.uniform(-IS / 4, IS / 4, len(shape))
        i1 = render(shape, pos, pk, sig, dtype=np.float32) + g.normal(0, 10, shape).astype(np.float32)
        i2 = render(shape, pos + shift[None, :], pk, sig, dtype=np.float32) + g.normal(0, 10, shape).astype(np.float32)
        masked = g.random() < frac_masked
        mask = ellipse_mask(g, shape) if masked else None
        alg = "nsqecc" if masked else str(g.choice(["fft", "zncc", "nsqecc"]))
        items.append(BatchItem(i1, i2, mask, IS, IS // 2, alg))
    return items


def taylor_green_displacement(pos, shape, t, amp=4.0, period=None):
    """Time-varying Taylor-Green displacement per frame at ``pos`` (2D or 3D)."""
    shape = np.asarray(shape, dtype=np.float64)
    k = 2 * math.pi / shape
    ph = 0.3 * t
    if len(shape) == 2:
        u1 = amp * np.sin(k[0] * pos[:, 0] + ph) * np.cos(k[1] * pos[:, 1])
        u2 = -amp * np.cos(k[0] * pos[:, 0] + ph) * np.sin(k[1] * pos[:, 1])
        return np.stack([u1, u2], axis=1)
    u1 = amp * np.sin(k[0] * pos[:, 0] + ph) * np.cos(k[1] * pos[:, 1]) * np.cos(k[2] * pos[:, 2])
    u2 = -amp * np.cos(k[0] * pos[:, 0] + ph) * np.sin(k[1] * pos[:, 1]) * np.cos(k[2] * pos[:, 2])
    u3 = np.zeros_like(u1)
    return np.stack([u1, u2, u3], axis=1)


class TaylorGreenStream:
    """A time-lapse stream: a persistent particle field advected frame to
    frame by the Taylor-Green field; ``next()`` renders the next frame."""

    def __init__(self, shape, seed_stream=4, density=None, sigma=None, amp=4.0):
        self.shape = tuple(shape)
        self.g = rng(seed_stream)
        nd = len(shape)
        density = density if density is not None else (0.02 if nd == 2 else 0.005)
        self.sigma = sigma if sigma is not None else (1.2 if nd == 2 else 1.0)
        self.pos, self.pk = _particles(self.g, shape, density, 0.0)
        self.t = 0
        self.amp = amp

    def next(self) -> np.ndarray:
        img = render(self.shape, self.pos, self.pk, self.sigma, dtype=np.float32)
        img += self.g.normal(0, 10, self.shape).astype(np.float32)
        d = taylor_green_displacement(self.pos, self.shape, self.t, self.amp)
        self.pos = np.mod(self.pos + d, np.asarray(self.shape, dtype=np.float64))
        self.t += 1
        return img
