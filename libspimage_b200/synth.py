"""Seeded synthetic diffraction patterns for the phasing workloads.

No public dataset is named for this path, so every workload is generated here
with the shapes, photon counts and beamstops of the benchmark configurations:

1. object: zeros with a centred ``blob``-sized cube of uniform[0,1) values
   (PCG64, ``seed``), smoothed by a Gaussian of sigma 2 px (constant padding);
2. intensities ``|FFT(object)|^2`` scaled to ``photons`` in total;
3. amplitudes ``sqrt(Poisson(I))`` (PCG64, ``seed + 1``);
4. a centred beamstop of radius ``beamstop`` px where the mask and the
   amplitudes are 0 (a disc in 2-D, a sphere in 3-D);
5. amplitudes and mask moved to the FFT-shifted layout the phaser expects
   (zero frequency at index 0, as in the reference's ``shifted`` images);
6. an initial support: a centred disc/sphere of radius ``0.75 * blob``,
   shifted the same way so the object forms around the origin.
"""
from __future__ import annotations

import numpy as np

WORKLOADS = {
    # name: (shape, blob, photons, beamstop radius)
    "hio256": ((256, 256), 64, 1e6, 4),
    "raar1024": ((1024, 1024), 256, 1e8, 8),
    "batch512": ((512, 512), 128, 1e7, 6),
    "vol128": ((128, 128, 128), 32, 1e8, 3),
    "hio1000": ((1000, 1000), 250, 1e7, 1000 / 85.0),
}


def _gaussian_smooth(obj: np.ndarray, sigma: float) -> np.ndarray:
    try:
        from scipy.ndimage import gaussian_filter

        return gaussian_filter(obj, sigma=sigma, mode="constant")
    except ImportError:  # separable fallback with the same truncation (4 sigma)
        r = int(4.0 * sigma + 0.5)
        x = np.arange(-r, r + 1)
        k = np.exp(-0.5 * (x / sigma) ** 2)
        k /= k.sum()
        out = obj
        for ax in range(obj.ndim):
            out = np.apply_along_axis(lambda v: np.convolve(v, k, mode="same"), ax, out)
        return out


def centred_radius(shape) -> np.ndarray:
    grids = np.meshgrid(*[np.arange(s) - s // 2 for s in shape], indexing="ij")
    return np.sqrt(sum(g.astype(np.float64) ** 2 for g in grids))


def make_object(shape, blob: int, seed: int = 0) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    obj = np.zeros(shape, np.float64)
    sl = tuple(slice(s // 2 - blob // 2, s // 2 - blob // 2 + blob) for s in shape)
    obj[sl] = rng.random([blob] * len(shape))
    return _gaussian_smooth(obj, 2.0)


def make_pattern(shape, blob: int, photons: float, beamstop: float, seed: int = 0):
    """Returns (amplitudes float32, mask int32, support float32, object float64), shifted layout."""
    shape = tuple(int(s) for s in shape)
    obj = make_object(shape, blob, seed)
    inten = np.abs(np.fft.fftn(obj)) ** 2
    inten *= photons / inten.sum()
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    amp = np.sqrt(rng.poisson(np.fft.fftshift(inten)).astype(np.float64))
    r = centred_radius(shape)
    mask = (r >= beamstop).astype(np.int32)
    amp[mask == 0] = 0.0
    support = (r < 0.75 * blob).astype(np.float32)
    return (
        np.ascontiguousarray(np.fft.ifftshift(amp).astype(np.float32)),
        np.ascontiguousarray(np.fft.ifftshift(mask).astype(np.int32)),
        np.ascontiguousarray(np.fft.ifftshift(support)),
        np.fft.ifftshift(obj),
    )


def workload(name: str, seed: int = 0):
    shape, blob, photons, bs = WORKLOADS[name]
    return make_pattern(shape, blob, photons, bs, seed)


def small_pattern(shape, seed: int = 0, photons: float = 1e6):
    """Tiny cases for parity tests: blob = n/4 per axis, beamstop n/32."""
    shape = tuple(int(s) for s in shape)
    blob = max(2, min(shape) // 4)
    return make_pattern(shape, blob, photons, max(1.0, min(shape) / 32.0), seed)
