"""Synthetic reconstructions for the PRTF tests: one object, shifted with
wrap-around, with random global phases, one of them reflected through the
origin (the reflection sp_image_superimpose corrects), plus a little noise."""
import numpy as np


def reconstructions(shape, n=6, seed=0, noise=1e-3):
    rng = np.random.default_rng(seed)
    obj = np.zeros(shape, np.complex64)
    sl = tuple(slice(s // 3, s // 3 + max(2, s // 4)) for s in shape)
    obj[sl] = rng.random(obj[sl].shape) + 0.2j * rng.random(obj[sl].shape)
    sup = (np.abs(obj) > 0).astype(np.int32)
    axes = tuple(range(len(shape)))
    ims, sups = [], []
    for k in range(n):
        shift = tuple(int(v) for v in rng.integers(-3, 4, len(shape)))
        o = np.roll(obj, shift, axes) * np.exp(1j * rng.uniform(0, 2 * np.pi))
        s = np.roll(sup, shift, axes)
        if k == n // 2:
            o = o[(slice(None, None, -1),) * len(shape)]
            s = s[(slice(None, None, -1),) * len(shape)]
        ims.append(o + noise * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)))
        sups.append(s)
    return np.array(ims, np.complex64), np.array(sups, np.int32)
