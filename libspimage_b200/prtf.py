"""PRTF of many reconstructions on the GPU (the reference's Python prtf,
src/_spimage_prtf.py:17-106), over spb_prtf_host.

    out = prtf(images_rs, supports)           # images_rs[N, ...] complex, supports[N, ...]
    out["prtf"]          # |mean unit phasor of the aligned spectra|, fftshifted
    out["super_image"]   # sum of the aligned images
    out["prtf_r"]        # (full_out) radial mean, shells of one pixel, from the centre
    out["super_mask"]    # (full_out) where some non-empty support left the pixel out

The reference's full output also lists every aligned image and mask; this
one does not (the alignment runs on the device and only the sum comes back).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import load


def _bind(lib):
    if not getattr(lib, "_prtf_bound", False):
        fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int)
        lib.spb_prtf_host.restype = C.c_int
        lib.spb_prtf_host.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, fp, ip, C.c_int, fp, fp, ip]
        lib._prtf_bound = True
    return lib


def radial_mean(img, shell_thickness=1.0):
    """Mean over spherical shells [r-1, r) around the pixel shape[0]//2 of
    every axis, r = 1, 2, ... up to the edge; empty shells are dropped (the
    reference's radial, src/_spimage_utils.py:42-69, as its prtf calls it)."""
    img = np.asarray(img, np.float64)
    dim = img.shape[0]
    c = dim // 2
    nshells = int((dim - c) / shell_thickness)
    r2 = sum((g - c) ** 2 for g in np.indices(img.shape))
    out = []
    for k in range(1, nshells + 1):
        r_out = k * shell_thickness
        sel = (r2 >= (r_out - 1) ** 2) & (r2 < r_out ** 2)
        v = img[sel].mean() if sel.any() else np.nan
        if np.isfinite(v):
            out.append(v)
    return np.array(out)


def prtf(images_rs, supports, translate=True, enantio=True, full_out=False):
    lib = _bind(load())
    ims = np.ascontiguousarray(images_rs, np.complex64)
    sups = np.ascontiguousarray(supports, np.int32)
    n = ims.shape[0]
    shape = ims.shape[1:]
    nz, ny, nx = (1,) + tuple(shape) if len(shape) == 2 else tuple(shape)
    out_prtf = np.zeros(shape, np.float32)
    out_img = np.zeros(shape, np.complex64)
    out_msk = np.zeros(shape, np.int32)
    flags = (1 if translate else 0) | (2 if enantio else 0)
    fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int)
    rc = lib.spb_prtf_host(nx, ny, nz, n, ims.ctypes.data_as(fp), sups.ctypes.data_as(ip), flags,
                           out_prtf.ctypes.data_as(fp), out_img.ctypes.data_as(fp), out_msk.ctypes.data_as(ip))
    if rc != 0:
        raise RuntimeError(f"spb_prtf_host failed: {lib.spb_error_string().decode()}")
    out = {"prtf": np.fft.fftshift(out_prtf), "super_image": out_img}
    if full_out:
        out["prtf_r"] = radial_mean(out["prtf"])
        out["super_mask"] = out_msk > 0
    return out
