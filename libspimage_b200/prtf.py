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


# ---- the reference's C PRTF and fractional superposition (include/spimage/prtf.h,
# sp_image_superimpose_fractional), on the GPU

def _bind_c(lib):
    if not getattr(lib, "_cprtf_bound", False):
        fp = C.POINTER(C.c_float)
        lib.spb_superimpose_fractional_host.restype = C.c_int
        lib.spb_superimpose_fractional_host.argtypes = [C.c_int, C.c_int, C.c_int, fp, fp, C.c_int, C.c_int]
        lib.spb_prtf_basic_host.restype = C.c_int
        lib.spb_prtf_basic_host.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, fp, fp]
        lib.spb_prtf_advanced_host.restype = C.c_int
        lib.spb_prtf_advanced_host.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, fp, C.c_int, C.c_int, fp]
        lib._cprtf_bound = True
    return lib


def _dims(shape):
    nz, ny, nx = (1,) + tuple(shape) if len(shape) == 2 else tuple(shape)
    return nx, ny, nz


def superimpose_fractional(a, b, flags=3, precision=4):
    """b superimposed on a (sp_image_superimpose_fractional): flags bit 0
    SpEnantiomorph, bit 1 SpCorrectPhaseShift."""
    lib = _bind_c(load())
    fp = C.POINTER(C.c_float)
    a = np.ascontiguousarray(a, np.complex64)
    out = np.ascontiguousarray(b, np.complex64).copy()
    rc = lib.spb_superimpose_fractional_host(*_dims(a.shape), a.ctypes.data_as(fp), out.ctypes.data_as(fp), int(flags),
                                             int(precision))
    if rc != 0:
        raise RuntimeError(lib.spb_error_string().decode())
    return out


def prtf_basic(images):
    """sp_prtf_basic of images[n, ...] (complex, Fourier space)."""
    lib = _bind_c(load())
    fp = C.POINTER(C.c_float)
    ims = np.ascontiguousarray(images, np.complex64)
    out = np.zeros(ims.shape[1:], np.complex64)
    rc = lib.spb_prtf_basic_host(*_dims(ims.shape[1:]), ims.shape[0], ims.ctypes.data_as(fp), out.ctypes.data_as(fp))
    if rc != 0:
        raise RuntimeError(lib.spb_error_string().decode())
    return out


def prtf_advanced(images, fourier_space=True, in_place=False):
    """(prtf, images) of sp_prtf_advanced; images are overwritten with the
    superimposed images when in_place."""
    lib = _bind_c(load())
    fp = C.POINTER(C.c_float)
    ims = np.ascontiguousarray(images, np.complex64).copy()
    out = np.zeros(ims.shape[1:], np.complex64)
    rc = lib.spb_prtf_advanced_host(*_dims(ims.shape[1:]), ims.shape[0], ims.ctypes.data_as(fp),
                                    1 if fourier_space else 2, 1 if in_place else 0, out.ctypes.data_as(fp))
    if rc != 0:
        raise RuntimeError(lib.spb_error_string().decode())
    return out, ims
