"""Oracle of the PRTF (test infrastructure only).

The reference's Python prtf (src/_spimage_prtf.py:17-106) restated step for
step, calling the reference's own C routines from oracle/_ref/libspref.so for
every image operation it delegates to libspimage: sp_image_superimpose
(src/image_util.c:2974-3007), sp_image_phase_match (:3160-3186), sp_image_add
(:1089-1091) and sp_image_fftw3 (src/fft.c:152-175, on the oracle FFT).  The
numpy steps (the first image's spectrum, the unit phasors, the zero counts,
the final division) are the reference's own numpy code.  Needs the reference
build; the parity test skips without it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _load_reference

_vp = C.c_void_p
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)


def _lib():
    lib = _load_reference()
    if not getattr(lib, "_prtf_bound", False):
        lib.sp_image_superimpose.argtypes = [_vp, _vp, C.c_int]
        lib.sp_image_phase_match.argtypes = [_vp, _vp, C.c_int]
        lib.sp_image_phase_match.restype = C.c_float
        lib.sp_image_add.argtypes = [_vp, _vp]
        lib.sp_image_fftw3.argtypes = [_vp]
        lib.sp_image_fftw3.restype = _vp
        lib._prtf_bound = True
    return lib


def _shape3(shape):
    return (1,) + tuple(shape) if len(shape) == 2 else tuple(shape)


class _Img:
    """A reference Image holding a numpy array (numpy_array_to_image of the reference)."""

    def __init__(self, lib, data, mask=None):
        self.lib = lib
        self.shape = data.shape
        nz, ny, nx = _shape3(data.shape)
        self.n = nx * ny * nz
        self.h = lib.ref_image_alloc(nx, ny, nz)
        d = np.ctypeslib.as_array(lib.ref_image_data(self.h), shape=(2 * self.n,))
        d[:] = np.ascontiguousarray(data, np.complex64).ravel().view(np.float32)
        if mask is not None:
            m = np.ctypeslib.as_array(lib.ref_image_mask(self.h), shape=(self.n,))
            m[:] = np.ascontiguousarray(mask, np.int32).ravel()

    @staticmethod
    def data_of(lib, h, n, shape):
        return np.ctypeslib.as_array(lib.ref_image_data(h), shape=(2 * n,)).copy().view(np.complex64).reshape(shape)

    def data(self):
        return _Img.data_of(self.lib, self.h, self.n, self.shape)

    def mask(self):
        return np.ctypeslib.as_array(self.lib.ref_image_mask(self.h), shape=(self.n,)).copy().reshape(self.shape)

    def free(self):
        self.lib.ref_image_free(self.h)


def prtf_reference(images_rs, supports, translate=True, enantio=True):
    """PRTF of the reconstructions images_rs[N, ...] with supports[N, ...]:
    {"prtf" (fftshifted), "super_image", "super_mask"}."""
    lib = _lib()
    images_rs = np.asarray(images_rs)
    N = images_rs.shape[0]
    shape = images_rs.shape[1:]
    image0_fs = np.fft.fftn(images_rs[0])
    sum_fs = image0_fs.copy()
    sum_fs[abs(sum_fs) > 0.] /= abs(sum_fs[abs(sum_fs) > 0.])
    zeros = np.zeros(shape, dtype="int")
    zeros[abs(sum_fs) <= 0.] = 1
    sum_fs = sum_fs.astype(np.complex64)
    avg = _Img(lib, images_rs[0])
    avg_msk = np.zeros(shape, dtype="float")
    for i in range(1, N):
        img = _Img(lib, images_rs[i], supports[i])
        if translate:
            lib.sp_image_superimpose(avg.h, img.h, 1 if enantio else 0)
            lib.sp_image_phase_match(avg.h, img.h, 2)
        lib.sp_image_add(avg.h, img.h)
        m = img.mask()
        if m.sum() > 0:
            avg_msk[m == 0] += 1
        th = lib.sp_image_fftw3(img.h)
        tmp = _Img.data_of(lib, th, img.n, shape)
        lib.ref_image_free(th)
        positive = abs(tmp) > 0.
        tmp[positive] /= abs(tmp)[positive]
        zeros += (positive == False)  # noqa: E712 (the reference's expression)
        sum_fs = (sum_fs + tmp).astype(np.complex64)
        img.free()
    prtf = (sum_fs / np.float32(N)).astype(np.complex64)
    prtf[zeros > 0] = 0.
    out = {"prtf": np.fft.fftshift(abs(prtf)).astype(np.float32), "super_image": avg.data(),
           "super_mask": avg_msk > 0}
    avg.free()
    return out


# ---- the reference's C PRTF (src/prtf.c:6-78) and fractional superposition
# (src/image_util.c:3024-3066), called in oracle/_ref

def _c_lib():
    lib = _lib()
    if not getattr(lib, "_cprtf_bound", False):
        lib.sp_prtf_basic.argtypes = [C.POINTER(_vp), C.c_int]
        lib.sp_prtf_basic.restype = _vp
        lib.sp_prtf_advanced.argtypes = [C.POINTER(_vp), C.c_int, C.c_int]
        lib.sp_prtf_advanced.restype = _vp
        lib.sp_image_superimpose_fractional.argtypes = [_vp, _vp, C.c_int, C.c_int]
        lib._cprtf_bound = True
    return lib


def superimpose_fractional(a, b, flags, precision):
    """b superimposed on a (both numpy, same shape) by the reference."""
    lib = _c_lib()
    ia, ib = _Img(lib, np.asarray(a)), _Img(lib, np.asarray(b))
    lib.sp_image_superimpose_fractional(ia.h, ib.h, int(flags), int(precision))
    out = ib.data()
    ia.free()
    ib.free()
    return out


def prtf_basic(images):
    lib = _c_lib()
    imgs = [_Img(lib, np.asarray(im)) for im in images]
    arr = (_vp * len(imgs))(*[im.h for im in imgs])
    h = lib.sp_prtf_basic(arr, len(imgs))
    out = _Img.data_of(lib, h, imgs[0].n, imgs[0].shape)
    lib.ref_image_free(h)
    for im in imgs:
        im.free()
    return out


def prtf_advanced(images, flags):
    """(prtf, images after the call) of the reference's sp_prtf_advanced; the
    inputs are marked phased and shifted (as spectra from sp_image_fft are)."""
    lib = _c_lib()
    imgs = [_Img(lib, np.asarray(im)) for im in images]
    for im in imgs:
        lib.ref_image_set_flags(im.h, 1, 1)
    arr = (_vp * len(imgs))(*[im.h for im in imgs])
    h = lib.sp_prtf_advanced(arr, len(imgs), int(flags))
    out = _Img.data_of(lib, h, imgs[0].n, imgs[0].shape)
    lib.ref_image_free(h)
    after = [im.data() for im in imgs]
    for im in imgs:
        im.free()
    return out, after
