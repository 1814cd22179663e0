"""spimage-b200: libspimage's phase-retrieval hot path on NVIDIA B200 (sm_100a).

The product is ``libspimage_b200.so``: the reference's C API (``sp_phaser_*``,
``sp_phasing_*_alloc``, ``sp_support_*``, ``sp_image_fft/ifft``) implemented in
C over this library's own CUDA kernels.  This module is a thin ctypes binding
of that C API -- the role the reference's SWIG module plays
(``src/spimage_pybackend.i``) -- used by the tests and ``bench.py``.

The library must be built first (``python -m libspimage_b200.build``); loading
fails loudly when it is missing or when no GPU is present, there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libspimage_b200.so")

# reference enums (include/spimage/phasing.h:14-20, support_update.h:9)
SpHIO, SpRAAR, SpDiffMap, SpER = 1, 2, 3, 4
SpNoConstraints, SpRealObject, SpPositiveRealObject, SpPositiveComplexObject = 0, 1, 2, 4
SpPositivityFlipping, SpCentrosymmetricObject, SpAmplitudeErrorMargin = 8, 16, 32
SpModelRandomPhases, SpModelZeroPhases, SpModelRandomValues, SpModelMaskedOutZeroed = 1, 2, 4, 256
SpSupportFromPatterson = 1
SpEngineAutomatic, SpEngineCPU, SpEngineCUDA = 0, 1, 2
SpPixelInsideSupport, SpPixelMeasuredAmplitude = 1, 2
SpRecoverPhases, SpRecoverAmplitudes = 0, 1
SpSupportThreshold, SpSupportArea, SpSupportCentreImage, SpSupportTemplate, SpSupportStatic, SpSupportClose = 1, 2, 3, 4, 5, 6


class sp_c3matrix(C.Structure):
    _fields_ = [("x", C.c_uint), ("y", C.c_uint), ("z", C.c_uint), ("data", C.c_void_p)]


class sp_i3matrix(C.Structure):
    _fields_ = [("x", C.c_uint), ("y", C.c_uint), ("z", C.c_uint), ("data", C.c_void_p)]


class Image(C.Structure):
    _fields_ = [
        ("phased", C.c_int),
        ("scaled", C.c_int),
        ("image", C.POINTER(sp_c3matrix)),
        ("mask", C.POINTER(sp_i3matrix)),
        ("detector", C.c_void_p),
        ("shifted", C.c_int),
        ("rec_coords", C.c_void_p),
        ("num_dimensions", C.c_int),
    ]


class SpPhaser(C.Structure):
    _fields_ = [
        ("amplitudes", C.c_void_p),
        ("amplitudes_min", C.c_void_p),
        ("amplitudes_max", C.c_void_p),
        ("phased_amplitudes", C.c_void_p),
        ("pixel_flags", C.c_void_p),
        ("phasing_objective", C.c_int),
        ("algorithm", C.c_void_p),
        ("sup_algorithm", C.c_void_p),
        ("iteration", C.c_int),
        ("image_size", C.c_int),
        ("nx", C.c_int),
        ("ny", C.c_int),
        ("nz", C.c_int),
    ]


_IMG = C.POINTER(Image)
_PH = C.POINTER(SpPhaser)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p
_lib = None


def load():
    """Loads libspimage_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m libspimage_b200.build`")
    lib = C.CDLL(LIB_PATH)
    sig = {
        "_sp_image_alloc": (_IMG, [C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_int]),
        "_sp_image_free": (None, [_IMG, C.c_char_p, C.c_int]),
        "spb_smap_create": (_vp, [C.c_int, _fp, _fp]),
        "spb_smap_free": (None, [_vp]),
        "spb_smap_interpolate": (C.c_float, [_vp, C.c_float]),
        "sp_srand": (None, [C.c_int]),
        "sp_phasing_hio_alloc": (_vp, [_vp, C.c_int]),
        "sp_phasing_raar_alloc": (_vp, [_vp, C.c_int]),
        "sp_phasing_er_alloc": (_vp, [C.c_int]),
        "sp_phasing_diff_map_alloc": (_vp, [_vp, C.c_float, C.c_float, C.c_int]),
        "sp_support_area_alloc": (_vp, [_vp, _vp]),
        "sp_support_threshold_alloc": (_vp, [_vp, _vp]),
        "sp_support_static_alloc": (_vp, []),
        "sp_support_close_alloc": (_vp, [C.c_int]),
        "sp_support_centre_image_alloc": (_vp, []),
        "sp_support_template_alloc": (_vp, [_IMG, C.c_float, _vp]),
        "sp_support_array_init": (_vp, [_vp, C.c_int]),
        "sp_support_array_append": (None, [_vp, _vp]),
        "sp_phaser_alloc": (_PH, []),
        "sp_phaser_free": (None, [_PH]),
        "sp_phaser_init": (C.c_int, [_PH, _vp, _vp, C.c_int]),
        "sp_phaser_set_phasing_algorithm": (C.c_int, [_PH, _vp]),
        "sp_phaser_set_amplitudes": (None, [_PH, _IMG]),
        "sp_phaser_set_amplitudes_margins": (None, [_PH, _IMG, _IMG]),
        "sp_phaser_set_phased_amplitudes": (None, [_PH, _IMG]),
        "sp_phaser_set_objective": (None, [_PH, C.c_int]),
        "sp_phaser_set_model": (None, [_PH, _IMG]),
        "sp_phaser_set_support": (None, [_PH, _IMG]),
        "sp_phaser_init_model": (C.c_int, [_PH, _IMG, C.c_int]),
        "sp_phaser_init_support": (C.c_int, [_PH, _IMG, C.c_int, C.c_float]),
        "sp_phaser_iterate": (C.c_int, [_PH, C.c_int]),
        "sp_phaser_model": (_IMG, [_PH]),
        "sp_phaser_old_model": (_IMG, [_PH]),
        "sp_phaser_model_before_projection": (_IMG, [_PH]),
        "sp_phaser_model_change": (_IMG, [_PH]),
        "sp_phaser_fmodel": (_IMG, [_PH]),
        "sp_phaser_fmodel_with_mask": (_IMG, [_PH]),
        "sp_phaser_model_with_support": (_IMG, [_PH]),
        "sp_phaser_support": (_IMG, [_PH]),
        "sp_phaser_amplitudes": (_IMG, [_PH]),
        "sp_phaser_efourier": (C.c_float, [_PH, _fp]),
        "sp_phaser_ereal": (C.c_float, [_PH]),
        "sp_phaser_support_fraction": (C.c_float, [_PH]),
        "sp_phaser_last_error": (C.c_char_p, []),
        "sp_image_fftw3": (_IMG, [_IMG]),
        "sp_image_ifftw3": (_IMG, [_IMG]),
        "sp_gaussian_blur": (_IMG, [_IMG, C.c_float]),
        "sp_phaser_set_cuda_stream": (C.c_int, [_PH, _vp]),
        "sp_phaser_device_context": (_vp, [_PH]),
        "spb_ctx_profile": (C.c_int, [_vp, C.c_int]),
        "spb_ctx_profile_read": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_double)]),
        "spb_kernel_name": (C.c_char_p, [C.c_int]),
        "spb_ctx_launch_count": (C.c_longlong, [_vp]),
        "spb_error_string": (C.c_char_p, []),
        "spb_device_count": (C.c_int, []),
        "spb_fft_host": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _fp, _fp]),
        "spb_blur_host": (C.c_int, [C.c_int, C.c_int, C.c_int, _fp, C.c_float, _fp]),
        "spb_support_from_blur_host": (C.c_int, [C.c_longlong, _fp, C.c_int, C.c_float, _ip]),
        "sp_phaser_set_starts": (C.c_int, [_PH, C.c_int]),
        "sp_phaser_autotune": (C.c_int, [_PH]),
        "spb_ctx_set_tuning": (C.c_int, [_vp, C.c_int, C.c_int]),
        "spb_ctx_get_tuning": (C.c_int, [_vp, C.c_int]),
        "sp_phaser_starts": (C.c_int, [_PH]),
        "sp_phaser_init_models": (C.c_int, [_PH, C.c_int, _ip]),
        "sp_phaser_init_models_device": (C.c_int, [_PH, C.c_int, C.POINTER(C.c_ulonglong)]),
        "sp_phaser_start_model": (C.c_int, [_PH, C.c_int, _IMG]),
        "sp_phaser_start_support": (C.c_int, [_PH, C.c_int, _IMG]),
        "sp_phaser_start_model_before_projection": (C.c_int, [_PH, C.c_int, _IMG]),
        "sp_phaser_start_fmodel": (C.c_int, [_PH, C.c_int, _IMG]),
        "sp_phaser_set_support_algorithm": (C.c_int, [_PH, _vp]),
        "sp_phaser_starts_efourier": (C.c_int, [_PH, _fp, _fp]),
        "sp_phaser_starts_ereal": (C.c_int, [_PH, _fp]),
        "sp_phaser_starts_support_fraction": (C.c_int, [_PH, _fp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    """Names the C-ABI headers declare (include/spimage/*.h)."""
    import re

    names = []
    inc = os.path.join(os.path.dirname(PKG), "include", "spimage")
    for fn in sorted(os.listdir(inc)):
        text = open(os.path.join(inc, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\([^;{]*\)\s*;", text, flags=re.M):
            if "static" in m.group(0).split("(")[0] or "#define" in m.group(0):
                continue
            names.append(m.group(1))
    return sorted(set(names))


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.complex64)


def _p(a, t=_fp):
    return a.ctypes.data_as(t)


def _check(rc, what):
    if rc != 0:
        lib = load()
        raise RuntimeError(f"{what} failed ({rc}): {lib.spb_error_string().decode()}")


def _shape3(shape):
    shape = tuple(int(s) for s in shape)
    return ((1,) + shape) if len(shape) == 2 else shape


def new_image(data=None, mask=None, shape=None, phased=1, shifted=0):
    """Allocates an Image (library-owned memory) from numpy arrays (z, y, x) or (y, x)."""
    lib = load()
    if shape is None:
        shape = np.shape(data)
    nz, ny, nx = _shape3(shape)
    img = lib._sp_image_alloc(nx, ny, nz, b"python", 0)
    n = nx * ny * nz
    if data is not None:
        d = np.ctypeslib.as_array(C.cast(img.contents.image.contents.data, _fp), shape=(2 * n,))
        d[:] = _c64(data).ravel().view(np.float32)
    if mask is not None:
        m = np.ctypeslib.as_array(C.cast(img.contents.mask.contents.data, _ip), shape=(n,))
        m[:] = np.ascontiguousarray(mask, dtype=np.int32).ravel()
    img.contents.phased = phased
    img.contents.shifted = shifted
    return img


def image_data(img, shape):
    n = int(np.prod(shape))
    d = np.ctypeslib.as_array(C.cast(img.contents.image.contents.data, _fp), shape=(2 * n,))
    return d.copy().view(np.complex64).reshape(shape)


def image_mask(img, shape):
    n = int(np.prod(shape))
    m = np.ctypeslib.as_array(C.cast(img.contents.mask.contents.data, _ip), shape=(n,))
    return m.copy().reshape(shape)


def free_image(img):
    load()._sp_image_free(img, b"python", 0)


def smap(schedule):
    """sp_smap from a float (constant) or a dict {iteration: value}."""
    lib = load()
    if isinstance(schedule, dict):
        items = sorted(schedule.items())
    else:
        items = [(0.0, float(schedule))]
    k = _f32([a for a, _ in items])
    v = _f32([b for _, b in items])
    return lib.spb_smap_create(len(items), _p(k), _p(v))


class Phaser:
    """An SpPhaser driven through the library's C API (GPU engine)."""

    def __init__(self, shape):
        self.lib = load()
        self.shape = tuple(int(s) for s in shape)
        self.nz, self.ny, self.nx = _shape3(self.shape)
        self.n = self.nx * self.ny * self.nz
        self.ph = self.lib.sp_phaser_alloc()
        self.alg = None
        self.sup = None
        self._owned = []

    def close(self):
        if self.ph:
            self.lib.sp_phaser_free(self.ph)
            self.ph = None
        for img in self._owned:
            free_image(img)
        self._owned = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _img(self, *a, **k):
        img = new_image(*a, **k)
        self._owned.append(img)
        return img

    # -- configuration (same call order as the reference's Reconstructor) --
    def set_algorithm(self, alg, beta=0.9, constraints=0, gamma1=float("inf"), gamma2=float("inf")):
        if alg == SpHIO:
            a = self.lib.sp_phasing_hio_alloc(smap(beta), constraints)
        elif alg == SpRAAR:
            a = self.lib.sp_phasing_raar_alloc(smap(beta), constraints)
        elif alg == SpER:
            a = self.lib.sp_phasing_er_alloc(constraints)
        else:
            a = self.lib.sp_phasing_diff_map_alloc(smap(beta), gamma1, gamma2, constraints)
        if self.alg is not None:
            _check(self.lib.sp_phaser_set_phasing_algorithm(self.ph, a), "sp_phaser_set_phasing_algorithm")
        self.alg = a

    def add_support_update(self, kind, period, blur, sel):
        if kind == SpSupportArea:
            s = self.lib.sp_support_area_alloc(smap(blur), smap(sel))
        elif kind == SpSupportThreshold:
            s = self.lib.sp_support_threshold_alloc(smap(blur), smap(sel))
        else:
            s = self.lib.sp_support_static_alloc()
        if self.sup is None:
            self.sup = self.lib.sp_support_array_init(s, period)
        else:
            self.lib.sp_support_array_append(self.sup, s)

    def _append_support(self, s, period):
        if self.sup is None:
            self.sup = self.lib.sp_support_array_init(s, period)
        else:
            self.lib.sp_support_array_append(self.sup, s)

    def add_support_close(self, period, size):
        self._append_support(self.lib.sp_support_close_alloc(size), period)

    def add_support_centre(self, period):
        self._append_support(self.lib.sp_support_centre_image_alloc(), period)

    def add_support_template(self, period, support, blur_radius, area):
        img = self._img(np.asarray(support, np.complex64))
        self._append_support(self.lib.sp_support_template_alloc(img, blur_radius, smap(area)), period)

    def start(self, engine=SpEngineCUDA):
        rc = self.lib.sp_phaser_init(self.ph, self.alg, self.sup, engine)
        if rc:
            raise RuntimeError(f"sp_phaser_init failed ({rc}): {self.lib.sp_phaser_last_error().decode()}")

    def set_amplitudes(self, amp, mask):
        self.lib.sp_phaser_set_amplitudes(self.ph, self._img(_f32(amp).astype(np.complex64), mask))

    def set_amplitudes_margins(self, amin, amax):
        self.lib.sp_phaser_set_amplitudes_margins(
            self.ph, self._img(_f32(amin).astype(np.complex64)), self._img(_f32(amax).astype(np.complex64))
        )

    def set_phased_amplitudes(self, pa, mask):
        self.lib.sp_phaser_set_phased_amplitudes(self.ph, self._img(pa, mask))

    def set_objective(self, obj):
        self.lib.sp_phaser_set_objective(self.ph, obj)

    def set_support(self, support):
        rc = self.lib.sp_phaser_init_support(self.ph, self._img(np.asarray(support, np.complex64)), 0, 0.0)
        _check(rc, "sp_phaser_init_support")

    def init_support_patterson(self, value):
        _check(self.lib.sp_phaser_init_support(self.ph, None, SpSupportFromPatterson, value), "Patterson support")

    def init_model(self, flags, seed=None, model=None):
        if seed is not None:
            self.lib.sp_srand(seed)
        img = self._img(model) if model is not None else None
        return self.lib.sp_phaser_init_model(self.ph, img, flags)

    def set_model(self, model):
        self.lib.sp_phaser_set_model(self.ph, self._img(model))

    def iterate(self, n):
        return self.lib.sp_phaser_iterate(self.ph, n)

    @property
    def iteration(self):
        return self.ph.contents.iteration

    # -- accessors --
    def _get(self, fn):
        img = fn(self.ph)
        if not img:
            raise RuntimeError(self.lib.sp_phaser_last_error().decode())
        return image_data(img, self.shape)

    def get(self, which):
        fn = {0: self.lib.sp_phaser_old_model, 1: self.lib.sp_phaser_model, 2: self.lib.sp_phaser_model_before_projection}
        return self._get(fn[which])

    def model(self):
        return self._get(self.lib.sp_phaser_model)

    def old_model(self):
        return self._get(self.lib.sp_phaser_old_model)

    def model_before_projection(self):
        return self._get(self.lib.sp_phaser_model_before_projection)

    def model_change(self):
        return self._get(self.lib.sp_phaser_model_change)

    def fmodel(self):
        return self._get(self.lib.sp_phaser_fmodel)

    def _get_masked(self, fn):
        img = fn(self.ph)
        if not img:
            raise RuntimeError(self.lib.sp_phaser_last_error().decode())
        return image_data(img, self.shape), image_mask(img, self.shape)

    def fmodel_with_mask(self):
        """(FFT of the model, measured-amplitude mask)"""
        return self._get_masked(self.lib.sp_phaser_fmodel_with_mask)

    def model_with_support(self):
        """(model, support as mask)"""
        return self._get_masked(self.lib.sp_phaser_model_with_support)

    def amplitudes_image(self):
        """(amplitudes as a complex image, measured mask)"""
        return self._get_masked(self.lib.sp_phaser_amplitudes)

    def support(self):
        img = self.lib.sp_phaser_support(self.ph)
        return (image_data(img, self.shape).real != 0).astype(np.int32)

    def flags(self):
        sup = self.support()
        amp = self.lib.sp_phaser_amplitudes(self.ph)
        meas = image_mask(amp, self.shape)
        return (sup * SpPixelInsideSupport + (meas != 0) * SpPixelMeasuredAmplitude).astype(np.int32)

    def efourier(self):
        f = C.c_float()
        e = self.lib.sp_phaser_efourier(self.ph, C.byref(f))
        return float(e), float(f.value)

    def ereal(self):
        return float(self.lib.sp_phaser_ereal(self.ph))

    def support_fraction(self):
        return float(self.lib.sp_phaser_support_fraction(self.ph))

    # -- extension: batched random starts of one pattern --
    def set_starts(self, nb):
        _check(self.lib.sp_phaser_set_starts(self.ph, int(nb)), "sp_phaser_set_starts")

    @property
    def starts(self):
        return int(self.lib.sp_phaser_starts(self.ph))

    def init_models(self, flags, seeds=None):
        """seeds[b] seeds start b; None draws the starts one after another
        from the current rand() stream"""
        if seeds is None:
            return self.lib.sp_phaser_init_models(self.ph, flags, None)
        s = np.ascontiguousarray(seeds, dtype=np.int32)
        assert s.size == self.starts
        return self.lib.sp_phaser_init_models(self.ph, flags, _p(s, _ip))

    def init_models_device(self, flags, seeds):
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        assert s.size == self.starts
        return self.lib.sp_phaser_init_models_device(self.ph, flags, s.ctypes.data_as(C.POINTER(C.c_ulonglong)))

    def _start_image(self, fn, b):
        img = self._img(np.zeros(self.shape, np.complex64))
        _check(fn(self.ph, int(b), img), fn.__name__)
        out = image_data(img, self.shape)
        self._owned.remove(img)
        free_image(img)
        return out

    def start_model(self, b):
        return self._start_image(self.lib.sp_phaser_start_model, b)

    def start_fmodel(self, b):
        return self._start_image(self.lib.sp_phaser_start_fmodel, b)

    def start_model_before_projection(self, b):
        return self._start_image(self.lib.sp_phaser_start_model_before_projection, b)

    def start_support(self, b):
        return (self._start_image(self.lib.sp_phaser_start_support, b).real != 0).astype(np.int32)

    def starts_efourier(self):
        e = np.zeros(self.starts, np.float32)
        f = np.zeros(self.starts, np.float32)
        _check(self.lib.sp_phaser_starts_efourier(self.ph, _p(e), _p(f)), "sp_phaser_starts_efourier")
        return e, f

    def starts_ereal(self):
        e = np.zeros(self.starts, np.float32)
        _check(self.lib.sp_phaser_starts_ereal(self.ph, _p(e)), "sp_phaser_starts_ereal")
        return e

    def starts_support_fraction(self):
        e = np.zeros(self.starts, np.float32)
        _check(self.lib.sp_phaser_starts_support_fraction(self.ph, _p(e)), "sp_phaser_starts_support_fraction")
        return e

    # -- extension: launch-shape autotuner --
    def autotune(self):
        _check(self.lib.sp_phaser_autotune(self.ph), "sp_phaser_autotune")
        ctx = self.lib.sp_phaser_device_context(self.ph)
        return {"row_lines": self.lib.spb_ctx_get_tuning(ctx, 0), "no_pdl": self.lib.spb_ctx_get_tuning(ctx, 1),
                "row_g0": self.lib.spb_ctx_get_tuning(ctx, 2), "split": self.lib.spb_ctx_get_tuning(ctx, 3),
                "persist": self.lib.spb_ctx_get_tuning(ctx, 4), "col_width": self.lib.spb_ctx_get_tuning(ctx, 5)}

    def set_tuning(self, knob, value):
        ctx = self.lib.sp_phaser_device_context(self.ph)
        _check(self.lib.spb_ctx_set_tuning(ctx, knob, value), "spb_ctx_set_tuning")

    # -- extensions: caller stream and per-kernel timing --
    def set_stream(self, stream_handle):
        _check(self.lib.sp_phaser_set_cuda_stream(self.ph, stream_handle), "sp_phaser_set_cuda_stream")

    def profile(self, enable):
        ctx = self.lib.sp_phaser_device_context(self.ph)
        _check(self.lib.spb_ctx_profile(ctx, 1 if enable else 0), "spb_ctx_profile")

    def launch_count(self):
        return int(self.lib.spb_ctx_launch_count(self.lib.sp_phaser_device_context(self.ph)))

    def kernel_times(self):
        """{kernel name: (launches, total ms)} since profiling was enabled."""
        ctx = self.lib.sp_phaser_device_context(self.ph)
        out = {}
        for k in range(20):
            n = C.c_longlong()
            ms = C.c_double()
            _check(self.lib.spb_ctx_profile_read(ctx, k, C.byref(n), C.byref(ms)), "spb_ctx_profile_read")
            if n.value:
                out[self.lib.spb_kernel_name(k).decode()] = (int(n.value), float(ms.value))
        return out


# ---- one-shot device entry points (numpy in, numpy out) ----

def fft(x, sign=-1):
    """Unnormalised FFT of a complex64 2-D/3-D array on the GPU (sign -1 forward)."""
    lib = load()
    a = _c64(x)
    nz, ny, nx = _shape3(a.shape)
    out = np.empty_like(a)
    _check(lib.spb_fft_host(nx, ny, nz, sign, _p(a), _p(out)), "spb_fft_host")
    return out


def gaussian_blur(x, radius):
    lib = load()
    a = _c64(x)
    nz, ny, nx = _shape3(a.shape)
    out = np.empty_like(a)
    _check(lib.spb_blur_host(nx, ny, nz, _p(a), radius, _p(out)), "spb_blur_host")
    return out


def support_from_blur(blur, kind, value, flags):
    """New pixel flags after thresholding an already blurred image (area or threshold rule)."""
    lib = load()
    b = _c64(blur).ravel()
    f = np.ascontiguousarray(flags, dtype=np.int32).ravel().copy()
    _check(lib.spb_support_from_blur_host(b.size, _p(b), kind, value, _p(f, _ip)), "spb_support_from_blur_host")
    return f.reshape(np.shape(flags))
