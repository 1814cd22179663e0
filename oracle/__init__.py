"""Oracle for the phase-retrieval hot path -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm may import this package.  It offers two CPU engines with one
interface:

* :class:`Restatement` -- ``oracle/sporacle.c``, a C restatement of the
  reference CPU engine (``src/phasing.c``, ``src/support_update.c``,
  ``src/image_filter.c:80-90``) over the oracle FFT ``oracle/cpufft``.  Its
  sources are committed, so it builds anywhere gcc exists.
* :class:`Reference` -- ``oracle/_ref/libspref.so``, the reference's own
  unmodified C sources compiled against the FFTW3 shim (``oracle/Makefile``
  target ``ref``).  Present only where the reference sources were available at
  build time.

The two are bit-identical on the same inputs (checked in
``tests/test_oracle_pin.py``); the restatement is therefore pinned to the
reference itself.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATE_SO = os.path.join(HERE, "build", "libsporacle.so")
REF_SO = os.path.join(HERE, "_ref", "libspref.so")
# the reference's CUDA engine (cuFFT, cuRAND, thrust), built by `make refcuda`
REF_CUDA_SO = os.path.join(HERE, "_ref", "libspref_cuda.so")

HIO, RAAR, DIFFMAP, ER = 1, 2, 3, 4
SUP_THRESHOLD, SUP_AREA, SUP_CENTRE, SUP_TEMPLATE, SUP_STATIC, SUP_CLOSE = 1, 2, 3, 4, 5, 6
NO_CONSTRAINTS, REAL, POS_REAL, POS_COMPLEX, FLIP, CENTROSYM, MARGIN = 0, 1, 2, 4, 8, 16, 32
RANDOM_PHASES, ZERO_PHASES, RANDOM_VALUES, MASKED_OUT_ZEROED = 1, 2, 4, 256
INSIDE, MEASURED = 1, 2

_lock = threading.Lock()
_libs: dict = {}

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p


def reference_root():
    """Root of the reference's source tree: ``$SPIMAGE_REFERENCE`` when set,
    else the ``REF`` default of ``oracle/Makefile``; None when that directory
    has no ``src/`` (the reference is not present on this machine)."""
    root = os.environ.get("SPIMAGE_REFERENCE")
    if not root:
        with open(os.path.join(HERE, "Makefile")) as f:
            for line in f:
                if line.startswith("REF ?="):
                    root = line.split("?=", 1)[1].strip()
                    break
    return root if root and os.path.isdir(os.path.join(root, "src")) else None


def build(ref: bool = False) -> None:
    """Compile the restatement (and the reference builds when ``ref``: its
    CPU engine, and its CUDA engine where nvcc, cuFFT and cuRAND are at hand --
    a baseline only, so a failure there is reported and not raised)."""
    target = ["all", "ref"] if ref else ["all"]
    extra = []
    if ref and os.environ.get("SPIMAGE_REFERENCE"):
        extra = [f"REF={os.environ['SPIMAGE_REFERENCE']}"]
    subprocess.run(["make", "-s", "-C", HERE] + target + extra, check=True)
    if ref:
        r = subprocess.run(["make", "-s", "-C", HERE, "refcuda"] + extra, capture_output=True, text=True)
        if r.returncode != 0:
            print("oracle: the reference's CUDA engine was not built:\n" + r.stderr[-2000:])


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.complex64)


def _ptr(a, t=_fp):
    return a.ctypes.data_as(t)


def _load_restatement():
    with _lock:
        if "rs" in _libs:
            return _libs["rs"]
        if not os.path.exists(RESTATE_SO):
            build(ref=False)
        lib = C.CDLL(RESTATE_SO)
        lib.spo_create.restype = _vp
        lib.spo_create.argtypes = [C.c_int, C.c_int, C.c_int]
        lib.spo_destroy.argtypes = [_vp]
        lib.spo_set_threads.argtypes = [_vp, C.c_int]
        lib.spo_srand.argtypes = [C.c_int]
        lib.spo_bezier.restype = C.c_float
        lib.spo_bezier.argtypes = [C.c_int, _fp, _fp, C.c_float]
        lib.spo_set_amplitudes.argtypes = [_vp, _fp, _ip]
        lib.spo_set_amplitudes_margins.argtypes = [_vp, _fp, _fp]
        lib.spo_set_phased_amplitudes.argtypes = [_vp, _fp, _ip]
        lib.spo_set_objective.argtypes = [_vp, C.c_int]
        lib.spo_set_support.argtypes = [_vp, _fp]
        lib.spo_init_support_patterson.argtypes = [_vp, C.c_float]
        lib.spo_set_algorithm.argtypes = [_vp, C.c_int, C.c_int, _fp, _fp, C.c_float, C.c_float, C.c_int]
        lib.spo_clear_support_updates.argtypes = [_vp]
        lib.spo_add_support_update.argtypes = [_vp, C.c_int, C.c_int, C.c_int, _fp, _fp, C.c_int, _fp, _fp]
        lib.spo_add_support_close.argtypes = [_vp, C.c_int, C.c_int]
        lib.spo_add_support_centre.argtypes = [_vp, C.c_int]
        lib.spo_add_support_template.argtypes = [_vp, C.c_int, _fp, C.c_float, C.c_int, _fp, _fp]
        lib.spo_init_model.restype = C.c_int
        lib.spo_init_model.argtypes = [_vp, C.c_int, _fp]
        lib.spo_set_model.argtypes = [_vp, _fp]
        lib.spo_iterate.restype = C.c_int
        lib.spo_iterate.argtypes = [_vp, C.c_int]
        lib.spo_iteration.restype = C.c_int
        lib.spo_iteration.argtypes = [_vp]
        lib.spo_get.argtypes = [_vp, C.c_int, _fp]
        lib.spo_get_flags.argtypes = [_vp, _ip]
        lib.spo_efourier.restype = C.c_float
        lib.spo_efourier.argtypes = [_vp, _fp]
        lib.spo_ereal.restype = C.c_float
        lib.spo_ereal.argtypes = [_vp]
        lib.spo_support_fraction.restype = C.c_float
        lib.spo_support_fraction.argtypes = [_vp]
        lib.spo_dm_gamma.restype = C.c_float
        lib.spo_dm_gamma.argtypes = [_vp, C.c_int]
        lib.spo_gaussian_blur.argtypes = [C.c_int, C.c_int, C.c_int, _fp, C.c_float, _fp]
        lib.spo_area_threshold.restype = C.c_float
        lib.spo_area_threshold.argtypes = [C.c_long, _fp, C.c_float]
        lib.spo_fft.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, _fp, _fp]
        lib.spo_module_projection.argtypes = [C.c_long, _fp, _fp, _ip, C.c_int]
        _libs["rs"] = lib
        return lib


def _load_reference(path=REF_SO):
    with _lock:
        if path in _libs:
            return _libs[path]
        if not os.path.exists(path):
            raise RuntimeError(f"oracle/_ref/{os.path.basename(path)} is not built (needs the reference sources)")
        lib = C.CDLL(path)
        lib.ref_image_alloc.restype = _vp
        lib.ref_image_alloc.argtypes = [C.c_int, C.c_int, C.c_int]
        lib.ref_image_free.argtypes = [_vp]
        lib.ref_image_data.restype = _fp
        lib.ref_image_data.argtypes = [_vp]
        lib.ref_image_mask.restype = _ip
        lib.ref_image_mask.argtypes = [_vp]
        lib.ref_image_set_flags.argtypes = [_vp, C.c_int, C.c_int]
        lib.ref_smap.restype = _vp
        lib.ref_smap.argtypes = [C.c_int, _fp, _fp]
        lib.ref_smap_interpolate.restype = C.c_float
        lib.ref_smap_interpolate.argtypes = [_vp, C.c_float]
        lib.ref_phaser_g.restype = _fp
        lib.ref_phaser_g.argtypes = [_vp, C.c_int]
        lib.ref_phaser_flags.restype = _ip
        lib.ref_phaser_flags.argtypes = [_vp]
        lib.ref_phaser_iteration.restype = C.c_int
        lib.ref_phaser_iteration.argtypes = [_vp]
        lib.ref_dm_gamma.restype = C.c_float
        lib.ref_dm_gamma.argtypes = [_vp, C.c_int]
        lib.sp_srand.argtypes = [C.c_int]
        for name in ("sp_phasing_hio_alloc", "sp_phasing_raar_alloc"):
            getattr(lib, name).restype = _vp
            getattr(lib, name).argtypes = [_vp, C.c_int]
        lib.sp_phasing_er_alloc.restype = _vp
        lib.sp_phasing_er_alloc.argtypes = [C.c_int]
        lib.sp_phasing_diff_map_alloc.restype = _vp
        lib.sp_phasing_diff_map_alloc.argtypes = [_vp, C.c_float, C.c_float, C.c_int]
        lib.sp_support_area_alloc.restype = _vp
        lib.sp_support_area_alloc.argtypes = [_vp, _vp]
        lib.sp_support_threshold_alloc.restype = _vp
        lib.sp_support_threshold_alloc.argtypes = [_vp, _vp]
        lib.sp_support_static_alloc.restype = _vp
        lib.sp_support_static_alloc.argtypes = []
        lib.sp_support_close_alloc.restype = _vp
        lib.sp_support_close_alloc.argtypes = [C.c_int]
        lib.sp_support_centre_image_alloc.restype = _vp
        lib.sp_support_centre_image_alloc.argtypes = []
        lib.sp_support_template_alloc.restype = _vp
        lib.sp_support_template_alloc.argtypes = [_vp, C.c_float, _vp]
        lib.sp_support_array_init.restype = _vp
        lib.sp_support_array_init.argtypes = [_vp, C.c_int]
        lib.sp_support_array_append.argtypes = [_vp, _vp]
        lib.sp_phaser_alloc.restype = _vp
        lib.sp_phaser_alloc.argtypes = []
        lib.sp_phaser_free.argtypes = [_vp]
        lib.sp_phaser_init.restype = C.c_int
        lib.sp_phaser_init.argtypes = [_vp, _vp, _vp, C.c_int]
        lib.sp_phaser_set_phasing_algorithm.restype = C.c_int
        lib.sp_phaser_set_phasing_algorithm.argtypes = [_vp, _vp]
        lib.sp_phaser_set_amplitudes.argtypes = [_vp, _vp]
        lib.sp_phaser_set_amplitudes_margins.argtypes = [_vp, _vp, _vp]
        lib.sp_phaser_set_phased_amplitudes.argtypes = [_vp, _vp]
        lib.sp_phaser_set_objective.argtypes = [_vp, C.c_int]
        lib.sp_phaser_set_model.argtypes = [_vp, _vp]
        lib.sp_phaser_set_support.argtypes = [_vp, _vp]
        lib.sp_phaser_init_model.restype = C.c_int
        lib.sp_phaser_init_model.argtypes = [_vp, _vp, C.c_int]
        lib.sp_phaser_init_support.restype = C.c_int
        lib.sp_phaser_init_support.argtypes = [_vp, _vp, C.c_int, C.c_float]
        lib.sp_phaser_iterate.restype = C.c_int
        lib.sp_phaser_iterate.argtypes = [_vp, C.c_int]
        lib.sp_phaser_efourier.restype = C.c_float
        lib.sp_phaser_efourier.argtypes = [_vp, _fp]
        lib.sp_phaser_ereal.restype = C.c_float
        lib.sp_phaser_ereal.argtypes = [_vp]
        lib.sp_phaser_support_fraction.restype = C.c_float
        lib.sp_phaser_support_fraction.argtypes = [_vp]
        lib.sp_gaussian_blur.restype = _vp
        lib.sp_gaussian_blur.argtypes = [_vp, C.c_float]
        lib.sp_image_fftw3.restype = _vp
        lib.sp_image_fftw3.argtypes = [_vp]
        lib.sp_image_ifftw3.restype = _vp
        lib.sp_image_ifftw3.argtypes = [_vp]
        lib.sp_init_fft.restype = C.c_int
        lib.sp_init_fft.argtypes = [C.c_int]
        _libs[path] = lib
        return lib


def _keys_values(smap):
    """A schedule is a float (constant) or a dict {iteration: value}."""
    if isinstance(smap, dict):
        items = sorted(smap.items())
        return _f32([k for k, _ in items]), _f32([v for _, v in items])
    return _f32([0.0]), _f32([float(smap)])


class _Engine:
    """Common interface of the two CPU engines; arrays are numpy (nz, ny, nx) or (ny, nx)."""

    def __init__(self, shape):
        shape = tuple(shape)
        if len(shape) == 2:
            shape = (1,) + shape
        self.shape3 = shape
        self.nz, self.ny, self.nx = shape
        self.n = self.nx * self.ny * self.nz
        self.out_shape = shape if self.nz > 1 else shape[1:]


class Restatement(_Engine):
    """The C restatement (oracle/sporacle.c)."""

    def __init__(self, shape, threads: int = 1):
        super().__init__(shape)
        self.lib = _load_restatement()
        self.ph = self.lib.spo_create(self.nx, self.ny, self.nz)
        self.lib.spo_set_threads(self.ph, threads)
        self._keep = []

    def __del__(self):
        try:
            self.lib.spo_destroy(self.ph)
        except Exception:
            pass

    def set_amplitudes(self, amp, mask):
        a = _f32(amp).ravel()
        m = np.ascontiguousarray(mask, dtype=np.int32).ravel()
        self.lib.spo_set_amplitudes(self.ph, _ptr(a), _ptr(m, _ip))

    def set_amplitudes_margins(self, amin, amax):
        a, b = _f32(amin).ravel(), _f32(amax).ravel()
        self.lib.spo_set_amplitudes_margins(self.ph, _ptr(a), _ptr(b))

    def set_phased_amplitudes(self, pa, mask):
        a = _c64(pa).ravel()
        m = np.ascontiguousarray(mask, dtype=np.int32).ravel()
        self.lib.spo_set_phased_amplitudes(self.ph, _ptr(a), _ptr(m, _ip))

    def set_objective(self, obj):
        self.lib.spo_set_objective(self.ph, obj)

    def set_support(self, support):
        s = _f32(np.real(support)).ravel()
        self.lib.spo_set_support(self.ph, _ptr(s))

    def init_support_patterson(self, value):
        self.lib.spo_init_support_patterson(self.ph, value)

    def set_algorithm(self, alg, beta=0.9, constraints=0, gamma1=float("inf"), gamma2=float("inf")):
        k, v = _keys_values(beta)
        self.lib.spo_set_algorithm(self.ph, alg, len(k), _ptr(k), _ptr(v), gamma1, gamma2, constraints)

    def add_support_update(self, kind, period, blur, sel):
        bk, bv = _keys_values(blur)
        sk, sv = _keys_values(sel)
        self.lib.spo_add_support_update(self.ph, kind, period, len(bk), _ptr(bk), _ptr(bv), len(sk), _ptr(sk), _ptr(sv))

    def add_support_close(self, period, size):
        self.lib.spo_add_support_close(self.ph, period, size)

    def add_support_centre(self, period):
        self.lib.spo_add_support_centre(self.ph, period)

    def add_support_template(self, period, support, blur_radius, area):
        s = _f32(np.real(support)).ravel()
        k, v = _keys_values(area)
        self.lib.spo_add_support_template(self.ph, period, _ptr(s), blur_radius, len(k), _ptr(k), _ptr(v))

    def init_model(self, flags, seed=None, model=None):
        if seed is not None:
            self.lib.spo_srand(seed)
        if model is not None:
            m = _c64(model).ravel()
            return self.lib.spo_init_model(self.ph, flags, _ptr(m))
        return self.lib.spo_init_model(self.ph, flags, None)

    def set_model(self, model):
        m = _c64(model).ravel()
        self.lib.spo_set_model(self.ph, _ptr(m))

    def iterate(self, n):
        return self.lib.spo_iterate(self.ph, n)

    @property
    def iteration(self):
        return self.lib.spo_iteration(self.ph)

    def get(self, which):
        out = np.empty(self.n, np.complex64)
        self.lib.spo_get(self.ph, which, _ptr(out))
        return out.reshape(self.out_shape)

    def model(self):
        return self.get(1)

    def old_model(self):
        return self.get(0)

    def model_before_projection(self):
        return self.get(2)

    def flags(self):
        out = np.empty(self.n, np.int32)
        self.lib.spo_get_flags(self.ph, _ptr(out, _ip))
        return out.reshape(self.out_shape)

    def support(self):
        return (self.flags() & INSIDE).astype(np.int32)

    def efourier(self):
        f = C.c_float()
        e = self.lib.spo_efourier(self.ph, C.byref(f))
        return float(e), float(f.value)

    def ereal(self):
        return float(self.lib.spo_ereal(self.ph))

    def support_fraction(self):
        return float(self.lib.spo_support_fraction(self.ph))


class Reference(_Engine):
    """The reference's own CPU engine (oracle/_ref/libspref.so), driven through its C API."""

    def __init__(self, shape, threads: int = 1):
        super().__init__(shape)
        self.lib = _load_reference()
        if threads > 1:
            self.lib.sp_init_fft(threads)
        self.ph = self.lib.sp_phaser_alloc()
        self.alg = None
        self.sup = None
        self.images = []
        self.amp_img = None
        self.objective = 0

    def _image(self, data=None, mask=None, phased=1, shifted=0):
        img = self.lib.ref_image_alloc(self.nx, self.ny, self.nz)
        self.images.append(img)
        if data is not None:
            d = np.ctypeslib.as_array(self.lib.ref_image_data(img), shape=(self.n * 2,))
            d[:] = _c64(data).ravel().view(np.float32)
        if mask is not None:
            mk = np.ctypeslib.as_array(self.lib.ref_image_mask(img), shape=(self.n,))
            mk[:] = np.ascontiguousarray(mask, dtype=np.int32).ravel()
        self.lib.ref_image_set_flags(img, phased, shifted)
        return img

    def set_algorithm(self, alg, beta=0.9, constraints=0, gamma1=float("inf"), gamma2=float("inf")):
        k, v = _keys_values(beta)
        bm = self.lib.ref_smap(len(k), _ptr(k), _ptr(v))
        if alg == HIO:
            a = self.lib.sp_phasing_hio_alloc(bm, constraints)
        elif alg == RAAR:
            a = self.lib.sp_phasing_raar_alloc(bm, constraints)
        elif alg == ER:
            a = self.lib.sp_phasing_er_alloc(constraints)
        else:
            a = self.lib.sp_phasing_diff_map_alloc(bm, gamma1, gamma2, constraints)
        if self.alg is None:
            self.alg = a
        else:
            self.lib.sp_phaser_set_phasing_algorithm(self.ph, a)
            self.alg = a

    def add_support_update(self, kind, period, blur, sel):
        bk, bv = _keys_values(blur)
        sk, sv = _keys_values(sel)
        bm = self.lib.ref_smap(len(bk), _ptr(bk), _ptr(bv))
        sm = self.lib.ref_smap(len(sk), _ptr(sk), _ptr(sv))
        if kind == SUP_AREA:
            s = self.lib.sp_support_area_alloc(bm, sm)
        elif kind == SUP_THRESHOLD:
            s = self.lib.sp_support_threshold_alloc(bm, sm)
        else:
            s = self.lib.sp_support_static_alloc()
        self._append_support(s, period)

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
        k, v = _keys_values(area)
        am = self.lib.ref_smap(len(k), _ptr(k), _ptr(v))
        img = self._image(np.asarray(support, np.complex64))
        self._append_support(self.lib.sp_support_template_alloc(img, blur_radius, am), period)

    def start(self):
        """sp_phaser_init with the CPU engine; call after set_algorithm/add_support_update."""
        return self.lib.sp_phaser_init(self.ph, self.alg, self.sup, 1)

    def set_amplitudes(self, amp, mask):
        self.lib.sp_phaser_set_amplitudes(self.ph, self._image(_f32(amp).astype(np.complex64), mask))

    def set_amplitudes_margins(self, amin, amax):
        self.lib.sp_phaser_set_amplitudes_margins(
            self.ph, self._image(_f32(amin).astype(np.complex64)), self._image(_f32(amax).astype(np.complex64))
        )

    def set_phased_amplitudes(self, pa, mask):
        self.lib.sp_phaser_set_phased_amplitudes(self.ph, self._image(pa, mask))

    def set_objective(self, obj):
        self.lib.sp_phaser_set_objective(self.ph, obj)

    def set_support(self, support):
        self.lib.sp_phaser_init_support(self.ph, self._image(np.asarray(support, np.complex64)), 0, 0.0)

    def init_support_patterson(self, value):
        self.lib.sp_phaser_init_support(self.ph, None, 1, value)

    def init_model(self, flags, seed=None, model=None):
        if seed is not None:
            self.lib.sp_srand(seed)
        img = self._image(model) if model is not None else None
        return self.lib.sp_phaser_init_model(self.ph, img, flags)

    def set_model(self, model):
        self.lib.sp_phaser_set_model(self.ph, self._image(model))

    def iterate(self, n):
        return self.lib.sp_phaser_iterate(self.ph, n)

    @property
    def iteration(self):
        return self.lib.ref_phaser_iteration(self.ph)

    def get(self, which):
        p = self.lib.ref_phaser_g(self.ph, which)
        a = np.ctypeslib.as_array(p, shape=(self.n * 2,)).copy().view(np.complex64)
        return a.reshape(self.out_shape)

    def model(self):
        return self.get(1)

    def old_model(self):
        return self.get(0)

    def model_before_projection(self):
        return self.get(2)

    def flags(self):
        p = self.lib.ref_phaser_flags(self.ph)
        return np.ctypeslib.as_array(p, shape=(self.n,)).copy().reshape(self.out_shape)

    def support(self):
        return (self.flags() & INSIDE).astype(np.int32)

    def efourier(self):
        f = C.c_float()
        e = self.lib.sp_phaser_efourier(self.ph, C.byref(f))
        return float(e), float(f.value)

    def ereal(self):
        return float(self.lib.sp_phaser_ereal(self.ph))

    def support_fraction(self):
        return float(self.lib.sp_phaser_support_fraction(self.ph))


def ref_cuda_available() -> bool:
    return os.path.exists(REF_CUDA_SO)


class ReferenceCuda(Reference):
    """The reference's own CUDA engine (oracle/_ref/libspref_cuda.so: its
    phasing.cu and friends over cuFFT, cuRAND and thrust, compiled for
    sm_100a), driven through its C API with SpEngineCUDA.  A baseline to time
    beside this project's kernels: its random starts come from cuRAND and its
    transforms from cuFFT, so its iterates are not the CPU engine's bits.  The
    model is read with sp_phaser_model (the engine keeps it on the device)."""

    def __init__(self, shape):
        _Engine.__init__(self, shape)
        self.lib = _load_reference(REF_CUDA_SO)
        self.lib.sp_phaser_model.restype = _vp
        self.lib.sp_phaser_model.argtypes = [_vp]
        self.ph = self.lib.sp_phaser_alloc()
        self.alg = None
        self.sup = None
        self.images = []
        self.amp_img = None
        self.objective = 0

    def start(self):
        """sp_phaser_init with the CUDA engine; call after set_algorithm/add_support_update."""
        return self.lib.sp_phaser_init(self.ph, self.alg, self.sup, 2)

    def model(self):
        img = self.lib.sp_phaser_model(self.ph)
        d = np.ctypeslib.as_array(self.lib.ref_image_data(img), shape=(self.n * 2,)).copy().view(np.complex64)
        return d.reshape(self.out_shape)


def fft(x, sign=-1):
    """Oracle FFT (oracle/cpufft) of a complex64 array (2-D or 3-D, x fastest)."""
    lib = _load_restatement()
    a = _c64(x)
    shape = a.shape if a.ndim == 3 else (1,) + a.shape
    out = np.empty_like(a)
    lib.spo_fft(shape[2], shape[1], shape[0], sign, _ptr(a), _ptr(out))
    return out


def gaussian_blur(x, radius):
    lib = _load_restatement()
    a = _c64(x)
    shape = a.shape if a.ndim == 3 else (1,) + a.shape
    out = np.empty_like(a)
    lib.spo_gaussian_blur(shape[2], shape[1], shape[0], _ptr(a), radius, _ptr(out))
    return out


def area_threshold(blur, area):
    lib = _load_restatement()
    a = _c64(blur).ravel()
    return float(lib.spo_area_threshold(a.size, _ptr(a), area))


def module_projection(G, amp, flags, constraints=0):
    """The Fourier-modulus projection alone (src/phasing.c:1070-1100)."""
    lib = _load_restatement()
    g = _c64(G).ravel().copy()
    a = _f32(amp).ravel()
    f = np.ascontiguousarray(flags, dtype=np.int32).ravel()
    lib.spo_module_projection(g.size, _ptr(g), _ptr(a), _ptr(f, _ip), constraints)
    return g.reshape(np.shape(G))


def bezier(smap, x):
    lib = _load_restatement()
    k, v = _keys_values(smap)
    return float(lib.spo_bezier(len(k), _ptr(k), _ptr(v), x))
