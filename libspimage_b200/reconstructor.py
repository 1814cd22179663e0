"""Reconstructor: the reference's Python driver of the phasing path
(src/_spimage_reconstructor.py:9-769), over this library's C API.

Same configuration calls, the same output cadence and the same result
dictionaries as the reference:

    R = Reconstructor()
    R.set_intensities(I)                      # non-shifted pattern
    R.set_mask(M)
    R.set_number_of_iterations(1000)
    R.set_number_of_outputs(11)
    R.set_initial_support(radius=20)
    R.set_support_algorithm("area", update_period=20, blur_init=3., blur_final=0.7,
                            area_init=0.05, area_final=0.05)
    R.set_phasing_algorithm("hio", beta_init=0.9, beta_final=0.9,
                            constraints=["enforce_positivity", "enforce_real"])
    out = R.reconstruct()                     # one reconstruction
    out = R.reconstruct_loop(512)             # many random starts

Differences from the reference, all deliberate:

* ``reconstruct_loop(N)`` runs the N starts together in one batched phaser
  (``sp_phaser_set_starts``) instead of one after another.  Start k draws its
  random phases as the k-th of N consecutive ``sp_phaser_init_model`` calls
  would (``sp_phaser_init_models`` with no seeds), so every result equals the
  sequential loop's.
* The "threshold" support algorithm works: the reference builds it from
  attributes it never sets (``self._blur_radius``, ``self._threshold``) and
  reads ``area_init``, which a threshold configuration does not have.  Here the
  blur and threshold schedules come from ``blur_init/blur_final`` and
  ``threshold_init/threshold_final``, as its docstring describes.
* Output arrays of ``reconstruct_loop`` have the pattern's shape (the reference
  allocates them as (N, Nx, Ny), which only matches square patterns).
* The 3-D initial support disc is built on a (z, y, x) grid; the reference's
  meshgrid call gives the same grid for cubic volumes only.
* Phasing runs on the GPU only: ``use_gpu=False`` raises, since this library
  has no CPU engine.
"""
from __future__ import annotations

import ctypes as C
import logging

import numpy as np

from . import (SpCentrosymmetricObject, SpEngineCPU, SpEngineCUDA, SpModelRandomPhases, SpNoConstraints,
               SpPositiveComplexObject, SpPositiveRealObject, SpRealObject, free_image, image_data, image_mask,
               load, new_image, smap)

logger = logging.getLogger("RECONSTRUCTOR")
logger.setLevel("WARNING")

_SUPPORT_KWARGS = {"area": ["update_period", "blur_init", "blur_final", "area_init", "area_final"],
                   "threshold": ["update_period", "blur_init", "blur_final", "threshold_init", "threshold_final"],
                   "static": []}
_PHASING_KWARGS = {"raar": ["beta_init", "beta_final"], "hio": ["beta_init", "beta_final"], "er": [],
                   "diffmap": ["beta_init", "beta_final", "gamma1", "gamma2"]}


def output_iterations(number_of_iterations, number_of_outputs):
    """Iterations at which the reference writes outputs
    (src/_spimage_reconstructor.py:439-446)."""
    return np.int64(np.linspace(0, number_of_iterations, number_of_outputs).round())


def initial_support_mask(shape, radius=None, area=None, support_mask=None):
    """The initial support of the reference (src/_spimage_reconstructor.py:401-437):
    a disc (sphere) of the given radius, or of the radius that covers the given
    area fraction, centred at ((N-1)/2) and shifted to the corner; or the given
    mask as it is."""
    shape = tuple(int(s) for s in shape)
    if support_mask is not None:
        return np.asarray(support_mask, np.float32)
    if len(shape) == 2:
        ny, nx = shape
        X, Y = np.meshgrid(np.arange(nx), np.arange(ny))
        R = np.sqrt((X - (nx - 1) / 2.) ** 2 + (Y - (ny - 1) / 2.) ** 2)
        n = nx * ny
    else:
        nz, ny, nx = shape
        # (z, y, x) indexing; the reference's default meshgrid indexing gives
        # the same grid for cubic volumes only
        Z, Y, X = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        R = np.sqrt((X - (nx - 1) / 2.) ** 2 + (Y - (ny - 1) / 2.) ** 2 + (Z - (nz - 1) / 2.) ** 2)
        n = nx * ny * nz
    r = radius if radius is not None else np.sqrt(area * n / np.pi)
    return np.float32(np.fft.fftshift(R) < r)


def phasing_constraints(constraints):
    """Constraint flags from the reference's constraint strings
    (src/_spimage_reconstructor.py:502-512)."""
    c = SpNoConstraints
    if "enforce_positivity" in constraints and "enforce_real" in constraints:
        c |= SpPositiveRealObject
    elif "enforce_real" in constraints:
        c |= SpRealObject
    elif "enforce_positivity" in constraints:
        c |= SpPositiveComplexObject
    if "enforce_centrosymmetry" in constraints:
        c |= SpCentrosymmetricObject
    return c


class Reconstructor:
    def __init__(self, use_gpu=True):
        self._lib = None
        self._use_gpu = use_gpu
        self._ph = None
        self._images = []
        self.clear()

    # ------------------------------------------------------------ configuration
    def clear(self):
        """Deletes all configuration and data."""
        self._free()
        self._amplitudes = None
        self._mask = None
        self._support_init_args = None
        self._n_iterations = None
        self._n_image_outputs = None
        self._n_score_outputs = None
        self._support_stages = []
        self._support_stage_idx = None
        self._phasing_stages = []
        self._phasing_stage_idx = None
        self._reconstruction = None
        self._iteration = None

    def _free(self):
        if self._ph is not None and self._lib is not None:
            self._lib.sp_phaser_free(self._ph)
        self._ph = None
        for img in self._images:
            free_image(img)
        self._images = []

    def __del__(self):
        try:
            self._free()
        except Exception:
            pass

    def _log(self, s, mode="INFO"):
        {"INFO": logger.info, "DEBUG": logger.debug, "WARNING": logger.warning, "ERROR": logger.error}[mode](" " + s)

    def set_intensities(self, intensities, shifted=False):
        """Intensities to phase; negative values are set to zero.  Non-shifted
        (zero frequency at the centre) unless shifted=True."""
        A = np.array(intensities, dtype="float")
        if (A < 0).sum() > 0:
            self._log("negative intensities clipped to zero")
            A[A < 0] = 0.
        A = np.sqrt(A)
        self._amplitudes = A if shifted else np.fft.fftshift(A)

    def set_mask(self, mask, shifted=False):
        """True where the intensity is measured.  Non-shifted unless shifted=True."""
        M = np.array(mask, dtype="bool")
        self._mask = M if shifted else np.fft.fftshift(M)

    def set_number_of_iterations(self, number_of_iterations):
        self._n_iterations = number_of_iterations

    def set_number_of_outputs_images(self, number_of_outputs_images):
        self._n_image_outputs = number_of_outputs_images

    def set_number_of_outputs_scores(self, number_of_outputs_scores):
        self._n_score_outputs = number_of_outputs_scores

    def set_number_of_outputs(self, number_of_outputs):
        self._n_image_outputs = number_of_outputs
        self._n_score_outputs = number_of_outputs

    def set_initial_support(self, **kwargs):
        """radius=..., area=... (fraction of the image) or support_mask=... (used as given)."""
        for k in ("radius", "area", "support_mask"):
            if k in kwargs:
                self._support_init_args = {k: kwargs[k]}
                return
        self._log("set_initial_support: give one of radius, area or support_mask", "ERROR")

    def set_support_algorithm(self, type, number_of_iterations=None, center_image=False, **kwargs):
        self._support_stages = []
        self._support_stage_idx = None
        self.append_support_algorithm(type, number_of_iterations=number_of_iterations, center_image=center_image,
                                      **kwargs)

    def append_support_algorithm(self, type, number_of_iterations, center_image=False, **kwargs):
        """area: update_period, blur_init, blur_final, area_init, area_final;
        threshold: update_period, blur_init, blur_final, threshold_init, threshold_final; static."""
        conf = {"type": type, "center_image": center_image, "number_of_iterations": number_of_iterations}
        if number_of_iterations is None and len(self._support_stages) > 0:
            self._log("only one support stage may leave its number of iterations open", "ERROR")
            return
        if type not in _SUPPORT_KWARGS:
            self._log("append_support_algorithm: known arguments are " + str(list(_SUPPORT_KWARGS)), "ERROR")
            return
        for k in _SUPPORT_KWARGS[type]:
            if k not in kwargs:
                self._log("append_support_algorithm: %s needs %s" % (type, k), "ERROR")
                return
            conf[k] = kwargs[k]
        if number_of_iterations is not None:
            if not self._support_stages:
                self._support_stage_idx = 0
            self._support_stage_idx += number_of_iterations
        self._support_stages.append(conf)

    def set_phasing_algorithm(self, type, **kwargs):
        self._phasing_stages = []
        self._phasing_stage_idx = None
        kw = dict(kwargs)
        kw.setdefault("number_of_iterations", None)
        self.append_phasing_algorithm(type, **kw)

    def append_phasing_algorithm(self, type, **kwargs):
        """er; hio / raar: beta_init, beta_final; diffmap: beta_init, beta_final,
        gamma1, gamma2; all take number_of_iterations and constraints (a list of
        enforce_positivity, enforce_real, enforce_centrosymmetry)."""
        if "number_of_iterations" not in kwargs:
            self._log("append_phasing_algorithm: number_of_iterations is required", "ERROR")
            return
        n = kwargs["number_of_iterations"]
        if n is None and len(self._phasing_stages) > 0:
            self._log("only one phasing stage may leave its number of iterations open", "ERROR")
            return
        if type not in _PHASING_KWARGS:
            self._log("append_phasing_algorithm: known arguments are %s" % list(_PHASING_KWARGS), "ERROR")
            return
        for k in _PHASING_KWARGS[type]:
            if k not in kwargs:
                self._log("append_phasing_algorithm: %s needs %s" % (type, k), "ERROR")
                return
        conf = {"type": type, "constraints": kwargs.get("constraints", "")}
        conf.update(kwargs)
        if n is not None:
            if not self._phasing_stages:
                self._phasing_stage_idx = 0
            self._phasing_stage_idx += n
        self._phasing_stages.append(conf)

    # ------------------------------------------------------------- preparation
    def _prepare(self):
        """The checks of the reference's _prepare_reconstruction
        (src/_spimage_reconstructor.py:310-345); False (with the error logged)
        when the configuration is incomplete."""
        ok = True
        if self._amplitudes is None:
            self._log("not ready: no intensities set", "ERROR")
            ok = False
        if self._support_init_args is None:
            self._log("not ready: no initial support set", "ERROR")
            ok = False
        if not self._support_stages:
            self._log("not ready: no support algorithm set", "ERROR")
            ok = False
        if not self._phasing_stages:
            self._log("not ready: no phasing algorithm set", "ERROR")
            ok = False
        if self._n_image_outputs is None or self._n_score_outputs is None:
            self._log("not ready: number of outputs not set", "ERROR")
            ok = False
        if self._support_stage_idx is not None and self._support_stage_idx != self._n_iterations:
            self._log("the support stages do not add up to the number of iterations", "ERROR")
            ok = False
        if self._phasing_stage_idx is not None and self._phasing_stage_idx != self._n_iterations:
            self._log("the phasing stages do not add up to the number of iterations", "ERROR")
            ok = False
        if ok and not self._use_gpu:
            raise RuntimeError("use_gpu=False: this library runs phasing on the GPU only")
        return ok

    def _algorithms(self):
        """Phasing algorithms and support arrays with their schedules
        (src/_spimage_reconstructor.py:452-533): beta, blur and area schedules
        run from the algorithm's first to its last iteration."""
        lib = self._lib
        N = self._n_iterations
        sups, i = [], 0
        for conf in self._support_stages:
            n = conf["number_of_iterations"] if conf["number_of_iterations"] is not None else N
            period = conf.get("update_period")
            if conf["type"] == "area":
                a = lib.sp_support_area_alloc(smap({i: conf["blur_init"], i + n: conf["blur_final"]}),
                                              smap({i: conf["area_init"], i + n: conf["area_final"]}))
            elif conf["type"] == "threshold":
                a = lib.sp_support_threshold_alloc(smap({i: conf["blur_init"], i + n: conf["blur_final"]}),
                                                   smap({i: conf["threshold_init"], i + n: conf["threshold_final"]}))
            else:
                period = n
                a = lib.sp_support_static_alloc()
            arr = lib.sp_support_array_init(a, period)
            if conf["center_image"]:
                lib.sp_support_array_append(arr, lib.sp_support_centre_image_alloc())
            sups.append((arr, n))
            i += n
        algs, i = [], 0
        for conf in self._phasing_stages:
            n = conf["number_of_iterations"] if conf["number_of_iterations"] is not None else N
            c = phasing_constraints(conf.get("constraints", ""))
            if conf["type"] in ("raar", "hio", "diffmap"):
                beta = smap({i: conf["beta_init"], i + n: conf["beta_final"]})
            if conf["type"] == "raar":
                a = lib.sp_phasing_raar_alloc(beta, c)
            elif conf["type"] == "hio":
                a = lib.sp_phasing_hio_alloc(beta, c)
            elif conf["type"] == "diffmap":
                a = lib.sp_phasing_diff_map_alloc(beta, conf["gamma1"], conf["gamma2"], c)
            else:
                a = lib.sp_phasing_er_alloc(c)
            algs.append((a, n))
            i += n
        return algs, sups

    def _image(self, data, mask=None):
        img = new_image(np.asarray(data, np.complex64), mask)
        self._images.append(img)
        return img

    def _start(self, starts):
        """A phaser as the reference's _init_phaser (src/_spimage_reconstructor.py:535-551);
        several starts draw their phases one after another from the rand() stream."""
        self._lib = lib = load()
        self._free()
        algs, sups = self._algorithms()
        A = self._amplitudes
        M = self._mask if self._mask is not None else np.ones(A.shape, bool)
        amp = self._image(A, M.astype(np.int32))
        support = initial_support_mask(A.shape, **self._support_init_args)
        self._initial_support = support
        sup_img = self._image(support)
        ph = lib.sp_phaser_alloc()
        self._ph = ph
        if starts > 1 and lib.sp_phaser_set_starts(ph, starts) != 0:
            raise RuntimeError("sp_phaser_set_starts failed")
        rc = lib.sp_phaser_init(ph, algs[0][0], sups[0][0], SpEngineCUDA if self._use_gpu else SpEngineCPU)
        if rc != 0:
            raise RuntimeError(f"sp_phaser_init failed ({rc}): {lib.sp_phaser_last_error().decode()}")
        lib.sp_phaser_set_amplitudes(ph, amp)
        if starts > 1:
            rc = lib.sp_phaser_init_models(ph, SpModelRandomPhases, None)
        else:
            rc = lib.sp_phaser_init_model(ph, None, SpModelRandomPhases)
        if rc != 0:
            raise RuntimeError(f"initial model failed ({rc}): {lib.sp_phaser_last_error().decode()}")
        lib.sp_phaser_init_support(ph, sup_img, 0, 0.0)
        return algs, sups

    # ---------------------------------------------------------------- outputs
    def _fetch(self, fn, *args):
        img = fn(self._ph, *args)
        if not img:
            raise RuntimeError(self._lib.sp_phaser_last_error().decode())
        return img

    def _scores(self, starts):
        lib, ph = self._lib, self._ph
        if starts == 1:
            f = C.c_float()
            ef = lib.sp_phaser_efourier(ph, C.byref(f))
            return [{"fourier_error": float(ef), "FcFo": float(f.value), "real_error": float(lib.sp_phaser_ereal(ph)),
                     "support_size": float(lib.sp_phaser_support_fraction(ph))}]
        ef = np.zeros(starts, np.float32)
        fc = np.zeros(starts, np.float32)
        er = np.zeros(starts, np.float32)
        sf = np.zeros(starts, np.float32)
        fp = C.POINTER(C.c_float)
        lib.sp_phaser_starts_efourier(ph, ef.ctypes.data_as(fp), fc.ctypes.data_as(fp))
        lib.sp_phaser_starts_ereal(ph, er.ctypes.data_as(fp))
        lib.sp_phaser_starts_support_fraction(ph, sf.ctypes.data_as(fp))
        return [{"fourier_error": float(ef[b]), "FcFo": float(fc[b]), "real_error": float(er[b]),
                 "support_size": float(sf[b])} for b in range(starts)]

    def _start_image(self, fn, b, shape):
        img = new_image(np.zeros(shape, np.complex64))
        try:
            if fn(self._ph, b, img) != 0:
                raise RuntimeError(self._lib.sp_phaser_last_error().decode())
            return image_data(img, shape)
        finally:
            free_image(img)

    def _models(self, starts):
        """[real space, support] of every start, non-shifted (the reference's
        _get_curr_model, state before_projection, src/_spimage_reconstructor.py:749-769)"""
        lib, shape = self._lib, self._amplitudes.shape
        out = []
        for b in range(starts):
            if self._iteration > 0:
                if starts == 1:
                    img = image_data(self._fetch(lib.sp_phaser_model_before_projection), shape)
                    msk = np.int32(image_data(self._fetch(lib.sp_phaser_support), shape).real)
                else:
                    img = self._start_image(lib.sp_phaser_start_model_before_projection, b, shape)
                    msk = np.int32(self._start_image(lib.sp_phaser_start_support, b, shape).real)
            else:
                if starts == 1:
                    img = image_data(self._fetch(lib.sp_phaser_model), shape)
                else:
                    img = self._start_image(lib.sp_phaser_start_model, b, shape)
                msk = np.array(self._initial_support.real, dtype="bool")
            out.append([np.fft.fftshift(img), np.fft.fftshift(msk)])
        return out

    def _fmodels(self, starts):
        """[Fourier space, mask] of every start, non-shifted (_get_curr_fmodel)"""
        lib, shape = self._lib, self._amplitudes.shape
        fmsk = image_mask(self._fetch(lib.sp_phaser_amplitudes), shape)
        out = []
        for b in range(starts):
            if starts == 1:
                fimg = image_data(self._fetch(lib.sp_phaser_fmodel), shape)
            else:
                fimg = self._start_image(lib.sp_phaser_start_fmodel, b, shape)
            out.append([np.fft.fftshift(fimg), np.fft.fftshift(fmsk)])
        return out

    # --------------------------------------------------------------- running
    def _run(self, starts):
        """The reference's reconstruct loop (src/_spimage_reconstructor.py:553-675)
        for `starts` starts at once; returns one output dictionary per start."""
        algs, sups = self._start(starts)
        lib, ph = self._lib, self._ph
        N = self._n_iterations
        out_img = output_iterations(N, self._n_image_outputs)
        out_sco = output_iterations(N, self._n_score_outputs)
        shape = self._amplitudes.shape
        res = [{"real_space": np.zeros((len(out_img),) + shape, np.complex128),
                "support": np.zeros((len(out_img),) + shape, bool),
                "fourier_space": np.zeros((len(out_img),) + shape, np.complex128),
                "mask": np.zeros((len(out_img),) + shape, bool),
                "real_error": np.zeros(len(out_sco)), "fourier_error": np.zeros(len(out_sco)),
                "support_size": np.zeros(len(out_sco))} for _ in range(starts)]
        i_alg = i_sup = i_img = i_sco = 0
        it0_alg = it0_sup = propagated = 0
        for self._iteration in range(N + 1):
            it = self._iteration
            change_alg = it - it0_alg == algs[i_alg][1] and it != N
            change_sup = it - it0_sup == sups[i_sup][1] and it != N
            if not (change_alg or change_sup or it in out_img or it in out_sco):
                continue
            if it != 0:
                rc = lib.sp_phaser_iterate(ph, it - propagated)
                if rc != 0:
                    raise RuntimeError(f"sp_phaser_iterate failed ({rc}): {lib.sp_phaser_last_error().decode()}")
                propagated = it
            if change_alg:
                i_alg += 1
                it0_alg = it
                lib.sp_phaser_set_phasing_algorithm(ph, algs[i_alg][0])
            if change_sup:
                i_sup += 1
                it0_sup = it
                lib.sp_phaser_set_support_algorithm(ph, sups[i_sup][0])
            if it in out_img:
                for r, (m, f) in zip(res, zip(self._models(starts), self._fmodels(starts))):
                    r["real_space"][i_img], r["support"][i_img] = m
                    r["fourier_space"][i_img], r["mask"][i_img] = f
                i_img += 1
            if it in out_sco:
                for r, s in zip(res, self._scores(starts)):
                    r["fourier_error"][i_sco] = s["fourier_error"]
                    r["real_error"][i_sco] = s["real_error"]
                    r["support_size"][i_sco] = s["support_size"]
                i_sco += 1
        self._iteration = None
        for r in res:
            r["iteration_index_images"] = out_img
            r["iteration_index_scores"] = out_sco
        return res

    def reconstruct(self):
        """One reconstruction; the reference's output dictionary (images and
        scores at the output iterations, non-shifted)."""
        if not self._prepare():
            return None
        return self._run(1)[0]

    def reconstruct_loop(self, Nrepeats, full_output=False):
        """Nrepeats reconstructions from consecutive random starts, run together
        on the GPU; the final images and scores of each (the reference's
        reconstruct_loop, src/_spimage_reconstructor.py:677-740)."""
        if not self._prepare():
            return None
        res = self._run(Nrepeats)
        out = {"real_space_final": np.stack([r["real_space"][-1] for r in res]),
               "fourier_space_final": np.stack([r["fourier_space"][-1] for r in res]),
               "support_final": np.stack([r["support"][-1] for r in res]),
               "scores_final": {k: np.array([r[k][-1] for r in res])
                                for k in ("real_error", "fourier_error", "support_size")}}
        if full_output:
            out["single_outputs"] = res
        return out
