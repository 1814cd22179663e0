"""ctypes binding of the reconstruction server (include/spimage/serve.h).

    srv = Server(max_active_jobs=8)
    jid = srv.submit(amp, mask, support, stages=[(SpHIO, 0.9, 1000), (SpER, 0.0, 100)],
                     starts=8, seed=0, support_period=20, area=0.05, blur=(3.0, 0.7))
    info = srv.wait(jid)            # dict with status and timestamps
    res = srv.result(jid)           # efourier[starts], support_fraction[starts] (+ models)
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import load

MAX_STAGES = 4


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_double), ("max_active_jobs", C.c_int), ("chunk_slots", C.c_int),
                ("chunks_ahead", C.c_int), ("no_autotune", C.c_int)]


class JobStage(C.Structure):
    _fields_ = [("algorithm", C.c_int), ("beta", C.c_float), ("iterations", C.c_int)]


class Job(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("starts", C.c_int),
                ("amplitudes", C.POINTER(C.c_float)), ("mask", C.POINTER(C.c_int)), ("support", C.POINTER(C.c_int)),
                ("constraints", C.c_int), ("nstages", C.c_int), ("stage", JobStage * MAX_STAGES),
                ("support_period", C.c_int), ("support_area", C.c_float), ("blur_start", C.c_float),
                ("blur_end", C.c_float), ("seed", C.c_ulonglong), ("keep_models", C.c_int),
                ("time_budget_s", C.c_double)]

# spb_job_info.status (include/spimage/serve.h)
JOB_DONE, JOB_RUNNING, JOB_FAILED, JOB_CANCELLED, JOB_NONFINITE, JOB_EXPIRED = 0, 1, -1, -2, -3, -4


class JobInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("starts", C.c_int), ("slots", C.c_longlong), ("t_submit", C.c_double),
                ("t_admit", C.c_double), ("t_finish", C.c_double)]


def _bind(lib):
    if getattr(lib, "_serve_bound", False):
        return lib
    vp = C.c_void_p
    sig = {
        "spb_server_create": (C.c_int, [C.POINTER(vp), C.POINTER(ServerConfig)]),
        "spb_server_destroy": (None, [vp]),
        "spb_server_submit": (C.c_longlong, [vp, C.POINTER(Job)]),
        "spb_server_wait": (C.c_int, [vp, C.c_longlong, C.c_double, C.POINTER(JobInfo)]),
        "spb_server_cancel": (C.c_int, [vp, C.c_longlong]),
        "spb_server_result": (C.c_int, [vp, C.c_longlong, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                        C.POINTER(C.c_float)]),
        "spb_server_stats": (C.c_int, [vp, C.POINTER(C.c_double)]),
        "spb_server_last_error": (C.c_char_p, []),
        "spb_server_job_error": (C.c_char_p, [vp, C.c_longlong]),
        "spb_ctx_footprint": (C.c_longlong, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    lib._serve_bound = True
    return lib


def _shape3(shape):
    shape = tuple(int(s) for s in shape)
    if len(shape) == 2:
        return 1, shape[0], shape[1]
    return shape


class Server:
    """A running reconstruction server (one native worker thread)."""

    def __init__(self, hbm_budget_bytes=0.0, max_active_jobs=0, chunk_slots=0, chunks_ahead=0, autotune=True):
        self.lib = _bind(load())
        cfg = ServerConfig(float(hbm_budget_bytes), int(max_active_jobs), int(chunk_slots), int(chunks_ahead),
                           0 if autotune else 1)
        h = C.c_void_p()
        if self.lib.spb_server_create(C.byref(h), C.byref(cfg)) != 0:
            raise RuntimeError(self.lib.spb_server_last_error().decode())
        self.h = h
        self._shapes = {}

    def close(self):
        if self.h:
            self.lib.spb_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, amplitudes, mask, support, stages, starts=1, seed=0, constraints=2, support_period=0,
               area=0.05, blur=(3.0, 0.7), keep_models=False, time_budget_s=0.0):
        amp = np.ascontiguousarray(amplitudes, np.float32)
        m = np.ascontiguousarray(mask, np.int32)
        s = np.ascontiguousarray(support, np.int32)
        nz, ny, nx = _shape3(amp.shape)
        j = Job()
        j.nx, j.ny, j.nz, j.starts = nx, ny, nz, int(starts)
        j.amplitudes = amp.ctypes.data_as(C.POINTER(C.c_float))
        j.mask = m.ctypes.data_as(C.POINTER(C.c_int))
        j.support = s.ctypes.data_as(C.POINTER(C.c_int))
        j.constraints = int(constraints)
        j.nstages = len(stages)
        for i, (alg, beta, nit) in enumerate(stages):
            j.stage[i] = JobStage(int(alg), float(beta if beta is not None else 0.0), int(nit))
        j.support_period = int(support_period)
        j.support_area = float(area)
        j.blur_start, j.blur_end = float(blur[0]), float(blur[1])
        j.seed = int(seed)
        j.keep_models = 1 if keep_models else 0
        j.time_budget_s = float(time_budget_s)
        jid = self.lib.spb_server_submit(self.h, C.byref(j))
        if jid < 0:
            raise RuntimeError(self.lib.spb_server_last_error().decode())
        self._shapes[int(jid)] = (amp.shape, int(starts), bool(keep_models))
        return int(jid)

    def wait(self, jid, timeout=-1.0):
        info = JobInfo()
        if self.lib.spb_server_wait(self.h, jid, float(timeout), C.byref(info)) != 0:
            raise RuntimeError(self.lib.spb_server_last_error().decode())
        return {"status": info.status, "starts": info.starts, "slots": info.slots, "t_submit": info.t_submit,
                "t_admit": info.t_admit, "t_finish": info.t_finish}

    def cancel(self, jid):
        """Cancels a pending or running job (a running one stops at its next chunk boundary)."""
        if self.lib.spb_server_cancel(self.h, jid) != 0:
            raise RuntimeError(self.lib.spb_server_last_error().decode())

    def job_error(self, jid):
        return self.lib.spb_server_job_error(self.h, jid).decode()

    def result(self, jid):
        """Results of a finished job (releases it); raises for a job that ended with an error."""
        shape, starts, keep = self._shapes.pop(jid)
        ef = np.zeros(starts, np.float32)
        sf = np.zeros(starts, np.float32)
        models = np.zeros((starts,) + tuple(shape), np.complex64) if keep else None
        mp = models.ctypes.data_as(C.POINTER(C.c_float)) if keep else None
        rc = self.lib.spb_server_result(self.h, jid, ef.ctypes.data_as(C.POINTER(C.c_float)),
                                        sf.ctypes.data_as(C.POINTER(C.c_float)), mp)
        if rc != 0:
            raise RuntimeError(self.lib.spb_server_last_error().decode())
        out = {"efourier": ef, "support_fraction": sf}
        if keep:
            out["models"] = models
        return out

    def stats(self):
        a = (C.c_double * 8)()
        self.lib.spb_server_stats(self.h, a)
        keys = ["jobs_done", "start_slots_done", "peak_active_jobs", "peak_bytes", "contexts_created",
                "contexts_evicted", "contexts_reused", "jobs_failed"]
        return dict(zip(keys, list(a)))


def footprint(shape, starts, dm=False):
    lib = _bind(load())
    nz, ny, nx = _shape3(shape)
    return int(lib.spb_ctx_footprint(nx, ny, nz, int(starts), 1 if dm else 0))
