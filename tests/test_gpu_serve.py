"""Reconstruction server: jobs of different sizes and algorithms admitted as
they arrive and run side by side on one GPU.  Every job's result must be bit
for bit the result of the same schedule run alone through the SpPhaser API."""
import time

import numpy as np
import pytest

from libspimage_b200 import synth

pytestmark = pytest.mark.gpu

HIO, RAAR, DM, ER = 1, 2, 3, 4
AREA = 2


def _pattern(shape, seed=1):
    amp, mask, support, _ = synth.small_pattern(shape, seed=seed)
    return amp, mask, support


def run_alone(lib, shape, stages, starts, seed, period, area=0.05, blur=(3.0, 0.7), constraints=2, pseed=1):
    """The job's schedule through a Phaser of its own (reference for the server)."""
    amp, mask, support = _pattern(shape, pseed)
    slots = sum(n for _, _, n in stages)
    ph = lib.Phaser(shape)
    handles = []
    for alg, beta, _ in stages:
        ph.set_algorithm(alg, beta=beta, constraints=constraints)
        handles.append(ph.alg)
    ph.alg = handles[0]
    if period:
        ph.add_support_update(AREA, period, {0: blur[0], slots: blur[1]}, area)
    ph.start()
    ph.lib.sp_phaser_set_phasing_algorithm(ph.ph, handles[0])
    ph.set_starts(starts)
    ph.set_amplitudes(amp, mask)
    assert ph.init_models_device(1, [seed + b for b in range(starts)]) == 0
    ph.set_support(support)
    for h, (_, _, n) in zip(handles, stages):
        ph.lib.sp_phaser_set_phasing_algorithm(ph.ph, h)
        assert ph.iterate(n) == 0
    ef, _ = ph.starts_efourier()
    sf = ph.starts_support_fraction()
    models = np.stack([ph.start_model(b) for b in range(starts)])
    ph.close()
    return ef, sf, models


def submit(srv, shape, stages, starts, seed, period, pseed=1, keep=True):
    amp, mask, support = _pattern(shape, pseed)
    return srv.submit(amp, mask != 0, support, stages, starts=starts, seed=seed, support_period=period, area=0.05,
                      blur=(3.0, 0.7), keep_models=keep)


JOBS = [
    ((64, 64), [(HIO, 0.9, 60), (ER, 0.0, 10)], 3, 5, 20),
    ((48, 40), [(RAAR, 0.87, 45)], 2, 9, 15),
    ((16, 16, 16), [(HIO, 0.9, 30), (ER, 0.0, 10)], 2, 11, 10),
    ((32, 32), [(DM, 0.8, 25)], 2, 13, 0),
    ((128, 128), [(ER, 0.0, 40)], 1, 17, 20),
    ((64, 64), [(RAAR, 0.75, 50)], 2, 19, 20),
]


def _check(lib, res, shape, stages, starts, seed, period):
    ef, sf, models = run_alone(lib, shape, stages, starts, seed, period)
    assert np.array_equal(res["models"].view(np.uint32), models.view(np.uint32)), f"{shape} models differ"
    assert np.array_equal(res["efourier"], ef)
    assert np.array_equal(res["support_fraction"], sf)


def test_mixed_jobs_equal_alone(lib):
    from libspimage_b200.serve import Server

    with Server(max_active_jobs=3, chunk_slots=16, chunks_ahead=2) as srv:
        ids = [submit(srv, *j) for j in JOBS]
        for jid in ids:
            info = srv.wait(jid, timeout=120)
            assert info["status"] == 0, srv.job_error(jid)
        results = [srv.result(jid) for jid in ids]
        st = srv.stats()
    assert st["jobs_done"] == len(JOBS) and st["jobs_failed"] == 0
    assert st["peak_active_jobs"] <= 3
    for res, job in zip(results, JOBS):
        _check(lib, res, *job)


def test_short_jobs_overtake_a_long_one(lib):
    """continuous batching: jobs that arrive while a long job runs are admitted
    at once and finish before it"""
    from libspimage_b200.serve import Server

    with Server(max_active_jobs=4, chunk_slots=50) as srv:
        long_id = submit(srv, (512, 512), [(HIO, 0.9, 3000)], 8, 100, 20, keep=False)
        t0 = time.time()
        while srv.wait(long_id, timeout=0.01)["t_admit"] < 0 and time.time() - t0 < 30:
            pass
        short = [submit(srv, (32, 32), [(HIO, 0.9, 30)], 1, 200 + k, 10) for k in range(3)]
        infos = [srv.wait(j, timeout=120) for j in short]
        linfo = srv.wait(long_id, timeout=300)
        assert linfo["status"] == 0
        for inf in infos:
            assert inf["status"] == 0
            assert inf["t_admit"] < linfo["t_finish"]
            assert inf["t_finish"] < linfo["t_finish"]
        res = srv.result(short[1])
        srv.result(long_id)
    _check(lib, res, (32, 32), [(HIO, 0.9, 30)], 1, 201, 10)


def test_budget_serialises_admission(lib):
    from libspimage_b200.serve import Server, footprint

    shape, stages = (64, 64), [(HIO, 0.9, 40)]
    budget = 1.5 * footprint(shape, 2)
    with Server(hbm_budget_bytes=budget, max_active_jobs=8, chunk_slots=20) as srv:
        ids = [submit(srv, shape, stages, 2, 30 + 7 * k, 20) for k in range(3)]
        infos = [srv.wait(j, timeout=120) for j in ids]
        res = [srv.result(j) for j in ids]
        st = srv.stats()
    for a, b in zip(infos, infos[1:]):
        assert b["t_admit"] >= a["t_finish"]
    assert st["peak_active_jobs"] == 1
    assert st["contexts_created"] == 1 and st["contexts_reused"] == 2
    for k, r in enumerate(res):
        _check(lib, r, shape, stages, 2, 30 + 7 * k, 20)


def test_job_larger_than_budget_fails_cleanly(lib):
    from libspimage_b200.serve import Server, footprint

    with Server(hbm_budget_bytes=footprint((64, 64), 1) * 1.2, max_active_jobs=2) as srv:
        big = submit(srv, (64, 64), [(HIO, 0.9, 10)], 4, 1, 0)
        ok = submit(srv, (64, 64), [(HIO, 0.9, 10)], 1, 1, 0)
        assert srv.wait(big, timeout=60)["status"] < 0
        assert "budget" in srv.job_error(big)
        assert srv.wait(ok, timeout=60)["status"] == 0
        with pytest.raises(RuntimeError):
            srv.result(big)
        with pytest.raises(RuntimeError):
            srv.submit(np.ones((8, 8), np.float32), np.ones((8, 8)), np.ones((8, 8)), [(9, 0.9, 10)])


# ---- failure handling: a job that diverges, is cancelled or runs out of time
# ends with its own status while the server and the other jobs carry on

def test_nonfinite_job_fails_and_others_are_unaffected(lib):
    """NaN amplitudes make every model non-finite after the first chunk: the
    job ends as SPB_JOB_NONFINITE; the jobs beside it give their alone results
    and the server takes new work afterwards."""
    from libspimage_b200.serve import JOB_NONFINITE, Server

    good = [JOBS[0], JOBS[1]]
    with Server(max_active_jobs=3, chunk_slots=20) as srv:
        amp, mask, support = _pattern((64, 64), 1)
        bad_amp = amp.copy()
        bad_amp[3, 5] = np.nan
        bad = srv.submit(bad_amp, mask != 0, support, [(HIO, 0.9, 200)], starts=2, seed=3, support_period=20)
        ids = [submit(srv, *j) for j in good]
        info = srv.wait(bad, timeout=120)
        assert info["status"] == JOB_NONFINITE
        assert "NaN or infinite" in srv.job_error(bad)
        with pytest.raises(RuntimeError, match="NaN or infinite"):
            srv.result(bad)
        results = []
        for jid in ids:
            assert srv.wait(jid, timeout=120)["status"] == 0, srv.job_error(jid)
            results.append(srv.result(jid))
        later = submit(srv, *JOBS[5])
        assert srv.wait(later, timeout=120)["status"] == 0
        later_res = srv.result(later)
        st = srv.stats()
    assert st["jobs_failed"] == 1
    for res, job in zip(results, good):
        _check(lib, res, *job)
    _check(lib, later_res, *JOBS[5])


def test_cancel_pending_and_running_jobs(lib):
    from libspimage_b200.serve import JOB_CANCELLED, Server

    with Server(max_active_jobs=1, chunk_slots=50) as srv:
        long_id = submit(srv, (64, 64), [(HIO, 0.9, 400000)], 2, 7, 20, keep=False)
        queued = submit(srv, (64, 64), [(HIO, 0.9, 40)], 2, 8, 20)
        srv.cancel(queued)  # not admitted yet (one job at a time): ends at once
        qinfo = srv.wait(queued, timeout=5)
        assert qinfo["status"] == JOB_CANCELLED and qinfo["t_admit"] < 0
        t0 = time.time()
        while srv.wait(long_id, timeout=0.01)["t_admit"] < 0 and time.time() - t0 < 30:
            pass
        time.sleep(0.2)
        srv.cancel(long_id)
        info = srv.wait(long_id, timeout=60)
        assert info["status"] == JOB_CANCELLED
        assert info["t_finish"] - info["t_admit"] < 30
        assert srv.job_error(long_id) == "cancelled"
        with pytest.raises(RuntimeError, match="already ended"):
            srv.cancel(long_id)
        with pytest.raises(RuntimeError, match="unknown job"):
            srv.cancel(123456)
        # the cancelled job's context is reused by the next job of its shape
        nxt = submit(srv, (64, 64), [(HIO, 0.9, 40)], 2, 9, 20)
        assert srv.wait(nxt, timeout=60)["status"] == 0
        res = srv.result(nxt)
        st = srv.stats()
    assert st["contexts_reused"] >= 1 and st["contexts_created"] == 1
    _check(lib, res, (64, 64), [(HIO, 0.9, 40)], 2, 9, 20)


def test_time_budget_expires_running_and_pending_jobs(lib):
    from libspimage_b200.serve import JOB_EXPIRED, Server

    amp, mask, support = _pattern((64, 64), 1)
    with Server(max_active_jobs=1, chunk_slots=50) as srv:
        first = srv.submit(amp, mask != 0, support, [(HIO, 0.9, 400000)], starts=2, seed=1, support_period=20,
                           time_budget_s=0.5)
        waiting = srv.submit(amp, mask != 0, support, [(HIO, 0.9, 40)], starts=2, seed=2, support_period=20,
                             time_budget_s=0.001)
        tiny = None
        info = srv.wait(first, timeout=60)
        assert info["status"] == JOB_EXPIRED and "time budget" in srv.job_error(first)
        assert info["t_finish"] - info["t_submit"] < 30
        winfo = srv.wait(waiting, timeout=60)
        assert winfo["status"] == JOB_EXPIRED and winfo["t_admit"] < 0
        tiny = srv.submit(amp, mask != 0, support, [(HIO, 0.9, 40)], starts=2, seed=3, support_period=20)
        assert srv.wait(tiny, timeout=60)["status"] == 0
        srv.result(tiny)
