#!/usr/bin/env python
"""Benchmark of the phase-retrieval hot path; prints ONE JSON line.

Workload (default ``raar1024``): single-instance RAAR on a 1024x1024 FP32
pattern (256x256 blob smoothed by sigma 2, 1e8 photons, Poisson, beamstop
radius 8 px), 5000 RAAR iterations (beta 0.87, positive real object) with an
area support update every 50 iterations (area 0.05, blur radius 3.0 -> 0.7),
then 200 ER iterations.  One step = that whole reconstruction = 5200
``sp_phaser_iterate`` iteration slots (a support update uses a slot, as in the
reference).  Data are synthetic (seeded, ``libspimage_b200.synth``).

value  : iteration slots / s with the inputs resident in HBM, device-timed with
         CUDA events on the stream the kernels run on; L2 is flushed (256 MiB
         write) before every timed step, outside the events.
e2e    : the same metric through the C API with host buffers: set amplitudes,
         random-phase start (host RNG as the reference), support, iterate,
         read the model and the Fourier error back -- wall clock per step.
Multi-GPU (torchrun): independent replicas, one per GPU (the path has no
exchange step); value sums all ranks' slots over the slowest rank's time.

``--impl reference`` times the reference's own CPU engine (oracle/_ref, built
from the reference sources; the oracle restatement if that build is absent) on
the host cores, each step a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "HIO/RAAR iters/sec, batched & served vs plain, at equal Fourier error; p50/p99"
UNIT = "iterations/s"

WORKLOADS = {
    "raar1024": dict(
        pattern="raar1024", shape=(1024, 1024), stages=[("RAAR", 0.87, 5000), ("ER", None, 200)], period=50,
        area=0.05, blur={0: 3.0, 5000: 0.7}, constraints=2,
        desc="single-instance RAAR 1024x1024 FP32: 5000 RAAR (beta 0.87, area support every 50, area 0.05, "
             "blur 3.0->0.7) + 200 ER",
    ),
    "batch512": dict(
        pattern="batch512", shape=(512, 512), stages=[("HIO", 0.9, 2000), ("ER", None, 200)], period=20,
        area=0.05, blur={0: 3.0, 2200: 0.7}, constraints=2, starts=512,
        desc="batched random starts: 512 reconstructions of one 512x512 FP32 pattern (128x128 blob, 1e7 photons, "
             "beamstop 6 px), seeds 0..511, each 2000 HIO (beta 0.9) + 200 ER, area support every 20 (area 0.05, "
             "blur 3.0->0.7)",
    ),
    "hio256": dict(
        pattern="hio256", shape=(256, 256), stages=[("HIO", 0.9, 1000)], period=20, area=0.05,
        blur={0: 3.0, 1000: 0.7}, constraints=2,
        desc="plain HIO 256x256 FP32: 1000 HIO (beta 0.9, area support every 20, area 0.05, blur 3.0->0.7)",
    ),
    "hio1000": dict(
        pattern="hio1000", shape=(1000, 1000), stages=[("HIO", 0.9, 1000)], period=20, area=0.05,
        blur={0: 3.0, 1000: 0.7}, constraints=2,
        desc="plain HIO 1000x1000 FP32 (a job size of the mixed batch: 250 blob, 1e7 photons, beamstop 11.8 px): "
             "1000 HIO (beta 0.9, area support every 20, area 0.05, blur 3.0->0.7)",
    ),
    "vol128": dict(
        pattern="vol128", shape=(128, 128, 128), stages=[("HIO", 0.9, 1000)], period=20, area=0.05,
        blur={0: 3.0, 1000: 0.7}, constraints=2,
        desc="plain HIO 128^3 FP32 (the volume of the mixed batch and the serving mix: 32^3 blob, 1e8 photons, "
             "spherical beamstop 3 px): 1000 HIO (beta 0.9, area support every 20, area 0.05, blur 3.0->0.7)",
    ),
}

# launch-shape knobs of spb_ctx_set_tuning by name (--tune; they change no
# arithmetic): for timing and profiling the other kernel forms
TUNE_KNOBS = {"row_lines": 0, "no_pdl": 1, "row_g0": 2, "split": 3, "persist": 4, "col_width": 5, "tma": 6, "plane": 7,
              "select": 8}


def parse_tune(items):
    out = {}
    for it in items or []:
        k, _, v = it.partition("=")
        if k not in TUNE_KNOBS or not v.lstrip("-").isdigit():
            raise SystemExit(f"--tune {it}: expected one of {sorted(TUNE_KNOBS)}=<int>")
        out[k] = int(v)
    return out

# algorithmic HBM bytes per pixel of the dominant 2-D kernels (bit-packed
# support/measured masks): row pass reads Y + g_prev, writes g_new + X
# (+ support bit); column pass reads X + amplitudes, writes Y (+ measured bit)
ALGO_BYTES_PER_PIXEL = {"row_iter": 32.0 + 1.0 / 8, "col_project": 20.0 + 1.0 / 8}


def slots_per_step(wl):
    return sum(n for _, _, n in wl["stages"])


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms",
                 "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 8:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for name, v in zip(names, parts[4:8]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
        os.unlink(self.path)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ------------------------------------------------------------------ GPU arm
def build_phaser(L, wl, amp, mask, support, seed, starts=None, device_phases=False):
    """Phaser for the workload; with starts > 1 a batch whose start b gets
    device-drawn random phases keyed by seed + b."""
    ph = L.Phaser(wl["shape"])
    handles = []
    for name, beta, _ in wl["stages"]:
        alg = {"HIO": L.SpHIO, "RAAR": L.SpRAAR, "ER": L.SpER, "DM": L.SpDiffMap}[name]
        ph.set_algorithm(alg, beta=beta if beta is not None else 0.9, constraints=wl["constraints"])
        handles.append(ph.alg)
    ph.alg = handles[0]
    ph.add_support_update(L.SpSupportArea, wl["period"], wl["blur"], wl["area"])
    ph.start()
    ph.lib.sp_phaser_set_phasing_algorithm(ph.ph, handles[0])
    if starts is None:
        starts = wl.get("starts", 1)
    if starts > 1 or device_phases:
        ph.set_starts(starts)
        ph.set_amplitudes(amp, mask)
        rc = ph.init_models_device(L.SpModelRandomPhases, [seed + b for b in range(starts)])
    else:
        ph.set_amplitudes(amp, mask)
        rc = ph.init_model(L.SpModelRandomPhases, seed=seed)
    assert rc == 0, rc
    ph.set_support(support)
    return ph, handles


def run_stages(ph, handles, wl):
    for h, (_, _, nit) in zip(handles, wl["stages"]):
        ph.lib.sp_phaser_set_phasing_algorithm(ph.ph, h)
        rc = ph.iterate(nit)
        if rc:
            raise RuntimeError(f"sp_phaser_iterate returned {rc}: {ph.lib.sp_phaser_last_error().decode()}")


def gpu_arm(args):
    import torch
    import torch.distributed as dist

    import libspimage_b200 as L
    from libspimage_b200 import synth

    from libspimage_b200 import replicas

    world, rank, local = replicas.dist_env()
    torch.cuda.set_device(local)
    replicas.init("nccl", timeout_s=300)
    wl = WORKLOADS[args.workload]
    n = int(np.prod(wl["shape"]))
    amp, mask, support, _ = synth.workload(wl["pattern"], seed=0)
    L.load()
    ph, handles = build_phaser(L, wl, amp, mask, support, seed=rank)
    tune = parse_tune(args.tune)
    for k, v in tune.items():
        ph.set_tuning(TUNE_KNOBS[k], v)
    stream = torch.cuda.Stream()
    ph.set_stream(stream.cuda_stream)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MiB > L2

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        run_stages(ph, handles, wl)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    evs = []
    launches0 = ph.launch_count()
    for k in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(float(k))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run_stages(ph, handles, wl)
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    launches_total = ph.launch_count() - launches0
    clocks = sampler.stop()
    # one more step with a CUDA event pair around every kernel launch (direct
    # launches, no graphs) for the per-kernel durations of the roofline
    with torch.cuda.stream(stream):
        flush.fill_(-1.0)
    ph.profile(True)
    run_stages(ph, handles, wl)
    torch.cuda.synchronize()
    ktimes = ph.kernel_times()
    ph.profile(False)
    total_ms = replicas.max_over_ranks(float(sum(step_ms)), device="cuda")
    slots = slots_per_step(wl)
    starts = wl.get("starts", 1)
    value = world * args.steps * slots * starts / (total_ms / 1e3)

    # ---- end to end through the C API with host buffers
    ph.set_stream(None)
    del ph
    e2e_val, h2d, d2h, efour = e2e_run(args, L, wl, amp, mask, support, rank, world, torch, dist)

    # ---- roofline of the dominant kernel
    peak, peak_kind = measured_peak()
    dom = max(ktimes.items(), key=lambda kv: kv[1][1]) if ktimes else ("none", (0, 0.0))
    name, (launches, ms) = dom
    per_pixel = ALGO_BYTES_PER_PIXEL.get(name)
    roof = None
    if per_pixel and launches:
        avg_s = ms / launches / 1e3
        achieved = per_pixel * n * starts / avg_s / 1e9
        traffic = profiled_traffic(name, args.workload)
        # the profiled step launches each kernel directly between its own event
        # pair (no graphs, no dependent launch); in the timed, graph-replayed
        # step the same kernel's time is estimated as its share of the profiled
        # step's kernel time applied to the timed step's device time
        share = ms / sum(v[1] for v in ktimes.values())
        in_step_s = (total_ms / args.steps / 1e3) * share / launches
        roof = {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": traffic, "algorithmic_bytes_per_launch": per_pixel * n * starts,
                "avg_launch_us": round(avg_s * 1e6, 3),
                "in_step_us": round(in_step_s * 1e6, 3),
                "frac_in_step": round(per_pixel * n * starts / in_step_s / 1e9 / peak, 4),
                "note": "achieved/frac: event pair around each directly launched kernel; in_step: the timed "
                        "graph-replayed step's device time x this kernel's share of the profiled kernel time"}

    batched = None
    if args.batch_steps > 0:
        batched = batched_run(args, L, torch, world)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            batched["cpu_baseline"] = cpu_baseline(WORKLOADS["batch512"], args.cpu_sample_slots,
                                                   wl_name="batch512", use="ii")
            batched["cpu_baseline"]["note"] = ("independent starts on the host: one single-threaded reference "
                                               "engine per core, each on its own start (mode ii), aggregate "
                                               "start-iterations/s")

    mixed = mixed_run(args, L) if args.mixed_jobs > 0 else None
    serving = serving_run(args, L) if args.serve_window > 0 else None

    cpu = fp64 = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(wl, args.cpu_sample_slots, wl_name=args.workload, use="iii")
        fp64 = error_vs_fp64(args.workload)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": wl["desc"], "shape": list(wl["shape"]), "slots_per_step": slots,
                       "parallelism": f"replicas x{world}", "l2": "flushed (256 MiB write) before each timed step",
                       "efourier_final_e2e": efour, "error_vs_fp64": fp64, **({"tuning": tune} if tune else {})},
            "e2e": {"value": round(e2e_val, 2), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches_total),
            "kernels": {k: {"launches": v[0], "avg_us": round(v[1] / max(v[0], 1) * 1e3, 3)} for k, v in ktimes.items()},
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "batched": batched,
            "mixed": mixed,
            "serving": serving,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def timed_jobs(ph, handles, wl, steps, stream, torch):
    """Device time (ms) of `steps` whole jobs, CUDA events on the phaser's stream."""
    evs = []
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run_stages(ph, handles, wl)
        e1.record(stream)
        evs.append((e0, e1))
    torch.cuda.synchronize()
    return float(sum(a.elapsed_time(b) for a, b in evs))


def batched_run(args, L, torch, world):
    """Batched random starts (512 starts of 512x512) against the plain
    single-start path on the same pattern and schedule; start 0 of the batch
    and the plain run begin from the same device-drawn phases, so their final
    Fourier errors must agree."""
    import ctypes as C

    from libspimage_b200 import replicas, synth

    wl = dict(WORKLOADS["batch512"])
    if args.batch_starts:  # a smaller batch of the same job (profiling captures)
        wl["starts"] = args.batch_starts
    nb = wl["starts"]
    n = int(np.prod(wl["shape"]))
    slots = slots_per_step(wl)
    amp, mask, support, _ = synth.workload(wl["pattern"], seed=0)
    stream = torch.cuda.Stream()
    out = {"workload": wl["desc"], "starts": nb, "unit": "start-iterations/s", "steps": args.batch_steps,
           "warmup": f"{args.batch_warm_slots} iteration slots (kernel warm-up and graph capture)",
           "init": "random phases drawn on the device (Philox4x32-10, seeds 0..511)",
           "l2": "inputs larger than L2 (8 GB of iterates)"}
    res = {}
    for label, starts in (("batched", nb), ("plain", 1)):
        ph, handles = build_phaser(L, wl, amp, mask, support, seed=0, starts=starts, device_phases=True)
        ph.set_stream(stream.cuda_stream)
        rc = ph.iterate(args.batch_warm_slots)
        assert rc == 0, rc
        torch.cuda.synchronize()
        l0 = ph.launch_count()
        ms = timed_jobs(ph, handles, wl, args.batch_steps, stream, torch)
        launches = ph.launch_count() - l0
        ms = replicas.max_over_ranks(ms, device="cuda")
        if starts > 1:
            ef, _ = ph.starts_efourier()
            e0 = float(ef[0])
            # then one support period with a CUDA event pair around every
            # launch (direct launches) for the per-kernel rooflines
            ph.profile(True)
            assert ph.iterate(wl["period"]) == 0
            torch.cuda.synchronize()
            ktimes = ph.kernel_times()
            ph.profile(False)
        else:
            e0 = ph.efourier()[0]
        res[label] = (ms, launches, e0)
        ph.set_stream(None)
        ph.close()
        del ph
        torch.cuda.empty_cache()
    bms, blaunch, bef = res["batched"]
    pms, _, pef = res["plain"]
    out["value"] = round(world * args.batch_steps * slots * nb / (bms / 1e3), 1)
    out["ms_per_step"] = round(bms / args.batch_steps, 3)
    out["gpu_launches"] = int(blaunch)
    out["plain"] = {"value": round(world * args.batch_steps * slots / (pms / 1e3), 1), "unit": "iterations/s",
                    "ms_per_step": round(pms / args.batch_steps, 3),
                    "config": "the same job for one start (the batch's start 0), same pattern and schedule"}
    out["speedup_vs_plain"] = round(out["value"] / out["plain"]["value"], 3)
    out["efourier_final"] = {"batched_start0": bef, "plain": pef, "equal": bef == pef}
    # HBM roofline: algorithmic bytes of each pass kernel over its live launch
    # time, and of a whole iteration (support updates included) over the
    # timed iteration rate
    peak, peak_kind = measured_peak()
    per_start = n * nb
    kern = {}
    for name, (nl, kms) in ktimes.items():
        per_pixel = ALGO_BYTES_PER_PIXEL.get(name)
        if per_pixel and nl:
            avg_s = kms / nl / 1e3
            tr = profiled_traffic(name, "batch512")
            kern[name] = {"achieved": round(per_pixel * per_start / avg_s / 1e9, 1),
                          "frac": round(per_pixel * per_start / avg_s / 1e9 / peak, 4),
                          "avg_launch_us": round(avg_s * 1e6, 2),
                          "algorithmic_bytes_per_launch": per_pixel * per_start,
                          "traffic": tr * nb if tr else None}
    it_s = bms / 1e3 / (args.batch_steps * slots)
    it_bytes = sum(ALGO_BYTES_PER_PIXEL.values()) * per_start
    dom = max(kern.items(), key=lambda kv: kv[1]["avg_launch_us"]) if kern else None
    out["roofline"] = {"bound": "hbm", "kernel": dom[0] if dom else None,
                       "achieved": dom[1]["achieved"] if dom else None, "peak": peak, "unit": "GB/s",
                       "frac": dom[1]["frac"] if dom else None,
                       "traffic": dom[1]["traffic"] if dom else None,
                       "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)", "kernels": kern,
                       "iteration": {"algorithmic_bytes": it_bytes, "ms": round(it_s * 1e3, 4),
                                     "achieved": round(it_bytes / it_s / 1e9, 1),
                                     "frac": round(it_bytes / it_s / 1e9 / peak, 4),
                                     "note": "whole batch iteration incl. amortised support updates"}}

    # end to end through the C API with host buffers: amplitudes, mask and
    # support up, device-drawn starts, the whole job, every start's model and
    # Fourier error down
    ph, handles = build_phaser(L, wl, amp, mask, support, seed=0, starts=nb)
    amp_img = L.new_image(np.asarray(amp, np.complex64), mask)
    sup_img = L.new_image(np.asarray(support, np.complex64))
    model_img = L.new_image(np.zeros(wl["shape"], np.complex64))
    lib = ph.lib
    seeds = np.arange(nb, dtype=np.uint64)
    efs = np.zeros(nb, np.float32)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(args.batch_e2e_steps):
        lib.sp_phaser_set_amplitudes(ph.ph, amp_img)
        assert lib.sp_phaser_init_models_device(ph.ph, L.SpModelRandomPhases,
                                                (seeds + 1000 * k).ctypes.data_as(C.POINTER(C.c_ulonglong))) == 0
        assert lib.sp_phaser_init_support(ph.ph, sup_img, 0, 0.0) == 0
        run_stages(ph, handles, wl)
        for b in range(nb):
            assert lib.sp_phaser_start_model(ph.ph, b, model_img) == 0
        assert lib.sp_phaser_starts_efourier(ph.ph, efs.ctypes.data_as(C.POINTER(C.c_float)), None) == 0
    dt = replicas.max_over_ranks(time.perf_counter() - t0, device="cuda")
    ph.close()
    for img in (amp_img, sup_img, model_img):
        L.free_image(img)
    out["e2e"] = {"value": round(world * args.batch_e2e_steps * slots * nb / dt, 1), "unit": "start-iterations/s",
                  "steps": args.batch_e2e_steps, "h2d_bytes_per_step": 4 * n + n + 8 * n + 8 * nb,
                  "d2h_bytes_per_step": 8 * n * nb + 4 * nb}
    return out


# ------------------------------------------------ mixed batch and serving
SERVE_SIZES = [((128, 128), 0.30), ((256, 256), 0.30), ((512, 512), 0.20), ((1024, 1024), 0.15),
               ((128, 128, 128), 0.05)]
MIXED_SIZES = [(128, 128), (192, 192), (256, 256), (384, 384), (512, 512), (1000, 1000)]
HIO_, RAAR_, DM_, ER_ = 1, 2, 3, 4


class PatternCache:
    """A few seeded synthetic patterns per shape (a job reuses one of them;
    its random starting phases come from its own seed)."""

    def __init__(self, variants=2):
        self.variants = variants
        self.cache = {}

    def get(self, shape, k):
        from libspimage_b200 import synth

        key = (tuple(shape), k % self.variants)
        if key not in self.cache:
            if len(shape) == 3:
                amp, mask, sup, _ = synth.make_pattern(shape, 32, 1e8, 3, seed=key[1])
            else:
                n = shape[0]
                amp, mask, sup, _ = synth.make_pattern(shape, n // 4, 1e7, n / 85.0, seed=key[1])
            self.cache[key] = (amp, mask, (sup != 0).astype(np.int32))
        return self.cache[key]


def _pct(xs, q):
    return float(np.percentile(np.asarray(xs, np.float64), q)) if len(xs) else None


def run_jobs(srv, jobs, arrivals, patterns):
    """Submits job k at arrivals[k] seconds (relative to the first), waits for
    all; returns per-job (submit, admit, finish, start-slots) on the server clock."""
    ids = []
    t0 = time.perf_counter()
    for k, job in enumerate(jobs):
        dt = arrivals[k] - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        amp, mask, sup = patterns.get(job["shape"], job["pattern"])
        ids.append(srv.submit(amp, mask, sup, job["stages"], starts=job["starts"], seed=job["seed"],
                              support_period=job["period"], area=0.05, blur=(3.0, 0.7)))
    out = []
    for jid, job in zip(ids, jobs):
        info = srv.wait(jid)
        if info["status"] != 0:
            raise RuntimeError(f"job {jid} failed: {srv.job_error(jid)}")
        srv.result(jid)
        out.append((info["t_submit"], info["t_admit"], info["t_finish"], job["starts"] * info["slots"]))
    return out


def summarise(rows):
    sub = np.array([r[0] for r in rows])
    adm = np.array([r[1] for r in rows])
    fin = np.array([r[2] for r in rows])
    lat = fin - sub
    span = float(fin.max() - sub.min())
    return {"jobs": len(rows), "makespan_s": round(span, 4), "jobs_per_s": round(len(rows) / span, 3),
            "start_iterations_per_s": round(sum(r[3] for r in rows) / span, 1),
            "latency_p50_s": round(_pct(lat, 50), 4), "latency_p99_s": round(_pct(lat, 99), 4),
            "queue_wait_p50_s": round(_pct(adm - sub, 50), 4), "queue_wait_p99_s": round(_pct(adm - sub, 99), 4)}


def tune_alone(Server, warm, patterns):
    """Runs the warm-up jobs one at a time: the server tunes the launch shapes
    of every new (shape, starts, algorithm) on its first job, and the choice
    is cached for the process -- timed with the GPU otherwise idle rather
    than beside the other jobs of a concurrent warm-up."""
    with Server(max_active_jobs=1, chunk_slots=100) as srv:
        run_jobs(srv, warm, [0.0] * len(warm), patterns)


def mixed_run(args, L):
    """Uneven mixed batch: single-start jobs of 2-D sizes drawn from
    {128, 192, 256, 384, 512, 1000}^2 with a random algorithm and beta, plus
    eight 128^3 volumes, 1000 iteration slots each, all submitted at once;
    against the same jobs run one at a time."""
    from libspimage_b200.serve import Server

    rng = np.random.default_rng(0)
    jobs = []
    for k in range(args.mixed_jobs):
        shape = MIXED_SIZES[rng.integers(len(MIXED_SIZES))]
        alg = int(rng.integers(1, 5))
        beta = float(rng.uniform(0.7, 0.95))
        jobs.append({"shape": shape, "stages": [(alg, beta, 1000)], "starts": 1, "seed": k, "period": 20,
                     "pattern": k})
    for k in range(8):
        alg = int(rng.integers(1, 5))
        jobs.append({"shape": (128, 128, 128), "stages": [(alg, float(rng.uniform(0.7, 0.95)), 1000)], "starts": 1,
                     "seed": 10000 + k, "period": 20, "pattern": k})
    patterns = PatternCache()
    for j in jobs:
        patterns.get(j["shape"], j["pattern"])
    res = {}
    # warm-up: one short job per shape and algorithm (launch-shape tuning,
    # module loading, graph capture)
    warm = [{"shape": sh, "stages": [(a, 0.9, 40)], "starts": 1, "seed": 0, "period": 20, "pattern": 0}
            for sh in MIXED_SIZES + [(128, 128, 128)] for a in (1, 2, 3, 4)]
    tune_alone(Server, warm, patterns)
    for label, active in (("concurrent", args.max_active_jobs), ("one_at_a_time", 1)):
        with Server(max_active_jobs=active, chunk_slots=100) as srv:
            run_jobs(srv, warm, [0.0] * len(warm), patterns)
            rows = run_jobs(srv, jobs, [0.0] * len(jobs), patterns)
            res[label] = summarise(rows)
            res[label]["server"] = srv.stats()
    out = {"workload": f"{args.mixed_jobs} single-start 2-D jobs, sizes U{{128,192,256,384,512,1000}}^2, algorithm "
                       "U{ER,HIO,RAAR,DM}, beta U[0.7,0.95], plus 8 x 128^3; 1000 iteration slots each, area "
                       "support every 20; all submitted at t=0",
           "unit": "start-iterations/s", "value": res["concurrent"]["start_iterations_per_s"],
           "concurrent": res["concurrent"], "one_at_a_time": res["one_at_a_time"],
           "speedup_vs_one_at_a_time": round(res["one_at_a_time"]["makespan_s"] / res["concurrent"]["makespan_s"], 3),
           "patterns": "2 seeded synthetic patterns per shape; phases from each job's seed (device Philox)"}
    return out


def serving_run(args, L):
    """Serving: Poisson arrivals of 8-start jobs (1000 HIO + 100 ER, area
    support every 20), sizes 128^2 .30, 256^2 .30, 512^2 .20, 1024^2 .15,
    128^3 .05, admitted as slots and memory free up; latency = finish - arrival."""
    from libspimage_b200.serve import Server

    patterns = PatternCache()
    for sh, _ in SERVE_SIZES:
        patterns.get(sh, 0)
        patterns.get(sh, 1)
    probs = np.array([w for _, w in SERVE_SIZES])

    def make_jobs(rate, window, seed):
        rng = np.random.default_rng(seed)
        t, arr, jobs = 0.0, [], []
        while True:
            t += rng.exponential(1.0 / rate)
            if t > window:
                break
            sh = SERVE_SIZES[rng.choice(len(SERVE_SIZES), p=probs)][0]
            arr.append(t)
            jobs.append({"shape": sh, "stages": [(HIO_, 0.9, 1000), (ER_, 0.0, 100)], "starts": 8,
                         "seed": 8 * len(jobs), "period": 20, "pattern": len(jobs)})
        return jobs, arr

    out = {"workload": f"Poisson arrivals at {args.serve_rate:g}/s for {args.serve_window:g} s (the stated window is 60 s; "
                       "reduced so that the benchmark run stays within minutes: at this overload the queue, and "
                       "with it the latency, grows linearly with the window); 8 starts x (1000 HIO beta 0.9 + "
                       "100 ER) per job, area support every 20; sizes 128^2 .30, 256^2 .30, 512^2 .20, "
                       "1024^2 .15, 128^3 .05",
           "unit": "jobs/s", "max_active_jobs": args.max_active_jobs}
    warm, _ = make_jobs(50.0, 0.2, 99)
    warm = [dict(j, stages=[(HIO_, 0.9, 40), (ER_, 0.0, 10)]) for j in warm]
    warm += [{"shape": sh, "stages": [(HIO_, 0.9, 40), (ER_, 0.0, 10)], "starts": 8, "seed": 0, "period": 20,
              "pattern": 0} for sh, _ in SERVE_SIZES]
    tune_alone(Server, [{"shape": sh, "stages": [(HIO_, 0.9, 40), (ER_, 0.0, 10)], "starts": 8, "seed": 0,
                         "period": 20, "pattern": 0} for sh, _ in SERVE_SIZES], patterns)
    with Server(max_active_jobs=args.max_active_jobs, chunk_slots=100) as srv:
        run_jobs(srv, warm, [0.0] * len(warm), patterns)
        # offered load at the configured rate (far above capacity): queueing-dominated
        jobs, arr = make_jobs(args.serve_rate, args.serve_window, 0)
        over = summarise(run_jobs(srv, jobs, arr, patterns))
        over["offered_jobs_per_s"] = args.serve_rate
        over["window_s"] = args.serve_window
        # a rate the server sustains: 70% of the throughput it reached above
        rate = 0.7 * over["jobs_per_s"]
        jobs, arr = make_jobs(rate, args.serve_sustained_window, 1)
        sus = summarise(run_jobs(srv, jobs, arr, patterns))
        sus["offered_jobs_per_s"] = round(rate, 3)
        sus["window_s"] = args.serve_sustained_window
        out["server"] = srv.stats()
    out["overload"] = over
    out["sustained"] = sus
    out["value"] = over["jobs_per_s"]
    out["latency_p50_s"] = sus["latency_p50_s"]
    out["latency_p99_s"] = sus["latency_p99_s"]
    return out


def e2e_run(args, L, wl, amp, mask, support, rank, world, torch, dist):
    """Full user flow per step with host inputs; wall clock, max over ranks."""
    import ctypes as C

    from libspimage_b200 import replicas

    n = int(np.prod(wl["shape"]))
    ph = L.Phaser(wl["shape"])
    handles = []
    for name, beta, _ in wl["stages"]:
        alg = {"HIO": L.SpHIO, "RAAR": L.SpRAAR, "ER": L.SpER, "DM": L.SpDiffMap}[name]
        ph.set_algorithm(alg, beta=beta if beta is not None else 0.9, constraints=wl["constraints"])
        handles.append(ph.alg)
    ph.add_support_update(L.SpSupportArea, wl["period"], wl["blur"], wl["area"])
    ph.start()
    amp_img = L.new_image(np.asarray(amp, np.complex64), mask)
    sup_img = L.new_image(np.asarray(support, np.complex64))
    # user's input buffers live in pinned host memory
    cudart = torch.cuda.cudart()
    pinned = []
    for img in (amp_img, sup_img):
        for ptr, nbytes in ((img.contents.image.contents.data, 8 * n), (img.contents.mask.contents.data, 4 * n)):
            if cudart.cudaHostRegister(ptr, nbytes, 0) == 0:
                pinned.append(ptr)
    lib = ph.lib
    fc = C.c_float()
    times, efour = [], None

    def one(seed):
        lib.sp_phaser_set_amplitudes(ph.ph, amp_img)
        lib.sp_srand(seed)
        assert lib.sp_phaser_init_model(ph.ph, None, L.SpModelRandomPhases) == 0
        assert lib.sp_phaser_init_support(ph.ph, sup_img, 0, 0.0) == 0
        run_stages(ph, handles, wl)
        m = lib.sp_phaser_model(ph.ph)
        assert m
        return float(lib.sp_phaser_efourier(ph.ph, C.byref(fc)))

    for w in range(args.warmup):
        one(1000 + w)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    for k in range(args.steps):
        t0 = time.perf_counter()
        efour = one(rank * 1000 + k)
        times.append(time.perf_counter() - t0)
    total = replicas.max_over_ranks(float(sum(times)), device="cuda")
    for ptr in pinned:
        cudart.cudaHostUnregister(ptr)
    ph.close()
    L.free_image(amp_img)
    L.free_image(sup_img)
    slots = slots_per_step(wl)
    # per step up: amplitudes (4N), pixel flags (1N, once: measured and support
    # bits together), the random-phase start's float phases (4N); down: model (8N)
    h2d = 4 * n + n + 4 * n
    d2h = 8 * n + 4 * 8
    return world * args.steps * slots / total, h2d, d2h, efour


def profiled_traffic(kernel, workload):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            parts = line.split()
            if len(parts) == 3 and not line.startswith("#") and parts[0] == workload and parts[1] == kernel:
                return int(parts[2])
    return None


# ------------------------------------------------------------- CPU engines
def cpu_engine(shape, threads):
    import oracle

    if oracle.ref_available():
        return oracle.Reference(shape, threads=threads), "reference"
    return oracle.Restatement(shape, threads=threads), "port"


def cpu_setup(wl, threads, seed=0):
    import oracle
    from libspimage_b200 import synth

    amp, mask, support, _ = synth.workload(wl["pattern"], seed=0)
    e, kind = cpu_engine(wl["shape"], threads)
    name, beta, _ = wl["stages"][0]
    alg = {"HIO": oracle.HIO, "RAAR": oracle.RAAR, "ER": oracle.ER, "DM": oracle.DIFFMAP}[name]
    e.set_algorithm(alg, beta=beta, constraints=wl["constraints"])
    e.add_support_update(oracle.SUP_AREA, wl["period"], wl["blur"], wl["area"])
    if hasattr(e, "start"):
        e.start()
    e.set_amplitudes(amp, mask)
    e.init_model(oracle.RANDOM_PHASES, seed=seed)
    e.set_support(support)
    return e, kind


def cpu_sample_rate(wl, threads, sample_slots, seed=0):
    """Iteration slots per second of one CPU engine with `threads` FFT threads
    over `sample_slots` slots of the workload's first stage."""
    e, kind = cpu_setup(wl, threads, seed=seed)
    t0 = time.perf_counter()
    e.iterate(sample_slots)
    return sample_slots / (time.perf_counter() - t0), kind


def cpu_worker(args):
    """One single-threaded CPU engine of the per-core throughput mode: waits
    for the common start signal (a line on stdin), times its sample and prints
    {"slots": ..., "seconds": ...}."""
    wl = WORKLOADS[args.cpu_worker]
    e, kind = cpu_setup(wl, 1, seed=args.cpu_worker_seed)
    sys.stdin.readline()
    t0 = time.perf_counter()
    e.iterate(args.cpu_sample_slots)
    print(json.dumps({"slots": args.cpu_sample_slots, "seconds": time.perf_counter() - t0, "kind": kind}), flush=True)


def cpu_per_core(wl_name, procs, sample_slots):
    """Mode (ii): one independent single-threaded engine per host core (the
    reference's FFTW planner is not thread-safe, so throughput on many cores
    means many processes), each on its own start; aggregate slots/s over the
    slowest process's timed span."""
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-worker", wl_name, "--cpu-sample-slots", str(sample_slots)]
    ps = [subprocess.Popen(cmd + ["--cpu-worker-seed", str(k)], stdin=subprocess.PIPE, stdout=subprocess.PIPE,
                           stderr=subprocess.DEVNULL, text=True) for k in range(procs)]
    time.sleep(0.5)
    for p in ps:  # all set up (imports, pattern, start); release them together
        p.stdin.write("go\n")
        p.stdin.flush()
    outs = [json.loads(p.communicate(timeout=600)[0].strip().splitlines()[-1]) for p in ps]
    slowest = max(o["seconds"] for o in outs)
    return sum(o["slots"] for o in outs) / slowest, outs[0]["kind"]


def cpu_modes(wl_name, sample_slots, per_core_slots):
    """The reference CPU engine in three modes on this host: (i) one job,
    one thread (the reference default: sp_init_fft not called); (ii) one
    single-threaded job per core, aggregate; (iii) one job with
    sp_init_fft(cores)."""
    wl = WORKLOADS[wl_name]
    cores = os.cpu_count() or 1
    single, kind = cpu_sample_rate(wl, 1, max(1, sample_slots // 4))
    per_core, _ = cpu_per_core(wl_name, cores, per_core_slots)
    threaded, _ = cpu_sample_rate(wl, cores, sample_slots)
    return {"i_single_thread": round(single, 3), "ii_per_core_aggregate": round(per_core, 3),
            "iii_one_job_all_threads": round(threaded, 3), "cores": cores, "kind": kind,
            "fft": "FFTW3 API served by the oracle CPU FFT (no libfftw3f on the box)",
            "samples": f"(i) {max(1, sample_slots // 4)} slots, (ii) {per_core_slots} slots per process x {cores}, "
                       f"(iii) {sample_slots} slots; first stage ({wl['stages'][0][0]}) of the same workload, "
                       "support updates included"}


def cpu_baseline(wl, sample_slots, wl_name="raar1024", per_core_slots=40, use="iii"):
    m = cpu_modes(wl_name, sample_slots, per_core_slots)
    key = {"i": "i_single_thread", "ii": "ii_per_core_aggregate", "iii": "iii_one_job_all_threads"}[use]
    return {"value": m[key], "unit": UNIT, "cores": m["cores"] if use != "i" else 1, "kind": m["kind"],
            "mode": key, "modes": m,
            "sample": m["samples"] + "; " + m["fft"]}


def error_vs_fp64(wl_name, iterations=10):
    """Relative L2 error of the float32 model after `iterations` slots against
    the FP64 restatement (oracle/fp64.py) from the same start.  The float32
    engine here is the oracle restatement, whose iterates the GPU library
    reproduces bit for bit (parity tests), so the figure is the GPU's."""
    import oracle
    from oracle.fp64 import Fp64Phaser, efourier64, rel_l2
    from libspimage_b200 import synth

    wl = WORKLOADS[wl_name]
    amp, mask, support, _ = synth.workload(wl["pattern"], seed=0)
    e = oracle.Restatement(wl["shape"], threads=os.cpu_count() or 1)
    f = Fp64Phaser(wl["shape"])
    name, beta, _ = wl["stages"][0]
    alg = {"HIO": oracle.HIO, "RAAR": oracle.RAAR, "ER": oracle.ER, "DM": oracle.DIFFMAP}[name]
    for eng in (e, f):
        eng.set_algorithm(alg, beta=beta, constraints=wl["constraints"])
        eng.add_support_update(oracle.SUP_AREA, wl["period"], wl["blur"], wl["area"])
    e.set_amplitudes(amp, mask)
    e.init_model(oracle.RANDOM_PHASES, seed=0)
    e.set_support(support)
    f.set_amplitudes(amp, mask)
    f.set_flags(e.flags())
    f.set_model(e.model())
    e.iterate(iterations)
    f.iterate(iterations)
    ef32, ef64 = efourier64(e.model(), amp, e.flags())[0], f.efourier()[0]
    return {"iterations": iterations, "model_rel_l2": float(f"{rel_l2(e.model(), f.model()):.3e}"),
            "efourier_rel": float(f"{abs(ef32 - ef64) / ef64:.3e}"),
            "note": "float32 result (bit-identical on GPU and reference engine) vs FP64 restatement, same start; "
                    "both Fourier errors summed in float64"}


def reference_arm(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    wl = WORKLOADS[args.workload]
    threads = os.cpu_count() or 1
    e, kind = cpu_setup(wl, threads)
    sample = args.cpu_sample_slots
    for _ in range(args.warmup):
        e.iterate(max(1, sample // 10))
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e.iterate(sample)
        times.append(time.perf_counter() - t0)
    total = float(sum(times))
    value = args.steps * sample / total
    modes = cpu_modes(args.workload, sample, 40)
    ref_gpu = reference_cuda_engine(wl, args.workload)
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total / args.steps * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": wl["desc"], "shape": list(wl["shape"]),
                   "step": f"bounded sample: {sample} iteration slots of the first stage per step"},
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{sample} iteration slots per step, FFT threads = cores, FFTW3 API served by "
                                   "the oracle CPU FFT (no libfftw3f on the box)",
                         "mode": "iii_one_job_all_threads", "modes": modes},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cuda_engine": ref_gpu,
    }
    print(json.dumps(line), flush=True)


def reference_cuda_engine(wl, wl_name, slots=520):
    """The reference's own CUDA engine (its phasing.cu kernels over cuFFT,
    cuRAND and thrust, compiled for sm_100a into oracle/_ref) on a bounded
    sample of the same workload on GPU 0: a second baseline beside the CPU
    engine.  Wall clock with the device synchronised (the engine works on the
    legacy default stream and synchronises inside its support updates)."""
    import oracle

    if not oracle.ref_cuda_available():
        return {"unavailable": "oracle/_ref/libspref_cuda.so is not built (needs the reference sources and nvcc)"}
    try:
        import torch

        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
        from libspimage_b200 import synth

        amp, mask, support, _ = synth.workload(wl["pattern"], seed=0)
        e = oracle.ReferenceCuda(wl["shape"])
        name, beta, _ = wl["stages"][0]
        e.set_algorithm({"HIO": oracle.HIO, "RAAR": oracle.RAAR, "ER": oracle.ER, "DM": oracle.DIFFMAP}[name],
                        beta=beta if beta is not None else 0.9, constraints=wl["constraints"])
        e.add_support_update(oracle.SUP_AREA, wl["period"], wl["blur"], wl["area"])
        if e.start() != 0:
            return {"unavailable": "sp_phaser_init with the reference's CUDA engine failed"}
        e.set_amplitudes(amp, mask)
        e.init_model(oracle.RANDOM_PHASES, seed=0)
        e.set_support(support)
        e.iterate(2 * wl["period"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = e.iterate(slots)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if rc != 0:
            return {"unavailable": f"the reference's CUDA engine returned {rc}"}
        return {"value": round(slots / dt, 3), "unit": UNIT, "us_per_slot": round(dt / slots * 1e6, 2),
                "sample": f"{slots} iteration slots of the first stage ({name}) of {wl_name}, support updates "
                          "included, after a warm-up of two support periods",
                "engine": "the reference's CUDA engine (src/phasing.cu, phasing_kernels.cu, support_update_cuda.cu, "
                          "image_filter_cuda.cu, fft.cu over cuFFT, cuRAND and thrust) compiled unmodified for sm_100a",
                "efourier_after": e.efourier()[0]}
    except Exception as ex:  # a baseline: report, do not fail the arm
        return {"unavailable": f"{type(ex).__name__}: {ex}"[:300]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="raar1024", choices=sorted(k for k in WORKLOADS if "starts" not in WORKLOADS[k]))
    ap.add_argument("--tune", action="append", default=[], metavar="KNOB=VALUE",
                    help=f"launch-shape knob of the headline phaser (repeatable): {', '.join(sorted(TUNE_KNOBS))}")
    ap.add_argument("--cpu-sample-slots", type=int, default=300)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-steps", type=int, default=2, help="timed whole jobs of the batched block (0: skip it)")
    ap.add_argument("--batch-warm-slots", type=int, default=60)
    ap.add_argument("--batch-starts", type=int, default=0, help="starts of the batched block (0: the workload's 512)")
    ap.add_argument("--batch-e2e-steps", type=int, default=1)
    ap.add_argument("--mixed-jobs", type=int, default=256, help="2-D jobs of the mixed batch (0: skip it)")
    ap.add_argument("--max-active-jobs", type=int, default=8,
                    help="server admission limit; mixed batch, start-iterations/s by limit on three boxes: "
                         "4/6/8: 67.9k/69.2k/63.6k; 8/12/16/24: 69.7k/63.1k/64.5k/50.9k; 16/32/64/96: 59.5k/56.5k/45.2k/50.3k")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="offered arrivals per second")
    ap.add_argument("--serve-window", type=float, default=3.0,
                    help="seconds of arrivals at --serve-rate (0: skip serving); the stated window is 60 s")
    ap.add_argument("--serve-sustained-window", type=float, default=5.0)
    ap.add_argument("--cpu-worker", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-worker-seed", type=int, default=0, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.cpu_worker:
        cpu_worker(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
