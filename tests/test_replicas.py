"""N > 1 host logic on CPU: two gloo ranks shard a set of reconstruction jobs,
run their share (on the CPU oracle -- no GPU here), gather the results and
reduce their times the way bench.py does for replicas."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_shard_is_a_partition_and_balanced():
    from libspimage_b200.replicas import shard

    fp = [4, 1, 9, 9, 2, 7, 3, 3, 1, 8]
    for world in (1, 2, 3, 4):
        parts = [shard(fp, world, r) for r in range(world)]
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(fp)))
        loads = [sum(fp[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(fp)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import oracle
    from libspimage_b200 import replicas, synth

    assert replicas.init("gloo", timeout_s=60)
    jobs = [(16, 16), (24, 24), (16, 24), (32, 32), (8, 8)]
    mine = replicas.shard([h * w for h, w in jobs], world, rank)
    results = {}
    for j in mine:
        shape = jobs[j]
        amp, mask, support, _ = synth.small_pattern(shape, seed=j)
        e = oracle.Restatement(shape)
        e.set_algorithm(oracle.HIO, beta=0.9, constraints=oracle.POS_REAL)
        e.set_amplitudes(amp, mask)
        e.init_model(oracle.RANDOM_PHASES, seed=100 + j)
        e.set_support(support)
        e.iterate(10)
        results[j] = e.efourier()[0]
    everything = replicas.gather(results)
    t = replicas.max_over_ranks(float(rank + 1))
    s = replicas.sum_over_ranks(1.0)
    if rank == 0:
        merged = {}
        for d in everything:
            merged.update(d)
        np.save(out_path, np.array([len(merged), t, s] + [merged[k] for k in sorted(merged)]))
    import torch.distributed as dist

    dist.destroy_process_group()


def test_two_gloo_ranks_shard_run_and_reduce(tmp_path, oracle_mod):
    import torch.multiprocessing as mp

    out = str(tmp_path / "res.npy")
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        assert p.exitcode == 0
    res = np.load(out)
    assert int(res[0]) == 5  # every job ran exactly once
    assert res[1] == 2.0  # max over ranks
    assert res[2] == 2.0  # sum over ranks
    # the same jobs on one process give the same errors
    import oracle
    from libspimage_b200 import synth

    jobs = [(16, 16), (24, 24), (16, 24), (32, 32), (8, 8)]
    for j, shape in enumerate(jobs):
        amp, mask, support, _ = synth.small_pattern(shape, seed=j)
        e = oracle.Restatement(shape)
        e.set_algorithm(oracle.HIO, beta=0.9, constraints=oracle.POS_REAL)
        e.set_amplitudes(amp, mask)
        e.init_model(oracle.RANDOM_PHASES, seed=100 + j)
        e.set_support(support)
        e.iterate(10)
        assert np.float32(e.efourier()[0]) == np.float32(res[3 + j])
