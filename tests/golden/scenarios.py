"""Golden scenarios: small phasing runs whose outputs were produced by the
reference's own CPU engine (oracle/_ref, built from the reference sources)
and stored as .npz fixtures by make_golden.py.  The same runner drives any
engine with the common interface (oracle.Reference, oracle.Restatement,
libspimage_b200.Phaser)."""
import numpy as np

HIO, RAAR, DIFFMAP, ER = 1, 2, 3, 4
THRESHOLD, AREA = 1, 2
POS_REAL, REAL, POS_COMPLEX = 2, 1, 4

SCENARIOS = {
    "hio_area_32": dict(shape=(32, 32), alg=HIO, beta=0.9, cons=POS_REAL, sup=[(AREA, 7, {0: 3.0, 60: 0.7}, 0.1)],
                        seed=5, iters=[40]),
    "raar_thr_32": dict(shape=(32, 32), alg=RAAR, beta=0.87, cons=POS_REAL, sup=[(THRESHOLD, 9, 2.0, 0.2)],
                        seed=6, iters=[25, 15]),
    "er_32x24": dict(shape=(24, 32), alg=ER, beta=0.9, cons=REAL, sup=None, seed=7, iters=[20]),
    "dm_area_32": dict(shape=(32, 32), alg=DIFFMAP, beta=0.9, cons=POS_REAL, sup=[(AREA, 10, 2.0, 0.12)], seed=8,
                       iters=[30]),
    "hio_3d_8": dict(shape=(8, 8, 8), alg=HIO, beta=0.8, cons=POS_REAL, sup=[(AREA, 5, 1.5, 0.15)], seed=9,
                     iters=[20]),
    "hio_patterson_40x24": dict(shape=(40, 24), alg=HIO, beta=0.9, cons=POS_COMPLEX, sup=None, seed=10, iters=[25],
                                patterson=0.004),
    "raar_sched_64": dict(shape=(64, 64), alg=RAAR, beta={0: 0.95, 30: 0.7}, cons=POS_REAL,
                          sup=[(AREA, 20, {0: 2.5, 40: 1.0}, 0.08)], seed=11, iters=[45]),
}


def inputs(name):
    from libspimage_b200 import synth

    cfg = SCENARIOS[name]
    amp, mask, support, _ = synth.small_pattern(cfg["shape"], seed=cfg["seed"])
    return amp, mask, support


def run(engine, name, amp, mask, support):
    cfg = SCENARIOS[name]
    engine.set_algorithm(cfg["alg"], beta=cfg["beta"], constraints=cfg["cons"])
    for s in cfg["sup"] or []:
        engine.add_support_update(*s)
    if hasattr(engine, "start"):
        engine.start()
    engine.set_amplitudes(amp, mask)
    assert engine.init_model(1, seed=cfg["seed"]) == 0
    if cfg.get("patterson") is not None:
        engine.init_support_patterson(cfg["patterson"])
    else:
        engine.set_support(support)
    for n in cfg["iters"]:
        assert engine.iterate(n) == 0
    ef, fc = engine.efourier()
    return dict(
        g0=np.ascontiguousarray(engine.get(0)), g1=np.ascontiguousarray(engine.get(1)),
        gp=np.ascontiguousarray(engine.get(2)), flags=np.ascontiguousarray(engine.flags()).astype(np.int32),
        iteration=np.int32(engine.iteration), efourier=np.float32(ef), fcfo=np.float32(fc),
        ereal=np.float32(engine.ereal()), support_fraction=np.float32(engine.support_fraction()),
    )
