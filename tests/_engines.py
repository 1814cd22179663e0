"""Runs one phasing scenario on any engine with the common interface
(oracle.Restatement, oracle.Reference, libspimage_b200.Phaser)."""
import numpy as np

from libspimage_b200 import synth

HIO, RAAR, DIFFMAP, ER = 1, 2, 3, 4
AREA, THRESHOLD, STATIC = 2, 1, 5
RANDOM_PHASES = 1


def setup(engine, shape, alg, sup=None, constraints=2, beta=0.9, seed=3, pattern_seed=1,
          init_flags=RANDOM_PHASES, patterson=None):
    amp, mask, support, _ = synth.small_pattern(shape, seed=pattern_seed)
    engine.set_algorithm(alg, beta=beta, constraints=constraints)
    for s in (sup or []):
        engine.add_support_update(*s)
    if hasattr(engine, "start"):
        engine.start()
    engine.set_amplitudes(amp, mask)
    engine.amplitudes_np = amp
    rc = engine.init_model(init_flags, seed=seed)
    assert rc == 0
    if patterson is not None:
        engine.init_support_patterson(patterson)
    else:
        engine.set_support(support)
    return engine


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype in (np.float32, np.complex64) else a


def same_bits(a, b):
    return np.array_equal(bits(a), bits(b))


def rel_l2(a, b):
    return float(np.linalg.norm((np.asarray(a) - np.asarray(b)).ravel()) / max(np.linalg.norm(np.asarray(b).ravel()), 1e-30))


# Scenarios of the closing, centre-image and template support updates:
# name, shape, algorithm, support steps, initial-support shift, iterations.
# A step is ("area"|"threshold", period, blur, value), ("close", period, size),
# ("centre", period) or ("template", period, blur, area schedule).
MORPH_SCENARIOS = [
    ("area_close", (48, 40), HIO, [("area", 7, 2.0, 0.1), ("close", 7, 2)], (0, 0), 50),
    ("area_centre_offset", (48, 40), RAAR, [("area", 7, 2.0, 0.1), ("centre", 7)], (5, -7), 50),
    ("template", (64, 48), HIO, [("template", 6, 3.0, {0: 1.3, 60: 0.8})], (0, 0), 50),
    ("threshold_close_centre", (32, 32), HIO, [("threshold", 5, 2.0, 0.2), ("close", 5, 1), ("centre", 5)], (3, 4), 40),
    ("3d_area_close_centre", (8, 16, 12), ER, [("area", 5, 1.5, 0.2), ("close", 5, 1), ("centre", 5)], (2, -3), 31),
]


def setup_morph(engine, shape, alg, steps, shift, seed=3):
    """A phaser with the scenario's support steps; the initial support disc is
    rolled by `shift` (last two axes) so that centring has work to do."""
    amp, mask, support, _ = synth.small_pattern(shape, seed=1)
    support = np.roll(support, shift, axis=(-2, -1))
    engine.set_algorithm(alg, beta=0.9, constraints=2)
    for st in steps:
        if st[0] in ("area", "threshold"):
            engine.add_support_update(AREA if st[0] == "area" else THRESHOLD, st[1], st[2], st[3])
        elif st[0] == "close":
            engine.add_support_close(st[1], st[2])
        elif st[0] == "centre":
            engine.add_support_centre(st[1])
        else:
            engine.add_support_template(st[1], support, st[2], st[3])
    if hasattr(engine, "start"):
        engine.start()
    engine.set_amplitudes(amp, mask)
    engine.amplitudes_np = amp
    assert engine.init_model(RANDOM_PHASES, seed=seed) == 0
    engine.set_support(support)
    return engine, support
