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
