"""Batched random starts: one SpPhaser advancing several reconstructions of one
pattern (sp_phaser_set_starts) gives, for every start, bit for bit what a
one-start phaser gives from the same seed.  This is the batched form of the
reference's sequential Reconstructor.reconstruct_loop
(src/_spimage_reconstructor.py:677-740)."""
import numpy as np
import pytest

from libspimage_b200 import synth
from tests._engines import AREA, DIFFMAP, ER, HIO, RAAR, RANDOM_PHASES, THRESHOLD, rel_l2, same_bits, setup

pytestmark = pytest.mark.gpu

RANDOM_VALUES = 4
MASKED_OUT_ZEROED = 256  # SpModelMaskedOutZeroed, include/spimage/phasing.h


def batch_setup(lib, shape, alg, sup, seeds, constraints=2, beta=0.9, init_flags=RANDOM_PHASES, patterson=None):
    amp, mask, support, _ = synth.small_pattern(shape, seed=1)
    ph = lib.Phaser(shape)
    ph.set_algorithm(alg, beta=beta, constraints=constraints)
    for s in (sup or []):
        ph.add_support_update(*s)
    ph.start()
    ph.set_starts(len(seeds))
    ph.set_amplitudes(amp, mask)
    assert ph.init_models(init_flags, seeds) == 0
    if patterson is not None:
        ph.init_support_patterson(patterson)
    else:
        ph.set_support(support)
    return ph


def check_start(batch, b, single):
    assert same_bits(batch.start_model(b), single.model()), f"start {b}: model rel {rel_l2(batch.start_model(b), single.model())}"
    assert np.array_equal(batch.start_support(b), single.support()), f"start {b}: support"
    assert same_bits(batch.start_model_before_projection(b), single.model_before_projection()), f"start {b}: gp"


BATCH = [
    # name, shape, alg, support updates, constraints, beta, seeds, iterate calls
    ("hio_area", (64, 48), HIO, [(AREA, 5, {0: 3.0, 40: 0.7}, 0.1)], 2, 0.9, [3, 11, 12, 400, 7], [23, 40]),
    ("raar_area_graphs", (128, 128), RAAR, [(AREA, 20, {0: 3.0, 200: 0.7}, 0.08)], 2, 0.87, [5, 6, 9], [120, 47]),
    ("er_area_3d", (8, 16, 12), ER, [(AREA, 5, 1.5, 0.2)], 2, 0.9, [1, 2, 3, 4], [31]),
    ("dm_area", (32, 32), DIFFMAP, [(AREA, 6, 2.0, 0.15)], 2, 0.8, [21, 22, 23], [40]),
    ("raar_thr", (24, 40), RAAR, [(THRESHOLD, 7, 2.0, 0.2)], 0, 0.9, [8, 9], [29]),
    ("hio_sched_nosup", (64, 64), HIO, None, 2, {0: 0.95, 150: 0.75}, [100, 101, 102, 103, 104, 105], [70, 61]),
]


@pytest.mark.parametrize("name,shape,alg,sup,cons,beta,seeds,calls", BATCH, ids=[s[0] for s in BATCH])
def test_batch_equals_single_starts(lib, name, shape, alg, sup, cons, beta, seeds, calls):
    batch = batch_setup(lib, shape, alg, sup, seeds, constraints=cons, beta=beta)
    singles = [setup(lib.Phaser(shape), shape, alg, sup, constraints=cons, beta=beta, seed=s) for s in seeds]
    for b, s in enumerate(singles):
        assert same_bits(batch.start_model(b), s.model()), f"initial model of start {b}"
    for n in calls:
        assert batch.iterate(n) == 0
        for s in singles:
            assert s.iterate(n) == 0
    for b, s in enumerate(singles):
        check_start(batch, b, s)
    # start 0 through the single-image accessors
    assert same_bits(batch.model(), singles[0].model())
    # per-start metrics: double reductions (block partition depends on the
    # number of starts, so the last float bit may differ)
    ef, fc = batch.starts_efourier()
    er = batch.starts_ereal()
    sf = batch.starts_support_fraction()
    for b, s in enumerate(singles):
        e1, f1 = s.efourier()
        assert abs(ef[b] - e1) <= 1e-6 * e1
        assert abs(fc[b] - f1) <= 1e-6 * f1
        assert abs(er[b] - s.ereal()) <= 1e-6 * s.ereal() + 1e-12
        assert sf[b] == s.support_fraction()


def test_batch_matches_oracle(lib, oracle_mod):
    """one start of a batch against the CPU restatement of the reference engine"""
    shape, alg, sup = (64, 48), HIO, [(AREA, 5, {0: 3.0, 40: 0.7}, 0.1)]
    seeds = [17, 18, 19]
    batch = batch_setup(lib, shape, alg, sup, seeds)
    ref = setup(oracle_mod.Restatement(shape), shape, alg, sup, seed=seeds[2])
    assert batch.iterate(33) == 0
    assert ref.iterate(33) == 0
    assert same_bits(batch.start_model(2), ref.model())
    assert np.array_equal(batch.start_support(2), ref.support())


def test_batch_random_values_and_masked_out(lib):
    shape, seeds = (32, 32), [4, 5, 6]
    flags = 4 | MASKED_OUT_ZEROED
    batch = batch_setup(lib, shape, HIO, [(AREA, 5, 2.0, 0.1)], seeds, init_flags=flags)
    singles = [setup(lib.Phaser(shape), shape, HIO, [(AREA, 5, 2.0, 0.1)], seed=s, init_flags=flags) for s in seeds]
    assert batch.iterate(12) == 0
    for b, s in enumerate(singles):
        assert s.iterate(12) == 0
        check_start(batch, b, s)


def test_batch_patterson(lib):
    shape, seeds = (32, 32), [2, 3]
    batch = batch_setup(lib, shape, HIO, [(AREA, 5, 2.0, 0.1)], seeds, patterson=0.05)
    singles = [setup(lib.Phaser(shape), shape, HIO, [(AREA, 5, 2.0, 0.1)], seed=s, patterson=0.05) for s in seeds]
    for b, s in enumerate(singles):
        assert np.array_equal(batch.start_support(b), s.support())
    assert batch.iterate(11) == 0
    for b, s in enumerate(singles):
        assert s.iterate(11) == 0
        check_start(batch, b, s)


def test_batch_column_grid_split(lib):
    """4097 starts of 16^3: the y-axis pass has 4097*16 outer lines, more
    than one grid's y dimension (65535), so it is launched in two pieces"""
    shape, nb = (16, 16, 16), 4097
    seeds = list(range(nb))
    sup = [(AREA, 5, 1.5, 0.2)]
    batch = batch_setup(lib, shape, ER, sup, seeds)
    assert batch.iterate(7) == 0
    for b in (0, 2048, 4096):
        s = setup(lib.Phaser(shape), shape, ER, sup, seed=seeds[b])
        assert s.iterate(7) == 0
        check_start(batch, b, s)


def test_device_random_phase_starts(lib, oracle_mod):
    shape = (64, 64)
    amp, mask, support, _ = synth.small_pattern(shape, seed=1)

    def make(seeds):
        ph = lib.Phaser(shape)
        ph.set_algorithm(HIO, beta=0.9, constraints=2)
        ph.start()
        ph.set_starts(len(seeds))
        ph.set_amplitudes(amp, mask)
        assert ph.init_models_device(RANDOM_PHASES, seeds) == 0
        ph.set_support(support)
        return ph

    a = make([1, 2, 3, 4])
    b = make([1, 2, 3, 5])
    for k in range(3):
        assert same_bits(a.start_model(k), b.start_model(k))
    assert not same_bits(a.start_model(3), b.start_model(3))
    assert not same_bits(a.start_model(0), a.start_model(1))
    # the start is IFFT(amp * exp(i phi)) / N: its transform has the amplitudes
    for k in range(4):
        F = oracle_mod.fft(a.start_model(k), -1)
        assert rel_l2(np.abs(F), amp) < 1e-5
        ph = np.angle(F[amp > 0])
        # uniform phases: the mean phasor of n of them is ~ 1/sqrt(n)
        assert ph.size > 200
        assert abs(np.mean(np.exp(1j * ph))) < 5.0 / np.sqrt(ph.size)
    assert a.iterate(30) == 0
    ef, _ = a.starts_efourier()
    assert np.all(np.isfinite(ef)) and np.all(ef > 0)
