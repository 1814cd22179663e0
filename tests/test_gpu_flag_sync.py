"""Pixel flags edited on the host between runs (src/phasing.c:207-232
sp_phaser_set_support, :294-333 sp_phaser_set_amplitudes): the host API
uploads only the flag bits it edited and fetches only those the device
changed, so a support update's support bits stay on the device while the
host replaces the measured bits, and a new support replaces the device's
support bits without fetching them first.  Each sequence runs on the GPU and
on the oracle (the reference CPU engine's restatement, which keeps one copy
of the flags) and must end in the same bits: iterates, support and measured
mask."""
import numpy as np
import pytest

from libspimage_b200 import synth
from tests._engines import AREA, HIO, RAAR, THRESHOLD, rel_l2, same_bits, setup

pytestmark = pytest.mark.gpu


def _same(gpu, ref):
    for which in (0, 1, 2):
        g, r = gpu.get(which), ref.get(which)
        assert same_bits(g, r), f"which={which} rel={rel_l2(g, r)}"
    assert np.array_equal(gpu.support(), ref.support())
    assert np.array_equal(gpu.flags(), ref.flags())


def _other_mask(shape, seed):
    amp, mask, _, _ = synth.small_pattern(shape, seed=seed)
    return amp, mask


@pytest.mark.parametrize("shape,alg,sup", [((48, 40), HIO, (AREA, 4, 2.0, 0.1)),
                                           ((16, 16, 12), RAAR, (THRESHOLD, 5, 1.5, 0.2))])
def test_new_amplitudes_after_support_updates(lib, oracle_mod, shape, alg, sup):
    """set_amplitudes after a run whose support updates changed the support
    on the device: the next iterations use the device's support bits and the
    new measured bits."""
    amp2, mask2 = _other_mask(shape, seed=7)
    gpu = setup(lib.Phaser(shape), shape, alg, [sup])
    ref = setup(oracle_mod.Restatement(shape), shape, alg, [sup])
    for e in (gpu, ref):
        assert e.iterate(11) == 0
        e.set_amplitudes(amp2, mask2)
        assert e.iterate(9) == 0
    _same(gpu, ref)


def test_new_support_and_amplitudes_then_new_start(lib, oracle_mod):
    """After a run: a new support (replacing the device's support bits without
    fetching them), new amplitudes, a new random start, then iterations --
    the flow of one reconstruction after another on the same phaser."""
    shape, alg, sup = (40, 48), RAAR, (AREA, 3, 1.5, 0.15)
    amp2, mask2, sup2, _ = synth.small_pattern(shape, seed=11)
    gpu = setup(lib.Phaser(shape), shape, alg, [sup])
    ref = setup(oracle_mod.Restatement(shape), shape, alg, [sup])
    for e in (gpu, ref):
        assert e.iterate(10) == 0
        e.set_support(sup2)
        e.set_amplitudes(amp2, mask2)
        assert e.init_model(1, seed=19) == 0  # random phases
        assert e.iterate(8) == 0
    _same(gpu, ref)


def test_read_support_between_host_edits(lib, oracle_mod):
    """Reading the support (which fetches the device's support bits) between
    a measured-bit edit and the next run keeps the edit."""
    shape, alg, sup = (32, 32), HIO, (AREA, 4, 2.0, 0.2)
    amp2, mask2 = _other_mask(shape, seed=13)
    gpu = setup(lib.Phaser(shape), shape, alg, [sup])
    ref = setup(oracle_mod.Restatement(shape), shape, alg, [sup])
    for e in (gpu, ref):
        assert e.iterate(9) == 0
        e.set_amplitudes(amp2, mask2)
    assert np.array_equal(gpu.support(), ref.support())
    assert np.array_equal(gpu.flags(), ref.flags())
    for e in (gpu, ref):
        assert e.iterate(6) == 0
    _same(gpu, ref)
