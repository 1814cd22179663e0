"""GPU parity of the API modes beside the plain phase-recovery run, against the
oracle (the CPU restatement of the reference engine):

* amplitude error margins, SpAmplitudeErrorMargin (src/phasing.c:1070-1100,
  sp_phaser_set_amplitudes_margins :335-363);
* amplitude recovery from phased amplitudes, SpRecoverAmplitudes
  (src/phasing.c:1103-1109, sp_phaser_set_phased_amplitudes :235-269);
* ZeroPhases, RandomValues and MaskedOutZeroed starting models on a one-start
  phaser (src/phasing.c:606-724);
* Patterson support (src/phasing.c:744-763);
* the accessors fmodel, fmodel_with_mask, old_model, model_change,
  model_with_support and amplitudes (src/phasing.c:365-554).

All bit-exact."""
import numpy as np
import pytest

from libspimage_b200 import synth
from tests._engines import AREA, DIFFMAP, ER, HIO, RAAR, RANDOM_PHASES, rel_l2, same_bits, setup

pytestmark = pytest.mark.gpu

POS_REAL, MARGIN = 2, 32
ZERO_PHASES, RANDOM_VALUES, MASKED_OUT_ZEROED = 2, 4, 256
RECOVER_AMPLITUDES = 1


def _same_run(gpu, ref):
    for which in (0, 1, 2):
        g, r = gpu.get(which), ref.get(which)
        assert same_bits(g, r), f"which={which} rel={rel_l2(g, r)}"
    assert np.array_equal(gpu.support(), ref.support())


def _margins(shape):
    amp, mask, support, _ = synth.small_pattern(shape, seed=1)
    rng = np.random.default_rng(5)
    amin = (amp * (1 - 0.2 * rng.random(shape))).astype(np.float32)
    amax = (amp * (1 + 0.2 * rng.random(shape))).astype(np.float32)
    return amp, mask, support, amin, amax


@pytest.mark.parametrize("shape,alg", [((48, 40), HIO), ((64, 64), RAAR), ((8, 16, 12), ER), ((64, 64, 16), HIO)])
def test_amplitude_margins_bit_exact(lib, oracle_mod, shape, alg):
    amp, mask, support, amin, amax = _margins(shape)
    engines = []
    for eng in (oracle_mod.Restatement(shape), lib.Phaser(shape)):
        eng.set_algorithm(alg, beta=0.9, constraints=POS_REAL | MARGIN)
        eng.add_support_update(AREA, 7, 2.0, 0.1)
        if hasattr(eng, "start"):
            eng.start()
        eng.set_amplitudes(amp, mask)
        eng.set_amplitudes_margins(amin, amax)
        assert eng.init_model(RANDOM_PHASES, seed=4) == 0
        eng.set_support(support)
        assert eng.iterate(30) == 0
        engines.append(eng)
    ref, gpu = engines
    _same_run(gpu, ref)
    # the margins change the result: a run without them differs
    plain = setup(lib.Phaser(shape), shape, alg, [(AREA, 7, 2.0, 0.1)], seed=4)
    assert plain.iterate(30) == 0
    assert not same_bits(plain.model(), gpu.model())


@pytest.mark.parametrize("shape,alg", [((48, 40), HIO), ((32, 32), ER), ((16, 8, 12), RAAR)])
def test_recover_amplitudes_bit_exact(lib, oracle_mod, shape, alg):
    """SpRecoverAmplitudes: the measured pixels of the Fourier iterate are
    replaced by the given phased amplitudes."""
    amp, mask, support, obj = synth.small_pattern(shape, seed=2)
    rng = np.random.default_rng(9)
    pa = (np.fft.fftn(obj) * np.exp(2j * np.pi * 0.05 * rng.standard_normal(shape))).astype(np.complex64)
    pmask = (rng.random(shape) < 0.7).astype(np.int32)
    engines = []
    for eng in (oracle_mod.Restatement(shape), lib.Phaser(shape)):
        eng.set_algorithm(alg, beta=0.85, constraints=POS_REAL)
        if hasattr(eng, "start"):
            eng.start()
        eng.set_amplitudes(amp, mask)
        assert eng.init_model(RANDOM_PHASES, seed=8) == 0
        eng.set_phased_amplitudes(pa, pmask)
        eng.set_objective(RECOVER_AMPLITUDES)
        eng.set_support(support)
        assert eng.iterate(21) == 0
        engines.append(eng)
    ref, gpu = engines
    _same_run(gpu, ref)


@pytest.mark.parametrize("init", [ZERO_PHASES, RANDOM_VALUES, RANDOM_PHASES | MASKED_OUT_ZEROED,
                                  RANDOM_VALUES | MASKED_OUT_ZEROED, ZERO_PHASES | MASKED_OUT_ZEROED])
@pytest.mark.parametrize("shape", [(40, 48), (8, 12, 16)])
def test_model_initialisations_bit_exact(lib, oracle_mod, init, shape):
    ref = setup(oracle_mod.Restatement(shape), shape, HIO, [(AREA, 5, 2.0, 0.1)], init_flags=init, seed=13)
    gpu = setup(lib.Phaser(shape), shape, HIO, [(AREA, 5, 2.0, 0.1)], init_flags=init, seed=13)
    assert same_bits(gpu.model(), ref.model()), f"initial model rel {rel_l2(gpu.model(), ref.model())}"
    assert ref.iterate(16) == 0 and gpu.iterate(16) == 0
    _same_run(gpu, ref)


@pytest.mark.parametrize("shape,value", [((32, 32), 0.05), ((40, 24), 0.1), ((8, 16, 16), 0.02), ((128, 128), 0.05)])
def test_patterson_support_bit_exact(lib, oracle_mod, shape, value):
    ref = setup(oracle_mod.Restatement(shape), shape, HIO, [(AREA, 5, 2.0, 0.1)], patterson=value)
    gpu = setup(lib.Phaser(shape), shape, HIO, [(AREA, 5, 2.0, 0.1)], patterson=value)
    assert np.array_equal(gpu.support(), ref.support())
    assert ref.support().sum() > 0
    assert ref.iterate(12) == 0 and gpu.iterate(12) == 0
    _same_run(gpu, ref)


@pytest.mark.parametrize("shape,alg", [((48, 40), HIO), ((32, 32), DIFFMAP), ((8, 16, 12), RAAR)])
def test_accessors_bit_exact(lib, oracle_mod, shape, alg):
    ref = setup(oracle_mod.Restatement(shape), shape, alg, [(AREA, 6, 2.0, 0.1)])
    gpu = setup(lib.Phaser(shape), shape, alg, [(AREA, 6, 2.0, 0.1)])
    assert ref.iterate(17) == 0 and gpu.iterate(17) == 0
    model, old = ref.model(), ref.old_model()
    flags = ref.flags()
    # old model (g0)
    assert same_bits(gpu.old_model(), old)
    # fmodel: forward FFT of the model (sp_image_fft_fast)
    fm = oracle_mod.fft(model, -1)
    assert same_bits(gpu.fmodel(), fm)
    data, mask = gpu.fmodel_with_mask()
    assert same_bits(data, fm)
    assert np.array_equal(mask != 0, (flags & 2) != 0)
    # model_change: model - g0, complex float subtraction (sp_image_sub)
    assert same_bits(gpu.model_change(), (model - old).astype(np.complex64))
    # model_with_support: the model with the support as its mask
    data, mask = gpu.model_with_support()
    assert same_bits(data, model)
    assert np.array_equal(mask != 0, (flags & 1) != 0)
    # amplitudes: the amplitudes as a real image, measured mask
    data, mask = gpu.amplitudes_image()
    assert same_bits(data.real.astype(np.float32), gpu.amplitudes_np.astype(np.float32))
    assert not np.any(data.imag)
    assert np.array_equal(mask != 0, (flags & 2) != 0)
    # cached per iteration: a second read is the same, and one more
    # iteration refreshes every accessor
    assert same_bits(gpu.fmodel(), fm)
    assert ref.iterate(1) == 0 and gpu.iterate(1) == 0
    assert same_bits(gpu.old_model(), ref.old_model())
    assert same_bits(gpu.fmodel(), oracle_mod.fft(ref.model(), -1))
    assert same_bits(gpu.model_change(), (ref.model() - ref.old_model()).astype(np.complex64))
