"""GPU parity: every kernel path against the oracle (CPU restatement of the
reference engine), through the library's C-ABI.  The device FFT and every
pointwise step follow the same arithmetic as the oracle, so the checks are
bit-exact unless a tolerance is written next to them."""
import numpy as np
import pytest

from tests._engines import AREA, DIFFMAP, ER, HIO, RAAR, STATIC, THRESHOLD, bits, rel_l2, same_bits, setup

pytestmark = pytest.mark.gpu

FFT_SHAPES = [(8, 8), (16, 16), (32, 32), (64, 48), (24, 40), (17, 19), (128, 128), (256, 256), (192, 384),
              (8, 16, 12), (16, 16, 16), (5, 7, 9), (1, 64), (1000, 8), (3, 1024),
              # register kernels of the 2^a 3^b 5^c lengths (rows and columns)
              (192, 192), (384, 40), (40, 384), (16, 1000), (1000, 24), (6, 192, 384)]


@pytest.mark.parametrize("shape", FFT_SHAPES)
@pytest.mark.parametrize("sign", [-1, 1])
def test_fft_bit_exact(lib, oracle_mod, shape, sign):
    rng = np.random.default_rng(hash(shape) % 1000)
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    got = lib.fft(x, sign)
    want = oracle_mod.fft(x, sign)
    assert same_bits(got, want), f"max abs diff {np.abs(got - want).max()}"


@pytest.mark.parametrize("shape", [(32, 32), (64, 48), (8, 16, 12), (128, 128), (192, 192), (1000, 40)])
@pytest.mark.parametrize("radius", [0.7, 3.0])
def test_blur_bit_exact(lib, oracle_mod, shape, radius):
    rng = np.random.default_rng(7)
    x = rng.random(shape).astype(np.complex64)
    got = lib.gaussian_blur(x, radius)
    want = oracle_mod.gaussian_blur(x, radius)
    assert same_bits(got, want), f"rel {rel_l2(got, want)}"


@pytest.mark.parametrize("area", [0.05, 0.1, 0.3333])
def test_area_mask_bit_exact_on_identical_blur(lib, oracle_mod, area):
    rng = np.random.default_rng(11)
    blur = (rng.random((64, 64)) + 1j * rng.random((64, 64)) * 1e-3).astype(np.complex64)
    blur.real[:4, :4] = 0.5  # ties at the threshold
    flags = rng.integers(0, 4, size=blur.shape).astype(np.int32)
    t = oracle_mod.area_threshold(blur, area)
    # |.| exactly as the reference: sqrt(im*im + re*re) in float
    a = np.sqrt((blur.imag * blur.imag + blur.real * blur.real).astype(np.float32))
    want = (flags & ~1) | (a > np.float32(t)).astype(np.int32)
    got = lib.support_from_blur(blur, AREA, area, flags)
    assert np.array_equal(got, want)


def test_threshold_mask_bit_exact_on_identical_blur(lib):
    rng = np.random.default_rng(12)
    blur = rng.random((48, 40)).astype(np.complex64)
    flags = np.zeros(blur.shape, np.int32)
    a = np.abs(blur.real).astype(np.float32)
    want = (a > np.float32(a.max() * np.float32(0.2))).astype(np.int32)
    got = lib.support_from_blur(blur, THRESHOLD, 0.2, flags)
    assert np.array_equal(got, want)


SCENARIOS = [
    ("hio", (32, 32), HIO, None, 2),
    ("raar", (32, 32), RAAR, None, 2),
    ("er", (32, 32), ER, None, 2),
    ("dm", (32, 32), DIFFMAP, None, 2),
    ("hio_area", (64, 48), HIO, [(AREA, 5, {0: 3.0, 40: 0.7}, 0.1)], 2),
    ("raar_thr", (24, 40), RAAR, [(THRESHOLD, 7, 2.0, 0.2)], 0),
    ("er_area_3d", (8, 16, 12), ER, [(AREA, 5, 1.5, 0.2)], 2),
    ("dm_area", (32, 32), DIFFMAP, [(AREA, 6, 2.0, 0.15)], 2),
    ("hio_3d", (16, 16, 16), HIO, [(AREA, 10, 2.0, 0.1)], 2),
    ("hio_nc", (48, 48), HIO, [(AREA, 9, 3.0, 0.1), (STATIC, 9, 0, 0)], 0),
    ("raar_flip", (40, 30), RAAR, None, 2 | 8),
    ("hio_complex", (32, 32), HIO, None, 4),
    ("hio_real_centro", (32, 32), HIO, None, 1 | 16),
    ("hio_area_192", (192, 192), HIO, [(AREA, 7, 2.0, 0.1)], 2),
    ("raar_thr_1000", (24, 1000), RAAR, [(THRESHOLD, 6, 2.0, 0.2)], 2),
    ("er_area_384", (384, 48), ER, [(AREA, 5, 1.5, 0.1)], 2),
    # difference map: register row pass (power-of-two rows) and general row pass
    ("dm_area_256", (128, 256), DIFFMAP, [(AREA, 9, 2.0, 0.1)], 2),
    ("dm_area_3d", (16, 16, 32), DIFFMAP, [(AREA, 5, 2.0, 0.1)], 2),
    ("dm_48", (40, 48), DIFFMAP, None, 2),
    ("dm_many_short_rows", (640, 32), DIFFMAP, [(AREA, 7, 2.0, 0.1)], 2),
]


@pytest.mark.parametrize("name,shape,alg,sup,cons", SCENARIOS, ids=[s[0] for s in SCENARIOS])
def test_phaser_bit_exact(lib, oracle_mod, name, shape, alg, sup, cons):
    nit = 23
    ref = setup(oracle_mod.Restatement(shape), shape, alg, sup, constraints=cons)
    gpu = setup(lib.Phaser(shape), shape, alg, sup, constraints=cons)
    assert same_bits(gpu.model(), ref.model()), "initial model"
    assert ref.iterate(nit) == 0
    assert gpu.iterate(nit) == 0
    assert gpu.iteration == ref.iteration == nit
    _compare(gpu, ref)


# long runs: iterations between support updates are replayed from captured
# CUDA graphs (beta from a device table); the schedule varies beta per iteration
LONG = [
    ("hio_sched", (64, 64), HIO, None, 2, {0: 0.95, 150: 0.75}, [70, 61, 33]),
    ("raar_area20", (128, 128), RAAR, [(AREA, 20, {0: 3.0, 200: 0.7}, 0.08)], 2, 0.87, [120, 47]),
    ("er_3d", (16, 32, 32), ER, [(AREA, 25, 2.0, 0.1)], 2, 0.9, [80]),
    ("dm_long", (64, 64), DIFFMAP, None, 2, 0.8, [40, 40]),
]


@pytest.mark.parametrize("name,shape,alg,sup,cons,beta,calls", LONG, ids=[s[0] for s in LONG])
def test_phaser_graph_replay_bit_exact(lib, oracle_mod, name, shape, alg, sup, cons, beta, calls):
    ref = setup(oracle_mod.Restatement(shape), shape, alg, sup, constraints=cons, beta=beta)
    gpu = setup(lib.Phaser(shape), shape, alg, sup, constraints=cons, beta=beta)
    for n in calls:
        assert ref.iterate(n) == 0
        assert gpu.iterate(n) == 0
        assert gpu.iteration == ref.iteration
        assert same_bits(gpu.model(), ref.model()), f"after {gpu.iteration} iterations"
    _compare(gpu, ref)


def _cabs(z):
    """|z| as the reference computes it: sqrt(im*im + re*re) in float."""
    z = np.asarray(z, np.complex64)
    return np.sqrt((z.imag * z.imag + z.real * z.real).astype(np.float32)).astype(np.float32)


def _metrics64(model, gp, flags, amp, oracle_mod):
    """Fourier and real-space errors (src/phasing.c:803-891) evaluated in FP64
    on given (bit-identical) arrays."""
    inside = (flags & 1) != 0
    meas = (flags & 2) != 0
    a = _cabs(gp).astype(np.float64) ** 2
    ereal = np.sqrt(a[~inside].sum() / a.sum())
    F = _cabs(oracle_mod.fft(model, -1)).astype(np.float64)
    A = np.abs(np.asarray(amp, np.float64))
    nom = ((F - A) ** 2)[meas].sum()
    den = (A ** 2)[meas].sum() + (F ** 2)[~meas].sum()
    return np.sqrt(nom / den), A[meas].sum() / F[meas].sum(), ereal


def _compare(gpu, ref, oracle_mod=None):
    assert np.array_equal(gpu.support(), ref.support())
    for which in (0, 1, 2):
        g, r = gpu.get(which), ref.get(which)
        assert same_bits(g, r), f"which={which} rel={rel_l2(g, r)}"
    assert gpu.support_fraction() == ref.support_fraction()
    if oracle_mod is None:
        import oracle as oracle_mod
    flags = ref.flags()
    amp = getattr(gpu, "amplitudes_np", None)
    ef_g, fc_g = gpu.efourier()
    ef_r, fc_r = ref.efourier()
    er_g, er_r = gpu.ereal(), ref.ereal()
    if amp is not None:
        ef64, fc64, er64 = _metrics64(ref.model(), ref.model_before_projection(), flags, amp, oracle_mod)
        # GPU reductions run in double: agree with FP64 to float rounding
        assert abs(ef_g - ef64) <= 2e-6 * ef64 + 1e-12
        assert abs(fc_g - fc64) <= 2e-6 * fc64
        assert abs(er_g - er64) <= 2e-6 * er64 + 1e-12
        # the reference accumulates in float, sequentially: looser
        assert abs(ef_r - ef64) <= 1e-3 * ef64 + 1e-9
        assert abs(er_r - er64) <= 1e-3 * er64 + 1e-9
    else:
        assert abs(ef_g - ef_r) <= 1e-4 * abs(ef_r) + 1e-12
        assert abs(er_g - er_r) <= 1e-3 * abs(er_r) + 1e-12


from tests._engines import MORPH_SCENARIOS, setup_morph  # noqa: E402


@pytest.mark.parametrize("name,shape,alg,steps,shift,nit", MORPH_SCENARIOS, ids=[s[0] for s in MORPH_SCENARIOS])
def test_close_centre_template_bit_exact(lib, oracle_mod, name, shape, alg, steps, shift, nit):
    """closing (device morphology), centre-image (host, per start) and
    template (device mask from the blurred template) against the oracle"""
    ref, _ = setup_morph(oracle_mod.Restatement(shape), shape, alg, steps, shift)
    gpu, _ = setup_morph(lib.Phaser(shape), shape, alg, steps, shift)
    assert ref.iterate(nit) == 0
    assert gpu.iterate(nit) == 0
    _compare(gpu, ref)


def test_close_centre_batched_starts(lib):
    """the same support steps on a batch of starts equal one-start phasers"""
    name, shape, alg, steps, shift, nit = MORPH_SCENARIOS[3]
    seeds = [4, 9, 16]
    amp, mask, support, _ = __import__("libspimage_b200").synth.small_pattern(shape, seed=1)
    support = np.roll(support, shift, axis=(-2, -1))
    batch = lib.Phaser(shape)
    batch.set_algorithm(alg, beta=0.9, constraints=2)
    batch.add_support_update(THRESHOLD, 5, 2.0, 0.2)
    batch.add_support_close(5, 1)
    batch.add_support_centre(5)
    batch.start()
    batch.set_starts(len(seeds))
    batch.set_amplitudes(amp, mask)
    assert batch.init_models(1, seeds) == 0
    batch.set_support(support)
    assert batch.iterate(nit) == 0
    for b, s in enumerate(seeds):
        one, _ = setup_morph(lib.Phaser(shape), shape, alg, steps, shift, seed=s)
        assert one.iterate(nit) == 0
        assert np.array_equal(batch.start_support(b), one.support())
        assert same_bits(batch.start_model(b), one.model())


@pytest.mark.parametrize("shape,alg,sup", [((256, 256), HIO, [(AREA, 20, 3.0, 0.05)]), ((64, 64), DIFFMAP, None),
                                           ((640, 32), DIFFMAP, [(AREA, 7, 2.0, 0.1)]),
                                           ((16, 16, 16), RAAR, [(AREA, 10, 2.0, 0.1)])])
def test_autotune_and_launch_shapes_leave_results_unchanged(lib, oracle_mod, shape, alg, sup):
    """the autotuner restores the reconstruction it times on, and every
    launch shape (row lines per block, dependent launch on/off, where the
    row pass stages the previous iterate) computes the same bits"""
    ref = setup(oracle_mod.Restatement(shape), shape, alg, sup)
    tuned = setup(lib.Phaser(shape), shape, alg, sup)
    assert tuned.iterate(7) == 0 and ref.iterate(7) == 0
    choice = tuned.autotune()
    assert choice["row_lines"] >= 0 and choice["no_pdl"] in (0, 1) and choice["row_g0"] in (1, 2)
    assert choice["split"] in (1, 2) and choice["persist"] in (1, 2)
    assert tuned.autotune() == choice  # cached
    assert tuned.iterate(45) == 0 and ref.iterate(45) == 0
    _compare(tuned, ref)
    for knob, value in ((0, 1), (0, 2), (1, 1), (2, 1), (2, 2), (3, 1), (3, 2), (4, 1), (4, 2)):
        other = setup(lib.Phaser(shape), shape, alg, sup)
        other.set_tuning(knob, value)
        assert other.iterate(52) == 0
        assert same_bits(other.model(), ref.model()), f"knob {knob}={value}"
