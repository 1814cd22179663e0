"""CPU tests of the oracle: pinned to the reference's own engine and to the
known answers of the reference's test suite.  No GPU needed."""
import glob
import os
import sys

import numpy as np
import pytest

from tests._engines import AREA, DIFFMAP, ER, HIO, RAAR, STATIC, THRESHOLD, same_bits, setup

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import scenarios  # noqa: E402

GOLDEN = sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(HERE, "golden", "*.npz")))


def _check_against(out, gold):
    assert int(out["iteration"]) == int(gold["iteration"])
    for k in ("g0", "g1", "gp"):
        assert same_bits(out[k], gold[k]), k
    assert np.array_equal(out["flags"], gold["flags"])
    for k in ("efourier", "fcfo", "ereal", "support_fraction"):
        assert np.float32(out[k]).view(np.uint32) == np.float32(gold[k]).view(np.uint32), k


def test_golden_fixtures_present():
    assert set(GOLDEN) == set(scenarios.SCENARIOS)


@pytest.mark.parametrize("name", GOLDEN)
def test_restatement_reproduces_reference_golden(oracle_mod, name):
    """The C restatement reproduces, bit for bit, outputs the reference engine produced."""
    gold = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    eng = oracle_mod.Restatement(scenarios.SCENARIOS[name]["shape"])
    out = scenarios.run(eng, name, gold["amp"], gold["mask"], gold["support"])
    _check_against(out, gold)


@pytest.mark.parametrize("name", GOLDEN)
def test_reference_still_produces_golden(oracle_mod, name):
    if not oracle_mod.ref_available():
        pytest.skip("reference engine not built here (needs the reference sources)")
    gold = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    eng = oracle_mod.Reference(scenarios.SCENARIOS[name]["shape"])
    out = scenarios.run(eng, name, gold["amp"], gold["mask"], gold["support"])
    _check_against(out, gold)


PIN = [
    ((32, 32), HIO, [(AREA, 5, {0: 3.0, 40: 0.7}, 0.1)], 2),
    ((24, 40), RAAR, [(THRESHOLD, 7, 2.0, 0.2)], 0),
    ((48, 30), ER, None, 1),
    ((32, 32), DIFFMAP, [(AREA, 6, 2.0, 0.15)], 2),
    ((8, 16, 12), HIO, [(AREA, 5, 1.5, 0.2), (STATIC, 5, 0, 0)], 4 | 8),
    ((27, 25), RAAR, None, 1 | 16),
]


@pytest.mark.parametrize("shape,alg,sup,cons", PIN)
def test_restatement_bit_identical_to_reference(oracle_mod, shape, alg, sup, cons):
    if not oracle_mod.ref_available():
        pytest.skip("reference engine not built here (needs the reference sources)")
    a = setup(oracle_mod.Restatement(shape), shape, alg, sup, constraints=cons)
    b = setup(oracle_mod.Reference(shape), shape, alg, sup, constraints=cons)
    a.iterate(23)
    b.iterate(23)
    assert a.iteration == b.iteration == 23
    for w in (0, 1, 2):
        assert same_bits(a.get(w), b.get(w))
    assert np.array_equal(a.flags(), b.flags())
    assert a.efourier() == b.efourier()
    assert a.ereal() == b.ereal()


@pytest.mark.parametrize("init", [2, 4, 1 | 256, 4 | 256])
def test_model_initialisations_match_reference(oracle_mod, init):
    if not oracle_mod.ref_available():
        pytest.skip("reference engine not built here")
    shape = (16, 24)
    a = setup(oracle_mod.Restatement(shape), shape, HIO, None, init_flags=init)
    b = setup(oracle_mod.Reference(shape), shape, HIO, None, init_flags=init)
    assert same_bits(a.get(1), b.get(1))


def test_dm_default_gammas_match_reference(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference engine not built here")
    import ctypes as C

    r = oracle_mod._load_reference()
    rs = oracle_mod._load_restatement()
    for beta in (0.7, 0.87, 0.9, 1.1):
        k = np.array([0], np.float32)
        v = np.array([beta], np.float32)
        alg = r.sp_phasing_diff_map_alloc(r.ref_smap(1, oracle_mod._ptr(k), oracle_mod._ptr(v)), float("inf"), 0.0, 0)
        ph = rs.spo_create(4, 4, 1)
        rs.spo_set_algorithm(ph, 3, 1, oracle_mod._ptr(k), oracle_mod._ptr(v), float("inf"), 0.0, 0)
        for which in (1, 2):
            assert np.float32(r.ref_dm_gamma(alg, which)) == np.float32(rs.spo_dm_gamma(ph, which))
        rs.spo_destroy(ph)


SCHEDULES = [{0: 0.9}, {0: 3.0, 1000: 0.7}, {0: 0.95, 150: 0.75}, {10: 1.0, 20: 2.0, 50: 0.5}, {0: 0.05, 5000: 0.02}]


@pytest.mark.parametrize("smap", SCHEDULES)
def test_bezier_schedule_matches_reference_and_library(oracle_mod, smap):
    import libspimage_b200 as L

    lib = L.load()
    m = L.smap(smap)
    xs = np.arange(-5, 5200, 7, dtype=np.float32)
    ours = np.array([lib.spb_smap_interpolate(m, float(x)) for x in xs], np.float32)
    orc = np.array([oracle_mod.bezier(smap, float(x)) for x in xs], np.float32)
    assert same_bits(ours, orc)
    if oracle_mod.ref_available():
        r = oracle_mod._load_reference()
        k = np.array(sorted(smap), np.float32)
        v = np.array([smap[kk] for kk in sorted(smap)], np.float32)
        rm = r.ref_smap(len(k), oracle_mod._ptr(k), oracle_mod._ptr(v))
        ref = np.array([r.ref_smap_interpolate(rm, float(x)) for x in xs], np.float32)
        assert same_bits(ref, orc)


# ---------------------------------------------------------------- FFT
FFT_SIZES = [(1, 2), (1, 3), (1, 5), (1, 7), (1, 16), (1, 17), (1, 97), (1, 128), (1, 1000), (1, 1024), (8, 8),
             (30, 42), (64, 64), (3, 5, 7), (16, 8, 4)]


@pytest.mark.parametrize("shape", FFT_SIZES)
def test_fft_accuracy_vs_fp64(oracle_mod, shape):
    rng = np.random.default_rng(sum(shape))
    x = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    y = oracle_mod.fft(x, -1)
    ref = np.fft.fftn(x.astype(np.complex128))
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 4e-7
    yi = oracle_mod.fft(x, +1)
    refi = np.fft.ifftn(x.astype(np.complex128)) * x.size
    assert np.linalg.norm(yi - refi) / np.linalg.norm(refi) < 4e-7


def test_fft_known_answers(oracle_mod):
    n = (16, 12)
    d = np.zeros(n, np.complex64)
    d[0, 0] = 1
    assert np.array_equal(oracle_mod.fft(d), np.ones(n, np.complex64))  # impulse -> flat
    t = np.zeros(n, np.complex64)
    ky, kx = 3, 5
    yy, xx = np.meshgrid(np.arange(n[0]), np.arange(n[1]), indexing="ij")
    t[:] = np.exp(2j * np.pi * (ky * yy / n[0] + kx * xx / n[1]))
    F = oracle_mod.fft(t)
    assert abs(F[ky, kx] - t.size) < 1e-3 * t.size
    F[ky, kx] = 0
    assert np.abs(F).max() < 1e-4 * t.size
    rng = np.random.default_rng(0)
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    X = oracle_mod.fft(x)
    assert abs(np.sum(np.abs(X.astype(np.complex128)) ** 2) / x.size - np.sum(np.abs(x) ** 2)) < 1e-5 * np.sum(
        np.abs(x) ** 2)  # Parseval
    back = oracle_mod.fft(X, +1) / x.size
    assert np.abs(back - x).max() < 1e-5


# ---------------------------------------------------- known answers of the reference's tests
def test_module_projection_keeps_phase_sets_modulus(oracle_mod):
    """tests/ProjTests.c:4-30: modulus = measured amplitude, phase unchanged (2 eps)."""
    rng = np.random.default_rng(3)
    G = (rng.random((8, 8)) + 1j * rng.random((8, 8))).astype(np.complex64)
    amp = rng.random((8, 8)).astype(np.float32)
    flags = np.full((8, 8), 2, np.int32)
    P = oracle_mod.module_projection(G, amp, flags)
    eps = np.finfo(np.float32).eps
    assert np.all(np.abs(np.abs(P) - amp) <= 2 * eps * amp + 1e-12)
    assert np.all(np.abs(np.angle(P) - np.angle(G)) <= 2 * eps * np.abs(np.angle(G)) + 1e-7)
    # unmeasured pixels are left alone; a zero Fourier value takes the amplitude with zero phase
    flags[0, 0] = 0
    G[1, 1] = 0
    P = oracle_mod.module_projection(G, amp, flags)
    assert P[0, 0] == G[0, 0]
    assert P[1, 1] == np.complex64(amp[1, 1])


@pytest.mark.parametrize("shape,pos", [((11, 11), (5, 5)), ((11, 11, 11), (3, 5, 1))])
def test_blur_of_impulse_keeps_integral_and_argmax(oracle_mod, shape, pos):
    """tests/ImageTests.c:194-243: integral within 1.5e-4, maximum in place."""
    a = np.zeros(shape, np.complex64)
    a[pos] = 1
    b = oracle_mod.gaussian_blur(a, 1.0)
    assert abs(b.sum() - 1) <= 1.5e-4
    assert np.unravel_index(np.argmax(np.abs(b)), shape) == pos


def make_test_problem(rng, size=4, oversampling=2, constraints=2, beamstop=0):
    """tests/PhasingTests.c:405-436 + :14-31: a size^2 object in the corner of an
    oversampled grid, its |FFT| as amplitudes, the object's footprint as support."""
    n = size * oversampling
    obj = np.zeros((n, n), np.complex64)
    if constraints & 1:
        blk = rng.random((size, size)) - 0.5
    elif constraints & 2:
        blk = rng.random((size, size))
    elif constraints & 4:
        blk = rng.random((size, size)) + 1j * rng.random((size, size))
    else:
        blk = (rng.random((size, size)) - 0.5) + 1j * (rng.random((size, size)) - 0.5)
    obj[:size, :size] = blk
    F = np.abs(np.fft.fft2(obj.astype(np.complex128))).astype(np.float32)
    yy, xx = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    dy, dx = np.minimum(yy, n - 1 - yy), np.minimum(xx, n - 1 - xx)
    mask = (np.sqrt(dx * dx + dy * dy) >= beamstop).astype(np.int32)
    F[mask == 0] = 0
    support = (np.abs(obj) != 0).astype(np.float32)
    return F, mask, support


def converges(engine_factory, alg, constraints, beamstop, seed0, beta=0.8, tol=1e-10, max_iter=300, attempts=11):
    """tests/PhasingTests.c:10-59: iterate one at a time until sum |model change|^2 <= tol."""
    for attempt in range(attempts):
        rng = np.random.default_rng(seed0 + attempt)
        amp, mask, support = make_test_problem(rng, constraints=constraints, beamstop=beamstop)
        e = engine_factory((8, 8))
        e.set_algorithm(alg, beta=beta, constraints=constraints)
        if hasattr(e, "start"):
            e.start()
        e.set_amplitudes(amp, mask)
        assert e.init_model(1, seed=seed0 * 100 + attempt) == 0
        e.set_support(support)
        for _ in range(max_iter):
            assert e.iterate(1) == 0
            d = (e.get(1) - e.get(0)).astype(np.complex128)
            if np.sum(np.abs(d) ** 2) <= tol:
                return True
    return False


@pytest.mark.parametrize("alg", [HIO, RAAR])
@pytest.mark.parametrize("constraints,beamstop", [(2, 0), (1, 0), (4, 0), (4, 1), (2, 1)])
def test_small_object_converges(oracle_mod, alg, constraints, beamstop):
    assert converges(oracle_mod.Restatement, alg, constraints, beamstop, seed0=17)


from tests._engines import MORPH_SCENARIOS, setup_morph  # noqa: E402


@pytest.mark.parametrize("name,shape,alg,steps,shift,nit", MORPH_SCENARIOS, ids=[s[0] for s in MORPH_SCENARIOS])
def test_restatement_equals_reference_close_centre_template(oracle_mod, name, shape, alg, steps, shift, nit):
    """closing, centre-image and template support updates of the restatement
    against the reference's own CPU engine (src/support_update.c:44-125,
    193-390), bit for bit"""
    if not oracle_mod.ref_available():
        pytest.skip("reference CPU engine not built")
    ref, s0 = setup_morph(oracle_mod.Reference(shape), shape, alg, steps, shift)
    res, _ = setup_morph(oracle_mod.Restatement(shape), shape, alg, steps, shift)
    assert ref.iterate(nit) == 0 and res.iterate(nit) == 0
    assert np.array_equal(res.support(), ref.support())
    assert not np.array_equal(res.support(), (np.real(s0) != 0).astype(np.int32)), "support never changed"
    assert same_bits(res.model(), ref.model())


def _margin_or_phased_run(eng, shape, mode):
    """Amplitude margins (SpAmplitudeErrorMargin, src/phasing.c:1070-1100) or
    amplitude recovery from phased amplitudes (SpRecoverAmplitudes,
    src/phasing.c:1103-1109) on one engine."""
    from libspimage_b200 import synth

    amp, mask, support, obj = synth.small_pattern(shape, seed=2)
    rng = np.random.default_rng(5)
    eng.set_algorithm(HIO, beta=0.9, constraints=2 | (32 if mode == "margins" else 0))
    eng.add_support_update(AREA, 7, 2.0, 0.1)
    if hasattr(eng, "start"):
        eng.start()
    eng.set_amplitudes(amp, mask)
    if mode == "margins":
        eng.set_amplitudes_margins((amp * (1 - 0.2 * rng.random(shape))).astype(np.float32),
                                   (amp * (1 + 0.2 * rng.random(shape))).astype(np.float32))
    assert eng.init_model(1, seed=4) == 0
    if mode == "phased":
        pa = (np.fft.fftn(obj) * np.exp(2j * np.pi * 0.05 * rng.standard_normal(shape))).astype(np.complex64)
        eng.set_phased_amplitudes(pa, (rng.random(shape) < 0.7).astype(np.int32))
        eng.set_objective(1)
    eng.set_support(support)
    assert eng.iterate(25) == 0
    return eng


@pytest.mark.parametrize("mode", ["margins", "phased"])
@pytest.mark.parametrize("shape", [(32, 40), (8, 12, 10)])
def test_margins_and_phased_amplitudes_match_reference(oracle_mod, mode, shape):
    if not oracle_mod.ref_available():
        pytest.skip("reference engine not built here")
    a = _margin_or_phased_run(oracle_mod.Restatement(shape), shape, mode)
    b = _margin_or_phased_run(oracle_mod.Reference(shape), shape, mode)
    for w in (0, 1, 2):
        assert same_bits(a.get(w), b.get(w)), w
    assert np.array_equal(a.flags(), b.flags())
