"""The FP64 oracle (oracle/fp64.py) on the CPU: it follows the same algorithm
as the float32 restatement (which is pinned bit for bit to the reference
engine), so from the same start the two stay within float32 rounding of each
other; and it passes the reference's own convergence test
(tests/PhasingTests.c:10-59, 1040-1065: a 4x4 object oversampled twice
reconstructed to sum |model change|^2 <= 1e-10 within 300 iterations)."""
import numpy as np
import pytest

from tests._engines import AREA, DIFFMAP, ER, HIO, RAAR, THRESHOLD, setup

CASES = [
    ("hio_area", (48, 40), HIO, [(AREA, 5, {0: 3.0, 40: 0.7}, 0.1)], 2),
    ("raar", (32, 32), RAAR, None, 2),
    ("er_3d", (8, 16, 12), ER, [(AREA, 6, 1.5, 0.2)], 2),
    ("dm_area", (32, 32), DIFFMAP, [(AREA, 6, 2.0, 0.15)], 2),
    ("hio_thr_complex", (40, 24), HIO, [(THRESHOLD, 4, 2.0, 0.2)], 4),
    ("raar_flip_centro", (30, 30), RAAR, None, 2 | 8 | 16),
]

# float32 rounding over 10 iterations from the same start: rel. L2 of order
# 1e-7 per step, allowed 1e-5 in all
TOL_10 = 1e-5


def fp64_from(ref, shape, alg, sup, cons, beta=0.9):
    from oracle.fp64 import Fp64Phaser

    f = Fp64Phaser(shape)
    f.set_algorithm(alg, beta=beta, constraints=cons)
    for s in sup or []:
        f.add_support_update(*s)
    f.set_amplitudes(ref.amplitudes_np, (ref.flags() & 2) != 0)
    f.set_flags(ref.flags())
    f.set_model(ref.model(), iteration=ref.iteration)
    return f


@pytest.mark.parametrize("name,shape,alg,sup,cons", CASES, ids=[c[0] for c in CASES])
def test_fp64_oracle_tracks_float32_restatement(oracle_mod, name, shape, alg, sup, cons):
    from oracle.fp64 import rel_l2

    ref = setup(oracle_mod.Restatement(shape), shape, alg, sup, constraints=cons)
    f64 = fp64_from(ref, shape, alg, sup, cons)
    assert ref.iterate(10) == 0 and f64.iterate(10) == 0
    assert f64.iteration == ref.iteration == 10
    assert np.array_equal(f64.support(), ref.support())
    err = rel_l2(ref.model(), f64.model())
    assert 0 < err <= TOL_10, err
    ef32, _ = ref.efourier()
    ef64, _ = f64.efourier()
    assert abs(ef32 - ef64) <= 1e-4 * ef64


def _test_object(rng, size=4, oversampling=2, constraints=2):
    """create_test_image (tests/PhasingTests.c:405-436): a size x size object
    in the corner of a (size*oversampling)^2 image."""
    a = np.zeros((size * oversampling, size * oversampling), np.complex128)
    if constraints & 1:
        a[:size, :size] = rng.random((size, size)) - 0.5
    elif constraints & 2:
        a[:size, :size] = rng.random((size, size))
    elif constraints & 4:
        a[:size, :size] = rng.random((size, size)) + 1j * rng.random((size, size))
    else:
        a[:size, :size] = (rng.random((size, size)) - 0.5) + 1j * (rng.random((size, size)) - 0.5)
    return a


def converges(make_engine, constraints, beamstop, seed, tol=1e-10, max_iter=300, attempts=11):
    """test_sp_phasing_common (tests/PhasingTests.c:10-59): amplitudes of a
    random test object with a corner beamstop, support = the object's
    non-zero pixels, iterate one at a time until sum |model change|^2 <= tol."""
    rng = np.random.default_rng(seed)
    for _ in range(attempts):
        obj = _test_object(rng, constraints=constraints)
        amp = np.abs(np.fft.fft2(obj))
        n = obj.shape[0]
        i = np.arange(n)
        d = np.minimum(i, n - i).astype(np.float64)
        dist = np.sqrt(d[:, None] ** 2 + d[None, :] ** 2)
        mask = (dist >= beamstop).astype(np.int32)
        amp[mask == 0] = 0
        support = (obj != 0).astype(np.float32)
        eng, step = make_engine(obj.shape, amp, mask, support, int(rng.integers(1 << 30)))
        for _ in range(max_iter):
            change = step(eng)
            if change <= tol:
                return True
    return False


def test_fp64_oracle_passes_reference_convergence_test():
    from oracle.fp64 import HIO as H, Fp64Phaser

    def make(shape, amp, mask, support, seed):
        f = Fp64Phaser(shape)
        f.set_algorithm(H, beta=0.8, constraints=cons)
        f.set_amplitudes(amp, mask)
        f.set_support(support)
        r = np.random.default_rng(seed)
        f.set_model(np.fft.ifft2(amp * np.exp(2j * np.pi * r.random(shape))))

        def step(e):
            e.iterate(1)
            return float(np.sum(np.abs(e.g1 - e.g0) ** 2))

        return f, step

    for cons, beamstop in ((2, 0), (1, 0), (4, 0), (4, 1), (2, 1)):
        assert converges(make, cons, beamstop, seed=cons * 10 + beamstop), (cons, beamstop)
