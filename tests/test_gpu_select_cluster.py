"""The support update's selection and mask against the oracle: the k-th
largest |blur| (src/support_update.c:136-151, descending index (int)(N*area))
and the threshold rule (maximum times the fraction,
src/support_update.c:153-179), then the strict '>' mask
(src/support_update.c:392-400).  The host entry point (one launch per radix
pass and one for the mask) over sizes from one pixel to above the cluster
form's limit; phaser runs with the cluster form (knob 2: one launch over a
cluster of thread blocks per start exchanging histograms through distributed
shared memory, where a start's |blur| fits: up to 327,680 pixels) and the
launch-per-pass form, against the oracle.  Shapes give slices of unequal
length (17x19, 5x7x9) and batched starts."""
import numpy as np
import pytest

from libspimage_b200 import synth
from tests._engines import AREA, HIO, RAAR, THRESHOLD
from tests.test_gpu_parity_large import assert_same_state, setup_pattern

pytestmark = pytest.mark.gpu

SELECT = 8   # tuning knob: 2 = the cluster form where it fits, 1 (or 0) = one launch per radix pass and one for the mask
PERSIST = 4  # tuning knob: 1 = the two-pass kernels


def _abs_ref(blur):
    # |.| exactly as the reference: sqrt(im*im + re*re) in float
    return np.sqrt((blur.imag * blur.imag + blur.real * blur.real).astype(np.float32))


@pytest.mark.parametrize("n", [1, 7, 9, 1000, 65536 + 5, 262144, 327680, 327681])
@pytest.mark.parametrize("area", [0.05, 0.3333])
def test_area_select_sizes(lib, oracle_mod, n, area):
    rng = np.random.default_rng(n)
    blur = (rng.random(n) + 1j * rng.random(n) * 1e-3).astype(np.complex64)
    blur.real[: min(n, 16)] = 0.5  # ties at the threshold
    blur.real[n // 2: n // 2 + min(n, 40)] = 0.25
    flags = rng.integers(0, 4, size=n).astype(np.int32)
    t = oracle_mod.area_threshold(blur.reshape(1, n), area)
    want = (flags & ~1) | (_abs_ref(blur) > np.float32(t)).astype(np.int32)
    got = lib.support_from_blur(blur, AREA, area, flags)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n", [1, 7, 4099, 327680, 327681])
def test_threshold_select_sizes(lib, n):
    rng = np.random.default_rng(n + 1)
    blur = rng.random(n).astype(np.complex64)
    flags = rng.integers(0, 4, size=n).astype(np.int32)
    a = _abs_ref(blur)
    want = (flags & ~1) | (a > np.float32(a.max() * np.float32(0.2))).astype(np.int32)
    got = lib.support_from_blur(blur, THRESHOLD, 0.2, flags)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("select", [2, 1], ids=["cluster", "per-pass"])
@pytest.mark.parametrize("shape,alg,sup,starts", [
    ((256, 256), HIO, (AREA, 7, {0: 3.0, 50: 0.7}, 0.05), None),
    ((512, 512), RAAR, (AREA, 9, 2.0, 0.1), 4),
    ((192, 192), HIO, (THRESHOLD, 6, 1.5, 0.2), None),
    ((48, 40, 36), RAAR, (AREA, 5, 1.5, 0.2), 3),
    ((17, 19), HIO, (AREA, 4, 1.0, 0.3), 2),
    ((5, 7, 9), RAAR, (THRESHOLD, 5, 1.0, 0.25), None),
])
def test_phaser_support_updates_bit_exact(lib, oracle_mod, shape, alg, sup, starts, select):
    pat = synth.make_pattern(shape, min(shape) // 4, 1e7, max(1.0, min(shape) / 32.0), seed=17)
    seeds = list(range(40, 40 + starts)) if starts else None
    gpu = setup_pattern(lib.Phaser(shape), pat, alg, 0.87, [sup], seed=40, starts=seeds)
    gpu.set_tuning(SELECT, select)
    gpu.set_tuning(PERSIST, 1)
    assert gpu.iterate(21) == 0
    for k in ([0, starts - 1] if starts else [None]):
        ref = setup_pattern(oracle_mod.Restatement(shape, threads=8), pat, alg, 0.87, [sup], seed=40 + (k or 0))
        assert ref.iterate(21) == 0
        assert_same_state(gpu, ref, start=k)


@pytest.mark.parametrize("sup", [(AREA, 6, 2.0, 0.1), (THRESHOLD, 6, 1.5, 0.2)], ids=["area", "threshold"])
def test_large_batch_streaming_select_bit_exact(lib, oracle_mod, sup):
    """300 starts of 128x128: two blocks per start, so each thread of the
    histogram and mask launches streams many keys and takes them four at a
    time (16-byte loads); starts 0 and 299 against the oracle."""
    shape, starts = (128, 128), 300
    pat = synth.make_pattern(shape, 32, 1e7, 4.0, seed=23)
    seeds = list(range(60, 60 + starts))
    gpu = setup_pattern(lib.Phaser(shape), pat, HIO, 0.9, [sup], seed=60, starts=seeds)
    gpu.set_tuning(PERSIST, 1)
    assert gpu.iterate(13) == 0
    for k in (0, starts - 1):
        ref = setup_pattern(oracle_mod.Restatement(shape, threads=8), pat, HIO, 0.9, [sup], seed=60 + k)
        assert ref.iterate(13) == 0
        assert_same_state(gpu, ref, start=k)
