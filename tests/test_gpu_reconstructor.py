"""Reconstructor driver on the GPU: a reconstruction equals the oracle
restatement run with the same schedule, and the batched reconstruct_loop
equals the reference's sequential loop."""
import numpy as np
import pytest

from libspimage_b200 import synth
from tests._engines import AREA, ER, HIO, same_bits

pytestmark = pytest.mark.gpu


def _configure(R, shape, n_hio=60, n_er=20, outputs=5):
    amp, mask, support, _ = synth.small_pattern(shape, seed=1)
    I = np.fft.fftshift(amp.astype(np.float64) ** 2)    # the driver takes a non-shifted pattern
    R.set_intensities(I)
    R.set_mask(np.fft.fftshift(mask != 0))
    R.set_number_of_iterations(n_hio + n_er)
    R.set_number_of_outputs(outputs)
    R.set_initial_support(radius=min(shape) / 8)
    R.set_support_algorithm("area", update_period=10, blur_init=3.0, blur_final=0.7, area_init=0.1,
                            area_final=0.05, center_image=False)
    R.append_phasing_algorithm("hio", number_of_iterations=n_hio, beta_init=0.95, beta_final=0.8,
                               constraints=["enforce_positivity", "enforce_real"])
    R.append_phasing_algorithm("er", number_of_iterations=n_er, constraints=["enforce_positivity", "enforce_real"])
    return amp, mask


def test_reconstruct_equals_oracle_schedule(lib, oracle_mod):
    from libspimage_b200.reconstructor import Reconstructor, initial_support_mask

    shape = (64, 48)
    R = Reconstructor()
    amp, mask = _configure(R, shape)
    lib.load().sp_srand(7)
    out = R.reconstruct()
    # the same schedule on the oracle: beta 0.95 -> 0.8 over iterations 0..60,
    # blur 3.0 -> 0.7 and area 0.1 -> 0.05 over 0..80
    amp_r = np.sqrt(np.fft.ifftshift(np.fft.fftshift(amp.astype(np.float64) ** 2)))
    ref = oracle_mod.Restatement(shape)
    ref.set_algorithm(HIO, beta={0: 0.95, 60: 0.8}, constraints=2)
    ref.add_support_update(AREA, 10, {0: 3.0, 80: 0.7}, {0: 0.1, 80: 0.05})
    ref.set_amplitudes(amp_r.astype(np.float32), mask != 0)
    assert ref.init_model(1, seed=7) == 0
    ref.set_support(initial_support_mask(shape, radius=min(shape) / 8))
    assert ref.iterate(60) == 0
    ref.set_algorithm(ER, constraints=2)
    assert ref.iterate(20) == 0
    assert list(out["iteration_index_images"]) == [0, 20, 40, 60, 80]
    assert same_bits(out["real_space"][-1].astype(np.complex64), np.fft.fftshift(ref.model_before_projection()))
    assert np.array_equal(out["support"][-1], np.fft.fftshift(ref.support()) != 0)
    ef, _ = ref.efourier()
    assert abs(out["fourier_error"][-1] - ef) <= 1e-3 * ef
    assert abs(out["support_size"][-1] - ref.support_fraction()) <= 1e-6


def test_reconstruct_loop_equals_sequential_loop(lib):
    from libspimage_b200.reconstructor import Reconstructor

    shape = (48, 48)
    R = Reconstructor()
    _configure(R, shape, n_hio=40, n_er=10, outputs=3)
    lib.load().sp_srand(11)
    seq = [R.reconstruct() for _ in range(3)]
    lib.load().sp_srand(11)
    loop = R.reconstruct_loop(3, full_output=True)
    for k in range(3):
        assert same_bits(loop["real_space_final"][k].astype(np.complex64), seq[k]["real_space"][-1].astype(np.complex64))
        assert np.array_equal(loop["support_final"][k], seq[k]["support"][-1])
        assert same_bits(loop["fourier_space_final"][k].astype(np.complex64),
                         seq[k]["fourier_space"][-1].astype(np.complex64))
        for key in ("fourier_error", "real_error"):
            a, b = loop["scores_final"][key][k], seq[k][key][-1]
            assert abs(a - b) <= 1e-5 * abs(b) + 1e-12
        assert loop["scores_final"]["support_size"][k] == seq[k]["support_size"][-1]
        # intermediate outputs too
        assert same_bits(loop["single_outputs"][k]["real_space"][1].astype(np.complex64),
                         seq[k]["real_space"][1].astype(np.complex64))
    assert not same_bits(loop["real_space_final"][0].astype(np.complex64),
                         loop["real_space_final"][1].astype(np.complex64))
