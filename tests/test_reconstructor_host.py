"""Reconstructor driver: configuration, cadence and support geometry (no GPU)."""
import numpy as np

from libspimage_b200.reconstructor import Reconstructor, initial_support_mask, output_iterations, phasing_constraints


def test_output_cadence_as_the_reference():
    # np.linspace(0, N, n).round() as int64 (src/_spimage_reconstructor.py:443-444)
    assert list(output_iterations(1000, 11)) == list(range(0, 1001, 100))
    assert list(output_iterations(10, 4)) == [0, 3, 7, 10]
    assert list(output_iterations(5, 1)) == [0]


def test_initial_support_disc_is_centred_on_the_corner():
    s = initial_support_mask((64, 48), radius=10)
    assert s.dtype == np.float32 and s[0, 0] == 1 and s[32, 24] == 0
    ys = np.fft.fftshift(s)
    cy, cx = np.argwhere(ys > 0).mean(axis=0)
    assert abs(cy - 31.5) < 1e-6 and abs(cx - 23.5) < 1e-6
    area = initial_support_mask((128, 128), area=0.05)
    assert abs(area.mean() - 0.05) < 0.005
    v = initial_support_mask((16, 20, 24), radius=5)
    assert v.shape == (16, 20, 24) and v[0, 0, 0] == 1
    m = np.zeros((8, 8), bool)
    m[2, 3] = True
    assert np.array_equal(initial_support_mask((8, 8), support_mask=m), m.astype(np.float32))


def test_constraint_strings():
    assert phasing_constraints(["enforce_positivity", "enforce_real"]) == 2
    assert phasing_constraints(["enforce_real"]) == 1
    assert phasing_constraints(["enforce_positivity"]) == 4
    assert phasing_constraints(["enforce_real", "enforce_centrosymmetry"]) == 1 | 16
    assert phasing_constraints("") == 0


def test_incomplete_configuration_returns_none():
    R = Reconstructor()
    assert R.reconstruct() is None
    R.set_intensities(np.ones((16, 16)))
    R.set_number_of_iterations(10)
    R.set_number_of_outputs(2)
    R.set_initial_support(radius=3)
    R.set_support_algorithm("area", update_period=5, blur_init=2., blur_final=1., area_init=.1, area_final=.1)
    assert R.reconstruct() is None                     # no phasing algorithm
    R.set_phasing_algorithm("hio", beta_init=0.9)      # beta_final missing: rejected
    assert R._phasing_stages == []
    R.append_phasing_algorithm("hio", number_of_iterations=6, beta_init=.9, beta_final=.9)
    assert R.reconstruct() is None                     # 6 of 10 iterations covered
    R.append_support_algorithm("threshold", number_of_iterations=5, update_period=5, blur_init=2.)
    assert len(R._support_stages) == 1     # missing arguments: rejected


def test_negative_intensities_and_shift():
    R = Reconstructor()
    I = np.arange(16.).reshape(4, 4) - 3
    R.set_intensities(I)
    A = np.sqrt(np.clip(I, 0, None))
    assert np.array_equal(R._amplitudes, np.fft.fftshift(A))
    R.set_intensities(I, shifted=True)
    assert np.array_equal(R._amplitudes, A)
