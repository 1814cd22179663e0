"""PRTF on the GPU against the oracle (the reference's algorithm over its own
C routines).  Translations and reflections come from bit-identical
correlation maps; the phase matching evaluates atan2/cos/sin on the GPU and
sums in double, so values agree to rounding: PRTF within 1e-4 absolute, the
superimposed image within 1e-4 relative L2, the mask exactly."""
import numpy as np
import pytest

from tests._prtf_cases import reconstructions

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def prtf_ref(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference CPU engine not built")
    from oracle.prtf import prtf_reference

    return prtf_reference


@pytest.mark.parametrize("shape,n,translate", [((32, 40), 6, True), ((48, 48), 9, True), ((32, 40), 6, False),
                                               ((12, 16, 14), 5, True)])
def test_prtf_matches_reference(lib, prtf_ref, shape, n, translate):
    from libspimage_b200.prtf import prtf

    ims, sups = reconstructions(shape, n=n, seed=n)
    want = prtf_ref(ims, sups, translate=translate)
    got = prtf(ims, sups, translate=translate, full_out=True)
    assert np.abs(got["prtf"] - want["prtf"]).max() <= 1e-4
    err = np.linalg.norm(got["super_image"] - want["super_image"]) / np.linalg.norm(want["super_image"])
    assert err <= 1e-4
    assert np.array_equal(got["super_mask"], want["super_mask"])
    if translate:
        assert got["prtf"].mean() > 0.99
    # the first shell is the centre pixel (shape[0]//2 on every axis)
    assert got["prtf_r"].ndim == 1
    assert abs(got["prtf_r"][0] - got["prtf"][(shape[0] // 2,) * len(shape)]) < 1e-6
