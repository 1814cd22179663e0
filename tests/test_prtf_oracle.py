"""The PRTF oracle (the reference's algorithm over its own C routines): sanity on the CPU."""
import numpy as np
import pytest

from tests._prtf_cases import reconstructions


@pytest.fixture(scope="module")
def prtf_ref(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference CPU engine not built")
    from oracle.prtf import prtf_reference

    return prtf_reference


def test_identical_reconstructions_give_one(prtf_ref):
    ims, sups = reconstructions((32, 32), n=1)
    out = prtf_ref(np.repeat(ims, 4, axis=0), np.repeat(sups, 4, axis=0))
    assert np.allclose(out["prtf"], 1.0, atol=1e-6)


def test_alignment_recovers_shifted_phased_and_mirrored_copies(prtf_ref):
    ims, sups = reconstructions((32, 40), n=6)
    aligned = prtf_ref(ims, sups)
    raw = prtf_ref(ims, sups, translate=False)
    assert aligned["prtf"].mean() > 0.99
    assert raw["prtf"].mean() < 0.8
