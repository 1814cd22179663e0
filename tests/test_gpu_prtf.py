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


# ---- the reference's C PRTF (src/prtf.c) and fractional superposition
# (src/image_util.c:3024-3066) against the same functions in the reference
# build.  sp_prtf_basic is bit-exact; the superposition's correlation peak
# (translation and enantiomorph choice) is decided from bit-identical
# surfaces, and its Fourier translation and phase shift evaluate cos/sin/atan2
# in double on the GPU, so the superimposed images agree within 1e-5 relative
# L2 and the PRTFs within 1e-5 absolute.

@pytest.fixture(scope="module")
def cref(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("reference CPU engine not built")
    from oracle import prtf as op

    return op


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


@pytest.mark.parametrize("shape", [(32, 40), (24, 24), (8, 12, 10)])
@pytest.mark.parametrize("flags", [0, 1, 2, 3])
@pytest.mark.parametrize("precision", [1, 2, 4])
def test_superimpose_fractional_matches_reference(lib, cref, shape, flags, precision):
    from libspimage_b200.prtf import superimpose_fractional

    ims, _ = reconstructions(shape, n=4, seed=len(shape) * 7 + flags)
    for k in (1, 2):  # image 2 of 4 is the reflected one
        want = cref.superimpose_fractional(ims[0], ims[k], flags, precision)
        got = superimpose_fractional(ims[0], ims[k], flags, precision)
        assert _rel(got, want) <= 1e-5, (k, _rel(got, want))


@pytest.mark.parametrize("shape,n", [((32, 40), 5), ((16, 16, 12), 3)])
def test_prtf_basic_bit_exact(lib, cref, shape, n):
    from libspimage_b200.prtf import prtf_basic

    ims, _ = reconstructions(shape, n=n, seed=3)
    specs = np.array([np.fft.fftn(im) for im in ims], np.complex64)
    specs[1][0] = 0  # a pixel where one spectrum vanishes
    specs[:, -1] = 0  # and one where all do (the sum stays)
    want = cref.prtf_basic(specs)
    got = prtf_basic(specs)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("shape,n", [((32, 40), 5), ((24, 24), 4), ((8, 12, 10), 3)])
@pytest.mark.parametrize("fourier_space", [True, False])
def test_prtf_advanced_matches_reference(lib, cref, shape, n, fourier_space):
    from libspimage_b200.prtf import prtf_advanced

    ims, _ = reconstructions(shape, n=n, seed=n + 11)
    inputs = np.array([np.fft.fftn(im) for im in ims], np.complex64) if fourier_space else ims
    flags = (1 if fourier_space else 2) | 65536  # SpInPlace
    want, want_after = cref.prtf_advanced(inputs, flags)
    got, got_after = prtf_advanced(inputs, fourier_space=fourier_space, in_place=True)
    assert np.abs(got - want).max() <= 1e-5
    for g, w in zip(got_after, want_after):
        assert _rel(g, w) <= 1e-5
    # the superimposed reconstructions agree: a PRTF near one at low frequencies
    assert np.abs(got).ravel()[0] > 0.99


def test_prtf_image_api(lib, cref):
    """sp_prtf_basic through the Image-level C API (Image ** in, Image * out)."""
    import ctypes as C

    import libspimage_b200 as L

    so = L.load()
    so.sp_prtf_basic.restype = C.POINTER(L.Image)
    so.sp_prtf_basic.argtypes = [C.POINTER(C.POINTER(L.Image)), C.c_int]
    ims, _ = reconstructions((20, 24), n=3, seed=5)
    specs = np.array([np.fft.fftn(im) for im in ims], np.complex64)
    imgs = [L.new_image(s) for s in specs]
    arr = (C.POINTER(L.Image) * 3)(*imgs)
    out = so.sp_prtf_basic(arr, 3)
    got = L.image_data(out, (20, 24))
    want = cref.prtf_basic(specs)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    L.free_image(out)
    for im in imgs:
        L.free_image(im)
