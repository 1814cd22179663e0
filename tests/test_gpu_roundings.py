"""The projection passes take |G| = sqrt(re^2 + im^2) and amp / |G|, and the
support passes |g| and |blur|, from branch-free Newton-Raphson forms with
fused multiply-adds instead of the IEEE intrinsics' slow-path branches.
These tests hold them to the intrinsics bit for bit: every float of the
square-root domain [2^-126, 2^126] (about 2.1e9 values) and of the
reciprocal's [2^-63, 2^63]; a billion pseudo-random quotients over the
quotient's domain; and the quotients of significand pairs (every divisor
significand, every 64th dividend significand here; all 2^46 pairs with
a_stride=1, about a minute on a B200)."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def _run(lo, hi, ndiv, seed, a_stride):
    import libspimage_b200 as L

    so = L.load()
    f = so.spb_check_roundings
    f.restype = C.c_int
    f.argtypes = [C.c_uint, C.c_uint, C.c_ulonglong, C.c_ulonglong, C.c_uint, C.POINTER(C.c_ulonglong)]
    bad = (C.c_ulonglong * 4)(99, 99, 99, 99)
    rc = f(lo, hi, ndiv, seed, a_stride, bad)
    assert rc == 0, so.spb_error_string()
    return list(bad)


def test_sqrt_and_reciprocal_every_float_of_their_domains():
    bad = _run(0x00800000, 0x7E800001, 0, 0, 0)
    assert bad[0] == 0 and bad[1] == 0


@pytest.mark.parametrize("seed", [1, 2])
def test_random_quotients(seed):
    assert _run(0, 0, 1 << 29, seed, 0)[2] == 0


def test_quotients_of_significand_pairs():
    assert _run(0, 0, 0, 0, 64)[3] == 0
