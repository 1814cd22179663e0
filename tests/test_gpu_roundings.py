"""The projection passes take |G| = sqrt(re^2 + im^2) and amp / |G| from a
branch-free evaluation in double precision rounded once to float; these
tests hold it to the IEEE intrinsics bit for bit: every float of the
square-root domain [2^-126, 2^126] (about 2.1e9 values), and a billion
pseudo-random quotients with the divisor in [2^-63, 2^63] and the dividend
any bit pattern (NaN results compare as NaN)."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def _fn():
    import libspimage_b200 as L

    so = L.load()
    f = so.spb_check_roundings
    f.restype = C.c_int
    f.argtypes = [C.c_uint, C.c_uint, C.c_ulonglong, C.c_ulonglong, C.POINTER(C.c_ulonglong),
                  C.POINTER(C.c_ulonglong)]
    return so, f


def _run(lo, hi, ndiv, seed):
    so, f = _fn()
    bs, bd = C.c_ulonglong(99), C.c_ulonglong(99)
    rc = f(lo, hi, ndiv, seed, C.byref(bs), C.byref(bd))
    assert rc == 0, so.spb_error_string()
    return bs.value, bd.value


def test_sqrt_every_float_of_the_domain():
    bad_sqrt, _ = _run(0x00800000, 0x7E800001, 0, 0)
    assert bad_sqrt == 0


@pytest.mark.parametrize("seed", [1, 2])
def test_quotients(seed):
    _, bad_div = _run(0, 0, 1 << 29, seed)
    assert bad_div == 0
