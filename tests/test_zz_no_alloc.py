"""spb_support_from_blur_noalloc (no device allocation, fixed file-scope
scratch) against spb_support_from_blur_host on the same inputs, called
through the C-ABI several times in a row so that each call runs on the
scratch contents the previous call left behind."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

AREA, THRESHOLD = 2, 1
MAX_PIXELS = 1 << 16


def _entry_points(lib):
    so = lib.load()
    fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int)
    for name in ("spb_support_from_blur_noalloc", "spb_support_from_blur_host"):
        f = getattr(so, name)
        f.restype = C.c_int
        f.argtypes = [C.c_longlong, fp, C.c_int, C.c_float, ip]
    return so


def _case(seed, shape, kind, value):
    rng = np.random.default_rng(seed)
    blur = (rng.random(shape) + 1j * rng.random(shape) * 1e-2).astype(np.complex64)
    blur.real[:3, :3] = 0.75  # ties
    flags = rng.integers(0, 16, size=shape).astype(np.int32)
    return blur, flags, kind, value


def _run(so, fn, blur, flags, kind, value):
    b = np.ascontiguousarray(blur, np.complex64)
    f = np.ascontiguousarray(flags, np.int32).copy()
    rc = getattr(so, fn)(b.size, b.ctypes.data_as(C.POINTER(C.c_float)), kind, value, f.ctypes.data_as(C.POINTER(C.c_int)))
    assert rc == 0, so.spb_error_string().decode()
    return f


def test_noalloc_matches_allocating_entry_point(lib):
    so = _entry_points(lib)
    cases = [
        _case(1, (256, 256), AREA, 0.05),     # the full scratch
        _case(2, (40, 50), THRESHOLD, 0.2),   # smaller: stale data past n
        _case(3, (100, 96), AREA, 0.3),
        _case(1, (256, 256), AREA, 0.05),     # the first case again
    ]
    results = []
    for blur, flags, kind, value in cases:
        want = _run(so, "spb_support_from_blur_host", blur, flags, kind, value)
        got = _run(so, "spb_support_from_blur_noalloc", blur, flags, kind, value)
        assert np.array_equal(got, want)
        assert np.any(got & 1) and not np.all(got & 1)
        results.append(got)
    assert np.array_equal(results[0], results[3])


def test_noalloc_rejects_sizes_beyond_its_scratch(lib):
    so = _entry_points(lib)
    n = MAX_PIXELS + 1
    blur = np.zeros(n, np.complex64)
    flags = np.zeros(n, np.int32)
    rc = so.spb_support_from_blur_noalloc(n, blur.ctypes.data_as(C.POINTER(C.c_float)), AREA, 0.1,
                                          flags.ctypes.data_as(C.POINTER(C.c_int)))
    assert rc == -1
    assert "65536-pixel limit" in so.spb_error_string().decode()


def _device_free_bytes():
    """Free device memory as the driver reports it (cuMemGetInfo on the
    context the library's calls made current on this thread)."""
    cu = C.CDLL("libcuda.so.1")
    free, total = C.c_size_t(), C.c_size_t()
    rc = cu.cuMemGetInfo_v2(C.byref(free), C.byref(total))
    assert rc == 0, f"cuMemGetInfo_v2 returned {rc}"
    return free.value


def test_noalloc_leaves_device_memory_unchanged(lib):
    """The property the entry point exists for: once its kernels are loaded
    and the scratch address is known (a first call of each case), further
    calls of interleaved sizes and kinds take no device memory."""
    so = _entry_points(lib)
    cases = [_case(4, (256, 256), AREA, 0.05), _case(5, (17, 31), THRESHOLD, 0.4), _case(6, (128, 200), AREA, 0.2)]
    for c in cases:
        _run(so, "spb_support_from_blur_noalloc", *c)
    before = _device_free_bytes()
    outs = {}
    for rep in range(3):
        for k in (2, 0, 1, 0, 2):
            got = _run(so, "spb_support_from_blur_noalloc", *cases[k])
            if k in outs:
                assert np.array_equal(got, outs[k])
            outs[k] = got
    assert _device_free_bytes() == before
