"""Random-phase starts on the host (sp_image_rephase, the reference's
src/image_util.c:1035-1067): the values come from the C library's rand()
sequence and libm's double cos/sin exactly as the reference computes them
one pixel at a time, although this library draws the sequence in bulk from
the generator's state -- each host thread jumping ahead to its own span of
pixels -- and evaluates cos/sin on those threads; and rand() continues
afterwards as if it had been called once per pixel.  Sizes cover draws
shorter than the generator's 31-word state, one thread, and uneven spans
over all host threads."""
import ctypes as C

import numpy as np
import pytest

SP_RANDOM_PHASE = 2
RAND_MAX = 2147483647


@pytest.fixture(scope="module")
def env():
    import libspimage_b200 as L

    so = L.load()
    so.sp_image_rephase.argtypes = [C.c_void_p, C.c_int]
    libc = C.CDLL("libc.so.6")
    libm = C.CDLL("libm.so.6")
    for f in (libm.cos, libm.sin):
        f.restype = C.c_double
        f.argtypes = [C.c_double]
    return L, so, libc, libm


def _expected(libc, libm, amp, seed, skip):
    """one rand() per pixel, cos/sin of the float phase in double, as the reference"""
    libc.srand(seed)
    for _ in range(skip):
        libc.rand()
    out = np.empty(amp.size, np.complex64)
    for i, a in enumerate(amp.ravel()):
        p = np.float32(float(libc.rand()) / RAND_MAX)
        phase = np.float32(float(p) * 3.14159265358979323846 * 2)
        av = float(np.sqrt(np.float32(a) * np.float32(a) + np.float32(0.0) * np.float32(0.0), dtype=np.float32))
        out[i] = complex(np.float32(libm.cos(float(phase)) * av), np.float32(libm.sin(float(phase)) * av))
    return out, libc.rand()


@pytest.mark.parametrize("shape,seed,skip", [((16, 16), 3, 0), ((300, 300), 11, 5), ((1, 70001), 0, 31),
                                             ((1, 7), 2, 1), ((1, 30), 4, 40), ((257, 263), 9, 2)])
def test_rephase_matches_per_pixel_draws(env, shape, seed, skip):
    L, so, libc, libm = env
    amp = (np.random.default_rng(seed).random(shape) * 4).astype(np.float32)
    img = L.new_image(amp.astype(np.complex64))
    try:
        libc.srand(seed)
        for _ in range(skip):
            libc.rand()
        so.sp_image_rephase(C.cast(img, C.c_void_p), SP_RANDOM_PHASE)
        after = libc.rand()
        n = amp.size
        fp = C.cast(img.contents.image.contents.data, C.POINTER(C.c_float))
        got = np.ctypeslib.as_array(fp, shape=(2 * n,)).copy().view(np.complex64)
    finally:
        L.free_image(img)
    exp, exp_after = _expected(libc, libm, amp, seed, skip)
    assert np.array_equal(got.view(np.uint32), exp.view(np.uint32))
    assert after == exp_after


def test_concurrent_rephase_keeps_the_generator(env):
    """Host threads rephasing at once (ctypes releases the GIL during the
    call) must not leave the C library's generator on the bulk draw's
    stand-in state: afterwards sp_srand(s) gives glibc's own sequence."""
    import threading

    L, so, libc, libm = env
    libc.srand(123)
    want = [libc.rand() for _ in range(64)]
    # many short calls from eight threads: the swaps of the generator state
    # overlap thousands of times (without the lock this lost the generator
    # on every run)
    imgs = [L.new_image((np.random.default_rng(k).random((32, 32))).astype(np.complex64)) for k in range(8)]
    errors = []

    def work(img):
        try:
            for _ in range(20000):
                so.sp_image_rephase(C.cast(img, C.c_void_p), SP_RANDOM_PHASE)
        except Exception as e:  # pragma: no cover
            errors.append(e)

    try:
        th = [threading.Thread(target=work, args=(im,)) for im in imgs]
        for t in th:
            t.start()
        for t in th:
            t.join()
    finally:
        for im in imgs:
            L.free_image(im)
    assert not errors
    so.sp_srand(123)
    assert [libc.rand() for _ in range(64)] == want


@pytest.mark.parametrize("n,seed,skip", [(5, 1, 0), (40, 3, 7), (600000, 8, 2)])
def test_uniform_draw_matches_rand(env, n, seed, skip):
    """The p_drand48() values of a random-values start (two per pixel), drawn
    on the host threads by jumping ahead in the generator, equal n calls of
    rand() / RAND_MAX, and rand() continues where those calls leave it."""
    L, so, libc, libm = env
    so.spb_random_uniforms.argtypes = [C.c_void_p, C.c_longlong]
    libc.srand(seed)
    for _ in range(skip):
        libc.rand()
    got = np.empty(n, np.float32)
    so.spb_random_uniforms(got.ctypes.data, n)
    after = libc.rand()
    libc.srand(seed)
    for _ in range(skip):
        libc.rand()
    want = np.array([np.float32(float(libc.rand()) / RAND_MAX) for _ in range(n)], np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert after == libc.rand()


def test_concurrent_bulk_draws_take_whole_blocks(env):
    """Large draws run their spans on the library's pool of host threads; a
    draw that finds the pool busy with another thread's draw runs on threads
    of its own.  Either way each draw is one whole block of the sequence: the
    outputs of concurrent draws are consecutive blocks of n values, in the
    order the draws took the generator."""
    import threading

    L, so, libc, libm = env
    so.spb_random_uniforms.argtypes = [C.c_void_p, C.c_longlong]
    n, threads, calls = 300000, 4, 2
    libc.srand(77)
    want = np.empty(n * threads * calls, np.float32)
    so.spb_random_uniforms(want.ctypes.data, want.size)
    blocks = {want[k * n:(k + 1) * n].tobytes(): k for k in range(threads * calls)}
    libc.srand(77)
    outs = [[np.empty(n, np.float32) for _ in range(calls)] for _ in range(threads)]

    def work(t):
        for c in range(calls):
            so.spb_random_uniforms(outs[t][c].ctypes.data, n)

    th = [threading.Thread(target=work, args=(t,)) for t in range(threads)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    got = sorted(blocks.get(o.tobytes(), -1) for row in outs for o in row)
    assert got == list(range(threads * calls))


@pytest.mark.filterwarnings("ignore:This process .* is multi-threaded")
def test_bulk_draw_in_forked_child(env):
    """A child forked after the pool's threads exist (they are not copied
    into it) draws on a fresh pool of its own."""
    import os
    import time

    L, so, libc, libm = env
    so.spb_random_uniforms.argtypes = [C.c_void_p, C.c_longlong]
    n = 400000
    warm = np.empty(n, np.float32)
    so.spb_random_uniforms(warm.ctypes.data, n)  # the pool exists in this process now
    libc.srand(5)
    want = np.empty(n, np.float32)
    so.spb_random_uniforms(want.ctypes.data, n)
    pid = os.fork()
    if pid == 0:  # child: no pytest machinery, exit status only
        try:
            libc.srand(5)
            got = np.empty(n, np.float32)
            so.spb_random_uniforms(got.ctypes.data, n)
            os._exit(0 if np.array_equal(got.view(np.uint32), want.view(np.uint32)) else 3)
        except BaseException:
            os._exit(4)
    deadline = time.time() + 60
    while True:
        done, status = os.waitpid(pid, os.WNOHANG)
        if done:
            break
        if time.time() > deadline:
            os.kill(pid, 9)
            os.waitpid(pid, 0)
            pytest.fail("the forked child's draw did not finish")
        time.sleep(0.05)
    assert os.WIFEXITED(status) and os.WEXITSTATUS(status) == 0, status


def test_parallel_for_spans_partition_the_range(env):
    """spb_parallel_for (the host loops of set_amplitudes, init_support and the
    flag conversions) runs fn over contiguous spans that cover [0, n) exactly
    once, on the pool or, when another caller holds the pool, on threads of
    its own; two callers at once both get whole partitions."""
    import threading

    L, so, libc, libm = env
    SPAN = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_longlong, C.c_longlong)
    so.spb_parallel_for.argtypes = [C.c_longlong, SPAN, C.c_void_p]
    so.spb_parallel_for.restype = C.c_int
    results = {}

    def run(key, n):
        got = []
        lock = threading.Lock()

        def fn(ctx, t, i0, i1):
            with lock:
                got.append((t, i0, i1))

        cb = SPAN(fn)
        spans = so.spb_parallel_for(n, cb, None)
        results[key] = (spans, sorted(got, key=lambda s: s[1]), n)

    for n in (5, 1 << 18, 1000003):
        run(n, n)
    th = [threading.Thread(target=run, args=(f"c{k}", 600000 + k)) for k in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for key, (spans, got, n) in results.items():
        assert 1 <= spans <= 8 and len(got) == spans, key
        assert sorted(t for t, _, _ in got) == list(range(spans)), key
        assert got[0][1] == 0 and got[-1][2] == n, key
        assert all(a[2] == b[1] for a, b in zip(got, got[1:])), key
