"""The C-ABI boundary without a GPU: the library loads, exports every symbol
include/spimage/*.h declares, keeps the reference's struct layouts, and its
host-side checks return the reference's error codes."""
import ctypes as C
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def L():
    import libspimage_b200 as L

    if not os.path.exists(L.LIB_PATH):
        from libspimage_b200 import build

        build.build()
    L.load()
    return L


def test_every_declared_symbol_is_exported(L):
    names = L.exported_symbols()
    assert len(names) > 60
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True, check=True)
    defined = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    missing = [n for n in names if n not in defined]
    assert not missing, missing


def test_no_device_means_init_fails_loudly(L):
    lib = L.load()
    if lib.spb_device_count() > 0:
        pytest.skip("a CUDA device is present")
    ph = lib.sp_phaser_alloc()
    alg = lib.sp_phasing_hio_alloc(L.smap(0.9), 0)
    assert lib.sp_phaser_init(ph, alg, None, L.SpEngineCUDA) == -3
    assert b"no CUDA device" in lib.sp_phaser_last_error()
    assert lib.sp_phaser_init(ph, alg, None, L.SpEngineCPU) == -3
    assert b"GPU only" in lib.sp_phaser_last_error()
    lib.sp_phaser_free(ph)


def test_iterate_error_codes(L):
    """src/phasing.c:898-998: -1 NULL phaser, -2 no algorithm, -3 no model."""
    lib = L.load()
    assert lib.sp_phaser_iterate(None, 1) == -1
    ph = lib.sp_phaser_alloc()
    assert lib.sp_phaser_iterate(ph, 1) == -2
    assert lib.sp_phaser_init(ph, None, None, 0) == -2
    ph.contents.algorithm = lib.sp_phasing_er_alloc(0)
    assert lib.sp_phaser_iterate(ph, 1) == -3
    lib.sp_phaser_free(ph)


def test_dm_default_gammas(L, oracle_mod):
    """src/phasing.c:16-45 gammas at beta(0) when gamma1 is INFINITY."""
    lib = L.load()

    class DMParams(C.Structure):
        _fields_ = [("beta", C.c_void_p), ("gamma1", C.c_float), ("gamma2", C.c_float), ("constraints", C.c_int)]

    class Alg(C.Structure):
        _fields_ = [("type", C.c_int), ("params", C.POINTER(DMParams))]

    for beta in (0.7, 0.9):
        a = C.cast(lib.sp_phasing_diff_map_alloc(L.smap(beta), float("inf"), 0.0, 0), C.POINTER(Alg))
        p = a.contents.params.contents
        b = np.float32(beta)
        s = np.float32(0.1)
        g1 = -(np.float32(4) + (np.float32(2) + b) * s + b * s * s) / (b * (np.float32(4) - s + s * s))
        g2 = (np.float32(3) - b) / (np.float32(2) * b)
        assert np.float32(p.gamma1) == np.float32(g1)
        assert np.float32(p.gamma2) == np.float32(g2)
        k = np.array([0], np.float32)
        v = np.array([beta], np.float32)
        rs = oracle_mod._load_restatement()
        ph = rs.spo_create(4, 4, 1)
        rs.spo_set_algorithm(ph, 3, 1, oracle_mod._ptr(k), oracle_mod._ptr(v), float("inf"), 0.0, 0)
        assert np.float32(rs.spo_dm_gamma(ph, 1)) == np.float32(p.gamma1)
        rs.spo_destroy(ph)


PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "spimage.h"
#define P(T, f) printf(#T "." #f " %zu\n", offsetof(T, f));
int main(void) {
  printf("sizeof.Image %zu\n", sizeof(Image));
  printf("sizeof.Complex %zu\n", sizeof(Complex));
  P(Image, image) P(Image, mask) P(Image, detector) P(Image, shifted) P(Image, num_dimensions)
  P(SpPhaser, algorithm) P(SpPhaser, sup_algorithm) P(SpPhaser, iteration) P(SpPhaser, nx) P(SpPhaser, model)
  P(SpPhaser, model_change) P(SpPhaser, support) P(SpPhaser, fmodel) P(SpPhaser, engine) P(SpPhaser, g0)
  P(SpPhaser, g1) P(SpPhaser, gp)
  P(SpSupportAlgorithm, function) P(SpSupportArray, update_period) P(SpPhasingDiffMapParameters, gamma2)
  P(sp_smap, values) P(sp_list, size) P(Detector, orientation)
  return 0;
}
"""


def _probe(include_dirs, defines=()):
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        with open(src, "w") as f:
            f.write(PROBE)
        cmd = ["gcc", "-std=gnu99", "-w", "-o", exe, src] + [f"-I{i}" for i in include_dirs] + list(defines)
        subprocess.run(cmd, check=True, capture_output=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return dict(line.split() for line in out.splitlines())


def test_struct_layouts_match_reference_headers():
    import oracle

    root = oracle.reference_root()
    if root is None:
        pytest.skip("reference headers not present")
    ref_inc = os.path.join(root, "include")
    ours = _probe([os.path.join(ROOT, "include")])
    theirs = _probe([ref_inc, os.path.join(ref_inc, "spimage"), os.path.join(ROOT, "oracle", "stubs"),
                     os.path.join(ROOT, "oracle", "fftw_shim")], ["-D_SP_SINGLE_PRECISION"])
    assert ours == theirs
