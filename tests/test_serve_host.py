"""Host-side checks of the reconstruction server that need no GPU."""
import pytest

import libspimage_b200 as L


@pytest.fixture(scope="module")
def serve():
    L.load()
    from libspimage_b200 import serve

    return serve


def test_footprint_accounts_for_starts_and_difference_map(serve):
    n = 64 * 64
    one = serve.footprint((64, 64), 1)
    four = serve.footprint((64, 64), 4)
    assert one > 53 * n
    # per start: six complex buffers, |blur| and flags = 53 bytes per pixel, plus selection state
    assert four - one >= 3 * 53 * n
    assert serve.footprint((64, 64), 4, dm=True) - four == 2 * 8 * 4 * n
    assert serve.footprint((0, 64), 1) == -1


def test_server_needs_a_device(serve):
    if L.load().spb_device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError, match="no CUDA device"):
        serve.Server()


def test_job_structs_match_the_c_header(serve, tmp_path):
    """ctypes layouts of spb_job, spb_job_info and spb_server_config equal the
    C compiler's for include/spimage/serve.h"""
    import ctypes as C
    import os
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    fields = {"spb_job": serve.Job, "spb_job_info": serve.JobInfo, "spb_server_config": serve.ServerConfig}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "spimage/serve.h"', 'int main(void) {']
    for cname, py in fields.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "probe.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-o", str(exe), str(src), f"-I{os.path.join(root, 'include')}"], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, py in fields.items():
        assert got[(cname, "size")] == C.sizeof(py)
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
