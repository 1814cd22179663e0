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
