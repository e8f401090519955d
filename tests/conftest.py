import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU and the built libjlcgpu.so")
    config.addinivalue_line("markers", "slow: larger sizes (still minutes at most)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def ctx():
    """A libjlcgpu context on cuda:0.  GPU tests fail (not skip) when the
    library or the device is missing: the GPU route has no fallback."""
    import jlc_b200
    c = jlc_b200.Context(0)
    yield c
    c.close()
