import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def mf():
    import __graft_entry__
    return __graft_entry__.load_package()


@pytest.fixture(scope="session")
def ref():
    from oracle import mfref
    return mfref


@pytest.fixture
def rng():
    return np.random.default_rng(0x5EED)


def bits(x):
    return np.ascontiguousarray(x).view(np.uint64)


def assert_bitwise(got, want, what=""):
    g, w = bits(got), bits(want)
    if not np.array_equal(g, w):
        bad = np.argwhere(g != w)
        raise AssertionError(f"{what}: {len(bad)} limbs differ bitwise, first at {bad[0].tolist()}: "
                             f"got {np.ascontiguousarray(got).flat[np.ravel_multi_index(bad[0], g.shape)]!r} "
                             f"want {np.ascontiguousarray(want).flat[np.ravel_multi_index(bad[0], w.shape)]!r}")
