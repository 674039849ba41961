"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
import os
import subprocess
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "owt-krylov_b200")
for p in (REPO, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


def _ensure_product_built():
    lib = os.path.join(PKG, "lib", "libowtk_b200.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", PKG, "-j8"], check=True)


@pytest.fixture(scope="session")
def native():
    _ensure_product_built()
    from owtk_b200 import native as n
    n.lib()
    return n


@pytest.fixture(scope="session")
def problems(native):
    from owtk_b200 import problems as p
    return p


@pytest.fixture(scope="session")
def restatement():
    import oracle
    return oracle.Restatement()


@pytest.fixture(scope="session")
def reference():
    import oracle
    try:
        return oracle.Reference()
    except FileNotFoundError:
        pytest.skip("reference harness not built (oracle/_ref)")


@pytest.fixture(scope="session")
def golden():
    path = os.path.join(GOLDEN, "reference_small.npz")
    return dict(np.load(path, allow_pickle=False))


@pytest.fixture(scope="session")
def ctx(native):
    c = native.Context(0)
    yield c
    c.close()


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint64 if a.dtype == np.float64 else np.uint32)


def assert_bitwise(actual, expected, what=""):
    actual, expected = np.asarray(actual), np.asarray(expected)
    assert actual.shape == expected.shape, (what, actual.shape, expected.shape)
    same = bits(actual) == bits(expected)
    if not same.all():
        i = int(np.argmin(same))
        raise AssertionError(f"{what}: {int((~same).sum())} of {same.size} differ; first at {i}: "
                             f"{actual.flat[i]!r} vs {expected.flat[i]!r}")
