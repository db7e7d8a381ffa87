"""Shared pytest set-up: markers, repository paths and the golden fixtures."""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ref_fixtures():
    """Golden vectors read from the reference's own unit tests."""
    with np.load(os.path.join(GOLDEN, "ref_fixtures.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def port():
    from oracle import oracle

    return oracle.port()


@pytest.fixture(scope="session")
def ref_lib():
    """The reference CPU library built from its sources, where it exists."""
    from oracle import oracle

    lib = oracle.ref()
    if lib is None:
        pytest.skip("reference CPU library not built on this machine")
    return lib


@pytest.fixture(scope="session")
def dpb():
    """The product package (CUDA extension loaded through its C-ABI)."""
    import __graft_entry__

    return __graft_entry__.load_package()
