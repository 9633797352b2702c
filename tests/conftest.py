import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def rsb():
    """The product package (C ABI through ctypes). The library must already be built
    (__graft_entry__.build()); loading fails loudly otherwise."""
    pkg = __graft_entry__.load_package()
    pkg.load()
    return pkg


@pytest.fixture(scope="session")
def O():
    """The CPU oracle (test infrastructure)."""
    from oracle import oracle

    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def golden():
    import json

    with open(os.path.join(ROOT, "tests", "golden", "reference_vectors.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def gpu(rsb):
    """GPU tests run only where a device exists; they fail (not skip) without one."""
    if rsb.device_check() != 0:
        raise RuntimeError("GPU test selected but no usable CUDA device")
    return rsb
