"""Test configuration: the ``gpu`` marker, import paths and in-tree builds.

Tests marked ``gpu`` need a B200 (they drive the CUDA library through its C
ABI); every other test runs on the CPU.
"""
import os
import sys

import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
HERE = os.path.abspath(os.path.dirname(__file__))
for _p in (ROOT, HERE):
    if _p not in sys.path:
        sys.path.insert(0, _p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the oracle and the CUDA library in-tree when missing."""
    import oracle

    if not os.path.exists(os.path.join(ROOT, "oracle", "_build", "libcavity_oracle.so")):
        oracle.build()
    lib = os.path.join(ROOT, "cfd_cavity_b200", "_build", "libcavity_b200.so")
    if not os.path.exists(lib):
        from cfd_cavity_b200 import build

        build.build()
    yield
