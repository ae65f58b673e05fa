"""Shared test setup.  GPU tests are marked `gpu`; everything else runs on the CPU."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs through libtamm_b200.so")


def _ensure_built():
    lib = os.path.join(ROOT, "tamm_b200", "libtamm_b200.so")
    if not os.path.exists(lib):
        from tamm_b200 import build as b
        b.build()
    port = os.path.join(ROOT, "oracle", "liboracle_port.so")
    if not os.path.exists(port):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "port"], check=True)


_ensure_built()


@pytest.fixture(scope="session")
def ec():
    """One execution context (4 GiB arena) for the GPU tests of a session."""
    import tamm_b200 as tb
    ctx = tb.ExecutionContext(0, 4 << 30)
    yield ctx
    ctx.close()
