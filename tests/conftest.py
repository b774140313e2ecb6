"""Test configuration: repository on sys.path, the `gpu` marker, shared fixtures."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a); the parity tests proper")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle

    pyoracle.lib()  # builds liboracle.so if needed
    return pyoracle


@pytest.fixture(scope="session")
def ref(oracle):
    if not oracle.ref_available():
        pytest.skip("reference checker oracle/_ref/xpir_ref not built (needs the reference sources)")
    return oracle


@pytest.fixture(scope="session")
def engine():
    """The CUDA engine on GPU 0.  A missing library is an error, not a skip: the engine
    has no CPU path.  Only the absence of a GPU (this container) skips."""
    import xpir_b200

    xpir_b200.lib()
    if xpir_b200.device_count() == 0:
        pytest.skip("no CUDA device")
    return xpir_b200
