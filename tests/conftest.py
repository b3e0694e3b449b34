"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
import os
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO / "oracle"))

import oracle as O  # noqa: E402  (test infrastructure: the checker)

pkg = O.load_package()  # the package binding, imported as `itlbm_b200`


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def itlbm():
    return pkg


@pytest.fixture(scope="session")
def oracle():
    return O


@pytest.fixture(scope="session")
def golden():
    import json
    d = REPO / "tests" / "golden"
    return {
        "lotes": json.loads((d / "lotes_subset.json").read_text()),
        "e0": json.loads((d / "e0_resultado.json").read_text()),
    }


@pytest.fixture(scope="session")
def gpu(itlbm):
    """The library with a usable device; GPU tests fail loudly when either is missing."""
    import ctypes
    L = itlbm.lib()
    n = ctypes.c_int(0)
    rc = L.itlbm_device_count(ctypes.byref(n))
    assert rc == 0 and n.value > 0, f"no CUDA device ({rc}): {L.itlbm_last_error().decode()}"
    return itlbm
