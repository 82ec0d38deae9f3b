"""Shared pytest setup: import paths, the `gpu` marker and small helpers."""

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "threejs-particle-fluids_b200"
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build()
    O.lib()
    return O


@pytest.fixture(scope="session")
def pfsim():
    import pfsim as P

    P.lib()
    return P


@pytest.fixture(params=["slots", "tiles"])
def nbr_path(request, monkeypatch):
    """Runs a test on each fluid neighbour path (one thread per slot, warp
    tiles) instead of the one the autotuner would pick."""
    monkeypatch.setenv("PFSIM_NBR_PATH", "0" if request.param == "slots" else "1")
    return request.param
