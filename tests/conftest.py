"""Shared fixtures. GPU tests carry @pytest.mark.gpu and run only on a B200 box."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device (run with -m gpu)")
    config.addinivalue_line("markers", "slow: long CPU oracle runs")


@pytest.fixture(scope="session")
def kat():
    return json.loads((ROOT / "tests" / "golden" / "quadrature_kat.json").read_text())


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle

    oracle.load()
    return oracle


@pytest.fixture(scope="session")
def ctx():
    """CUDA context of the library (GPU tests only): fails loudly without the extension."""
    import dvr3d_b200

    c = dvr3d_b200.Context(0)
    yield c
    c.close()
