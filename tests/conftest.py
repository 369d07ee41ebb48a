"""Test configuration: the `gpu` marker, and one-time builds of the native
library and of the CPU oracle (test infrastructure)."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) GPU")


@pytest.fixture(scope="session", autouse=True)
def _built():
    from bowshock_b200 import build
    from oracle import oracle

    build.build()
    oracle.build()
    yield
