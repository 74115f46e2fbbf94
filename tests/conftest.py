"""Shared pytest configuration.

Tests marked ``gpu`` run the CUDA path (libmog.so) on a B200 and compare it
with the oracle; everything else runs on the CPU.
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs libmog.so against the oracle)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    oracle.build_oracle()
    return oracle
