"""Shared pytest configuration.

Tests marked ``gpu`` run the CUDA path (libmog.so) on a B200 and compare it
with the oracle; everything else runs on the CPU.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs libmog.so against the oracle)")


# The core parity suites run first: their kernels carry the force-and-step
# path, and under -x a failure in a later feature suite must not hide them.
# test_zz_no_alloc stays last (it checks the process's allocator state).
_FIRST = ("test_gpu_parity.py", "test_golden_gpu.py", "test_batch_gpu.py", "test_learned_gpu.py",
          "test_dft_tc_gpu.py")


def pytest_collection_modifyitems(session, config, items):
    def rank(item):
        name = Path(str(item.fspath)).name
        if name in _FIRST:
            return (0, _FIRST.index(name))
        if name.startswith("test_zz_"):
            return (2, 0)
        return (1, 0)

    items.sort(key=rank)  # stable: the order inside each file is kept


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    oracle.build_oracle()
    return oracle
