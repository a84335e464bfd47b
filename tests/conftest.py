"""Test configuration: registers the `gpu` marker and exposes the package and the oracle.

`shakti_b200` is the package directory shakti.jl_b200/; `shakti_oracle` is oracle/oracle.py (the
CPU restatement used as the test oracle)."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

import __graft_entry__ as _entry  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 and the built libshakti_b200.so")


@pytest.fixture(scope="session")
def shk():
    return _entry.load_package()


@pytest.fixture(scope="session")
def orc():
    o = _entry.load_oracle()
    o.build()
    return o


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("this test needs a GPU (marked gpu)")
    return torch
