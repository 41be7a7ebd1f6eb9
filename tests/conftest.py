import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running check")


@pytest.fixture(scope="session")
def oracle():
    from oracle_lib import oracle_library
    return oracle_library()


@pytest.fixture(scope="session")
def engine():
    from coffee_sim_b200.sim import engine_library
    return engine_library()
