import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libaxon_b200.so")
    config.addinivalue_line("markers", "slow: minutes of CPU time (full-geometry oracle runs)")


@pytest.fixture(scope="session")
def oracle():
    import oracle_lib

    return oracle_lib.load()
