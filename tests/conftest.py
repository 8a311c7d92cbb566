import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libaxon_b200.so")
    config.addinivalue_line("markers", "slow: minutes of CPU time (full-geometry oracle runs); set AXON_SLOW=1 to run")


def pytest_collection_modifyitems(config, items):
    """Full-geometry oracle regenerations of committed fixtures run only with AXON_SLOW=1,
    so the default CPU suite stays within a few minutes."""
    if os.environ.get("AXON_SLOW") == "1":
        return
    skip = pytest.mark.skip(reason="full-geometry oracle run; set AXON_SLOW=1")
    for item in items:
        if "slow" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    import oracle_lib

    return oracle_lib.load()
