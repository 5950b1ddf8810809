import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def sq():
    """The engine package (GPU tests only)."""
    import simulador_quantico_b200 as sq_mod

    sq_mod.init(int(os.environ.get("HGM_DEVICE", "0")))
    return sq_mod
