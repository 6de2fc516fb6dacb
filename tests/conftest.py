import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine")


@pytest.fixture(scope="session")
def ctx():
    import kcgpu_b200 as kc

    c = kc.Context(0)
    yield c
    c.close()
