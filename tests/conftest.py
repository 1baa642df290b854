import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: larger sizes, minutes of CPU or GPU time")


@pytest.fixture(scope="session")
def gpu_ctx():
    import iccg_b200 as ib
    ctx = ib.Context(0)
    yield ctx
    ctx.close()
