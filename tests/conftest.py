import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libshb.so")


@pytest.fixture(scope="session")
def gpu_ctx():
    from sh_baker_b200 import build as B
    B.build()
    from sh_baker_b200 import Context
    ctx = Context(device=int(os.environ.get("SHB_DEVICE", "0")))
    yield ctx
    ctx.close()
