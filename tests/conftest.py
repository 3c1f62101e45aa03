import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) and the built libtcscf_gpu.so")


@pytest.fixture(scope="session")
def ctx():
    """One library context on cuda:0 for the GPU tests (fails loudly without a B200)."""
    from tcscf_b200 import build as _build
    from tcscf_b200.api import Context

    _build.build()
    c = Context(0)
    yield c
    c.close()
