import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the device path")


@pytest.fixture(scope="session", autouse=True)
def _build_oracle():
    """Build the oracle's C restatement (and the reference harness where the sources exist)."""
    import oracle
    oracle.build()


@pytest.fixture(scope="session")
def renderer():
    import torch  # noqa: F401  (initialises the CUDA driver the same way the bench does)
    from slimtracin_b200 import api, build
    build.build()
    r = api.Renderer(device=0)
    yield r
    r.close()
