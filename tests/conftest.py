import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the native test libraries (CPU-only builds are cheap and idempotent)."""
    from g3sa_b200 import build
    build.build_emu()
    build.build_emu16()
    build.build_synth()
    from tests import native
    native.build_oracle()
