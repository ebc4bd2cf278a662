import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the native library")
    config.addinivalue_line("markers", "slow: full-size workloads")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the host generator and the oracle once per session (cheap if current)."""
    from agipc_learning_b200 import build
    import oracle
    build.build_synth()
    oracle.build()
    yield
