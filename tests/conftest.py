import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (sm_100)")
    config.addinivalue_line("markers", "reference: needs the reference built from its sources (oracle/_ref)")


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Builds the native library and the CPU oracle in-tree if they are missing or stale."""
    from bg_flood_b200.build import build, build_oracle
    build()
    build_oracle()
    yield


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def have_reference():
    from oracle.pyoracle import ref_available
    if not ref_available():
        pytest.skip("reference oracle (oracle/_ref) not built")
    return True
