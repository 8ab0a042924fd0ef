import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
TESTS = Path(__file__).resolve().parent
if str(TESTS) not in sys.path:
    sys.path.insert(0, str(TESTS))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Both shared libraries exist before any test (built in-tree if missing)."""
    from continuum_b200 import build as cbuild
    from oracle import build as obuild

    if not cbuild.LIB.exists():
        cbuild.build()
    obuild.build()


@pytest.fixture(scope="session")
def kernel():
    from continuum_b200 import MaskConeKernel

    k = MaskConeKernel.new(0)
    if k is None:
        pytest.fail("no CUDA device: GPU tests need a B200")
    yield k
    k.close()
