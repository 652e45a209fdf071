import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ctx():
    """One library context on device 0 for the GPU tests (fails loudly without a GPU)."""
    import torch  # noqa: F401  (loads the CUDA runtime first; the library uses the same driver)

    from nanomap_b200.api import Context

    c = Context(0)
    yield c
    c.close()
