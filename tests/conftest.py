import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs through the C ABI")


@pytest.fixture(scope="session")
def built():
    """Builds the library and the oracle once per session (no-op when fresh)."""
    from epi_b200 import build as B
    from oracle import oracle as O
    B.build_library()
    O.build_oracle()
    return True
